"""Learned initial guess (ddc_guess_*, DDC_GUESS_LEARNED).

* The BF16-weight inference kernels against an FP32 torch forward of the same
  (BF16-rounded) weights.
* Training kernels: a few epochs on solver-generated rows lower the loss.
* The solve from the learned start converges to the same answer as the plain
  FP64 zero-guess solve (Esolv within 1e-9 relative, forces within 1e-7),
  single molecule and batched, on globules held out of training.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
WEIGHTS = os.path.join(ROOT, "ddpcm_b200", "guess_lmax6_g302.npz")
P6 = dict(lmax=6, ngrid=302, iconv=10, eps=78.3553, eta=0.1)


def _bf16(a):
    import torch
    return torch.as_tensor(a).to(torch.bfloat16).to(torch.float32)


def _torch_forward(model, feat):
    """FP32 reference of the network with the model's BF16-rounded weights."""
    import torch
    p = model.get_params()
    d = [model.nfeat, model.hidden, model.hidden, model.hidden, model.nout]
    o, W = 0, []
    for k in range(4):
        W.append(p[o:o + d[k] * d[k + 1]].reshape(d[k + 1], d[k]))
        o += d[k] * d[k + 1]
    b = []
    for k in range(4):
        b.append(p[o:o + d[k + 1]])
        o += d[k + 1]
    mean, istd = p[o:o + d[0]], p[o + d[0]:o + 2 * d[0]]
    dev = feat.device
    x = (feat - torch.tensor(mean, device=dev)) * torch.tensor(istd, device=dev)
    for k in range(4):
        x = x @ _bf16(W[k]).to(dev).T + torch.tensor(b[k], device=dev)
        if k < 3:
            x = torch.relu(x)
    return x


def test_inference_matches_fp32_forward():
    import torch
    from ddpcm_b200.ddcosmo import GuessModel
    model = GuessModel.load(WEIGHTS)
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(3)
    p = model.get_params()
    mean = torch.tensor(p[-(2 * model.nfeat + model.nout):-(model.nfeat + model.nout)])
    istd = torch.tensor(p[-(model.nfeat + model.nout):-model.nout])
    feat = (torch.randn(3000, model.nfeat, generator=g) / istd + mean).to(dev)
    out = torch.empty((3000, model.nout), dtype=torch.float32, device=dev)
    model.predict(feat.data_ptr(), out.data_ptr(), 3000)
    ref = _torch_forward(model, feat)
    err = (out - ref).abs().max().item() / ref.abs().max().item()
    assert err < 1e-5, err


def test_training_lowers_the_loss():
    import torch
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo, GuessModel
    dev = torch.device("cuda", 0)
    model = GuessModel(6, 64, 0)
    mols = [M.to_bohr(M.make_molecule(n, 812000 + k)) for k, n in enumerate((60, 90, 150, 230))]
    with DDCosmo(lmax=6, ngrid=110, iconv=8, eps=78.3553, eta=0.1) as dd:
        dd.set_guess_model(model)
        out = dd.batch_energy_forces(mols)
        n = int(out["off"][-1])
        f = torch.empty((n, model.nfeat), dtype=torch.float32, device=dev)
        t = torch.empty((n, model.nout), dtype=torch.float32, device=dev)
        dd.guess_rows(f.data_ptr(), t.data_ptr())
    # the rows: rhs, psi(00), radius and a histogram that counts every other
    # sphere of the molecule within 8 angstrom
    assert torch.isfinite(f).all() and torch.isfinite(t).all()
    assert (f[:, 49] != 0).any() and (f[:, 50] > 0).all()
    hist = f[:, 51:67]
    assert (hist >= 0).all() and (hist.sum(1) <= torch.tensor(
        np.repeat([60, 90, 150, 230], [60, 90, 150, 230]) - 1, device=dev)).all()
    model.fit_scaling(f.data_ptr(), t.data_ptr(), n)
    model.init_random(5)
    losses = [model.train_epoch(f.data_ptr(), t.data_ptr(), 0, n, 128, 2e-3) for _ in range(12)]
    assert losses[-1] < 0.8 * losses[0], losses
    assert all(b < a for a, b in zip(losses[:4], losses[1:5])), losses


def _solve(mol, guess, model=None, precision=0):
    from ddpcm_b200.ddcosmo import DDCosmo
    with DDCosmo(guess=guess, precision=precision, **P6) as dd:
        if model is not None:
            dd.set_guess_model(model)
        return dd.energy_forces(mol["q"], mol["x"], mol["y"], mol["z"], mol["r"])


@pytest.mark.parametrize("precision", [0, 1])
def test_learned_guess_converges_to_the_zero_guess_answer(precision):
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import GUESS_LEARNED, GUESS_REFERENCE, GUESS_ZERO, GuessModel
    from ddpcm_b200.train_guess import EVAL_SEEDS
    model = GuessModel.load(WEIGHTS)
    mol = M.to_bohr(M.make_molecule(1200, EVAL_SEEDS[0]))
    zero = _solve(mol, GUESS_ZERO)
    ref = _solve(mol, GUESS_REFERENCE)
    lrn = _solve(mol, GUESS_LEARNED, model, precision)
    assert abs(lrn["esolv"] - zero["esolv"]) <= 1e-9 * abs(zero["esolv"])
    assert np.abs(lrn["fx"] - zero["fx"]).max() <= 1e-7
    for key in ("direct", "adjoint"):
        assert lrn["info"][key]["converged"]
        if precision == 0:
            # the learned start is at least as good as the reference's
            assert lrn["info"][key]["iterations"] <= ref["info"][key]["iterations"], key


@pytest.mark.parametrize("precision", [0, 1])
def test_learned_guess_in_a_batch(precision):
    """FP64 reference-start batch against the learned start, batched in FP64
    or in mixed precision (the mixed refinement then starts from the
    learned guess with an FP64 residual)."""
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo, GUESS_LEARNED, GuessModel
    from ddpcm_b200.train_guess import EVAL_SEEDS
    model = GuessModel.load(WEIGHTS)
    mols = [M.to_bohr(M.make_molecule(n, EVAL_SEEDS[1] + k)) for k, n in enumerate((40, 300, 900))]
    with DDCosmo(**P6) as dd:
        a = dd.batch_energy_forces(mols)
    with DDCosmo(guess=GUESS_LEARNED, precision=precision, **P6) as dd:
        dd.set_guess_model(model)
        b = dd.batch_energy_forces(mols)
    assert b["info"]["direct"]["converged"] and b["info"]["adjoint"]["converged"]
    # Both starts run to the same stop test; as in the batched parity tests,
    # a molecule of at most 60 spheres stops within an iteration or two of
    # the other start's count, and the two iterates (both inside the 1e-10
    # test) give energies up to a few 1e-9 apart: those are held to 5e-9
    for k, m in enumerate(mols):
        rtol = 1e-9 if len(m["x"]) > 60 else 5e-9
        assert abs(b["esolv"][k] - a["esolv"][k]) <= rtol * abs(a["esolv"][k]), k
    for fa, fb in zip(a["fx"], b["fx"]):
        np.testing.assert_allclose(fb, fa, rtol=0, atol=1e-7)


def test_learned_guess_needs_a_model():
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmoError, GUESS_LEARNED
    mol = M.to_bohr(M.make_molecule(30, 5))
    with pytest.raises(DDCosmoError):
        _solve(mol, GUESS_LEARNED)
