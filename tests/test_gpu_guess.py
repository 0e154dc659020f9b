"""User-supplied initial guesses (the sigma slot of cosmo.f90:136-138, 174-176)
through ddc_energy_forces: the previous frame of a trajectory as the guess of
the next.  The converged answer must not depend on the guess (same bars as the
zero/reference guesses against the oracle: Esolv 1e-9 relative, forces 1e-7
Hartree/bohr) and a close guess must save iterations."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ESOLV_RTOL = 1e-9
FORCE_ATOL = 1e-7


def _frames(cfg, count=2):
    from ddpcm_b200 import molecules as M
    m = M.config_molecule(cfg)
    return [M.to_bohr(f) for f in M.trajectory(m, count, sigma=0.05, seed=77)]


@pytest.mark.parametrize("prec", [0, 1])
def test_previous_frame_guess_config1(oracle, prec):
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo, GUESS_REFERENCE, GUESS_USER
    c = M.CONFIGS[1]
    f0, f1 = _frames(1)
    kw = dict(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"], eta=c["eta"],
              precision=prec)
    with DDCosmo(guess=GUESS_REFERENCE, **kw) as dd:
        first = dd.energy_forces(f0["q"], f0["x"], f0["y"], f0["z"], f0["r"])
        cold = dd.energy_forces(f1["q"], f1["x"], f1["y"], f1["z"], f1["r"])
    with DDCosmo(guess=GUESS_USER, **kw) as dd:
        warm = dd.energy_forces(f1["q"], f1["x"], f1["y"], f1["z"], f1["r"],
                                sigma0=first["sigma"], s0=first["s"])
    ref = oracle.energy_forces(f1, c["lmax"], c["ngrid"], c["iconv"], c["eps"], c["eta"])
    for out in (cold, warm):
        assert out["info"]["direct"]["converged"] and out["info"]["adjoint"]["converged"]
        assert abs(out["esolv"] - ref["esolv"]) <= ESOLV_RTOL * abs(ref["esolv"])
        np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)
    for side in ("direct", "adjoint"):
        assert warm["info"][side]["iterations"] < cold["info"][side]["iterations"]


def test_user_guess_is_used_unchanged():
    """The converged solution as the guess: the first Jacobi increment is
    already below the tolerance, so the solve stops after one step, which
    moves Esolv by far less than the parity bar."""
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo, GUESS_USER
    c = M.CONFIGS[1]
    f0 = _frames(1, 1)[0]
    kw = dict(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"], eta=c["eta"])
    with DDCosmo(**kw) as dd:
        first = dd.energy_forces(f0["q"], f0["x"], f0["y"], f0["z"], f0["r"])
    with DDCosmo(guess=GUESS_USER, **kw) as dd:
        again = dd.energy_forces(f0["q"], f0["x"], f0["y"], f0["z"], f0["r"],
                                 sigma0=first["sigma"], s0=first["s"])
    assert again["info"]["direct"]["iterations"] <= 1
    assert again["info"]["adjoint"]["iterations"] <= 1
    assert abs(again["esolv"] - first["esolv"]) <= 1e-10 * abs(first["esolv"])


def test_user_guess_requires_arrays():
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDC_ERR_PARAM, DDCosmo, DDCosmoError, GUESS_USER
    f0 = _frames(0, 1)[0]
    c = M.CONFIGS[0]
    arr = {k: np.ascontiguousarray(f0[k], dtype=np.float64) for k in "qxyzr"}
    with DDCosmo(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eta=c["eta"],
                 guess=GUESS_USER) as dd:
        with pytest.raises(DDCosmoError) as e:
            dd.energy_forces_ptr(*(arr[k].ctypes.data for k in "qxyzr"), len(arr["q"]), 0, 0, 0)
        assert e.value.status == DDC_ERR_PARAM
