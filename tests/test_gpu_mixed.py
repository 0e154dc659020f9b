"""Mixed precision (FP32 operator inside FP64 iterative refinement) against
the FP64 oracle: the same bars as the FP64 path (Esolv 1e-9 relative, forces
1e-7 Hartree/bohr), because the refinement stops on the FP64 Jacobi
increment, the reference's own convergence test."""
import os

import numpy as np
import pytest

from conftest import GOLDEN, load_golden

pytestmark = pytest.mark.gpu

ESOLV_RTOL = 1e-9
FORCE_ATOL = 1e-7


def _run(mol, c, **kw):
    from ddpcm_b200.ddcosmo import DDCosmo, PREC_MIXED
    with DDCosmo(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"], eta=c["eta"],
                 precision=PREC_MIXED, **kw) as dd:
        return dd.energy_forces(mol["q"], mol["x"], mol["y"], mol["z"], mol["r"])


@pytest.mark.parametrize("cfg", [0, 1])
def test_mixed_configs_vs_oracle(oracle, cfg):
    from ddpcm_b200 import molecules as M
    c = M.CONFIGS[cfg]
    m = M.to_bohr(M.config_molecule(cfg))
    ref = oracle.energy_forces(m, c["lmax"], c["ngrid"], c["iconv"], c["eps"], c["eta"])
    out = _run(m, c)
    assert out["info"]["direct"]["converged"] and out["info"]["adjoint"]["converged"]
    assert out["info"]["direct"]["refinements"] >= 2
    assert abs(out["esolv"] - ref["esolv"]) <= ESOLV_RTOL * abs(ref["esolv"])
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)


@pytest.mark.parametrize("name", ["caffeine", "crambin"])
def test_mixed_golden_molecules(oracle, name):
    g = load_golden(name)
    p, m = dict(g["params"]), g["mol"]
    p["iconv"] = 10
    ref = oracle.energy_forces(m, p["lmax"], p["ngrid"], p["iconv"], p["eps"], p["eta"])
    out = _run(m, p)
    assert abs(out["esolv"] - ref["esolv"]) <= ESOLV_RTOL * abs(ref["esolv"])
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)


def test_mixed_zero_guess_full_size():
    """20,000 spheres, lmax 10: mixed precision from a zero guess against the
    stored FP64 oracle run."""
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import GUESS_ZERO
    c = M.CONFIGS[2]
    m = M.to_bohr(M.config_molecule(2))
    out = _run(m, c, guess=GUESS_ZERO)
    ref = np.load(os.path.join(GOLDEN, "config2_oracle.npz"))
    assert abs(out["esolv"] - float(ref["esolv"])) <= ESOLV_RTOL * abs(float(ref["esolv"]))
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)
