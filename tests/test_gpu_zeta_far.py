"""Grouped multipole far field of the cavity charges zeta at the nuclei (the
field of efld.f90:97-114 as main.f90:259-265 uses it for the forces) in the
mixed-precision energy+force flow: from 4,096 spheres on, the spheres are
grouped by grid cells and a group farther than three group radii from a
nucleus acts through its degree-16 multipole expansion (truncation about
1.2e-8 of the group's charge scale), nearer groups through FP32 pair sums as
in the direct path.  Both are FP32 approximations of the FP64 field: the
expansion sums round in FP32 like the pair sums do (about 1e-7 of each
group's field; measured force differences 0.7e-8 at 4,096 spheres and
1.3e-8 at 9,000, forces up to 0.12 Hartree/bohr).  The forces must agree
with those of the direct FP32 pair sums (DDC_ZFAR_OFF=1) to 3e-8, well
inside the force bar (1e-7 Hartree/bohr); the energy does not depend on
this field and must be identical.  The
20,000-sphere comparison with the stored FP64 oracle run
(test_gpu_mixed.py) covers the whole flow against the reference
restatement."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P10 = dict(lmax=10, ngrid=590, iconv=10, eps=78.3553, eta=0.1, precision=1)


def _solve(mol, zfar, **kw):
    from ddpcm_b200.ddcosmo import DDCosmo
    os.environ["DDC_ZFAR_OFF"] = "0" if zfar else "1"
    try:
        with DDCosmo(**kw) as dd:
            return dd.energy_forces(mol["q"], mol["x"], mol["y"], mol["z"], mol["r"])
    finally:
        os.environ.pop("DDC_ZFAR_OFF", None)


@pytest.mark.parametrize("n,seed", [(4096, 77), (9000, 78)])
def test_grouped_zeta_field_matches_direct_pairs(n, seed):
    from ddpcm_b200 import molecules as M
    mol = M.to_bohr(M.make_molecule(n, seed))
    a = _solve(mol, True, **P10)
    b = _solve(mol, False, **P10)
    assert a["esolv"] == b["esolv"]
    d = np.abs(a["fx"] - b["fx"]).max()
    print(f"n={n}: max |dF| = {d:.3e}, max |F| = {np.abs(b['fx']).max():.3e}")
    assert d <= 3e-8


def test_grouped_zeta_field_is_reproducible():
    from ddpcm_b200 import molecules as M
    mol = M.to_bohr(M.make_molecule(5000, 79))
    a = _solve(mol, True, **P10)
    b = _solve(mol, True, **P10)
    assert np.array_equal(a["fx"], b["fx"])
