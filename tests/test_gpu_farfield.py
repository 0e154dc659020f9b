"""Near / far split of the solute potential and field at the cavity points
(mkrhs.f90:102-114, main.f90:241): from 4,096 spheres on, charges farther
than 8 sphere radii enter through a degree-10 local expansion about each
sphere's centre.  The energy and forces with the split must equal those of
the direct sums (DDC_FAR_OFF=1) to well below the bars (Esolv 1e-9 relative,
forces 1e-7): the expansion is truncated at about 1e-10 of each far term.
The 20,000-sphere comparison with the stored FP64 oracle run
(test_gpu_mixed.py) covers the split against the reference restatement."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P6 = dict(lmax=6, ngrid=302, iconv=10, eps=78.3553, eta=0.1)


def _solve(mol, far, **kw):
    from ddpcm_b200.ddcosmo import DDCosmo
    os.environ["DDC_FAR_OFF"] = "0" if far else "1"
    try:
        with DDCosmo(**P6, **kw) as dd:
            return dd.energy_forces(mol["q"], mol["x"], mol["y"], mol["z"], mol["r"])
    finally:
        os.environ.pop("DDC_FAR_OFF", None)


@pytest.mark.parametrize("precision", [0, 1])
def test_far_split_matches_direct_sums(precision):
    from ddpcm_b200 import molecules as M
    mol = M.to_bohr(M.make_molecule(6000, 4242))
    a = _solve(mol, True, precision=precision)
    b = _solve(mol, False, precision=precision)
    assert abs(a["esolv"] - b["esolv"]) <= 1e-11 * abs(b["esolv"]) * (1 if precision == 0 else 100)
    assert np.abs(a["fx"] - b["fx"]).max() <= (1e-10 if precision == 0 else 1e-8)
    if precision == 0:
        assert a["info"]["direct"]["iterations"] == b["info"]["direct"]["iterations"]


def test_far_split_in_a_batch():
    """Three 2,000-sphere globules in one batch (6,000 spheres: the split is
    on, each sphere's far charges restricted to its own molecule)."""
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo
    mols = [M.to_bohr(M.make_molecule(2000, 4300 + k)) for k in range(3)]
    out = {}
    for far in (True, False):
        os.environ["DDC_FAR_OFF"] = "0" if far else "1"
        try:
            with DDCosmo(**P6) as dd:
                out[far] = dd.batch_energy_forces(mols)
        finally:
            os.environ.pop("DDC_FAR_OFF", None)
    np.testing.assert_allclose(out[True]["esolv"], out[False]["esolv"], rtol=1e-11, atol=0)
    for fa, fb in zip(out[True]["fx"], out[False]["fx"]):
        np.testing.assert_allclose(fa, fb, rtol=0, atol=1e-10)
