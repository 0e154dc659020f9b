"""Cell groups of one large molecule (4,096 spheres and more): the neighbour
list (ddcosmo.f90:308-324) is searched among the spheres of the groups whose
bounding spheres reach a sphere, and the near charges of the cavity far
field among the groups within 8 sphere radii.  The lists must be the ones
the all-pairs scans give (DDC_CELLS_OFF=1): the same pair count, and the
FP64 energy, forces and iteration counts equal up to the summation order of
the near charges (1e-13)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P6 = dict(lmax=6, ngrid=302, iconv=10, eps=78.3553, eta=0.1)


def _run(mol, cells):
    from ddpcm_b200.ddcosmo import DDCosmo
    os.environ["DDC_CELLS_OFF"] = "0" if cells else "1"
    try:
        with DDCosmo(**P6) as dd:
            return dd.energy_forces(mol["q"], mol["x"], mol["y"], mol["z"], mol["r"])
    finally:
        os.environ.pop("DDC_CELLS_OFF", None)


@pytest.mark.parametrize("n,seed", [(4096, 91), (12000, 92)])
def test_cell_lists_match_all_pairs(n, seed):
    from ddpcm_b200 import molecules as M
    mol = M.to_bohr(M.make_molecule(n, seed))
    a = _run(mol, True)
    b = _run(mol, False)
    for key in ("npairs", "ntriples", "ncav"):
        assert a["info"][key] == b["info"][key], key
    assert abs(a["esolv"] - b["esolv"]) <= 1e-13 * abs(b["esolv"])
    assert np.abs(a["fx"] - b["fx"]).max() <= 1e-12
    for key in ("direct", "adjoint"):
        assert a["info"][key]["iterations"] == b["info"][key]["iterations"]
