"""Forces when Lebedev points fall exactly on a neighbour's pole.

Spheres centred on the z axis put the grid points (0, 0, +-1) of one sphere
on the z axis of its neighbours, where the unit vector s has sin(theta) = 0:
the force kernel then takes the reference's dbasis branch for the pole
(ddcosmo.f90:904-1043, VC = 0 and VS = int(cos theta)) instead of the
recurrence against the ladder vectors.  A fourth, off-axis sphere keeps the
other triples on the general branch.  Both must match the oracle."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _mol():
    # bohr; the first three centres are exactly on the z axis
    return dict(q=np.array([0.4, -0.3, 0.2, -0.3]),
                x=np.array([0.0, 0.0, 0.0, 2.1]),
                y=np.array([0.0, 0.0, 0.0, 0.7]),
                z=np.array([0.0, 2.0, 4.2, 1.3]),
                r=np.array([2.5, 2.3, 2.6, 2.2]))


@pytest.mark.parametrize("prec, etol, ftol", [(0, 1e-9, 1e-8), (1, 1e-9, 1e-7)])
def test_forces_with_points_on_poles(oracle, prec, etol, ftol):
    from ddpcm_b200.ddcosmo import DDCosmo
    m = _mol()
    p = dict(lmax=8, ngrid=302, iconv=10, eps=78.3553, eta=0.1)
    ref = oracle.energy_forces(m, p["lmax"], p["ngrid"], p["iconv"], p["eps"], p["eta"])
    with DDCosmo(precision=prec, **p) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
    assert abs(out["esolv"] - ref["esolv"]) <= etol * abs(ref["esolv"])
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=ftol)
    # the forces are not trivially small
    assert np.abs(ref["fx"]).max() > 1e-4
