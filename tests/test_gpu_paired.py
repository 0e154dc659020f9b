"""Paired solves: ddc_energy_forces advancing the direct and adjoint
Jacobi/DIIS solves together, with L x and L* s from one fused pass over the
(sphere, point, neighbour) triples.  Each solve keeps its own history and
convergence test, so the iterations must equal those of the one-after-the-
other flow (pair_solves=0, the reference's order) and the results must meet
the same bars against the oracle."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def _run(m, p, **kw):
    from ddpcm_b200.ddcosmo import DDCosmo
    with DDCosmo(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"], eta=p["eta"],
                 **kw) as dd:
        return dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])


@pytest.mark.parametrize("prec", [0, 1])
@pytest.mark.parametrize("name", ["caffeine", "crambin"])
def test_paired_equals_sequential(oracle, name, prec):
    g = load_golden(name)
    p, m = dict(g["params"]), g["mol"]
    p["iconv"] = 10
    seq = _run(m, p, pair_solves=0, precision=prec)
    par = _run(m, p, pair_solves=1, precision=prec)
    ref = oracle.energy_forces(m, p["lmax"], p["ngrid"], p["iconv"], p["eps"], p["eta"])
    for side in ("direct", "adjoint"):
        a, b = seq["info"][side], par["info"][side]
        assert b["converged"]
        assert abs(a["iterations"] - b["iterations"]) <= 1
    for out in (seq, par):
        assert abs(out["esolv"] - ref["esolv"]) <= 1e-9 * abs(ref["esolv"])
        np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=1e-7)
    # the two flows round the operator sums differently; at tol 1e-10 on the
    # increments that moves Esolv by ~1e-10 relative
    assert abs(par["esolv"] - seq["esolv"]) <= 1e-9 * abs(seq["esolv"])


@pytest.mark.parametrize("lmax", list(range(0, 13)))
def test_fused_operator_all_lmax(oracle, lmax):
    """The fused kernel is instantiated per lmax: each against the oracle's
    lx and lstarx."""
    from ddpcm_b200.ddcosmo import DDCosmo
    g = load_golden("caffeine")
    m = g["mol"]
    ngrid = 302 if lmax > 8 else 110
    d = oracle.RefDD(lmax, ngrid, 10, 1, 78.3553, 0.1).init(m["x"], m["y"], m["z"], m["r"])
    rng = np.random.default_rng(lmax)
    x = rng.standard_normal((d.nsph, d.nylm))
    s = rng.standard_normal((d.nsph, d.nylm))
    with DDCosmo(lmax=lmax, ngrid=ngrid, iconv=10, eta=0.1) as dd:
        dd.ddinit(m["x"], m["y"], m["z"], m["r"])
        y, z = dd.lx_lstarx(x, s)
    for a, b in ((y, d.lx(x)), (z, d.lstarx(s))):
        assert np.abs(a - b).max() <= 1e-13 * max(np.abs(b).max(), 1e-300)


def test_paired_nonconvergence_reports_both():
    from ddpcm_b200.ddcosmo import DDC_ERR_NOCONV, DDCosmoError
    g = load_golden("caffeine")
    m = g["mol"]
    p = dict(lmax=6, ngrid=110, iconv=10, eps=78.3553, eta=0.1)
    with pytest.raises(DDCosmoError) as ei:
        _run(m, p, max_iter=3)
    assert ei.value.status == DDC_ERR_NOCONV
