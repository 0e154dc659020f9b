"""Parity of the CUDA library (through the C ABI) with the CPU oracle.

Bars: Esolv within 1e-9 relative, forces within 1e-7 Hartree/bohr max-abs
(the targets of the task); in practice both run in FP64 and agree far more
tightly, which the tighter asserts below pin.  Set-defining geometry (the
neighbour list, the cavity, ui) is computed in the same IEEE operation order
on both sides and must match exactly.
"""
import numpy as np
import pytest

from conftest import MOLS, TOKCAL, load_golden

pytestmark = pytest.mark.gpu

ESOLV_RTOL = 1e-9
FORCE_ATOL = 1e-7


def _iters_close(out, ref):
    """Late DIIS steps solve nearly singular bordered systems whose pivoting
    can differ on last-bit rounding; counts agree to within 20% (+1)."""
    for k, key in ((0, "direct"), (1, "adjoint")):
        a, b = out["info"][key]["iterations"], ref["iters"][k]
        assert abs(a - b) <= 1 + 0.2 * b, (key, a, b)


def gpu_ctx(**kw):
    from ddpcm_b200.ddcosmo import DDCosmo
    return DDCosmo(**kw)


def ref_ctx(oracle, p, m):
    d = oracle.RefDD(p["lmax"], p["ngrid"], p["iconv"], p.get("igrad", 1), p["eps"], p["eta"])
    return d.init(m["x"], m["y"], m["z"], m["r"])


@pytest.mark.parametrize("pair", [1, 0])
@pytest.mark.parametrize("name", MOLS)
def test_golden_decks_iteration_logs(name, pair):
    """Every Jacobi/DIIS increment norm the reference printed (4 significant
    digits), direct and adjoint, paired or one after the other."""
    g = load_golden(name)
    p, m = g["params"], g["mol"]
    with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"], pair_solves=pair) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
    for side in ("direct", "adjoint"):
        ref = np.array(g["norms_" + side])
        got = np.array(out["info"][side]["norms"])
        k = min(len(ref), len(got))
        assert k >= len(ref) - 1
        np.testing.assert_allclose(got[:k], ref[:k], rtol=1e-3, atol=0)


@pytest.mark.parametrize("name", MOLS)
def test_golden_decks_vs_reference_logs(name):
    """The reference's own decks at their own settings (iconv 7) against the
    printed results.  At tol 1e-7 the solution is defined to ~1e-7 relative,
    so the energy is checked at 1e-4 kcal/mol (6e-8 relative for crambin) and
    the forces at the 1e-7 bar; the CPU oracle, which sums in the
    reference's order, matches the same logs to print precision."""
    g = load_golden(name)
    p, m = g["params"], g["mol"]
    with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"]) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
        assert dd.launches > 0
    assert out["info"]["ngrid"] == g["ngrid_snapped"]
    assert abs(out["esolv"] * TOKCAL - g["energy_kcal"]) <= 1e-4
    np.testing.assert_allclose(out["fx"], np.array(g["forces"]), rtol=0, atol=FORCE_ATOL)
    assert abs(out["info"]["direct"]["iterations"] - len(g["norms_direct"])) <= 1
    assert abs(out["info"]["adjoint"]["iterations"] - len(g["norms_adjoint"])) <= 1


@pytest.mark.parametrize("name", MOLS)
def test_golden_molecules_vs_oracle_converged(oracle, name):
    """GPU against the oracle on the reference's molecules at tol 1e-10."""
    g = load_golden(name)
    p, m = dict(g["params"]), g["mol"]
    p["iconv"] = 10
    tol = 1e-10
    ref = oracle.energy_forces(m, p["lmax"], p["ngrid"], p["iconv"], p["eps"], p["eta"])
    with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"]) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
    assert out["info"]["ncav"] == ref["ncav"]
    assert abs(out["esolv"] - ref["esolv"]) <= ESOLV_RTOL * abs(ref["esolv"])
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)
    # secondary, 30x tighter than the bar: the iteration noise floor at tol
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=3e-9)
    _iters_close(out, ref)
    # the stop test bounds the H-norm of the increment (an RMS over spheres),
    # not each element: single elements sit up to a few tol away
    np.testing.assert_allclose(out["sigma"], ref["sigma"], rtol=0, atol=30 * tol)
    np.testing.assert_allclose(out["s"], ref["s"], rtol=0, atol=30 * tol)


@pytest.mark.parametrize("name", ["formaldehyde", "caffeine", "crambin"])
def test_init_geometry_exact(oracle, name):
    g = load_golden(name)
    p, m = g["params"], g["mol"]
    ref = ref_ctx(oracle, p, m)
    with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"]) as dd:
        dd.ddinit(m["x"], m["y"], m["z"], m["r"])
        assert (dd.nsph, dd.ncav, dd.nylm, dd.ngrid) == (ref.nsph, ref.ncav, ref.nylm, ref.ngrid)
        gr, w = dd.grid()
        np.testing.assert_array_equal(gr, ref.get("grid"))
        np.testing.assert_array_equal(w, ref.get("w"))
        np.testing.assert_array_equal(dd.ccav, ref.get("ccav"))
        np.testing.assert_array_equal(dd.ui, ref.get("ui"))
        np.testing.assert_array_equal(dd.csph, ref.get("csph"))


def _random_vec(rng, n, nylm):
    return rng.standard_normal((n, nylm))


@pytest.mark.parametrize("name", ["caffeine", "crambin"])
def test_operators_vs_oracle(oracle, name):
    g = load_golden(name)
    p, m = g["params"], g["mol"]
    ref = ref_ctx(oracle, p, m)
    rng = np.random.default_rng(11)
    x = _random_vec(rng, ref.nsph, ref.nylm)
    with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"]) as dd:
        dd.ddinit(m["x"], m["y"], m["z"], m["r"])
        for fn, rf in ((dd.lx, ref.lx), (dd.lstarx, ref.lstarx), (dd.ldm1x, ref.ldm1x)):
            a, b = fn(x), rf(x)
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
        s = _random_vec(rng, ref.nsph, ref.nylm)
        y, z = dd.lx_lstarx(x, s)
        for a, b in ((y, ref.lx(x)), (z, ref.lstarx(s))):
            assert np.abs(a - b).max() <= 1e-13 * np.abs(b).max()
        assert abs(dd.hnorm(x) - ref.hnorm(x)) <= 1e-14 * ref.hnorm(x)
        phi, _ = oracle.mkrhs(m["q"], m["x"], m["y"], m["z"], ref.get("ccav"), ref.nylm)
        np.testing.assert_allclose(dd.rhs(phi), ref.rhs(phi), rtol=0,
                                   atol=1e-14 * np.abs(ref.rhs(phi)).max())


def test_separate_entry_points_formaldehyde(oracle):
    """ddinit -> mkrhs -> cosmo -> cosmo* -> forces_dd -> ddmkzeta -> efld, one
    call each, as main.f90 drives them (pole geometry: atoms on the z axis)."""
    g = load_golden("formaldehyde")
    p, m = g["params"], g["mol"]
    ref = ref_ctx(oracle, p, m)
    with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"]) as dd:
        dd.ddinit(m["x"], m["y"], m["z"], m["r"])
        phi, psi = dd.mkrhs(m["q"], m["x"], m["y"], m["z"])
        rphi, rpsi = oracle.mkrhs(m["q"], m["x"], m["y"], m["z"], ref.get("ccav"), ref.nylm)
        np.testing.assert_allclose(phi, rphi, rtol=1e-13, atol=0)
        np.testing.assert_array_equal(psi, rpsi)
        phi2, _ = dd.mkrhs(m["q"], m["x"], m["y"], m["z"], ccav=ref.get("ccav"))
        np.testing.assert_allclose(phi2, rphi, rtol=1e-13, atol=0)
        X, es = dd.cosmo(False, True, phi=phi, psi=psi)
        rd = ref.cosmo(False, True, phi=rphi, psi=rpsi)
        assert abs(es - rd["esolv"]) <= 1e-12 * abs(rd["esolv"])
        np.testing.assert_allclose(X, np.array(g["X"]), atol=6e-9)
        S, _, info = dd.cosmo(True, False, psi=psi, return_info=True)
        ra = ref.cosmo(True, False, psi=rpsi)
        assert info["iterations"] == ra["iters"] and info["converged"]
        np.testing.assert_allclose(info["norms"], ra["norms"], rtol=1e-5)
        np.testing.assert_allclose(S, np.array(g["S"]), atol=6e-9)
        fx = dd.forces_dd(phi, X, S)
        np.testing.assert_allclose(fx, ref.forces_dd(rphi, rd["sigma"], ra["sigma"]), atol=1e-13)
        zeta = dd.ddmkzeta(S)
        # S is converged to 1e-7 here (the deck's iconv), so zeta/xi agree to that noise
        np.testing.assert_allclose(zeta, ref.mkzeta(ra["sigma"]), rtol=1e-8, atol=1e-15)
        np.testing.assert_allclose(dd.ddmkxi(S), ref.mkxi(ra["sigma"]), rtol=1e-8, atol=1e-15)
        # with the oracle's own S the GPU zeta/xi match to round-off
        np.testing.assert_allclose(dd.ddmkzeta(ra["sigma"]), ref.mkzeta(ra["sigma"]), rtol=1e-12,
                                   atol=1e-18)
        csph = dd.csph
        ccav = dd.ccav
        ef = dd.efld(m["q"], csph, ccav)
        np.testing.assert_allclose(ef, oracle.efld(m["q"], csph, ccav), rtol=1e-13, atol=1e-16)
        ef2 = dd.efld(zeta, ccav, csph)
        np.testing.assert_allclose(ef2, oracle.efld(zeta, ccav, csph), rtol=1e-12, atol=1e-17)
        # NULL coordinates: the module's own cavity / centres
        np.testing.assert_allclose(dd.efld(m["q"], None, None), ef, rtol=1e-15, atol=0)
        # main.f90:245-265 contractions give the logged total forces
        tot = fx.copy()
        ui = dd.ui
        ii = 0
        for i in range(dd.nsph):
            for n in range(dd.ngrid):
                if ui[i, n] > 0:
                    tot[i] -= zeta[ii] * ef[ii]
                    ii += 1
        tot -= ef2 * m["q"][:, None]
        np.testing.assert_allclose(tot, np.array(g["forces"]), atol=6e-9)


@pytest.mark.parametrize("cfg", [0, 1])
def test_configs_vs_oracle(oracle, cfg):
    from ddpcm_b200 import molecules as M
    c = M.CONFIGS[cfg]
    m = M.to_bohr(M.config_molecule(cfg))
    ref = oracle.energy_forces(m, c["lmax"], c["ngrid"], c["iconv"], c["eps"], c["eta"])
    with gpu_ctx(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"],
                 eta=c["eta"]) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
    assert abs(out["esolv"] - ref["esolv"]) <= ESOLV_RTOL * abs(ref["esolv"])
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=1e-10)
    _iters_close(out, ref)


def test_config2_full_size_properties():
    """20,000 spheres, lmax 10, ngrid 590: size-independent checks.
    <y, L x> = <L* y, x> (L* is the adjoint of L), and the total force
    vanishes (the discrete energy is translation invariant)."""
    from ddpcm_b200 import molecules as M
    c = M.CONFIGS[2]
    m = M.to_bohr(M.config_molecule(2))
    with gpu_ctx(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"],
                 eta=c["eta"]) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
        assert out["info"]["direct"]["converged"] and out["info"]["adjoint"]["converged"]
        rng = np.random.default_rng(5)
        x = rng.standard_normal((dd.nsph, dd.nylm))
        y = rng.standard_normal((dd.nsph, dd.nylm))
        lhs = np.vdot(y, dd.lx(x))
        rhs = np.vdot(dd.lstarx(y), x)
        assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), 1.0)
        lx, lsy = dd.lx_lstarx(x, y)        # fused pass
        assert abs(np.vdot(y, lx) - np.vdot(lsy, x)) <= 1e-11 * max(abs(lhs), 1.0)
        assert abs(np.vdot(y, lx) - lhs) <= 1e-12 * max(abs(lhs), 1.0)
        F = out["fx"]
        assert np.abs(F.sum(axis=0)).max() <= 1e-9 * np.abs(F).sum()
        assert np.isfinite(out["esolv"]) and out["esolv"] < 0
    # against the oracle's full-size run (tests/golden/make_config2.py)
    import os
    from conftest import GOLDEN
    ref = np.load(os.path.join(GOLDEN, "config2_oracle.npz"))
    assert out["info"]["ncav"] == int(ref["ncav"])
    assert abs(out["esolv"] - float(ref["esolv"])) <= ESOLV_RTOL * abs(float(ref["esolv"]))
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)
    _iters_close(out, dict(iters=[int(v) for v in ref["iters"]]))


def test_edge_single_and_separated_spheres(oracle):
    # one sphere: no neighbours, every point exposed, L = D
    p = dict(lmax=4, ngrid=50, iconv=10, eps=78.3553, eta=0.1)
    for m in (dict(q=np.array([0.3]), x=np.zeros(1), y=np.zeros(1), z=np.zeros(1),
                   r=np.array([3.0])),
              dict(q=np.array([0.5, -0.5]), x=np.array([0.0, 20.0]), y=np.zeros(2),
                   z=np.zeros(2), r=np.array([3.0, 2.5]))):
        ref = oracle.energy_forces(m, p["lmax"], p["ngrid"], p["iconv"], p["eps"], p["eta"])
        with gpu_ctx(**p) as dd:
            out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
            assert dd.ncav == len(m["q"]) * dd.ngrid
            assert np.abs(dd.lx(np.ones((dd.nsph, dd.nylm)))).max() == 0.0
        assert abs(out["esolv"] - ref["esolv"]) <= 1e-12 * abs(ref["esolv"])
        np.testing.assert_allclose(out["fx"], ref["fx"], atol=1e-13)


@pytest.mark.parametrize("lmax,ngrid", [(0, 6), (1, 14), (3, 26), (12, 302), (6, 5810)])
def test_lmax_ngrid_range(oracle, lmax, ngrid):
    g = load_golden("caffeine")
    m = g["mol"]
    p = dict(lmax=lmax, ngrid=ngrid, iconv=9, eps=78.3553, eta=0.1)
    ref = oracle.energy_forces(m, lmax, ngrid, p["iconv"], p["eps"], p["eta"])
    with gpu_ctx(**p) as dd:
        out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
    assert out["info"]["ngrid"] == ref["ngrid"]
    assert abs(out["esolv"] - ref["esolv"]) <= ESOLV_RTOL * abs(ref["esolv"])
    np.testing.assert_allclose(out["fx"], ref["fx"], rtol=0, atol=FORCE_ATOL)


def test_errors_and_nonconvergence():
    from ddpcm_b200.ddcosmo import DDCosmoError, DDC_ERR_NOCONV
    g = load_golden("caffeine")
    m = g["mol"]
    with pytest.raises(DDCosmoError):
        gpu_ctx(lmax=13)
    with pytest.raises(DDCosmoError):
        gpu_ctx(eta=0.0)
    with gpu_ctx(lmax=6, ngrid=110, iconv=10, max_iter=2) as dd:
        with pytest.raises(DDCosmoError) as ei:
            dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
        assert ei.value.status == DDC_ERR_NOCONV
    with gpu_ctx() as dd:
        with pytest.raises(DDCosmoError):
            dd.lx(np.zeros((3, 49)))  # before ddinit
        with pytest.raises(DDCosmoError):
            dd.ddinit([0.0], [0.0], [0.0], [-1.0])  # negative radius


def test_sizes_beyond_32bit_indexing_are_rejected():
    """Grid fields and triple lists use 32-bit indices: nsph * ngrid at or
    above 2^31 is refused with DDC_ERR_UNSUPPORTED before any allocation."""
    from ddpcm_b200.ddcosmo import DDCosmoError
    n = 369_700  # * 5810 points > 2^31
    x = np.arange(n, dtype=np.float64) * 10.0
    z = np.zeros(n)
    with gpu_ctx(lmax=2, ngrid=5810) as dd:
        with pytest.raises(DDCosmoError) as ei:
            dd.ddinit(x, z, z, np.ones(n))
        assert ei.value.status == 6


def test_zero_guess_and_no_diis_converge_to_same_solution(oracle):
    g = load_golden("taxol")
    p, m = g["params"], g["mol"]
    from ddpcm_b200.ddcosmo import GUESS_ZERO
    sols = []
    for kw in (dict(), dict(guess=GUESS_ZERO), dict(ndiis=0)):
        with gpu_ctx(lmax=p["lmax"], ngrid=p["ngrid"], iconv=11, eps=p["eps"], eta=p["eta"],
                     **kw) as dd:
            out = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
            sols.append(out)
    for o in sols[1:]:
        assert abs(o["esolv"] - sols[0]["esolv"]) <= 1e-9 * abs(sols[0]["esolv"])
        np.testing.assert_allclose(o["fx"], sols[0]["fx"], atol=1e-9)
