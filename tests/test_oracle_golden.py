"""The CPU oracle against the reference's own regression logs (tests/*.log).

Tolerances are the print precision of the logs: energies 6 decimals
(kcal/mol), forces and dumped intermediates 8 decimals, cavity points 6
decimals, iteration norms 4 significant digits.
"""
import numpy as np
import pytest

from conftest import MOLS, TOKCAL, load_golden


@pytest.mark.parametrize("name", MOLS)
def test_energy_forces_iterations(oracle, name):
    g = load_golden(name)
    p = g["params"]
    r = oracle.energy_forces(g["mol"], p["lmax"], p["ngrid"], p["iconv"], p["eps"], p["eta"])
    assert r["rc"] == 0
    assert abs(r["esolv"] * TOKCAL - g["energy_kcal"]) <= 1e-6
    assert r["iters"] == (len(g["norms_direct"]), len(g["norms_adjoint"]))
    assert r["ngrid"] == g["ngrid_snapped"]
    np.testing.assert_allclose(r["fx"], np.array(g["forces"]), rtol=0, atol=6e-9)


@pytest.mark.parametrize("name", ["formaldehyde", "benzene", "caffeine", "taxol"])
def test_iteration_norms(oracle, name):
    g = load_golden(name)
    p, m = g["params"], g["mol"]
    d = oracle.RefDD(p["lmax"], p["ngrid"], p["iconv"], p["igrad"], p["eps"], p["eta"])
    d.init(m["x"], m["y"], m["z"], m["r"])
    phi, psi = oracle.mkrhs(m["q"], m["x"], m["y"], m["z"], d.get("ccav"), d.nylm)
    rd = d.cosmo(False, True, phi=phi, psi=psi)
    ra = d.cosmo(True, False, psi=psi)
    np.testing.assert_allclose(rd["norms"], g["norms_direct"], rtol=6e-4)
    np.testing.assert_allclose(ra["norms"], g["norms_adjoint"], rtol=6e-4)


def test_formaldehyde_intermediates(oracle):
    g = load_golden("formaldehyde")
    p, m = g["params"], g["mol"]
    d = oracle.RefDD(p["lmax"], p["ngrid"], p["iconv"], p["igrad"], p["eps"], p["eta"])
    d.init(m["x"], m["y"], m["z"], m["r"])
    tol = 6e-9
    np.testing.assert_allclose(d.get("facs"), g["facs"], atol=tol)
    # the reference prints facs under the label 'facl' (ddcosmo.f90:276)
    np.testing.assert_allclose(d.get("facs"), g["facl_as_printed"], atol=tol)
    np.testing.assert_allclose(d.get("basis"), np.array(g["basis"]), atol=tol)
    flat = d.get("grid").ravel()
    ng = d.ngrid
    printed = np.stack([flat[c * ng:(c + 1) * ng] for c in range(3)])  # ptcart view
    np.testing.assert_allclose(printed, np.array(g["grid_as_printed"]), atol=tol)
    np.testing.assert_allclose(d.get("w"), g["weights"], atol=tol)
    inl, nl = d.csr()
    assert list(inl + 1) == g["inl"] and list(nl + 1) == g["nl"]
    np.testing.assert_allclose(d.get("fi"), np.array(g["fi"]), atol=tol)
    np.testing.assert_allclose(d.get("ui"), np.array(g["ui"]), atol=tol)
    np.testing.assert_allclose(d.get("ccav"), np.array(g["ccav"]), atol=6e-7)
    phi, psi = oracle.mkrhs(m["q"], m["x"], m["y"], m["z"], d.get("ccav"), d.nylm)
    np.testing.assert_allclose(d.rhs(phi), np.array(g["rhs"]), atol=tol)
    np.testing.assert_allclose(psi, np.array(g["psi"]), atol=tol)
    rd = d.cosmo(False, True, phi=phi, psi=psi)
    np.testing.assert_allclose(rd["sigma"], np.array(g["X"]), atol=tol)
    ra = d.cosmo(True, False, psi=psi)
    np.testing.assert_allclose(ra["sigma"], np.array(g["S"]), atol=tol)
    np.testing.assert_allclose(ra["sigma"] @ d.get("basis").T, np.array(g["xi"]), atol=tol)
    fep = 0.5 * (p["eps"] - 1.0) / p["eps"]
    # forces_dd prints before its final fep scaling (forces_dd.f90:139-161)
    fdd = d.forces_dd(phi, rd["sigma"], ra["sigma"])
    np.testing.assert_allclose(fdd / fep, np.array(g["forces_dd"]), atol=tol)
    np.testing.assert_allclose(d.mkzeta(ra["sigma"]), g["zeta"], atol=tol)


def test_benzene_solutions(oracle):
    g = load_golden("benzene")
    p, m = g["params"], g["mol"]
    d = oracle.RefDD(p["lmax"], p["ngrid"], p["iconv"], p["igrad"], p["eps"], p["eta"])
    d.init(m["x"], m["y"], m["z"], m["r"])
    phi, psi = oracle.mkrhs(m["q"], m["x"], m["y"], m["z"], d.get("ccav"), d.nylm)
    np.testing.assert_allclose(d.cosmo(False, True, phi=phi, psi=psi)["sigma"], np.array(g["X"]),
                               atol=6e-9)
    np.testing.assert_allclose(d.cosmo(True, False, psi=psi)["sigma"], np.array(g["S"]), atol=6e-9)


def test_lebedev_grids_integrate_polynomials(oracle):
    """Every Lebedev table integrates low-order monomials exactly."""
    sizes = [6, 14, 26, 38, 50, 74, 86, 110, 146, 170, 194, 230, 266, 302, 350, 434, 590, 770,
             974, 1202, 1454, 1730, 2030, 2354, 2702, 3074, 3470, 3890, 4334, 4802, 5294, 5810]
    fourpi = 4.0 * np.pi
    for n in sizes:
        g, w = oracle.llgrid(n)
        assert abs(w.sum() - fourpi) < 1e-12
        np.testing.assert_allclose(np.linalg.norm(g, axis=1), 1.0, atol=1e-14)
        x, y, z = g.T
        np.testing.assert_allclose(w @ (z * z), fourpi / 3, atol=1e-12)
        if n >= 14:
            np.testing.assert_allclose(w @ z ** 4, fourpi / 5, atol=1e-12)
            np.testing.assert_allclose(w @ (x * x * y * y), fourpi / 15, atol=1e-12)
        assert abs(w @ z) < 1e-13


def test_ngrid_snapping(oracle):
    # nearest size, ties to the smaller one (ddcosmo.f90:188-199)
    assert oracle.snap_ngrid(110) == 110
    assert oracle.snap_ngrid(100) == 110
    assert oracle.snap_ngrid(98) == 86  # |86-98| = 12 == |110-98|: first wins
    assert oracle.snap_ngrid(1) == 6
    assert oracle.snap_ngrid(100000) == 5810


def test_switch_function(oracle):
    eta = 0.1
    assert oracle.lib().ref_fsw(0.5, eta) == 1.0
    assert oracle.lib().ref_fsw(1.0, eta) == 0.0
    ts = np.linspace(0.9001, 0.9999, 50)
    f = np.array([oracle.lib().ref_fsw(t, eta) for t in ts])
    df = np.array([oracle.lib().ref_dfsw(t, eta) for t in ts])
    assert np.all(np.diff(f) < 0) and np.all((f > 0) & (f < 1))
    # derivative against a central difference
    h = 1e-7
    fd = np.array([(oracle.lib().ref_fsw(t + h, eta) - oracle.lib().ref_fsw(t - h, eta)) / (2 * h)
                   for t in ts])
    np.testing.assert_allclose(df, fd, rtol=1e-5, atol=1e-6)


def test_gjinv_singular_and_solve(oracle):
    import ctypes
    L = oracle.lib()
    a = np.array([[0.0, 1.0, 1.0], [1.0, 2.0, 0.5], [1.0, 0.5, 3.0]]).T.copy()
    b = np.array([1.0, 0.0, 0.0])
    ref = np.linalg.solve(a.T, b)
    dp = ctypes.POINTER(ctypes.c_double)
    ok = L.ref_gjinv(3, a.ctypes.data_as(dp), b.ctypes.data_as(dp))
    assert ok == 1
    np.testing.assert_allclose(b, ref, rtol=1e-14)
    s = np.ones((3, 3))
    bb = np.ones(3)
    assert L.ref_gjinv(3, s.ctypes.data_as(dp), bb.ctypes.data_as(dp)) == 0
