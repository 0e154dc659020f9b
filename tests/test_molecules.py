import numpy as np

from ddpcm_b200 import molecules as M


def test_generator_is_deterministic_and_valid():
    a = M.make_molecule(300, 7)
    b = M.make_molecule(300, 7)
    for k in "qxyzr":
        np.testing.assert_array_equal(a[k], b[k])
    pos = np.stack([a["x"], a["y"], a["z"]], 1)
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) + np.eye(300) * 10
    assert d.min() >= 1.0 - 1e-12
    R = (3 * 300 / (4 * np.pi * 0.1)) ** (1 / 3)
    assert np.linalg.norm(pos, axis=1).max() <= R + 1e-9
    assert abs(a["q"].sum()) < 1e-12 and np.all(np.abs(a["q"]) <= 1.0)
    assert set(np.round(a["r"], 6)) <= set(np.round(M.RADII, 6))


def test_walk_steps_and_unconfined_config0():
    m = M.config_molecule(0)
    assert m["n"] == 12
    pos = np.stack([m["x"], m["y"], m["z"]], 1)
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) + np.eye(12) * 10
    assert d.min() >= 1.0 - 1e-12


def test_input_roundtrip(tmp_path):
    m = M.make_molecule(20, 3)
    p = tmp_path / "Input.txt"
    M.write_input(str(p), m, lmax=6, ngrid=110, iconv=10, eps=78.3553, eta=0.1)
    params, m2 = M.read_input(str(p))
    assert params["lmax"] == 6 and params["iconv"] == 10 and abs(params["eta"] - 0.1) < 1e-12
    for k in "qxyzr":
        np.testing.assert_allclose(m2[k], m[k], atol=1e-8)


def test_batch_sizes():
    mols = M.batch_molecules(count=16, lo=20, hi=200, seed=5)
    ns = [m["n"] for m in mols]
    assert min(ns) >= 20 and max(ns) <= 200 and len(set(ns)) > 4


def test_trajectory_displacements():
    m = M.make_molecule(200, 5)
    tr = M.trajectory(m, 4, sigma=0.05, seed=9)
    assert len(tr) == 4 and tr[0]["x"] is m["x"]
    for a, b in zip(tr[:-1], tr[1:]):
        d = np.concatenate([b[k] - a[k] for k in "xyz"])
        assert abs(d.std() - 0.05) < 0.01
        assert np.array_equal(a["q"], b["q"]) and np.array_equal(a["r"], b["r"])
    again = M.trajectory(m, 4, sigma=0.05, seed=9)
    assert np.array_equal(again[3]["z"], tr[3]["z"])
