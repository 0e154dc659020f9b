"""Synthetic molecules and the reference's Input.txt format.

No public dataset exists for this path; molecules are generated from seeded
PCG64 streams (numpy ``default_rng``):

* radii drawn uniformly from {1.20, 1.70, 1.55, 1.52} angstrom, each x1.1;
* point charges at the centres, U[-0.5, 0.5], shifted to zero net charge;
* positions by a self-avoiding random walk: step length U[1.4, 1.6] angstrom
  in a uniform random direction, a step is rejected when it comes closer than
  1.0 angstrom to an existing centre or, for a globule, leaves the ball of
  radius R = (3N / (4 pi rho))^(1/3) with rho = 0.1 atoms/angstrom^3.  When a
  walk is stuck (64 rejections in a row) it restarts from a random existing
  centre, which keeps the globule compact.

Input.txt (main.f90:129-148): iprint, nproc, lmax, ngrid, iconv, igrad, eps,
eta, n, then n rows ``q x y z r`` in angstrom; main converts to bohr with
toang = 0.52917721092 (main.f90:99, 149-153).
"""
import math

import numpy as np

TOANG = 0.52917721092
RADII = np.array([1.20, 1.70, 1.55, 1.52]) * 1.1


def _walk(rng, n, confine_radius=None, min_dist=1.0, step=(1.4, 1.6), max_reject=64):
    cell = min_dist
    grid = {}
    pos = np.zeros((n, 3))

    def key(p):
        return (int(math.floor(p[0] / cell)), int(math.floor(p[1] / cell)),
                int(math.floor(p[2] / cell)))

    def ok(p, count):
        if confine_radius is not None and p[0] * p[0] + p[1] * p[1] + p[2] * p[2] > \
                confine_radius * confine_radius:
            return False
        kx, ky, kz = key(p)
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    for idx in grid.get((kx + dx, ky + dy, kz + dz), ()):
                        d = pos[idx] - p
                        if d[0] * d[0] + d[1] * d[1] + d[2] * d[2] < min_dist * min_dist:
                            return False
        return True

    pos[0] = 0.0
    grid.setdefault(key(pos[0]), []).append(0)
    cur = pos[0].copy()
    count = 1
    rejects = 0
    while count < n:
        d = rng.normal(size=3)
        d /= np.linalg.norm(d)
        cand = cur + d * rng.uniform(step[0], step[1])
        if ok(cand, count):
            pos[count] = cand
            grid.setdefault(key(cand), []).append(count)
            cur = cand
            count += 1
            rejects = 0
        else:
            rejects += 1
            if rejects >= max_reject:
                cur = pos[rng.integers(0, count)].copy()
                rejects = 0
    return pos


def make_molecule(n, seed, globule=True, density=0.1):
    """Synthetic molecule in angstrom: dict(q, x, y, z, r) (+ seed, n)."""
    rng = np.random.default_rng(seed)
    R = (3.0 * n / (4.0 * math.pi * density)) ** (1.0 / 3.0) if globule else None
    pos = _walk(rng, n, confine_radius=R)
    r = RADII[rng.integers(0, len(RADII), size=n)]
    q = rng.uniform(-0.5, 0.5, size=n)
    q -= q.mean()
    return dict(q=q, x=pos[:, 0].copy(), y=pos[:, 1].copy(), z=pos[:, 2].copy(), r=r, seed=seed,
                n=n)


def to_bohr(mol):
    """Convert x, y, z, r from angstrom to bohr as main.f90:149-153 does."""
    tobohr = 1.0 / TOANG
    out = dict(mol)
    for k in "xyzr":
        out[k] = np.asarray(mol[k], dtype=np.float64) * tobohr
    return out


# The benchmark configurations (sizes and solver settings).
CONFIGS = {
    0: dict(n=12, globule=False, lmax=6, ngrid=110, eta=0.1, eps=78.3553, iconv=10, seed=1000),
    1: dict(n=600, globule=True, lmax=8, ngrid=302, eta=0.1, eps=78.3553, iconv=10, seed=1001),
    2: dict(n=20000, globule=True, lmax=10, ngrid=590, eta=0.1, eps=78.3553, iconv=10, seed=1002),
    # profiling case: same settings as 2 at 5,000 spheres (working set above
    # L2, small enough for a full counter capture)
    9: dict(n=5000, globule=True, lmax=10, ngrid=590, eta=0.1, eps=78.3553, iconv=10, seed=1009),
}


# batched workload: 256 globules of log-uniform size in [20, 2000] spheres
BATCH_CONFIG = dict(count=256, lo=20, hi=2000, lmax=6, ngrid=302, eta=0.1, eps=78.3553, iconv=10,
                    seed=3000)


def config_molecule(k):
    c = CONFIGS[k]
    return make_molecule(c["n"], c["seed"], globule=c["globule"])


def batch_molecules(count=256, lo=20, hi=2000, seed=3000):
    """Config of uneven molecules: sizes log-uniform in [lo, hi], one seed each."""
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(math.log(lo), math.log(hi), size=count)).astype(int)
    return [make_molecule(int(s), seed + 1 + i) for i, s in enumerate(sizes)]


def trajectory(mol, frames, sigma=0.05, seed=0):
    """A synthetic trajectory from ``mol`` (angstrom): each frame moves every
    centre of the previous frame by a Gaussian displacement of ``sigma``
    angstrom per coordinate.  Returns a list of ``frames`` molecules, the first
    being ``mol`` itself; charges and radii do not change."""
    rng = np.random.default_rng(seed)
    out = [dict(mol)]
    for _ in range(frames - 1):
        prev = out[-1]
        nxt = dict(prev)
        for k in "xyz":
            nxt[k] = np.asarray(prev[k], dtype=np.float64) + rng.normal(0.0, sigma, size=len(prev[k]))
        out.append(nxt)
    return out


def write_input(path, mol, lmax, ngrid, iconv, eps, eta, igrad=1, iprint=1, nproc=1):
    """Write a reference-format Input.txt (angstrom)."""
    with open(path, "w") as f:
        for v, c in ((iprint, "print flag"), (nproc, "OpenMP threads"), (lmax, "lmax"),
                     (ngrid, "ngrid"), (iconv, "iconv"), (igrad, "igrad")):
            f.write(f"{v:<16d} ! {c}\n")
        f.write(f"{eps:<16.4f} ! eps\n{eta:<16.4f} ! eta\n{len(mol['q']):<16d} ! n\n")
        for i in range(len(mol["q"])):
            f.write(f"{mol['q'][i]: .8f} {mol['x'][i]: .8f} {mol['y'][i]: .8f} "
                    f"{mol['z'][i]: .8f} {mol['r'][i]: .8f}\n")


def read_input(path):
    """Read a reference-format Input.txt; returns (params, mol in angstrom)."""
    lines = open(path).read().splitlines()
    v = [ln.split()[0] for ln in lines[:9]]
    fnum = lambda s: float(s.replace("D", "E").replace("d", "e"))
    params = dict(iprint=int(v[0]), nproc=int(v[1]), lmax=int(v[2]), ngrid=int(v[3]),
                  iconv=int(v[4]), igrad=int(v[5]), eps=fnum(v[6]), eta=fnum(v[7]))
    n = int(v[8])
    rows = np.array([[fnum(t) for t in ln.split()[:5]] for ln in lines[9:9 + n]])
    mol = dict(q=rows[:, 0], x=rows[:, 1], y=rows[:, 2], z=rows[:, 3], r=rows[:, 4], n=n)
    return params, mol
