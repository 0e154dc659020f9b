"""ctypes wrapper around the CPU oracle ``ddc_ref.c``.

TEST INFRASTRUCTURE ONLY: used by ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` as the checker / baseline.  The product
library (``ddpcm_b200``) never imports this module.

Every function mirrors a reference routine (file:line given on each) and takes
and returns numpy arrays in the reference's column-major shapes, stored as
C-contiguous arrays of shape (ncol, nrow): e.g. X(nylm, nsph) is an array of
shape (nsph, nylm).
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _host_tag():
    """Build folder per host CPU: the oracle is compiled with -march=native."""
    import hashlib
    try:
        info = open("/proc/cpuinfo").read()
        model = next((ln for ln in info.splitlines() if ln.startswith("model name")), "")
        flags = next((ln for ln in info.splitlines() if ln.startswith("flags")), "")
        return hashlib.sha1((model + flags).encode()).hexdigest()[:10]
    except OSError:
        return "generic"


BUILD_DIR = os.path.join(HERE, "_build", _host_tag())
LIB_PATH = os.path.join(BUILD_DIR, "libddc_ref.so")

_lib = None
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def build():
    subprocess.run(["make", "-s", "-C", HERE, "OUT=" + BUILD_DIR], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        L.ref_create.restype = ctypes.c_void_p
        L.ref_create.argtypes = [ctypes.c_int] * 4 + [ctypes.c_double] * 2 + [ctypes.c_int]
        L.ref_destroy.argtypes = [ctypes.c_void_p]
        L.ref_init.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_dp] * 4
        L.ref_sizes.argtypes = [ctypes.c_void_p, _ip]
        L.ref_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
        L.ref_get_csr.argtypes = [ctypes.c_void_p, _ip, _ip]
        L.ref_lx.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ref_lstarx.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ref_ldm1x.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ref_hnorm.argtypes = [ctypes.c_void_p, _dp]
        L.ref_hnorm.restype = ctypes.c_double
        L.ref_rhs.argtypes = [ctypes.c_void_p, _dp, _dp]
        L.ref_cosmo.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp,
                                _dp, _ip, _dp]
        L.ref_forces_dd.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp]
        L.ref_forces_dd_range.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, ctypes.c_int,
                                          ctypes.c_int]
        L.ref_forces_dd_ranges.argtypes = [ctypes.c_void_p, _dp, _dp, _dp, _dp, _ip,
                                           ctypes.c_int]
        L.ref_num_threads.restype = ctypes.c_int
        L.ref_mkxi.argtypes = [ctypes.c_void_p, _dp, _dp, ctypes.c_int]
        L.ref_mkrhs.argtypes = [ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, _dp, _dp,
                                ctypes.c_int, _dp]
        L.ref_efld.argtypes = [ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp]
        L.ref_energy_forces.argtypes = [ctypes.c_void_p, ctypes.c_int] + [_dp] * 5 + [_dp] * 4 + [_ip]
        L.ref_energy_forces.restype = ctypes.c_int
        L.ref_snap_ngrid.argtypes = [ctypes.c_int]
        L.ref_snap_ngrid.restype = ctypes.c_int
        L.ref_llgrid.argtypes = [ctypes.c_int, _dp, _dp]
        L.ref_fsw.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_fsw.restype = ctypes.c_double
        L.ref_dfsw.argtypes = [ctypes.c_double, ctypes.c_double]
        L.ref_dfsw.restype = ctypes.c_double
        L.ref_gjinv.argtypes = [ctypes.c_int, _dp, _dp]
        L.ref_gjinv.restype = ctypes.c_int
        L.ref_diis_sample.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.ref_diis_sample.restype = ctypes.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(_dp)


def _c(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class RefDD:
    """Oracle context: the reference's module state after ``ddinit``."""

    def __init__(self, lmax, ngrid, iconv, igrad, eps, eta, nthreads=0):
        self.L = lib()
        self.h = self.L.ref_create(lmax, ngrid, iconv, igrad, eps, eta, nthreads)
        self.lmax, self.iconv, self.igrad, self.eps, self.eta = lmax, iconv, igrad, eps, eta

    def __del__(self):
        if getattr(self, "h", None):
            self.L.ref_destroy(self.h)
            self.h = None

    # ddinit (ddcosmo.f90:159)
    def init(self, x, y, z, r):
        x, y, z, r = map(_c, (x, y, z, r))
        self.L.ref_init(self.h, len(x), _p(x), _p(y), _p(z), _p(r))
        s = (ctypes.c_int * 5)()
        self.L.ref_sizes(self.h, s)
        self.nsph, self.ncav, self.nylm, self.ngrid, self.nnz = list(s)
        return self

    def get(self, name):
        shapes = {"grid": (self.ngrid, 3), "w": (self.ngrid,), "basis": (self.ngrid, self.nylm),
                  "facs": (self.nylm,), "facl": (self.nylm,), "fi": (self.nsph, self.ngrid),
                  "ui": (self.nsph, self.ngrid), "zi": (self.nsph, self.ngrid, 3),
                  "ccav": (self.ncav, 3), "csph": (self.nsph, 3), "rsph": (self.nsph,)}
        out = np.zeros(shapes[name])
        self.L.ref_get(self.h, name.encode(), _p(out))
        return out

    def csr(self):
        inl = np.zeros(self.nsph + 1, dtype=np.int32)
        nl = np.zeros(max(self.nnz, 1), dtype=np.int32)
        self.L.ref_get_csr(self.h, inl.ctypes.data_as(_ip), nl.ctypes.data_as(_ip))
        return inl, nl[: self.nnz]

    def _op(self, fn, x):
        x = _c(x)
        y = np.zeros_like(x)
        fn(self.h, _p(x), _p(y))
        return y

    def lx(self, x):           # matvec.f90:94
        return self._op(self.L.ref_lx, x)

    def lstarx(self, x):       # matvec.f90:161
        return self._op(self.L.ref_lstarx, x)

    def ldm1x(self, x):        # matvec.f90:246
        return self._op(self.L.ref_ldm1x, x)

    def hnorm(self, x):        # matvec.f90:281
        return self.L.ref_hnorm(self.h, _p(_c(x)))

    def rhs(self, phi):        # cosmo.f90:104-117 (wghpot + intrhs)
        phi = _c(phi)
        out = np.zeros((self.nsph, self.nylm))
        self.L.ref_rhs(self.h, _p(phi), _p(out))
        return out

    def cosmo(self, star, cart, phi=None, glm=None, psi=None):
        """cosmo(star, cart, phi, glm, psi, sigma, esolv) (cosmo.f90:1)."""
        z = np.zeros((self.nsph, self.nylm))
        phi = _c(phi) if phi is not None else np.zeros(max(self.ncav, 1))
        glm = _c(glm) if glm is not None else z.copy()
        psi = _c(psi) if psi is not None else z.copy()
        sigma = z.copy()
        es = ctypes.c_double(0.0)
        it = ctypes.c_int(0)
        norms = np.zeros(1024)
        rc = self.L.ref_cosmo(self.h, int(star), int(cart), _p(phi), _p(glm), _p(psi), _p(sigma),
                              ctypes.byref(es), ctypes.byref(it), _p(norms))
        return dict(sigma=sigma, esolv=es.value, iters=it.value, norms=norms[: it.value].copy(),
                    converged=(rc == 0))

    def forces_dd(self, phi, sigma, s):   # forces_dd.f90:1
        fx = np.zeros((self.nsph, 3))
        self.L.ref_forces_dd(self.h, _p(_c(phi)), _p(_c(sigma)), _p(_c(s)), _p(fx))
        return fx

    def forces_dd_range(self, phi, sigma, s, i0, i1):
        fx = np.zeros((self.nsph, 3))
        self.L.ref_forces_dd_range(self.h, _p(_c(phi)), _p(_c(sigma)), _p(_c(s)), _p(fx), i0, i1)
        return fx

    def diis_sample(self, iters):
        """Seconds of the reference's serial Jacobi/DIIS vector work over
        `iters` iterations at this context's size (operator excluded)."""
        sec, op = ctypes.c_double(0.0), ctypes.c_double(0.0)
        self.L.ref_diis_sample(self.h, iters, ctypes.byref(sec), ctypes.byref(op))
        return max(sec.value - op.value, 0.0)

    def forces_dd_ranges(self, phi, sigma, s, ranges):
        """forces_dd over several sphere ranges [(i0, i1), ...] in one call."""
        fx = np.zeros((self.nsph, 3))
        rg = np.ascontiguousarray(np.asarray(ranges, dtype=np.int32).reshape(-1))
        self.L.ref_forces_dd_ranges(self.h, _p(_c(phi)), _p(_c(sigma)), _p(_c(s)), _p(fx),
                                    rg.ctypes.data_as(_ip), len(rg) // 2)
        return fx

    def mkzeta(self, s):      # ddcosmo.f90:1787
        out = np.zeros(max(self.ncav, 1))
        self.L.ref_mkxi(self.h, _p(_c(s)), _p(out), 1)
        return out[: self.ncav]

    def mkxi(self, s):        # ddcosmo.f90:1758
        out = np.zeros(max(self.ncav, 1))
        self.L.ref_mkxi(self.h, _p(_c(s)), _p(out), 0)
        return out[: self.ncav]


def mkrhs(q, x, y, z, ccav, nylm):
    """mkrhs.f90:86-123: phi at cavity points and psi."""
    q, x, y, z, ccav = map(_c, (q, x, y, z, ccav))
    ncav = ccav.shape[0]
    phi = np.zeros(max(ncav, 1))
    psi = np.zeros((len(q), nylm))
    lib().ref_mkrhs(len(q), _p(q), _p(x), _p(y), _p(z), ncav, _p(ccav), _p(phi), nylm, _p(psi))
    return phi[:ncav], psi


def efld(src, csrc, ctrg):
    """efld.f90:81-116: field of point sources at targets; csrc (nsrc,3), ctrg (ntrg,3)."""
    src, csrc, ctrg = map(_c, (src, csrc, ctrg))
    ef = np.zeros((ctrg.shape[0], 3))
    lib().ref_efld(len(src), _p(src), _p(csrc), ctrg.shape[0], _p(ctrg), _p(ef))
    return ef


def energy_forces(mol, lmax, ngrid, iconv, eps, eta, igrad=1, nthreads=0):
    """The main.f90 flow (main.f90:164-265) on a molecule in bohr.

    mol: dict with q, x, y, z, r arrays (bohr).  Returns dict(esolv, sigma, s,
    fx, iters, ncav, ngrid, nylm)."""
    d = RefDD(lmax, ngrid, iconv, igrad, eps, eta, nthreads)
    n = len(mol["q"])
    nylm = (lmax + 1) ** 2
    q, x, y, z, r = (_c(mol[k]) for k in "qxyzr")
    es = ctypes.c_double(0.0)
    sigma = np.zeros((n, nylm))
    s = np.zeros((n, nylm))
    fx = np.zeros((n, 3))
    it = (ctypes.c_int * 2)()
    rc = lib().ref_energy_forces(d.h, n, _p(q), _p(x), _p(y), _p(z), _p(r), ctypes.byref(es),
                                 _p(sigma), _p(s), _p(fx), it)
    sz = (ctypes.c_int * 5)()
    lib().ref_sizes(d.h, sz)
    return dict(rc=rc, esolv=es.value, sigma=sigma, s=s, fx=fx, iters=(it[0], it[1]),
                ncav=sz[1], nylm=sz[2], ngrid=sz[3])


def num_threads():
    return lib().ref_num_threads()


def snap_ngrid(n):
    return lib().ref_snap_ngrid(n)


def llgrid(ngrid):
    w = np.zeros(ngrid)
    g = np.zeros((ngrid, 3))
    rc = lib().ref_llgrid(ngrid, _p(w), _p(g))
    assert rc == 0
    return g, w
