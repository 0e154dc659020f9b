"""Python mirror of the reference's ddCOSMO interface over the C ABI.

The reference is a Fortran module (``module ddcosmo``, ddcosmo.f90) whose
state is set by ``ddinit`` and used by ``cosmo``, ``forces_dd``, ``ddmkzeta``,
``ddmkxi`` and the user routines ``mkrhs``/``efld``.  ``DDCosmo`` holds one
such module state on the GPU (a ``ddc_ctx`` of ``libddcosmo_gpu.so``) and
exposes the same routines, with the same argument meaning, as methods.

Arrays follow the reference's column-major shapes, held as C-contiguous
numpy arrays with the axes reversed: X(nylm, nsph) is an array of shape
(nsph, nylm), ccav(3, ncav) one of shape (ncav, 3), ui(ngrid, nsph) one of
shape (nsph, ngrid).

There is no CPU fallback: constructing ``DDCosmo`` without the compiled
library or without a CUDA device raises ``DDCosmoError``.
"""
import ctypes
import os

import numpy as np

from .build import LIB

DDC_OK = 0
DDC_ERR_PARAM = 1
DDC_ERR_NOCONV = 5
PREC_FP64, PREC_MIXED = 0, 1
GUESS_REFERENCE, GUESS_ZERO, GUESS_USER, GUESS_LEARNED = 0, 1, 2, 3
TOANG = 0.52917721092          # main.f90:99
TOKCAL = 627.509469            # main.f90:99

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


class DDCosmoError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"ddcosmo status {status}: {msg}")
        self.status = status


class Params(ctypes.Structure):
    _fields_ = [("lmax", ctypes.c_int), ("ngrid", ctypes.c_int), ("iconv", ctypes.c_int),
                ("igrad", ctypes.c_int), ("eps", ctypes.c_double), ("eta", ctypes.c_double),
                ("iprint", ctypes.c_int), ("max_iter", ctypes.c_int), ("ndiis", ctypes.c_int),
                ("precision", ctypes.c_int), ("guess", ctypes.c_int), ("device", ctypes.c_int),
                ("device_pointers", ctypes.c_int), ("stream", ctypes.c_void_p),
                ("timing", ctypes.c_int), ("pair_solves", ctypes.c_int)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("converged", ctypes.c_int),
                ("diis_restarts", ctypes.c_int), ("refinements", ctypes.c_int),
                ("final_norm", ctypes.c_double), ("seconds", ctypes.c_double),
                ("norms", ctypes.c_double * 256)]

    def as_dict(self):
        it = self.iterations
        return dict(iterations=it, converged=bool(self.converged),
                    diis_restarts=self.diis_restarts, refinements=self.refinements,
                    final_norm=self.final_norm, seconds=self.seconds,
                    norms=list(self.norms[: min(it, 256)]))


class RunInfo(ctypes.Structure):
    _fields_ = [("direct", SolveInfo), ("adjoint", SolveInfo), ("t_init", ctypes.c_double),
                ("t_mkrhs", ctypes.c_double), ("t_direct", ctypes.c_double),
                ("t_adjoint", ctypes.c_double), ("t_forces", ctypes.c_double),
                ("t_efld", ctypes.c_double), ("nsph", ctypes.c_int), ("ncav", ctypes.c_int),
                ("nylm", ctypes.c_int), ("ngrid", ctypes.c_int), ("ntriples", ctypes.c_longlong),
                ("npairs", ctypes.c_int)]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k not in ("direct", "adjoint")}
        d["direct"] = self.direct.as_dict()
        d["adjoint"] = self.adjoint.as_dict()
        return d


_lib = None

# C ABI entry points and their argument types (include/ddcosmo_gpu.h)
_SIGS = {
    "ddc_default_params": [ctypes.POINTER(Params)],
    "ddc_create": [ctypes.POINTER(Params), ctypes.POINTER(ctypes.c_void_p)],
    "ddc_destroy": [ctypes.c_void_p],
    "ddc_init": [ctypes.c_void_p, ctypes.c_int] + [_dp] * 4,
    "ddc_sizes": [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_int)] * 4,
    "ddc_get_ccav": [ctypes.c_void_p, _dp],
    "ddc_get_ui": [ctypes.c_void_p, _dp],
    "ddc_get_csph": [ctypes.c_void_p, _dp],
    "ddc_get_grid": [ctypes.c_void_p, _dp, _dp],
    "ddc_mkrhs": [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp, _dp, ctypes.c_int, _dp, _dp,
                  ctypes.c_int, _dp],
    "ddc_cosmo": [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp, _dp, _dp,
                  ctypes.POINTER(SolveInfo)],
    "ddc_forces_dd": [ctypes.c_void_p, _dp, _dp, _dp, _dp],
    "ddc_mkzeta": [ctypes.c_void_p, _dp, _dp],
    "ddc_mkxi": [ctypes.c_void_p, _dp, _dp],
    "ddc_efld": [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp],
    "ddc_energy_forces": [ctypes.c_void_p, ctypes.c_int] + [_dp] * 5 + [_dp] * 4
                         + [ctypes.POINTER(RunInfo)],
    "ddc_lx": [ctypes.c_void_p, _dp, _dp],
    "ddc_lstarx": [ctypes.c_void_p, _dp, _dp],
    "ddc_lx_lstarx": [ctypes.c_void_p, _dp, _dp, _dp, _dp],
    "ddc_ldm1x": [ctypes.c_void_p, _dp, _dp],
    "ddc_hnorm": [ctypes.c_void_p, _dp, _dp],
    "ddc_rhs": [ctypes.c_void_p, _dp, _dp],
    "ddc_launch_count": [ctypes.c_void_p],
    "ddc_last_error": [ctypes.c_void_p],
    "ddc_status_string": [ctypes.c_int],
    "ddc_stage_count": [],
    "ddc_stage_name": [ctypes.c_int],
    "ddc_stage_times": [ctypes.c_void_p, _dp, ctypes.POINTER(ctypes.c_longlong)],
    "ddc_reset_stage_times": [ctypes.c_void_p],
    "ddc_set_timed_stages": [ctypes.c_void_p, ctypes.c_uint],
    "ddc_fp64_peak": [ctypes.c_int, _dp],
    "ddc_fp32_peak": [ctypes.c_int, _dp],
    "ddc_batch_energy_forces": [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
                               + [_dp] * 5 + [_dp, _dp, ctypes.POINTER(ctypes.c_int),
                                              ctypes.POINTER(RunInfo)],
    "ddc_guess_create": [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                         ctypes.POINTER(ctypes.c_void_p)],
    "ddc_guess_destroy": [ctypes.c_void_p],
    "ddc_guess_last_error": [ctypes.c_void_p],
    "ddc_guess_sizes": [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int),
                        ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_longlong)],
    "ddc_guess_get_params": [ctypes.c_void_p, _fp],
    "ddc_guess_set_params": [ctypes.c_void_p, _fp],
    "ddc_guess_init_random": [ctypes.c_void_p, ctypes.c_ulonglong],
    "ddc_guess_fit_scaling": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_longlong],
    "ddc_guess_train_epoch": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                              ctypes.c_longlong, ctypes.c_int, ctypes.c_float, _dp],
    "ddc_guess_predict": [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong],
    "ddc_guess_features": [ctypes.c_void_p, ctypes.c_void_p],
    "ddc_guess_targets": [ctypes.c_void_p, ctypes.c_void_p],
    "ddc_set_guess_model": [ctypes.c_void_p, ctypes.c_void_p],
}


def stage_mask(L, names=None):
    """Bit mask of ddc_set_timed_stages for the named stages (None: all);
    an unknown name raises ValueError."""
    if names is None:
        return 0xFFFFFFFF
    idx = {L.ddc_stage_name(k).decode(): k for k in range(L.ddc_stage_count())}
    mask = 0
    for n in names:
        if n not in idx:
            raise ValueError(f"unknown stage {n!r}; stages: {sorted(idx)}")
        mask |= 1 << idx[n]
    return mask


def load_library(path=None):
    """Load libddcosmo_gpu.so (building it first when the sources changed and
    nvcc is present).  Raises DDCosmoError when the library is missing."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB
    if not os.path.exists(path):
        try:
            from .build import build
            build()
        except Exception as e:  # no nvcc: fail loudly, there is no fallback
            raise DDCosmoError(-1, f"CUDA library {path} missing and could not be built: {e}")
    L = ctypes.CDLL(path)
    for name, args in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = ctypes.c_int
    L.ddc_launch_count.restype = ctypes.c_longlong
    L.ddc_last_error.restype = ctypes.c_char_p
    L.ddc_status_string.restype = ctypes.c_char_p
    L.ddc_stage_name.restype = ctypes.c_char_p
    L.ddc_guess_last_error.restype = ctypes.c_char_p
    _lib = L
    return L


def fp64_peak_gflops(device=0):
    """Measured FP64 FMA throughput of the device (GFLOP/s)."""
    v = ctypes.c_double()
    st = load_library().ddc_fp64_peak(device, ctypes.byref(v))
    if st != DDC_OK:
        raise DDCosmoError(st, "fp64 probe failed")
    return v.value


def fp32_peak_gflops(device=0):
    """Measured FP32 FMA throughput of the device (GFLOP/s)."""
    v = ctypes.c_double()
    st = load_library().ddc_fp32_peak(device, ctypes.byref(v))
    if st != DDC_OK:
        raise DDCosmoError(st, "fp32 probe failed")
    return v.value


def _p(a):
    if a is None:
        return None
    if isinstance(a, int):          # raw device pointer (device_pointers=1)
        return ctypes.cast(ctypes.c_void_p(a), _dp)
    return a.ctypes.data_as(_dp)


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


class DDCosmo:
    """One ddCOSMO module state on a GPU (ddcosmo.f90:87-127).

    Parameters mirror the Input.txt scalars (main.f90:129-136): lmax, ngrid,
    iconv, igrad, eps, eta, iprint; plus max_iter (200), ndiis (25),
    precision, guess, device and pair_solves (energy_forces solves the
    direct and adjoint systems together with the fused L / L* pass).
    """

    def __init__(self, lmax=6, ngrid=110, iconv=7, igrad=1, eps=78.3553, eta=0.2, iprint=0,
                 max_iter=200, ndiis=25, precision=PREC_FP64, guess=GUESS_REFERENCE, device=0,
                 device_pointers=0, stream=None, timing=0, pair_solves=1):
        self.L = load_library()
        p = Params()
        self.L.ddc_default_params(ctypes.byref(p))
        p.lmax, p.ngrid, p.iconv, p.igrad = lmax, ngrid, iconv, igrad
        p.eps, p.eta, p.iprint = eps, eta, iprint
        p.max_iter, p.ndiis, p.precision, p.guess, p.device = (max_iter, ndiis, precision, guess,
                                                                device)
        p.device_pointers, p.timing = int(device_pointers), int(timing)
        p.pair_solves = int(pair_solves)
        p.stream = stream
        self.params = p
        h = ctypes.c_void_p()
        st = self.L.ddc_create(ctypes.byref(p), ctypes.byref(h))
        if st != DDC_OK:
            raise DDCosmoError(st, self.L.ddc_status_string(st).decode())
        self.h = h
        self.nsph = self.ncav = self.nylm = 0
        self.ngrid = ngrid
        self.lmax, self.eps, self.igrad = lmax, eps, igrad

    def _check(self, st, allow_noconv=False):
        if st == DDC_OK or (allow_noconv and st == DDC_ERR_NOCONV):
            return st
        raise DDCosmoError(st, self.L.ddc_last_error(self.h).decode())

    def close(self):
        """memfree (ddcosmo.f90:491-523)."""
        if getattr(self, "h", None):
            self.L.ddc_destroy(self.h)
            self.h = None

    memfree = close

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def launches(self):
        return self.L.ddc_launch_count(self.h)

    def stage_times(self):
        """{stage: (ms, calls)} of the CUDA-event stage timers (timing=1)."""
        n = self.L.ddc_stage_count()
        ms = (ctypes.c_double * n)()
        calls = (ctypes.c_longlong * n)()
        self._check(self.L.ddc_stage_times(self.h, ms, calls))
        return {self.L.ddc_stage_name(k).decode(): (ms[k], calls[k]) for k in range(n)}

    def reset_stage_times(self):
        self._check(self.L.ddc_reset_stage_times(self.h))

    def set_timed_stages(self, names=None):
        """Time only the named stages (None: every stage)."""
        self._check(self.L.ddc_set_timed_stages(self.h, stage_mask(self.L, names)))

    def set_guess_model(self, model):
        """Model used by guess=GUESS_LEARNED (a GuessModel, or None)."""
        self._guess_model = model
        self._check(self.L.ddc_set_guess_model(self.h, model.h if model else None))

    def guess_rows(self, feat_ptr, target_ptr=None):
        """Training rows of the last energy+force call into device buffers
        (raw pointers): features [nsph][nfeat] and, if given, targets
        [nsph][nout] (needs a model attached for the row widths)."""
        self._check(self.L.ddc_guess_features(self.h, feat_ptr))
        if target_ptr is not None:
            self._check(self.L.ddc_guess_targets(self.h, target_ptr))

    # ddinit (ddcosmo.f90:159): coordinates and radii in bohr
    def ddinit(self, x, y, z, rvdw):
        x, y, z, r = map(_f64, (x, y, z, rvdw))
        self._check(self.L.ddc_init(self.h, len(x), _p(x), _p(y), _p(z), _p(r)))
        a = [ctypes.c_int() for _ in range(4)]
        self._check(self.L.ddc_sizes(self.h, *[ctypes.byref(v) for v in a]))
        self.nsph, self.ncav, self.nylm, self.ngrid = (v.value for v in a)
        return self

    @property
    def ccav(self):
        out = np.zeros((self.ncav, 3))
        self._check(self.L.ddc_get_ccav(self.h, _p(out)))
        return out

    @property
    def ui(self):
        out = np.zeros((self.nsph, self.ngrid))
        self._check(self.L.ddc_get_ui(self.h, _p(out)))
        return out

    @property
    def csph(self):
        out = np.zeros((self.nsph, 3))
        self._check(self.L.ddc_get_csph(self.h, _p(out)))
        return out

    def grid(self):
        g = np.zeros((self.ngrid, 3))
        w = np.zeros(self.ngrid)
        self._check(self.L.ddc_get_grid(self.h, _p(g), _p(w)))
        return g, w

    # mkrhs (mkrhs.f90:1): phi(ncav), psi(nylm, n); ccav=None uses the module's cavity
    def mkrhs(self, charge, x, y, z, ccav=None):
        q, x, y, z = map(_f64, (charge, x, y, z))
        n = len(q)
        ncav = self.ncav if ccav is None else len(ccav)
        cc = None if ccav is None else _f64(ccav)
        phi = np.zeros(max(ncav, 1))
        psi = np.zeros((n, self.nylm))
        self._check(self.L.ddc_mkrhs(self.h, n, _p(q), _p(x), _p(y), _p(z), ncav, _p(cc),
                                     _p(phi), self.nylm, _p(psi)))
        return phi[:ncav], psi

    # cosmo(star, cart, phi, glm, psi, sigma, esolv) (cosmo.f90:1)
    def cosmo(self, star, cart, phi=None, glm=None, psi=None, sigma=None, return_info=False):
        nv = (self.nsph, self.nylm)
        phi = None if phi is None else _f64(phi)
        glm = None if glm is None else _f64(glm)
        psi = None if psi is None else _f64(psi)
        sig = np.zeros(nv) if sigma is None else _f64(sigma).copy()
        es = ctypes.c_double(0.0)
        info = SolveInfo()
        st = self.L.ddc_cosmo(self.h, int(bool(star)), int(bool(cart)), _p(phi), _p(glm), _p(psi),
                              _p(sig), ctypes.byref(es), ctypes.byref(info))
        self._check(st)
        if return_info:
            return sig, es.value, info.as_dict()
        return sig, es.value

    # forces_dd(n, phi, sigma, s, fx) (forces_dd.f90:1)
    def forces_dd(self, phi, sigma, s):
        fx = np.zeros((self.nsph, 3))
        self._check(self.L.ddc_forces_dd(self.h, _p(_f64(phi)), _p(_f64(sigma)), _p(_f64(s)),
                                         _p(fx)))
        return fx

    def ddmkzeta(self, s):      # ddcosmo.f90:1787
        out = np.zeros(max(self.ncav, 1))
        self._check(self.L.ddc_mkzeta(self.h, _p(_f64(s)), _p(out)))
        return out[: self.ncav]

    def ddmkxi(self, s):        # ddcosmo.f90:1758
        out = np.zeros(max(self.ncav, 1))
        self._check(self.L.ddc_mkxi(self.h, _p(_f64(s)), _p(out)))
        return out[: self.ncav]

    # efld(nsrc, src, csrc, ntrg, ctrg, ef) (efld.f90:1); csrc/ctrg (n, 3)
    def efld(self, src, csrc, ctrg):
        src = _f64(src)
        cs = None if csrc is None else _f64(csrc)
        ct = None if ctrg is None else _f64(ctrg)
        nsrc = len(src)
        ntrg = len(ct) if ct is not None else (self.ncav if nsrc == self.nsph else self.nsph)
        ef = np.zeros((max(ntrg, 1), 3))
        self._check(self.L.ddc_efld(self.h, nsrc, _p(src), _p(cs), ntrg, _p(ct), _p(ef)))
        return ef[:ntrg]

    def _op(self, fn, x):
        x = _f64(x)
        y = np.zeros_like(x)
        self._check(fn(self.h, _p(x), _p(y)))
        return y

    def lx(self, x):            # matvec.f90:94
        return self._op(self.L.ddc_lx, x)

    def lstarx(self, x):        # matvec.f90:161
        return self._op(self.L.ddc_lstarx, x)

    def lx_lstarx(self, x, s):
        """(lx(x), lstarx(s)) from one fused pass over the triples."""
        x, s = _f64(x), _f64(s)
        y = np.zeros((self.nsph, self.nylm))
        z = np.zeros((self.nsph, self.nylm))
        self._check(self.L.ddc_lx_lstarx(self.h, _p(x), _p(y), _p(s), _p(z)))
        return y, z

    def ldm1x(self, x):         # matvec.f90:246
        return self._op(self.L.ddc_ldm1x, x)

    def hnorm(self, x):         # matvec.f90:281
        v = ctypes.c_double()
        self._check(self.L.ddc_hnorm(self.h, _p(_f64(x)), ctypes.byref(v)))
        return v.value

    def rhs(self, phi):         # cosmo.f90:104-117
        g = np.zeros((self.nsph, self.nylm))
        self._check(self.L.ddc_rhs(self.h, _p(_f64(phi)), _p(g)))
        return g

    def energy_forces_ptr(self, q, x, y, z, r, n, sigma, s, fx):
        """ddc_energy_forces on raw pointers (ints): device pointers when the
        context was created with device_pointers=1, else host pointers (e.g.
        pinned buffers).  0 for an output means "not requested".  Returns the
        run info dict with ``esolv`` added."""
        es = ctypes.c_double()
        info = RunInfo()
        self._check(self.L.ddc_energy_forces(self.h, n, _p(q), _p(x), _p(y), _p(z), _p(r),
                                             ctypes.byref(es), _p(sigma or None), _p(s or None),
                                             _p(fx or None), ctypes.byref(info)))
        d = info.as_dict()
        d["esolv"] = es.value
        self.nsph, self.ncav, self.nylm, self.ngrid = d["nsph"], d["ncav"], d["nylm"], d["ngrid"]
        return d

    def batch_energy_forces(self, mols):
        """Energy and forces of several independent molecules in one library
        call (each molecule as if solved alone).  mols: list of dicts with
        q, x, y, z, r (bohr).  Returns dict(esolv[nmol], fx list, iters
        (nmol, 2), info)."""
        sizes = [len(m["q"]) for m in mols]
        off = np.zeros(len(mols) + 1, dtype=np.int32)
        off[1:] = np.cumsum(sizes)
        cat = {k: _f64(np.concatenate([np.asarray(m[k], dtype=np.float64) for m in mols]))
               for k in "qxyzr"}
        nmol = len(mols)
        es = np.zeros(nmol)
        fx = np.zeros((int(off[-1]), 3))
        iters = np.zeros((nmol, 2), dtype=np.int32)
        info = RunInfo()
        ip = ctypes.POINTER(ctypes.c_int)
        self._check(self.L.ddc_batch_energy_forces(
            self.h, nmol, off.ctypes.data_as(ip), _p(cat["q"]), _p(cat["x"]), _p(cat["y"]),
            _p(cat["z"]), _p(cat["r"]), _p(es), _p(fx), iters.ctypes.data_as(ip),
            ctypes.byref(info)))
        return dict(esolv=es, fx=[fx[off[k]:off[k + 1]] for k in range(nmol)], iters=iters,
                    info=info.as_dict(), off=off)

    def energy_forces(self, charge, x, y, z, rvdw, sigma0=None, s0=None):
        """The main.f90 flow (main.f90:164-265) in one library call.  With
        guess=GUESS_USER, sigma0 and s0 (n, nylm) are the initial guesses of
        the direct and adjoint solves.  Returns dict(esolv, sigma, s, fx, info)."""
        q, x, y, z, r = map(_f64, (charge, x, y, z, rvdw))
        n = len(q)
        nylm = (self.lmax + 1) ** 2
        es = ctypes.c_double()
        sig = np.zeros((n, nylm)) if sigma0 is None else np.array(sigma0, dtype=np.float64, order="C")
        s = np.zeros((n, nylm)) if s0 is None else np.array(s0, dtype=np.float64, order="C")
        fx = np.zeros((n, 3))
        info = RunInfo()
        self._check(self.L.ddc_energy_forces(self.h, n, _p(q), _p(x), _p(y), _p(z), _p(r),
                                             ctypes.byref(es), _p(sig), _p(s), _p(fx),
                                             ctypes.byref(info)))
        a = [ctypes.c_int() for _ in range(4)]
        self._check(self.L.ddc_sizes(self.h, *[ctypes.byref(v) for v in a]))
        self.nsph, self.ncav, self.nylm, self.ngrid = (v.value for v in a)
        return dict(esolv=es.value, sigma=sig, s=s, fx=fx, info=info.as_dict())


class GuessModel:
    """Learned initial guess (ddc_guess_*): a per-sphere network from the
    sphere's right-hand side, charge, radius and neighbour-distance histogram
    to the corrections of X0 and S0 over facl * rhs.  BF16 weights, FP32
    accumulation, trained on device arrays of solver output."""

    def __init__(self, lmax, hidden=256, device=0, params=None):
        self.L = load_library()
        h = ctypes.c_void_p()
        st = self.L.ddc_guess_create(lmax, hidden, device, ctypes.byref(h))
        if st != DDC_OK:
            raise DDCosmoError(st, "ddc_guess_create failed")
        self.h = h
        self.lmax, self.hidden, self.device = lmax, hidden, device
        nf, no, npar = ctypes.c_int(), ctypes.c_int(), ctypes.c_longlong()
        self._check(self.L.ddc_guess_sizes(self.h, ctypes.byref(nf), ctypes.byref(no),
                                           ctypes.byref(npar)))
        self.nfeat, self.nout, self.nparams = nf.value, no.value, npar.value
        if params is not None:
            self.set_params(params)

    def _check(self, st):
        if st != DDC_OK:
            raise DDCosmoError(st, self.L.ddc_guess_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.L.ddc_guess_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def get_params(self):
        out = np.zeros(self.nparams, dtype=np.float32)
        self._check(self.L.ddc_guess_get_params(self.h, out.ctypes.data_as(_fp)))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.nparams:
            raise ValueError(f"expected {self.nparams} parameters, got {p.size}")
        self._check(self.L.ddc_guess_set_params(self.h, p.ctypes.data_as(_fp)))

    def init_random(self, seed=0):
        self._check(self.L.ddc_guess_init_random(self.h, seed))

    def fit_scaling(self, feat_ptr, target_ptr, n):
        self._check(self.L.ddc_guess_fit_scaling(self.h, feat_ptr, target_ptr, n))

    def train_epoch(self, feat_ptr, target_ptr, order_ptr, n, batch=4096, lr=1e-3):
        loss = ctypes.c_double()
        self._check(self.L.ddc_guess_train_epoch(self.h, feat_ptr, target_ptr, order_ptr, n,
                                                 batch, lr, ctypes.byref(loss)))
        return loss.value

    def predict(self, feat_ptr, out_ptr, n):
        self._check(self.L.ddc_guess_predict(self.h, feat_ptr, out_ptr, n))

    def save(self, path, **meta):
        np.savez_compressed(path, params=self.get_params(), lmax=self.lmax, hidden=self.hidden,
                            nfeat=self.nfeat, nout=self.nout, **meta)

    @classmethod
    def load(cls, path, device=0):
        d = np.load(path)
        return cls(int(d["lmax"]), int(d["hidden"]), device, params=d["params"])
