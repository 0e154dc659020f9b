"""ddc_efld_noalloc: the electric field without any device allocation.

It serves host programs that own all of the GPU's memory (for example a
QM/MM or MD code that reserves the HBM for its own pool at start-up), for
which a cudaMalloc issued by the library in the middle of a step would fail
or stall the device.  The test plays such a caller: it owns every device
buffer (allocated here through torch) and checks, through the C ABI, that two
calls in a row give the same field as the allocating entry point ddc_efld.
The sizes make the kernel split the sources into many chunks, so the fixed
scratch array inside the library is exercised, up to the case where it holds
fewer chunks than the kernel would use and the one near the target limit
where a single chunk writes the output directly; some calls go on a stream of
the caller's own.  This file is collected last
on purpose.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DDC_ERR_CAPACITY = 8
_dp = ctypes.POINTER(ctypes.c_double)


def _fn():
    from ddpcm_b200.ddcosmo import load_library
    L = load_library()
    f = L.ddc_efld_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int, _dp, _dp, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _ptr(t):
    return ctypes.cast(ctypes.c_void_p(t.data_ptr()), _dp)


def test_efld_noalloc_matches_efld_on_consecutive_calls():
    import torch
    from ddpcm_b200.ddcosmo import DDCosmo

    f = _fn()
    dev = torch.device("cuda", 0)
    # the one-time set-up call a caller makes at start-up: no targets, no work
    assert f(0, 0, None, None, 0, None, None, None) == 0
    rng = np.random.default_rng(17)
    side = torch.cuda.Stream(device=dev)
    # many source chunks; the same twice in a row; more chunks than the
    # scratch holds (the chunk count is clamped); one chunk near the target
    # limit (the field is written straight into ef)
    cases = ((200000, 2000, None), (150000, 3000, None), (20000, 100000, side),
             (3000, 349000, side))
    with DDCosmo() as dd:
        for nsrc, ntrg, stream in cases:
            src = rng.uniform(-0.5, 0.5, nsrc)
            csrc = rng.uniform(-40.0, 40.0, (nsrc, 3))
            ctrg = rng.uniform(-40.0, 40.0, (ntrg, 3))
            ref = dd.efld(src, csrc, ctrg)  # allocating entry point, host arrays
            d_src = torch.tensor(src, device=dev)
            d_csrc = torch.tensor(csrc, device=dev)
            d_ctrg = torch.tensor(ctrg, device=dev)
            d_ef = torch.full((ntrg, 3), float("nan"), dtype=torch.float64, device=dev)
            torch.cuda.synchronize(dev)
            handle = None if stream is None else stream.cuda_stream
            for _ in range(2):
                d_ef.fill_(float("nan"))
                torch.cuda.synchronize(dev)
                st = f(0, nsrc, _ptr(d_src), _ptr(d_csrc), ntrg, _ptr(d_ctrg), _ptr(d_ef),
                       handle)
                assert st == 0
                torch.cuda.synchronize(dev)
                # the chunk count (and with it the summation order) may differ
                # from ddc_efld's: agreement to 1e-13 of the field's scale
                got = d_ef.cpu().numpy()
                assert np.isfinite(got).all()
                assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_efld_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    f = _fn()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(16, dtype=torch.float64, device=dev)
    st = f(0, 1, _ptr(buf), _ptr(buf), 400000, _ptr(buf), _ptr(buf), None)
    assert st == DDC_ERR_CAPACITY
