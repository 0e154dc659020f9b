"""Device-pointer mode (device_pointers=1) on a caller's CUDA stream: the
call the benchmark times.  Inputs and outputs are device arrays (torch
tensors here); the results must equal those of host-array mode bit for bit
(same kernels, same summation orders), and the call must leave its results
ordered on the caller's stream."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [0, 1])
def test_device_pointers_on_caller_stream_match_host_mode(prec):
    import torch
    from ddpcm_b200 import molecules as M
    from ddpcm_b200.ddcosmo import DDCosmo
    c = M.CONFIGS[1]
    m = M.to_bohr(M.config_molecule(1))
    kw = dict(lmax=c["lmax"], ngrid=c["ngrid"], iconv=c["iconv"], eps=c["eps"], eta=c["eta"],
              precision=prec)
    with DDCosmo(**kw) as dd:
        host = dd.energy_forces(m["q"], m["x"], m["y"], m["z"], m["r"])
    dev = torch.device("cuda", 0)
    stream = torch.cuda.Stream(dev)
    n = len(m["q"])
    nylm = (c["lmax"] + 1) ** 2
    with torch.cuda.stream(stream):
        d_in = {k: torch.tensor(m[k], dtype=torch.float64, device=dev) for k in "qxyzr"}
        sig = torch.full((n, nylm), float("nan"), dtype=torch.float64, device=dev)
        s = torch.full_like(sig, float("nan"))
        fx = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
    with DDCosmo(device_pointers=1, stream=stream.cuda_stream, **kw) as dd:
        info = dd.energy_forces_ptr(*(d_in[k].data_ptr() for k in "qxyzr"), n, sig.data_ptr(),
                                    s.data_ptr(), fx.data_ptr())
        # results are ordered on the caller's stream: read them after it
        stream.synchronize()
        assert info["esolv"] == host["esolv"]
        np.testing.assert_array_equal(fx.cpu().numpy(), host["fx"])
        np.testing.assert_array_equal(sig.cpu().numpy(), host["sigma"])
        np.testing.assert_array_equal(s.cpu().numpy(), host["s"])
        assert info["direct"]["iterations"] == host["info"]["direct"]["iterations"]
