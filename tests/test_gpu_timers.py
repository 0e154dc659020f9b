"""Stage timers: with timing=1 every stage records CUDA events around its
launches; ddc_set_timed_stages restricts them to a subset, and the results
do not depend on which stages are timed."""
import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu


def test_timed_stage_subset():
    from ddpcm_b200.ddcosmo import DDCosmo
    g = load_golden("caffeine")
    p, m = dict(g["params"]), g["mol"]
    args = (m["q"], m["x"], m["y"], m["z"], m["r"])
    with DDCosmo(lmax=p["lmax"], ngrid=p["ngrid"], iconv=p["iconv"], eps=p["eps"],
                 eta=p["eta"], timing=1) as dd:
        full = dd.energy_forces(*args)
        every = dd.stage_times()
        timed = {k for k, (ms, calls) in every.items() if calls > 0}
        assert {"lx_lstarx", "jacobi_step", "diis_combine", "efield", "forces"} <= timed
        assert all(every[k][0] > 0.0 for k in timed)

        dd.reset_stage_times()
        dd.set_timed_stages(["lx_lstarx"])
        one = dd.energy_forces(*args)
        only = dd.stage_times()
        assert only["lx_lstarx"][1] == every["lx_lstarx"][1]
        assert all(calls == 0 for k, (ms, calls) in only.items() if k != "lx_lstarx")

        dd.reset_stage_times()
        dd.set_timed_stages(None)
        dd.energy_forces(*args)
        again = dd.stage_times()
        assert {k for k, (ms, calls) in again.items() if calls > 0} == timed
    assert one["esolv"] == full["esolv"]
    np.testing.assert_array_equal(one["fx"], full["fx"])
