"""The mixed-precision operators, whose projection onto the harmonics and
expansion to the grid run on the tensor cores (split TF32, tcgen05), against
the FP64 oracle's lx and lstarx (matvec.f90:94, :161).

A DDC_PREC_MIXED context's ddc_lx / ddc_lstarx / ddc_lx_lstarx apply the
operators of the inner solves: FP32 triple sums plus the two contractions.
They must agree with the FP64 operators to FP32 accuracy (bar: 1e-5 of the
largest entry), which is what the iterative refinement around them needs,
and the tensor-core contractions must be close to FP32 SIMT ones: the same
operators with the SIMT contractions (DDC_TC_OFF=1) set the reference error.
The three-term TF32 split carries about 2^-21 per product against 2^-24 for
an FP32 product, and the tensor cores accumulate in FP32 with their own
rounding, so the tensor-core error may be up to three times the SIMT one
(measured: 1.4e-6 against 1.0e-6 at lmax 0); a layout or descriptor mistake
would show as an error of order one.
The cases cover every harmonic count the tensor-core kernels take (lmax 0, 6,
8, 10: one to four 32-wide k-chunks of the expansion, one to five 128-row
grid tiles), tile widths from 16 to 64 spheres and the FP32 SIMT fallback
above 128 harmonics (lmax 11, 12).
"""
import os

import numpy as np
import pytest

from conftest import load_golden

pytestmark = pytest.mark.gpu

BAR = 1e-5


def _globule(n, seed):
    from ddpcm_b200.molecules import make_molecule, to_bohr
    return to_bohr(make_molecule(n, seed))


@pytest.mark.parametrize("lmax,ngrid,mol", [
    (0, 110, "caffeine"), (6, 302, "crambin"), (8, 302, "taxol"), (10, 590, "crambin"),
    (11, 590, "caffeine"), (12, 590, "caffeine")])
def test_mixed_operators_vs_oracle(oracle, lmax, ngrid, mol):
    from ddpcm_b200.ddcosmo import PREC_MIXED, DDCosmo
    m = load_golden(mol)["mol"]
    d = oracle.RefDD(lmax, ngrid, 10, 1, 78.3553, 0.1).init(m["x"], m["y"], m["z"], m["r"])
    rng = np.random.default_rng(100 + lmax)
    x = rng.standard_normal((d.nsph, d.nylm))
    s = rng.standard_normal((d.nsph, d.nylm))
    ref_y, ref_z = d.lx(x), d.lstarx(s)
    errs = {}
    for mode in ("tc", "simt"):
        os.environ["DDC_TC_OFF"] = "1" if mode == "simt" else "0"
        try:
            with DDCosmo(lmax=lmax, ngrid=ngrid, iconv=10, eta=0.1, precision=PREC_MIXED) as dd:
                dd.ddinit(m["x"], m["y"], m["z"], m["r"])
                y1, z1 = dd.lx(x), dd.lstarx(s)
                y2, z2 = dd.lx_lstarx(x, s)
        finally:
            os.environ.pop("DDC_TC_OFF", None)
        errs[mode] = [np.abs(a - b).max() / np.abs(b).max()
                      for a, b in ((y1, ref_y), (y2, ref_y), (z1, ref_z), (z2, ref_z))]
    for et, es in zip(errs["tc"], errs["simt"]):
        assert et <= BAR, errs
        assert et <= 3.0 * es + 1e-7, errs


@pytest.mark.parametrize("n", [2400, 9472])
def test_mixed_operators_wide_tiles(oracle, n):
    """Larger molecules: 2400 spheres (tiles of 32) and 9472 (64 per tile,
    one tile per SM) at lmax 6 / 302 points."""
    from ddpcm_b200.ddcosmo import PREC_MIXED, DDCosmo
    m = _globule(n, 7)
    d = oracle.RefDD(6, 302, 10, 1, 78.3553, 0.1).init(m["x"], m["y"], m["z"], m["r"])
    rng = np.random.default_rng(n)
    x = rng.standard_normal((d.nsph, d.nylm))
    s = rng.standard_normal((d.nsph, d.nylm))
    ref_y, ref_z = d.lx(x), d.lstarx(s)
    with DDCosmo(lmax=6, ngrid=302, iconv=10, eta=0.1, precision=PREC_MIXED) as dd:
        dd.ddinit(m["x"], m["y"], m["z"], m["r"])
        y, z = dd.lx_lstarx(x, s)
        y2 = dd.lx(x)
    for a, b in ((y, ref_y), (y2, ref_y), (z, ref_z)):
        err = np.abs(a - b).max() / np.abs(b).max()
        assert err <= BAR, err
