"""The precision form on B200 (gf_skygen_precision): the FP64 per-pixel expected
counts equal the FP64 oracle's (same bins, same anchors) to 1e-12; the FP32
Kahan-summed per-pixel counts equal the reference float counts (oracle) and the
crawl's own integrate; and the FP32 totals are within 1e-6 of FP64 (the
precision target), with per-bin errors up to ~1e-4 on far, faint bins."""
import numpy as np
import pytest

import galfast_b200 as G
from galfast_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_precision_report_against_fp64_oracle(lib):
    w = W.config1(lib, with_modules=False)
    ctx = G.Context(0)
    sk = G.Skygen(ctx, w)
    osk = O.OracleSkygen(w, "p")
    for m in range(3):
        rep, p32, p64, hist = sk.precision(m)
        _, _, pp = sk.integrate_counts(m, per_pixel=True)    # covered fraction is 1 in this footprint
        np.testing.assert_allclose(p32, pp, rtol=2e-7)
        for px in (0, 777, w.npixels - 1):
            a32, a64 = osk.expected_fp64(m, px)
            assert p64[px] == pytest.approx(a64, rel=1e-12), (m, px)
            assert p32[px] == pytest.approx(a32, rel=2e-7), (m, px)
        assert rep.expected64 == pytest.approx(p64.sum(), rel=1e-12)
        assert hist.sum() == pytest.approx(rep.expected64, rel=1e-12)
        assert rep.total_rel_err <= 1e-6, (m, rep.total_rel_err)
        # single bins far out in the disk: the float DM's rounding (~1e-6 mag) times an
        # exponent of tens of scale lengths gives ~1e-4; the mean and the totals stay small
        assert 0 < rep.bin_max_rel_err < 1e-3
        assert rep.bin_mean_rel_err < 1e-5
        assert rep.bins > 0
    sk.close()
    ctx.close()


def test_precision_of_bulge_and_broken_power_law(lib):
    """The FP64 evaluation of the LC bulge and the broken power law (per pixel,
    against the oracle's double-precision restatement) and the FP32 totals
    within 1e-6 of it."""
    from galfast_b200 import _abi as A
    w = W.build_workload(lib, foot=W.cap_footprint(5.0, 8.0, 1.5), dx_deg=0.25, m0=15.0, m1=19.0, with_modules=False)
    b = w.models[1]
    b.type = A.GF_MODEL_LCBULGE
    b.f, b.l, b.n, b.ba, b.ca = 10.0, 700.0, 2.0, 0.6, 0.4
    h = w.models[2]
    h.type = A.GF_MODEL_BROKEN_POWER_LAW
    h.nbreaks = 1
    h.n_brk[0], h.n_brk[1] = -2.5, -3.5
    h.rbreak[0] = 25000.0
    ctx = G.Context(0)
    sk = G.Skygen(ctx, w)
    osk = O.OracleSkygen(w, "p")
    for m in (1, 2):
        rep, p32, p64, hist = sk.precision(m)
        for px in (0, w.npixels // 2, w.npixels - 1):
            a32, a64 = osk.expected_fp64(m, px)
            assert p64[px] == pytest.approx(a64, rel=1e-12), (m, px)
            assert p32[px] == pytest.approx(a32, rel=2e-7), (m, px)
        assert rep.total_rel_err <= 1e-6, (m, rep.total_rel_err)
    sk.close()
    ctx.close()
