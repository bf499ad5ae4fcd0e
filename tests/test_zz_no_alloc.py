"""The allocation-free expected-count entry point (gf_skygen_integrate_static).

It serves hosts that own all GPU memory themselves (a framework with its own
arena, or a process that must not call cudaMalloc/cudaFree while it runs): they
pass their own device buffers, and the library's scratch is a fixed __device__
array.  The test calls it through the C ABI, twice in a row, and compares each
result with the regular entry point (gf_skygen_integrate), which allocates its
scratch, at the tolerance of the integrate parity tests (1e-12 relative).
The file is named to run last: a failure here leaves every other test run.
"""
import ctypes as C
import math

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_integrate_static_matches_regular_entry_point():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import galfast_b200 as G
    from galfast_b200 import workloads as W, _abi as A

    L = G.lib()
    L.gf_skygen_integrate_static.argtypes = [C.POINTER(G.SkygenConfig), C.c_void_p, C.c_int32, C.c_void_p,
                                              C.POINTER(G.Extinction), C.POINTER(G.ModelConfig), C.c_void_p, C.c_void_p]
    half = 2.5 * math.pi / 180
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LAMBERT_RECT
    foot.proj = 0
    foot.a, foot.b, foot.c, foot.d = -half, half, -half, half
    w = W.build_workload(L, foot=foot, dx_deg=0.25, m0=15.0, m1=21.0, with_modules=False)

    # the regular entry point: its own context, allocations and stream
    ctx = G.Context(0)
    sky = G.Skygen(ctx, w)
    expected = [sky.integrate_counts(m)[:2] for m in range(len(w.models))]
    sky.close()
    ctx.close()

    # the caller's own device buffers
    torch.cuda.set_device(0)
    d_pix = torch.frombuffer(bytearray(w.pixels), dtype=torch.uint8).cuda()
    d_ammin = torch.from_numpy(w.ammin.copy()).cuda()
    d_res = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for m, model in enumerate(w.models):
            d_res.fill_(-1.0)
            torch.cuda.synchronize()
            st = L.gf_skygen_integrate_static(C.byref(w.sky), C.c_void_p(d_pix.data_ptr()), w.npixels,
                                              C.c_void_p(d_ammin.data_ptr()), C.byref(w.ext), C.byref(model),
                                              C.c_void_p(d_res.data_ptr()), C.c_void_p(stream))
            assert st == 0, L.gf_last_error().decode()
            got = d_res.cpu().numpy()
            assert got[0] == pytest.approx(expected[m][0], rel=1e-12), (call, m)
            assert got[1] == pytest.approx(expected[m][1], rel=1e-12), (call, m)


def test_integrate_static_pixel_blocks_match_regular_entry_point():
    """nm * nM not a multiple of 10 (121 x 238 bins): the crawl runs in pixel blocks of
    2^21 / nthreads pixels that add into the same partial sums (skyconfig_impl.h:
    344-387).  With 7680 streams a block holds 273 pixels; the footprint has more
    than 1000, so several blocks run, each from its own offset into the caller's
    pixel buffer."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import galfast_b200 as G
    from galfast_b200 import workloads as W, _abi as A

    L = G.lib()
    L.gf_skygen_integrate_static.argtypes = [C.POINTER(G.SkygenConfig), C.c_void_p, C.c_int32, C.c_void_p,
                                              C.POINTER(G.Extinction), C.POINTER(G.ModelConfig), C.c_void_p, C.c_void_p]
    half = 4.5 * math.pi / 180
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LAMBERT_RECT
    foot.proj = 0
    foot.a, foot.b, foot.c, foot.d = -half, half, -half, half
    w = W.build_workload(L, foot=foot, dx_deg=0.25, m0=15.0, m1=21.05, M1=14.9, with_modules=False)
    info = (G.ModelInfo * len(w.models))()
    marr = (G.ModelConfig * len(w.models))(*w.models)
    assert L.gf_skygen_setup_host(C.byref(w.sky), w.npixels, marr, len(w.models), info, None) == 0
    assert (info[0].nm * info[0].nM) % 10 != 0
    assert w.npixels > 3 * (2 * 1024 * 1024 // w.sky.nthreads)

    ctx = G.Context(0)
    sky = G.Skygen(ctx, w)
    expected = [sky.integrate_counts(m)[:2] for m in range(len(w.models))]
    sky.close()
    ctx.close()

    torch.cuda.set_device(0)
    d_pix = torch.frombuffer(bytearray(w.pixels), dtype=torch.uint8).cuda()
    d_ammin = torch.from_numpy(w.ammin.copy()).cuda()
    d_res = torch.zeros(2, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for m, model in enumerate(w.models):
            d_res.fill_(-1.0)
            torch.cuda.synchronize()
            st = L.gf_skygen_integrate_static(C.byref(w.sky), C.c_void_p(d_pix.data_ptr()), w.npixels,
                                              C.c_void_p(d_ammin.data_ptr()), C.byref(w.ext), C.byref(model),
                                              C.c_void_p(d_res.data_ptr()), C.c_void_p(stream))
            assert st == 0, L.gf_last_error().decode()
            got = d_res.cpu().numpy()
            assert got[0] == pytest.approx(expected[m][0], rel=1e-12), (call, m)
            assert got[1] == pytest.approx(expected[m][1], rel=1e-12), (call, m)


def test_integrate_static_rejects_oversized_requests():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import galfast_b200 as G
    from galfast_b200 import workloads as W, _abi as A

    L = G.lib()
    L.gf_skygen_integrate_static.argtypes = [C.POINTER(G.SkygenConfig), C.c_void_p, C.c_int32, C.c_void_p,
                                              C.POINTER(G.Extinction), C.POINTER(G.ModelConfig), C.c_void_p, C.c_void_p]
    half = 0.5 * math.pi / 180
    foot = A.Footprint()
    foot.kind = A.GF_FOOT_LAMBERT_RECT
    foot.proj = 0
    foot.a, foot.b, foot.c, foot.d = -half, half, -half, half
    # 400 x 240 bins per pixel is above the 65536-bin limit of the fixed scratch
    w = W.build_workload(L, foot=foot, dx_deg=0.25, m0=5.0, m1=25.0, with_modules=False)
    d_pix = torch.frombuffer(bytearray(w.pixels), dtype=torch.uint8).cuda()
    d_res = torch.zeros(2, dtype=torch.float64, device="cuda")
    st = L.gf_skygen_integrate_static(C.byref(w.sky), C.c_void_p(d_pix.data_ptr()), w.npixels, None, C.byref(w.ext),
                                      C.byref(w.models[0]), C.c_void_p(d_res.data_ptr()), None)
    assert st == -1
    assert "65536 bins" in L.gf_last_error().decode()
