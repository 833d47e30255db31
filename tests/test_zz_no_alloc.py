"""bbrt_trace_noalloc: the trace entry point that allocates no device memory.

It exists for callers that must not allocate while tracing — a framework
whose device memory all belongs to its own arena or fixed budget, or a
latency-critical loop that cannot pay for the device synchronisation of
cudaMalloc / cudaFree.  The caller owns every input and output buffer; the
kernel's scratch (ray counter, statistics, per-object hit counters) sits in a
static device array of the library.

Checked here, through the C ABI: two calls in a row give exactly the outputs
of the allocating entry points (bbrt_trace on device pointers for the per-ray
results, bbrt_plane_source for the hit counts), so the second call is not
polluted by the first one's scratch; free device memory does not change
across the two calls, which run right after the scene's upload and before
any allocating trace; and the documented limits are enforced.  This file is
collected last so that a stopping run has already run every other test.
"""
import ctypes

import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes

pytestmark = pytest.mark.gpu

OUTS = (("status", np.int32, ()), ("bounce_count", np.int32, ()), ("exit_dir", np.float64, (3,)),
        ("end_point", np.float64, (3,)), ("hit_object", np.int32, ("K",)), ("hit_point", np.float64, ("K", 3)),
        ("err_object", np.int32, ()), ("err_value", np.float64, (2,)))


def _device_outputs(torch, n, K):
    tdt = {np.int32: torch.int32, np.float64: torch.float64}
    bufs = {}
    for name, dt, shape in OUTS:
        shp = (n,) + tuple(K if s == "K" else s for s in shape)
        bufs[name] = torch.full(shp, -7, dtype=tdt[dt], device="cuda")
    out = C.TraceOut()
    out.record_bounces = K
    for name, dt, _ in OUTS:
        ct = ctypes.c_int if dt == np.int32 else ctypes.c_double
        setattr(out, name, ctypes.cast(ctypes.c_void_p(bufs[name].data_ptr()), ctypes.POINTER(ct)))
    return bufs, out


def test_noalloc_trace_matches_allocating_entry_points(built):
    import torch
    lib = C.load_library()
    patches = scenes.scene_two_spheres()
    cfg = C.default_config(coarse_grid_n=9, newton_tol=1e-12)
    sc = api.Scene(patches, config=cfg)
    c0, c1, dd = (-3.0, -3.0, 4.0), (3.0, 3.0, 4.0), (0.3, 0.0, -1.0)
    src = scenes.plane_grid(c0, c1, 64, 48)
    dirs = np.tile(np.array(dd), (src.shape[0], 1))
    n, K = src.shape[0], 4
    to = torch.from_numpy(src).cuda()
    td = torch.from_numpy(dirs).cuda()
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)

    lib.bbrt_trace_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                       ctypes.c_int, ctypes.POINTER(C.TraceOut), ctypes.c_void_p, ctypes.c_int,
                                       ctypes.POINTER(C.TraceStats), ctypes.c_void_p]
    counts = torch.full((sc.n_objects,), -1, dtype=torch.int64, device="cuda")
    bufs, out = _device_outputs(torch, n, K)
    # the scene goes to the device first (the one step that allocates); from
    # here on, in a fresh process too, the allocation-free calls must leave
    # free device memory unchanged, the first one included
    sc.upload()
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    got_calls = []
    for call in range(2):
        for b in bufs.values():
            b.fill_(-7)
        counts.fill_(-1)
        torch.cuda.synchronize()
        st = C.TraceStats()
        C.check(lib, lib.bbrt_trace_noalloc(sc.h, ctypes.c_void_p(to.data_ptr()), ctypes.c_void_p(td.data_ptr()), n,
                                            20, ctypes.byref(out), ctypes.c_void_p(counts.data_ptr()), 1,
                                            ctypes.byref(st), ctypes.c_void_p(stream.cuda_stream)),
                "bbrt_trace_noalloc")
        torch.cuda.synchronize()
        got_calls.append(({k: v.cpu().numpy() for k, v in bufs.items()}, counts.cpu().numpy(),
                          (st.rays, st.bounces, sum(st.status_hist))))
    assert torch.cuda.mem_get_info()[0] == free_before

    # the allocating entry points on the same rays
    ref_bufs, ref_out = _device_outputs(torch, n, K)
    C.check(lib, lib.bbrt_trace(sc.h, ctypes.c_void_p(to.data_ptr()), ctypes.c_void_p(td.data_ptr()), n, 20,
                                C.DEVICE_PTRS, ctypes.byref(ref_out), None, ctypes.c_void_p(stream.cuda_stream)),
            "bbrt_trace")
    ref_counts = sc.plane_source(c0, c1, dd, 64, 48, 20, count_direct_hit=False)
    torch.cuda.synchronize()
    ref = {k: v.cpu().numpy() for k, v in ref_bufs.items()}
    for call, (got, cnt, (rays, bounces, hist_total)) in enumerate(got_calls):
        for k in got:
            assert np.array_equal(got[k], ref[k]), (call, k)
        assert np.array_equal(cnt, ref_counts), call
        assert rays == n
        assert bounces == int(ref["bounce_count"].sum())
        assert hist_total == n


def test_noalloc_limits(built):
    lib = C.load_library()
    lib.bbrt_trace_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                       ctypes.c_int, ctypes.POINTER(C.TraceOut), ctypes.c_void_p, ctypes.c_int,
                                       ctypes.POINTER(C.TraceStats), ctypes.c_void_p]
    # a scene that is not on the device yet: nothing may be allocated to put it there
    sc = api.Scene(scenes.scene_two_spheres()[:8], config=C.default_config(coarse_grid_n=5))
    rc = lib.bbrt_trace_noalloc(sc.h, None, None, 0, 5, None, None, 1, None, None)
    assert rc == C.BBRT_ERR_STATE
    assert b"not on the device" in lib.bbrt_last_error()
    # hit counters for more objects than the static array holds
    tris = [(k, 0, 0, k + 1, 0, 0, k, 1, 0) for k in range(32769)]
    big = api.Scene(triangles=tris)
    dummy = ctypes.c_longlong(0)
    rc = lib.bbrt_trace_noalloc(big.h, None, None, 0, 5, None, ctypes.byref(dummy), 1, None, None)
    assert rc == C.BBRT_ERR_ARG
    assert b"at most 32768 objects" in lib.bbrt_last_error()
