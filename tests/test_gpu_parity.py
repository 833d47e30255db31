"""GPU parity: the CUDA trace path (through the C ABI) against the oracle and
against the reference's own outputs (tests/golden/).

The FP64 path is bit-identical to the reference by construction, so status,
bounce counts and hit objects are compared exactly and hit points, end
points and exit directions are compared for exact equality as well (the
contract's bar is 1e-10 absolute; exact equality is stronger).
"""
import numpy as np
import pytest

import oracle
from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes
from conftest import golden
from test_oracle import TRACE_FIXTURES, _workload, bounce_map_scene_order, check_against_fixture

pytestmark = pytest.mark.gpu
POINT_TOL = 1e-10


def assert_same_trace(g, r, exact=True):
    for k in ("status", "bounce_count", "hit_object", "err_object"):
        assert np.array_equal(g[k], r[k]), k
    for k in ("hit_point", "end_point", "exit_dir", "hit_uv"):
        if exact:
            assert np.array_equal(g[k], r[k]), (k, np.max(np.abs(g[k] - r[k])))
        else:
            assert np.max(np.abs(g[k] - r[k])) <= POINT_TOL, k


@pytest.mark.parametrize("cull", [0, 1])
@pytest.mark.parametrize("name,n", [("two_spheres", None), ("tetra_spheres", 65536), ("ellipsoids", 32768)])
def test_trace_matches_oracle(built, workloads, name, n, cull):
    patches, o, d, maxb, cn, tol = workloads(name, n)
    cfg = C.default_config(coarse_grid_n=cn, newton_tol=tol, cull=cull)
    g = api.Scene(patches, config=cfg).trace(o, d, maxb, record=6)
    r = oracle.Oracle(patches, config=cfg).trace(o, d, maxb, K=6)
    assert_same_trace(g, r)
    st = g["stats"]
    assert st["rays"] == o.shape[0]
    assert sum(st["status_hist"]) == o.shape[0]
    assert st["bounces"] == int(g["bounce_count"].sum())
    assert st["status_hist"] == list(np.bincount(g["status"], minlength=C.RAY_STATUS_COUNT))


@pytest.mark.parametrize("fixture,n,cn,tol", TRACE_FIXTURES)
def test_trace_matches_reference_fixture(built, fixture, n, cn, tol):
    fx = golden(fixture)
    patches, o, d, maxb, cn, tol = _workload(fixture, n, cn, tol)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    g = sc.trace(o, d, maxb, record=fx["hit_object"].shape[1])
    check_against_fixture(g, fx, tol_point=0.0)
    err = np.nonzero(fx["err_zone"] >= 0)[0]
    assert np.array_equal(fx["zone_ids"][g["err_object"][err]], fx["err_zone"][err])
    assert sc.info()["scene_diagonal"] == float(fx["scene_diagonal"])


@pytest.mark.parametrize("mode", [C.QUERY_BVH, C.QUERY_BRUTE])
def test_single_queries_match_oracle(built, workloads, mode):
    patches, *_ = workloads("tetra_spheres", 4)
    cfg = C.default_config(coarse_grid_n=17, newton_tol=1e-12)
    rng = np.random.Generator(np.random.PCG64(5))
    n = 4096 if mode == C.QUERY_BVH else 512
    o = rng.uniform(-3.5, 3.5, (n, 3))
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    g = api.Scene(patches, config=cfg).intersect(o, d, mode)
    r = oracle.Oracle(patches, config=cfg).intersect(o, d, mode)
    assert np.array_equal(g, r)
    assert (g["object"] >= 0).sum() > n // 10


def test_single_object_queries(built, workloads):
    patches, *_ = workloads("two_spheres", 4)
    cfg = C.default_config(coarse_grid_n=9, newton_tol=1e-12)
    sc, orc = api.Scene(patches, config=cfg), oracle.Oracle(patches, config=cfg)
    rng = np.random.Generator(np.random.PCG64(6))
    for k in (0, 17, 101, 191):
        c = sc.object_info(k)["centroid"]
        o = c + rng.normal(size=(256, 3)) * 0.2 + sc.object_info(k)["centroid"] * 0.5
        d = c - o + rng.normal(size=(256, 3)) * 0.05
        g, r = sc.intersect(o, d, C.QUERY_OBJECT, k), orc.intersect(o, d, C.QUERY_OBJECT, k)
        diff = [i for i in range(len(g)) if g[i].tobytes() != r[i].tobytes()]
        assert not diff, (k, diff[:5], g[diff[0]], r[diff[0]], o[diff[0]], d[diff[0]])


def test_reference_triangle_unit_test(built):
    """tests/Triangle_Intersect.cpp on the GPU: BVH == brute force, t = 1, 1, miss, 5."""
    fx = golden("triangles")
    sc = api.Scene(triangles=list(fx["tris"]), config=C.default_config(leaf_threshold=1))
    bvh = sc.intersect(fx["origins"], fx["dirs"], C.QUERY_BVH)
    brute = sc.intersect(fx["origins"], fx["dirs"], C.QUERY_BRUTE)
    t_bvh = np.where(bvh["object"] >= 0, bvh["t"], -1.0)
    t_brute = np.where(brute["object"] >= 0, brute["t"], -1.0)
    assert np.array_equal(t_bvh, fx["bvh_t"])
    assert np.array_equal(t_brute, fx["brute_t"])
    assert list(bvh["object"]) == list(fx["bvh_obj"])


def test_edge_case_rays(built, workloads):
    patches, *_ = workloads("tetra_spheres", 4)
    cfg = C.default_config(coarse_grid_n=17, newton_tol=1e-12)
    c0 = np.array(scenes.tetrahedron_centers()[0])
    o = np.array([
        [0.0, 0.0, 6.0], [0.0, 0.0, 6.0], [np.nan, 0.0, 6.0], [0.0, 0.0, 6.0],
        c0 + [0.0, 0.0, 3.0], c0 + [3.0, 0.0, 0.0], c0,                    # axis-aligned; from the centre
        c0 + [0.0, 0.0, 1.0 + 1e-9], c0 + [0.0, 1.0, 1.0],                 # grazing the pole
        [1e6, 1e6, 1e6], [0.0, 0.0, 0.0], c0 + [0.3, 0.2, 0.1],
    ])
    d = np.array([
        [0.0, 0.0, -1.0], [0.0, 0.0, 0.0], [0.0, 0.0, -1.0], [np.inf, 0.0, -1.0],
        [0.0, 0.0, -1.0], [-1.0, 0.0, 0.0], [0.0, 0.0, 1.0],
        [1.0, 0.0, 0.0], [0.0, -1.0, 1e-12],
        [-1.0, -1.0, -1.0], [1e-200, 1e-200, 1e-200], [0.0, 1.0, 0.0],
    ])
    sc, orc = api.Scene(patches, config=cfg), oracle.Oracle(patches, config=cfg)
    for maxb in (0, 1, 50):
        g = sc.trace(o, d, maxb, record=4)
        r = orc.trace(o, d, maxb, K=4)
        for k in ("status", "bounce_count", "hit_object", "err_object"):
            assert np.array_equal(g[k], r[k]), (maxb, k)
        for k in ("hit_point", "end_point", "exit_dir"):
            assert np.array_equal(np.nan_to_num(g[k], nan=7.0), np.nan_to_num(r[k], nan=7.0)), (maxb, k)
    assert g["status"][1] == C.RAY_BAD_DIR
    assert g["status"][10] == C.RAY_BAD_DIR          # |d|^2 underflows below 1e-300
    empty = sc.trace(np.zeros((0, 3)), np.zeros((0, 3)), 10)
    assert empty["status"].shape == (0,)


def test_plane_source_counts(built):
    fx = golden("plane_counts")
    patches = scenes.scene_two_spheres()
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    args = (fx["corner0"], fx["corner1"], fx["direction"], int(fx["nx"]), int(fx["ny"]), int(fx["max_bounces"]))
    assert np.array_equal(sc.plane_source(*args, count_direct_hit=False), fx["counts"])
    assert np.array_equal(sc.plane_source(*args, count_direct_hit=True), fx["counts_direct"])
    with pytest.raises(RuntimeError, match="exactly one coordinate"):
        sc.plane_source((0, 0, 4), (1, 1, 5), (0, 0, -1), 4, 4, 5)


def test_bounce_map(built):
    fx = golden("bounce_map")
    patches = scenes.scene_two_spheres()
    order = bounce_map_scene_order(len(patches))
    sc = api.Scene([patches[k] for k in order], config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    samples = patches[int(fx["first"]) - 1:int(fx["last"])]
    mb, er, bd = sc.bounce_map(samples, int(fx["grid_n"]), int(fx["theta_n"]), int(fx["phi_n"]),
                               float(fx["cone"]), int(fx["max_bounces"]))
    assert np.array_equal(mb, fx["max_b"])
    assert np.array_equal(er, fx["errors"])
    orc = oracle.Oracle([patches[k] for k in order], config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    _, _, obd = orc.bounce_map(samples, int(fx["grid_n"]), int(fx["theta_n"]), int(fx["phi_n"]),
                               float(fx["cone"]), int(fx["max_bounces"]))
    assert np.array_equal(bd, obd)


def test_device_pointer_path_equals_host_path(built, workloads):
    import torch
    patches, o, d, maxb, cn, tol = workloads("tetra_spheres", 20000)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    host = sc.trace(o, d, maxb, record=0, outputs=("status", "bounce_count", "exit_dir", "end_point"))
    to = torch.from_numpy(o).cuda()
    td = torch.from_numpy(d).cuda()
    n = o.shape[0]
    st = torch.zeros(n, dtype=torch.int32, device="cuda")
    bc = torch.zeros(n, dtype=torch.int32, device="cuda")
    ed = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    ep = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
    side = torch.cuda.Stream()
    torch.cuda.set_stream(side)
    stream = side.cuda_stream
    stats = sc.trace_device(to.data_ptr(), td.data_ptr(), n, maxb,
                            dict(status=st.data_ptr(), bounce_count=bc.data_ptr(), exit_dir=ed.data_ptr(),
                                 end_point=ep.data_ptr()), stream=stream, want_stats=True)
    torch.cuda.synchronize()
    assert np.array_equal(st.cpu().numpy(), host["status"])
    assert np.array_equal(bc.cpu().numpy(), host["bounce_count"])
    assert np.array_equal(ed.cpu().numpy(), host["exit_dir"])
    assert np.array_equal(ep.cpu().numpy(), host["end_point"])
    assert stats["bounces"] == int(host["bounce_count"].sum())


def test_full_size_tetra_workload(built, workloads):
    """The full 1M-ray tetrahedron workload: culled == unculled bit for bit,
    consistent counters, and a 65k-ray sample against the oracle."""
    patches, o, d, maxb, cn, tol = workloads("tetra_spheres")
    outs = ("status", "bounce_count", "exit_dir", "end_point")
    a = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol, cull=1)).trace(
        o, d, maxb, record=0, outputs=outs)
    b = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol, cull=0)).trace(
        o, d, maxb, record=0, outputs=outs)
    for k in outs:
        assert np.array_equal(a[k], b[k]), k
    assert a["stats"]["bounces"] == int(a["bounce_count"].sum())
    assert a["stats"]["tri_tests"] < b["stats"]["tri_tests"] // 4
    sel = np.arange(0, o.shape[0], 16)
    r = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol)).trace(o[sel], d[sel], maxb, K=0)
    for k in outs:
        assert np.array_equal(a[k][sel], r[k]), k


def test_nested_spheres_many_solves_per_query(built):
    """Concentric spheres: a ray through the centre crosses many patches, so a
    single query needs several Newton solves (more than the wavefront's
    resolved list holds for some rays) — wavefront, overflow and tail paths
    against the oracle, plus the fused per-ray kernel on a small batch."""
    patches = []
    for k, r in enumerate((1.0, 1.4, 1.9, 2.5, 3.2)):
        patches += scenes.obstacle_patches(k, (0.0, 0.0, 0.0), (r, r, r), None, m=2, n_nodes=5)
    rng = np.random.Generator(np.random.PCG64(11))
    n = 20000
    o = rng.normal(size=(n, 3))
    o = 6.0 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o + rng.normal(size=(n, 3)) * 0.8
    cfg = C.default_config(coarse_grid_n=9, newton_tol=1e-12)
    sc, orc = api.Scene(patches, config=cfg), oracle.Oracle(patches, config=cfg)
    g = sc.trace(o, d, 30, record=4)
    r = orc.trace(o, d, 30, K=4)
    assert_same_trace(g, r)
    small = sc.trace(o[:500], d[:500], 30, record=4)
    for k in ("status", "bounce_count", "hit_object", "hit_point", "end_point", "exit_dir"):
        assert np.array_equal(small[k], g[k][:500]), k


TUNING_SCRIPT = r'''
import sys, numpy as np
sys.path.insert(0, sys.argv[1])
from billardballraytracing3d_b200 import scenes, api, _capi as C
patches, o, d, maxb, cn, tol = scenes.workload("tetra_spheres", 40000)
g = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol)).trace(o, d, maxb, record=4)
np.savez(sys.argv[2], **{k: g[k] for k in ("status", "bounce_count", "hit_object", "hit_point", "end_point", "exit_dir")})
'''


@pytest.mark.parametrize("env", [{"BBRT_WAVE_TAIL": "0"}, {"BBRT_WARP_TAIL": "0"}, {"BBRT_WAVE_TAIL": "100000"},
                                 {"BBRT_ORDER_RAYS": "0", "BBRT_WAVE_MIN": "1000000"},
                                 {"BBRT_GROUP_NEWTON": "1"}, {"BBRT_WARP_S1": "0", "BBRT_RESUME": "0"},
                                 {"BBRT_ADV_SHAPE": "0", "BBRT_TAIL_SHAPE": "2"}, {"BBRT_GRAPH": "0"},
                                 {"BBRT_GRAPH": "0", "BBRT_WAVE_TAIL": "0"}, {"BBRT_SORT_REQ": "0"},
                                 {"BBRT_SORT_REQ": "0", "BBRT_GRAPH": "0"}, {"BBRT_SORT_SIDE": "1"}, {"BBRT_ORDER_ENTRY": "0"},
                                 {"BBRT_CHILD_TEST": "1"}, {"BBRT_HALF_S1": "0"}, {"BBRT_QUARTER_S1": "1"},
                                 {"BBRT_QUARTER_S1": "1", "BBRT_GRAPH": "0"}, {"BBRT_NODE_F32": "0"},
                                 {"BBRT_NODE_F32": "0", "BBRT_GRAPH": "0"}, {"BBRT_NODE_F32": "0", "BBRT_CHILD_TEST": "1"},
                                 {"BBRT_NODE_F32": "0", "BBRT_TAIL_SHAPE": "3", "BBRT_WAVE_TAIL": "100000"},
                                 {"BBRT_ADAPT_LANES": "0"}, {"BBRT_ADAPT_LANES": "0", "BBRT_GRAPH": "0"},
                                 {"BBRT_WAVE_TAIL": "0", "BBRT_GRAPH": "0", "BBRT_ADAPT_LANES": "1"},
                                 {"BBRT_NEWTON_GROUP_MAX": "0"}, {"BBRT_NEWTON_GROUP_MAX": "100000000", "BBRT_GRAPH": "0"},
                                 {"BBRT_NEWTON_GROUP_MAX": "100000000", "BBRT_WAVE_TAIL": "1024"}])
def test_launch_shape_knobs_do_not_change_results(built, workloads, tmp_path, env):
    """Every schedule (all wavefront rounds, per-thread or per-warp tail, fused
    kernel only, unordered rays, host-driven or graph-launched rounds, Newton
    requests grouped by patch or not, BVH nodes tested in FP32 with an FP64
    re-test or in FP64 only, small rounds spread over every warp or not) gives
    the oracle's results bit for bit."""
    import os
    import subprocess
    import sys
    from conftest import ROOT
    out = tmp_path / "r.npz"
    subprocess.run([sys.executable, "-c", TUNING_SCRIPT, ROOT, str(out)], check=True, env={**os.environ, **env})
    g = np.load(out)
    patches, o, d, maxb, cn, tol = workloads("tetra_spheres", 40000)
    r = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol)).trace(o, d, maxb, K=4)
    for k in g.files:
        assert np.array_equal(g[k], r[k]), (env, k)


def test_autotune_keeps_results(built, workloads):
    """The autotuner only picks a launch schedule: the trace under the chosen
    schedule equals the trace under the defaults, bit for bit."""
    patches, o, d, maxb, cn, tol = workloads("tetra_spheres", 131072)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    base = sc.trace(o, d, maxb, record=4, outputs=("status", "bounce_count", "hit_object", "hit_point", "exit_dir"))
    best = sc.autotune(o, d, maxb, trials=1)
    assert best["ms"] > 0 and 0 <= best["advance_shape"] <= 6
    assert sc.tuning()["advance_shape"] == best["advance_shape"]
    tuned = sc.trace(o, d, maxb, record=4, outputs=("status", "bounce_count", "hit_object", "hit_point", "exit_dir"))
    for k in ("status", "bounce_count", "hit_object", "hit_point", "exit_dir"):
        assert np.array_equal(base[k], tuned[k]), k


def test_trace_batch_equals_single_scene_traces(built):
    """bbrt_trace_batch traces uneven scenes together; each scene's results are
    bit-identical to tracing it alone (wavefront and fused-kernel sizes mixed)."""
    import torch
    work = scenes.multi_scene_workload(4, seed=5, max_obstacles=6, min_rays=4000, max_rays=60000)
    scs, tens, outs, refs = [], [], [], []
    K = 4
    for patches, o, d, maxb, cn, tol in work:
        sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
        refs.append(sc.trace(o, d, maxb, record=K, outputs=("status", "bounce_count", "exit_dir", "hit_object",
                                                             "hit_point")))
        n = o.shape[0]
        t = dict(o=torch.from_numpy(o).cuda(), d=torch.from_numpy(d).cuda(),
                 status=torch.zeros(n, dtype=torch.int32, device="cuda"),
                 bounce_count=torch.zeros(n, dtype=torch.int32, device="cuda"),
                 exit_dir=torch.zeros((n, 3), dtype=torch.float64, device="cuda"),
                 hit_object=torch.zeros((n, K), dtype=torch.int32, device="cuda"),
                 hit_point=torch.zeros((n, K, 3), dtype=torch.float64, device="cuda"))
        scs.append(sc)
        tens.append(t)
        outs.append(dict(record=K, **{k: t[k].data_ptr() for k in ("status", "bounce_count", "exit_dir", "hit_object",
                                                                     "hit_point")}))
    assert min(o.shape[0] for _, o, _, _, _, _ in work) < 8192 <= max(o.shape[0] for _, o, _, _, _, _ in work)
    st, ms = api.trace_batch_device(scs, [t["o"].data_ptr() for t in tens], [t["d"].data_ptr() for t in tens],
                                    [w[1].shape[0] for w in work], 100, outs)
    torch.cuda.synchronize()
    assert ms > 0 and st["rays"] == sum(w[1].shape[0] for w in work)
    for ref, t in zip(refs, tens):
        for k in ("status", "bounce_count", "exit_dir", "hit_object", "hit_point"):
            assert np.array_equal(ref[k], t[k].cpu().numpy()), k
    assert st["bounces"] == sum(int(r["bounce_count"].sum()) for r in refs)


@pytest.mark.gpu
@pytest.mark.parametrize("graph_rounds", [1, 0])
def test_statistics_free_kernels_give_the_same_results(built, workloads, graph_rounds):
    """A call without statistics runs the k_advance and tail instances that
    keep no counters: the same results bit for bit as a call with them."""
    import torch
    patches, o, d, maxb, cn, tol = workloads("tetra_spheres", 65536)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    sc.tuning(graph_rounds=graph_rounds)
    n, K = o.shape[0], 8
    to = torch.from_numpy(np.ascontiguousarray(o)).cuda()
    td = torch.from_numpy(np.ascontiguousarray(d)).cuda()
    res = []
    for want_stats in (True, False):
        bufs = {"status": torch.full((n,), -1, dtype=torch.int32, device="cuda"),
                "bounce_count": torch.full((n,), -1, dtype=torch.int32, device="cuda"),
                "exit_dir": torch.zeros((n, 3), dtype=torch.float64, device="cuda"),
                "end_point": torch.zeros((n, 3), dtype=torch.float64, device="cuda"),
                "hit_object": torch.full((n, K), -9, dtype=torch.int32, device="cuda"),
                "hit_point": torch.zeros((n, K, 3), dtype=torch.float64, device="cuda")}
        st = sc.trace_device(to.data_ptr(), td.data_ptr(), n, maxb, {k: v.data_ptr() for k, v in bufs.items()},
                             record=K, want_stats=want_stats)
        torch.cuda.synchronize()
        res.append({k: v.cpu().numpy() for k, v in bufs.items()})
        if want_stats:
            assert st["node_tests"] > 0
    for k in res[0]:
        assert np.array_equal(res[0][k], res[1][k]), k
    # times only: kernel times, no counters
    sc.tuning(graph_rounds=0)
    st = sc.trace_device(to.data_ptr(), td.data_ptr(), n, maxb, {}, want_stats=True, times_only=True)
    assert st["node_tests"] == 0 and st["advance_ms"] > 0
