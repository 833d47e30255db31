"""The oracle port (oracle/bbrt_oracle.cpp) pinned against the reference.

CPU only.  The fixtures under tests/golden/ were produced by the reference's
own code (tests/golden/make_golden.py); where the compiled reference is
present (oracle/_ref) the oracle is also compared with it live.
"""
import numpy as np
import pytest

import oracle
from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import scenes
from conftest import golden
from golden.make_golden import ray_digest, scene_digest, array_digest

TRACE_FIXTURES = [("two_spheres", None, None, None), ("two_spheres_ref_constants", 2048, 100, 1e-3),
                  ("tetra_spheres", 4096, None, None), ("ellipsoids", 2048, None, None)]


def _workload(fixture, n, cn, tol):
    base = "two_spheres" if fixture.startswith("two_spheres") else fixture
    patches, o, d, maxb, wcn, wtol = scenes.workload(base, n)
    return patches, o, d, maxb, cn or wcn, tol or wtol


def check_against_fixture(res, fx, tol_point=0.0):
    """Exact status / bounce count / hit objects; points within tol_point."""
    assert np.array_equal(res["status"], fx["status"].astype(np.int32))
    assert np.array_equal(res["bounce_count"], fx["bounce_count"].astype(np.int32))
    b = fx["bounced"]
    K = fx["hit_object"].shape[1]
    assert np.array_equal(res["hit_object"][b][:, :K], fx["hit_object"])
    assert np.max(np.abs(res["hit_point"][b][:, :K] - fx["hit_point"]), initial=0.0) <= tol_point
    assert np.max(np.abs(res["end_point"][b] - fx["bounced_end_point"]), initial=0.0) <= tol_point
    e = fx["escaped_sample"]
    assert np.max(np.abs(res["end_point"][e] - fx["escaped_end_point"]), initial=0.0) <= max(tol_point, 0.0)
    assert np.max(np.abs(res["exit_dir"][e] - fx["escaped_exit_dir"]), initial=0.0) <= 1e-12


@pytest.mark.parametrize("fixture,n,cn,tol", TRACE_FIXTURES)
def test_scene_generator_is_deterministic(fixture, n, cn, tol):
    fx = golden(fixture)
    patches, o, d, *_ = _workload(fixture, n, cn, tol)
    assert scene_digest(patches) == str(fx["scene_sha256"])
    assert ray_digest(o, d) == str(fx["ray_sha256"])


@pytest.mark.parametrize("fixture,n,cn,tol", TRACE_FIXTURES)
def test_oracle_matches_reference_fixture(built, fixture, n, cn, tol):
    fx = golden(fixture)
    patches, o, d, maxb, cn, tol = _workload(fixture, n, cn, tol)
    orc = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    info = orc.info()
    assert info["scene_diagonal"] == float(fx["scene_diagonal"])
    assert info["max_patch_sagitta"] == float(fx["max_patch_sagitta"])
    for row, k in enumerate(fx["setup_index"]):
        s = orc.object_setup(int(k))
        assert np.array_equal(s["box"], fx["setup_box"][row])
        assert np.array_equal(s["centroid"], fx["setup_centroid"][row])
        assert s["max_sagitta"] == fx["setup_max_sagitta"][row]
        assert array_digest(s["coarse_xyz"], s["sagitta"], s["cell_normal"]) == str(fx["setup_coarse_sha256"][row])
    r = orc.trace(o, d, maxb, K=fx["hit_object"].shape[1], nthreads=0)
    check_against_fixture(r, fx, tol_point=0.0)
    # Newton failures name the same patch (the reference's message quotes its zoneID)
    err = np.nonzero(fx["err_zone"] >= 0)[0]
    zones = fx["zone_ids"]
    assert np.array_equal(zones[r["err_object"][err]], fx["err_zone"][err])


def test_triangle_unit_test_vectors(built):
    """tests/Triangle_Intersect.cpp: BVH(leaf 1) == brute force, t = 1, 1, miss, 5."""
    fx = golden("triangles")
    cfg = C.default_config(leaf_threshold=1)
    orc = oracle.Oracle(triangles=list(fx["tris"]), config=cfg)
    bvh = orc.intersect(fx["origins"], fx["dirs"], C.QUERY_BVH)
    brute = orc.intersect(fx["origins"], fx["dirs"], C.QUERY_BRUTE)
    t_bvh = np.where(bvh["object"] >= 0, bvh["t"], -1.0)
    t_brute = np.where(brute["object"] >= 0, brute["t"], -1.0)
    assert np.array_equal(t_bvh, fx["bvh_t"])
    assert np.array_equal(t_brute, fx["brute_t"])
    assert np.allclose(t_bvh, [1.0, 1.0, -1.0, 5.0], atol=1e-9)
    assert list(bvh["object"]) == list(fx["bvh_obj"])


def test_oracle_plane_counts_fixture(built):
    fx = golden("plane_counts")
    patches = scenes.scene_two_spheres()
    assert scene_digest(patches) == str(fx["scene_sha256"])
    orc = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    src = scenes.plane_grid(fx["corner0"], fx["corner1"], int(fx["nx"]), int(fx["ny"]))
    assert np.array_equal(orc.plane_counts(src, fx["direction"], int(fx["max_bounces"]), False), fx["counts"])
    assert np.array_equal(orc.plane_counts(src, fx["direction"], int(fx["max_bounces"]), True), fx["counts_direct"])


def bounce_map_scene_order(n):
    """Object order of the reference's sorted directory scan of p1.txt .. pN.txt."""
    names = sorted(f"p{k + 1}.txt" for k in range(n))
    return [int(s[1:-4]) - 1 for s in names]


def test_oracle_bounce_map_fixture(built):
    fx = golden("bounce_map")
    patches = scenes.scene_two_spheres()
    order = bounce_map_scene_order(len(patches))
    orc = oracle.Oracle([patches[k] for k in order], config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    samples = patches[int(fx["first"]) - 1:int(fx["last"])]
    mb, er, _ = orc.bounce_map(samples, int(fx["grid_n"]), int(fx["theta_n"]), int(fx["phi_n"]),
                               float(fx["cone"]), int(fx["max_bounces"]))
    assert np.array_equal(mb, fx["max_b"])
    assert np.array_equal(er, fx["errors"])


@pytest.mark.skipif(not oracle.reference_available(), reason="compiled reference not present")
def test_oracle_matches_live_reference_on_fresh_rays(built):
    """A ray set no fixture holds: grazing and axis-aligned rays on the tetrahedron scene."""
    patches = scenes.scene_tetra_spheres()
    rng = np.random.Generator(np.random.PCG64(99))
    n = 3000
    o = rng.uniform(-4, 4, (n, 3))
    d = rng.normal(size=(n, 3))
    d[:500, 1] = 0.0                       # axis-parallel components: inf in 1/d
    d[500:600, :2] = 0.0
    o[600:800] = scenes.tetrahedron_centers()[0] + np.array([0.0, 0.0, 1.0]) * 1.0000001  # grazing tops
    d[600:800] = np.column_stack([rng.normal(size=200), rng.normal(size=200), np.full(200, 1e-7)])
    ref = oracle.Reference.from_patches(patches, coarse_n=17, newton_tol=1e-12)
    rr = ref.trace(o, d, 50, K=4, nthreads=0)
    orc = oracle.Oracle(patches, config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    ro = orc.trace(o, d, 50, K=4)
    for k in ("status", "bounce_count", "hit_object", "hit_point", "end_point"):
        assert np.array_equal(rr[k], ro[k]), k
