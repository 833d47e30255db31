"""Scene compile on the GPU (scene_compile.cu) against the host scene compiler
(scene_host.cpp, itself pinned to the oracle and the reference by
test_capi.py): the coarse grids, cell normals and sagittas, boxes, centroids,
paddings, cull boxes and cull constants must be the same bit for bit, and so
must every trace of the two scenes.  NaNs compare equal to NaNs (the device
and the host spell a NaN made by arithmetic differently)."""
import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes

pytestmark = pytest.mark.gpu


def _bits_equal(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    if a.shape != b.shape:
        return False
    nan = np.isnan(a) & np.isnan(b)
    ia = a.view(np.uint64 if a.dtype == np.float64 else np.uint32)
    ib = b.view(np.uint64 if b.dtype == np.float64 else np.uint32)
    return bool(np.all((ia == ib) | nan))


def _uneven(patches):
    """The same surfaces sampled on 7 x 4 nodes (every other v node): patches
    whose two axes have different node counts."""
    out = []
    for p in patches:
        keep = np.arange(0, p.jmax, 2)
        f = {k: getattr(p, k).reshape(p.imax, p.jmax)[:, keep].reshape(-1) for k in scenes.Patch.FIELDS}
        out.append(scenes.Patch(imax=p.imax, jmax=keep.size, zone_id=p.zone_id, u_nodes=p.u_nodes,
                                v_nodes=p.v_nodes[keep], **f))
    return out


def _nan_patch(patches):
    """One patch with a non-finite node: set-up values turn NaN, culling goes off."""
    p = patches[0]
    x = p.x.copy()
    x[3] = np.nan
    f = {k: getattr(p, k) for k in scenes.Patch.FIELDS}
    f["x"] = x
    return [scenes.Patch(imax=p.imax, jmax=p.jmax, zone_id=p.zone_id, u_nodes=p.u_nodes, v_nodes=p.v_nodes, **f)] + \
        list(patches[1:])


CASES = {
    "two_spheres_n9": lambda: (scenes.scene_two_spheres(), (), 9),
    "tetra_n17": lambda: (scenes.scene_tetra_spheres(), (), 17),
    "ellipsoids_n17": lambda: (scenes.scene_ellipsoids(), (), 17),
    "reference_grid_n100": lambda: (scenes.scene_two_spheres(), (), 100),
    "grid_on_nodes_n3": lambda: (scenes.scene_two_spheres()[:24], (), 3),
    "uneven_nodes_with_triangles": lambda: (_uneven(scenes.scene_tetra_spheres(m=2)),
                                            [(4.0, 0.0, 0.0, 5.0, 0.0, 0.0, 4.0, 1.0, 0.5)], 9),
    "non_finite_node": lambda: (_nan_patch(scenes.scene_two_spheres()), (), 9),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_setup_equals_host_setup(built, case):
    patches, tris, cn = CASES[case]()
    host = api.Scene(patches, triangles=tris,
                     config=C.default_config(coarse_grid_n=cn, newton_tol=1e-12, setup_on_device=0))
    dev = api.Scene(patches, triangles=tris,
                    config=C.default_config(coarse_grid_n=cn, newton_tol=1e-12, setup_on_device=1))
    hi, di = host.info(), dev.info()
    assert hi["setup_on_device"] == 0 and di["setup_on_device"] == 1
    for k in ("n_objects", "n_nodes", "max_depth"):
        assert hi[k] == di[k], k
    for k in ("scene_diagonal", "max_patch_sagitta"):
        assert _bits_equal(np.float64(hi[k]), np.float64(di[k])), k
    ha, da = host.setup_arrays(), dev.setup_arrays()
    for k in ha:
        assert _bits_equal(ha[k], da[k]), k
    if case == "non_finite_node":
        assert ha["cull"][0] == 0.0
    else:
        assert ha["cull"][0] == 1.0 and ha["cell_boxes"].size > 0
    for k in range(hi["n_objects"]):
        a, b = host.object_info(k), dev.object_info(k)
        for f in ("box", "centroid"):
            assert _bits_equal(a[f], b[f]), (k, f)
        assert _bits_equal(np.float64(a["padding"]), np.float64(b["padding"])), k
    # one patch through the per-patch accessor, which reads the device copy
    ga, gb = host.coarse_grid(0), dev.coarse_grid(0)
    for f in ("coarse_xyz", "sagitta", "cell_normal"):
        assert _bits_equal(ga[f], gb[f]), f


def test_device_setup_scene_traces_like_the_host_setup_scene(built):
    patches = scenes.scene_tetra_spheres()
    o, d = scenes.cone_rays(65536, 1234, 5.0, 3.0, 10.0)
    runs = []
    for on_device in (0, 1):
        sc = api.Scene(patches, config=C.default_config(coarse_grid_n=17, newton_tol=1e-12,
                                                        setup_on_device=on_device))
        runs.append(sc.trace(o, d, 200, record=8))
    for k in ("status", "bounce_count", "hit_object", "hit_point", "hit_uv", "exit_dir", "end_point"):
        assert np.array_equal(runs[0][k], runs[1][k]), k


def test_default_setup_runs_on_the_gpu(built):
    """With a device present the default (-1) compiles on the GPU, and the
    scene traces with no further set-up upload."""
    patches = scenes.scene_two_spheres()
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    assert sc.info()["setup_on_device"] == 1
    o = scenes.plane_grid((-3.0, -3.0, 4.0), (3.0, 3.0, 4.0), 16, 16)
    d = np.tile(np.array([0.3, 0.0, -1.0]), (o.shape[0], 1))
    r = sc.trace(o, d, 20, record=2)
    assert r["stats"]["rays"] == o.shape[0]
