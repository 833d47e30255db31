"""C ABI boundary checks that need no GPU: the library loads, exports every
declared entry point, its structs match the header, and the host side of
scene creation (object set-up, BVH, scene scale) equals the oracle's."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

import oracle
from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes
from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "bbrt.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"BBRT_API\s+[\w\s\*]+?\b(bbrt_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol(built):
    syms = declared_symbols()
    assert len(syms) >= 20
    lib = ctypes.CDLL(C.LIB_PATH)
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_struct_layouts_match_header(built):
    structs = {"bbrt_config": C.Config, "bbrt_patch_desc": C.PatchDesc, "bbrt_object_desc": C.ObjectDesc,
               "bbrt_patch_file": C.PatchFile, "bbrt_scene_info": C.SceneInfo, "bbrt_object_info": C.ObjectInfo,
               "bbrt_hit": C.Hit, "bbrt_trace_out": C.TraceOut, "bbrt_trace_stats": C.TraceStats,
               "bbrt_tuning": C.Tuning, "bbrt_guess_train_config": C.GuessTrainConfig,
               "bbrt_guess_train_report": C.GuessTrainReport}
    src = '#include <stdio.h>\n#include "bbrt.h"\nint main(void){\n'
    for name in structs:
        src += f'printf("{name} %zu\\n", sizeof({name}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as tmp:
        c = os.path.join(tmp, "s.c")
        open(c, "w").write(src)
        exe = os.path.join(tmp, "s")
        subprocess.run(["gcc", "-std=c99", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    sizes = dict(line.split() for line in out.strip().splitlines())
    for name, cls in structs.items():
        assert int(sizes[name]) == ctypes.sizeof(cls), name
    assert C.HIT_DTYPE.itemsize == ctypes.sizeof(C.Hit)


def test_config_defaults_are_the_reference_constants(built):
    lib = C.load_library()
    c = C.Config()
    lib.bbrt_config_init(ctypes.byref(c))
    d = C.default_config()
    for k, _ in C.Config._fields_:
        assert getattr(c, k) == getattr(d, k), k
    assert (c.coarse_grid_n, c.newton_max_iters, c.newton_tol, c.leaf_threshold) == (100, 20, 1e-3, 4)


@pytest.mark.parametrize("name,n_patches", [("two_spheres", None), ("tetra_spheres", None), ("ellipsoids", 300)])
def test_host_scene_setup_equals_oracle(built, workloads, name, n_patches):
    patches, o, d, maxb, cn, tol = workloads(name, 8)
    patches = patches[:n_patches] if n_patches else patches
    cfg = C.default_config(coarse_grid_n=cn, newton_tol=tol)
    sc = api.Scene(patches, config=cfg)
    orc = oracle.Oracle(patches, config=cfg)
    si, oi = sc.info(), orc.info()
    assert si["n_nodes"] == oi["n_nodes"]
    assert si["scene_diagonal"] == oi["scene_diagonal"]
    assert si["max_patch_sagitta"] == oi["max_patch_sagitta"]
    for k in range(len(patches)):
        a, b, g = orc.object_setup(k), sc.object_info(k), sc.coarse_grid(k)
        assert np.array_equal(a["box"], b["box"])
        assert np.array_equal(a["centroid"], b["centroid"])
        assert a["max_sagitta"] == b["padding"]
        for key in ("coarse_xyz", "sagitta", "cell_normal"):
            assert np.array_equal(a[key], g[key]), (k, key)
        assert b["zone_id"] == patches[k].zone_id
    assert sc.self_intersect_epsilon(0) == max(1e-9 * si["scene_diagonal"], 5.0 * sc.object_info(0)["padding"])


def test_patch_file_roundtrip_and_dir_order(built, tmp_path):
    patches = scenes.scene_two_spheres()[:12]
    patches[3].edge_flags = (1, 0, 1, 0)
    scenes.write_scene_dir(str(tmp_path), patches)
    (tmp_path / "notes.dat").write_text("ignored: not a .txt file\n")
    files = sorted(p for p in os.listdir(tmp_path) if p.endswith(".txt"))
    f = api.read_patch_file(str(tmp_path / files[3]))
    for k in ("u_nodes", "v_nodes") + scenes.Patch.FIELDS:
        assert np.array_equal(f[k], getattr(patches[3], k)), k
    assert f["edge_flags"] == [1, 0, 1, 0]
    cfg = C.default_config(coarse_grid_n=9)
    from_dir = api.Scene(config=cfg, directory=str(tmp_path))
    direct = api.Scene(patches, config=cfg)
    assert from_dir.n_objects == 12
    for k in range(12):
        assert from_dir.object_info(k)["zone_id"] == patches[k].zone_id
        assert np.array_equal(from_dir.object_info(k)["box"], direct.object_info(k)["box"])


def test_range_constructor_uses_numeric_names(built, tmp_path):
    patches = scenes.scene_two_spheres()[:11]
    for k, p in enumerate(patches):
        scenes.write_patch_file(str(tmp_path / f"zone-{k + 1}.txt"), p)
    sc = api.Scene.from_range(str(tmp_path) + os.sep, "zone-", 2, 11, C.default_config(coarse_grid_n=5))
    assert [sc.object_info(k)["zone_id"] for k in range(10)] == [p.zone_id for p in patches[1:11]]


def test_errors_fail_loud(built, tmp_path):
    lib = C.load_library()
    h = ctypes.c_void_p()
    cfg = C.default_config()
    assert lib.bbrt_scene_create_from_dir(str(tmp_path / "missing").encode(), ctypes.byref(cfg), ctypes.byref(h)) == C.BBRT_ERR_IO
    assert b"not a directory" in lib.bbrt_last_error()
    assert lib.bbrt_scene_create_from_dir(str(tmp_path).encode(), ctypes.byref(cfg), ctypes.byref(h)) == C.BBRT_ERR_IO
    assert b"no *.txt patch files" in lib.bbrt_last_error()
    bad = tmp_path / "bad.txt"
    bad.write_text("5 5 1 7\n0 1 2\n")
    f = C.PatchFile()
    assert lib.bbrt_patch_file_read(str(bad).encode(), ctypes.byref(f)) == C.BBRT_ERR_FORMAT
    assert b"truncated patch file" in lib.bbrt_last_error()
    bad.write_text("x")
    assert lib.bbrt_patch_file_read(str(bad).encode(), ctypes.byref(f)) == C.BBRT_ERR_FORMAT
    assert b"bad header" in lib.bbrt_last_error()
    p = scenes.scene_two_spheres()[0]
    scenes.write_patch_file(str(bad), p)
    with open(bad, "a") as fh:
        fh.write("1 2 three\n")
    assert lib.bbrt_patch_file_read(str(bad).encode(), ctypes.byref(f)) == C.BBRT_ERR_FORMAT
    assert b"malformed sharp-edge" in lib.bbrt_last_error()
    assert lib.bbrt_scene_create_from_range(str(tmp_path).encode(), b"p", 3, 2, ctypes.byref(cfg), ctypes.byref(h)) == C.BBRT_ERR_ARG
    assert b"empty patch index range" in lib.bbrt_last_error()
    with pytest.raises(RuntimeError, match="kmax"):
        q = scenes.scene_two_spheres()[0]
        q.kmax = 2
        api.Scene([q])
    with pytest.raises(RuntimeError, match="at least one object"):
        api.Scene([])


@pytest.mark.skipif(C.load_library().bbrt_device_count() > 0, reason="a GPU is present")
def test_no_cpu_fallback_without_gpu(built, workloads):
    patches, o, d, maxb, cn, tol = workloads("two_spheres", 4)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn))
    with pytest.raises(RuntimeError, match="no CUDA device"):
        sc.trace(o, d, maxb)
    with pytest.raises(RuntimeError, match="no CUDA device"):
        sc.intersect(o, d)


def test_node_test_check_arguments(built):
    """bbrt_node_test_check: NULL arrays and negative counts are argument
    errors, an empty call succeeds, and on a machine without a GPU it fails
    loudly (the FP32 node test has no CPU path)."""
    lib = C.load_library()
    out = np.zeros(2, dtype=np.int32)
    v = np.zeros(3)
    assert lib.bbrt_node_test_check(None, None, None, 1, None, None) == C.BBRT_ERR_ARG
    assert lib.bbrt_node_test_check(C.ptr(v), C.ptr(v), C.ptr(v), -1, C.ptr(np.zeros(6)),
                                    C.ptr(out, ctypes.c_int)) == C.BBRT_ERR_ARG
    assert lib.bbrt_node_test_check(None, None, None, 0, None, None) == C.BBRT_OK
    if lib.bbrt_device_count() > 0:
        return
    rc = lib.bbrt_node_test_check(C.ptr(v), C.ptr(np.array([0.0, 0.0, -1.0])), C.ptr(np.array([np.inf])), 1,
                                  C.ptr(np.array([-1.0, -1.0, -1.0, 1.0, 1.0, 1.0])), C.ptr(out, ctypes.c_int))
    assert rc == C.BBRT_ERR_CUDA and b"no CUDA device" in lib.bbrt_last_error()


def test_bounce_map_rays_equal_oracle(built):
    """bbrt_bounce_map_rays is host code: the launch rays of
    BounceMapDriver::run (BounceMapDriver.hpp:119-237), bit for bit."""
    patches = scenes.scene_two_spheres()
    cfg = C.default_config(coarse_grid_n=9, newton_tol=1e-12)
    sc = api.Scene(patches, config=cfg)
    orc = oracle.Oracle(patches, config=cfg)
    samples = patches[3:6]
    for grid, theta, phi, cone in ((3, 2, 5, 180.0), (4, 3, 4, 37.5)):
        o, d = sc.bounce_map_rays(samples, grid, theta, phi, cone)
        ro, rd = orc.bounce_map_rays(samples, grid, theta, phi, cone)
        assert np.array_equal(o, ro) and np.array_equal(d, rd)
        pick = np.array([o.shape[0] - 1, 0, 17, 5, 17])
        so, sd = sc.bounce_map_rays(samples, grid, theta, phi, cone, ray_index=pick)
        assert np.array_equal(so, ro[pick]) and np.array_equal(sd, rd[pick])
    with pytest.raises(RuntimeError, match="out of range"):
        sc.bounce_map_rays(samples, 3, 2, 5, 180.0, ray_index=[3 * 9 * 10])
    with pytest.raises(RuntimeError, match="position_grid_n must be >= 2"):
        sc.bounce_map_rays(samples, 1, 2, 5, 180.0)


def test_scene_tuning_roundtrip_and_validation(built):
    sc = api.Scene(scenes.scene_two_spheres(), config=C.default_config(coarse_grid_n=9))
    t = sc.tuning()
    assert t["advance_shape"] == 3 and t["warp_stage1"] == 1 and t["wave_tail"] == 4096 and t["graph_rounds"] == 1
    t2 = sc.tuning(advance_shape=6, wave_tail=8192, graph_rounds=0)
    assert t2["advance_shape"] == 6 and t2["wave_tail"] == 8192 and t2["graph_rounds"] == 0 and sc.tuning() == t2
    with pytest.raises(RuntimeError, match="advance_shape"):
        sc.tuning(advance_shape=9)
    with pytest.raises(RuntimeError, match="graph_rounds"):
        sc.tuning(graph_rounds=2)
