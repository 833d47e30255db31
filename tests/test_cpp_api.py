"""The C++ mirror of the reference's API (billardballraytracing3d_b200/include/bbrt/).

Programs in tests/cpp/ use ScatObject, Triangle, SurfacePatch, BVH,
BruteForce, RayTracingDriver, PlaneSourceDriver and BounceMapDriver the way
the reference's own tests and examples do (tests/Triangle_Intersect.cpp,
src/main.cpp, tests/PlaneSource_Example.cpp, tests/BounceMap_Example.cpp).
They compile on CPU; on a GPU their outputs are compared with the oracle,
and their exception texts with the reference's (tests/golden/driver_errors.txt).
"""
import os
import struct
import subprocess
import sys

import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import scenes
import oracle

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
GOLDEN = os.path.join(ROOT, "tests", "golden")
sys.path.insert(0, GOLDEN)
from make_driver_errors import SAMPLE_PREFIX, write_driver_scene  # noqa: E402

PROGRAMS = ("triangle_intersect", "drivers", "driver_errors")
PKG = os.path.join(ROOT, "billardballraytracing3d_b200")


def compile_program(name, out_dir):
    exe = os.path.join(out_dir, name)
    cmd = ["g++", "-O1", "-std=c++17", "-Wall", "-Wextra", "-Werror",
           "-I", os.path.join(ROOT, "include"), "-I", os.path.join(PKG, "include", "bbrt"),
           os.path.join(ROOT, "tests", "cpp", name + ".cpp"), "-o", exe,
           "-L", PKG, "-lbbrt_cuda", "-Wl,-rpath," + PKG, "-pthread"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    return exe


@pytest.fixture(scope="module")
def programs(built, tmp_path_factory):
    d = str(tmp_path_factory.mktemp("cpp"))
    return {n: compile_program(n, d) for n in PROGRAMS}


@pytest.fixture(scope="module")
def driver_scene(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("scene")) + "/"
    patches = write_driver_scene(d)
    return d, patches


def test_cpp_headers_compile(programs):
    for n in PROGRAMS:
        assert os.access(programs[n], os.X_OK)


# ---------------------------------------------------------------------------
# GPU: outputs against the oracle and the reference's texts
# ---------------------------------------------------------------------------
def parse_paths(path):
    """drivers' dump: list of dicts (status, bounces, points[n,3], hits, error)."""
    out = []
    with open(path) as f:
        lines = f.read().split("\n")
    i = 0
    while i < len(lines) and lines[i].startswith("R "):
        _, st, b, npts = lines[i].split()
        pts = np.array([[float(v) for v in lines[i + 1 + k].split()[1:]] for k in range(int(npts))]).reshape(-1, 3)
        hits = [int(v) for v in lines[i + 1 + int(npts)].split()[1:]]
        err = lines[i + 2 + int(npts)][2:]
        out.append(dict(status=int(st), bounces=int(b), points=pts, hits=hits, error=err))
        i += 3 + int(npts)
    return out


def cpp_to_string(x):
    """std::to_string(double)."""
    return "%f" % x


def expected_error(r, i, patches):
    st = int(r["status"][i])
    if st == C.RAY_BAD_DIR:
        return "RayTracingDriver::trace_ray: zero-length direction"
    if st == C.RAY_WENT_INSIDE:
        return ("RayTracingDriver::trace_ray: hit back face of patch (dot(dir, normal) > 0) "
                "— ray likely tunneled through a triangulation gap")
    zone = patches[int(r["err_object"][i])].zone_id
    ev = r["err_value"][i]
    if st == C.RAY_NEWTON_SINGULAR:
        return (f"SurfacePatch::intersect: singular Jacobian during Newton refinement (zoneID {zone}), "
                "likely a grazing ray")
    if st == C.RAY_NEWTON_NOCONV:
        return (f"SurfacePatch::intersect: Newton refinement failed to converge in 20 iterations (zoneID {zone}), "
                f"final step norm {cpp_to_string(ev[0])}")
    if st == C.RAY_NEWTON_DOMAIN:
        return (f"SurfacePatch::intersect: Newton refinement converged outside the patch domain "
                f"(u={cpp_to_string(ev[0])}, v={cpp_to_string(ev[1])}, zoneID {zone})")
    raise AssertionError(f"unexpected status {st}")


def expected_paths(r, origins, patches):
    """RayPaths the reference builds (RayTracingDriver.hpp:172-242) from the oracle's trace."""
    out = []
    for i in range(origins.shape[0]):
        st = int(r["status"][i])
        b = int(r["bounce_count"][i])
        pts = [origins[i]] + [r["hit_point"][i, k] for k in range(b)]
        if st == C.RAY_ESCAPED:
            pts.append(r["end_point"][i])
        kind = 0 if st == C.RAY_ESCAPED else 1 if st == C.RAY_MAX_BOUNCES else 2
        out.append(dict(status=kind, bounces=b, points=np.array(pts).reshape(-1, 3),
                        hits=[int(v) for v in r["hit_object"][i, :b]],
                        error=expected_error(r, i, patches) if kind == 2 else ""))
    return out


def assert_same_paths(got, want):
    assert len(got) == len(want)
    for i, (g, w) in enumerate(zip(got, want)):
        assert g["status"] == w["status"], i
        assert g["bounces"] == w["bounces"], i
        assert np.array_equal(g["points"], w["points"]), (i, g["points"], w["points"])
        assert g["hits"] == w["hits"], i
        assert g["error"] == w["error"], i


def vtk_lines(paths, title, id_name):
    """The reference's legacy-VTK line writer (RayTracingDriver.hpp:270-310,
    BounceMapDriver.hpp:350-430): %g is C++'s default double output."""
    pts = [p for q in paths for p in q["points"]]
    segs = []
    base = 0
    for rid, q in enumerate(paths):
        n = len(q["points"])
        segs += [(base + k, base + k + 1, rid, k) for k in range(n - 1)]
        base += n
    s = [f"# vtk DataFile Version 3.0\n{title}\nASCII\nDATASET POLYDATA\n", f"POINTS {len(pts)} double\n"]
    s += ["%g %g %g\n" % tuple(p) for p in pts]
    s.append(f"LINES {len(segs)} {3 * len(segs)}\n")
    s += [f"2 {a} {b}\n" for a, b, _, _ in segs]
    s.append(f"CELL_DATA {len(segs)}\nSCALARS {id_name} int 1\nLOOKUP_TABLE default\n")
    s += [f"{r}\n" for _, _, r, _ in segs]
    s.append("SCALARS BounceIndex int 1\nLOOKUP_TABLE default\n")
    s += [f"{k}\n" for _, _, _, k in segs]
    return "".join(s)


def driver_rays(n=1536, seed=11):
    return scenes.cone_rays(n, seed, plane_z=3.0, half_extent=2.5, cone_half_deg=35.0)


@pytest.mark.gpu
def test_cpp_triangle_intersect(programs):
    r = subprocess.run([programs["triangle_intersect"]], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "All tests passed." in r.stdout


@pytest.mark.gpu
def test_cpp_driver_errors_match_reference(programs, driver_scene):
    d, _ = driver_scene
    r = subprocess.run([programs["driver_errors"], d, SAMPLE_PREFIX], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    with open(os.path.join(GOLDEN, "driver_errors.txt")) as f:
        want = f.read().splitlines()
    assert r.stdout.splitlines() == want


@pytest.mark.gpu
def test_cpp_ray_tracing_driver(programs, driver_scene, tmp_path):
    d, patches = driver_scene
    o, dirs = driver_rays()
    K = 20
    rays = tmp_path / "rays.bin"
    rays.write_bytes(struct.pack("<q", o.shape[0]) + o.astype("<f8").tobytes() + dirs.astype("<f8").tobytes())
    prefix = str(tmp_path) + "/"
    r = subprocess.run([programs["drivers"], "trace", d, str(rays), str(K), prefix],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    orc = oracle.Oracle(patches)
    ref = orc.trace(o, dirs, K, K=K)
    want = expected_paths(ref, o, patches)
    got = parse_paths(prefix + "paths.txt")
    assert_same_paths(got, want)
    assert_same_paths(parse_paths(prefix + "paths_one.txt"), want[:8])
    assert_same_paths(parse_paths(prefix + "paths_threads.txt"), want)
    assert {p["status"] for p in got} == {0, 2}   # escaped, and back-face errors
    assert max(p["bounces"] for p in got) >= 2
    with open(prefix + "traces.vtk") as f:
        assert f.read() == vtk_lines(want, "Billiard-ball ray traces", "RayID")
    n, eps_scene, eps_first = open(prefix + "info.txt").read().split()
    info = orc.info()
    assert int(n) == len(patches)
    assert float(eps_scene) == max(1e-9 * info["scene_diagonal"], 5.0 * info["max_patch_sagitta"])
    assert float(eps_first) == max(1e-9 * info["scene_diagonal"], 5.0 * orc.object_setup(0, False)["max_sagitta"])


@pytest.mark.gpu
def test_cpp_plane_source_driver(programs, driver_scene, tmp_path):
    d, patches = driver_scene
    c0, c1, direction, nx, ny, K = (-3.0, -1.2, 3.0), (3.0, 1.2, 3.0), (0.1, 0.05, -1.0), 48, 40, 20
    prefix = str(tmp_path) + "/"
    args = [str(v) for v in (*c0, *c1, *direction, nx, ny, K, 0)]
    r = subprocess.run([programs["drivers"], "plane", d, *args, prefix], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    got = np.loadtxt(prefix + "plane_counts.txt", dtype=np.int64)
    want = oracle.Oracle(patches).plane_counts(scenes.plane_grid(c0, c1, nx, ny), direction, K, False)
    assert np.array_equal(got, want)
    assert got.sum() > 0
    with open(prefix + "plane.vtk") as f:
        text = f.read()
    n_pts = sum(p.imax * p.jmax for p in patches)
    assert f"POINTS {n_pts} double\n" in text
    tail = text.split("SCALARS HitCount long 1\nLOOKUP_TABLE default\n")[1].split()
    assert [int(v) for v in tail] == [int(c) for p, c in zip(patches, want) for _ in range(p.imax * p.jmax)]


@pytest.mark.gpu
def test_cpp_bounce_map_driver(programs, driver_scene, tmp_path):
    d, patches = driver_scene
    grid, theta, phi, cone, K = 4, 4, 6, 120.0, 20
    prefix = str(tmp_path) + "/"
    r = subprocess.run([programs["drivers"], "bmap", d, SAMPLE_PREFIX, "1", "2", str(grid), str(theta), str(phi),
                        str(cone), str(K), prefix], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    samples = patches[:2]
    orc = oracle.Oracle(patches)
    mb, er, bd = orc.bounce_map(samples, grid, theta, phi, cone, K)
    got = np.loadtxt(prefix + "bmap.txt", dtype=np.int64)
    assert np.array_equal(got[:, 0], mb) and np.array_equal(got[:, 1], er)
    assert mb.max() >= 1
    # best path per point: the oracle's trace of the first direction reaching the maximum
    o, dirs = orc.bounce_map_rays(samples, grid, theta, phi, cone)
    per_point = theta * phi
    pick = [q * per_point + int(bd[q]) for q in range(mb.size) if bd[q] >= 0]
    ref = orc.trace(o[pick], dirs[pick], K, K=K)
    want_some = expected_paths(ref, o[pick], patches)
    want, j = [], 0
    for q in range(mb.size):
        if bd[q] >= 0:
            want.append(want_some[j]); j += 1
        else:
            want.append(dict(status=1, bounces=0, points=np.zeros((0, 3)), hits=[], error=""))
    best = parse_paths(prefix + "bmap_best.txt")
    assert_same_paths(best, want)
    assert all(w["bounces"] == m for w, m in zip(want, mb) if w["points"].size)
    for p in range(2):
        with open(os.path.join(prefix + "best_rays", f"best_rays_patch_{p + 1}.vtk")) as f:
            assert f.read() == vtk_lines(want[p * grid * grid:(p + 1) * grid * grid],
                                         "Best bounce ray per grid point", "PointID")
    with open(prefix + "bmap.vtk") as f:
        text = f.read()
    vals = text.split("SCALARS MaxBounces int 1\nLOOKUP_TABLE default\n")[1]
    mx, ec = vals.split("SCALARS ErrorCount int 1\nLOOKUP_TABLE default\n")
    assert [int(v) for v in mx.split()] == mb.tolist()
    assert [int(v) for v in ec.split()] == er.tolist()
