"""Oracle package — TEST INFRASTRUCTURE ONLY.

Python handles on the two CPU checkers of the trace path:

* ``Oracle``    : oracle/liboracle.so, a C++ restatement of the reference's
                  algorithm (oracle/bbrt_oracle.cpp), buildable anywhere.
* ``Reference`` : oracle/_ref/libbbrt_ref.so, the reference's own headers
                  compiled by oracle/build_ref.sh (only where the reference
                  sources were present at build time).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use
this package, and only as the checker or the timed CPU baseline; the product
(billardballraytracing3d_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import tempfile
from typing import Sequence

import numpy as np

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import scenes

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libbbrt_ref.so")
REF_TRI_BIN = os.path.join(HERE, "_ref", "triangle_intersect")
P = lambda a: None if a is None else a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731


def reference_root() -> str:
    """Where the reference project's sources are looked for: the environment
    variable BBRT_REFERENCE_ROOT, else a directory named `reference` beside
    this repository's root.  Neither exists on a machine that only runs the
    prebuilt oracle libraries."""
    env = os.environ.get("BBRT_REFERENCE_ROOT")
    if env:
        return env
    return os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference")


def build(reference_root_dir: str | None = None) -> None:
    """Compile the oracle port, and the reference oracle when its sources exist."""
    subprocess.run(["bash", os.path.join(HERE, "build_oracle.sh")], check=True)
    reference_root_dir = reference_root_dir or reference_root()
    if os.path.isdir(os.path.join(reference_root_dir, "include")):
        subprocess.run(["bash", os.path.join(HERE, "build_ref.sh"), reference_root_dir], check=True)


def reference_available() -> bool:
    return os.path.exists(REF_SO)


class TraceResult(dict):
    """Per-ray arrays: status, bounce_count, exit_dir, end_point, hit_object,
    hit_point, hit_uv, err_object, err_value (+ seconds, stats)."""


def _alloc_trace(n, K):
    return TraceResult(
        status=np.zeros(n, np.int32), bounce_count=np.zeros(n, np.int32),
        exit_dir=np.zeros((n, 3)), end_point=np.zeros((n, 3)),
        hit_object=np.full((n, K), -1, np.int32), hit_point=np.zeros((n, K, 3)),
        hit_uv=np.zeros((n, K, 2)), err_object=np.full(n, -1, np.int32), err_value=np.zeros((n, 2)))


def trace_out_struct(r, K):
    o = C.TraceOut()
    o.status = C.ptr(r["status"], ctypes.c_int)
    o.bounce_count = C.ptr(r["bounce_count"], ctypes.c_int)
    o.exit_dir = C.ptr(r["exit_dir"])
    o.end_point = C.ptr(r["end_point"])
    o.record_bounces = K
    o.hit_object = C.ptr(r["hit_object"], ctypes.c_int)
    o.hit_point = C.ptr(r["hit_point"])
    o.hit_uv = C.ptr(r["hit_uv"])
    o.err_object = C.ptr(r["err_object"], ctypes.c_int)
    o.err_value = C.ptr(r["err_value"])
    return o


class Oracle:
    """The C++ restatement (oracle/bbrt_oracle.cpp) over one scene."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(ORACLE_SO):
                raise RuntimeError("oracle/liboracle.so not built (oracle/build_oracle.sh)")
            L = ctypes.CDLL(ORACLE_SO)
            V = ctypes.c_void_p
            L.oracle_scene_create.restype = V
            L.oracle_scene_create.argtypes = [ctypes.POINTER(C.ObjectDesc), ctypes.c_int, ctypes.POINTER(C.Config)]
            L.oracle_scene_destroy.argtypes = [V]
            L.oracle_scene_info.argtypes = [V, V, V, V]
            L.oracle_object_setup.argtypes = [V, ctypes.c_int, V, V, V, V, V, V, V]
            L.oracle_bvh_nodes.argtypes = [V, V, V, V]
            L.oracle_intersect.argtypes = [V, ctypes.c_longlong, V, V, ctypes.c_int, ctypes.c_int, V]
            L.oracle_trace.argtypes = [V, ctypes.c_longlong, V, V, ctypes.c_int, ctypes.c_int,
                                       ctypes.POINTER(C.TraceOut), ctypes.POINTER(C.TraceStats), V]
            L.oracle_plane_counts.argtypes = [V, ctypes.c_longlong, V, V, ctypes.c_int, ctypes.c_int, V]
            L.oracle_sample_grid.argtypes = [ctypes.POINTER(C.PatchDesc), ctypes.c_int, V, V, V]
            L.oracle_bounce_map.argtypes = [V, ctypes.POINTER(C.PatchDesc), ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, V, V, V]
            L.oracle_bounce_map_rays.argtypes = [V, ctypes.POINTER(C.PatchDesc), ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, ctypes.c_int, ctypes.c_double, V, V]
            cls._lib = L
        return cls._lib

    def __init__(self, patches: Sequence = (), triangles: Sequence = (), config: C.Config = None):
        self.table = C.ObjectTable(patches, triangles)
        self.config = config if config is not None else C.default_config()
        self.h = self.lib().oracle_scene_create(self.table.descs, self.table.n, ctypes.byref(self.config))
        if not self.h:
            raise ValueError("oracle scene needs at least one object")
        self.n_objects = self.table.n

    def close(self):
        if self.h:
            self.lib().oracle_scene_destroy(self.h)
            self.h = None

    __del__ = close

    def info(self):
        n = ctypes.c_int(); d = ctypes.c_double(); s = ctypes.c_double()
        self.lib().oracle_scene_info(self.h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(s))
        return dict(n_nodes=n.value, scene_diagonal=d.value, max_patch_sagitta=s.value)

    def object_setup(self, idx, want_grid=True):
        box = np.zeros(6); cen = np.zeros(3); ms = np.zeros(1); n = ctypes.c_int()
        self.lib().oracle_object_setup(self.h, idx, P(box), P(cen), P(ms), ctypes.byref(n), None, None, None)
        out = dict(box=box, centroid=cen, max_sagitta=float(ms[0]), n=n.value)
        if want_grid and n.value > 0:
            g = n.value
            xyz = np.zeros((g * g, 3)); sag = np.zeros((g - 1) ** 2); nrm = np.zeros(((g - 1) ** 2, 3))
            self.lib().oracle_object_setup(self.h, idx, P(box), P(cen), P(ms), ctypes.byref(n), P(xyz), P(sag), P(nrm))
            out.update(coarse_xyz=xyz, sagitta=sag, cell_normal=nrm)
        return out

    def bvh_nodes(self):
        nn = self.info()["n_nodes"]
        boxes = np.zeros((nn, 6)); links = np.zeros((nn, 4), np.int32); leaf = np.zeros(self.n_objects, np.int32)
        self.lib().oracle_bvh_nodes(self.h, P(boxes), P(links), P(leaf))
        return boxes, links, leaf

    def intersect(self, origins, dirs, mode=C.QUERY_BVH, obj=0):
        o = np.ascontiguousarray(origins, dtype=np.float64); d = np.ascontiguousarray(dirs, dtype=np.float64)
        out = np.zeros(o.shape[0], dtype=C.HIT_DTYPE)
        self.lib().oracle_intersect(self.h, o.shape[0], P(o), P(d), mode, obj, P(out))
        return out

    def trace(self, origins, dirs, max_bounces, K=8, nthreads=0):
        o = np.ascontiguousarray(origins, dtype=np.float64); d = np.ascontiguousarray(dirs, dtype=np.float64)
        n = o.shape[0]
        r = _alloc_trace(n, K)
        st = C.TraceStats(); sec = np.zeros(1)
        self.lib().oracle_trace(self.h, n, P(o), P(d), max_bounces, nthreads,
                                ctypes.byref(trace_out_struct(r, K)), ctypes.byref(st), P(sec))
        r["seconds"] = float(sec[0]); r["stats"] = st.as_dict()
        return r

    def plane_counts(self, sources, direction, max_bounces, count_direct_hit=False):
        s = np.ascontiguousarray(sources, dtype=np.float64); d = np.ascontiguousarray(direction, dtype=np.float64)
        c = np.zeros(self.n_objects, np.int64)
        self.lib().oracle_plane_counts(self.h, s.shape[0], P(s), P(d), max_bounces, int(count_direct_hit), P(c))
        return c

    @classmethod
    def sample_grid(cls, patch, n):
        t = C.ObjectTable([patch])
        xyz = np.zeros((n * n, 3)); nrm = np.zeros((n * n, 3)); du = np.zeros((n * n, 3))
        cls.lib().oracle_sample_grid(t.pdescs, n, P(xyz), P(nrm), P(du))
        return xyz, nrm, du

    def bounce_map(self, sample_patches, grid_n, theta_n, phi_n, cone_deg, max_bounces):
        t = C.ObjectTable(sample_patches)
        m = len(sample_patches) * grid_n * grid_n
        mb = np.zeros(m, np.int32); er = np.zeros(m, np.int32); bd = np.zeros(m, np.int32)
        self.lib().oracle_bounce_map(self.h, t.pdescs, len(sample_patches), grid_n, theta_n, phi_n,
                                     cone_deg, max_bounces, P(mb), P(er), P(bd))
        return mb, er, bd

    def bounce_map_rays(self, sample_patches, grid_n, theta_n, phi_n, cone_deg):
        """Every launch ray of bounce_map, ray r at ((p*grid_n**2 + k)*theta_n + ti)*phi_n + pj."""
        t = C.ObjectTable(sample_patches)
        n = len(sample_patches) * grid_n * grid_n * theta_n * phi_n
        o = np.zeros((n, 3)); d = np.zeros((n, 3))
        self.lib().oracle_bounce_map_rays(self.h, t.pdescs, len(sample_patches), grid_n, theta_n, phi_n,
                                          cone_deg, P(o), P(d))
        return o, d


class Reference:
    """The reference's own code (oracle/_ref/libbbrt_ref.so) on a patch directory."""

    _lib = None

    @classmethod
    def lib(cls):
        if cls._lib is None:
            if not os.path.exists(REF_SO):
                raise RuntimeError("reference oracle not built (oracle/build_ref.sh needs the reference sources)")
            L = ctypes.CDLL(REF_SO)
            V = ctypes.c_void_p
            L.ref_last_error.restype = ctypes.c_char_p
            L.ref_set_constants.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double]
            L.ref_open.restype = V
            L.ref_open.argtypes = [ctypes.c_char_p]
            L.ref_close.argtypes = [V]
            L.ref_info.argtypes = [V, V, V, V]
            L.ref_zone_id.restype = ctypes.c_longlong
            L.ref_zone_id.argtypes = [V, ctypes.c_int]
            L.ref_patch_setup.argtypes = [V, ctypes.c_int, V, V, V, V, V, V, V]
            L.ref_trace.argtypes = [V, ctypes.c_longlong, V, V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    V, V, V, V, V, V, V, V]
            L.ref_intersect.argtypes = [V, ctypes.c_longlong, V, V, V, V, V, V, V]
            L.ref_plane_source.argtypes = [ctypes.c_char_p, V, V, V, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, ctypes.c_int, V, V]
            L.ref_bounce_map.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_int, V, V, V]
            L.ref_triangle_queries.argtypes = [ctypes.c_int, V, ctypes.c_int, ctypes.c_longlong, V, V, V, V, V, V]
            cls._lib = L
        return cls._lib

    def __init__(self, directory: str, coarse_n: int = 100, newton_tol: float = 1e-3, newton_max_iters: int = 20):
        L = self.lib()
        L.ref_set_constants(coarse_n, newton_max_iters, newton_tol)
        self.directory = directory
        self.h = L.ref_open(directory.encode())
        if not self.h:
            raise RuntimeError(L.ref_last_error().decode())
        n = ctypes.c_longlong(); d = ctypes.c_double(); s = ctypes.c_double()
        L.ref_info(self.h, ctypes.byref(n), ctypes.byref(d), ctypes.byref(s))
        self.n_objects, self.scene_diagonal, self.max_patch_sagitta = n.value, d.value, s.value

    @classmethod
    def from_patches(cls, patches, tmpdir=None, **kw):
        d = tmpdir or tempfile.mkdtemp(prefix="bbrt_ref_")
        scenes.write_scene_dir(d, patches)
        return cls(d, **kw)

    def close(self):
        if self.h:
            self.lib().ref_close(self.h)
            self.h = None

    __del__ = close

    def patch_setup(self, idx):
        box = np.zeros(6); cen = np.zeros(3); ms = np.zeros(1); n = ctypes.c_int()
        self.lib().ref_patch_setup(self.h, idx, P(box), P(cen), P(ms), ctypes.byref(n), None, None, None)
        g = n.value
        xyz = np.zeros((g * g, 3)); sag = np.zeros((g - 1) ** 2); nrm = np.zeros(((g - 1) ** 2, 3))
        self.lib().ref_patch_setup(self.h, idx, P(box), P(cen), P(ms), ctypes.byref(n), P(xyz), P(sag), P(nrm))
        return dict(box=box, centroid=cen, max_sagitta=float(ms[0]), n=g, coarse_xyz=xyz, sagitta=sag, cell_normal=nrm)

    def trace(self, origins, dirs, max_bounces, K=8, nthreads=0):
        o = np.ascontiguousarray(origins, dtype=np.float64); d = np.ascontiguousarray(dirs, dtype=np.float64)
        n = o.shape[0]
        r = _alloc_trace(n, K)
        ez = np.zeros(n, np.int64); sec = np.zeros(1)
        self.lib().ref_trace(self.h, n, P(o), P(d), max_bounces, nthreads, K, P(r["status"]), P(r["bounce_count"]),
                             P(r["exit_dir"]), P(r["end_point"]), P(r["hit_object"]), P(r["hit_point"]), P(ez), P(sec))
        r["err_zone"] = ez
        r["seconds"] = float(sec[0])
        return r

    def intersect(self, origins, dirs):
        o = np.ascontiguousarray(origins, dtype=np.float64); d = np.ascontiguousarray(dirs, dtype=np.float64)
        n = o.shape[0]
        t = np.zeros(n); pt = np.zeros((n, 3)); nr = np.zeros((n, 3)); ob = np.zeros(n, np.int32); st = np.zeros(n, np.int32)
        self.lib().ref_intersect(self.h, n, P(o), P(d), P(t), P(pt), P(nr), P(ob), P(st))
        return dict(t=t, point=pt, normal=nr, object=ob, status=st)

    def plane_source(self, c0, c1, direction, nx, ny, max_bounces, count_direct_hit=False, nthreads=0):
        c0 = np.asarray(c0, np.float64); c1 = np.asarray(c1, np.float64); d = np.asarray(direction, np.float64)
        counts = np.zeros(self.n_objects, np.int64); sec = np.zeros(1)
        rc = self.lib().ref_plane_source(self.directory.encode(), P(c0), P(c1), P(d), nx, ny, max_bounces,
                                         int(count_direct_hit), nthreads, P(counts), P(sec))
        if rc != 0:
            raise RuntimeError(self.lib().ref_last_error().decode())
        return counts, float(sec[0])

    @classmethod
    def bounce_map(cls, directory, prefix, first, last, grid_n, theta_n, phi_n, cone_deg, max_bounces, nthreads=0):
        m = (last - first + 1) * grid_n * grid_n
        mb = np.zeros(m, np.int32); er = np.zeros(m, np.int32); sec = np.zeros(1)
        rc = cls.lib().ref_bounce_map(directory.encode(), prefix.encode(), first, last, grid_n, theta_n, phi_n,
                                      cone_deg, max_bounces, nthreads, P(mb), P(er), P(sec))
        if rc != 0:
            raise RuntimeError(cls.lib().ref_last_error().decode())
        return mb, er, float(sec[0])

    @classmethod
    def triangle_queries(cls, tris, leaf_threshold, origins, dirs):
        t = np.ascontiguousarray(tris, dtype=np.float64)
        o = np.ascontiguousarray(origins, dtype=np.float64); d = np.ascontiguousarray(dirs, dtype=np.float64)
        n = o.shape[0]
        bt = np.zeros(n); bo = np.zeros(n, np.int32); ft = np.zeros(n); fo = np.zeros(n, np.int32)
        cls.lib().ref_triangle_queries(t.shape[0], P(t), leaf_threshold, n, P(o), P(d), P(bt), P(bo), P(ft), P(fo))
        return bt, bo, ft, fo
