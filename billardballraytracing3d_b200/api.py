"""Python face of the C ABI (include/bbrt.h) for tests, benchmarks and scripts.

Every method is one C-ABI call into libbbrt_cuda.so; nothing here computes a
trace result itself.  The C++ classes under include/bbrt/ are the drop-in
mirror of the reference's RayTracingDriver / BVH / PlaneSourceDriver /
BounceMapDriver API; this module is the same boundary seen from Python.
"""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Sequence

import numpy as np

from . import _capi as C

P = lambda a: None if a is None else ctypes.c_void_p(a.ctypes.data)  # noqa: E731


class TraceResult(dict):
    """Per-ray arrays keyed like bbrt_trace_out, plus 'stats'."""


class Scene:
    """One bbrt scene (device arrays + stream).  Build from patches
    (scenes.Patch), triangles (9 floats each), or a patch directory."""

    def __init__(self, patches: Sequence = (), triangles: Sequence = (), config: C.Config = None,
                 directory: str = None, _handle=None, table: C.ObjectTable = None):
        self.lib = C.load_library()
        self.config = config if config is not None else C.default_config()
        h = ctypes.c_void_p()
        if _handle is not None:
            h = _handle
        elif directory is not None:
            C.check(self.lib, self.lib.bbrt_scene_create_from_dir(directory.encode(), ctypes.byref(self.config),
                                                                   ctypes.byref(h)), "bbrt_scene_create_from_dir")
        else:
            # `table`: descriptors already built (another scene's), reused as they are
            self.table = table if table is not None else C.ObjectTable(patches, triangles)
            C.check(self.lib, self.lib.bbrt_scene_create(self.table.descs, self.table.n, ctypes.byref(self.config),
                                                         ctypes.byref(h)), "bbrt_scene_create")
        self.h = h
        inf = self.info()
        self.n_objects = inf["n_objects"]

    @classmethod
    def from_range(cls, directory: str, prefix: str, first: int, last: int, config: C.Config = None):
        lib = C.load_library()
        cfg = config if config is not None else C.default_config()
        h = ctypes.c_void_p()
        C.check(lib, lib.bbrt_scene_create_from_range(directory.encode(), prefix.encode(), first, last,
                                                      ctypes.byref(cfg), ctypes.byref(h)), "bbrt_scene_create_from_range")
        return cls(config=cfg, _handle=h)

    def close(self):
        if getattr(self, "h", None):
            self.lib.bbrt_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- host-side queries (no GPU needed) ---------------------------------
    def info(self) -> Dict:
        s = C.SceneInfo()
        C.check(self.lib, self.lib.bbrt_scene_info_get(self.h, ctypes.byref(s)), "bbrt_scene_info_get")
        return {k: getattr(s, k) for k, _ in s._fields_}

    def object_info(self, k: int) -> Dict:
        o = C.ObjectInfo()
        C.check(self.lib, self.lib.bbrt_object_info_get(self.h, k, ctypes.byref(o)), "bbrt_object_info_get")
        return dict(kind=o.kind, zone_id=o.zone_id, box=np.array(list(o.box_min) + list(o.box_max)),
                    centroid=np.array(list(o.centroid)), padding=o.padding)

    def coarse_grid(self, k: int) -> Dict:
        n = ctypes.c_int()
        C.check(self.lib, self.lib.bbrt_patch_coarse_grid(self.h, k, ctypes.byref(n), None, None, None, None, None),
                "bbrt_patch_coarse_grid")
        g = n.value
        u = np.zeros(g); v = np.zeros(g); xyz = np.zeros((g * g, 3))
        sag = np.zeros((g - 1) ** 2); nrm = np.zeros(((g - 1) ** 2, 3))
        C.check(self.lib, self.lib.bbrt_patch_coarse_grid(self.h, k, ctypes.byref(n), C.ptr(u), C.ptr(v), C.ptr(xyz),
                                                          C.ptr(sag), C.ptr(nrm)), "bbrt_patch_coarse_grid")
        return dict(n=g, u=u, v=v, coarse_xyz=xyz, sagitta=sag, cell_normal=nrm)

    def self_intersect_epsilon(self, k: int = -1) -> float:
        e = ctypes.c_double()
        C.check(self.lib, self.lib.bbrt_self_intersect_epsilon(self.h, k, ctypes.byref(e)), "bbrt_self_intersect_epsilon")
        return e.value

    # ---- GPU calls ------------------------------------------------------------
    def upload(self):
        C.check(self.lib, self.lib.bbrt_scene_upload(self.h), "bbrt_scene_upload")

    def intersect(self, origins, dirs, mode: int = C.QUERY_BVH, obj: int = 0) -> np.ndarray:
        o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        out = np.zeros(o.shape[0], dtype=C.HIT_DTYPE)
        C.check(self.lib, self.lib.bbrt_intersect(self.h, P(o), P(d), o.shape[0], mode, obj, 0, P(out), None),
                "bbrt_intersect")
        return out

    def setup_arrays(self) -> Dict[str, np.ndarray]:
        """The scene's whole set-up (bbrt_scene_setup_get): coarse grids, cell
        normals / sagittas, cull cell and block boxes, cull constants."""
        out = {}
        for name, what, dt in (("coarse", C.SETUP_COARSE, np.float64), ("cells", C.SETUP_CELLS, np.float64),
                               ("cell_boxes", C.SETUP_CELL_BOXES, np.float32),
                               ("block_boxes", C.SETUP_BLOCK_BOXES, np.float32), ("cull", C.SETUP_CULL, np.float64)):
            n = ctypes.c_longlong()
            C.check(self.lib, self.lib.bbrt_scene_setup_get(self.h, what, None, ctypes.byref(n)), "bbrt_scene_setup_get")
            a = np.zeros(n.value, dt)
            C.check(self.lib, self.lib.bbrt_scene_setup_get(self.h, what, ctypes.c_void_p(a.ctypes.data), ctypes.byref(n)),
                    "bbrt_scene_setup_get")
            out[name] = a
        return out

    def trace(self, origins, dirs, max_bounces: int, record: int = 8, want_stats: bool = True,
              outputs: Sequence[str] = ("status", "bounce_count", "exit_dir", "end_point", "hit_object",
                                        "hit_point", "hit_uv", "err_object", "err_value")) -> TraceResult:
        o = np.ascontiguousarray(origins, dtype=np.float64).reshape(-1, 3)
        d = np.ascontiguousarray(dirs, dtype=np.float64).reshape(-1, 3)
        n = o.shape[0]
        K = record
        shapes = dict(status=((n,), np.int32), bounce_count=((n,), np.int32), exit_dir=((n, 3), np.float64),
                      end_point=((n, 3), np.float64), hit_object=((n, K), np.int32),
                      hit_point=((n, K, 3), np.float64), hit_uv=((n, K, 2), np.float64),
                      err_object=((n,), np.int32), err_value=((n, 2), np.float64),
                      ray_work=((n, 4), np.int64))
        r = TraceResult()
        for k in outputs:
            shp, dt = shapes[k]
            r[k] = np.zeros(shp, dt)
        out = C.TraceOut()
        out.record_bounces = K
        for k in shapes:
            ct = {np.int32: ctypes.c_int, np.int64: ctypes.c_longlong}.get(shapes[k][1], ctypes.c_double)
            setattr(out, k, C.ptr(r.get(k), ct))
        st = C.TraceStats()
        C.check(self.lib, self.lib.bbrt_trace(self.h, P(o), P(d), n, max_bounces, 0, ctypes.byref(out),
                                              ctypes.byref(st) if want_stats else None, None), "bbrt_trace")
        if want_stats:
            r["stats"] = st.as_dict()
        return r

    def trace_device(self, origins_ptr: int, dirs_ptr: int, n: int, max_bounces: int, out_ptrs: Dict[str, int],
                     record: int = 0, stream: int = 0, want_stats: bool = False,
                     times_only: bool = False) -> Optional[Dict]:
        """bbrt_trace on device pointers (e.g. torch tensors' data_ptr()); with
        times_only the statistics hold the device times only (BBRT_TIMES_ONLY)."""
        out = C.TraceOut()
        out.record_bounces = record
        for k, v in out_ptrs.items():
            ct = ctypes.c_int if k in ("status", "bounce_count", "hit_object", "err_object") else ctypes.c_double
            setattr(out, k, ctypes.cast(ctypes.c_void_p(v), ctypes.POINTER(ct)))
        st = C.TraceStats()
        C.check(self.lib, self.lib.bbrt_trace(self.h, ctypes.c_void_p(origins_ptr), ctypes.c_void_p(dirs_ptr), n,
                                              max_bounces, C.DEVICE_PTRS | (C.TIMES_ONLY if times_only else 0),
                                              ctypes.byref(out),
                                              ctypes.byref(st) if want_stats else None,
                                              ctypes.c_void_p(stream) if stream else None), "bbrt_trace")
        return st.as_dict() if want_stats else None

    def plane_source(self, corner0, corner1, direction, nx: int, ny: int, max_bounces: int,
                     count_direct_hit: bool = False, want_stats: bool = False):
        c0 = np.ascontiguousarray(corner0, dtype=np.float64)
        c1 = np.ascontiguousarray(corner1, dtype=np.float64)
        dd = np.ascontiguousarray(direction, dtype=np.float64)
        counts = np.zeros(self.n_objects, np.int64)
        st = C.TraceStats()
        C.check(self.lib, self.lib.bbrt_plane_source(self.h, C.ptr(c0), C.ptr(c1), C.ptr(dd), nx, ny, max_bounces,
                                                     int(count_direct_hit), C.ptr(counts, ctypes.c_longlong),
                                                     ctypes.byref(st) if want_stats else None, None),
                "bbrt_plane_source")
        return (counts, st.as_dict()) if want_stats else counts

    def bounce_map(self, sample_patches: Sequence, grid_n: int, theta_n: int, phi_n: int,
                   cone_angle_deg: float = 180.0, max_bounces: int = 50):
        t = C.ObjectTable(sample_patches)
        m = len(sample_patches) * grid_n * grid_n
        mb = np.zeros(m, np.int32); er = np.zeros(m, np.int32); bd = np.zeros(m, np.int32)
        C.check(self.lib, self.lib.bbrt_bounce_map(self.h, t.pdescs, len(sample_patches), grid_n, theta_n, phi_n,
                                                   float(cone_angle_deg), max_bounces, C.ptr(mb, ctypes.c_int),
                                                   C.ptr(er, ctypes.c_int), C.ptr(bd, ctypes.c_int), None, None),
                "bbrt_bounce_map")
        return mb, er, bd

    def set_modes(self, precision: int = C.PREC_FP64, guess: int = C.GUESS_TRIANGLE):
        """Arithmetic mode (PREC_FP64 / PREC_SPLIT) and Newton start (GUESS_TRIANGLE / GUESS_LEARNED)."""
        C.check(self.lib, self.lib.bbrt_scene_set_modes(self.h, int(precision), int(guess)), "bbrt_scene_set_modes")

    def tuning(self, **set_fields) -> Dict:
        """The scene's launch schedule; keyword arguments change fields of it first."""
        t = C.Tuning()
        C.check(self.lib, self.lib.bbrt_scene_get_tuning(self.h, ctypes.byref(t)), "bbrt_scene_get_tuning")
        if set_fields:
            for k, v in set_fields.items():
                if not hasattr(t, k):
                    raise KeyError(k)
                setattr(t, k, v)
            C.check(self.lib, self.lib.bbrt_scene_set_tuning(self.h, ctypes.byref(t)), "bbrt_scene_set_tuning")
        return t.as_dict()

    def autotune(self, origins, dirs, max_bounces: int, trials: int = 2) -> Dict:
        """Picks the fastest launch schedule on these rays; returns it with its time."""
        o = np.ascontiguousarray(origins, dtype=np.float64)
        d = np.ascontiguousarray(dirs, dtype=np.float64)
        t = C.Tuning()
        ms = ctypes.c_double()
        C.check(self.lib, self.lib.bbrt_scene_autotune(self.h, C.ptr(o), C.ptr(d), o.shape[0], int(max_bounces),
                                                       int(trials), ctypes.byref(t), ctypes.byref(ms), None),
                "bbrt_scene_autotune")
        return dict(t.as_dict(), ms=ms.value)

    def guess_train(self, origins, dirs, max_bounces: int, **kw) -> Dict:
        """Records training samples from a plain trace of these rays and trains
        the learned-guess network on the GPU; returns the training report."""
        cfg = C.GuessTrainConfig()
        self.lib.bbrt_guess_train_config_init(ctypes.byref(cfg))
        for k, v in kw.items():
            if not hasattr(cfg, k):
                raise KeyError(k)
            setattr(cfg, k, v)
        o = np.ascontiguousarray(origins, dtype=np.float64)
        d = np.ascontiguousarray(dirs, dtype=np.float64)
        rep = C.GuessTrainReport()
        C.check(self.lib, self.lib.bbrt_guess_train(self.h, C.ptr(o), C.ptr(d), o.shape[0], int(max_bounces),
                                                    ctypes.byref(cfg), ctypes.byref(rep), None), "bbrt_guess_train")
        return rep.as_dict()

    def guess_params(self, params=None):
        """Gets (params=None) or sets the network's FP32 parameters."""
        n = self.lib.bbrt_guess_param_count(self.h)
        if params is None:
            out = np.zeros(n, np.float32)
            C.check(self.lib, self.lib.bbrt_guess_params(self.h, C.ptr(out, ctypes.c_float), n, 0), "bbrt_guess_params")
            return out
        p = np.ascontiguousarray(params, dtype=np.float32)
        C.check(self.lib, self.lib.bbrt_guess_params(self.h, C.ptr(p, ctypes.c_float), n, 1), "bbrt_guess_params")
        return p

    def bounce_map_rays(self, sample_patches: Sequence, grid_n: int, theta_n: int, phi_n: int,
                        cone_angle_deg: float = 180.0, ray_index=None):
        """The launch rays bounce_map traces, as (origins[n,3], dirs[n,3]).

        Ray r = ((p * grid_n**2 + k) * theta_n + ti) * phi_n + pj; ray_index
        picks some (default: all, in that order)."""
        t = C.ObjectTable(sample_patches)
        if ray_index is None:
            n = len(sample_patches) * grid_n * grid_n * theta_n * phi_n
            idx_p = None
        else:
            idx = np.ascontiguousarray(ray_index, dtype=np.int64)
            n = idx.size
            idx_p = C.ptr(idx, ctypes.c_longlong)
        o = np.zeros((n, 3)); d = np.zeros((n, 3))
        C.check(self.lib, self.lib.bbrt_bounce_map_rays(self.h, t.pdescs, len(sample_patches), grid_n, theta_n, phi_n,
                                                        float(cone_angle_deg), idx_p, n, C.ptr(o), C.ptr(d)),
                "bbrt_bounce_map_rays")
        return o, d


def trace_batch_device(scenes: Sequence["Scene"], origin_ptrs, dir_ptrs, ns, max_bounces: int, outs=None,
                       want_stats: bool = True):
    """bbrt_trace_batch: every scene's rays (device pointers, e.g. torch
    tensors' data_ptr()) traced with all scenes in flight together.
    outs: per scene a dict of device pointers (status, bounce_count, exit_dir,
    hit_object, hit_point with 'record'), or None.  Returns (stats, batch_ms)."""
    lib = C.load_library()
    k = len(scenes)
    hs = (ctypes.c_void_p * k)(*[s.h for s in scenes])
    op = (ctypes.c_void_p * k)(*[ctypes.c_void_p(p) for p in origin_ptrs])
    dp = (ctypes.c_void_p * k)(*[ctypes.c_void_p(p) for p in dir_ptrs])
    nn = (ctypes.c_longlong * k)(*[int(v) for v in ns])
    to = None
    if outs is not None:
        to = (C.TraceOut * k)()
        for j, od in enumerate(outs):
            if not od:
                continue
            to[j].record_bounces = int(od.get("record", 0))
            for key, v in od.items():
                if key == "record":
                    continue
                ct = ctypes.c_int if key in ("status", "bounce_count", "hit_object", "err_object") else ctypes.c_double
                setattr(to[j], key, ctypes.cast(ctypes.c_void_p(v), ctypes.POINTER(ct)))
    st = C.TraceStats()
    ms = ctypes.c_double()
    C.check(lib, lib.bbrt_trace_batch(hs, k, op, dp, nn, int(max_bounces), to, ctypes.byref(st) if want_stats else None,
                                      ctypes.byref(ms)), "bbrt_trace_batch")
    return (st.as_dict() if want_stats else None), ms.value


def _trace_outs(outs, k):
    """Per-scene dicts of device pointers (+ 'record') as a bbrt_trace_out array."""
    if outs is None:
        return None
    to = (C.TraceOut * k)()
    for j, od in enumerate(outs):
        if not od:
            continue
        to[j].record_bounces = int(od.get("record", 0))
        for key, v in od.items():
            if key == "record":
                continue
            ct = {"status": ctypes.c_int, "bounce_count": ctypes.c_int, "hit_object": ctypes.c_int,
                  "err_object": ctypes.c_int, "ray_work": ctypes.c_longlong}.get(key, ctypes.c_double)
            setattr(to[j], key, ctypes.cast(ctypes.c_void_p(v), ctypes.POINTER(ct)))
    return to


class SceneSet:
    """bbrt_scene_set: several scenes traced as one wavefront (one launch
    sequence for all members); results per member, in its own numbering."""

    def __init__(self, scenes: Sequence["Scene"]):
        self.lib = C.load_library()
        self.k = len(scenes)
        hs = (ctypes.c_void_p * self.k)(*[s.h for s in scenes])
        h = ctypes.c_void_p()
        C.check(self.lib, self.lib.bbrt_scene_set_create(hs, self.k, ctypes.byref(h)), "bbrt_scene_set_create")
        self.h = h

    def configure(self, precision: int = C.PREC_FP64, guess: int = C.GUESS_TRIANGLE, **tuning):
        t = None
        if tuning:
            t = C.Tuning()
            for k, v in tuning.items():
                setattr(t, k, v)
        C.check(self.lib, self.lib.bbrt_scene_set_configure(self.h, int(precision), int(guess),
                                                            ctypes.byref(t) if t else None), "bbrt_scene_set_configure")

    def guess_train(self, origins, dirs, max_bounces: int, **kw) -> Dict:
        """One network for every member (host ray arrays per member), trained on the GPU."""
        os_ = [np.ascontiguousarray(o, dtype=np.float64).reshape(-1, 3) for o in origins]
        ds_ = [np.ascontiguousarray(d, dtype=np.float64).reshape(-1, 3) for d in dirs]
        k = self.k
        op = (ctypes.c_void_p * k)(*[ctypes.c_void_p(a.ctypes.data) for a in os_])
        dp = (ctypes.c_void_p * k)(*[ctypes.c_void_p(a.ctypes.data) for a in ds_])
        nn = (ctypes.c_longlong * k)(*[a.shape[0] for a in os_])
        cfg = C.GuessTrainConfig()
        self.lib.bbrt_guess_train_config_init(ctypes.byref(cfg))
        for key, v in kw.items():
            setattr(cfg, key, v)
        rep = C.GuessTrainReport()
        C.check(self.lib, self.lib.bbrt_scene_set_guess_train(self.h, op, dp, nn, int(max_bounces), ctypes.byref(cfg),
                                                              ctypes.byref(rep)), "bbrt_scene_set_guess_train")
        return {key: getattr(rep, key) for key, _ in rep._fields_}

    def guess_export(self, member: int, scene: "Scene"):
        """Member `member`'s share of the set's network into `scene`."""
        C.check(self.lib, self.lib.bbrt_scene_set_guess_export(self.h, int(member), scene.h),
                "bbrt_scene_set_guess_export")

    def trace_device(self, origin_ptrs, dir_ptrs, ns, max_bounces: int, outs=None, want_stats: bool = True,
                     stream: int = 0):
        """Every member's rays (device pointers) in one trace; returns (stats, set_ms)."""
        k = self.k
        op = (ctypes.c_void_p * k)(*[ctypes.c_void_p(p) for p in origin_ptrs])
        dp = (ctypes.c_void_p * k)(*[ctypes.c_void_p(p) for p in dir_ptrs])
        nn = (ctypes.c_longlong * k)(*[int(v) for v in ns])
        st = C.TraceStats()
        ms = ctypes.c_double()
        C.check(self.lib, self.lib.bbrt_trace_set(self.h, op, dp, nn, int(max_bounces), _trace_outs(outs, k),
                                                  ctypes.byref(st) if want_stats else None, ctypes.byref(ms),
                                                  ctypes.c_void_p(stream) if stream else None), "bbrt_trace_set")
        return (st.as_dict() if want_stats else None), ms.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.bbrt_scene_set_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def sample_grid(patch, n: int):
    """SurfacePatch::sample_grid(n) through the C ABI: (xyz, normal, dX/du)."""
    lib = C.load_library()
    t = C.ObjectTable([patch])
    xyz = np.zeros((n * n, 3)); nrm = np.zeros((n * n, 3)); du = np.zeros((n * n, 3))
    C.check(lib, lib.bbrt_patch_sample_grid(t.pdescs, n, C.ptr(xyz), C.ptr(nrm), C.ptr(du)), "bbrt_patch_sample_grid")
    return xyz, nrm, du


def read_patch_file(path: str) -> Dict:
    """SurfacePatch::load_patch_file through the C ABI; returns numpy copies."""
    lib = C.load_library()
    f = C.PatchFile()
    C.check(lib, lib.bbrt_patch_file_read(path.encode(), ctypes.byref(f)), "bbrt_patch_file_read")
    try:
        d = f.desc
        n = d.imax * d.jmax * d.kmax
        arr = lambda p, m: np.ctypeslib.as_array(p, shape=(m,)).copy()  # noqa: E731
        out = dict(imax=d.imax, jmax=d.jmax, kmax=d.kmax, zone_id=d.zone_id,
                   u_nodes=arr(d.u_nodes, d.imax), v_nodes=arr(d.v_nodes, d.jmax),
                   mask=arr(f.mask, n), dS=arr(f.dS, n), edge_flags=list(f.edge_flags))
        for k in ("x", "y", "z", "dxdu", "dydu", "dzdu", "dxdv", "dydv", "dzdv", "nu_x", "nu_y", "nu_z"):
            out[k] = arr(getattr(d, k), n)
        return out
    finally:
        lib.bbrt_patch_file_free(ctypes.byref(f))


def trace_recording_all(scene: "Scene", origins, dirs, max_bounces: int, first_record: int = 16) -> TraceResult:
    """scene.trace with every bounce of every ray recorded: traces with
    `first_record` recorded bounces and, when some ray bounced more often,
    again with the largest bounce count."""
    r = scene.trace(origins, dirs, max_bounces, record=first_record)
    k = int(r["bounce_count"].max()) if r["bounce_count"].size else 0
    if k > first_record:
        r = scene.trace(origins, dirs, max_bounces, record=k)
    return r


def min_incidence_cos(origins, r: TraceResult) -> np.ndarray:
    """Per ray, the smallest incidence cosine over its recorded bounces,
    recomputed from the path alone: the ray arrives along d_in and leaves
    along d_out = d_in - 2 (d_in . n) n, so |d_in . n| = sqrt((1 - d_in . d_out) / 2).
    The leg after the last hit is exit_dir; rays without a hit get 1."""
    o = np.asarray(origins, dtype=np.float64).reshape(-1, 3)
    b = r["bounce_count"]
    n, K = r["hit_point"].shape[:2]
    pts = np.concatenate([o[:, None, :], r["hit_point"]], axis=1)            # [n, K+1, 3]
    legs = np.diff(pts, axis=1)                                                # leg k ends at hit k
    legs /= np.maximum(np.linalg.norm(legs, axis=2, keepdims=True), 1e-300)
    out_legs = np.concatenate([legs[:, 1:], np.zeros((n, 1, 3))], axis=1)
    last = np.clip(b - 1, 0, max(K - 1, 0))
    out_legs[np.arange(n), last] = r["exit_dir"]
    cos2 = np.clip((1.0 - np.sum(legs * out_legs, axis=2)) * 0.5, 0.0, 1.0)
    cos = np.sqrt(cos2)
    mask = np.arange(K)[None, :] < np.minimum(b, K)[:, None]
    return np.where(mask, cos, 1.0).min(axis=1) if K else np.ones(n)


def compare_traces(ref: TraceResult, other: TraceResult, origins=None, bound: float = 1e-10,
                   grazing_cos: float = 1e-3) -> Dict:
    """Ray-by-ray agreement of two traces of the same rays, both recorded
    with every bounce (trace_recording_all): the share of rays with the same
    status, bounce count and hit-object sequence, and over those rays the
    largest difference of any recorded hit point, of its patch parameters
    (u, v) and of the exit direction — the quantities held to `bound`.  The
    end point is reported beside them: for an escaped ray it is the tail
    point last hit + scene diagonal * exit direction, so its difference is
    the exit direction's scaled by the scene's size.

    With `origins`, rays whose incidence cosine (in `ref`) falls to
    `grazing_cos` or below at some bounce are set apart, as the accuracy bar
    sets them apart: the bound is held over the other agreeing rays, and the
    maxima over all agreeing rays are reported beside it."""
    K = ref["hit_object"].shape[1]
    if int(ref["bounce_count"].max(initial=0)) > K or int(other["bounce_count"].max(initial=0)) > other["hit_object"].shape[1]:
        raise ValueError("compare_traces: a trace did not record every bounce")
    if other["hit_object"].shape[1] != K:
        raise ValueError("compare_traces: the traces recorded different bounce counts")
    n = ref["status"].size
    same = (ref["status"] == other["status"]) & (ref["bounce_count"] == other["bounce_count"])
    same &= np.all(ref["hit_object"] == other["hit_object"], axis=1)
    mask = np.arange(K)[None, :] < np.minimum(ref["bounce_count"], K)[:, None]
    # per-ray maxima
    hit = np.where(mask, np.abs(ref["hit_point"] - other["hit_point"]).max(axis=2), 0.0).max(axis=1, initial=0.0) \
        if K else np.zeros(n)
    uv = np.zeros(n)
    if "hit_uv" in ref and "hit_uv" in other and K:
        uv = np.where(mask, np.abs(ref["hit_uv"] - other["hit_uv"]).max(axis=2), 0.0).max(axis=1, initial=0.0)
    ext = np.abs(ref["exit_dir"] - other["exit_dir"]).max(axis=1)
    end = np.abs(ref["end_point"] - other["end_point"]).max(axis=1)

    def mx(v, sel):
        return float(np.max(np.where(sel, v, 0.0), initial=0.0))

    out = {"rays": int(n), "sequence_agreement": float(np.mean(same)) if n else 1.0,
           "max_hit_err_agreeing": mx(hit, same), "max_uv_err_agreeing": mx(uv, same),
           "max_exit_dir_err_agreeing": mx(ext, same), "max_end_point_err_agreeing": mx(end, same),
           "bounces_compared": int(mask.sum()), "hit_err_bound": bound}
    held = same
    if origins is not None:
        cos = min_incidence_cos(origins, ref)
        ok = cos > grazing_cos
        held = same & ok
        out["grazing_cos"] = grazing_cos
        out["non_grazing_rays"] = int(ok.sum())
        out["sequence_agreement_non_grazing"] = float(np.mean(same[ok])) if ok.any() else 1.0
        out["max_hit_err_non_grazing"] = mx(hit, held)
        out["max_uv_err_non_grazing"] = mx(uv, held)
        out["max_exit_dir_err_non_grazing"] = mx(ext, held)
        if same.any():
            w = int(np.argmax(np.where(same, np.maximum(hit, np.maximum(uv, ext)), -1.0)))
            out["largest_err_ray_min_incidence_cos"] = float(cos[w])
    worst = np.maximum(hit, np.maximum(uv, ext))
    out["within_bound"] = bool(mx(worst, held) <= bound)
    # a ray agrees within the bound when its sequence agrees and every
    # recorded hit point, (u, v) and its exit direction are within `bound`
    # (differences of a few ulp at the first bounce grow by about twice the
    # obstacle spacing over the radius per bounce, so a long chain can leave
    # the bound although every bounce took the same patch)
    base = np.ones(n, bool) if origins is None else (min_incidence_cos(origins, ref) > grazing_cos)
    within = same & (worst <= bound)
    out["agreement_within_bound"] = float(np.mean(within[base])) if base.any() else 1.0
    out["rays_over_bound"] = int(np.sum(held & (worst > bound)))
    return out
