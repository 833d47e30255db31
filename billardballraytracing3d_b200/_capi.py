"""ctypes mirror of include/bbrt.h (the C ABI of libbbrt_cuda.so).

Struct layouts here must match the header field for field; the
`test_capi_layout` CPU test checks the sizes against a C compile of the
header.
"""
from __future__ import annotations

import ctypes
import os
from typing import List, Sequence

import numpy as np

c_double_p = ctypes.POINTER(ctypes.c_double)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_ll_p = ctypes.POINTER(ctypes.c_longlong)
c_float_p = ctypes.POINTER(ctypes.c_float)

# return codes
BBRT_OK = 0
BBRT_ERR_ARG = -1
BBRT_ERR_CUDA = -2
BBRT_ERR_IO = -3
BBRT_ERR_FORMAT = -4
BBRT_ERR_STATE = -5
BBRT_ERR_NOMEM = -6
BBRT_ERR_KERNEL = -7
BBRT_ERR_UNSUPPORTED = -8

# per-ray status
RAY_ESCAPED = 0
RAY_MAX_BOUNCES = 1
RAY_NEWTON_SINGULAR = 2
RAY_NEWTON_NOCONV = 3
RAY_NEWTON_DOMAIN = 4
RAY_WENT_INSIDE = 5
SETUP_COARSE, SETUP_CELLS, SETUP_CELL_BOXES, SETUP_BLOCK_BOXES, SETUP_CULL = 0, 1, 2, 3, 4
RAY_BAD_DIR = 6
RAY_STACK_OVERFLOW = 7
RAY_STATUS_COUNT = 8
STATUS_NAMES = ("escaped", "max_bounces", "newton_singular", "newton_noconv",
                "newton_domain", "went_inside", "bad_dir", "stack_overflow")

OBJ_PATCH = 0
OBJ_TRIANGLE = 1
PREC_FP64 = 0
PREC_SPLIT = 1
GUESS_TRIANGLE = 0
GUESS_LEARNED = 1
QUERY_BVH = 0
QUERY_BRUTE = 1
QUERY_OBJECT = 2
DEVICE_PTRS = 1
TIMES_ONLY = 2
PIPE_FP64 = 0
PIPE_FP32 = 1
PIPE_L2 = 2


class Config(ctypes.Structure):
    _fields_ = [
        ("coarse_grid_n", ctypes.c_int),
        ("newton_max_iters", ctypes.c_int),
        ("newton_tol", ctypes.c_double),
        ("leaf_threshold", ctypes.c_int),
        ("self_intersect_eps_factor", ctypes.c_double),
        ("sagitta_clearance_factor", ctypes.c_double),
        ("backface_tol", ctypes.c_double),
        ("precision", ctypes.c_int),
        ("guess", ctypes.c_int),
        ("cull", ctypes.c_int),
        ("setup_on_device", ctypes.c_int),
    ]


def default_config(**kw) -> Config:
    """The reference's hard-coded constants (SurfacePatch.hpp:117,121-122;
    BVH.hpp:67; RayTracingDriver.hpp:328,337,344), overridable by keyword."""
    c = Config(coarse_grid_n=100, newton_max_iters=20, newton_tol=1e-3, leaf_threshold=4,
               self_intersect_eps_factor=1e-9, sagitta_clearance_factor=5.0, backface_tol=1e-9,
               precision=PREC_FP64, guess=GUESS_TRIANGLE, cull=1, setup_on_device=-1)
    for k, v in kw.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


class PatchDesc(ctypes.Structure):
    _fields_ = [
        ("imax", ctypes.c_int), ("jmax", ctypes.c_int), ("kmax", ctypes.c_int),
        ("zone_id", ctypes.c_longlong),
        ("u_nodes", c_double_p), ("v_nodes", c_double_p),
        ("x", c_double_p), ("y", c_double_p), ("z", c_double_p),
        ("dxdu", c_double_p), ("dydu", c_double_p), ("dzdu", c_double_p),
        ("dxdv", c_double_p), ("dydv", c_double_p), ("dzdv", c_double_p),
        ("nu_x", c_double_p), ("nu_y", c_double_p), ("nu_z", c_double_p),
    ]


class ObjectDesc(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int),
        ("patch", ctypes.POINTER(PatchDesc)),
        ("tri", ctypes.c_double * 9),
    ]


class PatchFile(ctypes.Structure):
    _fields_ = [
        ("desc", PatchDesc),
        ("mask", c_int_p),
        ("dS", c_double_p),
        ("edge_flags", ctypes.c_int * 4),
        ("storage_", ctypes.c_void_p),
    ]


class SceneInfo(ctypes.Structure):
    _fields_ = [
        ("n_objects", ctypes.c_int), ("n_nodes", ctypes.c_int), ("max_depth", ctypes.c_int),
        ("scene_diagonal", ctypes.c_double), ("max_patch_sagitta", ctypes.c_double),
        ("device_bytes", ctypes.c_longlong), ("setup_on_device", ctypes.c_int),
    ]


class ObjectInfo(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int), ("zone_id", ctypes.c_longlong),
        ("box_min", ctypes.c_double * 3), ("box_max", ctypes.c_double * 3),
        ("centroid", ctypes.c_double * 3), ("padding", ctypes.c_double),
    ]


class Hit(ctypes.Structure):
    _fields_ = [
        ("t", ctypes.c_double), ("point", ctypes.c_double * 3), ("normal", ctypes.c_double * 3),
        ("uv", ctypes.c_double * 2), ("object", ctypes.c_int), ("status", ctypes.c_int),
        ("err_object", ctypes.c_int), ("pad_", ctypes.c_int), ("err_value", ctypes.c_double * 2),
    ]


HIT_DTYPE = np.dtype([("t", "f8"), ("point", "f8", 3), ("normal", "f8", 3), ("uv", "f8", 2),
                      ("object", "i4"), ("status", "i4"), ("err_object", "i4"), ("pad_", "i4"),
                      ("err_value", "f8", 2)], align=True)


class TraceOut(ctypes.Structure):
    _fields_ = [
        ("status", c_int_p), ("bounce_count", c_int_p), ("exit_dir", c_double_p),
        ("end_point", c_double_p), ("record_bounces", ctypes.c_int), ("hit_object", c_int_p),
        ("hit_point", c_double_p), ("hit_uv", c_double_p), ("err_object", c_int_p),
        ("err_value", c_double_p), ("ray_work", c_ll_p),
    ]


class TraceStats(ctypes.Structure):
    _fields_ = [
        ("rays", ctypes.c_longlong), ("bounces", ctypes.c_longlong), ("queries", ctypes.c_longlong),
        ("node_tests", ctypes.c_longlong), ("patch_tests", ctypes.c_longlong),
        ("cell_tests", ctypes.c_longlong), ("tri_tests", ctypes.c_longlong),
        ("newton_iters", ctypes.c_longlong), ("newton_iters_fp32", ctypes.c_longlong),
        ("status_hist", ctypes.c_longlong * RAY_STATUS_COUNT),
        ("kernel_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
        ("order_ms", ctypes.c_double), ("advance_ms", ctypes.c_double), ("newton_ms", ctypes.c_double),
        ("tail_ms", ctypes.c_double), ("rounds", ctypes.c_longlong), ("tail_rays", ctypes.c_longlong),
        ("tail_node_tests", ctypes.c_longlong), ("tail_cell_tests", ctypes.c_longlong),
        ("tail_tri_tests", ctypes.c_longlong), ("tail_newton_iters", ctypes.c_longlong),
        ("launches", ctypes.c_longlong),
        ("guess_used", ctypes.c_longlong), ("guess_fallback", ctypes.c_longlong), ("guess_ms", ctypes.c_double),
        ("off_patch", ctypes.c_longlong), ("node_tests_fp64", ctypes.c_longlong),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_ if k != "status_hist"}
        d["status_hist"] = list(self.status_hist)
        return d


class Tuning(ctypes.Structure):
    _fields_ = [
        ("advance_shape", ctypes.c_int), ("warp_stage1", ctypes.c_int), ("order_rays", ctypes.c_int),
        ("warp_tail", ctypes.c_int), ("wave_tail", ctypes.c_longlong), ("wave_min_rays", ctypes.c_longlong),
        ("graph_rounds", ctypes.c_int), ("watchdog_cycles", ctypes.c_longlong),
        ("mma_wait_cycles", ctypes.c_longlong),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GuessTrainConfig(ctypes.Structure):
    _fields_ = [
        ("epochs", ctypes.c_int), ("batch", ctypes.c_int), ("lr", ctypes.c_float),
        ("max_positive", ctypes.c_longlong), ("max_negative", ctypes.c_longlong),
        ("seed", ctypes.c_ulonglong), ("min_logit", ctypes.c_double), ("t_window", ctypes.c_double),
    ]


class GuessTrainReport(ctypes.Structure):
    _fields_ = [
        ("positives", ctypes.c_longlong), ("negatives", ctypes.c_longlong), ("steps", ctypes.c_longlong),
        ("first_loss", ctypes.c_double), ("last_loss", ctypes.c_double),
        ("collect_ms", ctypes.c_double), ("train_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def ptr(a, ctype=ctypes.c_double):
    """ctypes pointer to a numpy array's data (None passes NULL)."""
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class ObjectTable:
    """bbrt_object_desc[] for a list of patches (scenes.Patch) and/or
    triangles (9 floats each), keeping the numpy arrays alive."""

    def __init__(self, patches: Sequence = (), triangles: Sequence = ()):
        self._keep: List = []
        n = len(patches) + len(triangles)
        self.descs = (ObjectDesc * max(n, 1))()
        self.pdescs = (PatchDesc * max(len(patches), 1))()
        self.n = n
        for k, p in enumerate(patches):
            pd = self.pdescs[k]
            pd.imax, pd.jmax, pd.kmax, pd.zone_id = p.imax, p.jmax, p.kmax, int(p.zone_id)
            for name in ("u_nodes", "v_nodes", "x", "y", "z", "dxdu", "dydu", "dzdu",
                         "dxdv", "dydv", "dzdv", "nu_x", "nu_y", "nu_z"):
                a = np.ascontiguousarray(getattr(p, name), dtype=np.float64)
                self._keep.append(a)
                setattr(pd, name, ptr(a))
            self.descs[k].kind = OBJ_PATCH
            self.descs[k].patch = ctypes.pointer(pd)
        for k, t in enumerate(triangles):
            d = self.descs[len(patches) + k]
            d.kind = OBJ_TRIANGLE
            vals = [float(v) for v in np.asarray(t, dtype=np.float64).reshape(-1)]
            for q in range(9):
                d.tri[q] = vals[q]


PACKAGE_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PACKAGE_DIR, "libbbrt_cuda.so")

_lib = None


def load_library(path: str = None):
    """Load libbbrt_cuda.so from the package directory (in-tree build).
    Raises if it has not been built: there is no fallback implementation."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"libbbrt_cuda.so not built ({p}); run __graft_entry__.build()")
    lib = ctypes.CDLL(p)
    _declare(lib)
    if path is None:
        _lib = lib
    return lib


def _declare(lib):
    V, I, LL, D = ctypes.c_void_p, ctypes.c_int, ctypes.c_longlong, ctypes.c_double
    lib.bbrt_version.restype = ctypes.c_char_p
    lib.bbrt_last_error.restype = ctypes.c_char_p
    lib.bbrt_config_init.argtypes = [ctypes.POINTER(Config)]
    lib.bbrt_device_count.restype = I
    lib.bbrt_patch_file_read.argtypes = [ctypes.c_char_p, ctypes.POINTER(PatchFile)]
    lib.bbrt_patch_file_free.argtypes = [ctypes.POINTER(PatchFile)]
    lib.bbrt_scene_create.argtypes = [ctypes.POINTER(ObjectDesc), I, ctypes.POINTER(Config), ctypes.POINTER(V)]
    lib.bbrt_scene_create_from_dir.argtypes = [ctypes.c_char_p, ctypes.POINTER(Config), ctypes.POINTER(V)]
    lib.bbrt_scene_create_from_range.argtypes = [ctypes.c_char_p, ctypes.c_char_p, I, I,
                                                 ctypes.POINTER(Config), ctypes.POINTER(V)]
    lib.bbrt_scene_destroy.argtypes = [V]
    lib.bbrt_scene_destroy.restype = None
    lib.bbrt_scene_upload.argtypes = [V]
    lib.bbrt_scene_info_get.argtypes = [V, ctypes.POINTER(SceneInfo)]
    lib.bbrt_scene_setup_get.argtypes = [V, I, V, ctypes.POINTER(ctypes.c_longlong)]
    lib.bbrt_object_info_get.argtypes = [V, I, ctypes.POINTER(ObjectInfo)]
    lib.bbrt_patch_coarse_grid.argtypes = [V, I, c_int_p, c_double_p, c_double_p, c_double_p,
                                           c_double_p, c_double_p]
    lib.bbrt_self_intersect_epsilon.argtypes = [V, I, c_double_p]
    lib.bbrt_intersect.argtypes = [V, V, V, LL, I, I, I, V, V]
    lib.bbrt_trace.argtypes = [V, V, V, LL, I, I, ctypes.POINTER(TraceOut), ctypes.POINTER(TraceStats), V]
    lib.bbrt_plane_source.argtypes = [V, c_double_p, c_double_p, c_double_p, I, I, I, I, c_ll_p,
                                      ctypes.POINTER(TraceStats), V]
    lib.bbrt_patch_sample_grid.argtypes = [ctypes.POINTER(PatchDesc), I, c_double_p, c_double_p, c_double_p]
    lib.bbrt_measure_pipe_peak.argtypes = [I, c_double_p]
    lib.bbrt_umma_check.argtypes = [ctypes.POINTER(ctypes.c_ushort), ctypes.POINTER(ctypes.c_ushort),
                                    ctypes.POINTER(ctypes.c_float)]
    lib.bbrt_node_test_check.argtypes = [c_double_p, c_double_p, c_double_p, LL, c_double_p, c_int_p]
    lib.bbrt_scene_set_modes.argtypes = [V, I, I]
    lib.bbrt_trace_batch.argtypes = [ctypes.POINTER(V), I, ctypes.POINTER(V), ctypes.POINTER(V), c_ll_p, I,
                                     ctypes.POINTER(TraceOut), ctypes.POINTER(TraceStats), c_double_p]
    lib.bbrt_scene_set_create.argtypes = [ctypes.POINTER(V), I, ctypes.POINTER(V)]
    lib.bbrt_scene_set_destroy.argtypes = [V]
    lib.bbrt_scene_set_destroy.restype = None
    lib.bbrt_scene_set_configure.argtypes = [V, I, I, ctypes.POINTER(Tuning)]
    lib.bbrt_scene_set_guess_train.argtypes = [V, ctypes.POINTER(V), ctypes.POINTER(V), c_ll_p, I,
                                               ctypes.POINTER(GuessTrainConfig), ctypes.POINTER(GuessTrainReport)]
    lib.bbrt_scene_set_guess_export.argtypes = [V, I, V]
    lib.bbrt_trace_set.argtypes = [V, ctypes.POINTER(V), ctypes.POINTER(V), c_ll_p, I, ctypes.POINTER(TraceOut),
                                   ctypes.POINTER(TraceStats), c_double_p, V]
    lib.bbrt_scene_get_tuning.argtypes = [V, ctypes.POINTER(Tuning)]
    lib.bbrt_scene_set_tuning.argtypes = [V, ctypes.POINTER(Tuning)]
    lib.bbrt_scene_autotune.argtypes = [V, c_double_p, c_double_p, LL, I, I, ctypes.POINTER(Tuning), c_double_p, V]
    lib.bbrt_guess_train_config_init.argtypes = [ctypes.POINTER(GuessTrainConfig)]
    lib.bbrt_guess_train_config_init.restype = None
    lib.bbrt_guess_train.argtypes = [V, c_double_p, c_double_p, LL, I, ctypes.POINTER(GuessTrainConfig),
                                     ctypes.POINTER(GuessTrainReport), V]
    lib.bbrt_guess_param_count.argtypes = [V]
    lib.bbrt_guess_param_count.restype = LL
    lib.bbrt_guess_params.argtypes = [V, c_float_p, LL, I]
    lib.bbrt_mlp_check.argtypes = [c_float_p, I, c_float_p, c_int_p, c_float_p, c_float_p, I, c_float_p,
                                   c_float_p, c_float_p]
    lib.bbrt_mlp_infer_check.argtypes = [c_float_p, I, c_float_p, c_int_p, I, c_double_p]
    lib.bbrt_bounce_map.argtypes = [V, ctypes.POINTER(PatchDesc), I, I, I, I, D, I, c_int_p, c_int_p,
                                    c_int_p, ctypes.POINTER(TraceStats), V]
    lib.bbrt_bounce_map_rays.argtypes = [V, ctypes.POINTER(PatchDesc), I, I, I, I, D, c_ll_p, LL,
                                         c_double_p, c_double_p]


def check(lib, rc, what="bbrt call"):
    if rc != BBRT_OK:
        raise RuntimeError(f"{what} failed ({rc}): {lib.bbrt_last_error().decode(errors='replace')}")
    return rc
