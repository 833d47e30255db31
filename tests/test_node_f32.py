"""The FP32 BVH node test (k_advance and the warp-per-ray tail): wherever its
interval decides, it must give the FP64 test's answer (BVH.hpp:14-37
ray_box, the reference's test, restated in ray_box_exact) — checked here on
random rays and boxes and on cases built to sit on its decision boundaries:
faces through the ray's own FP64 points, best_t equal to the box's FP64
entry time, the origin on a face, flat boxes, nearly axis-parallel rays,
and rays outside the range its error bound covers."""
import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C

pytestmark = pytest.mark.gpu


def _run(o, d, best, boxes):
    lib = C.load_library()
    n = o.shape[0]
    out = np.zeros((n, 2), dtype=np.int32)
    rc = lib.bbrt_node_test_check(C.ptr(np.ascontiguousarray(o)), C.ptr(np.ascontiguousarray(d)),
                                  C.ptr(np.ascontiguousarray(best)), n, C.ptr(np.ascontiguousarray(boxes)),
                                  C.ptr(out, C.ctypes.c_int))
    C.check(lib, rc, "bbrt_node_test_check")
    return out[:, 0], out[:, 1]


def _fp64_slab(o, d, boxes):
    """Entry and exit times in the FP64 test's own arithmetic (numpy float64:
    fl(fl(b - o) * fl(1 / d)), swapped on the sign of 1/d)."""
    inv = 1.0 / d
    t1 = (boxes[:, :3] - o) * inv
    t2 = (boxes[:, 3:] - o) * inv
    lo = np.where(inv < 0, t2, t1)
    hi = np.where(inv < 0, t1, t2)
    return lo.max(axis=1), hi.min(axis=1)


def _unit(v):
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def _random_case(rng, n):
    o = rng.uniform(-6, 6, (n, 3))
    d = _unit(rng.normal(size=(n, 3)))
    c = rng.uniform(-4, 4, (n, 3))
    h = rng.uniform(0.01, 2.0, (n, 3))
    boxes = np.concatenate([c - h, c + h], axis=1)
    best = np.where(rng.random(n) < 0.3, np.inf, rng.uniform(0, 15, n))
    return o, d, best, boxes


def test_fp32_node_test_agrees_with_fp64_on_random_boxes(built):
    rng = np.random.default_rng(11)
    o, d, best, boxes = _random_case(rng, 400000)
    f64, f32 = _run(o, d, best, boxes)
    decided = f32 >= 0
    assert np.array_equal(f32[decided], f64[decided])
    assert (f32 == -2).sum() == 0
    assert decided.mean() > 0.995, decided.mean()
    # the FP64 test itself is the reference's slab test
    lo, hi = _fp64_slab(o, d, boxes)
    ref = (lo <= hi) & (lo <= best) & (hi >= 0)
    assert np.array_equal(ref.astype(np.int32), f64)


def test_fp32_node_test_on_its_decision_boundaries(built):
    rng = np.random.default_rng(12)
    n = 200000
    o, d, best, boxes = _random_case(rng, n)
    # cone rays like the tetrahedron workload's (small x and y components)
    d[: n // 4] = _unit(np.column_stack([rng.normal(0, 0.05, n // 4), rng.normal(0, 0.05, n // 4),
                                         -np.ones(n // 4)]))
    kind = np.arange(n) % 6
    t0 = rng.uniform(0.1, 12.0, n)
    p = o + t0[:, None] * d
    ax = rng.integers(0, 3, n)
    ulps = rng.integers(-3, 4, n)
    # 0: the min face on the ray's FP64 point (a few ulps either side)
    sel = kind == 0
    boxes[sel, ax[sel]] = p[sel, ax[sel]] + ulps[sel] * np.spacing(p[sel, ax[sel]])
    boxes[sel, ax[sel]] = np.minimum(boxes[sel, ax[sel]], boxes[sel, 3 + ax[sel]])
    # 1: the max face likewise
    sel = kind == 1
    boxes[sel, 3 + ax[sel]] = p[sel, ax[sel]] + ulps[sel] * np.spacing(p[sel, ax[sel]])
    boxes[sel, 3 + ax[sel]] = np.maximum(boxes[sel, 3 + ax[sel]], boxes[sel, ax[sel]])
    # 2: best_t on the box's FP64 entry time (the prune comparison)
    lo, hi = _fp64_slab(o, d, boxes)
    sel = (kind == 2) & np.isfinite(lo)
    best[sel] = lo[sel] + ulps[sel] * np.spacing(np.abs(lo[sel]) + 1e-300)
    # 3: the origin on a face (exit time near 0)
    sel = kind == 3
    boxes[sel, 3 + ax[sel]] = o[sel, ax[sel]] + ulps[sel] * np.spacing(o[sel, ax[sel]])
    boxes[sel, ax[sel]] = np.minimum(boxes[sel, ax[sel]], boxes[sel, 3 + ax[sel]])
    # 4: flat boxes (zero width on one axis) through the ray's point
    sel = kind == 4
    boxes[sel, ax[sel]] = p[sel, ax[sel]]
    boxes[sel, 3 + ax[sel]] = p[sel, ax[sel]]
    # 5: nearly axis-parallel rays
    sel = kind == 5
    d[sel, ax[sel]] = rng.choice([1e-4, -1e-7, 1e-10], sel.sum())
    d[sel] = _unit(d[sel])
    f64, f32 = _run(o, d, best, boxes)
    decided = f32 >= 0
    assert np.array_equal(f32[decided], f64[decided])
    assert (f32 == -2).sum() == 0
    # the boundary cases do reach the FP64 test (the interval does not decide them)
    assert (f32 == -1).sum() > 1000
    lo, hi = _fp64_slab(o, d, boxes)
    ref = (lo <= hi) & (lo <= best) & (hi >= 0)
    assert np.array_equal(ref.astype(np.int32), f64)


def test_fp32_node_test_range_limits(built):
    """Rays whose FP32 values leave the bound's range are never decided in
    FP32: a direction component below 2^-40 (1/d beyond 2^40), an origin
    beyond 2^40, a zero component; boxes with a coordinate beyond 2^40 turn
    the FP32 test off for every ray."""
    o = np.array([[0.0, 0.0, 5.0], [0.0, 0.0, 5.0], [2.0 ** 41, 0.0, 5.0], [0.0, 0.0, 5.0]])
    d = _unit(np.array([[1e-13, 0.3, -1.0], [0.2, 0.3, -1.0], [0.2, 0.3, -1.0], [0.0, 0.3, -1.0]]))
    boxes = np.tile(np.array([[-1.0, -1.0, -1.0, 1.0, 1.0, 1.0]]), (4, 1))
    best = np.full(4, np.inf)
    f64, f32 = _run(o, d, best, boxes)
    assert list(f32) == [-2, f64[1], -2, -2]
    big = boxes.copy()
    big[1, 3] = 2.0 ** 41
    _, f32b = _run(o, d, best, big)
    assert list(f32b) == [-2, -2, -2, -2]
