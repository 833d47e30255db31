"""The wavefront trace as one CUDA graph launch (tuning graph_rounds = 1, the
default) against the host-driven rounds (graph_rounds = 0): the same results
bit for bit and the same counters, in every arithmetic mode, with the round
loop taken many times, never, and with rays that overflow the resolved list.
"""
import os

import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes

pytestmark = pytest.mark.gpu

OUTS = ("status", "bounce_count", "exit_dir", "end_point", "hit_object", "hit_point", "hit_uv", "err_object",
        "err_value")
COUNTERS = ("rays", "bounces", "queries", "node_tests", "patch_tests", "cell_tests", "tri_tests", "newton_iters",
            "newton_iters_fp32", "guess_used", "guess_fallback", "tail_rays", "rounds")


def _both(sc, o, d, maxb, K=4, **tune):
    res = {}
    for g in (0, 1):
        sc.tuning(graph_rounds=g, **tune)
        res[g] = sc.trace(o, d, maxb, record=K, outputs=OUTS)
    sc.tuning(graph_rounds=1)
    return res[0], res[1]


def _assert_same(h, g):
    for k in OUTS:
        assert np.array_equal(h[k], g[k]), k
    for k in COUNTERS:
        assert h["stats"][k] == g["stats"][k], (k, h["stats"][k], g["stats"][k])


def test_graph_rounds_equal_host_rounds_every_mode(built):
    patches = scenes.scene_tetra_spheres()
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    to, td = scenes.cone_rays(400000, 99, 5.0, 3.0, 10.0)
    sc.guess_train(to, td, 200, epochs=6)
    o, d = scenes.cone_rays(131072, 1234, 5.0, 3.0, 10.0)
    for prec, guess in ((C.PREC_FP64, C.GUESS_TRIANGLE), (C.PREC_SPLIT, C.GUESS_TRIANGLE),
                        (C.PREC_SPLIT, C.GUESS_LEARNED)):
        sc.set_modes(prec, guess)
        h, g = _both(sc, o, d, 200)
        _assert_same(h, g)
        assert g["stats"]["rounds"] >= 2
        # the graph's launches: ordering, then per round advance / decide /
        # [four request-grouping kernels] / [inference] / Newton, then the two
        # tail kernels
        per_round = (4 if guess == C.GUESS_LEARNED else 3) + (4 if os.environ.get("BBRT_SORT_REQ", "1") != "0" else 0)
        assert g["stats"]["launches"] == 4 + per_round * g["stats"]["rounds"] + 2
        if guess == C.GUESS_LEARNED:
            assert g["stats"]["guess_used"] > 0
    sc.set_modes(C.PREC_FP64, C.GUESS_TRIANGLE)


@pytest.mark.parametrize("wave_tail", [0, 100000])
def test_graph_rounds_loop_always_or_never(built, wave_tail):
    """wave_tail 0: every round runs in the graph's loop until no ray waits;
    wave_tail 100000: the tail takes every ray after round 0 (the loop body
    never runs)."""
    patches, o, d, maxb, cn, tol = scenes.workload("tetra_spheres", 65536)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    h, g = _both(sc, o, d, maxb, wave_tail=wave_tail)
    _assert_same(h, g)
    if wave_tail == 0:
        assert g["stats"]["tail_rays"] == 0 and g["stats"]["rounds"] > 5
    else:
        assert g["stats"]["rounds"] == 1


def test_graph_rounds_overflow_rays(built):
    """Concentric spheres: queries needing more solves than the resolved list
    holds go to the overflow tail inside the graph."""
    patches = []
    for k, r in enumerate((1.0, 1.4, 1.9, 2.5, 3.2)):
        patches += scenes.obstacle_patches(k, (0.0, 0.0, 0.0), (r, r, r), None, m=2, n_nodes=5)
    rng = np.random.Generator(np.random.PCG64(11))
    n = 20000
    o = rng.normal(size=(n, 3))
    o = 6.0 * o / np.linalg.norm(o, axis=1, keepdims=True)
    d = -o + rng.normal(size=(n, 3)) * 0.8
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=9, newton_tol=1e-12))
    for tail in (0, 16384):
        h, g = _both(sc, o, d, 30, wave_tail=tail)
        _assert_same(h, g)


def test_graph_reused_and_rebuilt(built):
    """A second call with the same arguments reuses the captured graph; other
    output arrays or another ray count capture a new one; all give the same
    results."""
    patches, o, d, maxb, cn, tol = scenes.workload("tetra_spheres", 40000)
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=cn, newton_tol=tol))
    a = sc.trace(o, d, maxb, record=4, outputs=OUTS)
    b = sc.trace(o, d, maxb, record=4, outputs=OUTS)
    c = sc.trace(o, d, maxb, record=2, outputs=("status", "bounce_count", "exit_dir"))
    e = sc.trace(o[:30000], d[:30000], maxb, record=4, outputs=OUTS)
    _assert_same(a, b)
    for k in ("status", "bounce_count", "exit_dir"):
        assert np.array_equal(a[k], c[k]), k
    for k in OUTS:
        assert np.array_equal(a[k][:30000], e[k]), k
