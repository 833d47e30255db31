"""Scene sets (bbrt_scene_set_create / bbrt_trace_set): several scenes of
uneven sizes traced as one wavefront.  Every member's results must be the
results of tracing that member alone (which the other GPU tests pin to the
oracle), bit for bit, in the member's own object numbering — in every launch
schedule, in the precision split, with members that have no rays, and after
the member scenes themselves are gone."""
import ctypes

import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes

pytestmark = pytest.mark.gpu

OUTS = {"status": (np.int32, ()), "bounce_count": (np.int32, ()), "exit_dir": (np.float64, (3,)),
        "end_point": (np.float64, (3,)), "hit_object": (np.int32, ("K",)), "hit_point": (np.float64, ("K", 3)),
        "hit_uv": (np.float64, ("K", 2)), "err_object": (np.int32, ()), "err_value": (np.float64, (2,))}


def _members(n_scenes=6, seed=5, max_rays=60000):
    work = scenes.multi_scene_workload(n_scenes, seed=seed, max_obstacles=6, min_rays=3000, max_rays=max_rays)
    scs = [api.Scene(p, config=C.default_config(coarse_grid_n=cn, newton_tol=tol)) for p, o, d, mb, cn, tol in work]
    return work, scs


def _device_io(torch, work, K, ns=None):
    tens, outs = [], []
    for j, (patches, o, d, maxb, cn, tol) in enumerate(work):
        n = o.shape[0] if ns is None else ns[j]
        t = {"o": torch.from_numpy(np.ascontiguousarray(o[:n])).cuda(),
             "d": torch.from_numpy(np.ascontiguousarray(d[:n])).cuda()}
        tdt = {np.int32: torch.int32, np.float64: torch.float64}
        for k, (dt, shape) in OUTS.items():
            t[k] = torch.full((n,) + tuple(K if x == "K" else x for x in shape), -5, dtype=tdt[dt], device="cuda")
        tens.append(t)
        outs.append(dict(record=K, **{k: t[k].data_ptr() for k in OUTS}))
    return tens, outs


def _check(refs, tens):
    for j, (ref, t) in enumerate(zip(refs, tens)):
        for k in OUTS:
            assert np.array_equal(ref[k], t[k].cpu().numpy()), (j, k)


@pytest.mark.parametrize("schedule", [{}, {"graph_rounds": 0}, {"wave_tail": 0}, {"graph_rounds": 0, "wave_tail": 100000}])
def test_scene_set_equals_each_scene_alone(built, schedule):
    import torch
    work, scs = _members()
    K = 6
    refs = [sc.trace(o, d, maxb, record=K, outputs=tuple(OUTS)) for sc, (p, o, d, maxb, cn, tol) in zip(scs, work)]
    assert max(int(r["bounce_count"].max()) for r in refs) <= K
    ss = api.SceneSet(scs)
    if schedule:
        t = scs[0].tuning()
        t.update(schedule)
        ss.configure(C.PREC_FP64, C.GUESS_TRIANGLE, **t)
    tens, outs = _device_io(torch, work, K)
    for call in range(2):   # the second call reuses the captured graph
        for t in tens:
            for k in OUTS:
                t[k].fill_(-5)
        st, ms = ss.trace_device([t["o"].data_ptr() for t in tens], [t["d"].data_ptr() for t in tens],
                                 [w[1].shape[0] for w in work], 100, outs)
        torch.cuda.synchronize()
        _check(refs, tens)
        assert ms > 0 and st["rays"] == sum(w[1].shape[0] for w in work)
        assert st["bounces"] == sum(int(r["bounce_count"].sum()) for r in refs)


def test_scene_set_split_precision_empty_members_and_gone_members(built):
    import torch
    work, scs = _members(n_scenes=5, seed=9, max_rays=20000)
    K = 6
    ns = [w[1].shape[0] for w in work]
    ns[1] = 0          # a member without rays
    ns[3] = 700        # and a small one: the whole set below the wavefront size
    for sc in scs:
        sc.set_modes(C.PREC_SPLIT, C.GUESS_TRIANGLE)
    refs = [sc.trace(o[:n], d[:n], 100, record=K, outputs=tuple(OUTS)) for sc, (p, o, d, mb, cn, tol), n
            in zip(scs, work, ns)]
    ss = api.SceneSet(scs)
    ss.configure(C.PREC_SPLIT)
    for sc in scs:
        sc.close()      # the set keeps its own copy of every member
    tens, outs = _device_io(torch, work, K, ns)
    st, _ = ss.trace_device([t["o"].data_ptr() for t in tens], [t["d"].data_ptr() for t in tens], ns, 100, outs)
    torch.cuda.synchronize()
    _check(refs, tens)
    small = [w for w in ns]
    small_ns = [min(n, 1500) for n in small]
    tens2, outs2 = _device_io(torch, work, K, small_ns)
    st2, _ = ss.trace_device([t["o"].data_ptr() for t in tens2], [t["d"].data_ptr() for t in tens2], small_ns, 100,
                             outs2)
    torch.cuda.synchronize()
    assert sum(small_ns) < 8192 and st2["rays"] == sum(small_ns)
    for j, t in enumerate(tens2):
        for k in OUTS:
            assert np.array_equal(refs[j][k][:small_ns[j]], t[k].cpu().numpy()), (j, k)


def test_scene_set_rejects_mismatched_members(built):
    lib = C.load_library()
    a = api.Scene(scenes.scene_two_spheres(), config=C.default_config(coarse_grid_n=9))
    b = api.Scene(scenes.scene_two_spheres(), config=C.default_config(coarse_grid_n=17))
    hs = (ctypes.c_void_p * 2)(a.h, b.h)
    h = ctypes.c_void_p()
    assert lib.bbrt_scene_set_create(hs, 2, ctypes.byref(h)) == C.BBRT_ERR_ARG
    assert b"must share the coarse grid size" in lib.bbrt_last_error()
    hs = (ctypes.c_void_p * 2)(a.h, a.h)
    assert lib.bbrt_scene_set_create(hs, 2, ctypes.byref(h)) == C.BBRT_ERR_ARG


def test_scene_set_learned_network_of_two_scenes(built):
    """One network trained on the four-sphere and the ellipsoid scenes
    together (a set of the two): the set's learned form agrees with the plain
    form on >= 99.9% of each member's rays within 1e-10, and each member,
    given its share of the network, traces its learned form to the same bar
    against the set's trace of it."""
    import torch
    tet = api.Scene(scenes.scene_tetra_spheres(), config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    ell = api.Scene(scenes.scene_ellipsoids(), config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    ss = api.SceneSet([tet, ell])
    src = [(5.0, 3.0, 10.0), (8.0, 6.0, 20.0)]
    train = [scenes.cone_rays(200000, 99 + j, *src[j]) for j in range(2)]
    rep = ss.guess_train([t[0] for t in train], [t[1] for t in train], 100, epochs=4)
    assert rep["positives"] > 50000 and rep["last_loss"] < rep["first_loss"]
    rays = [scenes.cone_rays(65536, 1234 + j, *src[j]) for j in range(2)]
    K = 100   # every bounce recorded
    runs = {}
    for name, guess in (("plain", C.GUESS_TRIANGLE), ("learned", C.GUESS_LEARNED)):
        ss.configure(C.PREC_SPLIT if guess == C.GUESS_LEARNED else C.PREC_FP64, guess, wave_tail=1024,
                     **{k: v for k, v in tet.tuning().items() if k != "wave_tail"})
        work = [(None, o, d, 100, 17, 1e-12) for o, d in rays]
        tens, outs = _device_io(torch, work, K)
        st, _ = ss.trace_device([t["o"].data_ptr() for t in tens], [t["d"].data_ptr() for t in tens],
                                [o.shape[0] for o, _ in rays], 100, outs)
        torch.cuda.synchronize()
        runs[name] = [{k: t[k].cpu().numpy() for k in OUTS} for t in tens]
        if guess == C.GUESS_LEARNED:
            assert st["guess_used"] > 0
    for j in range(2):
        assert int(runs["plain"][j]["bounce_count"].max()) <= K
        cmp = api.compare_traces(runs["plain"][j], runs["learned"][j], rays[j][0])
        assert cmp["sequence_agreement"] >= 0.999 and cmp["agreement_within_bound"] >= 0.999, (j, cmp)
        assert cmp["max_hit_err_non_grazing"] <= 1e-10, (j, cmp)
    # a member alone with its share of the network: the same accuracy bar
    # against the set's learned trace (not bit for bit: which bounces the
    # wavefront rounds solve from the network's start, and which the tail
    # solves from the triangle's, depends on how many requests each round holds)
    for j, sc in enumerate((tet, ell)):
        ss.guess_export(j, sc)
        sc.set_modes(C.PREC_SPLIT, C.GUESS_LEARNED)
        sc.tuning(wave_tail=1024)
        alone = sc.trace(rays[j][0], rays[j][1], 100, record=K, outputs=tuple(OUTS))
        assert alone["stats"]["guess_used"] > 0
        cmp = api.compare_traces(alone, runs["learned"][j], rays[j][0])
        assert cmp["sequence_agreement"] >= 0.999 and cmp["agreement_within_bound"] >= 0.999, (j, cmp)
