"""The learned Newton initial guess: tensor-core kernels against the CPU
restatement in oracle/mlp_ref.py."""
import ctypes

import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api
from oracle import mlp_ref as R


@pytest.mark.gpu
def test_umma_operand_layouts(built):
    """D = A B^T through tcgen05 with A and B staged K-major and MN-major."""
    lib = C.load_library()
    rng = np.random.default_rng(5)
    a = R.bf16_bits(rng.standard_normal((128, 64)))
    b = R.bf16_bits(rng.standard_normal((128, 64)))
    d = np.zeros((4, 128, 128), np.float32)
    rc = lib.bbrt_umma_check(C.ptr(a, ctypes.c_ushort), C.ptr(b, ctypes.c_ushort), C.ptr(d, ctypes.c_float))
    C.check(lib, rc, "bbrt_umma_check")
    want = R.from_bf16_bits(a) @ R.from_bf16_bits(b).T
    for v in range(4):
        err = np.max(np.abs(d[v] - want))
        assert err < 1e-3 * np.max(np.abs(want)), (v, err)


def _mlp_case(P=7, B=300, seed=3):
    rng = np.random.default_rng(seed)
    params = R.init_params(P, seed)
    off = R.offsets()
    for name in ("b0", "b1", "b2"):
        params[off[name]:off[name] + R.N_H] = rng.normal(0.0, 0.05, R.N_H)
    params[off["b3"]:off["b3"] + 4] = rng.normal(0.0, 0.05, 4)
    feat = rng.normal(0.0, 1.0, (B, R.N_GEO)).astype(np.float32)
    pid = rng.integers(0, P, B).astype(np.int32)
    tgt = rng.normal(0.0, 0.5, (B, 3)).astype(np.float32)
    lbl = (rng.random(B) < 0.7).astype(np.float32)
    return params.astype(np.float32), P, feat, pid, tgt, lbl


def _device_check(lib, params, P, feat, pid, tgt, lbl):
    B = feat.shape[0]
    loss = np.zeros(1, np.float32)
    out = np.zeros((B, 4), np.float32)
    grads = np.zeros_like(params)
    F = ctypes.c_float
    rc = lib.bbrt_mlp_check(C.ptr(params, F), P, C.ptr(feat, F), C.ptr(pid, ctypes.c_int), C.ptr(tgt, F),
                            C.ptr(lbl, F), B, C.ptr(loss, F), C.ptr(out, F), C.ptr(grads, F))
    C.check(lib, rc, "bbrt_mlp_check")
    return float(loss[0]), out, grads


def test_oracle_mlp_gradients_match_finite_differences():
    """Pins the CPU restatement itself: its analytic backward pass against
    central differences of its loss (FP64, no BF16 rounding)."""
    params, P, feat, pid, tgt, lbl = _mlp_case(P=4, B=9, seed=11)
    p = params.astype(np.float64)
    _, _, g = R.forward_backward(p, P, feat, pid, tgt, lbl, rounding=False)
    off = R.offsets()
    picks = [off["W0"] + 5, off["W0"] + 64 * 3 + 20, off["b0"] + 7, off["W1"] + 300, off["b1"] + 1,
             off["W2"] + 9000, off["b2"] + 100, off["W3"] + 2 * 128 + 5, off["b3"] + 3, off["E"] + int(pid[0]) * 32 + 4]
    for k in picks:
        e = np.zeros_like(p)
        e[k] = 1e-6
        lp = R.forward_backward(p + e, P, feat, pid, tgt, lbl, rounding=False)[0]
        lm = R.forward_backward(p - e, P, feat, pid, tgt, lbl, rounding=False)[0]
        fd = (lp - lm) / 2e-6
        assert abs(fd - g[k]) <= 1e-6 + 1e-5 * abs(fd), (k, fd, g[k])


@pytest.mark.gpu
def test_mlp_forward_backward_matches_oracle(built):
    """Tensor-core forward + backward (BF16 operands, FP32 accumulation)
    against the oracle with the same BF16 roundings: loss, outputs and the
    gradient of every parameter block, over three 128-row tiles (one partial)."""
    lib = C.load_library()
    params, P, feat, pid, tgt, lbl = _mlp_case()
    loss, out, grads = _device_check(lib, params, P, feat, pid, tgt, lbl)
    rl, rout, rg = R.forward_backward(params.astype(np.float64), P, feat, pid, tgt, lbl)
    assert abs(loss - rl) <= 1e-3 * abs(rl)
    assert np.max(np.abs(out - rout)) <= 2e-2 * (1.0 + np.max(np.abs(rout)))
    assert np.mean(np.abs(out - rout)) <= 2e-3
    off = R.offsets()
    blocks = [(name, off[name], off[name] + int(np.prod(shp))) for name, shp in R.SHAPES]
    blocks.append(("E", off["E"], params.size))
    for name, a, b in blocks:
        ref = rg[a:b]
        err = np.linalg.norm(grads[a:b] - ref) / max(np.linalg.norm(ref), 1e-12)
        assert err < 2e-2, (name, err)
    # padding rows and columns get no gradient
    W0 = grads[off["W0"]:off["b0"]].reshape(R.N_H, R.N_IN)
    assert np.all(W0[:, R.N_GEO + R.N_EMB:] == 0.0)
    W3 = grads[off["W3"]:off["b3"]].reshape(R.N_OUT, R.N_H)
    assert np.all(W3[4:] == 0.0)


@pytest.mark.gpu
def test_mlp_inference_equals_training_forward(built):
    lib = C.load_library()
    params, P, feat, pid, tgt, lbl = _mlp_case(B=517, seed=8)
    _, out, _ = _device_check(lib, params, P, feat, pid, tgt, lbl)
    inf = np.zeros((feat.shape[0], 4))
    rc = lib.bbrt_mlp_infer_check(C.ptr(params, ctypes.c_float), P, C.ptr(feat, ctypes.c_float),
                                  C.ptr(pid, ctypes.c_int), feat.shape[0], C.ptr(inf))
    C.check(lib, rc, "bbrt_mlp_infer_check")
    assert np.max(np.abs(inf - out)) <= 1e-5 * (1.0 + np.max(np.abs(out)))


def _trace_forms(sc, o, d, maxb, forms):
    """Traces the rays in each (name, precision, guess) form, every bounce of
    every ray recorded (the same record length for all forms)."""
    runs = {}
    for name, prec, guess in forms:
        sc.set_modes(prec, guess)
        runs[name] = api.trace_recording_all(sc, o, d, maxb)
    K = max(r["hit_object"].shape[1] for r in runs.values())
    for name, prec, guess in forms:
        if runs[name]["hit_object"].shape[1] != K:
            sc.set_modes(prec, guess)
            runs[name] = sc.trace(o, d, maxb, record=K)
    sc.set_modes(C.PREC_FP64, C.GUESS_TRIANGLE)
    return runs


def _newton_failures(r):
    return int(np.isin(r["status"], [C.RAY_NEWTON_SINGULAR, C.RAY_NEWTON_NOCONV, C.RAY_NEWTON_DOMAIN]).sum())


@pytest.mark.gpu
def test_learned_guess_and_precision_split_trace(built):
    """Train the network on one seeded ray set of the four-sphere scene, then
    trace another: the learned and split forms keep the plain FP64 form's
    statuses and hit sequences, with every recorded hit point, (u, v) and the
    exit direction within 1e-10, on at least 99.9% of rays, and hit points
    within 1e-10 on every agreeing ray; the learned forms fail Newton no more often than the plain
    one; the split moves Newton work to FP32, and a learned start of the split
    saves FP64 iterations."""
    from billardballraytracing3d_b200 import scenes
    patches = scenes.scene_tetra_spheres()
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    to, td = scenes.cone_rays(400000, 99, 5.0, 3.0, 10.0)
    rep = sc.guess_train(to, td, 200, epochs=6)
    assert rep["positives"] > 50000 and rep["negatives"] > 50000
    assert rep["last_loss"] < 0.5 * rep["first_loss"], rep
    o, d = scenes.cone_rays(262144, 1234, 5.0, 3.0, 10.0)
    runs = _trace_forms(sc, o, d, 200, (("plain", C.PREC_FP64, C.GUESS_TRIANGLE),
                                         ("learned", C.PREC_FP64, C.GUESS_LEARNED),
                                         ("split", C.PREC_SPLIT, C.GUESS_TRIANGLE),
                                         ("both", C.PREC_SPLIT, C.GUESS_LEARNED)))
    plain = runs["plain"]
    for name in ("learned", "split", "both"):
        cmp = api.compare_traces(plain, runs[name], o)
        print(name, cmp)
        # every recorded bounce, its (u, v) and the exit direction of every agreeing non-grazing ray
        assert cmp["bounces_compared"] == int(plain["bounce_count"].sum()), name
        assert cmp["sequence_agreement"] >= 0.999, (name, cmp)
        assert cmp["agreement_within_bound"] >= 0.999, (name, cmp)
        assert cmp["max_hit_err_non_grazing"] <= 1e-10, (name, cmp)
    # the learned forms take roots outside their patch as misses and so fail less
    for name in ("learned", "both"):
        assert _newton_failures(runs[name]) <= _newton_failures(plain), name
    assert runs["both"]["stats"]["off_patch"] > 0 or _newton_failures(plain) == 0
    st_p, st_l, st_s, st_b = (runs[k]["stats"] for k in ("plain", "learned", "split", "both"))
    # the network's start is used for most wavefront solves and rarely abandoned
    assert st_l["guess_used"] > 0 and st_l["guess_fallback"] < 0.05 * st_l["guess_used"]
    # the FP32 phase takes over most of the iterations from FP64 ...
    assert st_s["newton_iters_fp32"] > 0 and st_s["newton_iters"] < 0.9 * st_p["newton_iters"]
    # ... and starting it from the learned guess saves FP64 iterations again
    assert st_b["newton_iters"] < st_s["newton_iters"]
