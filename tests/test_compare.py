"""Host-side comparison of two traces (api.compare_traces,
api.min_incidence_cos): the accuracy bar of the split and learned forms
(every recorded bounce, end point and exit direction; grazing rays)."""
import numpy as np
import pytest

from billardballraytracing3d_b200 import api


def _trace(n=4, K=3, seed=0):
    rng = np.random.default_rng(seed)
    return {"status": np.zeros(n, np.int32), "bounce_count": np.array([0, 1, 2, 3][:n], np.int32),
            "hit_object": np.where(np.arange(K)[None, :] < np.array([0, 1, 2, 3][:n])[:, None],
                                   rng.integers(0, 9, (n, K)), -1).astype(np.int32),
            "hit_point": rng.normal(size=(n, K, 3)), "hit_uv": rng.normal(size=(n, K, 2)),
            "exit_dir": rng.normal(size=(n, 3)),
            "end_point": rng.normal(size=(n, 3))}


def _copy(t):
    return {k: v.copy() for k, v in t.items()}


def test_compare_identical_and_every_bounce_counted():
    a = _trace()
    r = api.compare_traces(a, _copy(a))
    assert r["sequence_agreement"] == 1.0 and r["within_bound"]
    assert r["bounces_compared"] == 6


def test_compare_sees_a_late_bounce_its_parameters_and_the_exit_direction():
    a = _trace()
    for key, idx in (("hit_point", (3, 2, 1)), ("hit_uv", (2, 1, 0)), ("exit_dir", (1, 2))):
        b = _copy(a)
        b[key][idx] += 1e-9
        r = api.compare_traces(a, b)
        assert r["sequence_agreement"] == 1.0 and not r["within_bound"], key
    # the end point is reported, not held to the bound (an escaped ray's tail
    # point scales the exit direction's difference by the scene's size)
    b = _copy(a)
    b["end_point"][2, 0] += 1e-9
    r = api.compare_traces(a, b)
    assert r["within_bound"] and r["max_end_point_err_agreeing"] > 0
    # a difference past a ray's last bounce is not a recorded hit
    b = _copy(a)
    b["hit_point"][1, 2, 0] += 1.0
    assert api.compare_traces(a, b)["within_bound"]


def test_compare_sequence_disagreement():
    a = _trace()
    b = _copy(a)
    b["hit_object"][3, 2] += 1
    b["hit_point"][3] += 5.0   # ignored: the ray does not agree
    r = api.compare_traces(a, b)
    assert r["sequence_agreement"] == 0.75 and r["within_bound"]


def test_compare_refuses_truncated_records():
    a = _trace()
    b = _copy(a)
    b["bounce_count"][0] = 4
    with pytest.raises(ValueError):
        api.compare_traces(a, b)


def test_min_incidence_cos_of_a_mirror_path():
    # z = 0 mirror hit at 60 degrees from the normal, then a second hit on
    # x = 2 (normal -x) at its own angle
    d_in = np.array([np.sin(np.pi / 3), 0.0, -np.cos(np.pi / 3)])
    o = np.array([[0.0, 0.0, 1.0]])
    p1 = o[0] + d_in / np.cos(np.pi / 3)
    d1 = d_in * np.array([1, 1, -1])
    p2 = p1 + d1 * ((2.0 - p1[0]) / d1[0])
    d2 = d1 * np.array([-1, 1, 1])
    r = {"bounce_count": np.array([2]), "hit_point": np.array([[p1, p2]]), "exit_dir": np.array([d2])}
    cos = api.min_incidence_cos(o, r)
    assert np.isclose(cos[0], min(np.cos(np.pi / 3), abs(d1[0])))


def test_agreement_within_bound_counts_rays():
    a = _trace()
    b = _copy(a)
    b["hit_uv"][3, 2, 0] += 1e-9       # ray 3 agrees in sequence but not within the bound
    r = api.compare_traces(a, b)
    assert r["sequence_agreement"] == 1.0 and not r["within_bound"]
    assert r["agreement_within_bound"] == 0.75 and r["rays_over_bound"] == 1
