"""The device-side bounds that keep a trace from holding the GPU: the
k_advance watchdog and the tensor-core completion waits of the learned
guess.  Each is set, per scene, to a bound that every launch exceeds at once;
the call must then return BBRT_ERR_KERNEL with its message (the kernels
leave on their own: nothing hangs or faults), and the next call with the
default bounds must give the results of a call made before, bit for bit."""
import numpy as np
import pytest

from billardballraytracing3d_b200 import _capi as C
from billardballraytracing3d_b200 import api, scenes

pytestmark = pytest.mark.gpu

KEYS = ("status", "bounce_count", "hit_object", "hit_point", "exit_dir", "end_point")


def _same(a, b):
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("graph_rounds", [1, 0])
def test_watchdog_stops_the_round_and_the_next_call_is_clean(built, graph_rounds):
    patches = scenes.scene_tetra_spheres()
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    o, d = scenes.cone_rays(32768, 1234, 5.0, 3.0, 10.0)
    sc.tuning(graph_rounds=graph_rounds)
    before = sc.trace(o, d, 200, record=4)
    sc.tuning(watchdog_cycles=1)
    with pytest.raises(RuntimeError) as e:
        sc.trace(o, d, 200, record=4)
    assert f"({C.BBRT_ERR_KERNEL})" in str(e.value) and "watchdog" in str(e.value)
    sc.tuning(watchdog_cycles=0)
    _same(sc.trace(o, d, 200, record=4), before)


def test_tensor_core_wait_bound_reports_and_the_next_call_is_clean(built):
    patches = scenes.scene_tetra_spheres()
    sc = api.Scene(patches, config=C.default_config(coarse_grid_n=17, newton_tol=1e-12))
    to, td = scenes.cone_rays(262144, 99, 5.0, 3.0, 10.0)
    sc.guess_train(to, td, 200, epochs=4)
    o, d = scenes.cone_rays(65536, 1234, 5.0, 3.0, 10.0)
    sc.tuning(wave_tail=1024)   # wavefront rounds (which run the network) down to the last 1024 requests
    sc.set_modes(C.PREC_SPLIT, C.GUESS_LEARNED)
    before = sc.trace(o, d, 200, record=4)
    assert before["stats"]["guess_used"] > 0
    sc.tuning(mma_wait_cycles=1)
    with pytest.raises(RuntimeError) as e:
        sc.trace(o, d, 200, record=4)
    assert f"({C.BBRT_ERR_KERNEL})" in str(e.value) and "tensor-core completion wait" in str(e.value)
    sc.tuning(mma_wait_cycles=0)
    _same(sc.trace(o, d, 200, record=4), before)
