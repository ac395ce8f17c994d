"""Failure detection without a GPU fault.

(1) Bounded device waits run out on purpose: a debug hook bounds the first
wait of the radiance-cache kernels' tensor-core products and of the traversal's
shared-memory staging copy to one clock.  The kernels record the expiry, wait
for their own work in flight under the full limit, free their tensor memory and
return; the host reports VT_ERR_TIMEOUT / VT_ERR_BUILD, drops the failed
frame's samples, and the engine keeps rendering correctly afterwards (the
reference reports device errors through onError without killing the engine,
pt-webgpu/src/index.ts:736-750).

(2) Device allocation failures are injected on the host (a fake out-of-memory
cudaMalloc at the nth allocation): vt_set_scene is transactional -- at every
allocation stage the failure leaves the previous scene and its image as they
were (the reference's transactionalResourceReplacement.test.ts, which fails
each allocation stage of uploadPackedScene in turn).
"""
import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.engine import Engine, debug_fail_device_allocation

pytestmark = pytest.mark.gpu

VT_ERR_OUT_OF_MEMORY, VT_ERR_BUILD, VT_ERR_TIMEOUT = 4, 6, 7


def _room():
    return scenes.box_room(wall_cells=8, box_cells=4)


def _frame(e, cam, seed=5, spp=8):
    e.reset()
    e.render_frame(cam, 32, 32, samples=spp, frame_seed=seed)
    return e.capture_frame().copy()


def test_staging_wait_expiry_is_reported_and_the_engine_recovers(cuda):
    sc, cam = _room()
    ref = Engine(max_bounces=3)
    ref.set_scene(sc)
    want = _frame(ref, cam)
    ref.dispose()
    e = Engine(max_bounces=3, debug=True)
    e.set_scene(sc)
    e.set_tuning(wave_paths=1 << 20, stage_hot_nodes=True)
    assert _frame(e, cam).tobytes() == want.tobytes()   # staging on: same image
    e.debug.set_wait_limit(1)
    with pytest.raises(N.VtError) as err:
        _frame(e, cam)
    assert err.value.status == VT_ERR_BUILD and "staging" in str(err.value)
    # the expired CTAs traversed from global memory; the frame was dropped, not kept
    assert e.render_frame(cam, 32, 32, samples=0)["samplesAccumulated"] == 0
    e.debug.set_wait_limit(0)
    assert _frame(e, cam).tobytes() == want.tobytes()
    e.dispose()


def test_cache_wait_expiry_is_reported_and_the_engine_recovers(cuda):
    sc, cam = _room()
    e = Engine(max_bounces=3, debug=True)
    e.set_scene(sc)
    e.set_nrc(prefix_bounces=1, train_steps=1, train_batch=4096)
    e.render_frame(cam, 32, 32, samples=4, frame_seed=1)
    e.debug.set_wait_limit(1)
    with pytest.raises(N.VtError) as err:
        e.reset()
        e.render_frame(cam, 32, 32, samples=4, frame_seed=2)
    assert err.value.status == VT_ERR_TIMEOUT
    e.debug.set_wait_limit(0)
    e.reset()
    out = e.render_frame(cam, 32, 32, samples=4, frame_seed=3)
    img = e.capture_frame()
    assert out["samplesAccumulated"] == 4 and np.isfinite(img).all() and img[..., :3].mean() > 0
    # plain path tracing on the same engine equals a fresh engine's
    e.set_nrc(enabled=False)
    got = _frame(e, cam)
    ref = Engine(max_bounces=3)
    ref.set_scene(sc)
    want = _frame(ref, cam)
    ref.dispose()
    e.dispose()
    assert got.tobytes() == want.tobytes()


def test_set_scene_rolls_back_at_every_allocation_stage(cuda):
    room, cam = _room()
    other, _ = scenes.box_room(wall_cells=6, box_cells=3)
    e = Engine(max_bounces=3)
    e.set_scene(room)
    want = _frame(e, cam)
    stages = 0
    for k in range(1, 200):
        debug_fail_device_allocation(k)
        try:
            e.set_scene(other)
        except N.VtError as err:
            assert err.status == VT_ERR_OUT_OF_MEMORY and "injected" in str(err)
            stages += 1
            # the previous scene is intact: the same image, bit for bit
            assert _frame(e, cam).tobytes() == want.tobytes(), k
            continue
        finally:
            debug_fail_device_allocation(0)
        break
    assert stages >= 10, stages      # every staged buffer was a failure point
    other_img = _frame(e, cam)        # the new scene took effect once nothing failed
    assert other_img.tobytes() != want.tobytes()
    e.dispose()


def test_wait_limit_hook_needs_debug(cuda):
    sc, cam = _room()
    e = Engine(max_bounces=1)
    e.set_scene(sc)
    with pytest.raises(N.VtError):
        N.call("vt_engine_set_wait_limit", e.handle, 1)
    e.dispose()
