"""Batched rendering of many scenes (vt_batch_*) against the single-scene
engine: the same estimator on the same paths, so every scene's image matches
its own Engine frame up to the summation order of the accumulation."""
import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.batch import Batch, BatchItem
from vitrum_b200.engine import Engine

pytestmark = pytest.mark.gpu


def items(n=5):
    out = []
    for i, (tris, res, b, spp) in enumerate([(4096, 32, 2, 4), (20000, 48, 5, 3), (600, 24, 8, 6),
                                              (70000, 40, 3, 2), (9000, 16, 6, 5)][:n]):
        sc, cam = scenes.box_room_sized(tris)
        out.append(BatchItem(sc, cam, res, res, spp, b, frame_seed=11 + i))
    return out


@pytest.mark.parametrize("wave", [1024, 4096, 1 << 20])
@pytest.mark.parametrize("sort", [True, False])
def test_batch_matches_single_scene_engine(cuda, wave, sort):
    its = items()
    b = Batch(its)
    b.set_tuning(wave, sort_by_material=sort)
    st = b.render()
    assert st["waves"] >= 1 and st["closest_rays"] > 0
    for i, it in enumerate(its):
        e = Engine(max_bounces=8)
        e.set_scene(it.scene)
        e.render_frame(it.camera, it.width, it.height, samples=it.samples, bounces=it.bounces,
                       frame_seed=it.frame_seed)
        want = e.capture_frame()
        got = b.capture(i)
        assert np.allclose(got, want, rtol=1e-4, atol=1e-5), (i, np.abs(got - want).max())
        e.dispose()
    b.close()


def test_batch_rerender_and_autotune(cuda):
    its = items()
    b = Batch(its)
    b.render()
    a = [b.capture(i).copy() for i in range(len(its))]
    trials = b.autotune()
    assert len(trials) >= 3 and all(t["frame_ms"] > 0 for t in trials)
    best = b.tuning
    assert best["wave_paths"] in {t["wave_paths"] for t in trials}
    b.render()
    for i in range(len(its)):
        assert np.allclose(b.capture(i), a[i], rtol=1e-4, atol=1e-5)
    b.close()


def test_batch_validation(cuda):
    sc, cam = scenes.box_room_sized(1000)
    with pytest.raises(N.VtError):
        Batch([BatchItem(sc, cam, 20000, 16, 1)])
    with pytest.raises(N.VtError):
        Batch([BatchItem(sc, cam, 16, 16, 0)])
    inst, icam = scenes.instanced_cloud(n_instances=4, sphere_levels=(1,), torus_segments=(8, 4), cube_cells=(2,))
    with pytest.raises(N.VtError):
        Batch([BatchItem(inst, icam, 16, 16, 1)])
    b = Batch([BatchItem(sc, cam, 16, 16, 1)])
    with pytest.raises(N.VtError):  # one root per ray: nothing to stage
        b.set_tuning(1 << 20, stage_hot_nodes=True)
    b.set_tuning(1 << 20)
    assert b.tuning["stage_hot_nodes"] == 0
    b.close()
