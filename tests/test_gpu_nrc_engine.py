"""Path tracing with the neural radiance cache through the Engine: the cache
changes nothing while it warms up, and from a cold start the cache's frames
have at least 2x lower error than equal-time plain frames against the
65,536-spp FP64-accumulated oracle."""
import numpy as np
import pytest

from vitrum_b200 import _native as N
from vitrum_b200 import scenes
from vitrum_b200.engine import Camera, Engine
from vitrum_b200.nrc import NrcConfig

pytestmark = pytest.mark.gpu

SMALL = dict(train_steps=4, train_batch=16384)


def cloud():
    sc, _ = scenes.instanced_cloud(n_instances=96, seed=21, n_points=8, sphere_levels=(2, 3), torus_segments=(48, 16),
                                   cube_cells=(4, 8), extent=6.0)
    cam = Camera(eye=(0.0, 2.0, 19.0), target=(0.0, 0.0, 0.0), fov_y_deg=45.0, near=0.01, far=200.0)
    return sc, cam


def relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + 1e-2)))


def test_warmup_frames_are_plain_path_tracing(cuda):
    sc, cam = cloud()
    a = Engine(max_bounces=6)
    a.set_scene(sc)
    a.render_frame(cam, 48, 32, samples=4, frame_seed=3)
    b = Engine(max_bounces=6)
    b.set_scene(sc)
    b.set_nrc(prefix_bounces=1, warmup_frames=1, cache=NrcConfig(levels=8, log2_table_size=14), **SMALL)
    b.render_frame(cam, 48, 32, samples=4, frame_seed=3)
    assert np.array_equal(a.capture_frame(), b.capture_frame())
    st = b.profile_frame(cam, 48, 32, samples=4, frame_seed=3)  # second frame: cache queries
    assert st["nrc_train_ms"] > 0 and st["nrc_query_ms"] > 0
    assert np.isfinite(b.capture_frame()).all()
    a.dispose()
    b.dispose()


def test_nrc_options_validation(cuda):
    sc, cam = cloud()
    e = Engine(max_bounces=4)
    e.set_scene(sc)
    for bad in (dict(prefix_bounces=-1), dict(prefix_bounces=4), dict(train_batch=100), dict(train_steps=-1),
                dict(spread_c=-1.0), dict(fallback_error=-1.0)):
        kw = dict(SMALL)
        kw.update(bad)
        with pytest.raises(N.VtError):
            e.set_nrc(**kw)
    e.set_nrc(enabled=False)
    e.render_frame(cam, 16, 16, samples=1)
    e.dispose()


def test_trained_cache_lowers_equal_time_error(cuda):
    """From a cold start (fresh cache, 8 plain warm-up frames while it trains,
    online training every frame after that), the cache's frames against plain
    path tracing given each frame's device time (training included), on the
    cloud with 8 point lights, sky, metal and glass instances; both against a
    65,536-spp FP64-accumulated oracle (whose own variance is taken out of the
    squared error).  The steady-state frames (24 to 39) have at least 2x lower
    relMSE than equal-time plain frames (median over the frames)."""
    sc, cam = cloud()
    W, H, B = 320, 180, 8
    o = Engine(max_bounces=B, oracle_accumulation=True, max_samples_per_pixel=1 << 17)
    o.set_scene(sc)
    for _ in range(16):
        o.render_frame(cam, W, H, samples=4096, frame_seed=1 << 20)
    ref, var = o.capture_moments()
    o.dispose()
    ref_var = var / 65536

    def rel(img):
        return float(np.mean(((img - ref) ** 2 - ref_var) / (ref ** 2 + 1e-2)))

    n = Engine(max_bounces=B, max_samples_per_pixel=1 << 20)
    n.set_scene(sc)
    n.set_nrc(prefix_bounces=1, warmup_frames=8, **SMALL)
    e_nrc, t_nrc = [], []
    for f in range(40):
        n.reset()
        n.render_frame(cam, W, H, samples=16, frame_seed=(1 << 12) + 16 * f)
        if f >= 24:
            t_nrc.append(n.stats()["last_frame_ms"])
            e_nrc.append(rel(n.capture_frame()[..., :3]))
    n.dispose()

    p = Engine(max_bounces=B, max_samples_per_pixel=1 << 20)
    p.set_scene(sc)
    p.render_frame(cam, W, H, samples=16, frame_seed=2 << 12)
    p.render_frame(cam, W, H, samples=16, frame_seed=2 << 12)
    t16 = p.stats()["last_frame_ms"]
    spp = max(1, int(round(16 * np.median(t_nrc) / t16)))  # plain samples in one cache frame's time
    e_plain = []
    for f in range(16):
        p.reset()
        p.render_frame(cam, W, H, samples=spp, frame_seed=(3 << 12) + 64 * f)
        e_plain.append(rel(p.capture_frame()[..., :3]))
    p.dispose()
    gain = np.median(e_plain) / np.median(e_nrc)
    print(f"equal time ({np.median(t_nrc):.2f} ms per frame, plain {spp} spp vs 16 spp into the cache): relMSE "
          f"NRC {np.median(e_nrc):.4f} plain {np.median(e_plain):.4f} ({gain:.2f}x)")
    assert gain >= 2.0


def test_error_fallback_tiles_keep_path_tracing(cuda):
    """With a threshold below every tile's cache error estimate the render paths
    never end in the cache: the frame is plain path tracing, sample for sample."""
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    W = H = 32
    plain = Engine(max_bounces=5)
    plain.set_scene(sc)
    plain.render_frame(cam, W, H, samples=8, frame_seed=21)
    want = plain.capture_frame()
    plain.dispose()
    for thr, same in ((1e-9, True), (1e9, False)):
        e = Engine(max_bounces=5)
        e.set_scene(sc)
        e.set_nrc(prefix_bounces=1, fallback_error=thr, cache=NrcConfig(levels=8, log2_table_size=12), **SMALL)
        e.render_frame(cam, W, H, samples=8, frame_seed=21)
        got = e.capture_frame()
        assert np.array_equal(got, want) == same, thr
        e.dispose()


def test_spread_termination(cuda):
    """prefix_bounces 0: paths end in the cache where their accumulated spread
    exceeds c * a0 (spreadTermination.ts).  A huge c never triggers (the frame is
    plain path tracing, sample for sample); the default c queries the cache and
    keeps the image close to the oracle."""
    sc, cam = scenes.box_room(wall_cells=8, box_cells=4)
    W = H = 32
    plain = Engine(max_bounces=5)
    plain.set_scene(sc)
    plain.render_frame(cam, W, H, samples=8, frame_seed=31)
    want = plain.capture_frame()
    plain.dispose()
    e = Engine(max_bounces=5)
    e.set_scene(sc)
    e.set_nrc(prefix_bounces=0, spread_c=1e30, cache=NrcConfig(levels=8, log2_table_size=12), **SMALL)
    e.render_frame(cam, W, H, samples=8, frame_seed=31)
    assert np.array_equal(e.capture_frame(), want)
    e.dispose()
    e = Engine(max_bounces=5)
    e.set_scene(sc)
    e.set_nrc(prefix_bounces=0, cache=NrcConfig(levels=8, log2_table_size=12), **SMALL)
    for _ in range(24):
        e.render_frame(cam, W, H, samples=8, frame_seed=31)
    st = e.profile_frame(cam, W, H, samples=8, frame_seed=31)
    img = e.capture_frame()[..., :3]
    assert st["nrc_query_ms"] > 0 and np.isfinite(img).all()
    assert abs(img.mean() / want[..., :3].mean() - 1) < 0.1
    e.dispose()
