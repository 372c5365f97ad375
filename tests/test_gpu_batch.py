"""Batched persistent rendering: the one-launch batch path agrees with the
per-scene wavefront path on the same sample streams, is independent of the
launch shape, and covers scenes of uneven size and sample budget."""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes

pytestmark = pytest.mark.gpu


def _up(sa):
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    return s


def _batch_scenes():
    a = scenes.cornell_box(width=48, height=40, spp=12, max_depth=8)
    b = scenes.icosphere_field(n_spheres=30, subdiv=2, width=64, height=36, spp=8, max_depth=12, env_size=(128, 64))
    c = scenes.hidden_light_room(width=40, height=40, n_boxes=40, box_subdiv=2, spp=20, max_depth=10)
    return [a, b, c]


def test_batch_matches_wavefront_on_same_streams():
    sas = _batch_scenes()
    ss = [_up(sa) for sa in sas]
    imgs, st, cfg = pt.render_batch([(s, sa.spp) for s, sa in zip(ss, sas)], autotune=False, chunk_spp=4)
    for s, sa, img in zip(ss, sas, imgs):
        ref = pt.render(s, sa.spp)
        a, b = img[..., :3].astype(np.float64), ref[..., :3].astype(np.float64)
        rel = np.abs(a - b) / np.maximum(np.abs(b), 1e-3)
        assert np.median(rel) < 1e-5, (sa.name, np.median(rel))
        assert np.mean((a - b) ** 2 / (b ** 2 + 1e-2)) < 1e-4
    assert st["paths"] == sum(int(sa.camera["width"]) * int(sa.camera["height"]) * sa.spp for sa in sas)


def test_batch_independent_of_launch_shape():
    sas = _batch_scenes()
    ss = [_up(sa) for sa in sas]
    items = [(s, sa.spp, 5) for s, sa in zip(ss, sas)]
    r1, _, _ = pt.render_batch(items, block_size=64, blocks_per_sm=2, chunk_spp=4, autotune=False)
    r2, _, _ = pt.render_batch(items, block_size=256, blocks_per_sm=1, chunk_spp=4, autotune=False)
    for a, b in zip(r1, r2):
        assert np.array_equal(a, b)


def test_batch_autotuner_and_uneven_budgets():
    batch = scenes.uneven_batch(n_scenes=6, seed=9, env_size=(128, 64), tri_range=(1_000, 60_000))
    for sa in batch:
        sa.camera["width"], sa.camera["height"] = 64, 48
        sa.spp = max(4, sa.spp // 32)
    ss = [_up(sa) for sa in batch]
    imgs, st, cfg = pt.render_batch([(s, sa.spp) for s, sa in zip(ss, batch)], autotune=True)
    assert cfg["tuned_ms"] > 0
    if cfg["mode"] == pt.BATCH_PERSISTENT:
        assert cfg["block_size"] in (64, 128, 256) and cfg["blocks_per_sm"] >= 1
    else:
        assert cfg["mode"] == pt.BATCH_WAVEFRONT and cfg["paths_in_flight"] > 0
    assert st["paths"] == sum(64 * 48 * sa.spp for sa in batch)
    for img in imgs:
        assert np.isfinite(img).all() and img[..., :3].mean() > 0


def test_batch_wavefront_mode_matches_single_scene_renders():
    """Wavefront mode runs each item through the single-scene wavefront (as
    parallel graph branches): with spp a multiple of the frame size the images
    equal pt.render's bit for bit, whatever the share of path slots."""
    sas = _batch_scenes()
    ss = [_up(sa) for sa in sas]
    items = [(s, sa.spp) for s, sa in zip(ss, sas)]
    imgs, st, cfg = pt.render_batch(items, mode=pt.BATCH_WAVEFRONT)
    assert cfg["mode"] == pt.BATCH_WAVEFRONT
    small, _, _ = pt.render_batch(items, mode=pt.BATCH_WAVEFRONT, paths_in_flight=1 << 12)
    for s, sa, img, img2 in zip(ss, sas, imgs, small):
        ref = pt.render(s, sa.spp)
        assert np.array_equal(img, ref), sa.name
        assert np.array_equal(img2, ref), sa.name
    assert st["paths"] == sum(int(sa.camera["width"]) * int(sa.camera["height"]) * sa.spp for sa in sas)


def test_batch_modes_agree_and_autotuner_picks_one():
    batch = scenes.uneven_batch(n_scenes=5, seed=3, env_size=(128, 64), tri_range=(1_000, 40_000))
    for sa in batch:
        sa.camera["width"], sa.camera["height"] = 48, 40
        sa.spp = max(4, sa.spp // 64)
    ss = [_up(sa) for sa in batch]
    items = [(s, sa.spp, 3) for s, sa in zip(ss, batch)]
    a, _, _ = pt.render_batch(items, mode=pt.BATCH_PERSISTENT, autotune=False, chunk_spp=4)
    b, _, _ = pt.render_batch(items, mode=pt.BATCH_WAVEFRONT)
    c, st, cfg = pt.render_batch(items, mode=pt.BATCH_AUTO, autotune=True)
    assert cfg["mode"] in (pt.BATCH_PERSISTENT, pt.BATCH_WAVEFRONT)
    for x, y, z in zip(a, b, c):
        rel = np.abs(x[..., :3] - y[..., :3]) / np.maximum(np.abs(y[..., :3]), 1e-3)
        assert np.median(rel) < 1e-5
        assert np.isfinite(z).all()


def test_batch_item_cameras_share_one_scene():
    """Three cameras of one uploaded scene in one batch: each image equals the
    single-scene render with that camera (wavefront mode: bit for bit)."""
    sa = scenes.icosphere_field(n_spheres=30, subdiv=2, width=64, height=36, spp=8, max_depth=10, env_size=(128, 64))
    s = _up(sa)
    cams = [pt.make_camera(position=(0, 2, 14), look_at=(0, 0, 0), fov=50.0, width=64, height=36),
            pt.make_camera(position=(9, 4, 6), look_at=(0, 0.5, 0), fov=60.0, width=48, height=48),
            pt.make_camera(position=(-8, 1, -8), look_at=(0, 0, 0), fov=40.0, width=80, height=24)]
    items = [(s, 8, 0, c) for c in cams]
    imgs, st, cfg = pt.render_batch(items, mode=pt.BATCH_WAVEFRONT)
    pers, _, _ = pt.render_batch(items, mode=pt.BATCH_PERSISTENT, autotune=False, chunk_spp=4)
    assert st["paths"] == sum(int(c["width"]) * int(c["height"]) * 8 for c in cams)
    for c, img, img2 in zip(cams, imgs, pers):
        assert img.shape == (int(c["height"]), int(c["width"]), 4)
        s.update_camera(c)
        ref = pt.render(s, 8)
        assert np.array_equal(img, ref)
        rel = np.abs(img2[..., :3] - ref[..., :3]) / np.maximum(np.abs(ref[..., :3]), 1e-3)
        assert np.median(rel) < 1e-5


def test_batch_guided_items_match_single_guided_renders():
    """Guided items (two cameras sharing one trained guide, wavefront mode)
    render exactly what a single-scene guided render of the same frames does;
    asking for persistent mode with a guide is an error."""
    sa = scenes.hidden_light_room(width=40, height=40, n_boxes=40, box_subdiv=2, spp=8, max_depth=10)
    s = _up(sa)
    g = pt.Guide(s, seed=3)
    r = pt.Renderer(s)
    g.attach(r.integrator, pt.Guide.TRAIN)
    r.reset_accumulation()
    s.set_frame_count(1000)
    r.render_frames(8)
    r.synchronize()
    cams = [sa.camera, pt.make_camera(position=(2.0, 2.5, 3.0), look_at=(-1.0, 1.0, -1.0), fov=70.0,
                                      width=32, height=24)]
    imgs, st, cfg = pt.render_batch([(s, 8, 0, c, g) for c in cams])
    assert cfg["mode"] == pt.BATCH_WAVEFRONT
    for c, img in zip(cams, imgs):
        s.update_camera(c)
        rg = pt.Renderer(s)
        g.attach(rg.integrator, pt.Guide.USE)
        rg.reset_accumulation()
        s.set_frame_count(0)
        rg.render_frames(2)
        rg.synchronize()
        assert np.array_equal(img, rg.download_current_image())
    with pytest.raises(pt.PTError):
        pt.render_batch([(s, 8, 0, None, g)], mode=pt.BATCH_PERSISTENT, autotune=False)
    g.close()
