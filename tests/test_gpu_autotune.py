"""The autotuner (pt_autotune) and the traversal shapes it chooses from.

Every traversal shape (64, 128 or 256 threads per block; 32 or 64 stack
entries) and every queue capacity renders the same image bit for bit, so
the tuner changes speed only; its choice lands in the scene's settings and is
reused for scenes of the same class without timing.  The batch tuner times
the persistent kernel's shapes and the wavefront mode at three queue
capacities.
"""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes


def test_settings_reject_unknown_shapes():
    s = scenes.cornell_box(width=8, height=8).scene()
    with pytest.raises(pt.PTError, match="trace_block"):
        s.update_settings(trace_block=96)
    with pytest.raises(pt.PTError, match="stack_depth"):
        s.update_settings(stack_depth=48)
    s.update_settings(trace_block=256, stack_depth=32)
    assert (s.settings().trace_block, s.settings().stack_depth) == (256, 32)


def _up(sa):
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    return s


@pytest.mark.gpu
def test_every_traversal_shape_renders_the_same_image():
    sa = scenes.icosphere_field(n_spheres=30, subdiv=3, width=96, height=54, spp=8, env_size=(128, 64))
    s = _up(sa)
    assert s.info()["bvh_max_depth"] < 32
    ref = pt.render(s, 8)
    for block in (64, 128, 256):
        for depth in (32, 64):
            for pif in (0, 1 << 14):
                s.update_settings(trace_block=block, stack_depth=depth, paths_in_flight=pif)
                img = pt.render(s, 8)
                assert np.array_equal(img.view(np.uint32), ref.view(np.uint32)), (block, depth, pif)


@pytest.mark.gpu
def test_autotune_picks_a_shape_writes_settings_and_caches_per_class():
    sa = scenes.icosphere_field(n_spheres=30, subdiv=3, width=128, height=72, spp=8, env_size=(128, 64))
    s = _up(sa)
    ref = pt.render(s, 8)
    rep = s.autotune(calib_spp=16)
    assert not rep["cached"] and len(rep["candidates"]) >= 5
    assert rep["trace_block"] in (64, 128, 256) and rep["stack_depth"] in (32, 64)
    assert rep["best_ms"] == min(c["ms"] for c in rep["candidates"])
    st = s.settings()
    assert (st.trace_block, st.stack_depth, st.paths_in_flight) == \
        (rep["trace_block"], rep["stack_depth"], rep["paths_in_flight"])
    assert np.array_equal(pt.render(s, 8).view(np.uint32), ref.view(np.uint32))
    # a second scene of the same class: the cached choice, no timing
    sb = scenes.icosphere_field(n_spheres=30, subdiv=3, width=128, height=72, spp=8, env_size=(128, 64), seed=99)
    t = _up(sb)
    rep2 = t.autotune(calib_spp=16)
    assert rep2["cached"]
    assert (t.settings().trace_block, t.settings().stack_depth) == (rep["trace_block"], rep["stack_depth"])


@pytest.mark.gpu
def test_batch_autotuner_reports_its_queue_capacity():
    batch = scenes.uneven_batch(n_scenes=4, seed=5, env_size=(128, 64), tri_range=(1_000, 30_000))
    for sa in batch:
        sa.camera["width"], sa.camera["height"] = 64, 48
        sa.spp = 8
    ss = [_up(sa) for sa in batch]
    imgs, st, cfg = pt.render_batch([(s, sa.spp) for s, sa in zip(ss, batch)], autotune=True)
    if cfg["mode"] == pt.BATCH_WAVEFRONT:
        assert cfg["paths_in_flight"] in (1 << 25, 1 << 26, 1 << 27)
    else:
        assert cfg["chunk_spp"] == 16
    for s, sa, img in zip(ss, batch, imgs):
        ref, _, _ = pt.render_batch([(s, sa.spp)], mode=pt.BATCH_WAVEFRONT)
        rel = np.abs(img[..., :3] - ref[0][..., :3]) / np.maximum(np.abs(ref[0][..., :3]), 1e-3)
        assert np.median(rel) < 1e-5
