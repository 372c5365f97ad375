"""Output path: the preview's tone mapping as a CUDA kernel (headless buffer
instead of an OpenGL framebuffer), against the shader's formulas in float64."""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("exposure", [-2.8, 0.0, 1.5])
def test_tonemap_matches_shader_formula(exposure):
    from oracle.pyoracle import tonemap_ref
    rng = np.random.default_rng(4)
    img = np.ones((61, 97, 4), np.float32)
    img[..., :3] = np.exp(rng.uniform(-8, 8, (61, 97, 3))).astype(np.float32)
    img[0, :5, :3] = [0.0, 1e-6, 1e30]          # black, the linear segment, saturation
    out = pt.tonemap(img, exposure)
    ref = tonemap_ref(img, exposure)
    assert out.dtype == np.uint8 and out.shape == (61, 97, 4)
    assert np.abs(out.astype(int) - ref.astype(int)).max() <= 1
    assert (out[..., 3] == 255).all()


def test_tonemap_of_a_render():
    from oracle.pyoracle import tonemap_ref
    sa = scenes.cornell_box(width=48, height=48, spp=8)
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    img = pt.render(s, 8)
    out = pt.tonemap(img)
    assert np.abs(out.astype(int) - tonemap_ref(img).astype(int)).max() <= 1
    assert out[..., :3].mean() > 10


def test_film_download_waits_for_the_render():
    """Renderer.render_frames returns with the render queued on the
    integrator's stream; the film download (Film::downloadAccumulated) still
    returns the finished image, as the reference's blocking copy does."""
    sa = scenes.cornell_box(width=96, height=96)
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    r = pt.Renderer(s)
    r.reset_accumulation()
    r.render_frames(16)
    img = r.download_current_image()          # no synchronize in between
    ref = pt.render(s, 64)
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
