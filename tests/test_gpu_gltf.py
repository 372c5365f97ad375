"""A glTF scene (tests/test_gltf_io.py's synthetic file: Disney materials from
the KHR extensions, KHR_lights_punctual lights, transformed meshes) rendered
on the GPU and by the FP64 oracle on the same sample streams."""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes
from test_gltf_io import _write

pytestmark = pytest.mark.gpu


def test_gltf_scene_radiance_correlated_with_fp64_oracle(oracle, tmp_path):
    s = pt.SceneManager.load(str(_write(tmp_path, "glb")))
    cam = s.camera.copy()
    cam["width"], cam["height"] = 48, 32
    s.update_camera(cam)
    spp = 16
    s.update_settings(spp=spp, sample_per_frame=4, max_depth=8, sampler_type=pt.SAMPLER_SOBOL)
    sa = scenes.SceneArrays("gltf", s.vertices(), s.faces(), s.materials(), cam, None, spp=spp,
                            sample_per_frame=4, max_depth=8, sampler=pt.SAMPLER_SOBOL)
    sa.punctual = s.punctual_lights()
    assert len(sa.punctual) == 3
    s.build_accel()
    s.upload_to_device(0)
    img = pt.render(s, spp)[..., :3].astype(np.float64)
    prep = oracle.prepare(sa)
    (mean, _), _ = oracle.render(prep, 4, 8, pt.SAMPLER_SOBOL, frames=spp // 4, first_frame=0, precision=64,
                                 rtl=pt.DEVICE_ARG_ORDER, pcg_seed=0)
    assert mean.mean() > 0
    rel = np.abs(img - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert float(np.mean((img - mean) ** 2 / (mean ** 2 + 1e-2))) < 1e-3
