"""Generate the golden fixtures in tests/golden/ by running the REFERENCE's own
code (its host-compilable sources, built into oracle/_ref/libptref.so by
oracle/Makefile from the reference tree).  Run in the development container:

    make -C oracle all && python tests/golden/make_golden.py

Every array here is what the reference computes; the oracle and the CUDA path
are checked against these files on machines without the reference tree.
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pyoracle import RefHarness, FACE, VERTEX  # noqa: E402
from pathtracingtutorial_b200 import scenes  # noqa: E402
import pathtracingtutorial_b200 as pt  # noqa: E402


def random_triangles(n, seed):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-4, 4, (n, 1, 3))
    p = (c + rng.normal(scale=0.3, size=(n, 3, 3))).reshape(-1, 3).astype(np.float32)
    v = np.zeros(len(p), VERTEX)
    v["position"] = p
    v["normal"] = (0, 0, 1)
    f = np.zeros(n, FACE)
    f["v0"], f["v1"], f["v2"] = np.arange(0, 3 * n, 3), np.arange(1, 3 * n, 3), np.arange(2, 3 * n, 3)
    f["material_id"] = rng.integers(0, 3, n)
    m = np.zeros(3, pt.MATERIAL_DTYPE)
    for i in range(3):
        m[i] = pt.default_material(base_color=(0.5, 0.5, 0.5))
    m[2] = pt.default_material(emissive=(3.0, 2.0, 1.0), emissive_strength=2.0)
    return v, f, m


def rays_for(lo, hi, n, seed):
    rng = np.random.default_rng(seed)
    r = np.zeros((n, 8), np.float32)
    r[:, :3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    d[: n // 20, rng.integers(0, 3)] = 0.0
    r[:, 4:7] = d
    r[:, 7] = rng.uniform(0.05, 10.0, n)
    return r


def main():
    R = RefHarness()
    out = {}
    # -- sampler streams (Part_2/src/samplers) --
    for smp, name in ((0, "pcg"), (1, "sobol")):
        for frame, sif in ((0, 0), (7, 3)):
            out[f"sampler_{name}_f{frame}_s{sif}"] = R.sampler_stream(smp, 16, 8, frame, 4, sif, 16)
    # -- BVH, light tables and traversal on two scenes --
    v, f, m = random_triangles(300, 5)
    cb = scenes.cornell_box(width=24, height=24)
    for tag, (vv, ff, mm, env) in {"rand": (v, f, m, None),
                                   "cornell": (cb.vertices, cb.faces, cb.materials, None)}.items():
        b = R.build(vv, ff, mm, env)
        out[f"{tag}_vertices"], out[f"{tag}_faces_in"], out[f"{tag}_materials"] = vv, ff, mm
        out[f"{tag}_nodes"], out[f"{tag}_faces"] = b["nodes"], b["faces"]
        out[f"{tag}_emissive"], out[f"{tag}_tri_pmf"], out[f"{tag}_tri_alias"] = b["emissive"], b["tri_pmf"], b["tri_alias"]
        lo, hi = vv["position"].min(0), vv["position"].max(0)
        rays = rays_for(lo, hi, 4096, 9)
        out[f"{tag}_rays"] = rays
        out[f"{tag}_hits"] = R.trace(b["nodes"], vv, b["faces"], rays)
        out[f"{tag}_occluded"] = R.trace(b["nodes"], vv, b["faces"], rays, any_hit=True).astype(np.uint8)
    # -- environment tables --
    env = scenes.sky_env(64, 32, sun_peak=500.0, sun_sigma_deg=4.0)
    b = R.build(cb.vertices, cb.faces, cb.materials, env)
    out["env_image"], out["env_pmf"], out["env_alias"] = env, b["env_pmf"], b["env_alias"]
    # -- camera frames (test_math.cpp cases and the cornell camera) --
    cams = [pt.make_camera((0, 0, 4), (0, 0, 0), (0, 1, 0), 90.0, width=800, height=800),
            pt.make_camera((0, 0, 0), (1, 0, 0), (0, 1, 0), 60.0, width=1920, height=1080), cb.camera]
    out["cameras"] = np.stack([np.frombuffer(np.ascontiguousarray(c).tobytes(), np.uint8) for c in cams])
    out["camera_frames"] = np.stack([R.camera_frame(c) for c in cams])
    # -- rendered films: kernelPathTrace run on the host (g++ argument order) --
    cb = scenes.cornell_box(width=24, height=24, spp=8, max_depth=8, pcg_seed=0)
    st = np.array([cb.spp, cb.sample_per_frame, cb.max_depth, cb.sampler], np.int32)
    acc, new, stats = R.render(cb.vertices, cb.faces, cb.materials, cb.camera, st, None, num_frames=2)
    out["film_cornell"], out["film_cornell_new"] = acc, new
    out["film_cornell_rays"] = np.array([stats["closest_rays"], stats["shadow_rays"]], np.float64)
    sp = scenes.icosphere_field(n_spheres=12, subdiv=1, width=20, height=12, env_size=(64, 32))
    st = np.array([8, sp.sample_per_frame, sp.max_depth, sp.sampler], np.int32)
    acc, new, stats = R.render(sp.vertices, sp.faces, sp.materials, sp.camera, st, sp.env, num_frames=2)
    out["spheres_vertices"], out["spheres_faces_in"], out["spheres_materials"] = sp.vertices, sp.faces, sp.materials
    out["spheres_camera"] = np.frombuffer(np.ascontiguousarray(sp.camera).tobytes(), np.uint8)
    out["spheres_env"] = sp.env
    out["film_spheres"] = acc
    out["film_spheres_rays"] = np.array([stats["closest_rays"], stats["shadow_rays"]], np.float64)
    np.savez_compressed(os.path.join(HERE, "reference_vectors.npz"), **out)
    # -- the reference's own unit-test expectations (Part_2/tests) --
    with open(os.path.join(HERE, "reference_unit_tests.json"), "w") as fh:
        json.dump({
            "power_heuristic": [[0.25, 0.25, 0.5], [0.2, 0.8, 0.05882353]],
            "emissive_pmf_3tri": [0.0, 0.5, 0.5],
            "env_pmf_2x1": [0.25, 0.75],
            "camera_identity": {"forward_z": -1.0, "right_x": 1.0, "up_y": 1.0, "tan_half_fov": 1.0, "aspect": 1.0},
            "camera_off_axis": {"forward": [1.0, 0.0, 0.0], "tan_half_fov_deg": 30.0, "aspect": 1920.0 / 1080.0},
            "bvh": {"one_triangle_root_leaf": True, "two_triangles_leaf_count": 2, "five_triangles_root_inner": True,
                    "hundred_triangles_face_count": 100},
            "source": "Part_2/tests/test_math.cpp:51-85, test_bvh.cpp:27-82, test_sampling.cpp:20-111",
        }, fh, indent=1)
    print("wrote", os.path.join(HERE, "reference_vectors.npz"))


if __name__ == "__main__":
    main()
