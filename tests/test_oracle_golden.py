"""The oracle pinned against the reference: golden vectors written by running the
reference's own code (tests/golden/make_golden.py), and the reference's own
unit-test expectations (Part_2/tests).  CPU only."""
import json
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_vectors.npz"))
UT = json.load(open(os.path.join(HERE, "golden", "reference_unit_tests.json")))


def bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


@pytest.mark.parametrize("name,smp", [("pcg", 0), ("sobol", 1)])
@pytest.mark.parametrize("frame,sif", [(0, 0), (7, 3)])
def test_sampler_streams(oracle, name, smp, frame, sif):
    got = oracle.sampler_stream(smp, 16, 8, frame, 4, sif, 16)
    assert np.array_equal(got.view(np.uint32), G[f"sampler_{name}_f{frame}_s{sif}"].view(np.uint32))


def test_pcg_can_return_one_and_sobol_clamps(oracle):
    s = oracle.sampler_stream(1, 64, 64, 0, 4, 0, 8)
    assert s.max() <= np.float32(0.99999994) and s.min() >= 0.0
    p = oracle.sampler_stream(0, 64, 64, 0, 4, 0, 64)
    assert p.max() <= 1.0 and p.min() >= 0.0


@pytest.mark.parametrize("tag", ["rand", "cornell"])
def test_bvh_and_light_tables(oracle, tag):
    nodes, faces, _ = oracle.build_bvh(G[f"{tag}_vertices"], G[f"{tag}_faces_in"])
    assert np.array_equal(bits(nodes), bits(G[f"{tag}_nodes"]))
    assert np.array_equal(bits(faces), bits(G[f"{tag}_faces"]))
    refs, pmf, alias = oracle.emissive_tables(G[f"{tag}_vertices"], faces, G[f"{tag}_materials"])
    assert np.array_equal(bits(refs), bits(G[f"{tag}_emissive"]))
    assert np.array_equal(bits(pmf), bits(G[f"{tag}_tri_pmf"]))
    assert np.array_equal(bits(alias), bits(G[f"{tag}_tri_alias"]))


@pytest.mark.parametrize("tag", ["rand", "cornell"])
def test_traversal_hits_and_occlusion(oracle, tag):
    hits, cnt = oracle.trace(G[f"{tag}_nodes"], G[f"{tag}_vertices"], G[f"{tag}_faces"], G[f"{tag}_rays"])
    assert np.array_equal(hits.view(np.uint32), G[f"{tag}_hits"].view(np.uint32))
    occ, _ = oracle.trace(G[f"{tag}_nodes"], G[f"{tag}_vertices"], G[f"{tag}_faces"], G[f"{tag}_rays"], any_hit=True)
    assert np.array_equal(occ.astype(np.uint8), G[f"{tag}_occluded"])
    assert cnt["node_pops"] > 0 and cnt["tri_tests"] > 0


def test_env_tables(oracle):
    pmf, alias = oracle.env_tables(G["env_image"])
    assert np.array_equal(pmf.view(np.uint32), G["env_pmf"].view(np.uint32))
    assert np.array_equal(bits(alias), bits(G["env_alias"]))


def test_camera_frames(oracle):
    for cam, ref in zip(G["cameras"], G["camera_frames"]):
        assert np.array_equal(oracle.camera_frame(cam).view(np.uint32), ref.view(np.uint32))


def _film(oracle, prefix, spp_per_frame=4, frames=2, sampler=None, depth=None, cam=None):
    from pathtracingtutorial_b200.scenes import SceneArrays
    import pathtracingtutorial_b200 as pt
    v, f, m = G[f"{prefix}_vertices"], G[f"{prefix}_faces_in"], G[f"{prefix}_materials"]
    env = G[f"{prefix}_env"] if f"{prefix}_env" in G.files else None
    camera = np.frombuffer(G[f"{prefix}_camera"].tobytes(), pt.CAMERA_DTYPE)[0] if cam is None else cam
    sa = SceneArrays("golden", v, f, m, camera, env)
    prep = oracle.prepare(sa)
    return oracle.render(prep, spp_per_frame, depth, sampler, frames=frames, precision=32, rtl=1)


def test_film_cornell_bit_exact(oracle):
    from pathtracingtutorial_b200 import scenes
    cb = scenes.cornell_box(width=24, height=24, spp=8, max_depth=8, pcg_seed=0)
    prep = oracle.prepare(cb)
    img, cnt = oracle.render(prep, 4, 8, cb.sampler, frames=2, precision=32, rtl=1, pcg_seed=0)
    assert np.array_equal(img.view(np.uint32), G["film_cornell"].view(np.uint32))
    assert cnt["closest_rays"] == G["film_cornell_rays"][0] and cnt["shadow_rays"] == G["film_cornell_rays"][1]


def test_film_env_spheres_bit_exact(oracle):
    img, cnt = _film(oracle, "spheres", frames=2, sampler=1, depth=16)
    assert np.array_equal(img.view(np.uint32), G["film_spheres"].view(np.uint32))
    assert cnt["closest_rays"] == G["film_spheres_rays"][0] and cnt["shadow_rays"] == G["film_spheres_rays"][1]


def test_fp64_agrees_with_fp32_in_expectation(oracle):
    from pathtracingtutorial_b200 import scenes
    cb = scenes.cornell_box(width=16, height=16, spp=64, max_depth=8)
    prep = oracle.prepare(cb)
    img, _ = oracle.render(prep, 4, 8, 0, frames=16, precision=32, rtl=1, pcg_seed=1)
    (mean, var), _ = oracle.render(prep, 4, 8, 0, frames=16, precision=64, rtl=1, pcg_seed=1)
    # same sample streams: the two precisions track each other closely
    rel = np.abs(img[..., :3] - mean) / np.maximum(mean, 1e-3)
    assert np.median(rel) < 1e-4


# ---- the reference's unit tests, restated against the oracle ----
def test_reference_unit_emissive_pmf(oracle):
    import pathtracingtutorial_b200 as pt
    from oracle.pyoracle import VERTEX, FACE
    m = np.zeros(3, pt.MATERIAL_DTYPE)
    m[0] = pt.default_material(base_color=(1, 1, 1))
    m[1] = pt.default_material(base_color=(1, 1, 1), emissive=(2, 2, 2))
    m[2] = pt.default_material(base_color=(0.5, 0.5, 0.5), emissive=(1, 1, 1))
    v = np.zeros(9, VERTEX)
    tri = [((0, 0, 0), (1, 0, 0), (0, 1, 0)), ((0, 0, 0), (1, 0, 0), (0, 1, 0)), ((0, 0, 0), (2, 0, 0), (0, 1, 0))]
    for i, t in enumerate(tri):
        v["position"][3 * i:3 * i + 3] = t
    f = np.zeros(3, FACE)
    f["v0"], f["v1"], f["v2"], f["material_id"] = [0, 3, 6], [1, 4, 7], [2, 5, 8], [0, 1, 2]
    refs, pmf, alias = oracle.emissive_tables(v, f, m)
    assert len(refs) == 2
    assert np.allclose(pmf, UT["emissive_pmf_3tri"], atol=1e-5)
    assert abs(refs[-1]["cdf"] - 1.0) < 1e-5


def test_reference_unit_env_pmf_and_alias(oracle):
    img = np.array([[[1, 1, 1, 1], [3, 3, 3, 1]]], np.float32)
    pmf, alias = oracle.env_tables(img)
    assert np.allclose(pmf, UT["env_pmf_2x1"], atol=1e-5)
    img4 = np.array([[[1, 0, 0, 1], [2, 0, 0, 1], [3, 0, 0, 1], [4, 0, 0, 1]]], np.float32)
    pmf, alias = oracle.env_tables(img4)
    assert len(alias) == 4 and np.all((alias["prob"] >= 0) & (alias["prob"] <= 1)) and np.all(alias["alias"] < 4)


def test_reference_unit_camera(oracle):
    import pathtracingtutorial_b200 as pt
    f = oracle.camera_frame(pt.make_camera((0, 0, 4), (0, 0, 0), (0, 1, 0), 90.0, width=800, height=800))
    assert abs(f[5] + 1) < 1e-5 and abs(f[6] - 1) < 1e-5 and abs(f[10] - 1) < 1e-5
    assert abs(f[12] - 1) < 1e-4 and abs(f[13] - 1) < 1e-5
    f = oracle.camera_frame(pt.make_camera((0, 0, 0), (1, 0, 0), (0, 1, 0), 60.0, width=1920, height=1080))
    assert np.allclose(f[3:6], [1, 0, 0], atol=1e-5)
    assert abs(f[12] - np.tan(np.radians(30))) < 1e-4 and abs(f[13] - 1920 / 1080) < 1e-4


@pytest.mark.parametrize("n,root_leaf", [(1, True), (2, True), (5, False), (100, False)])
def test_reference_unit_bvh(oracle, n, root_leaf):
    from oracle.pyoracle import VERTEX, FACE
    v = np.zeros(3 * n, VERTEX)
    step = 3.0 if n == 5 else 1.0
    for i in range(n):
        x = i * step if n != 2 else (-1.0 if i == 0 else 1.0)
        v["position"][3 * i:3 * i + 3] = [(x, 0, 0), (x + 1, 0, 0), (x + 0.5, 1, 0)]
    f = np.zeros(n, FACE)
    f["v0"], f["v1"], f["v2"] = np.arange(0, 3 * n, 3), np.arange(1, 3 * n, 3), np.arange(2, 3 * n, 3)
    nodes, faces, _ = oracle.build_bvh(v, f)
    assert bool(nodes[0]["data0"] & 0x80000000) == root_leaf
    if n == 2:
        assert nodes[0]["data1"] == 2
    assert len(faces) == n


def test_power_heuristic_values(oracle):
    # powerHeuristic(a, b) = a^2 / (a^2 + b^2) (Part_2/src/math/sampling.h:34-39)
    for a, b, want in UT["power_heuristic"]:
        assert abs(a * a / (a * a + b * b) - want) < 1e-6
