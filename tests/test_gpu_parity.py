"""GPU parity: the CUDA path against the oracle, through the C ABI.

Integer work (sampler streams, hit triangle ids) must match bit for bit.
Radiance is compared with the FP64 oracle:
  * correlated: same pixels, same sample indices, same sampler streams -- the
    two estimates differ only by FP32-vs-FP64 rounding and the rare branch it
    flips, so the bound is tight (median relative error < 1e-4; whole-image
    relMSE < 1e-3);
  * independent: disjoint sample indices -- the squared per-pixel
    differences must add up to at most their expected value (the sum of both
    estimates' variances; ratio < 1.4, and > 0.6 for the independent PCG
    sampler -- Sobol's stratification makes the error smaller than the
    variance predicts), and the means of the image and of its four quadrants
    agree within 4 standard errors.  (Per-pixel or per-tile z-scores are not
    used: with a few dozen samples the variance estimates of heavy-tailed
    pixels are too noisy for a normal test.)
"""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes

pytestmark = pytest.mark.gpu

EPS_REL = 1e-2   # relMSE epsilon: mean((I - R)^2 / (R^2 + eps))


def _scene(sa):
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    return s


def _rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 50, rng.integers(0, 3)] = 0.0       # axis-parallel directions exercise the NaN slab path
    t = rng.uniform(0.05, 8.0, n).astype(np.float32)
    return o, d, t


@pytest.mark.parametrize("sampler", [pt.SAMPLER_PCG, pt.SAMPLER_SOBOL])
@pytest.mark.parametrize("frame,sif", [(0, 0), (3, 2), (1000, 3)])
def test_sampler_streams_bit_exact(oracle, sampler, frame, sif):
    gpu = pt.sampler_stream(sampler, 67, 23, frame, 4, sif, 24)
    ref = oracle.sampler_stream(sampler, 67, 23, frame, 4, sif, 24)
    assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32))


def test_pcg_user_seed_changes_stream(oracle):
    a = pt.sampler_stream(pt.SAMPLER_PCG, 16, 16, 0, 4, 0, 8, pcg_seed=1)
    assert np.array_equal(a.view(np.uint32), oracle.sampler_stream(pt.SAMPLER_PCG, 16, 16, 0, 4, 0, 8, 1).view(np.uint32))
    b = pt.sampler_stream(pt.SAMPLER_PCG, 16, 16, 0, 4, 0, 8, pcg_seed=0)
    assert not np.array_equal(a, b)


SCENES = {
    "cornell": lambda: scenes.cornell_box(width=64, height=64),
    "room": lambda: scenes.hidden_light_room(width=48, height=48, n_boxes=60, box_subdiv=3),
    "spheres": lambda: scenes.icosphere_field(n_spheres=40, subdiv=3, width=64, height=36, env_size=(128, 64)),
}


@pytest.mark.parametrize("name", list(SCENES))
def test_hit_ids_bit_exact(oracle, name):
    sa = SCENES[name]()
    s = _scene(sa)
    prep = oracle.prepare(sa)
    lo, hi = sa.vertices["position"].min(0), sa.vertices["position"].max(0)
    o, d, t = _rays(30000, lo, hi, 7)
    hits = pt.trace_closest(s, o, d)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, :3], rays[:, 4:7], rays[:, 7] = o, d, t
    ref, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays)
    gpu = np.stack([hits["t"], hits["prim"].view(np.float32), hits["u"], hits["v"]], 1)
    assert (hits["prim"] >= 0).mean() > 0.2
    assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32))
    occ = pt.trace_any(s, o, d, t)
    ref_occ, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays, any_hit=True)
    assert np.array_equal(occ, ref_occ)


def test_hit_ids_bit_exact_large_scene(oracle):
    """Seeded rays through a 51,202-triangle displaced-sphere field (BVH depth
    19): origins inside and outside the spheres, directions of every octant,
    plus rays whose origin lies on a bounding-box plane."""
    sa = scenes.icosphere_field(n_spheres=40, subdiv=3, width=64, height=36, env_size=(64, 32))
    s = _scene(sa)
    prep = oracle.prepare(sa)
    lo, hi = sa.vertices["position"].min(0), sa.vertices["position"].max(0)
    o, d, t = _rays(200000, lo - 1.0, hi + 1.0, 11)
    o[:2000] = sa.vertices["position"][np.random.default_rng(5).integers(0, len(sa.vertices), 2000)]
    hits = pt.trace_closest(s, o, d)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, :3], rays[:, 4:7], rays[:, 7] = o, d, t
    ref, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays)
    gpu = np.stack([hits["t"], hits["prim"].view(np.float32), hits["u"], hits["v"]], 1)
    assert (hits["prim"] >= 0).mean() > 0.2
    assert np.array_equal(gpu.view(np.uint32), ref.view(np.uint32))
    occ = pt.trace_any(s, o, d, t)
    ref_occ, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays, any_hit=True)
    assert np.array_equal(occ, ref_occ)


def test_camera_rays_hit_ids(oracle):
    """Primary rays generated on the host in the reference's arithmetic."""
    sa = scenes.icosphere_field(n_spheres=60, subdiv=3, width=96, height=54, env_size=(64, 32))
    s = _scene(sa)
    prep = oracle.prepare(sa)
    cf = prep.camera_frame
    pos, fwd, rgt, up = cf[0:3], cf[3:6], cf[6:9], cf[9:12]
    y, x = np.mgrid[0:54, 0:96].astype(np.float32)
    u = (np.float32(2) * (x + np.float32(0.5)) / np.float32(96) - np.float32(1)) * cf[12] * cf[13]
    v = (np.float32(2) * (y + np.float32(0.5)) / np.float32(54) - np.float32(1)) * cf[12]
    d = (u[..., None] * rgt + v[..., None] * up + fwd).reshape(-1, 3).astype(np.float32)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    o = np.broadcast_to(pos, d.shape).astype(np.float32)
    hits = pt.trace_closest(s, o, d)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, :3], rays[:, 4:7] = o, d
    ref, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays)
    assert np.array_equal(hits["prim"], ref[:, 1].view(np.int32))
    assert np.array_equal(hits["t"].view(np.uint32), ref[:, 0].view(np.uint32))


def test_bsdf_table_matches_oracle(oracle):
    rng = np.random.default_rng(3)
    mats = [pt.default_material(base_color=tuple(rng.uniform(0, 1, 3)), metallic=rng.uniform(0, 1),
                                roughness=rng.uniform(0.05, 1), clearcoat=rng.uniform(0, 1),
                                sheen=rng.uniform(0, 1), subsurface=rng.uniform(0, 1),
                                spec_trans=rng.uniform(0, 1) * (i % 3 == 0), anisotropic=rng.uniform(0, 0.9))
            for i in range(16)]
    m = np.zeros(len(mats), pt.MATERIAL_DTYPE)
    for i, x in enumerate(mats):
        m[i] = x
    sa = scenes.cornell_box(width=8, height=8)
    s = pt.SceneManager.from_arrays(sa.vertices, sa.faces, m, sa.camera)
    s.build_accel()
    s.upload_to_device(0)
    n = 20000
    def unit(k):
        v = rng.normal(size=(n, 3))
        return v / np.linalg.norm(v, axis=1, keepdims=True)
    N = unit(0)
    wo = unit(1); wo = np.where((wo * N).sum(1, keepdims=True) < 0, -wo, wo)
    wi = unit(2)
    rec = np.zeros((n, 13), np.float32)
    rec[:, 0] = rng.integers(0, len(mats), n)
    rec[:, 1:4], rec[:, 4:7], rec[:, 7:10] = wo, wi, N
    gpu = pt.bsdf_eval(s, rec)
    ref = oracle.bsdf_eval(m, rec)
    ok = np.isclose(gpu, ref, rtol=2e-4, atol=1e-6)
    assert ok.mean() > 0.999, ok.mean()
    assert (ref[:, 3] > 0).mean() > 0.3


def _oracle_mean(oracle, sa, frames, first_frame=0, rtl=None):
    prep = oracle.prepare(sa)
    (mean, var), cnt = oracle.render(prep, sa.sample_per_frame, sa.max_depth, sa.sampler, frames=frames,
                                     first_frame=first_frame, precision=64,
                                     rtl=pt.DEVICE_ARG_ORDER if rtl is None else rtl, pcg_seed=sa.pcg_seed)
    return mean, var, cnt


def _relmse(img, ref):
    return float(np.mean((img - ref) ** 2 / (ref ** 2 + EPS_REL)))


@pytest.mark.parametrize("name,spp", [("cornell", 16), ("spheres", 8), ("room", 8)])
def test_radiance_correlated_with_fp64_oracle(oracle, name, spp):
    sa = SCENES[name]()
    sa.spp = spp
    img = pt.render(_scene(sa), spp)[..., :3].astype(np.float64)
    mean, var, _ = _oracle_mean(oracle, sa, frames=spp // sa.sample_per_frame)
    rel = np.abs(img - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert _relmse(img, mean) < 1e-3, _relmse(img, mean)


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_radiance_independent_samples_unbiased(oracle, name):
    sa = SCENES[name]()
    spp = 64
    img = pt.render(_scene(sa), spp)[..., :3].astype(np.float64)
    # oracle on disjoint sample indices (frames 1000.. instead of 0..)
    frames = 64 // sa.sample_per_frame
    mean, var, _ = _oracle_mean(oracle, sa, frames=frames, first_frame=1000)
    n_ref = frames * sa.sample_per_frame
    var = np.maximum(var, 0.0)
    # (1) squared differences against their expectation
    ratio = ((img - mean) ** 2).sum() / (var * (1.0 / spp + 1.0 / n_ref)).sum()
    lo = 0.6 if sa.sampler == pt.SAMPLER_PCG else 0.0
    assert lo < ratio < 1.4, ratio
    # (2) means of the image and of its quadrants
    h, w = img.shape[0], img.shape[1]
    for ys, xs in [(slice(0, h), slice(0, w)), (slice(0, h // 2), slice(0, w // 2)), (slice(0, h // 2), slice(w // 2, w)),
                   (slice(h // 2, h), slice(0, w // 2)), (slice(h // 2, h), slice(w // 2, w))]:
        a, m, v = img[ys, xs], mean[ys, xs], var[ys, xs]
        diff = a.mean() - m.mean()
        se_mean = np.sqrt((v.mean() / spp + v.mean() / n_ref) / a[..., 0].size)
        assert abs(diff) < 4 * se_mean * np.sqrt(3) + 1e-6, (diff, se_mean)


def test_render_deterministic_and_graph_equivalent():
    sa = SCENES["cornell"]()
    s = _scene(sa)
    a = pt.render(s, 8)
    b = pt.render(s, 8)
    assert np.array_equal(a, b)
    s.update_settings(flags=pt.FLAG_NO_GRAPH)
    c = pt.render(s, 8)
    assert np.array_equal(a, c)
    s.update_settings(flags=pt.FLAG_STAGE_TIMING | pt.FLAG_COUNT_TRAVERSAL)
    d, st = pt.render(s, 8, stats=True)
    assert np.array_equal(a, d)
    assert st["extend_ms"] > 0 and st["node_visits"] > 0


def test_ray_counts_match_oracle(oracle):
    """The GPU traces exactly as many camera + extension rays as the oracle when
    the per-path decisions agree (PCG, cornell: same streams, same order)."""
    sa = SCENES["cornell"]()
    _, st = pt.render(_scene(sa), 8, stats=True)
    _, _, cnt = _oracle_mean(oracle, sa, frames=2)
    gpu_rays = st["camera_rays"] + st["extension_rays"]
    assert abs(gpu_rays - cnt["closest_rays"]) <= 1e-3 * cnt["closest_rays"]
    assert st["paths"] == cnt["paths"]
