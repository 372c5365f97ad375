"""GPU parity at the benchmark configurations' own sizes, through the C ABI.

  * Cornell box at its full configuration (36 triangles, 512 x 512, 64 spp,
    depth 8, PCG with seed 1): the render against the FP64 oracle on the same
    sample streams (correlated bounds), and on disjoint sample indices a
    per-pixel noise bound |mean - R| <= 4 sigma for at least 99.9 % of pixels;
  * the 2,048,002-triangle icosphere field at 1920 x 1080: triangle ids,
    distances and barycentrics of every camera ray and of one bounce of
    extension rays, plus occlusion of shadow rays, bit for bit against the
    oracle's restatement of the reference's traversal;
  * a thin-lens camera (aperture > 0), correlated with the FP64 oracle;
  * the batched renderer (persistent kernel and per-item wavefront branches)
    against the FP64 oracle directly.

References: Part_2/src/integrators/path.cu:31-59 (camera and thin lens),
:209-242 (per-pixel loop); Part_2/src/accel/bvh_traversal.cuh:43-133.
"""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes

pytestmark = pytest.mark.gpu

EPS_REL = 1e-2   # relMSE epsilon: mean((I - R)^2 / (R^2 + eps))


def _up(sa):
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    return s


def _oracle(oracle, sa, frames, first_frame=0, prep=None):
    prep = prep or oracle.prepare(sa)
    (mean, var), cnt = oracle.render(prep, sa.sample_per_frame, sa.max_depth, sa.sampler, frames=frames,
                                     first_frame=first_frame, precision=64, rtl=pt.DEVICE_ARG_ORDER,
                                     pcg_seed=sa.pcg_seed)
    return mean, var, cnt


def _correlated(img, mean):
    img = img[..., :3].astype(np.float64)
    rel = np.abs(img - mean) / np.maximum(np.abs(mean), 1e-3)
    return float(np.median(rel)), float(np.mean((img - mean) ** 2 / (mean ** 2 + EPS_REL)))


# ---------------------------------------------------------------------------
# Cornell box, full configuration
# ---------------------------------------------------------------------------
def test_cornell_full_config_correlated_with_fp64_oracle(oracle):
    sa = scenes.cornell_box()            # 512 x 512, 64 spp, depth 8, PCG seed 1
    assert (int(sa.camera["width"]), int(sa.camera["height"]), sa.spp, sa.max_depth, sa.pcg_seed) == \
        (512, 512, 64, 8, 1)
    img = pt.render(_up(sa), sa.spp)
    mean, _, _ = _oracle(oracle, sa, frames=sa.spp // sa.sample_per_frame)
    med, rmse = _correlated(img, mean)
    assert med < 1e-4, med
    assert rmse < 1e-3, rmse


def test_cornell_full_config_per_pixel_noise_bound(oracle):
    """Independent estimates of every pixel: the GPU's 64 spp (frames 0-15)
    and the oracle's 64 spp (frames 1000-1015).  Per pixel and channel,
    sigma^2 = max(var_gpu, var_oracle) * (1/64 + 1/64), where var_gpu comes
    from the spread of the GPU's 16 frame means (4 samples each) and
    var_oracle is the oracle's per-sample variance; the larger of the two
    estimates of the same distribution's variance keeps a pixel whose rare
    bright paths only one side drew from failing on an underestimate.  At
    least 99.9 % of pixels must lie within 4 sigma in every channel."""
    sa = scenes.cornell_box()
    s = _up(sa)
    r = pt.Renderer(s)
    r.reset_accumulation()
    frames = sa.spp // sa.sample_per_frame
    means = []
    for _ in range(frames):
        r.render_batch()
        means.append(r.film.download_new()[..., :3].astype(np.float64))
    fm = np.stack(means)
    m_gpu = fm.mean(0)
    var_gpu = sa.sample_per_frame * fm.var(0, ddof=1)
    acc = r.download_current_image()[..., :3].astype(np.float64)
    assert np.allclose(acc, m_gpu, rtol=1e-5, atol=1e-6)
    m_o, var_o, _ = _oracle(oracle, sa, frames=frames, first_frame=1000)
    n = frames * sa.sample_per_frame
    sigma = np.sqrt(np.maximum(var_gpu, var_o) * (2.0 / n))
    diff = np.abs(m_gpu - m_o)
    ok = np.where(sigma > 0, diff <= 4.0 * sigma, diff <= 1e-6 * np.abs(m_o) + 1e-7)
    pix_ok = ok.all(-1)
    frac_fail = 1.0 - float(pix_ok.mean())
    print(f"per-pixel 4-sigma bound: {frac_fail * 100:.4f} % of {pix_ok.size} pixels outside")
    assert frac_fail <= 1e-3, frac_fail
    assert (m_o.sum(-1) > 0).mean() > 0.8 and np.median(sigma) > 0


# ---------------------------------------------------------------------------
# icosphere field at its full size: hit ids of camera and extension rays
# ---------------------------------------------------------------------------
def _camera_rays(cf, w, h):
    pos, fwd, rgt, up = cf[0:3], cf[3:6], cf[6:9], cf[9:12]
    y, x = np.mgrid[0:h, 0:w].astype(np.float32)
    u = (np.float32(2) * (x + np.float32(0.5)) / np.float32(w) - np.float32(1)) * cf[12] * cf[13]
    v = (np.float32(2) * (y + np.float32(0.5)) / np.float32(h) - np.float32(1)) * cf[12]
    d = (u[..., None] * rgt + v[..., None] * up + fwd).reshape(-1, 3).astype(np.float32)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    return np.ascontiguousarray(np.broadcast_to(pos, d.shape), np.float32), d


def _pack(o, d, tmax=None):
    r = np.zeros((len(o), 8), np.float32)
    r[:, :3], r[:, 4:7] = o, d
    if tmax is not None:
        r[:, 7] = tmax
    return r


def _as_rows(hits):
    return np.stack([hits["t"], hits["prim"].view(np.float32), hits["u"], hits["v"]], 1)


def test_icosphere_field_full_size_hit_ids_bit_exact(oracle):
    sa = scenes.icosphere_field()        # 2,048,002 triangles, 1920 x 1080
    assert len(sa.faces) == 2_048_002
    s = _up(sa)
    prep = oracle.prepare(sa)
    assert np.array_equal(s.faces().view(np.uint8), prep.faces.view(np.uint8))
    w, h = int(sa.camera["width"]), int(sa.camera["height"])
    o, d = _camera_rays(prep.camera_frame, w, h)
    hits = pt.trace_closest(s, o, d)
    ref, cnt = oracle.trace(prep.nodes, prep.vertices, prep.faces, _pack(o, d))
    assert np.array_equal(_as_rows(hits).view(np.uint32), ref.view(np.uint32))
    hit = hits["prim"] >= 0
    assert hit.mean() > 0.5
    # one bounce: from every camera hit, offset along the geometric normal
    # (1e-4, as path.cu's spawn offset) into the hemisphere it faces
    f = prep.faces[hits["prim"][hit]]
    p = prep.vertices["position"]
    v0, v1, v2 = p[f["v0"]], p[f["v1"]], p[f["v2"]]
    ng = np.cross(v1 - v0, v2 - v0)
    ng = (ng / np.linalg.norm(ng, axis=1, keepdims=True)).astype(np.float32)
    ng = np.where(((ng * d[hit]).sum(1) > 0)[:, None], -ng, ng).astype(np.float32)
    x = (o[hit] + hits["t"][hit][:, None] * d[hit]).astype(np.float32)
    o2 = (x + np.float32(1e-4) * ng).astype(np.float32)
    rng = np.random.default_rng(21)
    d2 = rng.normal(size=o2.shape)
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    d2 = np.where(((d2 * ng).sum(1) < 0)[:, None], -d2, d2).astype(np.float32)
    hits2 = pt.trace_closest(s, o2, d2)
    ref2, cnt2 = oracle.trace(prep.nodes, prep.vertices, prep.faces, _pack(o2, d2))
    assert np.array_equal(_as_rows(hits2).view(np.uint32), ref2.view(np.uint32))
    assert 0.05 < (hits2["prim"] >= 0).mean() < 0.95
    tmax = rng.uniform(0.05, 60.0, len(o2)).astype(np.float32)
    occ = pt.trace_any(s, o2, d2, tmax)
    ref_occ, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, _pack(o2, d2, tmax), any_hit=True)
    assert np.array_equal(occ, ref_occ)
    print(f"{len(o)} camera rays ({hit.mean():.3f} hit), {len(o2)} extension and shadow rays; "
          f"{cnt['node_pops'] + cnt2['node_pops']} node pops")


# ---------------------------------------------------------------------------
# thin-lens camera
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_thin_lens_camera_correlated_with_fp64_oracle(oracle, name):
    if name == "cornell":
        sa = scenes.cornell_box(width=96, height=96, spp=16)
        sa.camera["aperture"], sa.camera["focal_distance"] = 0.04, 1.8
    else:
        sa = scenes.icosphere_field(n_spheres=40, subdiv=3, width=96, height=54, spp=8, env_size=(128, 64))
        sa.camera["aperture"], sa.camera["focal_distance"] = 0.6, 25.0
    img = pt.render(_up(sa), sa.spp)
    mean, _, _ = _oracle(oracle, sa, frames=sa.spp // sa.sample_per_frame)
    med, rmse = _correlated(img, mean)
    assert med < 1e-4, med
    assert rmse < 1e-3, rmse
    # the lens matters: the same scene through a pinhole differs
    sa.camera["aperture"] = 0.0
    pin, _, _ = _oracle(oracle, sa, frames=sa.spp // sa.sample_per_frame)
    _, rmse_pin = _correlated(img, pin)
    assert rmse_pin > 10 * rmse, (rmse_pin, rmse)


# ---------------------------------------------------------------------------
# batched renderer against the FP64 oracle
# ---------------------------------------------------------------------------
def _batch_scenes():
    a = scenes.cornell_box(width=64, height=48, spp=16, max_depth=8)
    b = scenes.icosphere_field(n_spheres=30, subdiv=2, width=64, height=36, spp=8, max_depth=12, env_size=(128, 64))
    c = scenes.hidden_light_room(width=40, height=40, n_boxes=40, box_subdiv=2, spp=16, max_depth=10)
    return [a, b, c]


@pytest.mark.parametrize("mode", [pt.BATCH_PERSISTENT, pt.BATCH_WAVEFRONT])
def test_batch_correlated_with_fp64_oracle(oracle, mode):
    sas = _batch_scenes()
    ss = [_up(sa) for sa in sas]
    first = [0, 3, 7]
    imgs, st, cfg = pt.render_batch([(s, sa.spp, f0) for s, sa, f0 in zip(ss, sas, first)], mode=mode,
                                    autotune=False, chunk_spp=4)
    assert cfg["mode"] == mode
    for sa, img, f0 in zip(sas, imgs, first):
        mean, _, _ = _oracle(oracle, sa, frames=sa.spp // sa.sample_per_frame, first_frame=f0)
        med, rmse = _correlated(img, mean)
        assert med < 1e-4, (sa.name, med)
        assert rmse < 1e-3, (sa.name, rmse)
