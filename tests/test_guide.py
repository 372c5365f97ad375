"""Learned guiding: the FP64 CPU restatement of the network is checked by
finite differences; the CUDA forward and backward (BF16 tensor cores, FP32
accumulation) are checked against it; guided rendering stays unbiased against
the plain integrator and lowers the error at equal sample count."""
import numpy as np
import pytest

from oracle import guide_ref


def _samples(n, seed, concentrated=False):
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, 1.0, (n, 3))
    d = rng.normal(size=(n, 3))
    if concentrated:
        d[:, 2] = np.abs(d[:, 2]) * 3.0
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.exponential(1.0, n)
    return pos.astype(np.float32), w.astype(np.float32), d.astype(np.float32)


@pytest.mark.parametrize("table_log2", [10, 13])
def test_oracle_backward_matches_finite_differences(table_log2):
    prm = guide_ref.random_params(table_log2, seed=3)
    pos, w, d = _samples(48, 1)
    gw, gg = guide_ref.backward(prm, pos, w, d)
    rng = np.random.default_rng(7)
    h = 1e-6

    def fd_weight(i):
        p1, p2 = dict(prm), dict(prm)
        p1["weights"] = prm["weights"].copy(); p1["weights"][i] += h
        p2["weights"] = prm["weights"].copy(); p2["weights"][i] -= h
        return (guide_ref.loss(p1, pos, w, d) - guide_ref.loss(p2, pos, w, d)) / (2 * h)

    def fd_grid(l, e, f):
        p1, p2 = dict(prm), dict(prm)
        p1["grid"] = prm["grid"].copy(); p1["grid"][l, e, f] += h
        p2["grid"] = prm["grid"].copy(); p2["grid"][l, e, f] -= h
        return (guide_ref.loss(p1, pos, w, d) - guide_ref.loss(p2, pos, w, d)) / (2 * h)

    used = [i for i in range(guide_ref.N_WEIGHTS) if not (i >= 10240 and (i - 10240) // 64 >= 40)]
    scale_w = np.abs(gw).max()
    for i in rng.choice(used, 24, replace=False):
        assert abs(fd_weight(i) - gw[i]) <= 1e-5 * scale_w + 1e-4 * abs(gw[i]), i
    nz = np.argwhere(gg != 0)
    scale_g = np.abs(gg).max()
    for l, e, f in nz[rng.choice(len(nz), 24, replace=False)]:
        assert abs(fd_grid(l, e, f) - gg[l, e, f]) <= 1e-5 * scale_g + 1e-4 * abs(gg[l, e, f]), (l, e, f)


def test_oracle_pdf_normalised():
    """q(. | x) integrates to one over the sphere (Fibonacci quadrature)."""
    prm = guide_ref.random_params(10, seed=4, feature_scale=0.5)
    m = 200_000
    k = np.arange(m) + 0.5
    z = 1 - 2 * k / m
    phi = np.pi * (1 + 5 ** 0.5) * k
    r = np.sqrt(1 - z * z)
    dirs = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    for p in ([0.3, 0.6, 0.2], [0.9, 0.1, 0.5]):
        q = guide_ref.pdf(prm, np.tile(np.array(p, np.float32), (m, 1)), dirs)
        assert abs(q.mean() * 4 * np.pi - 1.0) < 2e-3


# ---------------------------------------------------------------------------
# GPU: kernels against the FP64 restatement
# ---------------------------------------------------------------------------

def _scene(sa):
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    return s


def _render_from(s, spp, first_frame):
    """Plain render of spp samples per pixel starting at an arbitrary frame
    (independent of the frames pt.render uses)."""
    import pathtracingtutorial_b200 as pt
    r = pt.Renderer(s)
    r.reset_accumulation()
    s.set_frame_count(first_frame)
    spf = s.settings().sample_per_frame
    for _ in range((spp + spf - 1) // spf):
        r.render_batch()
    r.synchronize()
    return r.download_current_image()


def _layer_rel(a, b):
    out = []
    for o, (r, c) in zip(guide_ref.LAYER_OFFSETS, guide_ref.LAYER_SHAPES):
        x, y = a[o:o + r * c], b[o:o + r * c]
        out.append(np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30))
    return out


def _cos(a, b):
    return float(a.ravel() @ b.ravel() / (np.linalg.norm(a) * np.linalg.norm(b)))


def _check_gradients(g, seed, concentrated):
    prm = g.params()
    pos, w, d = _samples(4096, seed, concentrated)
    gw, gg = g.backward(pos, w, d)
    # (1) against the FP64 network with the kernels' BF16 storage points: only
    #     FP32 accumulation order and FP32 transcendentals differ
    rw, rg = guide_ref.backward(prm, pos, w, d, bf16=True)
    rel = _layer_rel(gw, rw)
    assert max(rel) < 1e-2, rel
    assert _cos(gw, rw) > 0.9999
    relg = np.linalg.norm(gg - rg) / np.linalg.norm(rg)
    assert relg < 1e-2, relg
    # (2) against the exact FP64 network: BF16 activations and upstream
    #     gradients (8-bit mantissa) flip a few ReLU masks and round every layer
    xw, xg = guide_ref.backward(prm, pos, w, d)
    relx = _layer_rel(gw, xw)
    assert max(relx) < 0.2, relx
    assert _cos(gw, xw) > 0.99 and _cos(gg, xg) > 0.99
    return rel, relg


@pytest.mark.gpu
def test_guide_gradients_match_fp64_oracle_at_init():
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    s = _scene(scenes.cornell_box(width=32, height=32, spp=4))
    g = pt.Guide(s, seed=5)
    g.set_schedule(ema=0.0)   # the parameters read back are then the ones training runs on
    _check_gradients(g, 11, False)
    g.close()


@pytest.mark.gpu
def test_guide_forward_and_gradients_after_training():
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    sa = scenes.hidden_light_room(width=64, height=64, n_boxes=40, box_subdiv=2, spp=8, max_depth=8)
    s = _scene(sa)
    g = pt.Guide(s, seed=1)
    g.set_schedule(ema=0.0)   # the parameters read back are then the ones training runs on
    img, g, _ = pt.render_guided(s, train_spp=64, spp=8, guide=g)
    assert g.info()["steps"] > 0
    prm = g.params()
    # forward: pdf at world positions inside the scene bounds
    rng = np.random.default_rng(2)
    lo, inv = prm["lo"].astype(np.float64), prm["inv_extent"].astype(np.float64)
    p01 = rng.uniform(0.05, 0.95, (2048, 3)).astype(np.float32)
    world = (lo + p01 / inv).astype(np.float32)
    d = rng.normal(size=(2048, 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    q_gpu = g.pdf(world, d.astype(np.float32)).astype(np.float64)
    pn = np.clip((world - prm["lo"]) * prm["inv_extent"], 0, 1).astype(np.float32)
    q_ref = guide_ref.pdf(prm, pn, d, bf16=True)
    rel = np.abs(q_gpu - q_ref) / q_ref
    assert np.median(rel) < 1e-3 and np.quantile(rel, 0.99) < 1e-2, (np.median(rel), np.quantile(rel, 0.99))
    q_x = guide_ref.pdf(prm, pn, d)
    assert np.median(np.abs(q_gpu - q_x) / q_x) < 0.05
    _check_gradients(g, 12, True)
    g.close()


@pytest.mark.gpu
def test_guide_training_is_deterministic():
    """Two guides trained from the same seed on the same samples end with the
    same parameters bit for bit, and render the same image: the samples are
    collected in path order and every gradient is summed in fixed point."""
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    sa = scenes.hidden_light_room(width=64, height=64, n_boxes=40, box_subdiv=2, spp=16, max_depth=10)
    s = _scene(sa)
    runs = []
    for _ in range(2):
        img, g, _ = pt.render_guided(s, train_spp=64, spp=16, guide=pt.Guide(s, seed=3))
        p = g.params(with_grid=True)
        runs.append((img, p["weights"], p["grid"], g.info()["steps"], g.loss()))
        g.close()
    (i0, w0, g0, n0, l0), (i1, w1, g1, n1, l1) = runs
    assert n0 == n1 > 0
    assert np.array_equal(w0.view(np.uint32), w1.view(np.uint32))
    assert np.array_equal(g0.view(np.uint32), g1.view(np.uint32))
    assert np.array_equal(i0.view(np.uint32), i1.view(np.uint32))
    assert l0 == l1


@pytest.mark.gpu
def test_guided_render_unbiased_and_lower_error():
    """Guided vs plain on the hidden-light room at equal samples per pixel
    (256): the image means agree with an 8192-spp plain render within four
    standard errors (estimated from eight independent 32-spp parts of each
    render), and the trained guide lowers the relative MSE against it.  The
    guide trains for 4096 spp: at 64 x 64 pixels that is 16M paths, 512
    optimiser steps (one per 2^15 paths) -- about what 16 spp give at
    1024 x 1024."""
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    sa = scenes.hidden_light_room(width=64, height=64, n_boxes=40, box_subdiv=2, spp=256, max_depth=10)
    s = _scene(sa)
    ref = _render_from(s, 8192, 1_000_000)[..., :3].astype(np.float64)
    g = pt.Guide(s, seed=1)
    pt.render_guided(s, train_spp=4096, spp=4, guide=g)
    spf = sa.sample_per_frame
    parts_plain = [_render_from(s, 32, k * (32 // spf))[..., :3].astype(np.float64) for k in range(8)]
    parts_guided = [pt.render_batch([(s, 32, k * (32 // spf), None, g)])[0][0][..., :3].astype(np.float64)
                    for k in range(8)]
    plain, guided = np.mean(parts_plain, 0), np.mean(parts_guided, 0)

    def relmse(x):
        return float(np.mean((x - ref) ** 2 / (ref ** 2 + 1e-2)))

    def se(parts):
        m = np.array([p.mean() for p in parts])
        return m.std(ddof=1) / np.sqrt(len(m))

    se_ref = se(parts_plain) * np.sqrt(256 / 8192)
    for img, parts in ((plain, parts_plain), (guided, parts_guided)):
        bound = 4 * np.sqrt(se(parts) ** 2 + se_ref ** 2)
        assert abs(img.mean() - ref.mean()) < bound, (img.mean(), ref.mean(), bound)
    e_plain, e_guided = relmse(plain), relmse(guided)
    print(f"relMSE at 256 spp: plain {e_plain:.4g}, guided {e_guided:.4g}")
    assert e_guided < e_plain, (e_guided, e_plain)
    g.close()


@pytest.mark.gpu
def test_guided_render_keeps_plain_expectation_with_clearcoat_and_sky():
    """Clear-coated Disney materials under the sky and sun: the clearcoat lobe
    is sampled from its visible normals while the BSDF's pdf counts its
    normal distribution, so the guided mixture must use the sampler's own
    density to keep the plain integrator's expectation.  Guided and plain
    image means (2048 spp each, after 256 spp of training) agree within four
    standard errors from eight independent parts of each.  The sky is
    dimmed so that no sample reaches the per-sample clamp at 100, which
    removes a different share of each estimator's energy."""
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    sa = scenes.icosphere_field(n_spheres=40, subdiv=3, width=64, height=36, spp=256, env_size=(256, 128))
    sa.materials["clearcoat"] = 1.0
    sa.materials["clearcoat_roughness"] = 0.3
    sa.env[..., :3] *= 1e-3
    s = _scene(sa)
    g = pt.Guide(s, seed=1)
    pt.render_guided(s, train_spp=256, spp=4, guide=g)
    spf = sa.sample_per_frame
    parts_plain = [_render_from(s, 256, k * (256 // spf))[..., :3].astype(np.float64) for k in range(8)]
    parts_guided = [pt.render_batch([(s, 256, 50_000 + k * (256 // spf), None, g)])[0][0][..., :3]
                    .astype(np.float64) for k in range(8)]
    mp = np.array([p.mean() for p in parts_plain])
    mg = np.array([p.mean() for p in parts_guided])
    se = np.sqrt(mp.var(ddof=1) / 8 + mg.var(ddof=1) / 8)
    print(f"plain {mp.mean():.6f} guided {mg.mean():.6f} se {se:.2e}")
    assert abs(mp.mean() - mg.mean()) < 4 * se, (mp.mean(), mg.mean(), se)
    g.close()


@pytest.mark.gpu
def test_guide_inference_kinds_agree_with_oracle():
    """The three ways of evaluating the network while rendering -- one fused
    mma.sync kernel, the encoding kernel then the MLP on mma.sync, and the
    encoding kernel then the MLP on the tcgen05 tensor cores -- give the
    FP64 oracle's densities (with the kernels' BF16 storage points) within
    the fused kernel's bounds; the two mma.sync kinds agree to FP32 rounding,
    and guided renders with each kind agree with the fused kind's."""
    import pathtracingtutorial_b200 as pt
    from pathtracingtutorial_b200 import scenes
    sa = scenes.hidden_light_room(width=64, height=64, n_boxes=40, box_subdiv=2, spp=8, max_depth=8)
    s = _scene(sa)
    _, g, _ = pt.render_guided(s, train_spp=64, spp=4)
    prm = g.params()
    rng = np.random.default_rng(7)
    lo, inv = prm["lo"].astype(np.float64), prm["inv_extent"].astype(np.float64)
    # 5512 queries: several 128-query tiles and a ragged last one; 512 of them
    # at the top of the unit cube and beyond it (clamped), where the dense
    # levels' cells reach the last layer of their index range
    p01 = np.concatenate([rng.uniform(0.02, 0.98, (5000, 3)),
                          rng.uniform(0.985, 1.02, (512, 3))]).astype(np.float32)
    world = (lo + p01 / inv).astype(np.float32)
    d = rng.normal(size=(len(p01), 3)); d /= np.linalg.norm(d, axis=1, keepdims=True)
    pn = np.clip((world - prm["lo"]) * prm["inv_extent"], 0, 1).astype(np.float32)
    q_ref = guide_ref.pdf(prm, pn, d, bf16=True)
    q, img = {}, {}
    for kind in (pt.Guide.INFER_FUSED, pt.Guide.INFER_SPLIT_MMA, pt.Guide.INFER_SPLIT_TC):
        g.set_inference(kind)
        q[kind] = g.pdf(world, d.astype(np.float32)).astype(np.float64)
        rel = np.abs(q[kind] - q_ref) / q_ref
        assert np.median(rel) < 1e-3 and np.quantile(rel, 0.99) < 1e-2, (kind, np.median(rel), np.quantile(rel, 0.99))
        img[kind] = pt.render_batch([(s, 16, 1000, None, g)])[0][0][..., :3].astype(np.float64)
    assert np.max(np.abs(q[pt.Guide.INFER_SPLIT_MMA] - q[pt.Guide.INFER_FUSED]) / q[pt.Guide.INFER_FUSED]) < 1e-5
    rel_tc = np.abs(q[pt.Guide.INFER_SPLIT_TC] - q[pt.Guide.INFER_FUSED]) / q[pt.Guide.INFER_FUSED]
    assert np.median(rel_tc) < 1e-4 and np.max(rel_tc) < 1e-2, (np.median(rel_tc), np.max(rel_tc))
    base = img[pt.Guide.INFER_FUSED]
    for kind in (pt.Guide.INFER_SPLIT_MMA, pt.Guide.INFER_SPLIT_TC):
        # same sample streams: only directions whose lobe or density choice sits
        # on an FP32 rounding boundary can differ
        assert abs(img[kind].mean() - base.mean()) < 0.01 * base.mean(), (kind, img[kind].mean(), base.mean())
        assert np.mean(np.abs(img[kind] - base)) < 0.02 * base.mean(), (kind, np.mean(np.abs(img[kind] - base)))
    g.close()

