"""Watertight intersection mode (PT_FLAG_WATERTIGHT; the reference has none).

Rays aimed exactly at the shared vertices and edge midpoints of a tessellated,
gently displaced grid, from above and steep enough that no such point is on
a silhouette: every one must hit some triangle.  The reference's
Moller-Trumbore test (Part_2/src/geometry/triangle.h:13-51) lets a share of
them slip through; the watertight mode (Woop, Benthin and Wald 2013 on the
shared vertices, box exits widened as in Ize 2013) lets none through.

CPU: the oracle's restatement of both modes.  GPU: the device kernels in
watertight mode against that restatement bit for bit (grid rays, and seeded
rays through a sphere field, closest and any hit), the rate at which hit ids
differ from the default mode, and a render in watertight mode correlated with
the FP64 oracle in the same mode.
"""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes


def grid_mesh(n=64, seed=3, amp=0.004):
    """(n x n) cells over [-1, 1]^2 in xz, heights uniform in +-amp, each cell
    split along a random diagonal; vertices shared between cells."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(-1, 1, n + 1)
    X, Z = np.meshgrid(xs, xs, indexing="xy")
    Y = rng.uniform(-amp, amp, X.shape)
    pos = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    idx = np.arange((n + 1) ** 2).reshape(n + 1, n + 1)
    a, b, c, d = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel(), idx[1:, 1:].ravel(), idx[1:, :-1].ravel()
    flip = rng.integers(0, 2, len(a)).astype(bool)
    t1 = np.where(flip[:, None], np.stack([a, b, d], 1), np.stack([a, b, c], 1))
    t2 = np.where(flip[:, None], np.stack([b, c, d], 1), np.stack([a, c, d], 1))
    tri = np.concatenate([t1, t2]).astype(np.uint32)
    v = np.zeros(len(pos), pt.VERTEX_DTYPE)
    v["position"] = pos
    v["normal"] = (0, 1, 0)
    f = np.zeros(len(tri), pt.FACE_DTYPE)
    f["v0"], f["v1"], f["v2"] = tri.T
    return v, f, n


def edge_rays(v, f, n, seed=5, per_target=4):
    """Rays through every interior vertex and interior edge midpoint, from
    origins 3 units away in directions at least ~56 degrees above the grid."""
    pos = v["position"]
    tri = np.stack([f["v0"], f["v1"], f["v2"]], 1)
    interior = np.arange((n + 1) ** 2).reshape(n + 1, n + 1)[1:-1, 1:-1].ravel()
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    mid = (np.float32(0.5) * (pos[e[:, 0]] + pos[e[:, 1]])).astype(np.float32)
    inner = (np.abs(mid[:, 0]) < 0.999) & (np.abs(mid[:, 2]) < 0.999)
    targets = np.repeat(np.concatenate([pos[interior], mid[inner]]), per_target, 0)
    rng = np.random.default_rng(seed)
    dirs = rng.normal(size=targets.shape)
    dirs[:, 1] = np.abs(dirs[:, 1]) + 1.5
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    o = (targets + 3.0 * dirs).astype(np.float32)
    d = (targets - o).astype(np.float32)
    d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, :3], rays[:, 4:7] = o, d
    return rays


def _misses(hits):
    return int((hits[:, 1].view(np.int32) < 0).sum())


def test_oracle_watertight_mode_has_no_leaks(oracle):
    v, f, n = grid_mesh()
    nodes, faces, _ = oracle.build_bvh(v, f)
    rays = edge_rays(v, faces, n)
    mt, _ = oracle.trace(nodes, v, faces, rays)
    wt, _ = oracle.trace(nodes, v, faces, rays, watertight=True)
    assert _misses(wt) == 0
    assert _misses(mt) > 0.01 * len(rays)          # the reference's test does leak here
    both = (mt[:, 1].view(np.int32) >= 0)
    assert np.allclose(mt[both, 0], wt[both, 0], rtol=1e-5)
    # shadow rays stopping short of the grid are never occluded; past it always
    short = np.concatenate([rays[:, :7], np.full((len(rays), 1), 2.9, np.float32)], 1)
    long_ = np.concatenate([rays[:, :7], np.full((len(rays), 1), 3.1, np.float32)], 1)
    assert not oracle.trace(nodes, v, faces, short, any_hit=True, watertight=True)[0].any()
    assert oracle.trace(nodes, v, faces, long_, any_hit=True, watertight=True)[0].all()


def test_watertight_hits_match_default_on_ordinary_rays(oracle):
    """Away from edges both modes find the same triangle (they differ only in
    rounding); the hit id differs on a small share of seeded rays."""
    sa = scenes.icosphere_field(n_spheres=20, subdiv=3, width=32, height=18, env_size=None)
    prep = oracle.prepare(sa)
    rng = np.random.default_rng(4)
    lo, hi = sa.vertices["position"].min(0), sa.vertices["position"].max(0)
    rays = np.zeros((50000, 8), np.float32)
    rays[:, :3] = rng.uniform(lo - 1, hi + 1, (50000, 3))
    rays[:, 4:7] = rng.normal(size=(50000, 3))
    mt, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays)
    wt, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays, watertight=True)
    pm, pw = mt[:, 1].view(np.int32), wt[:, 1].view(np.int32)
    assert (pm >= 0).mean() > 0.2
    assert (pm != pw).mean() < 1e-3


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _gpu_rows(hits):
    return np.stack([hits["t"], hits["prim"].view(np.float32), hits["u"], hits["v"]], 1)


@pytest.mark.gpu
def test_gpu_watertight_grid_bit_exact_and_leak_free(oracle):
    v, f, n = grid_mesh()
    s = pt.SceneManager.from_arrays(v, f, np.atleast_1d(pt.default_material()),
                                    pt.make_camera(position=(0, 3, 0.1), look_at=(0, 0, 0), width=64, height=64))
    s.build_accel()
    s.upload_to_device(0)
    faces = s.faces()
    nodes = s.bvh_nodes()
    rays = edge_rays(v, faces, n)
    o, d = rays[:, :3], rays[:, 4:7]
    mt_gpu = _gpu_rows(pt.trace_closest(s, o, d))
    s.update_settings(flags=pt.FLAG_WATERTIGHT)
    wt_gpu = _gpu_rows(pt.trace_closest(s, o, d))
    wt_ref, _ = oracle.trace(nodes, v, faces, rays, watertight=True)
    mt_ref, _ = oracle.trace(nodes, v, faces, rays)
    assert np.array_equal(wt_gpu.view(np.uint32), wt_ref.view(np.uint32))
    assert np.array_equal(mt_gpu.view(np.uint32), mt_ref.view(np.uint32))
    assert _misses(wt_gpu) == 0
    print(f"{len(rays)} rays through shared vertices and edges: default mode leaks {_misses(mt_gpu)} "
          f"({_misses(mt_gpu) / len(rays):.2%}), watertight mode 0")
    for tmax, expect in ((2.9, False), (3.1, True)):
        occ = pt.trace_any(s, o, d, np.full(len(o), tmax, np.float32))
        assert (occ == expect).all()
    # the allocation-free entry point follows the same flag
    k = pt.STATIC_TRACE_MAX_RAYS
    st = _gpu_rows(pt.trace_closest_static(s, o[:k], d[:k]))
    assert np.array_equal(st.view(np.uint32), wt_ref[:k].view(np.uint32))


@pytest.mark.gpu
def test_gpu_watertight_sphere_field_bit_exact_and_difference_rate(oracle):
    sa = scenes.icosphere_field(n_spheres=40, subdiv=3, width=64, height=36, env_size=(64, 32))
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    prep = oracle.prepare(sa)
    rng = np.random.default_rng(8)
    lo, hi = sa.vertices["position"].min(0), sa.vertices["position"].max(0)
    n = 200000
    o = rng.uniform(lo - 1, hi + 1, (n, 3)).astype(np.float32)
    o[:5000] = sa.vertices["position"][rng.integers(0, len(sa.vertices), 5000)]
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 50, rng.integers(0, 3)] = 0.0
    t = rng.uniform(0.05, 8.0, n).astype(np.float32)
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3], rays[:, 4:7], rays[:, 7] = o, d, t
    mt = pt.trace_closest(s, o, d)
    s.update_settings(flags=pt.FLAG_WATERTIGHT)
    wt = pt.trace_closest(s, o, d)
    ref, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays, watertight=True)
    assert np.array_equal(_gpu_rows(wt).view(np.uint32), ref.view(np.uint32))
    occ = pt.trace_any(s, o, d, t)
    ref_occ, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays, any_hit=True, watertight=True)
    assert np.array_equal(occ, ref_occ)
    diff = float((mt["prim"] != wt["prim"]).mean())
    print(f"hit ids differing between the default and the watertight mode: {diff:.5%} of {n} rays")
    assert diff < 1e-3


@pytest.mark.gpu
def test_gpu_watertight_render_correlated_with_fp64_oracle(oracle):
    sa = scenes.cornell_box(width=64, height=64, spp=16)
    s = sa.scene()
    s.update_settings(flags=pt.FLAG_WATERTIGHT)
    s.build_accel()
    s.upload_to_device(0)
    img = pt.render(s, sa.spp)[..., :3].astype(np.float64)
    prep = oracle.prepare(sa)
    (mean, _), _ = oracle.render(prep, sa.sample_per_frame, sa.max_depth, sa.sampler, frames=sa.spp // 4,
                                 precision=64, rtl=pt.DEVICE_ARG_ORDER, pcg_seed=sa.pcg_seed, watertight=True)
    rel = np.abs(img - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.median(rel) < 1e-4
    assert np.mean((img - mean) ** 2 / (mean ** 2 + 1e-2)) < 1e-3
