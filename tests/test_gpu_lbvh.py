"""The device BVH builder (pt_scene_build_accel_device) against its float32
restatement (oracle/lbvh_ref.py) and against the host-built reference tree.

  * bit for bit: faces in leaf order, every inner-node record, every triangle
    record, the root, depth and leaf count, and the reference-layout node
    array derived from them (pt_scene_get_bvh);
  * hits through the device-built tree on the GPU equal, bit for bit, the
    hits the oracle's traversal finds in the same tree, and have the same
    closest distances as the host-built tree;
  * renders of a device-built scene agree with renders of the host-built one
    within the noise of two independent renders, and with the FP64 oracle
    rendering the same device-built tree and light tables on the same sample
    streams to FP32 rounding;
  * a face with a vertex index out of range is reported, not traced.
"""
import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from oracle import lbvh_ref
from pathtracingtutorial_b200 import scenes
from pathtracingtutorial_b200._ffi import FACE_DTYPE, VERTEX_DTYPE
from test_lbvh_oracle import soup

pytestmark = pytest.mark.gpu


def _soup_scene(n, seed, dup=0):
    v, f = soup(n, seed, dup)
    mats = scenes._materials([scenes.default_material(base_color=(0.7, 0.7, 0.7))])
    cam = scenes.cornell_box(width=16, height=16).camera
    return pt.SceneManager.from_arrays(v, f, mats, cam, None), v, f


CASES = {
    "one_face": lambda: _soup_scene(1, 1),
    "two_faces": lambda: _soup_scene(2, 2),
    "seven_faces": lambda: _soup_scene(7, 7),
    "soup_dups": lambda: _soup_scene(5000, 5, dup=700),
    "cornell": lambda: (lambda sa: (sa.scene(), sa.vertices, sa.faces))(scenes.cornell_box(width=32, height=32)),
    "spheres": lambda: (lambda sa: (sa.scene(), sa.vertices, sa.faces))(
        scenes.icosphere_field(n_spheres=8, subdiv=3, width=32, height=18, env_size=(16, 8))),
    "spheres_large": lambda: (lambda sa: (sa.scene(), sa.vertices, sa.faces))(
        scenes.icosphere_field(n_spheres=40, subdiv=3, width=32, height=18, env_size=(16, 8))),
}
EXACT = [k for k in CASES if k != "spheres_large"]


@pytest.mark.parametrize("name", EXACT)
@pytest.mark.parametrize("max_leaf,treelet,passes,ct", [(1, 1, 1, 0.5), (8, 1, 1, 0.5), (1, 7, 1, 0.5), (8, 7, 1, 0.5),
                                                        (8, 4, 1, 0.5), (8, 7, 2, 1.0), (0, 0, 0, 0.0)])
def test_device_build_bit_exact(name, max_leaf, treelet, passes, ct):
    s, v, f = CASES[name]()
    kw = dict(builder="device", max_leaf=max_leaf, treelet=treelet, passes=passes, traversal_cost=ct)
    st = s.build_accel(**kw)
    if (max_leaf, treelet, passes, ct) == (0, 0, 0, 0.0):      # the library's defaults
        res = lbvh_ref.build(v["position"], f)
    else:
        res = lbvh_ref.build(v["position"], f, max_leaf, treelet if treelet >= 3 else 0, passes, ct)
    faces = s.faces()
    assert np.array_equal(faces.view(np.uint32), f[res["order"]].view(np.uint32))
    inner, tris, root = s.traversal_layout()
    assert root == res["root_ref"]
    assert np.array_equal(inner, res["inner"])
    assert np.array_equal(tris, lbvh_ref.tri_records(v["position"], faces, res["leaf_last"]))
    info = s.info()
    assert info["bvh_max_depth"] == res["depth"] == st["depth"]
    assert info["num_leaves"] == res["leaves"] == st["leaves"]
    assert info["num_inner_nodes"] == len(res["inner"]) == st["inner_nodes"]
    nodes = s.bvh_nodes()
    assert np.array_equal(nodes.view(np.uint32).reshape(-1, 8), lbvh_ref.reference_nodes(res, len(f)))
    # deterministic
    s.build_accel(**kw)
    inner2, tris2, _ = s.traversal_layout()
    assert np.array_equal(inner, inner2) and np.array_equal(tris, tris2)


def _rays(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 50, rng.integers(0, 3)] = 0.0
    return o, d


@pytest.mark.parametrize("name", ["cornell", "spheres_large", "soup_dups"])
def test_device_tree_hits(oracle, name):
    s, v, f = CASES[name]()
    s.build_accel(builder="device")
    s.upload_to_device(0)
    lo, hi = v["position"].min(0), v["position"].max(0)
    o, d = _rays(100000, lo - 0.5, hi + 0.5, 9)
    hits = pt.trace_closest(s, o, d)
    rays = np.zeros((len(o), 8), np.float32)
    rays[:, :3], rays[:, 4:7], rays[:, 7] = o, d, 1e30
    faces = s.faces()
    ours, _ = oracle.trace(s.bvh_nodes(), v, faces, rays)
    gpu = np.stack([hits["t"], hits["prim"].view(np.float32), hits["u"], hits["v"]], 1)
    assert (hits["prim"] >= 0).mean() > 0.05     # the soup is sparse: about 12% of its rays hit
    assert np.array_equal(gpu.view(np.uint32), ours.view(np.uint32))
    # the host-built (reference-order) tree: same closest distances
    h = CASES[name]()[0]
    h.build_accel()
    h.upload_to_device(0)
    href = pt.trace_closest(h, o, d)
    same = hits["t"].view(np.uint32) == href["t"].view(np.uint32)
    assert same.mean() > 0.999, same.mean()


def test_device_built_render_matches_host_built():
    sa = scenes.cornell_box(width=48, height=48)
    spp = 256
    imgs = {}
    for key, builder, first in (("host_a", "host", 0), ("host_b", "host", 10_000), ("dev", "device", 0)):
        s = sa.scene()
        s.build_accel(builder=builder)
        s.upload_to_device(0)
        r = pt.Renderer(s)
        r.reset_accumulation()
        s.set_frame_count(first)
        r.render_frames(spp // sa.sample_per_frame)
        r.synchronize()
        imgs[key] = r.download_current_image()[..., :3].astype(np.float64)

    def relmse(a, b):
        return float(np.mean((a - b) ** 2 / (b ** 2 + 1e-2)))

    control = relmse(imgs["host_b"], imgs["host_a"])
    assert relmse(imgs["dev"], imgs["host_a"]) < 1.5 * control + 1e-4
    assert abs(imgs["dev"].mean() / imgs["host_a"].mean() - 1) < 0.02


def test_bad_vertex_index_is_reported():
    s, v, f = _soup_scene(100, 3)
    f = f.copy()
    f["v1"][37] = len(v) + 5
    mats = scenes._materials([scenes.default_material(base_color=(0.7, 0.7, 0.7))])
    cam = scenes.cornell_box(width=16, height=16).camera
    bad = pt.SceneManager.from_arrays(v, f, mats, cam, None)
    with pytest.raises(pt.PTError, match="face 37"):
        bad.build_accel(builder="device")
    with pytest.raises(pt.PTError):
        bad.upload_to_device(0)


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_device_built_radiance_correlated_with_fp64_oracle(oracle, name):
    """The FP64 oracle renders with the device-built tree, its face order and
    its light tables (read back through the C ABI) on the same sample streams:
    the images agree to FP32 rounding, as for host-built scenes."""
    from oracle.pyoracle import Prepared
    sa = {"cornell": lambda: scenes.cornell_box(width=48, height=48),
          "spheres": lambda: scenes.icosphere_field(n_spheres=20, subdiv=3, width=64, height=36,
                                                    env_size=(128, 64))}[name]()
    spp = 8
    s = sa.scene()
    s.build_accel(builder="device")
    s.upload_to_device(0)
    img = pt.render(s, spp)[..., :3].astype(np.float64)
    base = oracle.prepare(sa)
    refs, pmf, alias = s.emissive_tables()
    prep = Prepared(base.vertices, np.ascontiguousarray(s.faces()), base.materials,
                    np.ascontiguousarray(s.bvh_nodes()), s.info()["bvh_max_depth"], refs, pmf, alias, base.env,
                    base.env_pmf, base.env_alias, base.camera_frame, base.width, base.height, base.punctual)
    (mean, _), _ = oracle.render(prep, sa.sample_per_frame, sa.max_depth, sa.sampler, frames=spp // sa.sample_per_frame,
                                 first_frame=0, precision=64, rtl=pt.DEVICE_ARG_ORDER, pcg_seed=sa.pcg_seed)
    assert mean.mean() > 0
    rel = np.abs(img - mean) / np.maximum(np.abs(mean), 1e-3)
    assert np.median(rel) < 1e-4, np.median(rel)
    assert float(np.mean((img - mean) ** 2 / (mean ** 2 + 1e-2))) < 1e-3
