"""The GPU BVH builder's float32 restatement (oracle/lbvh_ref.py) on its own:
Morton codes of known points, trees (with and without treelet restructuring)
that are valid BVHs, restructuring that lowers the SAH cost, and traversal
that finds the same closest hits as in the reference-order tree (both
traversed by the oracle's C restatement of the reference's traversal)."""
import numpy as np
import pytest

from oracle import lbvh_ref
from pathtracingtutorial_b200 import scenes
from pathtracingtutorial_b200._ffi import FACE_DTYPE, VERTEX_DTYPE


def soup(n, seed, dup=0):
    """n random triangles in the unit cube; `dup` of them repeated exactly
    (equal Morton codes)."""
    rng = np.random.default_rng(seed)
    c = rng.uniform(0, 1, (n, 1, 3))
    p = (c + rng.normal(0, 0.02, (n, 3, 3))).astype(np.float32)
    if dup:
        p[-dup:] = p[:dup]
    v = np.zeros(3 * n, VERTEX_DTYPE)
    v["position"] = p.reshape(-1, 3)
    f = np.zeros(n, FACE_DTYPE)
    f["v0"], f["v1"], f["v2"] = np.arange(0, 3 * n, 3), np.arange(1, 3 * n, 3), np.arange(2, 3 * n, 3)
    return v, f


def test_morton_known_values():
    lo = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 1]], np.float32)
    codes = lbvh_ref.morton_codes(lo, lo)
    # centre bounds [0, 1]: 1.0 quantises to 2^21 - 1 on its axis
    full = (1 << 21) - 1
    x = sum(1 << (3 * b + 2) for b in range(21))
    assert codes[0] == 0
    assert codes[1] == x and codes[2] == x >> 1 and codes[3] == x >> 2
    assert codes[4] == (1 << 63) - 1
    assert full == 2097151


@pytest.mark.parametrize("treelet,passes,ct", [(0, 1, 0.5), (7, 1, 0.5), (7, 2, 1.0)])
@pytest.mark.parametrize("n,dup,max_leaf", [(1, 0, 8), (2, 0, 8), (7, 0, 8), (500, 0, 8), (1500, 300, 8),
                                            (1500, 0, 1), (1500, 0, 4)])
def test_oracle_tree_is_a_bvh(n, dup, max_leaf, treelet, passes, ct):
    v, f = soup(n, n + dup, dup)
    res = lbvh_ref.build(v["position"], f, max_leaf, treelet, passes, ct)
    lo, hi = lbvh_ref.face_boxes(v["position"], f)
    order = res["order"]
    assert sorted(order.tolist()) == list(range(n))
    nodes = lbvh_ref.reference_nodes(res, n).view(np.float32).reshape(-1, 8)
    raw = nodes.view(np.uint32)
    seen = np.zeros(n, int)
    stack = [(0, 0)]
    depth = 0
    while stack:
        k, d = stack.pop()
        depth = max(depth, d)
        nlo, nhi = nodes[k, :3], nodes[k, 4:7]
        if raw[k, 3] & lbvh_ref.LEAF:
            first, cnt = int(raw[k, 3]) & 0x7fffffff, int(raw[k, 7])
            assert 1 <= cnt <= max(max_leaf, 1) or k == 0 and n <= max_leaf
            seen[first:first + cnt] += 1
            fl, fh = lo[order[first:first + cnt]], hi[order[first:first + cnt]]
            assert np.array_equal(nlo, fl.min(0)) and np.array_equal(nhi, fh.max(0))
        else:
            for c in (int(raw[k, 3]), int(raw[k, 7])):
                assert np.all(nodes[c, :3] >= nlo) and np.all(nodes[c, 4:7] <= nhi)
                stack.append((c, d + 1))
    assert np.all(seen == 1)
    assert depth == res["depth"]


def test_restructuring_lowers_sah_cost():
    v, f = soup(2000, 11)
    plain = lbvh_ref.build(v["position"], f, 8, 0)["sah_cost"]
    opt = lbvh_ref.build(v["position"], f, 8, 7)["sah_cost"]
    assert opt < 0.95 * plain, (opt, plain)


@pytest.mark.parametrize("name", ["cornell", "spheres"])
def test_oracle_tree_finds_the_reference_tree_hits(oracle, name):
    sa = {"cornell": lambda: scenes.cornell_box(width=32, height=32),
          "spheres": lambda: scenes.icosphere_field(n_spheres=6, subdiv=3, width=32, height=18,
                                                    env_size=(16, 8))}[name]()
    res = lbvh_ref.build(sa.vertices["position"], sa.faces)
    faces = sa.faces[res["order"]]
    nodes = lbvh_ref.reference_nodes(res, len(faces))
    prep = oracle.prepare(sa)
    lo, hi = sa.vertices["position"].min(0), sa.vertices["position"].max(0)
    rng = np.random.default_rng(3)
    n = 20000
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = rng.uniform(lo, hi, (n, 3))
    rays[:, 4:7] = rng.normal(size=(n, 3))
    rays[:, 7] = 1e30
    ours, _ = oracle.trace(np.ascontiguousarray(nodes), sa.vertices, faces, rays)
    ref, _ = oracle.trace(prep.nodes, prep.vertices, prep.faces, rays)
    assert (ref[:, 1].view(np.int32) >= 0).mean() > 0.3
    same_t = ours[:, 0].view(np.uint32) == ref[:, 0].view(np.uint32)
    assert same_t.mean() > 0.999, same_t.mean()
    # the same triangle, named by its vertex indices (the two trees order faces
    # differently), except where two coplanar triangles overlap (a tie at equal t,
    # e.g. the cornell box's blocks standing on the floor)
    hit = (ref[:, 1].view(np.int32) >= 0) & same_t
    a = faces[ours[hit, 1].view(np.int32)]
    b = prep.faces[ref[hit, 1].view(np.int32)]
    diff = np.nonzero(a[["v0", "v1", "v2"]] != b[["v0", "v1", "v2"]])[0]
    P = sa.vertices["position"].astype(np.float64)
    for i in diff:
        pa = P[[a[i]["v0"], a[i]["v1"], a[i]["v2"]]]
        pb = P[[b[i]["v0"], b[i]["v1"], b[i]["v2"]]]
        nrm = np.cross(pa[1] - pa[0], pa[2] - pa[0])
        nrm /= np.linalg.norm(nrm)
        assert np.abs((pb - pa[0]) @ nrm).max() < 1e-5
    assert len(diff) < 0.01 * hit.sum()
