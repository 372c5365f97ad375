"""TEST INFRASTRUCTURE: float32 restatement of the GPU BVH builder.

The device builder (pathtracingtutorial_b200/csrc/lbvh.cu) has no reference
counterpart -- the reference builds its SAH tree on the host
(Part_2/src/accel/bvh_builder.cpp:56-221), and host_prep.cpp reproduces that
one -- so this module is the CPU judge of the device build.  Only tests/
import it.  It computes the same tree by a different route and must agree bit
for bit:

  face box = min/max of the three positions; centre c = 0.5 (lo + hi);
  centre bounds [cmin, cmax] over all faces; per axis s = 2^21 / (cmax - cmin)
      (0 when the extent is 0), q = clamp(floor((c - cmin) s), 0, 2^21 - 1);
  code: bit b of qx at 3b+2, of qy at 3b+1, of qz at 3b (a plain bit loop);
  faces stably sorted by code;
  radix tree, built TOP-DOWN here (the device builds it bottom-up by Karras's
      per-node search): the key of sorted position i is (code << 32) | i; the
      node covering [f, l] splits after the last position whose key has a 0 at
      the highest bit where keys f and l differ; its children are the leaf
      gamma (if gamma == f) or inner node gamma, and the leaf gamma + 1 (if
      gamma + 1 == l) or inner node gamma + 1; the root is inner node 0;
  post-order: box = union of the children; A = dx dy + dy dz + dz dx;
      tree cost = (0.5 A + cost_left) + cost_right (a single face costs its A),
      leaf cost = count * A, the node becomes a leaf when count <= min(3,
      max_leaf) (the reference's LeafThreshold rule, bvh_builder.cpp:10,99) or
      when count <= max_leaf and leaf cost <= tree cost;
  surviving inner nodes (no collapsed ancestor, not collapsed) are numbered
      in increasing inner-node index; each becomes one 16-word record.
All float arithmetic is numpy float32, one rounding per operation, in the
device's order.
"""
from __future__ import annotations

import bisect

import numpy as np

F = np.float32
LEAF = 0x80000000


def face_boxes(positions: np.ndarray, faces: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    p = positions.astype(np.float32)
    v = np.stack([faces["v0"], faces["v1"], faces["v2"]], axis=1).astype(np.int64)
    t = p[v]                                     # [n, 3, 3]
    lo = np.minimum(np.minimum(t[:, 0], t[:, 1]), t[:, 2])
    hi = np.maximum(np.maximum(t[:, 0], t[:, 1]), t[:, 2])
    return lo, hi


def morton_codes(lo: np.ndarray, hi: np.ndarray) -> np.ndarray:
    c = (lo + hi) * F(0.5)
    cmin, cmax = c.min(axis=0), c.max(axis=0)
    q = np.zeros(c.shape, np.uint64)
    for a in range(3):
        ext = F(cmax[a] - cmin[a])
        s = F(F(2097152.0) / ext) if ext > 0 else F(0.0)
        t = np.floor((c[:, a] - cmin[a]) * s).astype(np.float32)
        q[:, a] = np.clip(t, 0.0, 2097151.0).astype(np.uint64)
    code = np.zeros(len(c), np.uint64)
    for b in range(21):
        for a in range(3):
            bit = (q[:, a] >> np.uint64(b)) & np.uint64(1)
            code |= bit << np.uint64(3 * b + 2 - a)
    return code


def _half_area(lo, hi) -> np.float32:
    dx, dy, dz = F(hi[0] - lo[0]), F(hi[1] - lo[1]), F(hi[2] - lo[2])
    return F(F(F(dx * dy) + F(dy * dz)) + F(dz * dx))


def build(positions: np.ndarray, faces: np.ndarray, max_leaf: int = 8) -> dict:
    """The device builder's outputs: order (sorted face index per position),
    inner (uint32[k, 16]), leaf_last (positions whose record ends a leaf),
    root_ref, root box, depth, leaves."""
    n = len(faces)
    lo, hi = face_boxes(positions, faces)
    codes = morton_codes(lo, hi)
    order = np.argsort(codes, kind="stable")
    keys = [(int(codes[order[i]]) << 32) | i for i in range(n)]
    slo, shi = lo[order], hi[order]
    m = n - 1

    # top-down radix tree (inner node index = the split rule's numbering)
    child = np.zeros((max(m, 0), 2), np.uint64)
    rng = np.zeros((max(m, 0), 2), np.int64)
    parent = np.full(max(m, 0), -1, np.int64)
    post = []
    if m > 0:
        stack = [(0, 0, n - 1)]
        while stack:
            node, f, l = stack.pop()
            rng[node] = (f, l)
            p = (keys[f] ^ keys[l]).bit_length() - 1
            thr = (keys[l] >> p) << p
            gamma = bisect.bisect_left(keys, thr, f, l + 1) - 1
            post.append(node)
            kids = []
            for c, (cf, cl) in ((gamma, (f, gamma)), (gamma + 1, (gamma + 1, l))):
                if cf == cl:
                    kids.append(LEAF | c)
                else:
                    kids.append(c)
                    parent[c] = node
                    stack.append((c, cf, cl))
            child[node] = kids
    post.reverse()   # children before parents

    nlo = np.zeros((max(m, 0), 3), np.float32)
    nhi = np.zeros((max(m, 0), 3), np.float32)
    cost = np.zeros(max(m, 0), np.float32)
    cnt = np.zeros(max(m, 0), np.int64)
    col = np.zeros(max(m, 0), bool)

    def info(c):
        c = int(c)
        if c & LEAF:
            p = c & ~LEAF
            return slo[p], shi[p], _half_area(slo[p], shi[p]), 1
        return nlo[c], nhi[c], cost[c], int(cnt[c])

    for node in post:
        la, ha, ca, na = info(child[node, 0])
        lb, hb, cbb, nb = info(child[node, 1])
        blo, bhi = np.minimum(la, lb), np.maximum(ha, hb)
        area = _half_area(blo, bhi)
        tree = F(F(F(F(0.5) * area) + ca) + cbb)
        k = na + nb
        leaf = F(F(k) * area)
        c_ = k <= min(max_leaf, 3) or (k <= max_leaf and leaf <= tree)
        nlo[node], nhi[node], cnt[node], col[node] = blo, bhi, k, c_
        cost[node] = leaf if c_ else tree

    keep = np.zeros(max(m, 0), bool)
    depth = np.zeros(max(m, 0), np.int64)
    for node in reversed(post):                  # parents before children
        par = parent[node]
        if col[node] or (par >= 0 and not keep[par]):
            continue
        keep[node] = True
        depth[node] = 0 if par < 0 else depth[par] + 1
    scan = np.cumsum(keep) - keep
    kept = int(keep.sum())

    inner = np.zeros((kept, 16), np.uint32)
    leaf_last = []

    def ref(c):
        c = int(c)
        if c & LEAF:
            p = c & ~LEAF
            leaf_last.append(p)
            return slo[p], shi[p], c
        if col[c]:
            leaf_last.append(int(rng[c, 1]))
            return nlo[c], nhi[c], LEAF | int(rng[c, 0])
        return nlo[c], nhi[c], int(scan[c])

    for i in range(max(m, 0)):
        if not keep[i]:
            continue
        l0, h0, r0 = ref(child[i, 0])
        l1, h1, r1 = ref(child[i, 1])
        d = nhi[i] - nlo[i]
        axis = 0 if (d[0] > d[1] and d[0] > d[2]) else (1 if d[1] > d[2] else 2)
        c0 = F(F(l0[axis] + h0[axis]) * F(0.5))
        c1 = F(F(l1[axis] + h1[axis]) * F(0.5))
        fl = np.array([l0[0], l0[1], l0[2], h0[0], h0[1], h0[2], l1[0], l1[1], l1[2], h1[0], h1[1], h1[2]],
                      np.float32)
        inner[scan[i], :12] = fl.view(np.uint32)
        inner[scan[i], 12:] = (r0, r1, axis | (4 if c0 < c1 else 0), 0)

    if kept == 0:
        root_ref = LEAF
        leaf_last = [n - 1]
        rlo, rhi = (nlo[0], nhi[0]) if m > 0 else (slo[0], shi[0])
    else:
        root_ref = 0
        rlo, rhi = nlo[0], nhi[0]
    return {"order": order, "inner": inner, "leaf_last": np.array(sorted(leaf_last), np.int64),
            "root_ref": root_ref, "root_lo": rlo, "root_hi": rhi,
            "depth": int(depth[keep].max() + 1) if kept else 0, "leaves": len(leaf_last)}


def tri_records(positions: np.ndarray, faces_sorted: np.ndarray, leaf_last: np.ndarray) -> np.ndarray:
    """uint32[n, 12]: v0, v1 - v0, v2 - v0, flags (bit 0 = last of its leaf), 0, 0."""
    p = positions.astype(np.float32)
    v0 = p[faces_sorted["v0"].astype(np.int64)]
    e1 = p[faces_sorted["v1"].astype(np.int64)] - v0
    e2 = p[faces_sorted["v2"].astype(np.int64)] - v0
    out = np.zeros((len(faces_sorted), 12), np.uint32)
    out[:, 0:3] = v0.view(np.uint32)
    out[:, 3:6] = e1.view(np.uint32)
    out[:, 6:9] = e2.view(np.uint32)
    out[leaf_last, 9] = 1
    return out


def reference_nodes(res: dict, n_faces: int) -> np.ndarray:
    """The tree in the reference's BVHNode layout (uint32[k, 8]: bmin xyz,
    data0, bmax xyz, data1): inner node k keeps index k, leaves follow in the
    order their parents list them, a node's box is the one its parent carries."""
    inner = res["inner"]
    last = set(int(x) for x in res["leaf_last"])

    def count(first):
        i = first
        while i not in last:
            i += 1
        return i - first + 1

    def box(lo, hi):
        return np.concatenate([np.asarray(lo, np.float32), np.asarray(hi, np.float32)]).view(np.uint32)

    if res["root_ref"] & LEAF:
        b = box(res["root_lo"], res["root_hi"])
        return np.array([[b[0], b[1], b[2], res["root_ref"], b[3], b[4], b[5], count(res["root_ref"] & ~LEAF)]],
                        np.uint32)
    k = len(inner)
    nodes = [[0] * 8 for _ in range(k)]
    b = box(res["root_lo"], res["root_hi"])
    nodes[0][0:3], nodes[0][4:7] = b[0:3], b[3:6]
    for i in range(k):
        idx = []
        for c in range(2):
            w = inner[i, 6 * c: 6 * c + 6]
            ref = int(inner[i, 12 + c])
            if ref & LEAF:
                idx.append(len(nodes))
                nodes.append([w[0], w[1], w[2], ref, w[3], w[4], w[5], count(ref & ~LEAF)])
            else:
                idx.append(ref)
                nodes[ref][0:3], nodes[ref][4:7] = w[0:3], w[3:6]
        nodes[i][3], nodes[i][7] = idx
    return np.array(nodes, np.uint32)
