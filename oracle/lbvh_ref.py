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
  every inner node after its subtree (the device's bottom-up order): with
      treelet >= 3 its treelet is re-topologised first (see restructure:
      open the largest-area inner leaf until `treelet` leaves, dynamic
      programming over the leaf subsets, the first strict minimum in
      descending-submask order of the splits holding the lowest leaf, inner
      nodes reused depth first from a LIFO stack); then box = union of the
      children; A = dx dy + dy dz + dz dx;
      tree cost = ct A + (cost_left + cost_right) (ct = traversal_cost, 1.0
      by default as on the device, the reference's model has 0.5; a single
      face costs its A),
      leaf cost = count * A, the node becomes a leaf when count <= min(3,
      max_leaf) (the reference's LeafThreshold rule, bvh_builder.cpp:10,99) or
      when count <= max_leaf and leaf cost <= tree cost;
  surviving inner nodes (no collapsed ancestor, not collapsed) are numbered
      in increasing inner-node index; each becomes one 16-word record; faces
      take their depth-first position in the final tree.
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


def _node_cost(area, children, cnt, min_leaf, max_leaf, ct=F(0.5)):
    tree = F(F(F(ct) * area) + children)
    leaf = F(F(cnt) * area)
    col = cnt <= min_leaf or (cnt <= max_leaf and leaf <= tree)
    return (leaf if col else tree), col


def _low_index(x: int) -> int:
    return (x & -x).bit_length() - 1


def build(positions: np.ndarray, faces: np.ndarray, max_leaf: int = 8, treelet: int = 7, passes: int = 3,
          traversal_cost: float = 1.0) -> dict:
    """The device builder's outputs: order (face index per final position),
    inner (uint32[k, 16]), leaf_last (positions whose record ends a leaf),
    root_ref, root box, depth, leaves.  treelet < 3: no restructuring;
    otherwise `passes` bottom-up passes, each over the tree the last one left."""
    n = len(faces)
    min_leaf = min(max_leaf, 3)
    ct = F(traversal_cost)
    lo, hi = face_boxes(positions, faces)
    codes = morton_codes(lo, hi)
    order = np.argsort(codes, kind="stable")
    keys = [(int(codes[order[i]]) << 32) | i for i in range(n)]
    slo, shi = lo[order], hi[order]
    m = n - 1

    # top-down radix tree (inner node index = the split rule's numbering)
    child = [[0, 0] for _ in range(max(m, 0))]
    parent = [-1] * max(m, 0)
    parent_leaf = [-1] * n
    pre = []
    if m > 0:
        stack = [(0, 0, n - 1)]
        while stack:
            node, f, l = stack.pop()
            p = (keys[f] ^ keys[l]).bit_length() - 1
            thr = (keys[l] >> p) << p
            gamma = bisect.bisect_left(keys, thr, f, l + 1) - 1
            pre.append(node)
            kids = []
            for c, (cf, cl) in ((gamma, (f, gamma)), (gamma + 1, (gamma + 1, l))):
                if cf == cl:
                    kids.append(LEAF | c)
                    parent_leaf[c] = node
                else:
                    kids.append(c)
                    parent[c] = node
                    stack.append((c, cf, cl))
            child[node] = kids

    nlo = np.zeros((max(m, 0), 3), np.float32)
    nhi = np.zeros((max(m, 0), 3), np.float32)
    cost = [F(0)] * max(m, 0)
    cnt = [0] * max(m, 0)
    col = [False] * max(m, 0)

    def info(c):
        if c & LEAF:
            p = c & ~LEAF
            return slo[p], shi[p], _half_area(slo[p], shi[p]), 1
        return nlo[c], nhi[c], cost[c], cnt[c]

    def set_parent(c, p):
        if c & LEAF:
            parent_leaf[c & ~LEAF] = p
        else:
            parent[c] = p

    def restructure(node):
        leaf = list(child[node])
        larea = [_half_area(*info(c)[:2]) for c in leaf]
        inner_pool = [node]
        while len(leaf) < treelet:
            best, ba = -1, F(0)
            for i, c in enumerate(leaf):
                if not (c & LEAF) and (best < 0 or larea[i] > ba):
                    best, ba = i, larea[i]
            if best < 0:
                break
            x = leaf[best]
            a, b = child[x]
            inner_pool.append(x)
            leaf[best], larea[best] = a, _half_area(*info(a)[:2])
            leaf.append(b)
            larea.append(_half_area(*info(b)[:2]))
        nl = len(leaf)
        if nl < 3:
            return
        li = [info(c) for c in leaf]
        full = (1 << nl) - 1
        dp = [F(0)] * (full + 1)
        split = [0] * (full + 1)

        def members(S):
            idx = [i for i in range(nl) if (S >> i) & 1]
            blo = np.min(np.stack([li[i][0] for i in idx]), 0)
            bhi = np.max(np.stack([li[i][1] for i in idx]), 0)
            return blo, bhi, sum(li[i][3] for i in idx)

        for S in range(1, full + 1):
            if S & (S - 1) == 0:
                dp[S] = li[_low_index(S)][2]
                continue
            blo, bhi, k = members(S)
            low = S & -S
            best, bp = None, low
            P = (S - 1) & S
            while P:
                if P & low:
                    c = F(dp[P] + dp[S ^ P])
                    if best is None or c < best:
                        best, bp = c, P
                P = (P - 1) & S
            dp[S] = _node_cost(_half_area(blo, bhi), best, k, min_leaf, max_leaf, ct)[0]
            split[S] = bp
        stack = [(full, node)]
        nxt = 1
        made = []
        while stack:
            S, me = stack.pop()
            made.append((S, me))
            refs = []
            for part in (split[S], S ^ split[S]):
                if part & (part - 1) == 0:
                    r = leaf[_low_index(part)]
                else:
                    r = inner_pool[nxt]
                    nxt += 1
                    stack.append((part, r))
                set_parent(r, me)
                refs.append(r)
            child[me] = refs
        for S, me in reversed(made[1:]):
            blo, bhi, k = members(S)
            nlo[me], nhi[me], cnt[me] = blo, bhi, k
            cost[me] = dp[S]
            col[me] = _node_cost(_half_area(blo, bhi), F(dp[split[S]] + dp[S ^ split[S]]), k, min_leaf, max_leaf, ct)[1]

    for _ in range(passes if treelet >= 3 else 1):
        if m > 0 and not pre:                    # preorder of the tree the last pass left
            stack = [0]
            while stack:
                x = stack.pop()
                pre.append(x)
                stack.extend(c for c in child[x] if not c & LEAF)
        for node in reversed(pre):               # every node after its subtree
            if treelet >= 3:
                restructure(node)
            la, ha, ca, na = info(child[node][0])
            lb, hb, cbb, nb = info(child[node][1])
            blo, bhi = np.minimum(la, lb), np.maximum(ha, hb)
            nlo[node], nhi[node], cnt[node] = blo, bhi, na + nb
            cost[node], col[node] = _node_cost(_half_area(blo, bhi), F(ca + cbb), na + nb, min_leaf, max_leaf, ct)
        pre = []

    def count_of(c):
        return 1 if c & LEAF else cnt[c]

    keep = np.zeros(max(m, 0), bool)
    depth = np.zeros(max(m, 0), np.int64)
    offset = [0] * max(m, 0)
    for i in range(max(m, 0)):
        kp, off, d = not col[i], 0, 0
        c, a = i, parent[i]
        while a >= 0:
            if col[a]:
                kp = False
            if child[a][1] == c:
                off += count_of(child[a][0])
            d += 1
            c, a = a, parent[a]
        keep[i], offset[i], depth[i] = kp, off, d
    pos = np.zeros(n, np.int64)
    for p in range(n):
        a = parent_leaf[p]
        if a >= 0:
            pos[p] = offset[a] + (count_of(child[a][0]) if child[a][1] == (LEAF | p) else 0)
    final = np.empty(n, np.int64)
    final[pos] = order
    scan = np.cumsum(keep) - keep
    kept = int(keep.sum())

    inner = np.zeros((kept, 16), np.uint32)
    leaf_last = []

    def ref(c):
        if c & LEAF:
            p = c & ~LEAF
            leaf_last.append(int(pos[p]))
            return slo[p], shi[p], LEAF | int(pos[p])
        if col[c]:
            leaf_last.append(offset[c] + cnt[c] - 1)
            return nlo[c], nhi[c], LEAF | offset[c]
        return nlo[c], nhi[c], int(scan[c])

    for i in range(max(m, 0)):
        if not keep[i]:
            continue
        l0, h0, r0 = ref(child[i][0])
        l1, h1, r1 = ref(child[i][1])
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
    return {"order": final, "inner": inner, "leaf_last": np.array(sorted(leaf_last), np.int64),
            "root_ref": root_ref, "root_lo": rlo, "root_hi": rhi,
            "depth": int(depth[keep].max() + 1) if kept else 0, "leaves": len(leaf_last),
            "sah_cost": float(cost[0] / _half_area(rlo, rhi)) if m > 0 else 1.0}


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
