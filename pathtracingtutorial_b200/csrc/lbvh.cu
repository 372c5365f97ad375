// lbvh.cu -- BVH construction on the GPU.
//
// The host builder (host_prep.cpp) reproduces the reference's binned-SAH tree
// node for node (Part_2/src/accel/bvh_builder.cpp:56-221) and is what the
// parity mode uses; for 20M triangles it takes seconds.  This builder makes a
// tree of the same kind on the device in milliseconds:
//
//   1. face boxes and the bounds of their centres         k_lbvh_boxes
//   2. 63-bit Morton codes of the centres (21 bits/axis)  k_lbvh_morton
//   3. stable radix sort of (code, face index)            cub::DeviceRadixSort
//   4. binary radix tree over the sorted codes (Karras,
//      "Maximizing parallelism in the construction of
//      BVHs, octrees and k-d trees", HPG 2012; equal codes
//      ordered by index)                                  k_lbvh_tree
//   5. bottom-up boxes and SAH costs with the reference's
//      cost model (traversal 0.5, one per triangle,
//      bvh_builder.cpp:144-172); a subtree of at most
//      3 faces, or of at most max_leaf faces whose leaf
//      cost is not above its tree cost, becomes one leaf k_lbvh_bottom_up
//   6. surviving inner nodes numbered by a scan           k_lbvh_keep + cub scan
//   7. faces gathered into leaf order as triangle records k_lbvh_gather
//   8. inner nodes in the traversal layout (both child
//      boxes, child refs, the reference's child-order
//      rule), last-in-leaf flags                         k_lbvh_emit
//
// Every step is deterministic: the sort is stable, the tree is a function of
// the sorted codes, boxes are min/max, and every float operation is an
// explicitly rounded intrinsic in a fixed order, so the output is bit for bit
// that of the float32 restatement in oracle/lbvh_ref.py.
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <memory>
#include <string>
#include <thread>
#include <vector>

#include "device_api.h"
#include "engine.h"

namespace ptb {
namespace {

#define LB_CU(call)                                                                        \
    do {                                                                                   \
        cudaError_t e_ = (call);                                                           \
        if (e_ != cudaSuccess) {                                                           \
            set_error(std::string("CUDA error in GPU BVH build: ") + cudaGetErrorString(e_)); \
            return PT_ERR_CUDA;                                                            \
        }                                                                                  \
    } while (0)

constexpr uint32_t kNone = 0xffffffffu;
constexpr int kLbThreads = 256;
constexpr int kMaxTreelet = 7;   // leaves of a restructured treelet (2^7 subsets)
constexpr uint32_t kMaxWalk = 1u << 12;   // bound on any climb to the root (a tree is far shallower)

__device__ __forceinline__ uint32_t ord_of(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_of(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// Half the surface area of a box.
__device__ __forceinline__ float half_area(float4 lo, float4 hi) {
    const float dx = __fsub_rn(hi.x, lo.x), dy = __fsub_rn(hi.y, lo.y), dz = __fsub_rn(hi.z, lo.z);
    return __fadd_rn(__fadd_rn(__fmul_rn(dx, dy), __fmul_rn(dy, dz)), __fmul_rn(dz, dx));
}

__device__ __forceinline__ float centre(float lo, float hi) { return __fmul_rn(0.5f, __fadd_rn(lo, hi)); }

// Face boxes; centre bounds as order-preserving integers in cb[0..5]
// (min x y z, max x y z); the first face with a vertex index or material id
// out of range in cb[6] (atomicMin), whose box is then left empty.
__global__ void __launch_bounds__(kLbThreads) k_lbvh_boxes(const pt_vertex* __restrict__ v, uint32_t nv,
                                                          const pt_face* __restrict__ f, uint32_t n, int32_t nm,
                                                          float4* __restrict__ blo, float4* __restrict__ bhi,
                                                          uint32_t* __restrict__ cb) {
    float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const pt_face fc = f[i];
        if (fc.v0 >= nv || fc.v1 >= nv || fc.v2 >= nv || fc.material_id < 0 || fc.material_id >= nm) {
            atomicMin(&cb[6], i);
            blo[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            bhi[i] = make_float4(0.f, 0.f, 0.f, 0.f);
            continue;
        }
        const float* p0 = v[fc.v0].position;
        const float* p1 = v[fc.v1].position;
        const float* p2 = v[fc.v2].position;
        float lo[3], hi[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            lo[a] = fminf(fminf(p0[a], p1[a]), p2[a]);
            hi[a] = fmaxf(fmaxf(p0[a], p1[a]), p2[a]);
            const float c = centre(lo[a], hi[a]);
            mn[a] = fminf(mn[a], c);
            mx[a] = fmaxf(mx[a], c);
        }
        blo[i] = make_float4(lo[0], lo[1], lo[2], 0.f);
        bhi[i] = make_float4(hi[0], hi[1], hi[2], 0.f);
    }
#pragma unroll
    for (int a = 0; a < 3; ++a) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            mn[a] = fminf(mn[a], __shfl_xor_sync(0xffffffffu, mn[a], o));
            mx[a] = fmaxf(mx[a], __shfl_xor_sync(0xffffffffu, mx[a], o));
        }
    }
    if ((threadIdx.x & 31) == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            atomicMin(&cb[a], ord_of(mn[a]));
            atomicMax(&cb[3 + a], ord_of(mx[a]));
        }
    }
}

// Bit b of x goes to bit 3b (21 bits in, 63 bits out).
__device__ __forceinline__ uint64_t spread3(uint32_t x) {
    uint64_t v = x & 0x1fffffu;
    v = (v | (v << 32)) & 0x001f00000000ffffull;
    v = (v | (v << 16)) & 0x001f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

// code = x bits at 3b+2, y at 3b+1, z at 3b; q = floor((c - lo) * (2^21 / extent)),
// clamped to [0, 2^21 - 1] (a zero extent quantises to 0).
__global__ void __launch_bounds__(kLbThreads) k_lbvh_morton(const float4* __restrict__ blo,
                                                           const float4* __restrict__ bhi, uint32_t n,
                                                           const uint32_t* __restrict__ cb,
                                                           uint64_t* __restrict__ keys, uint32_t* __restrict__ idx) {
    float lo[3], sc[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        lo[a] = float_of(cb[a]);
        const float ext = __fsub_rn(float_of(cb[3 + a]), lo[a]);
        sc[a] = ext > 0.0f ? __fdiv_rn(2097152.0f, ext) : 0.0f;
    }
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float4 l = blo[i], h = bhi[i];
        const float c[3] = {centre(l.x, h.x), centre(l.y, h.y), centre(l.z, h.z)};
        uint64_t code = 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const float t = floorf(__fmul_rn(__fsub_rn(c[a], lo[a]), sc[a]));
            const uint32_t q = static_cast<uint32_t>(fminf(fmaxf(t, 0.0f), 2097151.0f));
            code |= spread3(q) << (2 - a);
        }
        keys[i] = code;
        idx[i] = i;
    }
}

// Length of the common prefix of sorted codes i and j; equal codes compare
// their positions instead (64 + common prefix of the indices); -1 outside.
__device__ __forceinline__ int lb_delta(const uint64_t* __restrict__ k, int64_t n, int64_t i, int64_t j) {
    if (j < 0 || j >= n) return -1;
    const uint64_t a = k[i], b = k[j];
    if (a != b) return __clzll(static_cast<long long>(a ^ b));
    return 64 + __clz(static_cast<int>(static_cast<uint32_t>(i) ^ static_cast<uint32_t>(j)));
}

// Inner node i of the radix tree over n sorted codes (i < n - 1): the range
// it covers, the split, and its children (kLeafBit | position for a leaf).
__global__ void __launch_bounds__(kLbThreads) k_lbvh_tree(const uint64_t* __restrict__ k, uint32_t n,
                                                         uint2* __restrict__ child,
                                                         uint32_t* __restrict__ parent_inner,
                                                         uint32_t* __restrict__ parent_leaf) {
    const int64_t nn = n;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t ii = blockIdx.x * blockDim.x + threadIdx.x; ii + 1 < n; ii += stride) {
        const int64_t i = ii;
        const int d = (lb_delta(k, nn, i, i + 1) - lb_delta(k, nn, i, i - 1)) > 0 ? 1 : -1;
        const int dmin = lb_delta(k, nn, i, i - d);
        int64_t lmax = 2;
        while (lb_delta(k, nn, i, i + lmax * d) > dmin) lmax <<= 1;
        int64_t l = 0;
        for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
            if (lb_delta(k, nn, i, i + (l + t) * d) > dmin) l += t;
        const int64_t j = i + l * d;
        const int dnode = lb_delta(k, nn, i, j);
        int64_t s = 0, t = l;
        do {
            t = (t + 1) >> 1;
            if (lb_delta(k, nn, i, i + (s + t) * d) > dnode) s += t;
        } while (t > 1);
        const int64_t gamma = i + s * d + (d < 0 ? -1 : 0);
        const int64_t first = i < j ? i : j, last = i < j ? j : i;
        uint32_t c0, c1;
        if (first == gamma) { c0 = kLeafBit | static_cast<uint32_t>(gamma); parent_leaf[gamma] = ii; }
        else { c0 = static_cast<uint32_t>(gamma); parent_inner[gamma] = ii; }
        if (last == gamma + 1) { c1 = kLeafBit | static_cast<uint32_t>(gamma + 1); parent_leaf[gamma + 1] = ii; }
        else { c1 = static_cast<uint32_t>(gamma + 1); parent_inner[gamma + 1] = ii; }
        child[ii] = make_uint2(c0, c1);
        if (ii == 0) parent_inner[0] = kNone;
    }
}

struct ChildInfo {
    float4 lo, hi;   // hi.w = SAH cost of the child
    uint32_t count;
};

// Children written by other threads of the same launch are read through L2.
__device__ __forceinline__ ChildInfo child_info(uint32_t c, const uint32_t* __restrict__ sorted,
                                                const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                                const float4* nlo, const float4* nhi, const uint32_t* ncount) {
    ChildInfo r;
    if (c & kLeafBit) {
        const uint32_t f = sorted[c & ~kLeafBit];
        r.lo = blo[f];
        r.hi = bhi[f];
        r.hi.w = half_area(r.lo, r.hi);   // one triangle
        r.count = 1;
    } else {
        r.lo = __ldcg(nlo + c);
        r.hi = __ldcg(nhi + c);
        r.count = __ldcg(ncount + c);
    }
    return r;
}

// SAH cost of a node of `cnt` faces and half area `area` whose children cost
// `children` together: tree = ct A + children, leaf = cnt A (ct = cost of a
// node visit in triangle tests; the reference's model has 0.5).  It becomes a
// leaf when it holds at most min_leaf faces (the reference's rule: fewer than
// LeafThreshold = 4, bvh_builder.cpp:10,99) or at most max_leaf faces at a
// leaf cost not above its tree cost.
__device__ __forceinline__ float node_cost(float area, float children, uint32_t cnt, uint32_t min_leaf,
                                           uint32_t max_leaf, float ct, bool& col) {
    const float tree = __fadd_rn(__fmul_rn(ct, area), children);
    const float leaf = __fmul_rn(__uint2float_rn(cnt), area);
    col = cnt <= min_leaf || (cnt <= max_leaf && leaf <= tree);
    return col ? leaf : tree;
}

__device__ __forceinline__ float ref_area(uint32_t c, const uint32_t* __restrict__ sorted,
                                          const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                          const float4* nlo, const float4* nhi) {
    if (c & kLeafBit) {
        const uint32_t f = sorted[c & ~kLeafBit];
        return half_area(blo[f], bhi[f]);
    }
    return half_area(__ldcg(nlo + c), __ldcg(nhi + c));
}

__device__ __forceinline__ void set_parent(uint32_t c, uint32_t p, uint32_t* parent_inner, uint32_t* parent_leaf) {
    if (c & kLeafBit) __stcg(parent_leaf + (c & ~kLeafBit), p);
    else __stcg(parent_inner + c, p);
}

// Leaf subsets of a treelet ordered by size (then value): the dynamic program
// handles one size at a time, the subsets of a size in parallel.
struct SubsetTable {
    uint8_t mask[127];
    uint8_t start[9];   // subsets of size k: mask[start[k] .. start[k + 1])
};
constexpr SubsetTable make_subset_table() {
    SubsetTable t{};
    int j = 0;
    for (int k = 0; k <= 8; ++k) {
        t.start[k] = static_cast<uint8_t>(j);
        for (int m = 1; m < 128 && k >= 1; ++m) {
            int bits = 0;
            for (int b = 0; b < 7; ++b) bits += (m >> b) & 1;
            if (bits == k) t.mask[j++] = static_cast<uint8_t>(m);
        }
    }
    return t;
}
__constant__ SubsetTable c_subsets = make_subset_table();

// One warp's tables for the treelet it is restructuring.
struct TreeletScratch {
    float4 lo[kMaxTreelet], hi[kMaxTreelet];   // leaf boxes, hi.w = leaf cost
    uint32_t cnt[kMaxTreelet];
    float cost[1 << kMaxTreelet];
    uint8_t split[1 << kMaxTreelet];
};

// Treelet restructuring (Karras and Aila, "Fast parallel construction of
// high-quality bounding volume hierarchies", HPG 2013), by all 32 lanes of a
// warp for one node.  The treelet of `node`: start from its two children and
// repeatedly open the inner-node leaf of largest area (first on ties) until
// `max_leaves` leaves; the treelet's inner nodes (node first, then in opening
// order) are reused.  Dynamic programming over the leaf subsets, smaller
// subsets first (one subset per lane), finds the topology of least SAH cost:
// for subset S the splits P containing S's lowest leaf, in descending order,
// the first strict minimum wins; P becomes the left child.  Lane 0 writes
// the new topology with the inner nodes handed out depth first, right part
// first (a LIFO stack), and recomputes the moved nodes' summaries children
// first.
__device__ void warp_restructure(uint32_t node, int max_leaves, int lane, TreeletScratch& ts, uint2* child,
                                 uint32_t* parent_inner, uint32_t* parent_leaf, const uint32_t* __restrict__ sorted,
                                 const float4* __restrict__ blo, const float4* __restrict__ bhi, float4* nlo,
                                 float4* nhi, uint32_t* ncount, uint8_t* __restrict__ collapse, uint32_t min_leaf,
                                 uint32_t max_leaf, float ct) {
    // treelet formation: every lane computes the same (reads broadcast)
    uint32_t leaf[kMaxTreelet];
    float larea[kMaxTreelet];
    uint32_t inner[kMaxTreelet - 1];
    const uint2 ch = __ldcg(child + node);
    leaf[0] = ch.x;
    leaf[1] = ch.y;
    larea[0] = ref_area(ch.x, sorted, blo, bhi, nlo, nhi);
    larea[1] = ref_area(ch.y, sorted, blo, bhi, nlo, nhi);
    inner[0] = node;
    int nl = 2, ni = 1;
    while (nl < max_leaves) {
        int best = -1;
        float ba = 0.0f;
        for (int i = 0; i < nl; ++i)
            if (!(leaf[i] & kLeafBit) && (best < 0 || larea[i] > ba)) { ba = larea[i]; best = i; }
        if (best < 0) break;
        const uint32_t x = leaf[best];
        const uint2 cc = __ldcg(child + x);
        inner[ni++] = x;
        leaf[best] = cc.x;
        larea[best] = ref_area(cc.x, sorted, blo, bhi, nlo, nhi);
        leaf[nl] = cc.y;
        larea[nl] = ref_area(cc.y, sorted, blo, bhi, nlo, nhi);
        ++nl;
    }
    if (nl < 3) return;   // the same on every lane
    if (lane < nl) {
        const ChildInfo ci = child_info(leaf[lane], sorted, blo, bhi, nlo, nhi, ncount);
        ts.lo[lane] = ci.lo;
        ts.hi[lane] = ci.hi;
        ts.cnt[lane] = ci.count;
        ts.cost[1u << lane] = ci.hi.w;
    }
    __syncwarp();
    const uint32_t full = (1u << nl) - 1u;
    for (int k = 2; k <= nl; ++k) {
        for (int j = c_subsets.start[k] + lane; j < c_subsets.start[k + 1]; j += 32) {
            const uint32_t S = c_subsets.mask[j];
            if (S > full) continue;
            float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
            uint32_t cnt = 0;
            for (int i = 0; i < nl; ++i) {
                if (!((S >> i) & 1u)) continue;
                const float4 a = ts.lo[i], b = ts.hi[i];
                lo.x = fminf(lo.x, a.x); lo.y = fminf(lo.y, a.y); lo.z = fminf(lo.z, a.z);
                hi.x = fmaxf(hi.x, b.x); hi.y = fmaxf(hi.y, b.y); hi.z = fmaxf(hi.z, b.z);
                cnt += ts.cnt[i];
            }
            // the splits P holding S's lowest leaf, in descending order: P = low | Q
            // for the submasks Q of the other leaves R, Q < R descending
            const uint32_t low = S & (0u - S), R = S ^ low;
            float best = INFINITY;
            uint32_t bp = low;
            for (uint32_t Q = (R - 1u) & R;; Q = (Q - 1u) & R) {
                const float c = __fadd_rn(ts.cost[Q | low], ts.cost[R ^ Q]);
                if (c < best) { best = c; bp = Q | low; }
                if (Q == 0) break;
            }
            bool col;
            ts.cost[S] = node_cost(half_area(lo, hi), best, cnt, min_leaf, max_leaf, ct, col);
            ts.split[S] = static_cast<uint8_t>(bp);
        }
        __syncwarp();
    }
    if (lane == 0) {
        // write the topology: (subset, inner node) on a LIFO stack
        uint8_t st_s[kMaxTreelet];
        uint32_t st_n[kMaxTreelet];
        uint8_t made_s[kMaxTreelet - 1];
        uint32_t made_n[kMaxTreelet - 1];
        int sp = 0, next = 1, nm = 0;
        st_s[sp] = static_cast<uint8_t>(full);
        st_n[sp++] = node;
        while (sp) {
            --sp;
            const uint32_t S = st_s[sp], me = st_n[sp];
            made_s[nm] = static_cast<uint8_t>(S);
            made_n[nm++] = me;
            const uint32_t parts[2] = {ts.split[S], S ^ ts.split[S]};
            uint32_t ref[2];
            for (int q = 0; q < 2; ++q) {
                if ((parts[q] & (parts[q] - 1u)) == 0) {
                    ref[q] = leaf[__ffs(parts[q]) - 1];
                } else {
                    ref[q] = inner[next++];
                    st_s[sp] = static_cast<uint8_t>(parts[q]);
                    st_n[sp++] = ref[q];
                }
                set_parent(ref[q], me, parent_inner, parent_leaf);
            }
            __stcg(child + me, make_uint2(ref[0], ref[1]));
        }
        // summaries of the moved inner nodes, children first (the root's is
        // written by the caller)
        for (int j = nm - 1; j >= 1; --j) {
            const uint32_t S = made_s[j], me = made_n[j];
            float4 lo = make_float4(INFINITY, INFINITY, INFINITY, 0.f), hi = make_float4(-INFINITY, -INFINITY, -INFINITY, 0.f);
            uint32_t cnt = 0;
            for (int i = 0; i < nl; ++i) {
                if (!((S >> i) & 1u)) continue;
                const float4 a = ts.lo[i], b = ts.hi[i];
                lo.x = fminf(lo.x, a.x); lo.y = fminf(lo.y, a.y); lo.z = fminf(lo.z, a.z);
                hi.x = fmaxf(hi.x, b.x); hi.y = fmaxf(hi.y, b.y); hi.z = fmaxf(hi.z, b.z);
                cnt += ts.cnt[i];
            }
            hi.w = ts.cost[S];
            bool col;
            node_cost(half_area(lo, hi), __fadd_rn(ts.cost[ts.split[S]], ts.cost[S ^ ts.split[S]]), cnt, min_leaf,
                      max_leaf, ct, col);
            __stcg(nlo + me, lo);
            __stcg(nhi + me, hi);
            __stcg(ncount + me, cnt);
            collapse[me] = col ? 1 : 0;
        }
    }
    __syncwarp();
}

// One thread per leaf climbs while it is the second to reach a node; the
// first one stops.  At each node reached second: the warp restructures the
// node's treelet (when treelet >= 3; the warp takes its lanes' nodes one at a
// time), then the owner lane writes box = union of the children, count, SAH
// cost and the leaf decision of node_cost.  Every climb ends within kMaxWalk
// steps or raises `fault`.
__global__ void __launch_bounds__(kLbThreads) k_lbvh_bottom_up(
    uint2* child, uint32_t* parent_inner, uint32_t* parent_leaf, const uint32_t* __restrict__ sorted,
    const float4* __restrict__ blo, const float4* __restrict__ bhi, uint32_t n, uint32_t min_leaf, uint32_t max_leaf,
    float ct, int treelet, float4* nlo, float4* nhi, uint32_t* ncount, uint8_t* __restrict__ collapse,
    uint32_t* __restrict__ counter, uint32_t* __restrict__ fault) {
    __shared__ TreeletScratch scratch[kLbThreads / 32];
    const int lane = threadIdx.x & 31;
    TreeletScratch& ts = scratch[threadIdx.x >> 5];
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t nr = (n + 31u) & ~31u;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < nr; p += stride) {   // whole warps
        uint32_t node = p < n ? __ldcg(parent_leaf + p) : kNone;
        uint32_t steps = 0;
        while (__any_sync(0xffffffffu, node != kNone)) {
            bool mine = false;
            if (node != kNone) {
                if (steps++ >= kMaxWalk) {
                    atomicExch(fault, 1u);
                    node = kNone;
                } else {
                    __threadfence();
                    mine = atomicAdd(counter + node, 1u) != 0;
                    if (mine) __threadfence();
                    else node = kNone;
                }
            }
            if (treelet >= 3) {
                uint32_t need = __ballot_sync(0xffffffffu, mine);
                __syncwarp();
                while (need) {
                    const int src = __ffs(need) - 1;
                    need &= need - 1u;
                    const uint32_t t = __shfl_sync(0xffffffffu, node, src);
                    warp_restructure(t, treelet, lane, ts, child, parent_inner, parent_leaf, sorted, blo, bhi, nlo,
                                     nhi, ncount, collapse, min_leaf, max_leaf, ct);
                }
            }
            if (mine) {
                const uint2 ch = __ldcg(child + node);
                const ChildInfo a = child_info(ch.x, sorted, blo, bhi, nlo, nhi, ncount);
                const ChildInfo b = child_info(ch.y, sorted, blo, bhi, nlo, nhi, ncount);
                float4 lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), 0.f);
                float4 hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), 0.f);
                const uint32_t cnt = a.count + b.count;
                bool col;
                hi.w = node_cost(half_area(lo, hi), __fadd_rn(a.hi.w, b.hi.w), cnt, min_leaf, max_leaf, ct, col);
                __stcg(nlo + node, lo);
                __stcg(nhi + node, hi);
                __stcg(ncount + node, cnt);
                collapse[node] = col ? 1 : 0;
                node = __ldcg(parent_inner + node);
            }
        }
    }
}

__device__ __forceinline__ uint32_t ref_count(uint32_t c, const uint32_t* __restrict__ ncount) {
    return (c & kLeafBit) ? 1u : ncount[c];
}

// Per inner node i, walking to the root: keep[i] = neither it nor an
// ancestor became a leaf; offset[i] = its first face in depth-first order
// (the faces of the left siblings of it and its ancestors); depth[0] = max
// over survivors of (edges from the root + 1).
__global__ void __launch_bounds__(kLbThreads) k_lbvh_keep(const uint8_t* __restrict__ collapse,
                                                         const uint32_t* __restrict__ parent_inner,
                                                         const uint2* __restrict__ child,
                                                         const uint32_t* __restrict__ ncount, uint32_t m,
                                                         uint32_t* __restrict__ keep, uint32_t* __restrict__ offset,
                                                         uint32_t* __restrict__ depth, uint32_t* __restrict__ fault) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t mr = (m + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < mr; i += stride) {
        uint32_t kp = 0, dd = 0;
        if (i < m) {
            kp = collapse[i] ? 0u : 1u;
            uint32_t off = 0;
            for (uint32_t c = i, a = parent_inner[i]; a != kNone; c = a, a = parent_inner[a]) {
                if (dd >= kMaxWalk) { atomicExch(fault, 1u); break; }
                if (collapse[a]) kp = 0;
                const uint2 ch = child[a];
                if (ch.y == c) off += ref_count(ch.x, ncount);
                ++dd;
            }
            keep[i] = kp;
            offset[i] = off;
        }
        const uint32_t wmax = __reduce_max_sync(0xffffffffu, kp ? dd + 1 : 0u);
        if ((threadIdx.x & 31) == 0 && wmax) atomicMax(depth, wmax);
    }
}

// Depth-first position of every face: its parent's offset, plus the left
// sibling's faces when it is a right child.  With one face, position 0.
__global__ void __launch_bounds__(kLbThreads) k_lbvh_positions(const uint32_t* __restrict__ parent_leaf,
                                                              const uint2* __restrict__ child,
                                                              const uint32_t* __restrict__ ncount,
                                                              const uint32_t* __restrict__ offset, uint32_t n,
                                                              uint32_t* __restrict__ pos) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const uint32_t a = parent_leaf[p];
        if (a == kNone) { pos[p] = 0; continue; }
        const uint2 ch = child[a];
        pos[p] = offset[a] + (ch.y == (kLeafBit | p) ? ref_count(ch.x, ncount) : 0u);
    }
}

// Faces in leaf order and their triangle records (v0, v1 - v0, v2 - v0).
// A face with a vertex index out of range (already reported by k_lbvh_boxes)
// gets a zero record.
__global__ void __launch_bounds__(kLbThreads) k_lbvh_gather(const pt_vertex* __restrict__ v, uint32_t nv,
                                                           const pt_face* __restrict__ f,
                                                           const uint32_t* __restrict__ sorted,
                                                           const uint32_t* __restrict__ pos, uint32_t n,
                                                           pt_face* __restrict__ fout, float4* __restrict__ tout) {
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += stride) {
        const pt_face fc = f[sorted[p]];
        const uint32_t q = pos[p];
        if (q >= n) continue;   // only a malformed tree; the host walk rejects it
        fout[q] = fc;
        if (fc.v0 >= nv || fc.v1 >= nv || fc.v2 >= nv) {
            const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
            tout[3 * q + 0] = z;
            tout[3 * q + 1] = z;
            tout[3 * q + 2] = z;
            continue;
        }
        const float* p0 = v[fc.v0].position;
        const float* p1 = v[fc.v1].position;
        const float* p2 = v[fc.v2].position;
        const float x0 = p0[0], y0 = p0[1], z0 = p0[2];
        tout[3 * q + 0] = make_float4(x0, y0, z0, __fsub_rn(p1[0], x0));
        tout[3 * q + 1] = make_float4(__fsub_rn(p1[1], y0), __fsub_rn(p1[2], z0), __fsub_rn(p2[0], x0),
                                      __fsub_rn(p2[1], y0));
        tout[3 * q + 2] = make_float4(__fsub_rn(p2[2], z0), 0.f, 0.f, 0.f);
    }
}

__device__ __forceinline__ void child_ref(uint32_t c, const uint32_t* __restrict__ sorted,
                                          const float4* __restrict__ blo, const float4* __restrict__ bhi,
                                          const float4* __restrict__ nlo, const float4* __restrict__ nhi,
                                          const uint8_t* __restrict__ collapse, const uint32_t* __restrict__ ncount,
                                          const uint32_t* __restrict__ offset, const uint32_t* __restrict__ pos,
                                          const uint32_t* __restrict__ scan, float4& lo, float4& hi, uint32_t& ref,
                                          uint32_t& last) {
    if (c & kLeafBit) {
        const uint32_t p = c & ~kLeafBit;
        const uint32_t f = sorted[p];
        lo = blo[f];
        hi = bhi[f];
        ref = kLeafBit | pos[p];
        last = pos[p];
    } else {
        lo = nlo[c];
        hi = nhi[c];
        if (collapse[c]) {
            ref = kLeafBit | offset[c];
            last = offset[c] + ncount[c] - 1u;
        } else {
            ref = scan[c];
            last = kNone;
        }
    }
}

// Surviving inner node i -> InnerNode scan[i]; leaves flag their last record.
__global__ void __launch_bounds__(kLbThreads) k_lbvh_emit(
    const uint2* __restrict__ child, const uint32_t* __restrict__ sorted, const float4* __restrict__ blo,
    const float4* __restrict__ bhi, const float4* __restrict__ nlo, const float4* __restrict__ nhi,
    const uint8_t* __restrict__ collapse, const uint32_t* __restrict__ ncount, const uint32_t* __restrict__ offset,
    const uint32_t* __restrict__ pos, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ scan,
    uint32_t m, uint32_t n, InnerNode* __restrict__ out, float4* __restrict__ tris, uint32_t* __restrict__ leaves) {
    const uint32_t stride = gridDim.x * blockDim.x;
    const uint32_t mr = (m + 31u) & ~31u;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < mr; i += stride) {
        uint32_t nleaf = 0;
        if (i < m && keep[i]) {
            const uint2 ch = child[i];
            float4 l0, h0, l1, h1;
            uint32_t r0, r1, last0, last1;
            child_ref(ch.x, sorted, blo, bhi, nlo, nhi, collapse, ncount, offset, pos, scan, l0, h0, r0, last0);
            child_ref(ch.y, sorted, blo, bhi, nlo, nhi, collapse, ncount, offset, pos, scan, l1, h1, r1, last1);
            // (last >= n only in a malformed tree, which the host walk rejects)
            if (last0 != kNone) { if (last0 < n) tris[3 * last0 + 2].y = __uint_as_float(1u); ++nleaf; }
            if (last1 != kNone) { if (last1 < n) tris[3 * last1 + 2].y = __uint_as_float(1u); ++nleaf; }
            // child order rule: the node's max-extent axis and the child centres on it
            const float4 pl = nlo[i], ph = nhi[i];
            const float dx = __fsub_rn(ph.x, pl.x), dy = __fsub_rn(ph.y, pl.y), dz = __fsub_rn(ph.z, pl.z);
            const uint32_t axis = (dx > dy && dx > dz) ? 0u : (dy > dz ? 1u : 2u);
            const float c0 = axis == 0 ? centre(l0.x, h0.x) : (axis == 1 ? centre(l0.y, h0.y) : centre(l0.z, h0.z));
            const float c1 = axis == 0 ? centre(l1.x, h1.x) : (axis == 1 ? centre(l1.y, h1.y) : centre(l1.z, h1.z));
            float4* o = reinterpret_cast<float4*>(out + scan[i]);
            o[0] = make_float4(l0.x, l0.y, l0.z, h0.x);
            o[1] = make_float4(h0.y, h0.z, l1.x, l1.y);
            o[2] = make_float4(l1.z, h1.x, h1.y, h1.z);
            o[3] = make_float4(__uint_as_float(r0), __uint_as_float(r1),
                               __uint_as_float(axis | (c0 < c1 ? 4u : 0u)), 0.f);
        }
        const uint32_t w = __reduce_add_sync(0xffffffffu, nleaf);
        if ((threadIdx.x & 31) == 0 && w) atomicAdd(leaves, w);
    }
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

// Fault in freshly allocated host pages from several cores (each thread
// zeroes its own slice) before a device-to-host copy writes them: the copy
// then runs at the speed of resident memory.
void touch_pages(void* p, size_t bytes) {
    if (bytes < (size_t(64) << 20)) { std::memset(p, 0, bytes); return; }
    const unsigned nt = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    const size_t chunk = (bytes + nt - 1) / nt;
    std::vector<std::thread> pool;
    for (unsigned i = 0; i < nt; ++i) {
        const size_t a = i * chunk;
        if (a >= bytes) break;
        const size_t len = std::min(chunk, bytes - a);
        pool.emplace_back([p, a, len] { std::memset(static_cast<char*>(p) + a, 0, len); });
    }
    for (std::thread& t : pool) t.join();
}

int grid_for(uint32_t n, int sms) {
    const uint64_t want = (static_cast<uint64_t>(n) + kLbThreads - 1) / kLbThreads;
    const uint64_t cap = static_cast<uint64_t>(sms) * 8;
    return static_cast<int>(want < 1 ? 1 : (want > cap ? cap : want));
}

// Check the built tree on the host before anything traverses it, in linear
// passes: every child reference in range, every inner node but the root
// referenced exactly once and the root never (so the part reachable from the
// root is a tree), and the leaves tiling the triangle records exactly (each
// leaf starts where the previous flagged record ends, the last record is
// flagged).  Traversal then ends and reads only within the arrays.
bool check_tree(const SceneTables& t, uint32_t n, std::string& why) {
    const uint32_t ni = static_cast<uint32_t>(t.inner.size());
    std::vector<uint8_t> indeg(ni, 0), starts(n, 0);
    auto leaf = [&](uint32_t first) {
        if (first >= n) { why = "leaf start " + std::to_string(first) + " out of range"; return false; }
        if (starts[first]++) { why = "two leaves start at " + std::to_string(first); return false; }
        return true;
    };
    if (t.root_ref & kLeafBit) {
        if (ni != 0 || (t.root_ref & ~kLeafBit) != 0) { why = "one-leaf tree with inner nodes"; return false; }
        if (!leaf(0)) return false;
    } else {
        if (ni == 0 || t.root_ref != 0) { why = "no root"; return false; }
        for (uint32_t k = 0; k < ni; ++k) {
            for (const uint32_t r : {t.inner[k].ref0, t.inner[k].ref1}) {
                if (r & kLeafBit) {
                    if (!leaf(r & ~kLeafBit)) return false;
                } else if (r == 0 || r >= ni || indeg[r]++) {
                    why = "inner node reference " + std::to_string(r) + " out of range or repeated";
                    return false;
                }
            }
        }
        for (uint32_t k = 1; k < ni; ++k)
            if (!indeg[k]) { why = "inner node " + std::to_string(k) + " unreferenced"; return false; }
    }
    for (uint32_t i = 0; i < n; ++i) {
        const bool should_start = i == 0 || (t.tris[i - 1].flags & 1u);
        if (static_cast<bool>(starts[i]) != should_start) {
            why = "leaves do not tile the triangle records at " + std::to_string(i);
            return false;
        }
    }
    if (!(t.tris[n - 1].flags & 1u)) { why = "last triangle record not flagged"; return false; }
    return true;
}

}  // namespace

int build_accel_device(pt_scene* s, int device, uint32_t max_leaf, int treelet, int passes, float ct,
                       pt_build_stats* stats) {
    using clock = std::chrono::steady_clock;
    const auto t_start = clock::now();
    HostScene& hs = s->host;
    SceneTables& t = s->tables;
    const size_t n64 = hs.faces.size();
    if (n64 >= kLeafBit) { set_error("too many faces for the GPU BVH builder"); return PT_ERR_INVALID; }
    if (hs.vertices.size() >= 0xffffffffull) { set_error("too many vertices"); return PT_ERR_INVALID; }
    const uint32_t n = static_cast<uint32_t>(n64), nv = static_cast<uint32_t>(hs.vertices.size());
    const uint32_t m = n > 0 ? n - 1 : 0;
    pt_build_stats st{};
    t = SceneTables{};
    if (n == 0) {
        build_emissive_tables(hs, t);
        build_env_tables(hs, t);
        t.built = true;
        if (stats) *stats = st;
        return PT_OK;
    }
    LB_CU(cudaSetDevice(device));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

    // cub scratch sizes
    size_t sort_tmp = 0, scan_tmp = 0;
    LB_CU(cub::DeviceRadixSort::SortPairs(nullptr, sort_tmp, static_cast<const uint64_t*>(nullptr),
                                          static_cast<uint64_t*>(nullptr), static_cast<const uint32_t*>(nullptr),
                                          static_cast<uint32_t*>(nullptr), static_cast<int>(n), 0, 63));
    if (m > 0)
        LB_CU(cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, static_cast<const uint32_t*>(nullptr),
                                            static_cast<uint32_t*>(nullptr), static_cast<int>(m)));

    // one arena
    size_t off = 0;
    auto take = [&](size_t bytes) { const size_t o = off; off += align_up(bytes ? bytes : 1); return o; };
    const size_t o_v = take(size_t(nv) * sizeof(pt_vertex)), o_f = take(size_t(n) * sizeof(pt_face));
    const size_t o_blo = take(size_t(n) * 16), o_bhi = take(size_t(n) * 16), o_cb = take(16 * 4);
    const size_t o_k0 = take(size_t(n) * 8), o_k1 = take(size_t(n) * 8);
    const size_t o_i0 = take(size_t(n) * 4), o_i1 = take(size_t(n) * 4);
    const size_t o_sort = take(sort_tmp), o_scan = take(scan_tmp);
    const size_t o_child = take(size_t(m) * 8), o_off = take(size_t(m) * 4), o_pos = take(size_t(n) * 4);
    const size_t o_pin = take(size_t(m) * 4), o_pleaf = take(size_t(n) * 4);
    const size_t o_nlo = take(size_t(m) * 16), o_nhi = take(size_t(m) * 16), o_ncnt = take(size_t(m) * 4);
    const size_t o_col = take(size_t(m)), o_ctr = take(size_t(m) * 4);
    const size_t o_keep = take(size_t(m) * 4), o_scn = take(size_t(m) * 4);
    const size_t o_inner = take(size_t(m) * sizeof(InnerNode)), o_tris = take(size_t(n) * sizeof(TriRecord));
    const size_t o_fout = take(size_t(n) * sizeof(pt_face));
    char* arena = nullptr;
    LB_CU(cudaMalloc(&arena, off));
    struct Free { char* p; ~Free() { if (p) cudaFree(p); } } guard{arena};
    auto at = [&](size_t o) { return static_cast<void*>(arena + o); };
    pt_vertex* d_v = static_cast<pt_vertex*>(at(o_v));
    pt_face* d_f = static_cast<pt_face*>(at(o_f));
    float4* blo = static_cast<float4*>(at(o_blo));
    float4* bhi = static_cast<float4*>(at(o_bhi));
    uint32_t* cb = static_cast<uint32_t*>(at(o_cb));
    uint64_t* k0 = static_cast<uint64_t*>(at(o_k0));
    uint64_t* k1 = static_cast<uint64_t*>(at(o_k1));
    uint32_t* i0 = static_cast<uint32_t*>(at(o_i0));
    uint32_t* i1 = static_cast<uint32_t*>(at(o_i1));
    uint2* child = static_cast<uint2*>(at(o_child));
    uint32_t* offset = static_cast<uint32_t*>(at(o_off));
    uint32_t* pos = static_cast<uint32_t*>(at(o_pos));
    uint32_t* pin = static_cast<uint32_t*>(at(o_pin));
    uint32_t* pleaf = static_cast<uint32_t*>(at(o_pleaf));
    float4* nlo = static_cast<float4*>(at(o_nlo));
    float4* nhi = static_cast<float4*>(at(o_nhi));
    uint32_t* ncnt = static_cast<uint32_t*>(at(o_ncnt));
    uint8_t* col = static_cast<uint8_t*>(at(o_col));
    uint32_t* ctr = static_cast<uint32_t*>(at(o_ctr));
    uint32_t* keep = static_cast<uint32_t*>(at(o_keep));
    uint32_t* scn = static_cast<uint32_t*>(at(o_scn));
    InnerNode* d_inner = static_cast<InnerNode*>(at(o_inner));
    float4* d_tris = static_cast<float4*>(at(o_tris));
    pt_face* d_fout = static_cast<pt_face*>(at(o_fout));

    cudaStream_t stream;
    LB_CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    struct SFree { cudaStream_t s; ~SFree() { cudaStreamDestroy(s); } } sguard{stream};
    cudaEvent_t ev[3];
    for (auto& e : ev) LB_CU(cudaEventCreate(&e));
    struct EFree { cudaEvent_t* e; ~EFree() { for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]); } } eguard{ev};

    const auto t_setup = clock::now();
    LB_CU(cudaEventRecord(ev[0], stream));
    LB_CU(cudaMemcpyAsync(d_v, hs.vertices.data(), size_t(nv) * sizeof(pt_vertex), cudaMemcpyHostToDevice, stream));
    LB_CU(cudaMemcpyAsync(d_f, hs.faces.data(), size_t(n) * sizeof(pt_face), cudaMemcpyHostToDevice, stream));
    LB_CU(cudaEventRecord(ev[1], stream));

    // centre bounds start empty; cb[6] = first bad face; cb[7] = depth; cb[8] = a climb
    // that did not reach the root
    const uint32_t init[9] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u, 0xffffffffu, 0u, 0u};
    LB_CU(cudaMemcpyAsync(cb, init, sizeof(init), cudaMemcpyHostToDevice, stream));
    const int g = grid_for(n, sms);
    k_lbvh_boxes<<<g, kLbThreads, 0, stream>>>(d_v, nv, d_f, n, static_cast<int32_t>(hs.materials.size()), blo, bhi,
                                               cb);
    k_lbvh_morton<<<g, kLbThreads, 0, stream>>>(blo, bhi, n, cb, k0, i0);
    LB_CU(cub::DeviceRadixSort::SortPairs(at(o_sort), sort_tmp, k0, k1, i0, i1, static_cast<int>(n), 0, 63, stream));
    LB_CU(cudaMemsetAsync(pleaf, 0xff, size_t(n) * 4, stream));
    if (m > 0) {
        const int gm = grid_for(m, sms);
        const uint32_t min_leaf = max_leaf < 3 ? max_leaf : 3;
        k_lbvh_tree<<<gm, kLbThreads, 0, stream>>>(k1, n, child, pin, pleaf);
        // later passes restructure the treelets of the restructured tree
        for (int pass = 0; pass < (treelet >= 3 ? passes : 1); ++pass) {
            LB_CU(cudaMemsetAsync(ctr, 0, size_t(m) * 4, stream));
            k_lbvh_bottom_up<<<g, kLbThreads, 0, stream>>>(child, pin, pleaf, i1, blo, bhi, n, min_leaf, max_leaf,
                                                           ct, treelet, nlo, nhi, ncnt, col, ctr, cb + 8);
        }
        k_lbvh_keep<<<gm, kLbThreads, 0, stream>>>(col, pin, child, ncnt, m, keep, offset, cb + 7, cb + 8);
        LB_CU(cub::DeviceScan::ExclusiveSum(at(o_scan), scan_tmp, keep, scn, static_cast<int>(m), stream));
    }
    k_lbvh_positions<<<g, kLbThreads, 0, stream>>>(pleaf, child, ncnt, offset, n, pos);
    k_lbvh_gather<<<g, kLbThreads, 0, stream>>>(d_v, nv, d_f, i1, pos, n, d_fout, d_tris);
    if (m > 0) {
        // the bottom-up arrival counters are done with: ctr[0] counts leaves
        LB_CU(cudaMemsetAsync(ctr, 0, 4, stream));
        k_lbvh_emit<<<grid_for(m, sms), kLbThreads, 0, stream>>>(child, i1, blo, bhi, nlo, nhi, col, ncnt, offset, pos,
                                                                 keep, scn, m, n, d_inner, d_tris, ctr);
    }
    LB_CU(cudaGetLastError());
    LB_CU(cudaEventRecord(ev[2], stream));

    // the environment tables do not depend on the tree: build them while the device works
    const auto t_env0 = clock::now();
    build_env_tables(hs, t);
    const double env_ms = std::chrono::duration<double, std::milli>(clock::now() - t_env0).count();

    // scalars: bad face, depth, leaves, survivors, root collapse, root box
    uint32_t h_cb[9];
    uint32_t h_leaves = 0, h_keep_last = 0, h_scan_last = 0;
    float4 h_root[2] = {};
    LB_CU(cudaMemcpyAsync(h_cb, cb, sizeof(h_cb), cudaMemcpyDeviceToHost, stream));
    if (m > 0) {
        LB_CU(cudaMemcpyAsync(&h_leaves, ctr, 4, cudaMemcpyDeviceToHost, stream));
        LB_CU(cudaMemcpyAsync(&h_keep_last, keep + (m - 1), 4, cudaMemcpyDeviceToHost, stream));
        LB_CU(cudaMemcpyAsync(&h_scan_last, scn + (m - 1), 4, cudaMemcpyDeviceToHost, stream));
        LB_CU(cudaMemcpyAsync(h_root, nlo, 16, cudaMemcpyDeviceToHost, stream));
        LB_CU(cudaMemcpyAsync(h_root + 1, nhi, 16, cudaMemcpyDeviceToHost, stream));
    } else {
        LB_CU(cudaMemcpyAsync(h_root, blo, 16, cudaMemcpyDeviceToHost, stream));
        LB_CU(cudaMemcpyAsync(h_root + 1, bhi, 16, cudaMemcpyDeviceToHost, stream));
    }
    LB_CU(cudaStreamSynchronize(stream));
    if (h_cb[6] != 0xffffffffu) {
        const pt_face& f = hs.faces[h_cb[6]];
        set_error("face " + std::to_string(h_cb[6]) + " has vertex indices (" + std::to_string(f.v0) + ", " +
                  std::to_string(f.v1) + ", " + std::to_string(f.v2) + ") or material id " +
                  std::to_string(f.material_id) + " out of range (" + std::to_string(nv) + " vertices, " +
                  std::to_string(hs.materials.size()) + " materials)");
        return PT_ERR_INVALID;
    }
    if (h_cb[8]) {
        set_error("GPU BVH build: a climb to the root did not end (malformed tree)");
        return PT_ERR_DEVICE;
    }
    const uint32_t kept = m > 0 ? h_scan_last + h_keep_last : 0;
    const uint32_t depth = h_cb[7];
    if (depth >= static_cast<uint32_t>(kStackDepth)) {
        set_error("GPU BVH depth " + std::to_string(depth) + " exceeds the traversal stack (" +
                  std::to_string(kStackDepth) + "); build on the host instead");
        return PT_ERR_INVALID;
    }

    const auto t_dl0 = clock::now();
    t.inner.resize(kept);
    t.tris.resize(n);
    // the reordered faces land in a staging array and replace the scene's
    // only once the tree has passed its check
    std::unique_ptr<pt_face[]> faces_out(new pt_face[n]);
    touch_pages(t.inner.data(), size_t(kept) * sizeof(InnerNode));
    touch_pages(t.tris.data(), size_t(n) * sizeof(TriRecord));
    touch_pages(faces_out.get(), size_t(n) * sizeof(pt_face));
    if (kept)
        LB_CU(cudaMemcpyAsync(t.inner.data(), d_inner, size_t(kept) * sizeof(InnerNode), cudaMemcpyDeviceToHost,
                              stream));
    LB_CU(cudaMemcpyAsync(t.tris.data(), d_tris, size_t(n) * sizeof(TriRecord), cudaMemcpyDeviceToHost, stream));
    LB_CU(cudaMemcpyAsync(faces_out.get(), d_fout, size_t(n) * sizeof(pt_face), cudaMemcpyDeviceToHost, stream));
    LB_CU(cudaStreamSynchronize(stream));
    const auto t_dl = clock::now();

    {
        std::string why;
        if (kept == 0) t.tris[n - 1].flags |= 1u;
        t.root_ref = kept == 0 ? kLeafBit : 0u;
        if (!check_tree(t, n, why)) {
            set_error("GPU BVH build produced a malformed tree (" + why + ")");
            t = SceneTables{};
            return PT_ERR_DEVICE;
        }
    }
    std::memcpy(hs.faces.data(), faces_out.get(), size_t(n) * sizeof(pt_face));
    for (int a = 0; a < 3; ++a) {
        t.root_lo[a] = (&h_root[0].x)[a];
        t.root_hi[a] = (&h_root[1].x)[a];
    }
    t.num_leaves = kept == 0 ? 1u : h_leaves;   // kept == 0: the whole scene is one leaf
    t.bvh_depth = depth;
    build_emissive_tables(hs, t);
    t.built = true;
    const auto t_end = clock::now();

    float ms_up = 0, ms_build = 0;
    cudaEventElapsedTime(&ms_up, ev[0], ev[1]);
    cudaEventElapsedTime(&ms_build, ev[1], ev[2]);
    st.upload_ms = ms_up;
    st.device_ms = ms_build;
    st.download_ms = std::chrono::duration<double, std::milli>(t_dl - t_dl0).count();
    st.tables_ms = std::chrono::duration<double, std::milli>(t_end - t_dl).count() + env_ms;
    st.setup_ms = std::chrono::duration<double, std::milli>(t_setup - t_start).count();
    st.total_ms = std::chrono::duration<double, std::milli>(t_end - t_start).count();
    st.inner_nodes = kept;
    st.leaves = t.num_leaves;
    st.depth = depth;
    if (stats) *stats = st;
    return PT_OK;
}

}  // namespace ptb
