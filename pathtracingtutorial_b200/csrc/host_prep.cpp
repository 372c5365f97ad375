// host_prep.cpp -- scene preparation on the host: SAH BVH, light tables,
// camera basis, and the traversal layout uploaded to the GPU.
//
// The BVH must reproduce the reference's node order and face order exactly,
// because triangle ids (BVH-ordered face indices) are compared bit for bit.
// The reference algorithm (Part_2/src/accel/bvh_builder.cpp:56-221):
//   * per-primitive boxes from the three vertex positions;
//   * a node over [start, end) becomes a leaf below 4 primitives;
//   * otherwise 24 centroid buckets along the centroid-box max axis, forward and
//     backward sweeps of count * surface area, the first minimum over the 23
//     split positions, cost 0.5 + min/SA(node); a leaf if count < that cost;
//   * std::partition of the primitive range by "bucket <= best bucket" (the
//     partition algorithm itself fixes the resulting order, so the same
//     libstdc++ std::partition is called here);
//   * left-first depth-first renumbering of the nodes; faces permuted to the
//     final primitive order.
// This implementation differs in how it gets there: large ranges bin and
// bound in parallel chunks (min/max and counts are order independent, so the
// result is bit-identical), subtrees are built by a bounded set of worker
// threads, and the renumbering is iterative.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <future>
#include <queue>
#include <thread>

#include "engine.h"

namespace ptb {

namespace {

constexpr int kLeafThreshold = 4;
constexpr int kBuckets       = 24;
constexpr int kSplits        = kBuckets - 1;
constexpr uint32_t kParallelMin   = 1024;     // subtree size worth a task
constexpr uint32_t kChunkedMin    = 1u << 18; // range size worth chunked binning
constexpr int      kMaxTaskDepth  = 10;

struct Prim {
    float lo[3];
    float hi[3];
    uint32_t index;
    float centroid(int a) const { return 0.5f * (lo[a] + hi[a]); }
};

struct Box {
    float lo[3], hi[3];
    void reset() {
        lo[0] = lo[1] = lo[2] = FLT_MAX;
        hi[0] = hi[1] = hi[2] = -FLT_MAX;
    }
    void grow(const float* l, const float* h) {
        for (int i = 0; i < 3; ++i) { lo[i] = std::fmin(lo[i], l[i]); hi[i] = std::fmax(hi[i], h[i]); }
    }
    void grow_point(float x, float y, float z) {
        lo[0] = std::fmin(lo[0], x); hi[0] = std::fmax(hi[0], x);
        lo[1] = std::fmin(lo[1], y); hi[1] = std::fmax(hi[1], y);
        lo[2] = std::fmin(lo[2], z); hi[2] = std::fmax(hi[2], z);
    }
    float area() const {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
        return 2.0f * (dx * dy + dx * dz + dy * dz);
    }
    int max_axis() const {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (dx > dy && dx > dz) return 0;
        return dy > dz ? 1 : 2;
    }
};

struct Bucket { Box box; uint32_t count; };

int hardware_threads() {
    unsigned n = std::thread::hardware_concurrency();
    return n == 0 ? 1 : static_cast<int>(std::min(n, 64u));
}

class SahBuilder {
public:
    SahBuilder(std::vector<Prim>& prims, std::vector<pt_bvh_node>& nodes)
        : prims_(prims), nodes_(nodes), threads_(hardware_threads()) {}

    uint32_t build(uint32_t start, uint32_t end, int depth) {
        const uint32_t me = counter_.fetch_add(1, std::memory_order_relaxed);
        Box node_box, cent_box;
        bounds(start, end, node_box, cent_box);
        const uint32_t count = end - start;
        if (count < static_cast<uint32_t>(kLeafThreshold)) return make_leaf(me, node_box, start, count);
        const uint32_t mid = split(start, end, node_box, cent_box);
        if (mid == end) return make_leaf(me, node_box, start, count);
        uint32_t left, right;
        if (count > kParallelMin && depth < kMaxTaskDepth) {
            auto fut = std::async(std::launch::async, &SahBuilder::build, this, start, mid, depth + 1);
            right = build(mid, end, depth + 1);
            left = fut.get();
        } else {
            left = build(start, mid, depth + 1);
            right = build(mid, end, depth + 1);
        }
        pt_bvh_node& n = nodes_[me];
        for (int i = 0; i < 3; ++i) { n.bmin[i] = node_box.lo[i]; n.bmax[i] = node_box.hi[i]; }
        n.data0 = left;
        n.data1 = right;
        return me;
    }

    uint32_t node_count() const { return counter_.load(); }

private:
    uint32_t make_leaf(uint32_t me, const Box& b, uint32_t first, uint32_t count) {
        pt_bvh_node& n = nodes_[me];
        for (int i = 0; i < 3; ++i) { n.bmin[i] = b.lo[i]; n.bmax[i] = b.hi[i]; }
        n.data0 = first | 0x80000000u;
        n.data1 = count;
        return me;
    }

    // Node bounds and centroid bounds; chunked over threads for big ranges.
    void bounds(uint32_t start, uint32_t end, Box& nb, Box& cb) const {
        nb.reset(); cb.reset();
        const uint32_t count = end - start;
        if (count < kChunkedMin || threads_ == 1) {
            for (uint32_t i = start; i < end; ++i) {
                const Prim& p = prims_[i];
                nb.grow(p.lo, p.hi);
                cb.grow_point(p.centroid(0), p.centroid(1), p.centroid(2));
            }
            return;
        }
        const int nt = threads_;
        std::vector<Box> nbs(nt), cbs(nt);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) {
            pool.emplace_back([&, t] {
                const uint32_t a = start + static_cast<uint32_t>((uint64_t)count * t / nt);
                const uint32_t b = start + static_cast<uint32_t>((uint64_t)count * (t + 1) / nt);
                nbs[t].reset(); cbs[t].reset();
                for (uint32_t i = a; i < b; ++i) {
                    const Prim& p = prims_[i];
                    nbs[t].grow(p.lo, p.hi);
                    cbs[t].grow_point(p.centroid(0), p.centroid(1), p.centroid(2));
                }
            });
        }
        for (auto& th : pool) th.join();
        for (int t = 0; t < nt; ++t) { nb.grow(nbs[t].lo, nbs[t].hi); cb.grow(cbs[t].lo, cbs[t].hi); }
    }

    static int bucket_of(const Prim& p, int dim, const Box& cb) {
        const float c = p.centroid(dim);
        const float d = cb.hi[dim] - cb.lo[dim];
        const float off = d > 0 ? (c - cb.lo[dim]) / d : 0.0f;
        const int b = static_cast<int>(kBuckets * off);
        return b >= kBuckets ? kBuckets - 1 : b;
    }

    void bin(uint32_t start, uint32_t end, int dim, const Box& cb, Bucket* out) const {
        for (int b = 0; b < kBuckets; ++b) { out[b].box.reset(); out[b].count = 0; }
        const uint32_t count = end - start;
        if (count < kChunkedMin || threads_ == 1) {
            for (uint32_t i = start; i < end; ++i) {
                const int b = bucket_of(prims_[i], dim, cb);
                out[b].count++;
                out[b].box.grow(prims_[i].lo, prims_[i].hi);
            }
            return;
        }
        const int nt = threads_;
        std::vector<Bucket> part(static_cast<size_t>(nt) * kBuckets);
        std::vector<std::thread> pool;
        for (int t = 0; t < nt; ++t) {
            pool.emplace_back([&, t] {
                Bucket* my = part.data() + static_cast<size_t>(t) * kBuckets;
                for (int b = 0; b < kBuckets; ++b) { my[b].box.reset(); my[b].count = 0; }
                const uint32_t a = start + static_cast<uint32_t>((uint64_t)count * t / nt);
                const uint32_t e = start + static_cast<uint32_t>((uint64_t)count * (t + 1) / nt);
                for (uint32_t i = a; i < e; ++i) {
                    const int b = bucket_of(prims_[i], dim, cb);
                    my[b].count++;
                    my[b].box.grow(prims_[i].lo, prims_[i].hi);
                }
            });
        }
        for (auto& th : pool) th.join();
        for (int t = 0; t < nt; ++t)
            for (int b = 0; b < kBuckets; ++b) {
                const Bucket& s = part[static_cast<size_t>(t) * kBuckets + b];
                out[b].count += s.count;
                out[b].box.grow(s.box.lo, s.box.hi);
            }
    }

    // Returns the partition point, or `end` for "make a leaf".
    uint32_t split(uint32_t start, uint32_t end, const Box& nb, const Box& cb) {
        const int dim = cb.max_axis();
        Bucket bk[kBuckets];
        bin(start, end, dim, cb, bk);
        float cost[kSplits];
        uint32_t n_fwd = 0;
        Box fwd; fwd.reset();
        for (int i = 0; i < kSplits; ++i) {
            n_fwd += bk[i].count;
            fwd.grow(bk[i].box.lo, bk[i].box.hi);
            cost[i] = 0.0f;
            cost[i] += n_fwd * fwd.area();
        }
        uint32_t n_bwd = 0;
        Box bwd; bwd.reset();
        for (int i = kSplits - 1; i >= 0; --i) {
            n_bwd += bk[i + 1].count;
            bwd.grow(bk[i + 1].box.lo, bk[i + 1].box.hi);
            cost[i] += n_bwd * bwd.area();
        }
        int best = 0;
        for (int i = 1; i < kSplits; ++i)
            if (cost[i] < cost[best]) best = i;
        const float node_area = nb.area();
        const float split_cost = 0.5f + (node_area > 0.0f ? cost[best] / node_area : 0.0f);
        const float leaf_cost = static_cast<float>(end - start);
        if (leaf_cost < split_cost) return end;
        auto it = std::partition(prims_.begin() + start, prims_.begin() + end,
                                 [&](const Prim& p) { return bucket_of(p, dim, cb) <= best; });
        return static_cast<uint32_t>(it - prims_.begin());
    }

    std::vector<Prim>&        prims_;
    std::vector<pt_bvh_node>& nodes_;
    std::atomic<uint32_t>     counter_{0};
    int                       threads_;
};

}  // namespace

bool build_bvh(const std::vector<pt_vertex>& vertices, std::vector<pt_face>& faces,
               std::vector<pt_bvh_node>& out, uint32_t& depth) {
    out.clear();
    depth = 0;
    const size_t n = faces.size();
    if (n == 0) return true;
    if (n >= 0x7fffffffu) { set_error("too many faces for 31-bit primitive ids"); return false; }
    std::vector<Prim> prims(n);
    for (size_t i = 0; i < n; ++i) {
        const pt_face& f = faces[i];
        if (f.v0 >= vertices.size() || f.v1 >= vertices.size() || f.v2 >= vertices.size()) {
            set_error("face " + std::to_string(i) + " references a vertex out of range");
            return false;
        }
        const float* p0 = vertices[f.v0].position;
        const float* p1 = vertices[f.v1].position;
        const float* p2 = vertices[f.v2].position;
        Prim& p = prims[i];
        p.index = static_cast<uint32_t>(i);
        for (int a = 0; a < 3; ++a) {
            p.lo[a] = std::fmin(std::fmin(p0[a], p1[a]), p2[a]);
            p.hi[a] = std::fmax(std::fmax(p0[a], p1[a]), p2[a]);
        }
    }
    std::vector<pt_bvh_node> tmp(2 * n);
    uint32_t count;
    {
        SahBuilder b(prims, tmp);
        b.build(0, static_cast<uint32_t>(n), 0);
        count = b.node_count();
    }
    // Left-first depth-first renumbering.
    out.resize(count);
    struct Item { uint32_t old_idx; uint32_t parent_new; uint8_t side; uint32_t level; };
    std::vector<Item> stack;
    stack.push_back({0u, 0xffffffffu, 0, 0});
    uint32_t next = 0;
    while (!stack.empty()) {
        const Item it = stack.back();
        stack.pop_back();
        const uint32_t me = next++;
        out[me] = tmp[it.old_idx];
        depth = std::max(depth, it.level);
        if (it.parent_new != 0xffffffffu) {
            if (it.side == 0) out[it.parent_new].data0 = me; else out[it.parent_new].data1 = me;
        }
        const pt_bvh_node& src = tmp[it.old_idx];
        if (!(src.data0 & 0x80000000u)) {
            stack.push_back({src.data1, me, 1, it.level + 1});
            stack.push_back({src.data0, me, 0, it.level + 1});
        }
    }
    std::vector<pt_face> reordered(n);
    for (size_t i = 0; i < n; ++i) reordered[i] = faces[prims[i].index];
    faces.swap(reordered);
    return true;
}

// ---------------------------------------------------------------------------
// Light tables (Part_2/src/lights/light_sampler.cpp:7-149).
// ---------------------------------------------------------------------------
std::vector<pt_alias_entry> build_alias_table(const std::vector<float>& weights) {
    const uint32_t n = static_cast<uint32_t>(weights.size());
    if (n == 0) return {};
    float total = 0.0f;
    for (float w : weights) total += w;
    if (total <= 0.0f) return {};
    std::vector<float> scaled(n);
    for (uint32_t i = 0; i < n; ++i) scaled[i] = weights[i] / total * static_cast<float>(n);
    std::vector<pt_alias_entry> table(n);
    std::queue<uint32_t> lo, hi;
    for (uint32_t i = 0; i < n; ++i) (scaled[i] < 1.0f ? lo : hi).push(i);
    while (!lo.empty() && !hi.empty()) {
        const uint32_t s = lo.front(); lo.pop();
        const uint32_t l = hi.front(); hi.pop();
        table[s].prob = scaled[s];
        table[s].alias = l;
        scaled[l] = (scaled[l] + scaled[s]) - 1.0f;
        (scaled[l] < 1.0f ? lo : hi).push(l);
    }
    while (!hi.empty()) { const uint32_t l = hi.front(); hi.pop(); table[l].prob = 1.0f; table[l].alias = l; }
    while (!lo.empty()) { const uint32_t s = lo.front(); lo.pop(); table[s].prob = 1.0f; table[s].alias = s; }
    return table;
}

static float face_area(const pt_vertex& a, const pt_vertex& b, const pt_vertex& c) {
    const f3 e1 = ld3(b.position) - ld3(a.position);
    const f3 e2 = ld3(c.position) - ld3(a.position);
    return 0.5f * length(cross(e1, e2));
}

void build_emissive_tables(const HostScene& hs, SceneTables& t) {
    t.emissive.clear();
    t.tri_pmf.assign(hs.faces.size(), 0.0f);
    t.tri_alias.clear();
    std::vector<float> w;
    for (uint32_t i = 0; i < static_cast<uint32_t>(hs.faces.size()); ++i) {
        const pt_face& f = hs.faces[i];
        if (f.material_id < 0 || f.material_id >= static_cast<int>(hs.materials.size())) continue;
        const pt_material& m = hs.materials[f.material_id];
        const bool emits = m.emissive_strength > 0.0f &&
                           (m.emissive[0] > 0.0f || m.emissive[1] > 0.0f || m.emissive[2] > 0.0f);
        if (!emits) continue;
        const float area = face_area(hs.vertices[f.v0], hs.vertices[f.v1], hs.vertices[f.v2]);
        if (area <= 0.0f) continue;
        const f3 le = ld3(m.emissive) * m.emissive_strength;
        const float wt = area * std::fmax(luminance(le), 0.0f);
        if (wt <= 0.0f) continue;
        pt_emissive_ref r{};
        r.triangle_index = i;
        t.emissive.push_back(r);
        w.push_back(wt);
    }
    if (t.emissive.empty()) return;
    float total = 0.0f;
    for (float x : w) total += x;
    if (total <= 0.0f) { t.emissive.clear(); return; }
    float acc = 0.0f;
    for (size_t i = 0; i < t.emissive.size(); ++i) {
        const float pmf = w[i] / total;
        acc += pmf;
        t.emissive[i].selection_pmf = pmf;
        t.emissive[i].cdf = acc;
        t.tri_pmf[t.emissive[i].triangle_index] = pmf;
    }
    t.emissive.back().cdf = 1.0f;
    t.tri_alias = build_alias_table(w);
}

void build_env_tables(const HostScene& hs, SceneTables& t) {
    t.env_pmf.clear();
    t.env_alias.clear();
    t.env_w = t.env_h = 0;
    if (hs.env_w <= 0 || hs.env_h <= 0 || hs.env_rgba.size() < static_cast<size_t>(hs.env_w) * hs.env_h * 4) return;
    const int w = hs.env_w, h = hs.env_h;
    const size_t n = static_cast<size_t>(w) * h;
    std::vector<float> wt(n, 0.0f);
    for (int y = 0; y < h; ++y) {
        const float theta = kPi * (static_cast<float>(y) + 0.5f) / static_cast<float>(h);
        const float st = std::fmax(std::sin(theta), 0.0f);
        for (int x = 0; x < w; ++x) {
            const size_t idx = static_cast<size_t>(y) * w + x;
            const float* px = &hs.env_rgba[idx * 4];
            wt[idx] = std::fmax(luminance(mk(px[0], px[1], px[2])), 0.0f) * st;
        }
    }
    float total = 0.0f;
    for (float x : wt) total += x;
    if (total <= 0.0f) return;
    t.env_w = w;
    t.env_h = h;
    t.env_pmf.resize(n);
    for (size_t i = 0; i < n; ++i) t.env_pmf[i] = wt[i] / total;
    t.env_alias = build_alias_table(wt);
}

// ---------------------------------------------------------------------------
// Traversal layout: inner nodes carrying both child boxes, triangle records.
// ---------------------------------------------------------------------------
bool build_traversal_layout(const HostScene& hs, SceneTables& t) {
    t.inner.clear();
    t.tris.clear();
    t.num_leaves = 0;
    const std::vector<pt_bvh_node>& nodes = t.bvh;
    if (nodes.empty()) { t.root_ref = 0; return true; }
    std::vector<uint32_t> inner_index(nodes.size(), 0xffffffffu);
    uint32_t ni = 0;
    for (size_t i = 0; i < nodes.size(); ++i) {
        if (nodes[i].data0 & 0x80000000u) ++t.num_leaves;
        else inner_index[i] = ni++;
    }
    auto child_ref = [&](uint32_t c) -> uint32_t {
        const pt_bvh_node& n = nodes[c];
        return (n.data0 & 0x80000000u) ? (kLeafBit | (n.data0 & 0x7fffffffu)) : inner_index[c];
    };
    t.inner.resize(ni);
    for (size_t i = 0; i < nodes.size(); ++i) {
        const pt_bvh_node& n = nodes[i];
        if (n.data0 & 0x80000000u) continue;
        const pt_bvh_node& l = nodes[n.data0];
        const pt_bvh_node& r = nodes[n.data1];
        InnerNode& o = t.inner[inner_index[i]];
        o.c0lo[0] = l.bmin[0]; o.c0lo[1] = l.bmin[1]; o.c0lo[2] = l.bmin[2];
        o.c0hi_x = l.bmax[0]; o.c0hi_yz[0] = l.bmax[1]; o.c0hi_yz[1] = l.bmax[2];
        o.c1lo_xy[0] = r.bmin[0]; o.c1lo_xy[1] = r.bmin[1]; o.c1lo_z = r.bmin[2];
        o.c1hi[0] = r.bmax[0]; o.c1hi[1] = r.bmax[1]; o.c1hi[2] = r.bmax[2];
        o.ref0 = child_ref(n.data0);
        o.ref1 = child_ref(n.data1);
        // order rule: parent's max-extent axis, child centroids (bvh_common.h:43-53)
        const float dx = n.bmax[0] - n.bmin[0], dy = n.bmax[1] - n.bmin[1], dz = n.bmax[2] - n.bmin[2];
        const uint32_t axis = (dx > dy && dx > dz) ? 0u : (dy > dz ? 1u : 2u);
        const float cl = 0.5f * (l.bmin[axis] + l.bmax[axis]);
        const float cr = 0.5f * (r.bmin[axis] + r.bmax[axis]);
        o.meta = axis | ((cl < cr) ? 4u : 0u);
        o.pad = 0;
    }
    const size_t nf = hs.faces.size();
    t.tris.resize(nf);
    for (size_t i = 0; i < nf; ++i) {
        const pt_face& f = hs.faces[i];
        const float* p0 = hs.vertices[f.v0].position;
        const float* p1 = hs.vertices[f.v1].position;
        const float* p2 = hs.vertices[f.v2].position;
        TriRecord& r = t.tris[i];
        r.v0[0] = p0[0]; r.v0[1] = p0[1]; r.v0[2] = p0[2];
        r.e1x = p1[0] - p0[0]; r.e1yz[0] = p1[1] - p0[1]; r.e1yz[1] = p1[2] - p0[2];
        r.e2xy[0] = p2[0] - p0[0]; r.e2xy[1] = p2[1] - p0[1]; r.e2z = p2[2] - p0[2];
        r.flags = 0; r.pad[0] = r.pad[1] = 0;
    }
    for (size_t i = 0; i < nodes.size(); ++i) {
        const pt_bvh_node& n = nodes[i];
        if (!(n.data0 & 0x80000000u)) continue;
        const uint32_t first = n.data0 & 0x7fffffffu, cnt = n.data1;
        if (cnt == 0 || first + cnt > nf) { set_error("malformed BVH leaf"); return false; }
        t.tris[first + cnt - 1].flags |= 1u;
    }
    const pt_bvh_node& root = nodes[0];
    for (int a = 0; a < 3; ++a) { t.root_lo[a] = root.bmin[a]; t.root_hi[a] = root.bmax[a]; }
    t.root_ref = (root.data0 & 0x80000000u) ? (kLeafBit | (root.data0 & 0x7fffffffu)) : 0u;
    return true;
}

// The reference's node layout (BVHNode, Part_2/src/accel/bvh.h) recovered from
// the traversal layout, for trees that exist only in that layout (built on the
// device): inner node k keeps index k, leaves follow in the order their parents
// list them; a node's box is the one its parent carries (the root's is
// root_lo/hi), a leaf's count runs to its flagged last triangle record.
bool nodes_from_traversal_layout(const SceneTables& t, std::vector<pt_bvh_node>& nodes) {
    nodes.clear();
    if (!t.built || t.tris.empty()) return true;
    const uint32_t ni = static_cast<uint32_t>(t.inner.size());
    const uint32_t nt = static_cast<uint32_t>(t.tris.size());
    auto leaf_count = [&](uint32_t first, uint32_t& cnt) {
        uint32_t i = first;
        while (i < nt && !(t.tris[i].flags & 1u)) ++i;
        if (i >= nt) return false;
        cnt = i - first + 1;
        return true;
    };
    auto set_box = [](pt_bvh_node& n, const float* lo, const float* hi) {
        for (int a = 0; a < 3; ++a) { n.bmin[a] = lo[a]; n.bmax[a] = hi[a]; }
    };
    if (t.root_ref & kLeafBit) {
        nodes.resize(1);
        uint32_t cnt = 0;
        if (!leaf_count(t.root_ref & ~kLeafBit, cnt)) { set_error("malformed leaf"); return false; }
        set_box(nodes[0], t.root_lo, t.root_hi);
        nodes[0].data0 = t.root_ref;
        nodes[0].data1 = cnt;
        return true;
    }
    nodes.resize(ni);
    set_box(nodes[0], t.root_lo, t.root_hi);
    for (uint32_t k = 0; k < ni; ++k) {
        const InnerNode& o = t.inner[k];
        const float lo0[3] = {o.c0lo[0], o.c0lo[1], o.c0lo[2]}, hi0[3] = {o.c0hi_x, o.c0hi_yz[0], o.c0hi_yz[1]};
        const float lo1[3] = {o.c1lo_xy[0], o.c1lo_xy[1], o.c1lo_z}, hi1[3] = {o.c1hi[0], o.c1hi[1], o.c1hi[2]};
        uint32_t idx[2];
        const uint32_t refs[2] = {o.ref0, o.ref1};
        const float* los[2] = {lo0, lo1};
        const float* his[2] = {hi0, hi1};
        for (int c = 0; c < 2; ++c) {
            pt_bvh_node n{};
            set_box(n, los[c], his[c]);
            if (refs[c] & kLeafBit) {
                uint32_t cnt = 0;
                if (!leaf_count(refs[c] & ~kLeafBit, cnt)) { set_error("malformed leaf"); return false; }
                n.data0 = refs[c];
                n.data1 = cnt;
                idx[c] = static_cast<uint32_t>(nodes.size());
                nodes.push_back(n);
            } else {
                if (refs[c] >= ni || refs[c] == 0) { set_error("malformed inner node reference"); return false; }
                idx[c] = refs[c];
                set_box(nodes[refs[c]], los[c], his[c]);
            }
        }
        nodes[k].data0 = idx[0];
        nodes[k].data1 = idx[1];
    }
    return true;
}

// ---------------------------------------------------------------------------
// Camera basis (Part_2/src/camera/camera.h:36-51).
// ---------------------------------------------------------------------------
pt_camera_frame camera_frame(const pt_camera& cam) {
    const f3 pos = ld3(cam.position);
    const f3 fwd = normalize(ld3(cam.look_at) - pos);
    const f3 rgt = normalize(cross(fwd, ld3(cam.up)));
    const f3 cup = cross(rgt, fwd);
    pt_camera_frame f{};
    f.position[0] = pos.x; f.position[1] = pos.y; f.position[2] = pos.z;
    f.forward[0] = fwd.x;  f.forward[1] = fwd.y;  f.forward[2] = fwd.z;
    f.right[0] = rgt.x;    f.right[1] = rgt.y;    f.right[2] = rgt.z;
    f.up[0] = cup.x;       f.up[1] = cup.y;       f.up[2] = cup.z;
    f.tan_half_fov = std::tan(cam.fov * kPi / 360.0f);
    f.aspect = static_cast<float>(cam.width) / cam.height;
    f.aperture = cam.aperture;
    f.focal_distance = cam.focal_distance;
    return f;
}

pt_render_settings default_settings() {
    pt_render_settings s{};
    s.spp = 100000;
    s.sample_per_frame = 4;
    s.max_depth = 8;
    s.sampler_type = PT_SAMPLER_SOBOL;
    s.pcg_seed = 0;
    s.arg_order = PT_ARGS_LTR;
    s.flags = 0;
    return s;
}

pt_camera default_camera() {
    pt_camera c{};
    c.position[0] = 0; c.position[1] = 0; c.position[2] = 4;
    c.look_at[0] = 0; c.look_at[1] = 0; c.look_at[2] = 0;
    c.up[0] = 0; c.up[1] = 1; c.up[2] = 0;
    c.fov = 90.0f; c.aperture = 0.0f; c.focal_distance = 10.0f;
    c.width = 1600; c.height = 1600;
    return c;
}

pt_material default_material() {
    pt_material m{};
    m.base_color[0] = m.base_color[1] = m.base_color[2] = 0.8f;
    m.metallic = 0.0f; m.roughness = 0.5f; m.specular_tint = 0.0f; m.anisotropic = 0.0f;
    m.sheen = 0.0f; m.sheen_tint = 0.5f; m.clearcoat = 0.0f; m.clearcoat_roughness = 0.03f;
    m.spec_trans = 0.0f; m.ior = 1.5f; m.subsurface = 0.0f; m.specular_factor = 1.0f;
    m.specular_color_r = m.specular_color_g = m.specular_color_b = 1.0f;
    m.anisotropy_rotation = 0.0f; m.normal_scale = 1.0f;
    m.emissive[0] = m.emissive[1] = m.emissive[2] = 0.0f;
    m.emissive_strength = 1.0f; m.alpha_cutoff = 0.0f; m.alpha_mode = 0; m.base_alpha = 1.0f;
    m.double_sided = 0;
    m.sheen_color_r = m.sheen_color_g = m.sheen_color_b = 1.0f;
    m.occlusion_strength = 1.0f; m.thickness_factor = 0.0f; m.attenuation_distance = 1e30f;
    m.att_color_r = m.att_color_g = m.att_color_b = 1.0f;
    m.uv_offset_x = m.uv_offset_y = 0.0f; m.uv_scale_x = m.uv_scale_y = 1.0f; m.uv_rotation = 0.0f;
    m.base_color_tex = m.metallic_roughness_tex = m.normal_tex = m.emissive_tex = -1;
    m.occlusion_tex = m.clearcoat_tex = m.clearcoat_roughness_tex = m.clearcoat_normal_tex = -1;
    m.transmission_tex = m.sheen_color_tex = m.sheen_roughness_tex = -1;
    return m;
}

}  // namespace ptb
