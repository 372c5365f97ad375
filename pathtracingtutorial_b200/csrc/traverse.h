// traverse.h -- closest-hit and any-hit BVH traversal (host + device).
//
// Semantics are those of the reference's stack traversal
// (Part_2/src/accel/bvh_traversal.cuh:29-133) and Moller-Trumbore tests
// (Part_2/src/geometry/triangle.h:13-76), so that hit triangle ids and hit
// distances are bit-identical to the reference's IEEE (non-contracted) build:
//
//  * Box test: the reference's per-axis recurrence with t_min starting at 0
//    and t_max at the current best distance.  For NaN-free rays (every 1/d
//    finite) it equals  entry <= best && entry <= exit  with entry/exit the
//    usual slab max/min, which is what the fast path evaluates; rays with a
//    zero (or denormal) direction component take the literal recurrence, whose
//    NaN handling (an axis with a NaN bound is ignored) differs.
//  * Order: the reference pops the near child first, where "near" comes from
//    the parent's max-extent axis and the children's centroids compared with
//    the ray sign (bvh_traversal.cuh:81-92).  Here each inner node stores both
//    child boxes, so both are tested at the parent with the same best distance
//    the reference uses when it pops the near child; the far child is pushed
//    with its entry distance and re-tested against the best distance when
//    popped.  Visited set and visit order equal the reference's.
//  * Closest hit keeps the first hit found under strict '<' (ties resolved
//    exactly as in the reference); any-hit returns on the first triangle with
//    1e-4 < t < tMax, which is order independent.
//
// Watertight mode (PT_FLAG_WATERTIGHT; the reference has none): the triangle
// test is Woop, Benthin and Wald's (JCGT 2013) on the triangle's own shared
// vertex positions, so that two triangles sharing an edge see bit-identical
// transformed edge endpoints and exactly opposite edge functions, and the box
// test's exit distance is widened (Ize 2013, "Robust BVH Ray Traversal"), so
// no box that the ray touches is culled by rounding.  Visit order and the
// acceptance rules (t >= 1e-4, shadow t > 1e-4) are those of the default mode.
#pragma once

#include "pt_internal.h"

#if !defined(__CUDACC__)
#include <vector_types.h>
#endif

namespace ptb {

struct RayInv {
    float ox, oy, oz;
    float dx, dy, dz;
    float ix, iy, iz;
    float xs;          // box exit scale: 1 (the reference's test) or kWatertightExitScale
    int   sx, sy, sz;
    bool  nan_free;
};

// Widening of a box's exit distance.  A slab distance (l - o) * (1 / d) is
// off by a factor in [1 - gamma(3), 1 + gamma(3)], gamma(n) = n u / (1 - n u),
// u = 2^-24 (Ize 2013), so a box the ray touches passes whenever the exit is
// scaled by (1 + gamma(3)) / (1 - gamma(3)), just above 1 + 2 gamma(3) =
// 1 + 3.0000005 ulp; 1 + 4 ulp covers it and the rounding of the product.
constexpr float kWatertightExitScale = 1.0f + 4.0f * 1.1920929e-7f;

PT_HD RayInv make_ray_inv(float ox, float oy, float oz, float dx, float dy, float dz) {
    RayInv r;
    r.ox = ox; r.oy = oy; r.oz = oz;
    r.dx = dx; r.dy = dy; r.dz = dz;
    r.ix = x_rcp(dx); r.iy = x_rcp(dy); r.iz = x_rcp(dz);
    r.xs = 1.0f;
    r.sx = r.ix < 0.0f ? 1 : 0;
    r.sy = r.iy < 0.0f ? 1 : 0;
    r.sz = r.iz < 0.0f ? 1 : 0;
    r.nan_free = fabsf(r.ix) <= FLT_MAX && fabsf(r.iy) <= FLT_MAX && fabsf(r.iz) <= FLT_MAX;
    return r;
}

PT_HD float exit_scale(bool watertight) { return watertight ? kWatertightExitScale : 1.0f; }

// entry / exit of a box, with the reference's arithmetic; the exit is
// multiplied by r.xs (exact for the default 1).
PT_HD void box_span(const RayInv& r, float lx, float ly, float lz, float hx, float hy, float hz,
                    float& entry, float& exit_) {
    const float t1x = x_mul(x_sub(lx, r.ox), r.ix), t2x = x_mul(x_sub(hx, r.ox), r.ix);
    const float t1y = x_mul(x_sub(ly, r.oy), r.iy), t2y = x_mul(x_sub(hy, r.oy), r.iy);
    const float t1z = x_mul(x_sub(lz, r.oz), r.iz), t2z = x_mul(x_sub(hz, r.oz), r.iz);
    if (r.nan_free) {
        entry = fmaxf(fmaxf(fminf(t1x, t2x), fminf(t1y, t2y)), fmaxf(fminf(t1z, t2z), 0.0f));
        exit_ = x_mul(fminf(fminf(fmaxf(t1x, t2x), fmaxf(t1y, t2y)), fmaxf(t1z, t2z)), r.xs);
    } else {
        // literal recurrence (bvh_traversal.cuh:33-39) with t_max starting at +inf
        float tn = 0.0f, tf = INFINITY;
        tn = fminf(fmaxf(t1x, tn), fmaxf(t2x, tn)); tf = fmaxf(fminf(t1x, tf), fminf(t2x, tf));
        tn = fminf(fmaxf(t1y, tn), fmaxf(t2y, tn)); tf = fmaxf(fminf(t1y, tf), fminf(t2y, tf));
        tn = fminf(fmaxf(t1z, tn), fmaxf(t2z, tn)); tf = fmaxf(fminf(t1z, tf), fminf(t2z, tf));
        entry = tn; exit_ = x_mul(tf, r.xs);
    }
}

// Moller-Trumbore on a precomputed record.  Returns t (or -1).  `shadow`
// selects the reference's shadow acceptance (t > 1e-4) instead of the
// closest-hit one (t >= 1e-4).
PT_HD float tri_mt(const RayInv& r, float v0x, float v0y, float v0z,
                   float e1x, float e1y, float e1z, float e2x, float e2y, float e2z,
                   bool shadow, float& u_out, float& v_out) {
    const float px = x_sub(x_mul(r.dy, e2z), x_mul(r.dz, e2y));
    const float py = x_sub(x_mul(r.dz, e2x), x_mul(r.dx, e2z));
    const float pz = x_sub(x_mul(r.dx, e2y), x_mul(r.dy, e2x));
    const float det = x_add(x_add(x_mul(e1x, px), x_mul(e1y, py)), x_mul(e1z, pz));
    if (fabsf(det) < FLT_EPSILON) return -1.0f;
    const float inv = x_rcp(det);
    const float tx = x_sub(r.ox, v0x), ty = x_sub(r.oy, v0y), tz = x_sub(r.oz, v0z);
    const float u = x_mul(x_add(x_add(x_mul(tx, px), x_mul(ty, py)), x_mul(tz, pz)), inv);
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const float qx = x_sub(x_mul(ty, e1z), x_mul(tz, e1y));
    const float qy = x_sub(x_mul(tz, e1x), x_mul(tx, e1z));
    const float qz = x_sub(x_mul(tx, e1y), x_mul(ty, e1x));
    const float v = x_mul(x_add(x_add(x_mul(r.dx, qx), x_mul(r.dy, qy)), x_mul(r.dz, qz)), inv);
    if (v < 0.0f || x_add(u, v) > 1.0f) return -1.0f;
    const float t = x_mul(x_add(x_add(x_mul(e2x, qx), x_mul(e2y, qy)), x_mul(e2z, qz)), inv);
    if (shadow ? !(t > 1e-4f) : (t < 1e-4f)) return -1.0f;
    u_out = u; v_out = v;
    return t;
}

// Watertight ray/triangle test (Woop, Benthin, Wald 2013) on the absolute
// vertex positions p0, p1, p2 (the shared vertices of the mesh, not a
// per-triangle edge record): translate to the ray origin, shear and scale so
// the ray runs along +z, evaluate the three 2D edge functions, and redo them
// in double when one is exactly zero (products of floats are exact in
// double, so the signs are exact).  Every operation is explicitly rounded, so
// host and device agree bit for bit.  Barycentrics as the default test:
// u weights p1, v weights p2.
PT_HD float tri_watertight(const RayInv& r, const float* p0, const float* p1, const float* p2, bool shadow,
                           float& u_out, float& v_out) {
    const float adx = fabsf(r.dx), ady = fabsf(r.dy), adz = fabsf(r.dz);
    int kz = (adx > ady) ? (adx > adz ? 0 : 2) : (ady > adz ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    const float d[3] = {r.dx, r.dy, r.dz};
    if (d[kz] < 0.0f) { const int t = kx; kx = ky; ky = t; }
    const float sx = x_div(d[kx], d[kz]), sy = x_div(d[ky], d[kz]), sz = x_rcp(d[kz]);
    const float o[3] = {r.ox, r.oy, r.oz};
    float a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) {
        a[k] = x_sub(p0[k], o[k]);
        b[k] = x_sub(p1[k], o[k]);
        c[k] = x_sub(p2[k], o[k]);
    }
    const float ax = x_sub(a[kx], x_mul(sx, a[kz])), ay = x_sub(a[ky], x_mul(sy, a[kz]));
    const float bx = x_sub(b[kx], x_mul(sx, b[kz])), by = x_sub(b[ky], x_mul(sy, b[kz]));
    const float cx = x_sub(c[kx], x_mul(sx, c[kz])), cy = x_sub(c[ky], x_mul(sy, c[kz]));
    float U = x_sub(x_mul(cx, by), x_mul(cy, bx));
    float V = x_sub(x_mul(ax, cy), x_mul(ay, cx));
    float W = x_sub(x_mul(bx, ay), x_mul(by, ax));
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = static_cast<float>(xd_sub(xd_mul(cx, by), xd_mul(cy, bx)));
        V = static_cast<float>(xd_sub(xd_mul(ax, cy), xd_mul(ay, cx)));
        W = static_cast<float>(xd_sub(xd_mul(bx, ay), xd_mul(by, ax)));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return -1.0f;
    const float det = x_add(x_add(U, V), W);
    if (det == 0.0f) return -1.0f;
    const float az = x_mul(sz, a[kz]), bz = x_mul(sz, b[kz]), cz = x_mul(sz, c[kz]);
    const float T = x_add(x_add(x_mul(U, az), x_mul(V, bz)), x_mul(W, cz));
    const float inv = x_rcp(det);
    const float t = x_mul(T, inv);
    if (shadow ? !(t > 1e-4f) : (t < 1e-4f)) return -1.0f;
    u_out = x_mul(V, inv); v_out = x_mul(W, inv);
    return t;
}

struct TraceCounters { uint32_t inner; uint32_t tris; };

#if defined(__CUDA_ARCH__)
#  define PT_LDG4(p) __ldg(reinterpret_cast<const float4*>(p))
#  define PT_LDGU4(p) __ldg(reinterpret_cast<const uint4*>(p))
#else
#  define PT_LDG4(p) (*reinterpret_cast<const float4*>(p))
#  define PT_LDGU4(p) (*reinterpret_cast<const uint4*>(p))
#endif

PT_HD float tri_test(const DeviceScene& s, const RayInv& r, uint32_t ti, bool shadow, bool watertight,
                     float& u, float& v, bool& last) {
    const float* base = reinterpret_cast<const float*>(s.tris + ti);
    if (watertight) {
        last = (__float_as_uint_hd(PT_LDG4(base + 8).y) & 1u) != 0u;
        const uint4 f = PT_LDGU4(s.faces + ti);
        const float4 p0 = PT_LDG4(s.vertices[f.x].position);
        const float4 p1 = PT_LDG4(s.vertices[f.y].position);
        const float4 p2 = PT_LDG4(s.vertices[f.z].position);
        const float q0[3] = {p0.x, p0.y, p0.z}, q1[3] = {p1.x, p1.y, p1.z}, q2[3] = {p2.x, p2.y, p2.z};
        return tri_watertight(r, q0, q1, q2, shadow, u, v);
    }
    const float4 a = PT_LDG4(base);
    const float4 b = PT_LDG4(base + 4);
    const float4 c = PT_LDG4(base + 8);
    last = (__float_as_uint_hd(c.y) & 1u) != 0u;
    return tri_mt(r, a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, shadow, u, v);
}

// Closest hit.  Returns prim (BVH-ordered face index) or -1; t = FLT_MAX on miss.
PT_HD int trace_closest(const DeviceScene& s, const RayInv& ray, bool watertight,
                        float& t_out, float& u_out, float& v_out, uint32_t& err, TraceCounters& cnt) {
    RayInv r = ray;
    r.xs = exit_scale(watertight);
    float best = FLT_MAX;
    int prim = -1;
    float bu = 0.0f, bv = 0.0f;
    t_out = FLT_MAX; u_out = 0.0f; v_out = 0.0f;
    if (s.num_faces == 0) return -1;
    float en, ex;
    box_span(r, s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], en, ex);
    if (!(en <= best && en <= ex)) return -1;
    uint32_t stack_ref[kStackDepth];
    float    stack_t[kStackDepth];
    int sp = 0;
    uint32_t ref = s.root_ref;
    const int sgn[3] = {r.sx, r.sy, r.sz};
    for (;;) {
        if (ref & kLeafBit) {
            uint32_t ti = ref & ~kLeafBit;
            for (;;) {
                float u, v; bool last;
                const float t = tri_test(s, r, ti, false, watertight, u, v, last);
                ++cnt.tris;
                if (t >= 0.0f && t < best) { best = t; prim = (int)ti; bu = u; bv = v; }
                if (last) break;
                ++ti;
            }
        } else {
            ++cnt.inner;
            const float* nb = reinterpret_cast<const float*>(s.inner + ref);
            const float4 q0 = PT_LDG4(nb);
            const float4 q1 = PT_LDG4(nb + 4);
            const float4 q2 = PT_LDG4(nb + 8);
            const uint4  q3 = PT_LDGU4(nb + 12);
            float e0, x0, e1, x1;
            box_span(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, e0, x0);
            box_span(r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, e1, x1);
            const bool h0 = e0 <= best && e0 <= x0;
            const bool h1 = e1 <= best && e1 <= x1;
            const uint32_t axis = q3.z & 3u;
            const int lt = (int)((q3.z >> 2) & 1u);
            const bool right_first = sgn[axis] == lt;
            const uint32_t nref = right_first ? q3.y : q3.x;
            const uint32_t fref = right_first ? q3.x : q3.y;
            const bool hn = right_first ? h1 : h0;
            const bool hf = right_first ? h0 : h1;
            const float ef = right_first ? e0 : e1;
            if (hn) {
                if (hf) {
                    if (sp >= kStackDepth) { err |= kErrStackOverflow; break; }
                    stack_ref[sp] = fref; stack_t[sp] = ef; ++sp;
                }
                ref = nref;
                continue;
            }
            if (hf) { ref = fref; continue; }
        }
        // pop the next deferred child that still passes against the current best
        bool found = false;
        while (sp > 0) {
            --sp;
            if (stack_t[sp] <= best) { ref = stack_ref[sp]; found = true; break; }
        }
        if (!found) break;
    }
    if (prim >= 0) { t_out = best; u_out = bu; v_out = bv; }
    return prim;
}

// Any hit in (1e-4, tmax).
PT_HD bool trace_any(const DeviceScene& s, const RayInv& ray, float tmax, bool watertight,
                     uint32_t& err, TraceCounters& cnt) {
    if (s.num_faces == 0) return false;
    RayInv r = ray;
    r.xs = exit_scale(watertight);
    float en, ex;
    box_span(r, s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], en, ex);
    if (!(en <= tmax && en <= ex)) return false;
    uint32_t stack_ref[kStackDepth];
    int sp = 0;
    uint32_t ref = s.root_ref;
    const int sgn[3] = {r.sx, r.sy, r.sz};
    for (;;) {
        if (ref & kLeafBit) {
            uint32_t ti = ref & ~kLeafBit;
            for (;;) {
                float u, v; bool last;
                const float t = tri_test(s, r, ti, true, watertight, u, v, last);
                ++cnt.tris;
                if (t > 0.0f && t < tmax) return true;
                if (last) break;
                ++ti;
            }
        } else {
            ++cnt.inner;
            const float* nb = reinterpret_cast<const float*>(s.inner + ref);
            const float4 q0 = PT_LDG4(nb);
            const float4 q1 = PT_LDG4(nb + 4);
            const float4 q2 = PT_LDG4(nb + 8);
            const uint4  q3 = PT_LDGU4(nb + 12);
            float e0, x0, e1, x1;
            box_span(r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, e0, x0);
            box_span(r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, e1, x1);
            const bool h0 = e0 <= tmax && e0 <= x0;
            const bool h1 = e1 <= tmax && e1 <= x1;
            const uint32_t axis = q3.z & 3u;
            const int lt = (int)((q3.z >> 2) & 1u);
            const bool right_first = sgn[axis] == lt;
            const uint32_t nref = right_first ? q3.y : q3.x;
            const uint32_t fref = right_first ? q3.x : q3.y;
            const bool hn = right_first ? h1 : h0;
            const bool hf = right_first ? h0 : h1;
            if (hn) {
                if (hf) {
                    if (sp >= kStackDepth) { err |= kErrStackOverflow; return false; }
                    stack_ref[sp++] = fref;
                }
                ref = nref;
                continue;
            }
            if (hf) { ref = fref; continue; }
        }
        if (sp == 0) break;
        ref = stack_ref[--sp];
    }
    return false;
}

#if defined(__CUDACC__)
// ---------------------------------------------------------------------------
// Warp-scheduled traversal for the wavefront kernels.  Each lane walks its own
// ray with the visit order, tests and results of trace_closest / trace_any
// above, but the warp alternates two phases: all lanes that stand on inner
// nodes step through inner nodes until each reaches a leaf, then all lanes
// at a leaf test its triangles together.  A lane whose ray is finished takes
// its next ray (i + stride) at once instead of waiting for the warp's longest
// ray.  All 32 lanes of the warp must call these loops.
// ---------------------------------------------------------------------------
// Deferred children of one walk; Depth entries (the tuner picks 32 or 64; a
// tree needs more entries than its depth only never: the stack holds at most
// one far child per level).
template <int Depth = kStackDepth>
struct StepStack {
    uint32_t ref[Depth];
    float    t[Depth];
};

struct ClosestWalk {
    RayInv   r;
    float    best, bu, bv;
    int      prim;
    uint32_t ref;
    int      sp;
};

// Root test; false when the ray misses the scene box (or the scene is empty).
__device__ __forceinline__ bool closest_begin(const DeviceScene& s, ClosestWalk& w) {
    w.best = FLT_MAX; w.prim = -1; w.bu = 0.0f; w.bv = 0.0f; w.sp = 0;
    if (s.num_faces == 0) return false;
    float en, ex;
    box_span(w.r, s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], en, ex);
    if (!(en <= w.best && en <= ex)) return false;
    w.ref = s.root_ref;
    return true;
}

// Next deferred child that still passes against the current best; false at the end.
template <int Depth>
__device__ __forceinline__ bool closest_pop(ClosestWalk& w, const StepStack<Depth>& st) {
    while (w.sp > 0) {
        --w.sp;
        if (st.t[w.sp] <= w.best) { w.ref = st.ref[w.sp]; return true; }
    }
    return false;
}

// Inner node w.ref: both child boxes, then the next node; false at the end.
template <int Depth>
__device__ __forceinline__ bool closest_inner(const DeviceScene& s, ClosestWalk& w, StepStack<Depth>& st, uint32_t& err,
                                              TraceCounters& cnt) {
    ++cnt.inner;
    const float* nb = reinterpret_cast<const float*>(s.inner + w.ref);
    const float4 q0 = PT_LDG4(nb);
    const float4 q1 = PT_LDG4(nb + 4);
    const float4 q2 = PT_LDG4(nb + 8);
    const uint4  q3 = PT_LDGU4(nb + 12);
    float e0, x0, e1, x1;
    box_span(w.r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, e0, x0);
    box_span(w.r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, e1, x1);
    const bool h0 = e0 <= w.best && e0 <= x0;
    const bool h1 = e1 <= w.best && e1 <= x1;
    const uint32_t axis = q3.z & 3u;
    const int lt = static_cast<int>((q3.z >> 2) & 1u);
    const int sg = axis == 0 ? w.r.sx : (axis == 1 ? w.r.sy : w.r.sz);
    const bool right_first = sg == lt;
    const uint32_t nref = right_first ? q3.y : q3.x;
    const uint32_t fref = right_first ? q3.x : q3.y;
    const bool hn = right_first ? h1 : h0;
    const bool hf = right_first ? h0 : h1;
    const float ef = right_first ? e0 : e1;
    if (hn) {
        if (hf) {
            if (w.sp >= Depth) { err |= kErrStackOverflow; return false; }
            st.ref[w.sp] = fref; st.t[w.sp] = ef; ++w.sp;
        }
        w.ref = nref;
        return true;
    }
    if (hf) { w.ref = fref; return true; }
    return closest_pop(w, st);
}

// Leaf w.ref: its triangles, then the next node; false at the end.
template <int Depth>
__device__ __forceinline__ bool closest_leaf(const DeviceScene& s, ClosestWalk& w, StepStack<Depth>& st, bool watertight,
                                             TraceCounters& cnt) {
    uint32_t ti = w.ref & ~kLeafBit;
    for (;;) {
        float u, v; bool last;
        const float t = tri_test(s, w.r, ti, false, watertight, u, v, last);
        ++cnt.tris;
        if (t >= 0.0f && t < w.best) { w.best = t; w.prim = static_cast<int>(ti); w.bu = u; w.bv = v; }
        if (last) break;
        ++ti;
    }
    return closest_pop(w, st);
}

// Closest hits of rays first, first + stride, ... < n.  fetch(i, RayInv&)
// loads ray i; done(i, const ClosestWalk&) stores its result (prim < 0: miss).
template <int Depth = kStackDepth, class Fetch, class Done>
__device__ __forceinline__ void closest_loop(const DeviceScene& s, uint32_t i, uint32_t n, uint32_t stride,
                                             bool watertight, uint32_t& err, TraceCounters& cnt, Fetch&& fetch,
                                             Done&& done) {
    StepStack<Depth> st;
    ClosestWalk w;
    bool have = false;
    for (;;) {
        while (!have && i < n) {
            fetch(i, w.r);
            w.r.xs = exit_scale(watertight);
            if (closest_begin(s, w)) { have = true; }
            else { done(i, w); i += stride; }
        }
        if (!__any_sync(0xffffffffu, have)) break;
        bool fin = false;
        if (have) {
            while (!(w.ref & kLeafBit)) {
                if (!closest_inner(s, w, st, err, cnt)) { fin = true; break; }
            }
        }
        __syncwarp();
        if (have && !fin) fin = !closest_leaf(s, w, st, watertight, cnt);
        if (fin) { done(i, w); i += stride; have = false; }
    }
}

// Packet walk of the rays of one warp whose direction signs agree (sgn3: the
// shared sign bits x | y << 1 | z << 2).  The child order of every inner
// node depends only on the parent's axis and the ray's sign along it, so all
// lanes share one depth-first order, and the warp walks it together: every
// lane tests the boxes of the node in hand against its own best distance,
// the warp descends where any lane needs to, and a lane is active in exactly
// the nodes its own walk (closest_inner / closest_leaf) would visit, in the
// same order and with the same best distance at each -- so hits, distances
// and counters equal the per-lane walk's.  Stacked far children keep each
// lane's entry distance (+inf for lanes that do not need them); a pop takes
// the next entry some lane still needs.  Node and triangle loads are the same
// address on every lane.  `act` is false for lanes without a live ray.
template <int Depth>
__device__ __forceinline__ void closest_packet(const DeviceScene& s, ClosestWalk& w, bool act, int sgn3,
                                               StepStack<Depth>& st, bool watertight, uint32_t& err,
                                               TraceCounters& cnt) {
    uint32_t ref = s.root_ref;
    int sp = 0;
    for (;;) {
        if (!(ref & kLeafBit)) {
            if (act) ++cnt.inner;
            const float* nb = reinterpret_cast<const float*>(s.inner + ref);
            const float4 q0 = PT_LDG4(nb);
            const float4 q1 = PT_LDG4(nb + 4);
            const float4 q2 = PT_LDG4(nb + 8);
            const uint4  q3 = PT_LDGU4(nb + 12);
            float e0, x0, e1, x1;
            box_span(w.r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, e0, x0);
            box_span(w.r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, e1, x1);
            const bool h0 = act && e0 <= w.best && e0 <= x0;
            const bool h1 = act && e1 <= w.best && e1 <= x1;
            const uint32_t axis = q3.z & 3u;
            const int lt = static_cast<int>((q3.z >> 2) & 1u);
            const bool right_first = ((sgn3 >> axis) & 1) == lt;
            const uint32_t nref = right_first ? q3.y : q3.x;
            const uint32_t fref = right_first ? q3.x : q3.y;
            const bool hn = right_first ? h1 : h0;
            const bool hf = right_first ? h0 : h1;
            const float ef = right_first ? e0 : e1;
            const bool any_n = __any_sync(0xffffffffu, hn), any_f = __any_sync(0xffffffffu, hf);
            if (any_n) {
                if (any_f) {
                    if (sp >= Depth) { err |= kErrStackOverflow; break; }
                    st.ref[sp] = fref;
                    st.t[sp] = hf ? ef : INFINITY;
                    ++sp;
                }
                act = hn;
                ref = nref;
                continue;
            }
            if (any_f) { act = hf; ref = fref; continue; }
        } else if (act) {
            uint32_t ti = ref & ~kLeafBit;
            for (;;) {
                float u, v; bool last;
                const float t = tri_test(s, w.r, ti, false, watertight, u, v, last);
                ++cnt.tris;
                if (t >= 0.0f && t < w.best) { w.best = t; w.prim = static_cast<int>(ti); w.bu = u; w.bv = v; }
                if (last) break;
                ++ti;
            }
        }
        // the next stacked node some lane still needs
        bool found = false;
        while (sp > 0) {
            --sp;
            const bool need = st.t[sp] <= w.best;
            if (__any_sync(0xffffffffu, need)) { act = need; ref = st.ref[sp]; found = true; break; }
        }
        if (!found) break;
    }
}

// Closest hits of rays 32 t .. 32 t + 31 for the warp's tiles t = warp,
// warp + warps, ... (< n rays): a tile whose live rays share their direction
// signs is walked as a packet (closest_packet), any other lane by lane.  For
// coherent rays (camera rays of neighbouring pixels).  All 32 lanes call it.
template <int Depth = kStackDepth, class Fetch, class Done>
__device__ __forceinline__ void closest_packet_loop(const DeviceScene& s, uint32_t warp, uint32_t warps, uint32_t n,
                                                    bool watertight, uint32_t& err, TraceCounters& cnt,
                                                    Fetch&& fetch, Done&& done) {
    const uint32_t lane = threadIdx.x & 31u;
    StepStack<Depth> st;
    for (uint32_t base = warp * 32u; base < n; base += warps * 32u) {
        const uint32_t i = base + lane;
        const bool have = i < n;
        ClosestWalk w;
        w.best = FLT_MAX; w.prim = -1; w.bu = 0.0f; w.bv = 0.0f; w.sp = 0;
        bool alive = false;
        if (have) {
            fetch(i, w.r);
            w.r.xs = exit_scale(watertight);
            alive = closest_begin(s, w);
        }
        const int sgn3 = alive ? (w.r.sx | (w.r.sy << 1) | (w.r.sz << 2)) : -1;
        const uint32_t live = __ballot_sync(0xffffffffu, alive);
        if (live) {
            const int lead = __shfl_sync(0xffffffffu, sgn3, __ffs(live) - 1);
            if (__all_sync(0xffffffffu, !alive || sgn3 == lead)) {
                closest_packet<Depth>(s, w, alive, lead, st, watertight, err, cnt);
            } else if (alive) {
                for (;;) {
                    if (w.ref & kLeafBit) {
                        if (!closest_leaf(s, w, st, watertight, cnt)) break;
                    } else if (!closest_inner(s, w, st, err, cnt)) {
                        break;
                    }
                }
            }
        }
        if (have) done(i, w);
    }
}

struct AnyWalk {
    RayInv   r;
    float    tmax;
    uint32_t ref;
    int      sp;
    bool     hit;
};

__device__ __forceinline__ bool any_begin(const DeviceScene& s, AnyWalk& w) {
    w.sp = 0; w.hit = false;
    if (s.num_faces == 0) return false;
    float en, ex;
    box_span(w.r, s.root_lo[0], s.root_lo[1], s.root_lo[2], s.root_hi[0], s.root_hi[1], s.root_hi[2], en, ex);
    if (!(en <= w.tmax && en <= ex)) return false;
    w.ref = s.root_ref;
    return true;
}

template <int Depth>
__device__ __forceinline__ bool any_inner(const DeviceScene& s, AnyWalk& w, uint32_t* stack, uint32_t& err,
                                          TraceCounters& cnt) {
    ++cnt.inner;
    const float* nb = reinterpret_cast<const float*>(s.inner + w.ref);
    const float4 q0 = PT_LDG4(nb);
    const float4 q1 = PT_LDG4(nb + 4);
    const float4 q2 = PT_LDG4(nb + 8);
    const uint4  q3 = PT_LDGU4(nb + 12);
    float e0, x0, e1, x1;
    box_span(w.r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, e0, x0);
    box_span(w.r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, e1, x1);
    const bool h0 = e0 <= w.tmax && e0 <= x0;
    const bool h1 = e1 <= w.tmax && e1 <= x1;
    const uint32_t axis = q3.z & 3u;
    const int lt = static_cast<int>((q3.z >> 2) & 1u);
    const int sg = axis == 0 ? w.r.sx : (axis == 1 ? w.r.sy : w.r.sz);
    const bool right_first = sg == lt;
    const uint32_t nref = right_first ? q3.y : q3.x;
    const uint32_t fref = right_first ? q3.x : q3.y;
    const bool hn = right_first ? h1 : h0;
    const bool hf = right_first ? h0 : h1;
    if (hn) {
        if (hf) {
            if (w.sp >= Depth) { err |= kErrStackOverflow; return false; }
            stack[w.sp++] = fref;
        }
        w.ref = nref;
        return true;
    }
    if (hf) { w.ref = fref; return true; }
    if (w.sp == 0) return false;
    w.ref = stack[--w.sp];
    return true;
}

__device__ __forceinline__ bool any_leaf(const DeviceScene& s, AnyWalk& w, uint32_t* stack, bool watertight,
                                         TraceCounters& cnt) {
    uint32_t ti = w.ref & ~kLeafBit;
    for (;;) {
        float u, v; bool last;
        const float t = tri_test(s, w.r, ti, true, watertight, u, v, last);
        ++cnt.tris;
        if (t > 0.0f && t < w.tmax) { w.hit = true; return false; }
        if (last) break;
        ++ti;
    }
    if (w.sp == 0) return false;
    w.ref = stack[--w.sp];
    return true;
}

// Any-hit tests of rays first, first + stride, ... < n.  fetch(i, AnyWalk&)
// sets r and tmax; done(i, bool occluded) consumes the result.
template <int Depth = kStackDepth, class Fetch, class Done>
__device__ __forceinline__ void any_loop(const DeviceScene& s, uint32_t i, uint32_t n, uint32_t stride,
                                         bool watertight, uint32_t& err, TraceCounters& cnt, Fetch&& fetch,
                                         Done&& done) {
    uint32_t stack[Depth];
    AnyWalk w;
    bool have = false;
    for (;;) {
        while (!have && i < n) {
            fetch(i, w);
            w.r.xs = exit_scale(watertight);
            if (any_begin(s, w)) { have = true; }
            else { done(i, false); i += stride; }
        }
        if (!__any_sync(0xffffffffu, have)) break;
        bool fin = false;
        if (have) {
            while (!(w.ref & kLeafBit)) {
                if (!any_inner<Depth>(s, w, stack, err, cnt)) { fin = true; break; }
            }
        }
        __syncwarp();
        if (have && !fin) fin = !any_leaf(s, w, stack, watertight, cnt);
        if (fin) { done(i, w.hit); i += stride; have = false; }
    }
}
// Any-hit packet walk of one warp (see closest_packet): the warp walks the
// depth-first order of the sign bits sgn3; a lane takes part in the nodes
// whose box it passes on its own ray, and leaves once it finds an occluder.
// The answer does not depend on the visit order.  A stacked node records, per
// lane, whether that lane passed its box (bit sp of need).
template <int Depth>
__device__ __forceinline__ void any_packet(const DeviceScene& s, AnyWalk& w, bool act, int sgn3, uint32_t* stack,
                                           bool watertight, uint32_t& err, TraceCounters& cnt) {
    static_assert(Depth <= 64, "one bit per stack entry");
    uint32_t ref = s.root_ref;
    int sp = 0;
    unsigned long long need = 0ull;
    for (;;) {
        if (!(ref & kLeafBit)) {
            if (act) ++cnt.inner;
            const float* nb = reinterpret_cast<const float*>(s.inner + ref);
            const float4 q0 = PT_LDG4(nb);
            const float4 q1 = PT_LDG4(nb + 4);
            const float4 q2 = PT_LDG4(nb + 8);
            const uint4  q3 = PT_LDGU4(nb + 12);
            float e0, x0, e1, x1;
            box_span(w.r, q0.x, q0.y, q0.z, q0.w, q1.x, q1.y, e0, x0);
            box_span(w.r, q1.z, q1.w, q2.x, q2.y, q2.z, q2.w, e1, x1);
            const bool h0 = act && e0 <= w.tmax && e0 <= x0;
            const bool h1 = act && e1 <= w.tmax && e1 <= x1;
            const uint32_t axis = q3.z & 3u;
            const int lt = static_cast<int>((q3.z >> 2) & 1u);
            const bool right_first = ((sgn3 >> axis) & 1) == lt;
            const uint32_t nref = right_first ? q3.y : q3.x;
            const uint32_t fref = right_first ? q3.x : q3.y;
            const bool hn = right_first ? h1 : h0;
            const bool hf = right_first ? h0 : h1;
            const bool any_n = __any_sync(0xffffffffu, hn), any_f = __any_sync(0xffffffffu, hf);
            if (any_n) {
                if (any_f) {
                    if (sp >= Depth) { err |= kErrStackOverflow; break; }
                    stack[sp] = fref;
                    if (hf) need |= 1ull << sp;
                    else need &= ~(1ull << sp);
                    ++sp;
                }
                act = hn;
                ref = nref;
                continue;
            }
            if (any_f) { act = hf; ref = fref; continue; }
        } else if (act) {
            uint32_t ti = ref & ~kLeafBit;
            for (;;) {
                float u, v; bool last;
                const float t = tri_test(s, w.r, ti, true, watertight, u, v, last);
                ++cnt.tris;
                if (t > 0.0f && t < w.tmax) { w.hit = true; break; }
                if (last) break;
                ++ti;
            }
        }
        bool found = false;
        while (sp > 0) {
            --sp;
            const bool nd = !w.hit && ((need >> sp) & 1ull);
            if (__any_sync(0xffffffffu, nd)) { act = nd; ref = stack[sp]; found = true; break; }
        }
        if (!found) break;
    }
}

// Any-hit tests of the warp's tiles of 32 rays (see closest_packet_loop):
// a tile whose live rays share their direction signs walks as a packet, any
// other lane by lane.  fetch(i, AnyWalk&) sets r and tmax; done(i, occluded).
template <int Depth = kStackDepth, class Fetch, class Done>
__device__ __forceinline__ void any_packet_loop(const DeviceScene& s, uint32_t warp, uint32_t warps, uint32_t n,
                                                bool watertight, uint32_t& err, TraceCounters& cnt, Fetch&& fetch,
                                                Done&& done) {
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t stack[Depth];
    for (uint32_t base = warp * 32u; base < n; base += warps * 32u) {
        const uint32_t i = base + lane;
        const bool have = i < n;
        AnyWalk w;
        w.sp = 0; w.hit = false;
        bool alive = false;
        if (have) {
            fetch(i, w);
            w.r.xs = exit_scale(watertight);
            alive = any_begin(s, w);
        }
        const int sgn3 = alive ? (w.r.sx | (w.r.sy << 1) | (w.r.sz << 2)) : -1;
        const uint32_t live = __ballot_sync(0xffffffffu, alive);
        if (live) {
            const int lead = __shfl_sync(0xffffffffu, sgn3, __ffs(live) - 1);
            if (__all_sync(0xffffffffu, !alive || sgn3 == lead)) {
                any_packet<Depth>(s, w, alive, lead, stack, watertight, err, cnt);
            } else if (alive) {
                for (;;) {
                    if (w.ref & kLeafBit) {
                        if (!any_leaf(s, w, stack, watertight, cnt)) break;
                    } else if (!any_inner<Depth>(s, w, stack, err, cnt)) {
                        break;
                    }
                }
            }
        }
        if (have) done(i, w.hit);
    }
}
#endif  // __CUDACC__

}  // namespace ptb
