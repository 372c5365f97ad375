// pt_oracle.cpp -- TEST INFRASTRUCTURE: CPU oracle for the path-tracing hot
// path of Neroued/PathTracingTutorial Part_2.  Used only by tests/, the smoke
// check and bench.py's CPU-baseline leg; nothing in the library links it.
//
// Each function restates the reference algorithm cited beside it.  The
// arithmetic is written operation by operation in the reference's order and
// compiled without contraction, so Real = float reproduces the reference's
// IEEE host build exactly (pinned against it by the tests and the golden
// fixtures); Real = double evaluates the same estimator in FP64 and is the
// radiance judge for GPU renders.  `rtl` selects the order of the paired
// sampler draws the reference takes inside one argument list (the C++
// evaluation order there is unspecified: g++ host code draws the second
// argument first, rtl = 1).
#include "pt_oracle.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <queue>
#include <thread>
#include <vector>

#include <cfloat>

#include "tex_filter.h"

namespace {

// ---------------------------------------------------------------------------
// C-layout records (the reference's struct layouts)
// ---------------------------------------------------------------------------
struct Vtx { float p[3]; float _a; float n[3]; float _b; float uv[2]; float _c[2]; float t[4]; };
struct Face { uint32_t v0, v1, v2; int32_t mat; };
struct Mat {
    float base[3], _p0;
    float metallic, roughness, spec_tint, anisotropic;
    float sheen, sheen_tint, clearcoat, cc_roughness;
    float spec_trans, ior, subsurface, spec_factor;
    float spec_r, spec_g, spec_b, aniso_rot;
    float normal_scale, _p1[3];
    float emissive[3], _p2;
    float emissive_strength, alpha_cutoff; int32_t alpha_mode; float base_alpha;
    int32_t double_sided; float sheen_r, sheen_g, sheen_b;
    float occlusion, thickness, att_distance, att_r;
    float att_g, att_b, uvox, uvoy;
    float uvsx, uvsy, uvrot, _p3;
    float _p4; int32_t tex[11]; int32_t _p5[4];
};
static_assert(sizeof(Mat) == 256, "material layout");
struct Node { float lo[3]; uint32_t d0; float hi[3]; uint32_t d1; };
struct Alias { float prob; uint32_t alias; };
struct EmRef { uint32_t tri; float pmf; float cdf; float pad; };
struct Cam { float pos[3], _a; float look[3], _b; float up[3], _c; float fov, aperture, focal; int32_t w, h; int32_t _d[3]; };
struct CamFrame { float pos[3], fwd[3], rgt[3], up[3]; float tan_half_fov, aspect, aperture, focal; };
struct Punctual { float pos[3], _a; float range, _b[3]; float color[3], _c; float intensity, _d[3];
                  float dir[3], _e; float inner, outer; int32_t type; float _f[5]; };
static_assert(sizeof(Punctual) == 112, "punctual layout");
constexpr uint32_t kLeaf = 0x80000000u;

// ---------------------------------------------------------------------------
// Real-typed math mirroring the reference's float wrappers (math_utils.h)
// ---------------------------------------------------------------------------
template <class R> struct K;
template <> struct K<float> {
    static constexpr float Pi = 3.14159265358979323846f, InvPi = 0.31830988618379067154f,
                           Inv2Pi = 0.15915494309189533577f, TwoPi = 6.28318530717958647692f;
};
template <> struct K<double> {
    static constexpr double Pi = 3.14159265358979323846, InvPi = 0.31830988618379067154,
                            Inv2Pi = 0.15915494309189533577, TwoPi = 6.28318530717958647692;
};

template <class R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    explicit V3(R s) : x(s), y(s), z(s) {}
};
template <class R> inline V3<R> operator+(const V3<R>& a, const V3<R>& b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(const V3<R>& a, const V3<R>& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(const V3<R>& a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(const V3<R>& a, R s) { return {a.x * s, a.y * s, a.z * s}; }
template <class R> inline V3<R> operator*(R s, const V3<R>& a) { return a * s; }
template <class R> inline V3<R> operator*(const V3<R>& a, const V3<R>& b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
template <class R> inline V3<R> operator/(const V3<R>& a, R s) { return {a.x / s, a.y / s, a.z / s}; }
template <class R> inline R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline V3<R> cross(const V3<R>& a, const V3<R>& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
template <class R> inline R len(const V3<R>& a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
template <class R> inline V3<R> nrm(const V3<R>& a) { R l = len(a); return l > 0 ? a / l : V3<R>(); }
template <class R> inline bool eq0(const V3<R>& a) { return a.x == 0 && a.y == 0 && a.z == 0; }
template <class R> inline R fmn(R a, R b) { return std::fmin(a, b); }
template <class R> inline R fmx(R a, R b) { return std::fmax(a, b); }
template <class R> inline R clampr(R x, R lo, R hi) { return fmn(fmx(x, lo), hi); }
template <class R> inline V3<R> ld(const float* p) { return {R(p[0]), R(p[1]), R(p[2])}; }

template <class R> struct Frm {
    V3<R> t, b, n;
    explicit Frm(const V3<R>& nn) : n(nn) {
        V3<R> helper(R(1), R(0), R(0));
        if (std::fabs(nn.x) > R(0.999f)) helper = V3<R>(R(0), R(0), R(1));
        t = nrm(cross(nn, helper));
        b = nrm(cross(nn, t));
    }
    V3<R> world(const V3<R>& v) const { return t * v.x + b * v.y + n * v.z; }
    V3<R> local(const V3<R>& v) const { return {dot(v, t), dot(v, b), dot(v, n)}; }
};

// ---------------------------------------------------------------------------
// Samplers (Part_2/src/samplers/pcg.cuh:11-27, sobol.cuh:14-117, sampler.cuh:10-36)
// ---------------------------------------------------------------------------
inline uint32_t brev(uint32_t x) {
    uint32_t r = 0;
    for (int i = 0; i < 32; ++i) { r = (r << 1) | (x & 1u); x >>= 1; }
    return r;
}
inline uint32_t mixer(uint32_t x) {
    x ^= x >> 17; x ^= x * 0xed5ad4bbu; x ^= x >> 11; x ^= x * 0xac4c1b51u;
    x ^= x >> 15; x ^= x * 0x31848babu; x ^= x >> 14;
    return x;
}
inline uint32_t nested_hash(uint32_t x, uint32_t seed) {
    x += seed; x ^= x * 0x6c50b47cu; x ^= x * 0xb82f1e52u; x ^= x * 0xc7afe638u; x ^= x * 0x8d22f6e6u;
    return x;
}
inline uint32_t scramble(uint32_t v, uint32_t seed) { return brev(nested_hash(brev(v), seed)); }
inline uint32_t dim_seed(int px, int py, uint32_t dim) {
    uint32_t h = mixer(static_cast<uint32_t>(px) + 0x9e3779b9u);
    h ^= static_cast<uint32_t>(py) + 0x9e3779b9u + (h << 6) + (h >> 2);
    h = mixer(h);
    h ^= dim + 0x9e3779b9u + (h << 6) + (h >> 2);
    return mixer(h);
}

struct Smp {
    int type = 0;
    int px = 0, py = 0;
    uint32_t index = 0, dim = 0, state = 0;
    void sobol(int x, int y, uint32_t idx) { type = 1; px = x; py = y; index = idx; dim = 0; }
    void pcg(int x, int y, uint32_t frame, uint32_t sample, uint32_t user_seed) {
        type = 0;
        uint32_t s = static_cast<uint32_t>(x) * 1973u + static_cast<uint32_t>(y) * 9277u + frame * 26699u +
                     sample * 12149u + user_seed * 0x9e3779b1u;
        s = s * 747796405u + 2891336453u;
        state = s | 1u;
    }
    float next() {
        if (type == 1) {
            const uint32_t h = dim_seed(px, py, dim);
            const uint32_t idx = scramble(index, h);
            const uint32_t raw = brev(idx);                   // base-2 radical inverse
            const uint32_t v = scramble(raw, mixer(h));
            ++dim;
            return std::fmin(static_cast<float>(v) * (1.0f / 4294967296.0f), 0.99999994f);
        }
        const uint32_t old = state;
        state = old * 747796405u + 2891336453u;
        const uint32_t word = ((old >> ((old >> 28u) + 4u)) ^ old) * 277803737u;
        return static_cast<float>((word >> 22u) ^ word) / 4294967296.0f;
    }
    void pair(int rtl, float& a, float& b) {
        const float d0 = next(), d1 = next();
        if (rtl) { b = d0; a = d1; } else { a = d0; b = d1; }
    }
};

// ---------------------------------------------------------------------------
// Traversal on the reference node layout (bvh_traversal.cuh:16-133,
// triangle.h:13-76), counting node pops and triangle tests.
// ---------------------------------------------------------------------------
struct Cnt { uint64_t pops = 0, tris = 0; };

struct Hit {
    bool hit = false;
    float t = FLT_MAX;
    int prim = -1;
    float u = 0, v = 0;
};

inline bool slab(const float o[3], const float inv[3], const Node& n, float tmax) {
    float tn = 0.0f, tf = tmax;
    for (int i = 0; i < 3; ++i) {
        const float t1 = (n.lo[i] - o[i]) * inv[i];
        const float t2 = (n.hi[i] - o[i]) * inv[i];
        tn = std::fmin(std::fmax(t1, tn), std::fmax(t2, tn));
        tf = std::fmax(std::fmin(t1, tf), std::fmin(t2, tf));
    }
    return tn <= tf;
}

// Moller-Trumbore; returns t or -1.  closest: accept t >= 1e-4; shadow: t > 1e-4.
inline float mt(const float o[3], const float d[3], const Vtx& a, const Vtx& b, const Vtx& c, bool shadow,
                float& uu, float& vv) {
    const V3<float> e1 = ld<float>(b.p) - ld<float>(a.p), e2 = ld<float>(c.p) - ld<float>(a.p);
    const V3<float> dir(d[0], d[1], d[2]), org(o[0], o[1], o[2]);
    const V3<float> pv = cross(dir, e2);
    const float det = dot(e1, pv);
    if (std::fabs(det) < FLT_EPSILON) return -1.0f;
    const float inv = 1.0f / det;
    const V3<float> tv = org - ld<float>(a.p);
    const float u = dot(tv, pv) * inv;
    if (u < 0.0f || u > 1.0f) return -1.0f;
    const V3<float> qv = cross(tv, e1);
    const float v = dot(dir, qv) * inv;
    if (v < 0.0f || u + v > 1.0f) return -1.0f;
    const float t = dot(e2, qv) * inv;
    if (shadow) return t > 1e-4f ? t : -1.0f;
    if (t < 1e-4f) return -1.0f;
    uu = u; vv = v;
    return t;
}

// Watertight mode (added; the reference has none): the slab test of the
// reference with the exit distance widened by kWtExit (Ize 2013: the slab
// distances are within a factor 1 +- gamma(3) of exact, and 1 + 4 ulp covers
// (1 + gamma(3)) / (1 - gamma(3)) and the product's own rounding), and Woop,
// Benthin and Wald's triangle test (JCGT 2013) on the shared vertex
// positions.  The tmax of the reference's recurrence is compared apart from
// the widened exit.
constexpr float kWtExit = 1.0f + 4.0f * 1.1920929e-7f;

inline bool slab_wt(const float o[3], const float inv[3], const Node& n, float tmax) {
    float tn = 0.0f, tf = INFINITY;
    for (int i = 0; i < 3; ++i) {
        const float t1 = (n.lo[i] - o[i]) * inv[i];
        const float t2 = (n.hi[i] - o[i]) * inv[i];
        tn = std::fmin(std::fmax(t1, tn), std::fmax(t2, tn));
        tf = std::fmax(std::fmin(t1, tf), std::fmin(t2, tf));
    }
    return tn <= tf * kWtExit && tn <= tmax;
}

inline float woop(const float o[3], const float d[3], const Vtx& p0, const Vtx& p1, const Vtx& p2, bool shadow,
                  float& uu, float& vv) {
    const float adx = std::fabs(d[0]), ady = std::fabs(d[1]), adz = std::fabs(d[2]);
    int kz = (adx > ady) ? (adx > adz ? 0 : 2) : (ady > adz ? 1 : 2);
    int kx = kz + 1 == 3 ? 0 : kz + 1;
    int ky = kx + 1 == 3 ? 0 : kx + 1;
    if (d[kz] < 0.0f) std::swap(kx, ky);
    const float sx = d[kx] / d[kz], sy = d[ky] / d[kz], sz = 1.0f / d[kz];
    float a[3], b[3], c[3];
    for (int k = 0; k < 3; ++k) { a[k] = p0.p[k] - o[k]; b[k] = p1.p[k] - o[k]; c[k] = p2.p[k] - o[k]; }
    const float ax = a[kx] - sx * a[kz], ay = a[ky] - sy * a[kz];
    const float bx = b[kx] - sx * b[kz], by = b[ky] - sy * b[kz];
    const float cx = c[kx] - sx * c[kz], cy = c[ky] - sy * c[kz];
    float U = cx * by - cy * bx, V = ax * cy - ay * cx, W = bx * ay - by * ax;
    if (U == 0.0f || V == 0.0f || W == 0.0f) {
        U = static_cast<float>(double(cx) * double(by) - double(cy) * double(bx));
        V = static_cast<float>(double(ax) * double(cy) - double(ay) * double(cx));
        W = static_cast<float>(double(bx) * double(ay) - double(by) * double(ax));
    }
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return -1.0f;
    const float det = U + V + W;
    if (det == 0.0f) return -1.0f;
    const float az = sz * a[kz], bz = sz * b[kz], cz = sz * c[kz];
    const float T = U * az + V * bz + W * cz;
    const float inv = 1.0f / det;
    const float t = T * inv;
    if (shadow) { if (!(t > 1e-4f)) return -1.0f; }
    else if (t < 1e-4f) return -1.0f;
    uu = V * inv; vv = W * inv;
    return t;
}

struct Geo {
    const Node* nodes;
    const Vtx* v;
    const Face* f;
    uint32_t nn;
    bool wt = false;
};

Hit closest(const Geo& g, const float o[3], const float d[3], Cnt& c) {
    Hit h;
    if (g.nn == 0) return h;
    const float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    const int sg[3] = {inv[0] < 0.0f, inv[1] < 0.0f, inv[2] < 0.0f};
    uint32_t st[128];
    int top = 0;
    st[top++] = 0;
    while (top > 0) {
        const Node& n = g.nodes[st[--top]];
        ++c.pops;
        if (!(g.wt ? slab_wt(o, inv, n, h.t) : slab(o, inv, n, h.t))) continue;
        if (n.d0 & kLeaf) {
            const uint32_t first = n.d0 & ~kLeaf;
            for (uint32_t i = 0; i < n.d1; ++i) {
                const Face& f = g.f[first + i];
                float u = 0, v = 0;
                ++c.tris;
                const float t = g.wt ? woop(o, d, g.v[f.v0], g.v[f.v1], g.v[f.v2], false, u, v)
                                     : mt(o, d, g.v[f.v0], g.v[f.v1], g.v[f.v2], false, u, v);
                if (t >= 0.0f && t < h.t) { h.hit = true; h.t = t; h.prim = static_cast<int>(first + i); h.u = u; h.v = v; }
            }
        } else {
            const Node& L = g.nodes[n.d0];
            const Node& Rn = g.nodes[n.d1];
            const float dx = n.hi[0] - n.lo[0], dy = n.hi[1] - n.lo[1], dz = n.hi[2] - n.lo[2];
            const int axis = (dx > dy && dx > dz) ? 0 : (dy > dz ? 1 : 2);
            const float cl = 0.5f * (L.lo[axis] + L.hi[axis]);
            const float cr = 0.5f * (Rn.lo[axis] + Rn.hi[axis]);
            if ((sg[axis] != 0) == (cl < cr)) { st[top++] = n.d0; st[top++] = n.d1; }
            else { st[top++] = n.d1; st[top++] = n.d0; }
        }
    }
    return h;
}

bool occluded(const Geo& g, const float o[3], const float d[3], float tmax, Cnt& c) {
    if (g.nn == 0) return false;
    const float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
    uint32_t st[128];
    int top = 0;
    st[top++] = 0;
    while (top > 0) {
        const Node& n = g.nodes[st[--top]];
        ++c.pops;
        if (!(g.wt ? slab_wt(o, inv, n, tmax) : slab(o, inv, n, tmax))) continue;
        if (n.d0 & kLeaf) {
            const uint32_t first = n.d0 & ~kLeaf;
            for (uint32_t i = 0; i < n.d1; ++i) {
                const Face& f = g.f[first + i];
                float u, v;
                ++c.tris;
                const float t = g.wt ? woop(o, d, g.v[f.v0], g.v[f.v1], g.v[f.v2], true, u, v)
                                     : mt(o, d, g.v[f.v0], g.v[f.v1], g.v[f.v2], true, u, v);
                if (t > 0.0f && t < tmax) return true;
            }
        } else {
            st[top++] = n.d0;
            st[top++] = n.d1;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------
// Disney BSDF (disney_bsdf.cuh:53-410, microfacet.cuh:10-113)
// ---------------------------------------------------------------------------
template <class R> struct ME {
    V3<R> base;
    R metallic, roughness, spec_trans, ior, clearcoat, cc_roughness, sheen, sheen_tint, subsurface;
    R anisotropic, spec_tint, spec_factor;
    V3<R> spec_color, sheen_color;
    R thickness, att_distance;
    V3<R> att_color;
};
template <class R> ME<R> fetch(const Mat& m) {
    ME<R> e;
    e.base = ld<R>(m.base);
    e.metallic = R(m.metallic); e.roughness = R(m.roughness); e.spec_trans = R(m.spec_trans); e.ior = R(m.ior);
    e.clearcoat = R(m.clearcoat); e.cc_roughness = R(m.cc_roughness); e.sheen = R(m.sheen);
    e.sheen_tint = R(m.sheen_tint); e.subsurface = R(m.subsurface); e.anisotropic = R(m.anisotropic);
    e.spec_tint = R(m.spec_tint); e.spec_factor = R(m.spec_factor);
    e.spec_color = V3<R>(R(m.spec_r), R(m.spec_g), R(m.spec_b));
    e.sheen_color = V3<R>(R(m.sheen_r), R(m.sheen_g), R(m.sheen_b));
    e.thickness = R(m.thickness); e.att_distance = R(m.att_distance);
    e.att_color = V3<R>(R(m.att_r), R(m.att_g), R(m.att_b));
    e.roughness = clampr(e.roughness, R(0.001f), R(1));
    e.metallic = clampr(e.metallic, R(0), R(1));
    e.cc_roughness = clampr(e.cc_roughness, R(0.001f), R(1));
    return e;
}
template <class R> R lum(const V3<R>& c) { return R(0.2126f) * c.x + R(0.7152f) * c.y + R(0.0722f) * c.z; }
template <class R> void alpha_xy(R rough, R aniso, R& ax, R& ay) {
    const R aspect = std::sqrt(R(1) - R(0.9f) * aniso);
    const R a = rough * rough;
    ax = fmx(a / aspect, R(0.001f));
    ay = fmx(a * aspect, R(0.001f));
}
template <class R> V3<R> diffuse(const ME<R>& m, R nol, R nov, R hol) {
    const R fd90 = R(0.5f) + R(2) * hol * hol * m.roughness;
    const R fl = R(1) + (fd90 - R(1)) * std::pow(R(1) - nol, R(5));
    const R fv = R(1) + (fd90 - R(1)) * std::pow(R(1) - nov, R(5));
    V3<R> d = m.base * (K<R>::InvPi * fl * fv);
    if (m.subsurface > R(0)) {
        const R f90 = hol * hol * m.roughness;
        const R sl = R(1) + (f90 - R(1)) * std::pow(R(1) - nol, R(5));
        const R sv = R(1) + (f90 - R(1)) * std::pow(R(1) - nov, R(5));
        const R ss = R(1.25f) * (sl * sv * (R(1) / (nol + nov + R(1e-5f)) - R(0.5f)) + R(0.5f));
        const V3<R> sd = m.base * (K<R>::InvPi * ss);
        d = (R(1) - m.subsurface) * d + m.subsurface * sd;
    }
    return d;
}
template <class R> V3<R> tint(const V3<R>& base) {
    const R l = lum(base);
    return l > R(0) ? base / l : V3<R>(R(1));
}
template <class R> V3<R> sheen(const ME<R>& m, R hol) {
    if (m.sheen <= R(0)) return V3<R>(R(0));
    const V3<R> bs = (R(1) - m.sheen_tint) * V3<R>(R(1)) + m.sheen_tint * tint(m.base);
    const V3<R> fs = bs * m.sheen_color;
    const R fh = std::pow(R(1) - hol, R(5));
    return m.sheen * fs * fh;
}
template <class R> V3<R> f0(const ME<R>& m) {
    const R eta = m.ior;
    const R r0 = ((eta - R(1)) * (eta - R(1))) / ((eta + R(1)) * (eta + R(1)));
    V3<R> s = r0 * ((R(1) - m.spec_tint) * V3<R>(R(1)) + m.spec_tint * tint(m.base));
    s = s * m.spec_factor * m.spec_color;
    return (R(1) - m.metallic) * s + m.metallic * m.base;
}
template <class R> struct LW { R d, s, c, t, sh; };
template <class R> LW<R> weights(const ME<R>& m) {
    const R dw = (R(1) - m.metallic) * (R(1) - m.spec_trans);
    const R sw = R(1);
    const R tw = (R(1) - m.metallic) * m.spec_trans;
    const R cw = R(0.25f) * m.clearcoat;
    const R shw = (R(1) - m.metallic) * m.sheen * R(0.1f);
    const R total = dw + sw + cw + tw + shw;
    LW<R> w{R(0), R(0), R(0), R(0), R(0)};
    if (total <= R(0)) return w;
    const R inv = R(1) / total;
    w.d = dw * inv; w.s = sw * inv; w.c = cw * inv; w.t = tw * inv; w.sh = shw * inv;
    return w;
}
template <class R> R d_ggx(R noh, R a) {
    const R a2 = a * a;
    const R d = noh * noh * (a2 - R(1)) + R(1);
    return a2 / (K<R>::Pi * d * d + R(1e-7f));
}
template <class R> R d_aniso(R noh, R hx_, R hy_, R ax, R ay) {
    const R hx = hx_ / ax, hy = hy_ / ay;
    const R d = hx * hx + hy * hy + noh * noh;
    return R(1) / (K<R>::Pi * ax * ay * d * d + R(1e-7f));
}
template <class R> R g1(R nov, R a) {
    const R a2 = a * a;
    return R(2) * nov / (nov + std::sqrt(a2 + (R(1) - a2) * nov * nov) + R(1e-7f));
}
template <class R> R g2(R nol, R nov, R a) {
    const R a2 = a * a;
    const R gv = nol * std::sqrt(a2 + (R(1) - a2) * nov * nov);
    const R gl = nov * std::sqrt(a2 + (R(1) - a2) * nol * nol);
    return R(2) * nol * nov / (gv + gl + R(1e-7f));
}
template <class R> R schlick1(R c, R F0) {
    const R t = clampr(R(1) - c, R(0), R(1));
    const R t2 = t * t;
    return F0 + (R(1) - F0) * t2 * t2 * t;
}
template <class R> V3<R> schlick3(R c, const V3<R>& F0) {
    const R t = clampr(R(1) - c, R(0), R(1));
    const R t2 = t * t;
    const R t5 = t2 * t2 * t;
    return F0 + (V3<R>(R(1)) - F0) * t5;
}
template <class R> R fdiel(R ci_, R eta) {
    const R s2t = eta * eta * (R(1) - ci_ * ci_);
    if (s2t >= R(1)) return R(1);
    const R ct = std::sqrt(fmx(R(0), R(1) - s2t));
    const R ci = std::fabs(ci_);
    const R rs = (ci - eta * ct) / (ci + eta * ct + R(1e-7f));
    const R rp = (eta * ci - ct) / (eta * ci + ct + R(1e-7f));
    return R(0.5f) * (rs * rs + rp * rp);
}
template <class R> V3<R> vndf(const V3<R>& wo, R ax, R ay, R u1, R u2) {
    V3<R> wh = nrm(V3<R>(ax * wo.x, ay * wo.y, wo.z));
    if (wh.z < R(0)) wh = -wh;
    const V3<R> T1 = (wh.z < R(0.9999f)) ? nrm(cross(V3<R>(R(0), R(0), R(1)), wh)) : V3<R>(R(1), R(0), R(0));
    const V3<R> T2 = cross(wh, T1);
    const R r = std::sqrt(u1);
    const R phi = K<R>::TwoPi * u2;
    const R t1 = r * std::cos(phi);
    R t2 = r * std::sin(phi);
    const R s = R(0.5f) * (R(1) + wh.z);
    t2 = (R(1) - s) * std::sqrt(fmx(R(0), R(1) - t1 * t1)) + s * t2;
    const V3<R> nh = t1 * T1 + t2 * T2 + std::sqrt(fmx(R(0), R(1) - t1 * t1 - t2 * t2)) * wh;
    return nrm(V3<R>(ax * nh.x, ay * nh.y, fmx(R(0), nh.z)));
}
template <class R> R pvndf(const V3<R>& wo, const V3<R>& h, R ax, R ay) {
    const R nov = fmx(wo.z, R(1e-5f));
    const R noh = fmx(h.z, R(0));
    const R voh = fmx(dot(wo, h), R(0));
    const R D = d_aniso(noh, h.x, h.y, ax, ay);
    const R G = g1(nov, std::sqrt(ax * ay));
    return D * G * voh / (nov + R(1e-7f));
}
template <class R> bool refr(const V3<R>& wi, const V3<R>& n, R eta, V3<R>& wt) {
    const R ci = dot(wi, n);
    const R s2i = fmx(R(0), R(1) - ci * ci);
    const R s2t = eta * eta * s2i;
    if (s2t >= R(1)) return false;
    const R ct = std::sqrt(R(1) - s2t);
    wt = eta * (-wi) + (eta * ci - ct) * n;
    return true;
}
template <class R> V3<R> refl(const V3<R>& i, const V3<R>& n) { return i - R(2) * dot(i, n) * n; }

template <class R> struct BE { V3<R> f; R pdf = R(0); };
template <class R> BE<R> eval(const ME<R>& m, const V3<R>& wo, const V3<R>& wi, const V3<R>& N, bool entering = true) {
    BE<R> r;
    const R nol = dot(N, wi), nov = dot(N, wo);
    const bool reflect = nol > R(0);
    if (!reflect && m.spec_trans <= R(0)) return r;
    if (!reflect) {
        const R anol = std::fabs(nol), anov = std::fabs(nov);
        if (anol < R(1e-5f) || anov < R(1e-5f)) return r;
        const R eta = entering ? (R(1) / m.ior) : m.ior;
        const V3<R> ht = -nrm(wo * eta + wi);
        const R hov = std::fabs(dot(ht, wo));
        R ax, ay; alpha_xy(m.roughness, m.anisotropic, ax, ay);
        const Frm<R> fr(N);
        const V3<R> hl = fr.local(ht);
        const R D = d_aniso(std::fabs(hl.z), hl.x, hl.y, ax, ay);
        const R G = g2(anol, anov, std::sqrt(ax * ay));
        const R F = fdiel(hov, eta);
        const R sd = dot(wo, ht) * eta + dot(wi, ht);
        const R factor = std::fabs(dot(wo, ht)) * std::fabs(dot(wi, ht)) / (anov * anol * sd * sd + R(1e-7f));
        const R tw = (R(1) - m.metallic) * m.spec_trans;
        const V3<R> ft = m.base * tw * D * G * (R(1) - F) * factor;
        const LW<R> w = weights(m);
        const R jac = eta * eta * std::fabs(dot(wi, ht)) / (sd * sd + R(1e-7f));
        const R tp = D * g1(anov, std::sqrt(ax * ay)) * hov / (anov + R(1e-7f)) * jac;
        r.f = ft;
        r.pdf = w.t * tp;
        return r;
    }
    if (nol < R(1e-5f) || nov < R(1e-5f)) return r;
    const V3<R> H = nrm(wo + wi);
    const R noh = fmx(dot(N, H), R(0));
    const R hol = fmx(dot(H, wi), R(0));
    const Frm<R> fr(N);
    const V3<R> hl = fr.local(H);
    R ax, ay; alpha_xy(m.roughness, m.anisotropic, ax, ay);
    const LW<R> w = weights(m);
    V3<R> ft(R(0));
    R pt = R(0);
    const R dw = (R(1) - m.metallic) * (R(1) - m.spec_trans);
    if (dw > R(0)) {
        const V3<R> fd = diffuse(m, nol, nov, hol);
        ft = ft + dw * fd;
        pt = pt + w.d * (nol * K<R>::InvPi);
    }
    if (m.sheen > R(0) && m.metallic < R(1)) {
        const V3<R> fs = sheen(m, hol);
        ft = ft + (R(1) - m.metallic) * fs;
        pt = pt + w.sh * (nol * K<R>::InvPi);
    }
    {
        const R D = d_aniso(noh, hl.x, hl.y, ax, ay);
        const R G = g2(nol, nov, std::sqrt(ax * ay));
        const V3<R> F = schlick3(hol, f0(m));
        const V3<R> spec = D * G * F / (R(4) * nol * nov + R(1e-7f));
        ft = ft + spec;
        const V3<R> wol = fr.local(wo);
        const R sp = pvndf(wol, hl, ax, ay) / (R(4) * hol + R(1e-7f));
        pt = pt + w.s * sp;
    }
    if (m.clearcoat > R(0)) {
        const R ca = fmx(m.cc_roughness * m.cc_roughness, R(0.001f));
        const R Dc = d_ggx(noh, ca);
        const R Gc = g2(nol, nov, ca);
        const R Fc = schlick1(hol, R(0.04f));
        const R cs = R(0.25f) * m.clearcoat * Dc * Gc * Fc / (R(4) * nol * nov + R(1e-7f));
        ft = ft + V3<R>(cs);
        const R cp = Dc * noh / (R(4) * hol + R(1e-7f));
        pt = pt + w.c * cp;
    }
    r.f = ft * nol;
    r.pdf = pt;
    return r;
}

template <class R> struct BS { V3<R> wi, weight; R pdf = R(0); bool delta = false, valid = false; };
template <class R> BS<R> sample(const ME<R>& m, const V3<R>& wo, const V3<R>& N, Smp& rng, int rtl, bool entering) {
    BS<R> r;
    const R nov = dot(N, wo);
    if (nov < R(1e-5f)) return r;
    const LW<R> w = weights(m);
    const R choice = R(rng.next());
    const Frm<R> fr(N);
    const V3<R> wol = fr.local(wo);
    R ax, ay; alpha_xy(m.roughness, m.anisotropic, ax, ay);
    V3<R> wi;
    bool delta = false;
    float a1, a2;
    if (choice < w.d + w.sh) {
        rng.pair(rtl, a1, a2);
        const R u1 = R(a1), u2 = R(a2);
        const R rr = std::sqrt(u1);
        const R phi = K<R>::TwoPi * u2;
        wi = fr.world(V3<R>(rr * std::cos(phi), rr * std::sin(phi), std::sqrt(fmx(R(0), R(1) - u1))));
    } else if (choice < w.d + w.sh + w.s) {
        rng.pair(rtl, a1, a2);
        const V3<R> H = fr.world(vndf(wol, ax, ay, R(a1), R(a2)));
        wi = refl(-wo, H);
        if (dot(wi, N) <= R(0)) return r;
        delta = m.roughness < R(0.01f);
    } else if (choice < w.d + w.sh + w.s + w.c) {
        const R ca = fmx(m.cc_roughness * m.cc_roughness, R(0.001f));
        rng.pair(rtl, a1, a2);
        const V3<R> H = fr.world(vndf(wol, ca, ca, R(a1), R(a2)));
        wi = refl(-wo, H);
        if (dot(wi, N) <= R(0)) return r;
    } else {
        rng.pair(rtl, a1, a2);
        const V3<R> H = fr.world(vndf(wol, ax, ay, R(a1), R(a2)));
        const R eta = entering ? (R(1) / m.ior) : m.ior;
        V3<R> wt;
        if (!refr(wo, H, eta, wt)) {
            wi = refl(-wo, H);
            if (dot(wi, N) <= R(0)) return r;
        } else {
            wi = nrm(wt);
            delta = m.roughness < R(0.01f);
        }
    }
    const BE<R> ev = eval(m, wo, wi, N, entering);
    if (ev.pdf <= R(0)) return r;
    r.wi = wi; r.pdf = ev.pdf; r.delta = delta; r.valid = true;
    if (delta) {
        if (dot(N, wi) < R(0)) {
            r.weight = m.base;
        } else {
            const V3<R> H = nrm(wo + wi);
            r.weight = schlick3(fmx(dot(H, wi), R(0)), f0(m));
        }
    } else {
        r.weight = ev.f / (ev.pdf + R(1e-7f));
    }
    return r;
}
template <class R> R power(R a, R b) {
    const R a2 = a * a, b2 = b * b, s = a2 + b2;
    return s > R(0) ? a2 / s : R(0);
}

// ---------------------------------------------------------------------------
// Scene context and lights (direct_lighting.cuh, light_pdf.cuh, envmap.h)
// ---------------------------------------------------------------------------
// A material texture: float RGBA texels and the address modes of its glTF sampler.
struct OTex { const float* rgba; int32_t width, height, wrap_s, wrap_t; };

struct Ctx {
    Geo geo;
    const Mat* mats;
    uint32_t nmat;
    const OTex* texs;     // material textures (null / 0 when the scene has none)
    uint32_t ntex;
    const EmRef* em;
    uint32_t nem;
    const float* tri_pmf;
    const Alias* tri_alias;
    HostTexture tex;
    bool has_tex;
    const float* env_pmf;
    const Alias* env_alias;
    uint32_t n_env;
    int env_w, env_h;
    const Punctual* pl;
    uint32_t npl;
    CamFrame cam;
    int width, height;
    int spf, max_depth, rtl;
};

template <class R> void sph_uv(const V3<R>& d, R& u, R& v) {
    u = std::atan2(d.z, d.x);
    v = std::asin(d.y);
    u = u * K<R>::Inv2Pi;
    v = v * K<R>::InvPi;
    u = u + R(0.5f);
    v = v + R(0.5f);
    v = R(1) - v;
}
template <class R> V3<R> dir_uv(R u, R v) {
    const R phi = (u - R(0.5f)) * K<R>::TwoPi;
    const R th = v * K<R>::Pi;
    const R st = std::sin(th);
    return nrm(V3<R>(std::cos(phi) * st, std::cos(th), std::sin(phi) * st));
}
template <class R> V3<R> env_rad(const Ctx& c, const V3<R>& d) {
    if (!c.has_tex) return V3<R>(R(0));
    R u, v;
    sph_uv(d, u, v);
    const float4 t = ptref_tex_fetch(&c.tex, static_cast<float>(u), static_cast<float>(v));
    return V3<R>(R(t.x), R(t.y), R(t.z)) * K<R>::TwoPi;
}
template <class R> R env_pdf(const Ctx& c, const V3<R>& d) {
    if (!c.has_tex || !c.env_pmf || c.n_env == 0 || c.env_w <= 0 || c.env_h <= 0) return R(0);
    R u, v;
    sph_uv(d, u, v);
    const int x = static_cast<int>(clampr(u * R(c.env_w), R(0), R(c.env_w - 1)));
    const int y = static_cast<int>(clampr(v * R(c.env_h), R(0), R(c.env_h - 1)));
    const R st = std::sqrt(fmx(R(0), R(1) - d.y * d.y));
    if (st <= R(1e-5f)) return R(0);
    const int idx = y * c.env_w + x;
    return R(c.env_pmf[idx]) * R(static_cast<float>(c.env_w * c.env_h)) / (K<R>::TwoPi * K<R>::Pi * st);
}
template <class R> V3<R> vpos(const Ctx& c, uint32_t i) { return ld<R>(c.geo.v[i].p); }
template <class R> V3<R> vnr(const Ctx& c, uint32_t i) { return ld<R>(c.geo.v[i].n); }

// ---- material textures (shading_utils.cuh:17-68, disney_bsdf.cuh:79-116) ----
enum { kTexBase = 0, kTexMR = 1, kTexNormal = 2, kTexCC = 5, kTexCCR = 6, kTexTrans = 8, kTexSheenC = 9,
       kTexSheenR = 10 };
inline bool tex_live(const Ctx& c, int32_t id) {
    return id >= 0 && static_cast<uint32_t>(id) < c.ntex && c.texs[id].rgba != nullptr && c.texs[id].width > 0 &&
           c.texs[id].height > 0;
}
// the device's tex2D<float4> (bilinear, normalized coordinates, the sampler's
// address modes), through the measured B200 filter model
inline float4 tex_at(const Ctx& c, int32_t id, float u, float v) {
    const OTex& t = c.texs[id];
    const HostTexture h{t.rgba, t.width, t.height};
    return ptref_tex_fetch_mode(&h, u, v, ptref_gl_mode(t.wrap_s), ptref_gl_mode(t.wrap_t));
}
template <class R> V3<R> tex_linear(float4 t) {
    return {std::pow(R(t.x), R(2.2f)), std::pow(R(t.y), R(2.2f)), std::pow(R(t.z), R(2.2f))};
}

// fetchMaterial with textures: factors times texel channels, then the clamps.
template <class R> ME<R> fetch_tex(const Ctx& c, const Mat& m, float u, float v) {
    ME<R> e = fetch<R>(m);
    R rough = R(m.roughness), metal = R(m.metallic), ccr = R(m.cc_roughness);
    if (tex_live(c, m.tex[kTexBase])) e.base = e.base * tex_linear<R>(tex_at(c, m.tex[kTexBase], u, v));
    if (tex_live(c, m.tex[kTexMR])) {
        const float4 t = tex_at(c, m.tex[kTexMR], u, v);
        rough = rough * R(t.y);
        metal = metal * R(t.z);
    }
    if (tex_live(c, m.tex[kTexCC])) e.clearcoat = e.clearcoat * R(tex_at(c, m.tex[kTexCC], u, v).x);
    if (tex_live(c, m.tex[kTexCCR])) ccr = ccr * R(tex_at(c, m.tex[kTexCCR], u, v).y);
    if (tex_live(c, m.tex[kTexTrans])) e.spec_trans = e.spec_trans * R(tex_at(c, m.tex[kTexTrans], u, v).x);
    if (tex_live(c, m.tex[kTexSheenC])) e.sheen_color = e.sheen_color * tex_linear<R>(tex_at(c, m.tex[kTexSheenC], u, v));
    if (tex_live(c, m.tex[kTexSheenR])) e.sheen = e.sheen * R(tex_at(c, m.tex[kTexSheenR], u, v).w);
    e.roughness = clampr(rough, R(0.001f), R(1));
    e.metallic = clampr(metal, R(0), R(1));
    e.cc_roughness = clampr(ccr, R(0.001f), R(1));
    return e;
}
template <class R> R face_area(const Ctx& c, const Face& f) {
    return R(0.5f) * len(cross(vpos<R>(c, f.v1) - vpos<R>(c, f.v0), vpos<R>(c, f.v2) - vpos<R>(c, f.v0)));
}
template <class R> V3<R> face_normal(const Ctx& c, const Face& f) {
    return nrm(cross(vpos<R>(c, f.v1) - vpos<R>(c, f.v0), vpos<R>(c, f.v2) - vpos<R>(c, f.v0)));
}
bool emits(const Mat& m) {
    return m.emissive_strength > 0.0f && (m.emissive[0] > 0.0f || m.emissive[1] > 0.0f || m.emissive[2] > 0.0f);
}
template <class R> V3<R> emission(const Mat& m) { return ld<R>(m.emissive) * R(m.emissive_strength); }

uint32_t alias_pick(const Alias* t, uint32_t n, float u1, float u2) {
    uint32_t i = static_cast<uint32_t>(u1 * n);
    if (i >= n) i = n - 1;
    return (u2 < t[i].prob) ? i : t[i].alias;
}

struct Stats { uint64_t closest = 0, shadow = 0; Cnt cc, sc; };

template <class R> bool occl(const Ctx& c, const V3<R>& p, const V3<R>& n, const V3<R>& wi, R maxd, Stats& st) {
    const R sg = dot(wi, n) >= R(0) ? R(1) : R(-1);
    const V3<R> org = p + n * (R(1e-4f) * sg);
    const V3<R> dir = nrm(wi);
    const R tmax = (maxd < R(FLT_MAX)) ? (maxd - R(1e-3f)) : R(FLT_MAX);
    const float o[3] = {float(org.x), float(org.y), float(org.z)};
    const float d[3] = {float(dir.x), float(dir.y), float(dir.z)};
    ++st.shadow;
    return occluded(c.geo, o, d, static_cast<float>(tmax), st.sc);
}

template <class R> struct LS { V3<R> wi, rad; R pdf = R(0); bool valid = false; };

template <class R> struct Shade {
    static LS<R> area(const Ctx& c, const V3<R>& p, const V3<R>& N, Smp& rng, Stats& st) {
        LS<R> s;
        float a1, a2;
        rng.pair(c.rtl, a1, a2);
        const EmRef& ref = c.em[alias_pick(c.tri_alias, c.nem, a1, a2)];
        const Face& f = c.geo.f[ref.tri];
        const float t1 = rng.next();
        const float t2 = rng.next();
        const R su0 = std::sqrt(R(t1));
        const R b0 = R(1) - su0, b1 = R(t2) * su0, b2 = R(1) - b0 - b1;
        const V3<R> lp = vpos<R>(c, f.v0) * b0 + vpos<R>(c, f.v1) * b1 + vpos<R>(c, f.v2) * b2;
        V3<R> ln = nrm(vnr<R>(c, f.v0) * b0 + vnr<R>(c, f.v1) * b1 + vnr<R>(c, f.v2) * b2);
        if (len(ln) == R(0)) ln = face_normal<R>(c, f);
        const V3<R> to = lp - p;
        const R d2 = dot(to, to);
        if (d2 <= R(1e-8f)) return s;
        const R dist = std::sqrt(d2);
        const V3<R> wi = to / dist;
        const R cs = fmx(R(0), dot(N, wi));
        if (cs <= R(0)) return s;
        const R ar = face_area<R>(c, f);
        if (ar <= R(0)) return s;
        const R cl = std::fabs(dot(ln, -wi));
        if (cl <= R(1e-5f)) return s;
        const R pdf = (R(ref.pmf) / ar) * d2 / cl;
        if (pdf <= R(0)) return s;
        if (occl(c, p, N, wi, dist, st)) return s;
        s.wi = wi; s.rad = emission<R>(c.mats[f.mat]); s.pdf = pdf; s.valid = true;
        return s;
    }
    static LS<R> env(const Ctx& c, const V3<R>& p, const V3<R>& N, Smp& rng, Stats& st) {
        LS<R> s;
        float a1, a2;
        rng.pair(c.rtl, a1, a2);
        const uint32_t texel = alias_pick(c.env_alias, c.n_env, a1, a2);
        const int x = static_cast<int>(texel % static_cast<uint32_t>(c.env_w));
        const int y = static_cast<int>(texel / static_cast<uint32_t>(c.env_w));
        float j1, j2;
        rng.pair(c.rtl, j1, j2);
        const R u = (R(static_cast<float>(x)) + R(j1)) / R(static_cast<float>(c.env_w));
        const R v = (R(static_cast<float>(y)) + R(j2)) / R(static_cast<float>(c.env_h));
        const V3<R> wi = dir_uv(u, v);
        const R cs = fmx(R(0), dot(N, wi));
        if (cs <= R(0)) return s;
        const R pdf = env_pdf(c, wi);
        if (pdf <= R(0)) return s;
        if (occl(c, p, N, wi, R(FLT_MAX), st)) return s;
        s.wi = wi; s.rad = env_rad(c, wi); s.pdf = pdf; s.valid = true;
        return s;
    }
    static V3<R> direct(const LS<R>& s, const ME<R>& m, const V3<R>& wo, const V3<R>& N) {
        if (!s.valid) return V3<R>(R(0));
        const BE<R> b = eval(m, wo, s.wi, N);
        if (b.pdf <= R(0)) return V3<R>(R(0));
        const R sp = s.pdf * R(1);
        const R mis = power(sp, b.pdf);
        return s.rad * b.f * (mis / (sp + R(1e-7f)));
    }
    static V3<R> punctual(const Ctx& c, const V3<R>& p, const ME<R>& m, const V3<R>& wo, const V3<R>& N, Stats& st) {
        if (c.npl == 0 || c.pl == nullptr) return V3<R>(R(0));
        V3<R> Ld(R(0));
        for (uint32_t i = 0; i < c.npl; ++i) {
            const Punctual& L = c.pl[i];
            V3<R> wi;
            R dist = R(FLT_MAX);
            V3<R> inten(R(0));
            if (L.type == 0 || L.type == 2) {
                const V3<R> to = ld<R>(L.pos) - p;
                const R d2 = dot(to, to);
                if (d2 < R(1e-8f)) continue;
                dist = std::sqrt(d2);
                wi = to / dist;
                R att = dist >= R(L.range) ? R(0) : R(1) / (dist * dist + R(1e-7f));
                if (L.type == 2) {
                    const R ca = dot(nrm(-to), ld<R>(L.dir));
                    R sa;
                    if (ca < R(L.outer)) sa = R(0);
                    else if (ca > R(L.inner)) sa = R(1);
                    else { const R t = (ca - R(L.outer)) / (R(L.inner) - R(L.outer) + R(1e-7f)); sa = t * t; }
                    att = att * sa;
                }
                inten = ld<R>(L.color) * (R(L.intensity) * att);
            } else {
                wi = -ld<R>(L.dir);
                dist = R(FLT_MAX);
                inten = ld<R>(L.color) * R(L.intensity);
            }
            const R nol = dot(N, wi);
            if (nol <= R(0)) continue;
            if (occl(c, p, N, wi, dist, st)) continue;
            const BE<R> b = eval(m, wo, wi, N);
            Ld = Ld + inten * b.f;
        }
        return Ld;
    }
};

template <class R> R emissive_pdf(const Ctx& c, int prim, R dist, const V3<R>& d, uint32_t nfaces) {
    if (prim < 0 || prim >= static_cast<int>(nfaces) || c.tri_pmf == nullptr) return R(0);
    const R pmf = R(c.tri_pmf[prim]);
    if (pmf <= R(0)) return R(0);
    const Face& f = c.geo.f[prim];
    const R ar = face_area<R>(c, f);
    if (ar <= R(0)) return R(0);
    const V3<R> ln = face_normal<R>(c, f);
    const R cl = std::fabs(dot(ln, -d));
    if (cl <= R(1e-5f)) return R(0);
    return pmf * dist * dist / (ar * cl);
}

struct RayF { float o[3], d[3]; };

template <class R> RayF make_ray(const V3<R>& o, const V3<R>& d) {
    const V3<R> dn = nrm(d);
    return RayF{{float(o.x), float(o.y), float(o.z)}, {float(dn.x), float(dn.y), float(dn.z)}};
}

// pathTrace (path.cu:31-206) for pixel (x, y).
template <class R> V3<R> path(const Ctx& c, uint32_t nfaces, int x, int y, Smp& rng, Stats& st) {
    const CamFrame& cf = c.cam;
    V3<R> Lo(R(0)), T(R(1));
    // camera ray (emitRay, path.cu:31-59)
    const float jx = rng.next();
    const float jy = rng.next();
    const R u = (R(2) * (R(static_cast<float>(x)) + R(jx)) / R(static_cast<float>(c.width)) - R(1)) * R(cf.tan_half_fov) * R(cf.aspect);
    const R v = (R(2) * (R(static_cast<float>(y)) + R(jy)) / R(static_cast<float>(c.height)) - R(1)) * R(cf.tan_half_fov);
    V3<R> pos = ld<R>(cf.pos);
    const V3<R> fwd = ld<R>(cf.fwd), rgt = ld<R>(cf.rgt), cup = ld<R>(cf.up);
    V3<R> dir = nrm(u * rgt + v * cup + fwd);
    if (cf.aperture > 0.0f) {
        const V3<R> fp = pos + dir * (R(cf.focal) / dot(dir, fwd));
        const float l1 = rng.next();
        const float l2 = rng.next();
        const R r = std::sqrt(R(l1)) * R(cf.aperture);
        const R th = K<R>::TwoPi * R(l2);
        pos = pos + (rgt * (r * std::cos(th)) + cup * (r * std::sin(th)));
        dir = nrm(fp - pos);
    }
    RayF ray = make_ray(pos, dir);
    R last_pdf = R(0);
    bool last_delta = true;
    for (int d = 0; d < c.max_depth; ++d) {
        ++st.closest;
        const Hit h = closest(c.geo, ray.o, ray.d, st.cc);
        const V3<R> ro(R(ray.o[0]), R(ray.o[1]), R(ray.o[2]));
        const V3<R> rd(R(ray.d[0]), R(ray.d[1]), R(ray.d[2]));
        if (!h.hit) {
            const V3<R> env = env_rad(c, rd);
            if (!eq0(env)) {
                R w = R(1);
                if (d > 0 && !last_delta) w = power(last_pdf, env_pdf(c, rd));
                Lo = Lo + T * env * w;
            }
            break;
        }
        const Face& f = c.geo.f[h.prim];
        const R t = R(h.t), bu = R(h.u), bv = R(h.v);
        const R bw = R(1) - bu - bv;
        const V3<R> hp = ro + t * rd;
        const V3<R> n = nrm(bw * vnr<R>(c, f.v0) + bu * vnr<R>(c, f.v1) + bv * vnr<R>(c, f.v2));
        const Mat& mat = c.mats[f.mat];
        bool entering = dot(n, rd) < R(0);
        V3<R> gn;
        if (mat.double_sided && !entering) { gn = -n; entering = true; }
        else gn = entering ? n : -n;
        const V3<R> wo = -rd;
        V3<R> N = gn;
        float su = 0.0f, sv = 0.0f, tu = 0.0f, tv = 0.0f;
        if (c.ntex > 0) {
            // surface uv (triangle.h:46), applyUvTransform, applyNormalMap with
            // interpolateTangent (shading_utils.cuh:17-68)
            const Vtx& a = c.geo.v[f.v0];
            const Vtx& b = c.geo.v[f.v1];
            const Vtx& cc = c.geo.v[f.v2];
            const R u = bw * R(a.uv[0]) + bu * R(b.uv[0]) + bv * R(cc.uv[0]);
            const R v = bw * R(a.uv[1]) + bu * R(b.uv[1]) + bv * R(cc.uv[1]);
            su = static_cast<float>(u);
            sv = static_cast<float>(v);
            R ttu = u, ttv = v;
            if (!(mat.uvrot == 0.0f && mat.uvsx == 1.0f && mat.uvsy == 1.0f && mat.uvox == 0.0f && mat.uvoy == 0.0f)) {
                const R cr = std::cos(R(mat.uvrot)), sr = std::sin(R(mat.uvrot));
                const R ru = cr * u + sr * v, rv = -sr * u + cr * v;
                ttu = ru * R(mat.uvsx) + R(mat.uvox);
                ttv = rv * R(mat.uvsy) + R(mat.uvoy);
            }
            tu = static_cast<float>(ttu);
            tv = static_cast<float>(ttv);
            if (tex_live(c, mat.tex[kTexNormal])) {
                V3<R> Tg = nrm(V3<R>(bw * R(a.t[0]) + bu * R(b.t[0]) + bv * R(cc.t[0]),
                                     bw * R(a.t[1]) + bu * R(b.t[1]) + bv * R(cc.t[1]),
                                     bw * R(a.t[2]) + bu * R(b.t[2]) + bv * R(cc.t[2])));
                const R sign = a.t[3] >= 0.0f ? R(1) : R(-1);
                const float4 nm = tex_at(c, mat.tex[kTexNormal], tu, tv);
                V3<R> mn(R(nm.x) * R(2) - R(1), R(nm.y) * R(2) - R(1), R(nm.z) * R(2) - R(1));
                mn.x = mn.x * R(mat.normal_scale);
                mn.y = mn.y * R(mat.normal_scale);
                mn = nrm(mn);
                if (Tg.x != R(0) || Tg.y != R(0) || Tg.z != R(0)) {
                    Tg = nrm(Tg - gn * dot(gn, Tg));
                    const V3<R> B = cross(gn, Tg) * sign;
                    N = nrm(Tg * mn.x + B * mn.y + gn * mn.z);
                } else {
                    N = nrm(Frm<R>(gn).world(mn));
                }
            }
        }
        const ME<R> me = c.ntex > 0 ? fetch_tex<R>(c, mat, tu, tv) : fetch<R>(mat);
        if (emits(mat)) {
            R w = R(1);
            if (d > 0 && !last_delta) w = power(last_pdf, emissive_pdf(c, h.prim, t, rd, nfaces));
            Lo = Lo + T * emission<R>(mat) * w;
            break;
        }
        if (mat.alpha_mode == 1) {
            R alpha = R(1);
            if (tex_live(c, mat.tex[kTexBase])) alpha = R(tex_at(c, mat.tex[kTexBase], su, sv).w);
            if (alpha < R(mat.alpha_cutoff)) { ray = make_ray(hp + rd * R(1e-4f), rd); continue; }
        } else if (mat.alpha_mode == 2) {
            R alpha = R(mat.base_alpha);
            if (tex_live(c, mat.tex[kTexBase])) alpha = alpha * R(tex_at(c, mat.tex[kTexBase], su, sv).w);
            if (R(rng.next()) >= alpha) { ray = make_ray(hp + rd * R(1e-4f), rd); continue; }
        }
        const bool delta_surface = (me.metallic >= R(1) && me.roughness < R(0.01f)) ||
                                   (me.spec_trans >= R(1) && me.roughness < R(0.01f));
        if (!delta_surface) {
            const bool has_area = c.nem > 0 && c.em != nullptr;
            const bool has_env = c.has_tex && c.env_alias != nullptr && c.n_env > 0 && c.env_w > 0 && c.env_h > 0;
            V3<R> Ld(R(0));
            if (has_area && has_env) {
                Ld = Ld + Shade<R>::direct(Shade<R>::area(c, hp, N, rng, st), me, wo, N);
                Ld = Ld + Shade<R>::direct(Shade<R>::env(c, hp, N, rng, st), me, wo, N);
            } else if (has_area) {
                Ld = Shade<R>::direct(Shade<R>::area(c, hp, N, rng, st), me, wo, N);
            } else if (has_env) {
                Ld = Shade<R>::direct(Shade<R>::env(c, hp, N, rng, st), me, wo, N);
            }
            Lo = Lo + T * Ld;
            Lo = Lo + T * Shade<R>::punctual(c, hp, me, wo, N, st);
        }
        const BS<R> bs = sample(me, wo, N, rng, c.rtl, entering);
        if (!bs.valid) break;
        T = T * bs.weight;
        const bool transmitted = dot(bs.wi, gn) < R(0);
        const V3<R> off = transmitted ? -gn : gn;
        ray = make_ray(hp + off * R(1e-4f), bs.wi);
        if (transmitted && me.thickness > R(0) && me.att_distance < R(1e20f)) {
            const R th = me.thickness, ad = me.att_distance;
            const V3<R> ac = me.att_color;
            T = T * V3<R>(std::exp(-th * fmx(-std::log(fmx(ac.x, R(1e-6f))), R(0)) / ad),
                          std::exp(-th * fmx(-std::log(fmx(ac.y, R(1e-6f))), R(0)) / ad),
                          std::exp(-th * fmx(-std::log(fmx(ac.z, R(1e-6f))), R(0)) / ad));
        }
        last_pdf = bs.pdf;
        last_delta = bs.delta;
        if (d > 2) {
            const R mc = fmx(fmx(T.x, T.y), T.z);
            const R sp = fmn(mc, R(0.95f));
            if (R(rng.next()) >= sp) break;
            T = T / sp;
        }
    }
    Lo.x = fmn(Lo.x, R(100));
    Lo.y = fmn(Lo.y, R(100));
    Lo.z = fmn(Lo.z, R(100));
    return Lo;
}

// ---------------------------------------------------------------------------
// SAH BVH restated (bvh_builder.cpp:56-221), single threaded.
// ---------------------------------------------------------------------------
struct BPrim { float lo[3], hi[3]; uint32_t idx; float c(int a) const { return 0.5f * (lo[a] + hi[a]); } };
struct BB {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX}, hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const float* l, const float* h) { for (int i = 0; i < 3; ++i) { lo[i] = std::fmin(lo[i], l[i]); hi[i] = std::fmax(hi[i], h[i]); } }
    float area() const {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
        return 2.0f * (dx * dy + dx * dz + dy * dz);
    }
    int axis() const {
        const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (dx > dy && dx > dz) return 0;
        return dy > dz ? 1 : 2;
    }
};
struct SahRef {
    std::vector<BPrim>& P;
    std::vector<Node>& N;
    uint32_t count = 0;
    uint32_t build(uint32_t s, uint32_t e) {
        const uint32_t me = count++;
        BB nb;
        for (uint32_t i = s; i < e; ++i) nb.grow(P[i].lo, P[i].hi);
        auto leaf = [&] {
            Node& n = N[me];
            for (int i = 0; i < 3; ++i) { n.lo[i] = nb.lo[i]; n.hi[i] = nb.hi[i]; }
            n.d0 = s | kLeaf; n.d1 = e - s;
            return me;
        };
        if (e - s < 4u) return leaf();
        BB cb;
        for (uint32_t i = s; i < e; ++i) { const float p[3] = {P[i].c(0), P[i].c(1), P[i].c(2)}; cb.grow(p, p); }
        const int dim = cb.axis();
        auto bucket = [&](const BPrim& p) {
            const float c = p.c(dim), d = cb.hi[dim] - cb.lo[dim];
            const int b = static_cast<int>(24 * (d > 0 ? (c - cb.lo[dim]) / d : 0.0f));
            return b >= 24 ? 23 : b;
        };
        BB bb[24];
        uint32_t bc[24] = {};
        for (uint32_t i = s; i < e; ++i) { const int b = bucket(P[i]); bc[b]++; bb[b].grow(P[i].lo, P[i].hi); }
        float cost[23] = {};
        uint32_t nf = 0;
        BB fw;
        for (int i = 0; i < 23; ++i) { nf += bc[i]; fw.grow(bb[i].lo, bb[i].hi); cost[i] += nf * fw.area(); }
        uint32_t nbk = 0;
        BB bw;
        for (int i = 22; i >= 0; --i) { nbk += bc[i + 1]; bw.grow(bb[i + 1].lo, bb[i + 1].hi); cost[i] += nbk * bw.area(); }
        int best = static_cast<int>(std::min_element(cost, cost + 23) - cost);
        const float sa = nb.area();
        const float mc = 0.5f + (sa > 0.0f ? cost[best] / sa : 0.0f);
        if (static_cast<float>(e - s) < mc) return leaf();
        const uint32_t mid = static_cast<uint32_t>(
            std::partition(P.begin() + s, P.begin() + e, [&](const BPrim& p) { return bucket(p) <= best; }) - P.begin());
        if (mid == e) return leaf();
        const uint32_t l = build(s, mid);
        const uint32_t r = build(mid, e);
        Node& n = N[me];
        for (int i = 0; i < 3; ++i) { n.lo[i] = nb.lo[i]; n.hi[i] = nb.hi[i]; }
        n.d0 = l; n.d1 = r;
        return me;
    }
};
uint32_t dfs(const std::vector<Node>& in, std::vector<Node>& out, uint32_t i, uint32_t lvl, uint32_t& depth) {
    out.push_back(in[i]);
    const uint32_t me = static_cast<uint32_t>(out.size() - 1);
    depth = std::max(depth, lvl);
    if (!(in[i].d0 & kLeaf)) {
        const uint32_t l = dfs(in, out, in[i].d0, lvl + 1, depth);
        out[me].d0 = l;
        const uint32_t r = dfs(in, out, in[i].d1, lvl + 1, depth);
        out[me].d1 = r;
    }
    return me;
}

std::vector<Alias> alias_table(const std::vector<float>& w) {
    const uint32_t n = static_cast<uint32_t>(w.size());
    if (n == 0) return {};
    float sum = 0.0f;
    for (float x : w) sum += x;
    if (sum <= 0.0f) return {};
    std::vector<float> p(n);
    for (uint32_t i = 0; i < n; ++i) p[i] = w[i] / sum * static_cast<float>(n);
    std::vector<Alias> t(n);
    std::queue<uint32_t> sm, lg;
    for (uint32_t i = 0; i < n; ++i) (p[i] < 1.0f ? sm : lg).push(i);
    while (!sm.empty() && !lg.empty()) {
        const uint32_t a = sm.front(); sm.pop();
        const uint32_t b = lg.front(); lg.pop();
        t[a] = Alias{p[a], b};
        p[b] = (p[b] + p[a]) - 1.0f;
        (p[b] < 1.0f ? sm : lg).push(b);
    }
    while (!lg.empty()) { const uint32_t b = lg.front(); lg.pop(); t[b] = Alias{1.0f, b}; }
    while (!sm.empty()) { const uint32_t a = sm.front(); sm.pop(); t[a] = Alias{1.0f, a}; }
    return t;
}

}  // namespace

extern "C" {

int oracle_build_bvh(const void* vertices, uint32_t nv, void* faces_inout, uint32_t nf, void* nodes_out,
                     uint32_t cap, uint32_t* num_nodes, uint32_t* depth) {
    *num_nodes = 0; *depth = 0;
    if (nf == 0) return 0;
    const Vtx* V = static_cast<const Vtx*>(vertices);
    Face* F = static_cast<Face*>(faces_inout);
    std::vector<BPrim> P(nf);
    for (uint32_t i = 0; i < nf; ++i) {
        if (F[i].v0 >= nv || F[i].v1 >= nv || F[i].v2 >= nv) return 1;
        const float* a = V[F[i].v0].p; const float* b = V[F[i].v1].p; const float* c = V[F[i].v2].p;
        for (int k = 0; k < 3; ++k) {
            P[i].lo[k] = std::fmin(std::fmin(a[k], b[k]), c[k]);
            P[i].hi[k] = std::fmax(std::fmax(a[k], b[k]), c[k]);
        }
        P[i].idx = i;
    }
    std::vector<Node> tmp(2 * static_cast<size_t>(nf));
    SahRef b{P, tmp};
    b.build(0, nf);
    tmp.resize(b.count);
    std::vector<Node> out;
    out.reserve(tmp.size());
    uint32_t dep = 0;
    dfs(tmp, out, 0, 0, dep);
    if (out.size() > cap) return 2;
    std::memcpy(nodes_out, out.data(), out.size() * sizeof(Node));
    std::vector<Face> rf(nf);
    for (uint32_t i = 0; i < nf; ++i) rf[i] = F[P[i].idx];
    std::memcpy(F, rf.data(), nf * sizeof(Face));
    *num_nodes = static_cast<uint32_t>(out.size());
    *depth = dep;
    return 0;
}

int oracle_alias_table(const float* weights, uint32_t n, void* out) {
    const std::vector<Alias> t = alias_table(std::vector<float>(weights, weights + n));
    if (!t.empty()) std::memcpy(out, t.data(), t.size() * sizeof(Alias));
    return t.empty() ? 1 : 0;
}

int oracle_emissive_tables(const void* vertices, const void* faces, uint32_t nf, const void* materials, uint32_t nm,
                           void* refs_out, float* pmf_out, void* alias_out, uint32_t* count) {
    const Vtx* V = static_cast<const Vtx*>(vertices);
    const Face* F = static_cast<const Face*>(faces);
    const Mat* M = static_cast<const Mat*>(materials);
    std::vector<EmRef> refs;
    std::vector<float> w;
    for (uint32_t i = 0; i < nf; ++i) pmf_out[i] = 0.0f;
    for (uint32_t i = 0; i < nf; ++i) {
        if (F[i].mat < 0 || F[i].mat >= static_cast<int>(nm)) continue;
        const Mat& m = M[F[i].mat];
        if (!emits(m)) continue;
        const V3<float> e1 = ld<float>(V[F[i].v1].p) - ld<float>(V[F[i].v0].p);
        const V3<float> e2 = ld<float>(V[F[i].v2].p) - ld<float>(V[F[i].v0].p);
        const float area = 0.5f * len(cross(e1, e2));
        if (area <= 0.0f) continue;
        const float wt = area * std::fmax(lum(emission<float>(m)), 0.0f);
        if (wt <= 0.0f) continue;
        refs.push_back(EmRef{i, 0.0f, 0.0f, 0.0f});
        w.push_back(wt);
    }
    *count = 0;
    if (refs.empty()) return 0;
    float sum = 0.0f;
    for (float x : w) sum += x;
    if (sum <= 0.0f) return 0;
    float acc = 0.0f;
    for (size_t i = 0; i < refs.size(); ++i) {
        const float p = w[i] / sum;
        acc += p;
        refs[i].pmf = p;
        refs[i].cdf = acc;
        pmf_out[refs[i].tri] = p;
    }
    refs.back().cdf = 1.0f;
    const std::vector<Alias> t = alias_table(w);
    std::memcpy(refs_out, refs.data(), refs.size() * sizeof(EmRef));
    std::memcpy(alias_out, t.data(), t.size() * sizeof(Alias));
    *count = static_cast<uint32_t>(refs.size());
    return 0;
}

int oracle_env_tables(const float* rgba, int32_t w, int32_t h, float* pmf_out, void* alias_out) {
    if (w <= 0 || h <= 0) return 1;
    const size_t n = static_cast<size_t>(w) * h;
    std::vector<float> wt(n, 0.0f);
    for (int y = 0; y < h; ++y) {
        const float th = K<float>::Pi * (static_cast<float>(y) + 0.5f) / static_cast<float>(h);
        const float st = std::fmax(std::sin(th), 0.0f);
        for (int x = 0; x < w; ++x) {
            const size_t i = static_cast<size_t>(y) * w + x;
            wt[i] = std::fmax(lum(V3<float>(rgba[i * 4], rgba[i * 4 + 1], rgba[i * 4 + 2])), 0.0f) * st;
        }
    }
    float sum = 0.0f;
    for (float x : wt) sum += x;
    if (sum <= 0.0f) return 1;
    for (size_t i = 0; i < n; ++i) pmf_out[i] = wt[i] / sum;
    const std::vector<Alias> t = alias_table(wt);
    std::memcpy(alias_out, t.data(), t.size() * sizeof(Alias));
    return 0;
}

int oracle_camera_frame(const void* camera, void* out) {
    const Cam& c = *static_cast<const Cam*>(camera);
    const V3<float> pos = ld<float>(c.pos);
    const V3<float> fwd = nrm(ld<float>(c.look) - pos);
    const V3<float> rgt = nrm(cross(fwd, ld<float>(c.up)));
    const V3<float> cup = cross(rgt, fwd);
    CamFrame f{};
    f.pos[0] = pos.x; f.pos[1] = pos.y; f.pos[2] = pos.z;
    f.fwd[0] = fwd.x; f.fwd[1] = fwd.y; f.fwd[2] = fwd.z;
    f.rgt[0] = rgt.x; f.rgt[1] = rgt.y; f.rgt[2] = rgt.z;
    f.up[0] = cup.x; f.up[1] = cup.y; f.up[2] = cup.z;
    f.tan_half_fov = std::tan(c.fov * K<float>::Pi / 360.0f);
    f.aspect = static_cast<float>(c.w) / c.h;
    f.aperture = c.aperture;
    f.focal = c.focal;
    std::memcpy(out, &f, sizeof(f));
    return 0;
}

int oracle_sampler_stream(int32_t type, int32_t w, int32_t h, uint32_t frame, int32_t spf, int32_t sif,
                          uint32_t ndims, uint32_t pcg_seed, float* out) {
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            Smp s;
            if (type == 1) s.sobol(x, y, frame * static_cast<uint32_t>(spf) + static_cast<uint32_t>(sif));
            else s.pcg(x, y, frame, static_cast<uint32_t>(sif), pcg_seed);
            float* o = out + (static_cast<size_t>(y) * w + x) * ndims;
            for (uint32_t k = 0; k < ndims; ++k) o[k] = s.next();
        }
    return 0;
}

int oracle_trace(const void* nodes, const void* vertices, const void* faces, const float* rays, uint32_t n,
                 int32_t any, float* hits_out, uint8_t* occl_out, oracle_counters* counters) {
    return oracle_trace_mode(nodes, vertices, faces, rays, n, any, 0, hits_out, occl_out, counters);
}

int oracle_trace_mode(const void* nodes, const void* vertices, const void* faces, const float* rays, uint32_t n,
                      int32_t any, int32_t watertight, float* hits_out, uint8_t* occl_out,
                      oracle_counters* counters) {
    Geo g{static_cast<const Node*>(nodes), static_cast<const Vtx*>(vertices), static_cast<const Face*>(faces), 1,
          watertight != 0};
    // rays in blocks of 4096 handed out to the host threads; counters summed
    const uint32_t block = 4096;
    const uint32_t nblocks = (n + block - 1) / block;
    const int threads = static_cast<int>(std::min<uint32_t>(std::max(1u, std::thread::hardware_concurrency()),
                                                            std::max(1u, nblocks)));
    std::atomic<uint32_t> next{0};
    std::atomic<uint64_t> pops{0}, tris{0};
    auto worker = [&]() {
        Cnt c;
        for (uint32_t b = next++; b < nblocks; b = next++) {
            const uint32_t end = std::min(n, (b + 1) * block);
            for (uint32_t i = b * block; i < end; ++i) {
                const float* r = rays + static_cast<size_t>(i) * 8;
                const float o[3] = {r[0], r[1], r[2]}, d[3] = {r[4], r[5], r[6]};
                if (any) {
                    occl_out[i] = occluded(g, o, d, r[7], c) ? 1 : 0;
                } else {
                    const Hit h = closest(g, o, d, c);
                    float* out = hits_out + static_cast<size_t>(i) * 4;
                    out[0] = h.t;
                    std::memcpy(&out[1], &h.prim, 4);
                    out[2] = h.u;
                    out[3] = h.v;
                }
            }
        }
        pops += c.pops;
        tris += c.tris;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(worker);
    worker();
    for (auto& th : pool) th.join();
    Cnt c;
    c.pops = pops;
    c.tris = tris;
    if (counters) {
        std::memset(counters, 0, sizeof(*counters));
        if (any) { counters->shadow_rays = n; counters->shadow_node_pops = c.pops; counters->shadow_tri_tests = c.tris; }
        else { counters->closest_rays = n; counters->node_pops = c.pops; counters->tri_tests = c.tris; }
    }
    return 0;
}

int oracle_render(const oracle_scene* sc, const oracle_render_args* a, float* out_f32, double* out_mean,
                  double* out_var, oracle_counters* counters) {
    Ctx c{};
    c.geo = Geo{static_cast<const Node*>(sc->nodes), static_cast<const Vtx*>(sc->vertices),
                static_cast<const Face*>(sc->faces), sc->num_nodes, a->watertight != 0};
    c.mats = static_cast<const Mat*>(sc->materials);
    c.nmat = sc->num_materials;
    c.texs = static_cast<const OTex*>(sc->textures);
    c.ntex = sc->textures ? sc->num_textures : 0u;
    c.em = sc->num_emissive ? static_cast<const EmRef*>(sc->emissive) : nullptr;
    c.nem = sc->num_emissive;
    c.tri_pmf = sc->tri_pmf;
    c.tri_alias = static_cast<const Alias*>(sc->tri_alias);
    c.has_tex = sc->env_rgba != nullptr && sc->env_w > 0 && sc->env_h > 0;
    c.tex = HostTexture{sc->env_rgba, sc->env_w, sc->env_h};
    c.env_pmf = sc->env_pmf;
    c.env_alias = static_cast<const Alias*>(sc->env_alias);
    c.n_env = sc->num_env_texels;
    c.env_w = sc->env_tw;
    c.env_h = sc->env_th;
    c.pl = static_cast<const Punctual*>(sc->punctual);
    c.npl = sc->num_punctual;
    std::memcpy(&c.cam, sc->camera_frame, sizeof(CamFrame));
    c.width = sc->width;
    c.height = sc->height;
    c.spf = a->sample_per_frame;
    c.max_depth = a->max_depth;
    c.rtl = a->arg_rtl;
    const int w = c.width, h = c.height;
    const uint32_t nfaces = sc->num_faces;
    int threads = a->threads > 0 ? a->threads : static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    const int step = a->row_step > 0 ? a->row_step : 1;
    const int y_end = a->row_end > 0 ? std::min(a->row_end, h) : h;
    const int x0 = std::max(a->col0, 0), x1 = a->col1 > 0 ? std::min(a->col1, w) : w;
    std::vector<int> rows;
    for (int y = a->row0; y < y_end; y += step) rows.push_back(y);
    std::atomic<uint64_t> acc_c{0}, acc_s{0}, np{0}, nt{0}, snp{0}, snt{0};
    std::atomic<size_t> next_row{0};
    const auto t0 = std::chrono::steady_clock::now();
    auto worker = [&](int) {
        Stats st;
        for (size_t k = next_row++; k < rows.size(); k = next_row++) {
            const int y = rows[k];
            for (int x = x0; x < x1; ++x) {
                const size_t p = static_cast<size_t>(y) * w + x;
                if (a->precision == 64) {
                    double s[3] = {0, 0, 0}, q[3] = {0, 0, 0};
                    uint64_t n = 0;
                    for (uint32_t f = a->first_frame; f < a->first_frame + a->num_frames; ++f)
                        for (int i = 0; i < c.spf; ++i) {
                            Smp rng;
                            if (a->sampler_type == 1) rng.sobol(x, y, f * static_cast<uint32_t>(c.spf) + static_cast<uint32_t>(i));
                            else rng.pcg(x, y, f, static_cast<uint32_t>(i), a->pcg_seed);
                            const V3<double> L = path<double>(c, nfaces, x, y, rng, st);
                            const double v[3] = {L.x, L.y, L.z};
                            for (int ch = 0; ch < 3; ++ch) { s[ch] += v[ch]; q[ch] += v[ch] * v[ch]; }
                            ++n;
                        }
                    for (int ch = 0; ch < 3; ++ch) {
                        const double m = n ? s[ch] / n : 0.0;
                        if (out_mean) out_mean[p * 3 + ch] = m;
                        if (out_var) out_var[p * 3 + ch] = n > 1 ? (q[ch] - n * m * m) / (n - 1) : 0.0;
                    }
                } else {
                    // kernelPathTrace (path.cu:209-242): per-frame mean, running mean across frames
                    float4 accs = make_float4(0, 0, 0, 0);
                    for (uint32_t f = a->first_frame; f < a->first_frame + a->num_frames; ++f) {
                        V3<float> acc(0.0f);
                        for (int i = 0; i < c.spf; ++i) {
                            Smp rng;
                            if (a->sampler_type == 1) rng.sobol(x, y, f * static_cast<uint32_t>(c.spf) + static_cast<uint32_t>(i));
                            else rng.pcg(x, y, f, static_cast<uint32_t>(i), a->pcg_seed);
                            acc = acc + path<float>(c, nfaces, x, y, rng, st);
                        }
                        acc = acc / static_cast<float>(c.spf);
                        const float inv = 1.0f / static_cast<float>(f + 1);
                        accs.x = accs.x * (1.0f - inv) + acc.x * inv;
                        accs.y = accs.y * (1.0f - inv) + acc.y * inv;
                        accs.z = accs.z * (1.0f - inv) + acc.z * inv;
                        accs.w = accs.w * (1.0f - inv) + 1.0f * inv;
                    }
                    if (out_f32) { out_f32[p * 4] = accs.x; out_f32[p * 4 + 1] = accs.y; out_f32[p * 4 + 2] = accs.z; out_f32[p * 4 + 3] = accs.w; }
                }
            }
        }
        acc_c += st.closest; acc_s += st.shadow;
        np += st.cc.pops; nt += st.cc.tris; snp += st.sc.pops; snt += st.sc.tris;
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t) pool.emplace_back(worker, t);
    for (auto& th : pool) th.join();
    if (counters) {
        counters->closest_rays = acc_c; counters->shadow_rays = acc_s;
        counters->node_pops = np; counters->tri_tests = nt;
        counters->shadow_node_pops = snp; counters->shadow_tri_tests = snt;
        counters->paths = static_cast<uint64_t>(rows.size()) * static_cast<uint64_t>(std::max(x1 - x0, 0)) * c.spf * a->num_frames;
        counters->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    }
    return 0;
}

int oracle_bsdf_eval(const void* materials, uint32_t nm, const float* in, uint32_t n, float* out) {
    const Mat* M = static_cast<const Mat*>(materials);
    for (uint32_t i = 0; i < n; ++i) {
        const float* r = in + static_cast<size_t>(i) * 13;
        float* o = out + static_cast<size_t>(i) * 4;
        const uint32_t mi = static_cast<uint32_t>(r[0]);
        if (mi >= nm) { o[0] = o[1] = o[2] = o[3] = 0.0f; continue; }
        const ME<float> me = fetch<float>(M[mi]);
        const BE<float> b = eval(me, V3<float>(r[1], r[2], r[3]), V3<float>(r[4], r[5], r[6]), V3<float>(r[7], r[8], r[9]));
        o[0] = b.f.x; o[1] = b.f.y; o[2] = b.f.z; o[3] = b.pdf;
    }
    return 0;
}

}  // extern "C"
