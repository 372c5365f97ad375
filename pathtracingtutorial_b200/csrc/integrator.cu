// integrator.cu -- wavefront path-tracing integrator for sm_100a.
//
// Replaces the reference's megakernel kernelPathTrace/pathTrace
// (Part_2/src/integrators/path.cu:31-255) by stages over structure-of-arrays
// queues; one sample pass covers every pixel once:
//
//   raygen   camera rays for all pixels               (path.cu:31-59, 217-225)
//   extend   closest-hit traversal of the ray queue   (bvh_traversal.cuh:43-96)
//   shade    miss/emission MIS, NEE sampling, BSDF sampling, Russian roulette
//            -> next ray queue + shadow queue         (path.cu:69-199,
//                                                      direct_lighting.cuh:55-249)
//   shadow   any-hit traversal of the shadow queue; visible contributions are
//            added to per-(path, light slot) accumulators (one writer each, so
//            the result is deterministic)           (bvh_traversal.cuh:98-133)
//   finalize per-sample firefly clamp and compensated (Neumaier) FP32
//            accumulation into the film              (path.cu:201-204, 228-241)
//
// Kernels grid-stride over a queue length that lives in device memory, so a
// whole batch (sample_per_frame passes x max_depth bounces) is a fixed launch
// sequence that is captured once into a CUDA graph and replayed.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"
#include "bsdf.h"
#include "traverse.h"
#include <cub/device/device_scan.cuh>

#include "guide.cuh"
#include "guide_tc.cuh"
#include "guide_host.cuh"

namespace ptb {

#define PT_CU(call)                                                                      \
    do {                                                                                 \
        cudaError_t e__ = (call);                                                        \
        if (e__ != cudaSuccess) {                                                        \
            set_error(std::string("CUDA error: ") + cudaGetErrorString(e__) + " in " #call); \
            return PT_ERR_CUDA;                                                          \
        }                                                                                \
    } while (0)

enum StatIdx {
    kStatCameraRays = 0, kStatExtRays, kStatShadowRays, kStatNodes, kStatTris,
    kStatShadowNodes, kStatShadowTris, kStatPaths, kStatCount
};

struct PassState { uint32_t frame; uint32_t pad[3]; };

struct WaveParams {
    DeviceScene scene;
    pt_camera_frame cam;
    int      width, height, npix;
    int      npath;     // path slots: npix x lanes (lanes = samples per pixel in flight)
    int      spf, max_depth, sampler_type, arg_rtl, flags;
    uint32_t pcg_seed;
    int      n_slots;
    uint32_t* queue[2];
    float4*  ray_o[2];
    float4*  ray_d[2];
    float4*  hit;
    float4*  thr;       // xyz throughput, w last BSDF pdf
    float4*  lo;        // xyz radiance from emission / env hits, w last-was-delta
    uint32_t* rng;      // sobol dimension or pcg state
    float4*  nee;       // n_slots x npath visible NEE contributions
    uint32_t* sq_path;
    float4*  sq_o;      // w = slot (bits)
    float4*  sq_d;      // w = tmax
    float4*  sq_c;
    uint32_t* counts;   // [0], [1] path queues, [2] shadow queue, [4] sampling list
    uint32_t* slist;    // queue entries that continue by sampling (k_shade_front -> k_shade_back)
    unsigned long long* stats;
    uint32_t* err;
    PassState* pass;
    float4*  f_sum;
    float4*  f_comp;
    float4*  f_batch;
    float4*  f_new;
    // learned guiding (null when off)
    const float* gmix;   // queue-ordered mixtures, kGMix floats per entry
    float    galpha;     // probability of sampling the mixture (one-sample MIS)
    float4*  grec;       // training records [depth][npath][4]
    // traversal kernel shape (threads per block, stack entries)
    int      trace_block, stack_depth;
};

// ---------------------------------------------------------------------------
// Device helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t warp_append(uint32_t* counter, bool want) {
    const uint32_t active = __activemask();
    const uint32_t ballot = __ballot_sync(active, want);
    if (!want) return 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(ballot) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(counter, static_cast<uint32_t>(__popc(ballot)));
    base = __shfl_sync(ballot, base, leader);
    return base + static_cast<uint32_t>(__popc(ballot & ((1u << lane) - 1u)));
}

__device__ __forceinline__ f3 f3of(float4 v) { return mk(v.x, v.y, v.z); }
__device__ __forceinline__ float4 f4of(f3 v, float w) { return make_float4(v.x, v.y, v.z, w); }

// Equirectangular mapping (Part_2/src/lights/envmap.h:15-33).
__device__ __forceinline__ void spherical_uv(f3 d, float& u, float& v) {
    u = atan2f(d.z, d.x) * kInv2Pi + 0.5f;
    v = 1.0f - (asinf(d.y) * kInvPi + 0.5f);
}
__device__ __forceinline__ f3 dir_from_uv(float u, float v) {
    const float phi = (u - 0.5f) * kTwoPi;
    const float theta = v * kPi;
    const float st = sinf(theta);
    return normalize(mk(cosf(phi) * st, cosf(theta), sinf(phi) * st));
}
// Environment radiance: hardware bilinear lookup (wrap, normalized) x 2*pi
// (envmap.h:36-45; the reference samples the same texture configuration).
__device__ __forceinline__ f3 env_radiance(const DeviceScene& s, f3 d) {
    if (s.env_tex == 0) return mk(0.0f);
    float u, v;
    spherical_uv(d, u, v);
    const float4 c = tex2D<float4>(static_cast<cudaTextureObject_t>(s.env_tex), u, v);
    return mk(c.x, c.y, c.z) * kTwoPi;
}
__device__ __forceinline__ bool has_env_light(const DeviceScene& s) {
    return s.env_tex != 0 && s.env_alias != nullptr && s.num_env_texels > 0 && s.env_w > 0 && s.env_h > 0;
}
// environmentPdf (Part_2/src/lights/light_pdf.cuh:12-29)
__device__ float env_pdf(const DeviceScene& s, f3 d) {
    if (s.env_tex == 0 || s.env_pmf == nullptr || s.num_env_texels == 0 || s.env_w <= 0 || s.env_h <= 0) return 0.0f;
    float u, v;
    spherical_uv(d, u, v);
    const int x = static_cast<int>(clampf(u * s.env_w, 0.0f, static_cast<float>(s.env_w - 1)));
    const int y = static_cast<int>(clampf(v * s.env_h, 0.0f, static_cast<float>(s.env_h - 1)));
    const float st = sqrtf(fmaxf(0.0f, 1.0f - d.y * d.y));
    if (st <= 1e-5f) return 0.0f;
    return __ldg(s.env_pmf + (y * s.env_w + x)) * static_cast<float>(s.env_w * s.env_h) / (kTwoPi * kPi * st);
}
__device__ __forceinline__ f3 vpos(const DeviceScene& s, uint32_t i) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(s.vertices + i));
    return mk(a.x, a.y, a.z);
}
__device__ __forceinline__ f3 vnrm(const DeviceScene& s, uint32_t i) {
    const float4 a = __ldg(reinterpret_cast<const float4*>(s.vertices + i) + 1);
    return mk(a.x, a.y, a.z);
}
__device__ __forceinline__ pt_face load_face(const DeviceScene& s, uint32_t i) {
    const uint4 f = __ldg(reinterpret_cast<const uint4*>(s.faces + i));
    pt_face r; r.v0 = f.x; r.v1 = f.y; r.v2 = f.z; r.material_id = static_cast<int32_t>(f.w);
    return r;
}
// ---- material textures (Part_2/src/materials/shading_utils.cuh:17-68 and
//      disney_bsdf.cuh:79-116) ----
// A texture id is looked up only when it names a texture with an image.
__device__ __forceinline__ bool tex_live(const DeviceScene& s, int32_t id) {
    return id >= 0 && static_cast<uint32_t>(id) < s.num_textures && s.textures[id] != 0ull;
}
__device__ __forceinline__ float4 tex_at(const DeviceScene& s, int32_t id, float u, float v) {
    return tex2D<float4>(static_cast<cudaTextureObject_t>(s.textures[id]), u, v);
}
// texel colour to linear (the reference's pow(c, 2.2) per channel)
__device__ __forceinline__ f3 tex_linear(float4 c) { return mk(powf(c.x, 2.2f), powf(c.y, 2.2f), powf(c.z, 2.2f)); }
__device__ __forceinline__ float2 vuv(const DeviceScene& s, uint32_t i) {
    return __ldg(reinterpret_cast<const float2*>(s.vertices + i) + 4);
}
__device__ __forceinline__ float4 vtan(const DeviceScene& s, uint32_t i) {
    return __ldg(reinterpret_cast<const float4*>(s.vertices + i) + 3);
}

// fetchMaterial with textures: the factors times the texel channels, then
// the reference's clamps.  (The emissive texture only changes the evaluated
// material's emission, which the path loop never reads: emission comes from
// the material record, path.cu:105-111.)
__device__ MatEval resolve_material_textured(const DeviceScene& s, const pt_material& m, float u, float v) {
    MatEval e = resolve_material(m);
    float rough = m.roughness, metal = m.metallic, ccr = m.clearcoat_roughness;
    if (tex_live(s, m.base_color_tex)) e.base = e.base * tex_linear(tex_at(s, m.base_color_tex, u, v));
    if (tex_live(s, m.metallic_roughness_tex)) {
        const float4 t = tex_at(s, m.metallic_roughness_tex, u, v);
        rough *= t.y;
        metal *= t.z;
    }
    if (tex_live(s, m.clearcoat_tex)) e.clearcoat *= tex_at(s, m.clearcoat_tex, u, v).x;
    if (tex_live(s, m.clearcoat_roughness_tex)) ccr *= tex_at(s, m.clearcoat_roughness_tex, u, v).y;
    if (tex_live(s, m.transmission_tex)) e.spec_trans *= tex_at(s, m.transmission_tex, u, v).x;
    if (tex_live(s, m.sheen_color_tex)) e.sheen_color = e.sheen_color * tex_linear(tex_at(s, m.sheen_color_tex, u, v));
    if (tex_live(s, m.sheen_roughness_tex)) e.sheen *= tex_at(s, m.sheen_roughness_tex, u, v).w;
    e.roughness = clampf(rough, 0.001f, 1.0f);
    e.metallic = clampf(metal, 0.0f, 1.0f);
    e.cc_roughness = clampf(ccr, 0.001f, 1.0f);
    return e;
}

// The surface at a hit as the path loop sees it (path.cu:84-102): the
// interpolated normal oriented towards the ray (double-sided materials
// flipped), and -- for textured scenes -- the surface uv, the material's
// transformed uv and the normal-mapped shading normal.  Front and back
// shading kernels both call it, so they see the same surface.
struct SurfaceAt {
    f3    gn, N;          // oriented geometric normal, shading normal
    bool  entering;
    float su, sv;         // interpolated uv (alpha lookups)
    float tu, tv;         // after the material's uv transform (texture lookups)
};

template <bool Textured>
__device__ __forceinline__ void surface_at(const DeviceScene& s, const pt_face& f, const pt_material& m, float bu,
                                           float bv, f3 rd, SurfaceAt& g) {
    const float bw = 1.0f - bu - bv;
    const f3 n = normalize(bw * vnrm(s, f.v0) + bu * vnrm(s, f.v1) + bv * vnrm(s, f.v2));
    bool entering = dot(n, rd) < 0.0f;
    if (m.double_sided && !entering) { g.gn = -n; entering = true; }
    else g.gn = entering ? n : -n;
    g.entering = entering;
    g.N = g.gn;
    g.su = g.sv = g.tu = g.tv = 0.0f;
    if (!Textured) return;
    const float2 a = vuv(s, f.v0), b = vuv(s, f.v1), c = vuv(s, f.v2);
    g.su = bw * a.x + bu * b.x + bv * c.x;
    g.sv = bw * a.y + bu * b.y + bv * c.y;
    // applyUvTransform (shading_utils.cuh:17-28)
    g.tu = g.su;
    g.tv = g.sv;
    if (!(m.uv_rotation == 0.0f && m.uv_scale_x == 1.0f && m.uv_scale_y == 1.0f && m.uv_offset_x == 0.0f &&
          m.uv_offset_y == 0.0f)) {
        const float cr = cosf(m.uv_rotation), sr = sinf(m.uv_rotation);
        const float ru = cr * g.su + sr * g.sv;
        const float rv = -sr * g.su + cr * g.sv;
        g.tu = ru * m.uv_scale_x + m.uv_offset_x;
        g.tv = rv * m.uv_scale_y + m.uv_offset_y;
    }
    // applyNormalMap (shading_utils.cuh:43-68) with interpolateTangent (:30-41);
    // the reference's tangent flip for double-sided back faces cannot trigger
    // (entering is true by then), so none is applied here either
    if (tex_live(s, m.normal_tex)) {
        const float4 t0 = vtan(s, f.v0), t1 = vtan(s, f.v1), t2 = vtan(s, f.v2);
        f3 T = normalize(mk(bw * t0.x + bu * t1.x + bv * t2.x, bw * t0.y + bu * t1.y + bv * t2.y,
                            bw * t0.z + bu * t1.z + bv * t2.z));
        const float sign = t0.w >= 0.0f ? 1.0f : -1.0f;
        const float4 nm = tex_at(s, m.normal_tex, g.tu, g.tv);
        f3 mn = mk(nm.x * 2.0f - 1.0f, nm.y * 2.0f - 1.0f, nm.z * 2.0f - 1.0f);
        mn.x *= m.normal_scale;
        mn.y *= m.normal_scale;
        mn = normalize(mn);
        if (T.x != 0.0f || T.y != 0.0f || T.z != 0.0f) {
            T = normalize(T - g.gn * dot(g.gn, T));
            const f3 B = cross(g.gn, T) * sign;
            g.N = normalize(T * mn.x + B * mn.y + g.gn * mn.z);
        } else {
            const Frame tbn = make_frame(g.gn);
            g.N = normalize(to_world(tbn, mn));
        }
    }
}

// hit point o + t d with explicit fused multiply-adds (the same value wherever computed)
__device__ __forceinline__ f3 hit_point(f3 o, f3 d, float t) {
    return mk(fmaf(t, d.x, o.x), fmaf(t, d.y, o.y), fmaf(t, d.z, o.z));
}

// emissiveTrianglePdf (light_pdf.cuh:31-54)
__device__ float emissive_pdf(const DeviceScene& s, int prim, float dist, f3 dir) {
    if (prim < 0 || prim >= static_cast<int>(s.num_faces) || s.tri_light_pmf == nullptr) return 0.0f;
    const float pmf = __ldg(s.tri_light_pmf + prim);
    if (pmf <= 0.0f) return 0.0f;
    const pt_face f = load_face(s, prim);
    const f3 p0 = vpos(s, f.v0), p1 = vpos(s, f.v1), p2 = vpos(s, f.v2);
    const f3 c = cross(p1 - p0, p2 - p0);
    const float area = 0.5f * length(c);
    if (area <= 0.0f) return 0.0f;
    const float cl = fabsf(dot(normalize(c), -dir));
    if (cl <= 1e-5f) return 0.0f;
    return pmf * dist * dist / (area * cl);
}
__device__ __forceinline__ uint32_t sample_alias(const pt_alias_entry* t, uint32_t n, float u1, float u2) {
    uint32_t i = static_cast<uint32_t>(u1 * n);
    if (i >= n) i = n - 1;
    const float2 e = __ldg(reinterpret_cast<const float2*>(t + i));
    return (u2 < e.x) ? i : __float_as_uint(e.y);
}
// evaluateDirectLight (direct_lighting.cuh:204-218) without the visibility term.
// A guided vertex weighs its light samples exactly as the plain integrator
// does (power heuristic against the BSDF's pdf), so the light sample and the
// directional sample together keep the plain integrator's expectation.
__device__ __forceinline__ f3 direct_term(const MatEval& me, f3 wo, f3 wi, f3 n, f3 radiance, float light_pdf) {
    const BsdfEval b = PT_BSDF_EVAL(me, wo, wi, n, true);
    if (b.pdf <= 0.0f) return mk(0.0f);
    const float mis = power_heuristic(light_pdf, b.pdf);
    return radiance * b.f * (mis / (light_pdf + 1e-7f));
}

// Guiding inputs of one shaded vertex: its mixture (nullptr = plain BSDF
// sampling) and, while training, the record slot that receives
// (position, direction, pdf, throughput after the vertex).
struct GuideVertex {
    const float* mix;
    float4* rec;
    float alpha;
};

__device__ __forceinline__ void emit_shadow(const WaveParams& P, bool want, uint32_t path, uint32_t slot,
                                            f3 o, f3 d, float tmax, f3 c) {
    const uint32_t j = warp_append(P.counts + 2, want);
    if (!want) return;
    const uint32_t cap = static_cast<uint32_t>(P.npath) * static_cast<uint32_t>(P.n_slots);
    if (j >= cap) { atomicOr(P.err, kErrQueueOverflow); return; }
    P.sq_path[j] = path;
    P.sq_o[j] = make_float4(o.x, o.y, o.z, __uint_as_float(slot));
    P.sq_d[j] = make_float4(d.x, d.y, d.z, tmax);
    P.sq_c[j] = make_float4(c.x, c.y, c.z, 0.0f);
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------
__global__ void k_begin(PassState* ps, uint32_t frame) { ps->frame = frame; }

// Sampler for pixel (x, y), sample (frame, i) (kernelPathTrace, path.cu:217-225).
__device__ __forceinline__ PathRng make_rng(int type, int x, int y, uint32_t frame, uint32_t spf, uint32_t i,
                                            uint32_t user_seed) {
    PathRng rng;
    rng.type = type; rng.px = x; rng.py = y; rng.sample_index = frame * spf + i;
    rng.s = (type == PT_SAMPLER_SOBOL) ? 0u : pcg_seed(x, y, frame, i, user_seed);
    return rng;
}

// Camera ray for pixel (x, y): 2 jitter draws, +2 lens draws with aperture
// (emitRay, path.cu:31-59).  The direction is renormalised as Ray's
// constructor does (core/ray.h:13).
__device__ __forceinline__ void camera_ray(const pt_camera_frame& c, int width, int height, int x, int y,
                                           PathRng& rng, f3& pos, f3& dir) {
    const f3 fwd = ld3(c.forward), rgt = ld3(c.right), cup = ld3(c.up);
    const float jx = rng_next(rng);
    const float jy = rng_next(rng);
    const float u = (2.0f * (x + jx) / width - 1.0f) * c.tan_half_fov * c.aspect;
    const float v = (2.0f * (y + jy) / height - 1.0f) * c.tan_half_fov;
    pos = ld3(c.position);
    dir = normalize(u * rgt + v * cup + fwd);
    if (c.aperture > 0.0f) {
        const f3 focal = pos + dir * (c.focal_distance / dot(dir, fwd));
        const float lx = rng_next(rng);
        const float ly = rng_next(rng);
        const float r = sqrtf(lx) * c.aperture;
        const float th = kTwoPi * ly;
        pos = pos + rgt * (r * cosf(th)) + cup * (r * sinf(th));
        dir = normalize(focal - pos);
    }
    dir = normalize(dir);
}

// Paths of one pass: for every pixel the samples s0 .. s0+count-1 counted
// from the first sample of frame P.pass->frame (so a pass may span frames);
// path p = lane * npix + pixel takes sample s0 + lane.
__global__ void __launch_bounds__(256) k_raygen(WaveParams P, int s0, int count) {
    const int n = P.npix * count;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.counts[0] = static_cast<uint32_t>(n);
        P.counts[1] = 0;
        P.counts[2] = 0;
        atomicAdd(P.stats + kStatPaths, static_cast<unsigned long long>(n));
    }
    const uint32_t frame = P.pass->frame;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const int pix = p % P.npix, rel = s0 + p / P.npix;
        const int x = pix % P.width, y = pix / P.width;
        PathRng rng = make_rng(P.sampler_type, x, y, frame + static_cast<uint32_t>(rel / P.spf),
                               static_cast<uint32_t>(P.spf), static_cast<uint32_t>(rel % P.spf), P.pcg_seed);
        f3 pos, dir;
        camera_ray(P.cam, P.width, P.height, x, y, rng, pos, dir);
        P.queue[0][p] = static_cast<uint32_t>(p);
        P.ray_o[0][p] = f4of(pos, 1.0f);   // w: roulette throughput of the guided integrator
        P.ray_d[0][p] = f4of(dir, 0.0f);
        P.thr[p] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
        P.lo[p] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
        P.rng[p] = rng.s;
        for (int k = 0; k < P.n_slots; ++k) P.nee[static_cast<size_t>(k) * P.npath + p] = make_float4(0, 0, 0, 0);
    }
}

__device__ __forceinline__ void warp_count(unsigned long long* dst, uint32_t v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(__activemask(), v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, static_cast<unsigned long long>(v));
}

// Closest hits of queue q.  Packet: the queue holds camera rays, 32
// neighbouring pixels of one sample per warp, walked as packets
// (closest_packet_loop); else lane by lane with refill (closest_loop).
template <int Block, int Depth, bool Packet = false>
__global__ void __launch_bounds__(Block) k_extend(WaveParams P, int q, int depth) {
    const uint32_t n = min(P.counts[q], static_cast<uint32_t>(P.npath));
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.counts[q ^ 1] = 0;
        P.counts[2] = 0;
        P.counts[4] = 0;
        atomicAdd(P.stats + (depth == 0 ? kStatCameraRays : kStatExtRays), static_cast<unsigned long long>(n));
    }
    const bool watertight = (P.flags & PT_FLAG_WATERTIGHT) != 0;
    const bool count = (P.flags & PT_FLAG_COUNT_TRAVERSAL) != 0;
    uint32_t err = 0;
    TraceCounters tc{0, 0};
    const uint32_t stride = gridDim.x * blockDim.x;
    const float4* __restrict__ ro = P.ray_o[q];
    const float4* __restrict__ rd = P.ray_d[q];
    float4* __restrict__ hit = P.hit;
    auto fetch = [&](uint32_t i, RayInv& r) {
        const float4 o = ro[i];
        const float4 d = rd[i];
        r = make_ray_inv(o.x, o.y, o.z, d.x, d.y, d.z);
    };
    auto done = [&](uint32_t i, const ClosestWalk& w) {
        hit[i] = w.prim >= 0 ? make_float4(w.best, __int_as_float(w.prim), w.bu, w.bv)
                             : make_float4(FLT_MAX, __int_as_float(-1), 0.0f, 0.0f);
    };
    if (Packet) {
        closest_packet_loop<Depth>(P.scene, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, stride >> 5, n, watertight,
                                   err, tc, fetch, done);
    } else {
        closest_loop<Depth>(P.scene, blockIdx.x * blockDim.x + threadIdx.x, n, stride, watertight, err, tc, fetch,
                            done);
    }
    if (err) atomicOr(P.err, err);
    if (count) {
        warp_count(P.stats + kStatNodes, tc.inner);
        warp_count(P.stats + kStatTris, tc.tris);
    }
}

// Shadow-ray sinks for shade_path: the wavefront queues a shadow ray per light
// slot; the persistent (batched) kernel traces it on the spot.
struct QueueSink {
    const WaveParams& P;
    uint32_t path;
    __device__ __forceinline__ void emit(bool want, uint32_t slot, f3 o, f3 d, float tmax, f3 c) {
        emit_shadow(P, want, path, slot, o, d, tmax, c);
    }
};

struct InlineSink {
    const DeviceScene& s;
    bool watertight;
    f3 acc;
    uint32_t err;
    uint32_t rays;
    TraceCounters tc;
    __device__ __forceinline__ void emit(bool want, uint32_t, f3 o, f3 d, float tmax, f3 c) {
        if (!want) return;
        ++rays;
        const RayInv r = make_ray_inv(o.x, o.y, o.z, d.x, d.y, d.z);
        if (!trace_any(s, r, tmax, watertight, err, tc)) acc += c;
    }
};

// The shading point a bounce continues from.
struct ShadePoint {
    f3 hp, gn, N;        // N: the shading normal (gn unless a normal map bends it)
    bool entering;
    MatEval me;
    const float* gmix;   // guided vertex: its mixture, else nullptr
};

// First half of one bounce of pathTrace (path.cu:69-185): environment or
// emitter hit (the path ends), alpha pass-through, next-event estimation.
// Returns 0 when the path ends here, 1 when it continues by sampling at `sp`
// (shade_back), 2 when it continues straight through with ray (no, nd).
template <bool Guided, class Sink, bool Textured = false>
__device__ int shade_front(const DeviceScene& s, int arg_rtl, int depth, f3 ro, f3 rd, float4 h, const f3& T,
                           float last_pdf, bool last_delta, f3& L, PathRng& rng, f3& no, f3& nd, Sink& sink,
                           GuideVertex gv, ShadePoint& sp) {
    const int prim = __float_as_int(h.y);
    if (prim < 0) {
        const f3 env = env_radiance(s, rd);
        if (!is_zero(env)) {
            float w = 1.0f;
            if (depth > 0 && !last_delta) w = power_heuristic(last_pdf, env_pdf(s, rd));
            L += T * env * w;
        }
        return 0;
    }
    const float t = h.x, bu = h.z, bv = h.w;
    const pt_face f = load_face(s, static_cast<uint32_t>(prim));
    const pt_material& m = s.materials[f.material_id];
    f3 hp, gn, N;
    bool entering;
    SurfaceAt g;
    if (Textured) {
        hp = hit_point(ro, rd, t);
        surface_at<true>(s, f, m, bu, bv, rd, g);
        gn = g.gn;
        N = g.N;
        entering = g.entering;
    } else {
        hp = ro + t * rd;
        const float bw = 1.0f - bu - bv;
        const f3 n = normalize(bw * vnrm(s, f.v0) + bu * vnrm(s, f.v1) + bv * vnrm(s, f.v2));
        entering = dot(n, rd) < 0.0f;
        if (m.double_sided && !entering) { gn = -n; entering = true; }
        else gn = entering ? n : -n;
        N = gn;   // no normal map without textures
    }
    const f3 wo = -rd;
    if (material_emits(m)) {
        float w = 1.0f;
        if (depth > 0 && !last_delta) w = power_heuristic(last_pdf, emissive_pdf(s, prim, t, rd));
        L += T * material_emission(m) * w;
        return 0;
    }
    // alpha (path.cu:136-158): MASK alpha is the base colour texture's alpha
    // (else 1), BLEND alpha is baseAlpha times it; both looked up at the
    // surface's own uv, without the material's uv transform, as the reference does
    if (m.alpha_mode == 1) {
        float alpha = 1.0f;
        if (Textured && tex_live(s, m.base_color_tex)) alpha = tex_at(s, m.base_color_tex, g.su, g.sv).w;
        if (alpha < m.alpha_cutoff) { no = hp + rd * 1e-4f; nd = normalize(rd); return 2; }
    } else if (m.alpha_mode == 2) {
        float alpha = m.base_alpha;
        if (Textured && tex_live(s, m.base_color_tex)) alpha *= tex_at(s, m.base_color_tex, g.su, g.sv).w;
        if (rng_next(rng) >= alpha) { no = hp + rd * 1e-4f; nd = normalize(rd); return 2; }
    }
    const MatEval me = Textured ? resolve_material_textured(s, m, g.tu, g.tv) : resolve_material(m);
    const bool delta_surface = (me.metallic >= 1.0f && me.roughness < 0.01f) ||
                               (me.spec_trans >= 1.0f && me.roughness < 0.01f);
    // guided vertex: a mixture is available and no lobe can be a delta
    const float* gmix = (Guided && gv.mix != nullptr && me.roughness >= 0.01f) ? gv.mix : nullptr;
    if (!delta_surface) {
        const bool has_area = s.num_emissive > 0 && s.emissive != nullptr;
        const bool has_env = has_env_light(s);
        // area light sample (sampleAreaLight, direct_lighting.cuh:75-121)
        if (has_area) {
            float u1, u2;
            rng_pair(rng, arg_rtl, u1, u2);
            const uint32_t li = sample_alias(s.tri_alias, s.num_emissive, u1, u2);
            const uint32_t tri = __ldg(&s.emissive[li].triangle_index);
            const float pmf = __ldg(&s.emissive[li].selection_pmf);
            const pt_face lf = load_face(s, tri);
            const float tu = rng_next(rng);
            const float tv = rng_next(rng);
            const f3 p0 = vpos(s, lf.v0), p1 = vpos(s, lf.v1), p2 = vpos(s, lf.v2);
            const float su0 = sqrtf(tu);
            const float b0 = 1.0f - su0, b1 = tv * su0, b2 = 1.0f - b0 - b1;
            const f3 lp = p0 * b0 + p1 * b1 + p2 * b2;
            f3 ln = normalize(vnrm(s, lf.v0) * b0 + vnrm(s, lf.v1) * b1 + vnrm(s, lf.v2) * b2);
            if (length(ln) == 0.0f) ln = normalize(cross(p1 - p0, p2 - p0));
            const f3 to = lp - hp;
            const float d2 = dot(to, to);
            bool ok = d2 > 1e-8f;
            float dist = 0.0f, pdf = 0.0f;
            f3 wi = mk(0.0f), contrib = mk(0.0f);
            if (ok) {
                dist = sqrtf(d2);
                wi = to / dist;
                ok = fmaxf(0.0f, dot(N, wi)) > 0.0f;
            }
            if (ok) {
                const float area = 0.5f * length(cross(p1 - p0, p2 - p0));
                const float cl = fabsf(dot(ln, -wi));
                ok = area > 0.0f && cl > 1e-5f;
                if (ok) {
                    pdf = (pmf / area) * d2 / cl;
                    ok = pdf > 0.0f;
                }
            }
            if (ok) {
                const f3 le = material_emission(s.materials[lf.material_id]);
                contrib = T * direct_term(me, wo, wi, N, le, pdf);
                ok = !is_zero(contrib);
            }
            const float sg = dot(wi, N) >= 0.0f ? 1.0f : -1.0f;
            sink.emit(ok, 0, hp + N * (1e-4f * sg), normalize(wi), dist - 1e-3f, contrib);
        }
        // environment sample (sampleEnvironmentLight, direct_lighting.cuh:123-154)
        if (has_env) {
            float u1, u2;
            rng_pair(rng, arg_rtl, u1, u2);
            const uint32_t texel = sample_alias(s.env_alias, s.num_env_texels, u1, u2);
            const int x = static_cast<int>(texel % static_cast<uint32_t>(s.env_w));
            const int y = static_cast<int>(texel / static_cast<uint32_t>(s.env_w));
            float j1, j2;
            rng_pair(rng, arg_rtl, j1, j2);
            const float uu = (static_cast<float>(x) + j1) / static_cast<float>(s.env_w);
            const float vv = (static_cast<float>(y) + j2) / static_cast<float>(s.env_h);
            const f3 wi = dir_from_uv(uu, vv);
            bool ok = fmaxf(0.0f, dot(N, wi)) > 0.0f;
            float pdf = 0.0f;
            f3 contrib = mk(0.0f);
            if (ok) { pdf = env_pdf(s, wi); ok = pdf > 0.0f; }
            if (ok) {
                contrib = T * direct_term(me, wo, wi, N, env_radiance(s, wi), pdf);
                ok = !is_zero(contrib);
            }
            const float sg = dot(wi, N) >= 0.0f ? 1.0f : -1.0f;
            sink.emit(ok, 1, hp + N * (1e-4f * sg), normalize(wi), FLT_MAX, contrib);
        }
        // punctual lights, no MIS (evaluatePunctualLights, direct_lighting.cuh:158-200)
        for (uint32_t j = 0; j < s.num_punctual; ++j) {
            const pt_punctual_light& pl = s.punctual[j];
            f3 wi;
            float dist = FLT_MAX;
            f3 inten;
            bool ok = true;
            if (pl.type == 0 || pl.type == 2) {
                const f3 to = ld3(pl.position) - hp;
                const float d2 = dot(to, to);
                ok = !(d2 < 1e-8f);
                dist = sqrtf(d2);
                wi = to / dist;
                float att = dist >= pl.range ? 0.0f : 1.0f / (dist * dist + 1e-7f);
                if (pl.type == 2) {
                    const float ca = dot(normalize(-to), ld3(pl.direction));
                    float sa;
                    if (ca < pl.outer_cone) sa = 0.0f;
                    else if (ca > pl.inner_cone) sa = 1.0f;
                    else { const float tt = (ca - pl.outer_cone) / (pl.inner_cone - pl.outer_cone + 1e-7f); sa = tt * tt; }
                    att *= sa;
                }
                inten = ld3(pl.color) * (pl.intensity * att);
            } else {
                wi = -ld3(pl.direction);
                inten = ld3(pl.color) * pl.intensity;
            }
            f3 contrib = mk(0.0f);
            if (ok) ok = dot(N, wi) > 0.0f;
            if (ok) {
                contrib = T * (inten * PT_BSDF_EVAL(me, wo, wi, N, true).f);
                ok = !is_zero(contrib);
            }
            const float sg = dot(wi, N) >= 0.0f ? 1.0f : -1.0f;
            const float tmax = dist < FLT_MAX ? dist - 1e-3f : FLT_MAX;
            sink.emit(ok, 2 + j, hp + N * (1e-4f * sg), normalize(wi), tmax, contrib);
        }
    }
    sp.hp = hp;
    sp.gn = gn;
    sp.N = N;
    sp.entering = entering;
    sp.me = me;
    sp.gmix = gmix;
    return 1;
}

// Second half of one bounce (path.cu:186-199): BSDF (or guide/BSDF mixture)
// sampling, throughput, Russian roulette.  Returns true when the path
// continues with ray (no, nd).
template <bool Guided>
__device__ bool shade_back(int arg_rtl, int depth, f3 rd, const ShadePoint& sp, f3& T, float& last_pdf,
                           bool& last_delta, PathRng& rng, f3& no, f3& nd, GuideVertex gv, float* rr_w) {
    const MatEval& me = sp.me;
    const f3 hp = sp.hp, gn = sp.gn, N = sp.N, wo = -rd;
    const bool entering = sp.entering;
    const float* gmix = Guided ? sp.gmix : nullptr;
    BsdfSample bs;
    float plain_w = 0.0f;   // guided: max3(f cos / p_bsdf) of this vertex, for the roulette
    float mix_p = 0.0f;     // guided: the density the direction was drawn with (training records)
    if (Guided && gmix) {
        // One-sample MIS between the learned mixture q and the BSDF's own
        // sampler (density pB): the direction comes from q with probability
        // alpha, else from the BSDF, and the plain integrator's weight f / pdf
        // is scaled by pB / (alpha q + (1 - alpha) pB).  Its expectation is
        // the plain integrator's, including where the reference's pdf is not
        // the sampler's density (disney_sample_density).  bs.pdf stays the
        // BSDF's pdf, for the emitter hit's power heuristic.
        // Either branch only picks the direction; the BSDF is then evaluated
        // once for the whole warp (a lane that drew from q and one that drew
        // from the BSDF would otherwise each run an evaluation in turn).  No
        // guided vertex has a delta lobe, so both weights are f / pdf.
        const float sel = rng_next(rng);
        const bool from_q = sel < gv.alpha;
        bool have_dir;
        bool delta = false;
        if (from_q) {
            const float u0 = rng_next(rng), u1 = rng_next(rng), u2 = rng_next(rng);
            bs.wi = mix_sample(gmix, u0, u1, u2);
            have_dir = true;
        } else {
            have_dir = disney_sample_dir(me, wo, N, rng, arg_rtl, entering, bs.wi, delta);
        }
        bs.valid = false;
        bs.delta = false;
        if (have_dir) {
            const BsdfEval ev = PT_BSDF_EVAL(me, wo, bs.wi, N, entering);
            bs.pdf = ev.pdf;
            bs.valid = ev.pdf > 0.0f && (!from_q || !is_zero(ev.f));
            bs.weight = ev.f / (ev.pdf + 1e-7f);   // the plain integrator's weight
        }
        if (bs.valid) {
            const float pB = disney_sample_density(me, wo, bs.wi, N, bs.pdf);
            mix_p = gv.alpha * mix_pdf(gmix, bs.wi) + (1.0f - gv.alpha) * pB;
            bs.valid = mix_p > 0.0f && pB > 0.0f;
            plain_w = max3(bs.weight);
            bs.weight = bs.weight * (pB / fmaxf(mix_p, 1e-30f));
        }
    } else {
        bs = PT_BSDF_SAMPLE(me, wo, N, rng, arg_rtl, entering);
        plain_w = max3(bs.weight);
    }
    if (!bs.valid) return false;
    T *= bs.weight;
    if (Guided && rr_w) *rr_w *= plain_w;
    const bool transmitted = dot(bs.wi, gn) < 0.0f;
    const f3 off = transmitted ? -gn : gn;
    no = hp + off * 1e-4f;
    nd = normalize(bs.wi);
    if (transmitted && me.thickness > 0.0f && me.att_distance < 1e20f) {
        const float th = me.thickness, ad = me.att_distance;
        const f3 ac = me.att_color;
        const f3 tr = mk(expf(-th * fmaxf(-logf(fmaxf(ac.x, 1e-6f)), 0.0f) / ad),
                         expf(-th * fmaxf(-logf(fmaxf(ac.y, 1e-6f)), 0.0f) / ad),
                         expf(-th * fmaxf(-logf(fmaxf(ac.z, 1e-6f)), 0.0f) / ad));
        T *= tr;
        if (Guided && rr_w) *rr_w *= max3(tr);
    }
    last_pdf = bs.pdf;
    last_delta = bs.delta;
    if (depth > 2) {
        // Russian roulette (path.cu:193-196).  A guided path decides on the
        // throughput it would have had under BSDF sampling: its own throughput
        // is small exactly where the guide sent it towards bright light, and
        // rouletting on it would end the paths the guide is there to find.
        const float surv = fminf((Guided && rr_w) ? *rr_w : max3(T), 0.95f);
        if (rng_next(rng) >= surv) return false;
        T = T / surv;
        if (Guided && rr_w) *rr_w /= surv;
    }
    if (Guided && gv.rec && !bs.delta) {
        // training record: where, which way, with which pdf, the throughput
        // that scales everything found along this direction, |cos| to the normal
        gv.rec[0] = make_float4(hp.x, hp.y, hp.z, mix_p);
        gv.rec[1] = make_float4(nd.x, nd.y, nd.z, 1.0f);
        gv.rec[2] = make_float4(T.x, T.y, T.z, fabsf(dot(N, nd)));
    }
    return true;
}

// One bounce of pathTrace (path.cu:69-199).  Returns true when the path
// continues with ray (no, nd).  Shadow rays go to `sink`.  Guided = false
// compiles the plain integrator without any of the guiding code.
template <bool Guided, class Sink>
__device__ bool shade_path(const DeviceScene& s, int arg_rtl, int depth, bool last, f3 ro, f3 rd, float4 h,
                           f3& T, float& last_pdf, bool& last_delta, f3& L, PathRng& rng, f3& no, f3& nd,
                           Sink& sink, GuideVertex gv = GuideVertex{nullptr, nullptr}, float* rr_w = nullptr) {
    ShadePoint sp;
    const int r = shade_front<Guided>(s, arg_rtl, depth, ro, rd, h, T, last_pdf, last_delta, L, rng, no, nd, sink,
                                      gv, sp);
    if (r != 1) return r == 2;
    if (last) return false;   // the sampled continuation would never be traced
    return shade_back<Guided>(arg_rtl, depth, rd, sp, T, last_pdf, last_delta, rng, no, nd, gv, rr_w);
}

// Sampler state of path p in pass-relative sample s0.
__device__ __forceinline__ PathRng path_rng(const WaveParams& P, uint32_t p, uint32_t sidx0) {
    PathRng rng;
    rng.type = P.sampler_type;
    const uint32_t pix = p % static_cast<uint32_t>(P.npix);
    rng.px = static_cast<int>(pix % static_cast<uint32_t>(P.width));
    rng.py = static_cast<int>(pix / static_cast<uint32_t>(P.width));
    rng.sample_index = sidx0 + p / static_cast<uint32_t>(P.npix);
    rng.s = P.rng[p];
    return rng;
}

// Appends path p's continuation (no, nd) to the next queue.
__device__ __forceinline__ void push_continuation(const WaveParams& P, int q, bool cont, uint32_t p, f3 no, f3 nd,
                                                  float rr_w) {
    const uint32_t cap = static_cast<uint32_t>(P.npath);
    const uint32_t j = warp_append(P.counts + (q ^ 1), cont);
    if (!cont) return;
    if (j < cap) {
        P.queue[q ^ 1][j] = p;
        P.ray_o[q ^ 1][j] = f4of(no, rr_w);
        P.ray_d[q ^ 1][j] = f4of(nd, 0.0f);
    } else {
        atomicOr(P.err, kErrQueueOverflow);
    }
}

// Shading is two kernels per bounce: k_shade_front (hit, emission, NEE) and
// k_shade_back (BSDF sampling, roulette, the next ray).  Each is about half
// the code of one shading kernel, so divergent warps miss the instruction
// cache less (on the 1080p bench render: shading 325 -> 243 ms); the front
// hands the shading point to the back in the queue entry's own slots:
// hit[i] = (point, prim | entering << 30, or -1 when the path needs no
// sampling), ray_o[q][i] = (geometric normal, roulette weight).  Both run 6
// blocks of 128 per SM (80 registers): 224 ms against 243 ms at 5 blocks.
constexpr uint32_t kEnteringBit = 0x40000000u;

template <bool Guided, bool Textured = false>
__global__ void __launch_bounds__(128, 6) k_shade_front(WaveParams P, int q, int depth, int s0) {
    const uint32_t cap = static_cast<uint32_t>(P.npath);
    const uint32_t n = min(P.counts[q], cap);
    const uint32_t sidx0 = P.pass->frame * static_cast<uint32_t>(P.spf) + static_cast<uint32_t>(s0);
    const bool last = depth == P.max_depth - 1;
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t p = P.queue[q][i];
        if (p >= cap) { atomicOr(P.err, kErrQueueOverflow); continue; }
        const float4 o4 = P.ray_o[q][i];
        const float4 d4 = P.ray_d[q][i];
        const float4 h = P.hit[i];
        const float4 thr = P.thr[p];
        const float4 lo = P.lo[p];
        const f3 T = f3of(thr);
        f3 L = f3of(lo);
        PathRng rng = path_rng(P, p, sidx0);
        f3 no = mk(0.0f), nd = mk(0.0f);
        QueueSink sink{P, p};
        GuideVertex gv{Guided && P.gmix ? P.gmix + static_cast<size_t>(i) * kGMix : nullptr, nullptr, P.galpha};
        if (Guided && P.grec) {
            float4* rec = P.grec + (static_cast<size_t>(depth) * P.npath + p) * 4;
            rec[1].w = 0.0f;
            if (depth > 0) {
                // radiance gathered through the previous vertex: the part of the
                // final estimate that did not arrive along its sampled direction
                float4* prev = P.grec + (static_cast<size_t>(depth - 1) * P.npath + p) * 4;
                if (prev[1].w != 0.0f) {
                    f3 S = L;
                    for (int k = 0; k < P.n_slots; ++k) S += f3of(P.nee[static_cast<size_t>(k) * P.npath + p]);
                    prev[3] = f4of(S, 0.0f);
                }
            }
        }
        ShadePoint sp;
        const int r = shade_front<Guided, QueueSink, Textured>(P.scene, P.arg_rtl, depth, f3of(o4), f3of(d4), h, T,
                                                               thr.w, lo.w != 0.0f, L, rng, no, nd, sink, gv, sp);
        P.lo[p] = f4of(L, lo.w);
        P.rng[p] = rng.s;
        // the back kernel takes only the entries that continue by sampling, so
        // its warps start full
        const bool samp = r == 1 && !last;
        const uint32_t js = warp_append(P.counts + 4, samp);
        if (samp) P.slist[js] = i;
        if (Textured) {
            // the back kernel recomputes the surface from the untouched hit and
            // ray; a negative primitive tells it that this path needs no sampling
            if (!(r == 1 && !last)) P.hit[i].y = __int_as_float(-1);
        } else if (r == 1 && !last) {
            const uint32_t prim = static_cast<uint32_t>(__float_as_int(h.y));
            P.hit[i] = make_float4(sp.hp.x, sp.hp.y, sp.hp.z, __uint_as_float(prim | (sp.entering ? kEnteringBit : 0u)));
            P.ray_o[q][i] = make_float4(sp.gn.x, sp.gn.y, sp.gn.z, o4.w);
        } else {
            P.hit[i].w = __int_as_float(-1);
        }
        push_continuation(P, q, r == 2 && !last, p, no, nd, Guided ? o4.w : 1.0f);
    }
}

template <bool Guided, bool Textured = false>
__global__ void __launch_bounds__(128, 6) k_shade_back(WaveParams P, int q, int depth, int s0) {
    const uint32_t cap = static_cast<uint32_t>(P.npath);
    const uint32_t n = min(P.counts[4], cap);
    const uint32_t sidx0 = P.pass->frame * static_cast<uint32_t>(P.spf) + static_cast<uint32_t>(s0);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += stride) {
        const uint32_t i = P.slist[j];
        const float4 h = P.hit[i];
        const int code = Textured ? __float_as_int(h.y) : __float_as_int(h.w);
        bool cont = false;
        uint32_t p = 0;
        f3 no = mk(0.0f), nd = mk(0.0f);
        float rr_w = 1.0f;
        if (code >= 0) {
            p = P.queue[q][i];
            const float4 o4 = P.ray_o[q][i];
            const float4 d4 = P.ray_d[q][i];
            const float4 thr = P.thr[p];
            const float4 lo = P.lo[p];
            f3 T = f3of(thr);
            float last_pdf = thr.w;
            bool last_delta = lo.w != 0.0f;
            PathRng rng = path_rng(P, p, sidx0);
            ShadePoint sp;
            if (Textured) {
                const pt_face f = load_face(P.scene, static_cast<uint32_t>(code));
                const pt_material& m = P.scene.materials[f.material_id];
                SurfaceAt g;
                surface_at<true>(P.scene, f, m, h.z, h.w, f3of(d4), g);
                sp.hp = hit_point(f3of(o4), f3of(d4), h.x);
                sp.gn = g.gn;
                sp.N = g.N;
                sp.entering = g.entering;
                sp.me = resolve_material_textured(P.scene, m, g.tu, g.tv);
            } else {
                sp.hp = mk(h.x, h.y, h.z);
                sp.gn = f3of(o4);
                sp.N = sp.gn;
                sp.entering = (static_cast<uint32_t>(code) & kEnteringBit) != 0u;
                const pt_face f = load_face(P.scene, static_cast<uint32_t>(code) & ~kEnteringBit);
                sp.me = resolve_material(P.scene.materials[f.material_id]);
            }
            sp.gmix = (Guided && P.gmix && sp.me.roughness >= 0.01f) ? P.gmix + static_cast<size_t>(i) * kGMix
                                                                     : nullptr;
            GuideVertex gv{sp.gmix, nullptr, P.galpha};
            if (Guided && P.grec) gv.rec = P.grec + (static_cast<size_t>(depth) * P.npath + p) * 4;
            rr_w = Guided ? o4.w : 1.0f;
            cont = shade_back<Guided>(P.arg_rtl, depth, f3of(d4), sp, T, last_pdf, last_delta, rng, no, nd, gv,
                                      &rr_w);
            P.thr[p] = f4of(T, last_pdf);
            P.lo[p] = make_float4(lo.x, lo.y, lo.z, last_delta ? 1.0f : 0.0f);
            P.rng[p] = rng.s;
        }
        push_continuation(P, q, cont, p, no, nd, Guided ? rr_w : 1.0f);
    }
}

// Any-hit tests of the shadow queue.  Packet: the queue holds the shadow rays
// of the camera bounce, emitted warp by warp from neighbouring pixels, tested
// as packets where a tile's directions share their signs (any_packet_loop).
template <int Block, int Depth, bool Packet = false>
__global__ void __launch_bounds__(Block) k_shadow(WaveParams P) {
    const uint32_t n = min(P.counts[2], static_cast<uint32_t>(P.npath) * static_cast<uint32_t>(P.n_slots));
    if (blockIdx.x == 0 && threadIdx.x == 0)
        atomicAdd(P.stats + kStatShadowRays, static_cast<unsigned long long>(n));
    const bool watertight = (P.flags & PT_FLAG_WATERTIGHT) != 0;
    const bool count = (P.flags & PT_FLAG_COUNT_TRAVERSAL) != 0;
    uint32_t err = 0;
    TraceCounters tc{0, 0};
    const uint32_t stride = gridDim.x * blockDim.x;
    auto fetch = [&](uint32_t i, AnyWalk& w) {
        const float4 o = P.sq_o[i];
        const float4 d = P.sq_d[i];
        w.r = make_ray_inv(o.x, o.y, o.z, d.x, d.y, d.z);
        w.tmax = d.w;
    };
    auto done = [&](uint32_t i, bool occluded) {
        if (occluded) return;
        const uint32_t slot = __float_as_uint(P.sq_o[i].w);
        const uint32_t path = P.sq_path[i];
        if (slot < static_cast<uint32_t>(P.n_slots) && path < static_cast<uint32_t>(P.npath)) {
            float4* acc = P.nee + static_cast<size_t>(slot) * P.npath + path;
            const float4 c = P.sq_c[i];
            float4 a = *acc;
            a.x += c.x; a.y += c.y; a.z += c.z;
            *acc = a;
        } else {
            err |= kErrQueueOverflow;
        }
    };
    if (Packet)
        any_packet_loop<Depth>(P.scene, (blockIdx.x * blockDim.x + threadIdx.x) >> 5, stride >> 5, n, watertight, err,
                               tc, fetch, done);
    else
        any_loop<Depth>(P.scene, blockIdx.x * blockDim.x + threadIdx.x, n, stride, watertight, err, tc, fetch, done);
    if (err) atomicOr(P.err, err);
    if (count) {
        warp_count(P.stats + kStatShadowNodes, tc.inner);
        warp_count(P.stats + kStatShadowTris, tc.tris);
    }
}

__device__ __forceinline__ void neumaier(float& s, float& c, float x) {
    const float t = s + x;
    if (fabsf(s) >= fabsf(x)) c += (s - t) + x;
    else c += (x - t) + s;
    s = t;
}

// Adds the pass's samples to the film, per pixel in sample order (the order
// of one-sample-per-pass rendering, so the sums do not depend on the lanes);
// a completed frame's mean becomes the "new" image (the reference's surfNew).
__global__ void __launch_bounds__(256) k_finalize(WaveParams P, int s0, int count) {
    const float spf = static_cast<float>(P.spf);
    for (int pix = blockIdx.x * blockDim.x + threadIdx.x; pix < P.npix; pix += gridDim.x * blockDim.x) {
        float4 s = P.f_sum[pix], c = P.f_comp[pix], b = P.f_batch[pix];
        for (int lane = 0; lane < count; ++lane) {
            const int p = lane * P.npix + pix;
            f3 L = f3of(P.lo[p]);
            for (int k = 0; k < P.n_slots; ++k) L += f3of(P.nee[static_cast<size_t>(k) * P.npath + p]);
            // per-sample firefly clamp (path.cu:201-204); fminf maps NaN to the clamp value as the reference does
            L = mk(fminf(L.x, 100.0f), fminf(L.y, 100.0f), fminf(L.z, 100.0f));
            neumaier(s.x, c.x, L.x);
            neumaier(s.y, c.y, L.y);
            neumaier(s.z, c.z, L.z);
            s.w += 1.0f;
            b.x += L.x; b.y += L.y; b.z += L.z;
            if ((s0 + lane) % P.spf == P.spf - 1) {
                P.f_new[pix] = make_float4(b.x / spf, b.y / spf, b.z / spf, 1.0f);
                b = make_float4(0, 0, 0, 0);
            }
        }
        P.f_sum[pix] = s;
        P.f_comp[pix] = c;
        P.f_batch[pix] = b;
    }
}

// Turn this pass's guide records into training samples: for each recorded
// vertex, the incident radiance along its sampled direction is the part of the
// path's final estimate gathered after it, divided by the throughput after it
// (luminance, clamped like a sample); weight = L_in |cos| / p, so the guide
// learns the cosine-weighted incident radiance.  The samples are stored in
// path order, each path's in depth order (k_guide_count, an exclusive scan of
// the counts, k_guide_collect), so the minibatches -- and with them the
// trained network -- are the same on every run.  Records are cleared.
__device__ __forceinline__ float guide_record_weight(const WaveParams& P, int p, int d, f3 Lf, float4& r0,
                                                    float4& r1) {
    const float4* r = P.grec + (static_cast<size_t>(d) * P.npath + p) * 4;
    r1 = r[1];
    r0 = make_float4(0, 0, 0, 0);
    if (r1.w == 0.0f) return 0.0f;
    r0 = r[0];
    const f3 Ta = f3of(r[2]);
    const f3 S = f3of(r[3]);
    const f3 Lin = mk(Ta.x > 0.0f ? (Lf.x - S.x) / Ta.x : 0.0f, Ta.y > 0.0f ? (Lf.y - S.y) / Ta.y : 0.0f,
                      Ta.z > 0.0f ? (Lf.z - S.z) / Ta.z : 0.0f);
    const float lum = fminf(fmaxf(luminance(Lin), 0.0f), 100.0f) * r[2].w;
    float w = r0.w > 0.0f ? lum / r0.w : 0.0f;
    if (!(w < 1e30f)) w = 0.0f;
    return w;
}

__device__ __forceinline__ f3 guide_path_estimate(const WaveParams& P, int p) {
    f3 Lf = f3of(P.lo[p]);
    for (int k = 0; k < P.n_slots; ++k) Lf += f3of(P.nee[static_cast<size_t>(k) * P.npath + p]);
    return Lf;
}

// counts[p] = training samples of path p; counts[npaths] = 0 (the scan's total).
__global__ void __launch_bounds__(256) k_guide_count(WaveParams P, int npaths, uint32_t* counts) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p <= npaths; p += gridDim.x * blockDim.x) {
        uint32_t k = 0;
        if (p < npaths) {
            const f3 Lf = guide_path_estimate(P, p);
            for (int d = 0; d + 1 < P.max_depth; ++d) {
                float4 r0, r1;
                k += guide_record_weight(P, p, d, Lf, r0, r1) > 0.0f ? 1u : 0u;
            }
        }
        counts[p] = k;
    }
}

__global__ void __launch_bounds__(256) k_guide_collect(WaveParams P, int npaths, GuideNet net, GuideSample* out,
                                                       const uint32_t* offsets, uint32_t* count, uint32_t cap) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = offsets[npaths];
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npaths; p += gridDim.x * blockDim.x) {
        const f3 Lf = guide_path_estimate(P, p);
        uint32_t j = offsets[p];
        for (int d = 0; d + 1 < P.max_depth; ++d) {
            float4 r0, r1;
            const float w = guide_record_weight(P, p, d, Lf, r0, r1);
            if (r1.w != 0.0f) P.grec[(static_cast<size_t>(d) * P.npath + p) * 4 + 1].w = 0.0f;
            if (w > 0.0f) {
                if (j < cap) {
                    const f3 x = guide_normalise(net, mk(r0.x, r0.y, r0.z));
                    out[j] = GuideSample{make_float4(x.x, x.y, x.z, w), make_float4(r1.x, r1.y, r1.z, 0.0f)};
                }
                ++j;
            }
        }
    }
}

__global__ void k_film_mean(const float4* sum, const float4* comp, float4* out, int n) {
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        const float4 s = sum[p], c = comp[p];
        if (s.w > 0.0f) out[p] = make_float4((s.x + c.x) / s.w, (s.y + c.y) / s.w, (s.z + c.z) / s.w, 1.0f);
        else out[p] = make_float4(0, 0, 0, 0);
    }
}

// ---- diagnostics ----
__global__ void k_trace_rays(DeviceScene s, const float* rays, uint32_t n, pt_hit* hits, uint8_t* occl,
                             int any, int watertight, uint32_t* err_out) {
    // the warp-scheduled loops of the wavefront kernels
    uint32_t err = 0;
    TraceCounters tc{0, 0};
    const uint32_t first = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
    const float4* r4 = reinterpret_cast<const float4*>(rays);
    if (any) {
        any_loop(s, first, n, stride, watertight != 0, err, tc,
                 [&](uint32_t i, AnyWalk& w) {
                     const float4 o = r4[2 * i], d = r4[2 * i + 1];
                     w.r = make_ray_inv(o.x, o.y, o.z, d.x, d.y, d.z);
                     w.tmax = d.w;
                 },
                 [&](uint32_t i, bool occluded) { occl[i] = occluded ? 1 : 0; });
    } else {
        closest_loop(s, first, n, stride, watertight != 0, err, tc,
                     [&](uint32_t i, RayInv& r) {
                         const float4 o = r4[2 * i], d = r4[2 * i + 1];
                         r = make_ray_inv(o.x, o.y, o.z, d.x, d.y, d.z);
                     },
                     [&](uint32_t i, const ClosestWalk& w) {
                         pt_hit h;
                         h.prim = w.prim;
                         h.t = w.prim >= 0 ? w.best : FLT_MAX;
                         h.u = w.prim >= 0 ? w.bu : 0.0f;
                         h.v = w.prim >= 0 ? w.bv : 0.0f;
                         hits[i] = h;
                     });
    }
    if (err) atomicOr(err_out, err);
}

__global__ void k_sampler_stream(int type, int w, int h, uint32_t frame, int spf, int sif, uint32_t ndims,
                                 uint32_t seed, float* out) {
    const int npix = w * h;
    for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npix; p += gridDim.x * blockDim.x) {
        PathRng r;
        r.type = type; r.px = p % w; r.py = p / w;
        r.sample_index = frame * static_cast<uint32_t>(spf) + static_cast<uint32_t>(sif);
        r.s = type == PT_SAMPLER_SOBOL ? 0u : pcg_seed(r.px, r.py, frame, static_cast<uint32_t>(sif), seed);
        for (uint32_t k = 0; k < ndims; ++k) out[static_cast<size_t>(p) * ndims + k] = rng_next(r);
    }
}

__global__ void k_bsdf_eval(const pt_material* mats, uint32_t nmat, const float* in, uint32_t n, float* out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float* r = in + static_cast<size_t>(i) * 13;
        const uint32_t mi = static_cast<uint32_t>(r[0]);
        float* o = out + static_cast<size_t>(i) * 4;
        if (mi >= nmat) { o[0] = o[1] = o[2] = o[3] = 0.0f; continue; }
        const MatEval me = resolve_material(mats[mi]);
        const BsdfEval b = disney_eval(me, mk(r[1], r[2], r[3]), mk(r[4], r[5], r[6]), mk(r[7], r[8], r[9]), true);
        o[0] = b.f.x; o[1] = b.f.y; o[2] = b.f.z; o[3] = b.pdf;
    }
}

// The traversal kernels' shapes: 64, 128 or 256 threads per block and a
// stack of 32 or 64 entries (six instantiations of k_extend and k_shadow).
inline int trace_shape_index(int block, int depth) {
    return (block == 64 ? 0 : (block == 256 ? 2 : 1)) * 2 + (depth == 32 ? 0 : 1);
}
inline int trace_shape_block(int k) { return k < 2 ? 64 : (k < 4 ? 128 : 256); }
inline int trace_shape_depth(int k) { return (k & 1) ? 64 : 32; }

#define PT_TRACE_SHAPES(X) X(0, 64, 32) X(1, 64, 64) X(2, 128, 32) X(3, 128, 64) X(4, 256, 32) X(5, 256, 64)

inline const void* extend_kernel(int k) {
    switch (k) {
#define PT_CASE(i, b, d) case i: return reinterpret_cast<const void*>(k_extend<b, d>);
        PT_TRACE_SHAPES(PT_CASE)
#undef PT_CASE
    }
    return reinterpret_cast<const void*>(k_extend<128, 64>);
}
inline const void* shadow_kernel(int k) {
    switch (k) {
#define PT_CASE(i, b, d) case i: return reinterpret_cast<const void*>(k_shadow<b, d>);
        PT_TRACE_SHAPES(PT_CASE)
#undef PT_CASE
    }
    return reinterpret_cast<const void*>(k_shadow<128, 64>);
}
inline void launch_extend(int k, int grid, cudaStream_t st, const WaveParams& P, int q, int d) {
    switch (k) {
#define PT_CASE(i, b, dd)                                                   \
    case i:                                                                 \
        if (d == 0) k_extend<b, dd, true><<<grid, b, 0, st>>>(P, q, d);     \
        else k_extend<b, dd><<<grid, b, 0, st>>>(P, q, d);                  \
        return;
        PT_TRACE_SHAPES(PT_CASE)
#undef PT_CASE
    }
}
inline void launch_shadow(int k, int grid, cudaStream_t st, const WaveParams& P, int depth) {
    switch (k) {
#define PT_CASE(i, b, d)                                                    \
    case i:                                                                 \
        if (depth == 0) k_shadow<b, d, true><<<grid, b, 0, st>>>(P);        \
        else k_shadow<b, d><<<grid, b, 0, st>>>(P);                         \
        return;
        PT_TRACE_SHAPES(PT_CASE)
#undef PT_CASE
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
struct Wavefront {
    int device = -1;
    cudaStream_t own_stream = nullptr;
    int npath = 0, n_slots = 0;   // path slots the arena holds
    void* arena = nullptr;
    size_t arena_bytes = 0;
    WaveParams base{};
    // graph cache
    cudaGraphExec_t graph = nullptr;
    std::vector<unsigned char> graph_key;
    cudaStream_t graph_stream = nullptr;
    // launch shapes
    int sms = 0;
    int grid_raygen = 0, grid_shade = 0, grid_finalize = 0;
    int grid_extend[6] = {}, grid_shadow[6] = {};   // per traversal shape (trace_shape_index)
    // stats
    unsigned long long host_stats[kStatCount] = {};
    double stage_ms[5] = {0, 0, 0, 0, 0};   // extend, shade, shadow, other, guide
    GuideState* guide = nullptr;           // not owned
    double total_ms = 0.0;
    uint64_t extend_launches = 0;
    uint64_t kernel_launches = 0;
};

namespace {

template <typename T>
T* carve(char*& cur, size_t count) {
    const uintptr_t a = (reinterpret_cast<uintptr_t>(cur) + 255) & ~uintptr_t(255);
    T* p = reinterpret_cast<T*>(a);
    cur = reinterpret_cast<char*>(a + sizeof(T) * count);
    return p;
}

int ensure_device(int device) {
    int cur = -1;
    PT_CU(cudaGetDevice(&cur));
    if (cur != device) PT_CU(cudaSetDevice(device));
    return PT_OK;
}

int grid_for(const void* kernel, int block, int sms) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, block, 0) != cudaSuccess || per_sm < 1) per_sm = 1;
    return per_sm * sms;
}

// Size of the wavefront arena for npath path slots and n_slots light slots.
size_t arena_size(int npath, int n_slots) {
    const size_t P = static_cast<size_t>(npath);
    const size_t S = P * static_cast<size_t>(n_slots);
    size_t b = 0;
    b += 2 * (P * 4 + 256);          // queues
    b += 4 * (P * 16 + 256);         // ray_o/ray_d x2
    b += P * 16 + 256;               // hit
    b += 2 * (P * 16 + 256);         // thr, lo
    b += P * 4 + 256;                // rng
    b += S * 16 + 256;               // nee
    b += S * 4 + 256;                // sq_path
    b += 3 * (S * 16 + 256);         // sq_o, sq_d, sq_c
    b += 64 * 4 + 256;               // counts
    b += P * 4 + 256;                // slist
    b += kStatCount * 8 + 256;       // stats
    b += 4 * 4 + 256;                // err
    b += sizeof(PassState) + 256;
    return b;
}

int wavefront_prepare(Wavefront& wf, int device, int npath, int n_slots) {
    if (wf.device != device) {
        if (wf.arena) { cudaSetDevice(wf.device); cudaFree(wf.arena); wf.arena = nullptr; wf.arena_bytes = 0; }
        if (wf.graph) { cudaGraphExecDestroy(wf.graph); wf.graph = nullptr; wf.graph_key.clear(); }
        if (wf.own_stream) { cudaStreamDestroy(wf.own_stream); wf.own_stream = nullptr; }
        if (int rc = ensure_device(device)) return rc;
        PT_CU(cudaStreamCreateWithFlags(&wf.own_stream, cudaStreamNonBlocking));
        int sms = 0;
        PT_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
        wf.sms = sms;
        wf.grid_raygen = grid_for(reinterpret_cast<const void*>(k_raygen), 256, sms);
        wf.grid_shade = grid_for(reinterpret_cast<const void*>(k_shade_front<false>), 128, sms);
        for (int k = 0; k < 6; ++k) {
            wf.grid_extend[k] = grid_for(extend_kernel(k), trace_shape_block(k), sms);
            wf.grid_shadow[k] = grid_for(shadow_kernel(k), trace_shape_block(k), sms);
        }
        wf.grid_finalize = grid_for(reinterpret_cast<const void*>(k_finalize), 256, sms);
        wf.device = device;
        wf.npath = 0;
    } else if (int rc = ensure_device(device)) {
        return rc;
    }
    if (wf.npath == npath && wf.n_slots == n_slots && wf.arena) return PT_OK;
    std::memset(&wf.base, 0, sizeof(wf.base));
    const size_t need = arena_size(npath, n_slots);
    if (need > wf.arena_bytes) {
        if (wf.arena) { cudaFree(wf.arena); wf.arena = nullptr; wf.arena_bytes = 0; }
        if (cudaMalloc(&wf.arena, need) != cudaSuccess) {
            cudaGetLastError();
            set_error("cannot allocate " + std::to_string(need) + " bytes of wavefront state");
            return PT_ERR_NOMEM;
        }
        wf.arena_bytes = need;
    }
    char* cur = static_cast<char*>(wf.arena);
    WaveParams& b = wf.base;
    const size_t P = static_cast<size_t>(npath), S = P * static_cast<size_t>(n_slots);
    b.queue[0] = carve<uint32_t>(cur, P);
    b.queue[1] = carve<uint32_t>(cur, P);
    b.ray_o[0] = carve<float4>(cur, P);
    b.ray_d[0] = carve<float4>(cur, P);
    b.ray_o[1] = carve<float4>(cur, P);
    b.ray_d[1] = carve<float4>(cur, P);
    b.hit = carve<float4>(cur, P);
    b.thr = carve<float4>(cur, P);
    b.lo = carve<float4>(cur, P);
    b.rng = carve<uint32_t>(cur, P);
    b.nee = carve<float4>(cur, S);
    b.sq_path = carve<uint32_t>(cur, S);
    b.sq_o = carve<float4>(cur, S);
    b.sq_d = carve<float4>(cur, S);
    b.sq_c = carve<float4>(cur, S);
    b.counts = carve<uint32_t>(cur, 64);
    b.slist = carve<uint32_t>(cur, P);
    b.stats = carve<unsigned long long>(cur, kStatCount);
    b.err = carve<uint32_t>(cur, 4);
    b.pass = carve<PassState>(cur, 1);
    PT_CU(cudaMemset(b.counts, 0, 64 * 4));
    PT_CU(cudaMemset(b.stats, 0, kStatCount * 8));
    PT_CU(cudaMemset(b.err, 0, 16));
    PT_CU(cudaMemset(b.pass, 0, sizeof(PassState)));
    wf.npath = npath;
    wf.n_slots = n_slots;
    if (wf.graph) { cudaGraphExecDestroy(wf.graph); wf.graph = nullptr; wf.graph_key.clear(); }
    return PT_OK;
}

// Enqueue one batch (all sample passes) on `st`.  When `ev` is non-null,
// stage events are recorded (ev holds pairs per launch: kind, start, stop).
struct StageEvent { int kind; cudaEvent_t a, b; };

// Enqueues `total` samples per pixel, counted from the first sample of frame
// P.pass->frame, as passes of the wavefront's lanes.
// Guide inference over queue q (the hit points of its rays) into the guide's
// mixture buffer, by the guide's inference kind.
void launch_guide_infer(const GuideState& gs, const WaveParams& P, int q, int sms, cudaStream_t st) {
    const uint32_t cap = static_cast<uint32_t>(P.npath);
    GuideState g = gs;
    g.net = guide_infer_view(gs.net);
    if (g.infer == PT_GUIDE_INFER_FUSED) {
        k_guide_infer<<<sms * kGInferBlocksPerSm, 32 * kGInferWarps, kGInferSmem, st>>>(g.net, P.counts, q, cap,
                                                                                      P.ray_o[q], P.ray_d[q], P.hit,
                                                                                      g.mix);
        return;
    }
    if (g.net.quad) k_guide_quad<<<sms * 2, 256, 0, st>>>(g.net);
    k_guide_encode<<<sms * 8, 256, 0, st>>>(g.net, P.counts, q, cap, P.ray_o[q], P.ray_d[q], P.hit, nullptr, 0u,
                                            g.feat);
    if (g.infer == PT_GUIDE_INFER_SPLIT_MMA)
        k_guide_mlp_mma<<<sms * kGInferBlocksPerSm, 32 * kGInferWarps, kGInferSmem, st>>>(g.net, P.counts, q, cap, 0u,
                                                                                        g.feat, g.mix);
    else
        k_guide_mlp_tc<<<sms * kGTcBlocksPerSm, kGTcThreads, kGTcSmem, st>>>(g.net, P.counts, q, cap, 0u, g.feat,
                                                                             g.mix, P.err);
}

int enqueue_batch(Wavefront& wf, const WaveParams& P, int64_t total_samples, cudaStream_t st,
                  std::vector<StageEvent>* ev, GuideState* gs = nullptr) {
    const bool infer = gs && gs->mode != 0 && P.gmix;
    const bool train = infer && P.grec;
    auto timed = [&](int kind, auto&& launch) -> int {
        if (ev) {
            StageEvent e{kind, nullptr, nullptr};
            PT_CU(cudaEventCreate(&e.a));
            PT_CU(cudaEventCreate(&e.b));
            PT_CU(cudaEventRecord(e.a, st));
            launch();
            PT_CU(cudaEventRecord(e.b, st));
            ev->push_back(e);
        } else {
            launch();
        }
        return PT_OK;
    };
    const int lanes = std::max(1, P.npath / std::max(P.npix, 1));
    const int total = static_cast<int>(total_samples);
    const int tsi = trace_shape_index(P.trace_block, P.stack_depth);
    for (int s0 = 0; s0 < total; s0 += lanes) {
        const int count = std::min(lanes, total - s0);
        if (int rc = timed(3, [&] { k_raygen<<<wf.grid_raygen, 256, 0, st>>>(P, s0, count); })) return rc;
        for (int d = 0; d < P.max_depth; ++d) {
            const int q = d & 1;
            if (int rc = timed(0, [&] { launch_extend(tsi, wf.grid_extend[tsi], st, P, q, d); })) return rc;
            if (infer) {
                if (int rc = timed(4, [&] { launch_guide_infer(*gs, P, q, wf.sms, st); })) return rc;
            }
            if (int rc = timed(1, [&] {
                    const bool tex = P.scene.num_textures > 0;
                    if (P.gmix) {
                        if (tex) k_shade_front<true, true><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                        else k_shade_front<true><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                    } else {
                        if (tex) k_shade_front<false, true><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                        else k_shade_front<false><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                    }
                    if (d + 1 < P.max_depth) {
                        if (P.gmix) {
                            if (tex) k_shade_back<true, true><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                            else k_shade_back<true><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                        } else {
                            if (tex) k_shade_back<false, true><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                            else k_shade_back<false><<<wf.grid_shade, 128, 0, st>>>(P, q, d, s0);
                        }
                    }
                })) return rc;
            if (int rc = timed(2, [&] { launch_shadow(tsi, wf.grid_shadow[tsi], st, P, d); })) return rc;
        }
        if (int rc = timed(3, [&] { k_finalize<<<wf.grid_finalize, 256, 0, st>>>(P, s0, count); })) return rc;
        if (train) {
            if (int rc = timed(4, [&] {
                    const int np = P.npix * count;
                    k_guide_count<<<wf.grid_finalize, 256, 0, st>>>(P, np, gs->scan_counts);
                    size_t tmp = gs->scan_tmp_bytes;
                    cub::DeviceScan::ExclusiveSum(gs->scan_tmp, tmp, gs->scan_counts, gs->scan_offsets, np + 1, st);
                    k_guide_collect<<<wf.grid_finalize, 256, 0, st>>>(P, np, gs->net, gs->samples, gs->scan_offsets,
                                                                      gs->counters, gs->sample_cap);
                    // optimiser steps over this pass's samples in minibatches
                    const int nmb = guide_minibatches(int64_t(P.npix) * count, gs->paths_per_step);
                    const uint32_t step_cap = guide_step_cap(gs->samples_per_step);
                    for (int mb = 0; mb < nmb; ++mb) {
                        k_guide_train<<<wf.sms, 32 * kGTrainWarps, kGTrainSmem, st>>>(gs->net, gs->samples, gs->counters,
                                                                         gs->sample_cap, mb, nmb, step_cap, gs->rows);
                        k_guide_dw<<<dim3(kGDwChunks, 4), 128, 0, st>>>(gs->counters, gs->sample_cap, mb, nmb, step_cap,
                                                                        gs->rows, gs->partial);
                        k_guide_dw_reduce<<<(kGWeights + 255) / 256, 256, 0, st>>>(gs->counters, gs->sample_cap, mb, nmb,
                                                                                   step_cap, gs->partial,
                                                                                   gs->net.w_grad);
                        k_guide_adam<<<wf.sms * 8, 256, 0, st>>>(gs->net, gs->counters, gs->sample_cap, mb, nmb,
                                                                 gs->step, gs->lr, gs->lr, 0.9f, 0.99f, 1e-10f,
                                                                 gs->lr_half_life, gs->lr_floor);
                    }
                    k_guide_step<<<1, 1, 0, st>>>(gs->counters, gs->step, gs->net.loss, gs->net.loss_fix,
                                                  gs->sample_cap, nmb);
                })) return rc;
        }
    }
    PT_CU(cudaGetLastError());
    return PT_OK;
}

}  // namespace

DeviceScene device_view(const pt_scene* s) {
    DeviceScene v;
    std::memset(&v, 0, sizeof(v));
    const SceneTables& t = s->tables;
    const DeviceSceneBuffers& d = s->dev;
    v.inner = static_cast<const InnerNode*>(d.inner);
    v.tris = static_cast<const TriRecord*>(d.tris);
    for (int a = 0; a < 3; ++a) { v.root_lo[a] = t.root_lo[a]; v.root_hi[a] = t.root_hi[a]; }
    v.root_ref = t.root_ref;
    v.num_faces = static_cast<uint32_t>(s->host.faces.size());
    v.vertices = static_cast<const pt_vertex*>(d.vertices);
    v.faces = static_cast<const pt_face*>(d.faces);
    v.materials = static_cast<const pt_material*>(d.materials);
    v.num_materials = static_cast<uint32_t>(s->host.materials.size());
    v.emissive = static_cast<const pt_emissive_ref*>(d.emissive);
    v.num_emissive = static_cast<uint32_t>(t.emissive.size());
    v.tri_light_pmf = static_cast<const float*>(d.tri_pmf);
    v.tri_alias = static_cast<const pt_alias_entry*>(d.tri_alias);
    v.env_pmf = static_cast<const float*>(d.env_pmf);
    v.env_alias = static_cast<const pt_alias_entry*>(d.env_alias);
    v.num_env_texels = static_cast<uint32_t>(t.env_pmf.size());
    v.env_w = t.env_w;
    v.env_h = t.env_h;
    v.env_tex = d.env_tex;
    v.punctual = static_cast<const pt_punctual_light*>(d.punctual);
    v.num_punctual = static_cast<uint32_t>(s->host.punctual.size());
    v.textures = static_cast<const unsigned long long*>(d.tex_table);
    v.num_textures = d.tex_table ? static_cast<uint32_t>(d.tex_objs.size()) : 0u;
    return v;
}

void free_scene_device(pt_scene* s) {
    DeviceSceneBuffers& d = s->dev;
    if (d.device >= 0) cudaSetDevice(d.device);
    if (d.env_tex) cudaDestroyTextureObject(static_cast<cudaTextureObject_t>(d.env_tex));
    if (d.env_array) cudaFreeArray(static_cast<cudaArray_t>(d.env_array));
    for (unsigned long long t : d.tex_objs) if (t) cudaDestroyTextureObject(static_cast<cudaTextureObject_t>(t));
    for (void* a : d.tex_arrays) if (a) cudaFreeArray(static_cast<cudaArray_t>(a));
    if (d.tex_table) cudaFree(d.tex_table);
    void* bufs[] = {d.inner, d.tris, d.vertices, d.faces, d.materials, d.emissive, d.tri_pmf,
                    d.tri_alias, d.env_pmf, d.env_alias, d.punctual};
    for (void* b : bufs) if (b) cudaFree(b);
    d = DeviceSceneBuffers{};
}

void unpin_host_arrays(pt_scene* s) {
    for (void* p : s->pinned) cudaHostUnregister(p);
    s->pinned.clear();
    cudaGetLastError();
}

// Page-lock the large host arrays once so that every upload copies from pinned
// memory (they are not resized after the build).
static void pin_host_arrays(pt_scene* s) {
    if (!s->pinned.empty()) return;
    auto pin = [&](void* p, size_t bytes) {
        if (!p || bytes < (1u << 20)) return;
        if (cudaHostRegister(p, bytes, cudaHostRegisterDefault) == cudaSuccess) s->pinned.push_back(p);
        else cudaGetLastError();
    };
    pin(s->tables.inner.data(), s->tables.inner.size() * sizeof(InnerNode));
    pin(s->tables.tris.data(), s->tables.tris.size() * sizeof(TriRecord));
    pin(s->host.vertices.data(), s->host.vertices.size() * sizeof(pt_vertex));
    pin(s->host.faces.data(), s->host.faces.size() * sizeof(pt_face));
    pin(s->host.env_rgba.data(), s->host.env_rgba.size() * sizeof(float));
    pin(s->tables.env_pmf.data(), s->tables.env_pmf.size() * sizeof(float));
    pin(s->tables.env_alias.data(), s->tables.env_alias.size() * sizeof(pt_alias_entry));
}

// GL wrap mode -> CUDA address mode (CudaTexture, Part_2/src/cuda/cuda_texture.cu:27-34).
static cudaTextureAddressMode gl_wrap_mode(int gl) {
    if (gl == 33071) return cudaAddressModeClamp;    // CLAMP_TO_EDGE
    if (gl == 33648) return cudaAddressModeMirror;   // MIRRORED_REPEAT
    return cudaAddressModeWrap;                      // REPEAT and anything else
}

// Material textures as the reference's CudaTexture (cuda_texture.cu:37-62):
// float4 arrays, bilinear filtering, normalized coordinates, the sampler's wrap
// modes; a texture without an image gets no object (lookups skip it).
static int upload_textures(const HostScene& h, DeviceSceneBuffers& d) {
    const size_t nt = h.textures.size();
    d.tex_arrays.assign(nt, nullptr);
    d.tex_objs.assign(nt, 0ull);
    d.tex_sizes.assign(nt, 0);
    d.tex_wraps.assign(nt, 0);
    if (nt == 0) return PT_OK;
    for (size_t i = 0; i < nt; ++i) {
        const HostTextureImage& t = h.textures[i];
        if (t.width <= 0 || t.height <= 0 || t.rgba.size() != size_t(t.width) * t.height * 4) continue;
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
        cudaArray_t arr = nullptr;
        if (cudaMallocArray(&arr, &ch, t.width, t.height) != cudaSuccess) {
            cudaGetLastError();
            set_error("texture " + std::to_string(i) + ": cannot allocate " + std::to_string(t.width) + "x" +
                      std::to_string(t.height));
            return PT_ERR_NOMEM;
        }
        d.tex_arrays[i] = arr;
        const size_t pitch = static_cast<size_t>(t.width) * 4 * sizeof(float);
        PT_CU(cudaMemcpy2DToArray(arr, 0, 0, t.rgba.data(), pitch, pitch, t.height, cudaMemcpyHostToDevice));
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = gl_wrap_mode(t.wrap_s);
        td.addressMode[1] = gl_wrap_mode(t.wrap_t);
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        cudaTextureObject_t tex = 0;
        PT_CU(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
        d.tex_objs[i] = tex;
        d.tex_sizes[i] = size_t(t.width) * t.height;
        d.tex_wraps[i] = (t.wrap_s << 16) ^ t.wrap_t;
        d.bytes += static_cast<uint64_t>(t.width) * t.height * 16;
    }
    PT_CU(cudaMalloc(&d.tex_table, nt * sizeof(unsigned long long)));
    PT_CU(cudaMemcpy(d.tex_table, d.tex_objs.data(), nt * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    return PT_OK;
}

int upload_scene(pt_scene* s, int device) {
    if (!s->tables.built) { set_error("scene not built: call pt_scene_build_accel first"); return PT_ERR_STATE; }
    const HostScene& hs = s->host;
    const SceneTables& ts = s->tables;
    DeviceSceneBuffers& d = s->dev;
    void** bufs[11] = {&d.inner, &d.tris, &d.vertices, &d.faces, &d.materials, &d.emissive, &d.tri_pmf,
                       &d.tri_alias, &d.env_pmf, &d.env_alias, &d.punctual};
    const void* srcs[11] = {ts.inner.data(), ts.tris.data(), hs.vertices.data(), hs.faces.data(),
                            hs.materials.data(), ts.emissive.data(), ts.tri_pmf.data(), ts.tri_alias.data(),
                            ts.env_pmf.data(), ts.env_alias.data(), hs.punctual.data()};
    const size_t sizes[11] = {ts.inner.size() * sizeof(InnerNode), ts.tris.size() * sizeof(TriRecord),
                              hs.vertices.size() * sizeof(pt_vertex), hs.faces.size() * sizeof(pt_face),
                              hs.materials.size() * sizeof(pt_material), ts.emissive.size() * sizeof(pt_emissive_ref),
                              ts.tri_pmf.size() * sizeof(float), ts.tri_alias.size() * sizeof(pt_alias_entry),
                              ts.env_pmf.size() * sizeof(float), ts.env_alias.size() * sizeof(pt_alias_entry),
                              hs.punctual.size() * sizeof(pt_punctual_light)};
    // Same device and the same buffer sizes: copy into the existing buffers.
    // The device addresses stay, so a render graph captured for them stays valid.
    bool same = d.uploaded && d.device == device && d.env_w == hs.env_w && d.env_h == hs.env_h &&
                d.tex_objs.size() == hs.textures.size();
    for (int i = 0; i < 11 && same; ++i) same = d.sizes[i] == sizes[i];
    for (size_t i = 0; i < hs.textures.size() && same; ++i) {
        const HostTextureImage& t = hs.textures[i];
        const bool has = t.width > 0 && t.height > 0 && t.rgba.size() == size_t(t.width) * t.height * 4;
        same = has == (d.tex_objs[i] != 0) && (!has || (d.tex_sizes[i] == size_t(t.width) * t.height &&
                                                         d.tex_wraps[i] == ((t.wrap_s << 16) ^ t.wrap_t)));
    }
    if (same) {
        if (int rc = ensure_device(device)) return rc;
        pin_host_arrays(s);
        for (int i = 0; i < 11; ++i)
            if (sizes[i]) PT_CU(cudaMemcpy(*bufs[i], srcs[i], sizes[i], cudaMemcpyHostToDevice));
        if (hs.env_w > 0 && hs.env_h > 0) {
            const size_t pitch = static_cast<size_t>(hs.env_w) * 4 * sizeof(float);
            PT_CU(cudaMemcpy2DToArray(static_cast<cudaArray_t>(d.env_array), 0, 0, hs.env_rgba.data(), pitch, pitch,
                                      hs.env_h, cudaMemcpyHostToDevice));
        }
        for (size_t i = 0; i < hs.textures.size(); ++i) {
            const HostTextureImage& t = hs.textures[i];
            if (!d.tex_arrays[i]) continue;
            const size_t pitch = static_cast<size_t>(t.width) * 4 * sizeof(float);
            PT_CU(cudaMemcpy2DToArray(static_cast<cudaArray_t>(d.tex_arrays[i]), 0, 0, t.rgba.data(), pitch, pitch,
                                      t.height, cudaMemcpyHostToDevice));
        }
        return PT_OK;
    }
    free_scene_device(s);
    if (int rc = ensure_device(device)) return rc;
    pin_host_arrays(s);
    d.device = device;
    for (int i = 0; i < 11; ++i) d.sizes[i] = sizes[i];
    d.env_w = hs.env_w;
    d.env_h = hs.env_h;
    auto up = [&](void** dst, const void* src, size_t bytes) -> int {
        if (bytes == 0) { *dst = nullptr; return PT_OK; }
        if (cudaMalloc(dst, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_error("cudaMalloc of " + std::to_string(bytes) + " bytes failed");
            return PT_ERR_NOMEM;
        }
        PT_CU(cudaMemcpy(*dst, src, bytes, cudaMemcpyHostToDevice));
        d.bytes += bytes;
        return PT_OK;
    };
    const HostScene& h = s->host;
    const SceneTables& t = s->tables;
    int rc = PT_OK;
    if ((rc = up(&d.inner, t.inner.data(), t.inner.size() * sizeof(InnerNode)))) return rc;
    if ((rc = up(&d.tris, t.tris.data(), t.tris.size() * sizeof(TriRecord)))) return rc;
    if ((rc = up(&d.vertices, h.vertices.data(), h.vertices.size() * sizeof(pt_vertex)))) return rc;
    if ((rc = up(&d.faces, h.faces.data(), h.faces.size() * sizeof(pt_face)))) return rc;
    if ((rc = up(&d.materials, h.materials.data(), h.materials.size() * sizeof(pt_material)))) return rc;
    if ((rc = up(&d.emissive, t.emissive.data(), t.emissive.size() * sizeof(pt_emissive_ref)))) return rc;
    if ((rc = up(&d.tri_pmf, t.tri_pmf.data(), t.tri_pmf.size() * sizeof(float)))) return rc;
    if ((rc = up(&d.tri_alias, t.tri_alias.data(), t.tri_alias.size() * sizeof(pt_alias_entry)))) return rc;
    if ((rc = up(&d.env_pmf, t.env_pmf.data(), t.env_pmf.size() * sizeof(float)))) return rc;
    if ((rc = up(&d.env_alias, t.env_alias.data(), t.env_alias.size() * sizeof(pt_alias_entry)))) return rc;
    if ((rc = up(&d.punctual, h.punctual.data(), h.punctual.size() * sizeof(pt_punctual_light)))) return rc;
    if (h.env_w > 0 && h.env_h > 0) {
        // float4 array, linear filtering, wrap, normalized coordinates
        // (CudaTexture, Part_2/src/cuda/cuda_texture.cu:39-63)
        cudaChannelFormatDesc ch = cudaCreateChannelDesc<float4>();
        cudaArray_t arr = nullptr;
        PT_CU(cudaMallocArray(&arr, &ch, h.env_w, h.env_h));
        d.env_array = arr;
        const size_t pitch = static_cast<size_t>(h.env_w) * 4 * sizeof(float);
        PT_CU(cudaMemcpy2DToArray(arr, 0, 0, h.env_rgba.data(), pitch, pitch, h.env_h, cudaMemcpyHostToDevice));
        cudaResourceDesc rd;
        std::memset(&rd, 0, sizeof(rd));
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = arr;
        cudaTextureDesc td;
        std::memset(&td, 0, sizeof(td));
        td.addressMode[0] = cudaAddressModeWrap;
        td.addressMode[1] = cudaAddressModeWrap;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        cudaTextureObject_t tex = 0;
        PT_CU(cudaCreateTextureObject(&tex, &rd, &td, nullptr));
        d.env_tex = tex;
        d.bytes += static_cast<uint64_t>(h.env_w) * h.env_h * 16;
    }
    if (int rc2 = upload_textures(h, d)) return rc2;
    d.uploaded = true;
    return PT_OK;
}

int film_alloc(pt_film* f) {
    if (int rc = ensure_device(f->device)) return rc;
    const size_t bytes = static_cast<size_t>(f->width) * f->height * sizeof(float4);
    void** bufs[] = {&f->sum, &f->comp, &f->batch, &f->fresh, &f->resolve};
    for (void** b : bufs) {
        if (cudaMalloc(b, bytes) != cudaSuccess) {
            cudaGetLastError();
            set_error("cannot allocate film buffers");
            return PT_ERR_NOMEM;
        }
        PT_CU(cudaMemset(*b, 0, bytes));
    }
    return PT_OK;
}

void film_free(pt_film* f) {
    if (f->device >= 0) cudaSetDevice(f->device);
    void* bufs[] = {f->sum, f->comp, f->batch, f->fresh, f->resolve};
    for (void* b : bufs) if (b) cudaFree(b);
    f->sum = f->comp = f->batch = f->fresh = f->resolve = nullptr;
}

// Film::clear and Film::downloadAccumulated are blocking calls on the legacy
// stream in the reference (film.cu:8-59), ordered after every render launch;
// renders here run on the integrator's or the caller's stream, so both wait
// for the device first.
int film_clear(pt_film* f) {
    if (int rc = ensure_device(f->device)) return rc;
    PT_CU(cudaDeviceSynchronize());
    const size_t bytes = static_cast<size_t>(f->width) * f->height * sizeof(float4);
    void* bufs[] = {f->sum, f->comp, f->batch, f->fresh};
    for (void* b : bufs) PT_CU(cudaMemset(b, 0, bytes));
    return PT_OK;
}

int film_download(const pt_film* f, float* host, bool fresh, bool host_ptr) {
    if (int rc = ensure_device(f->device)) return rc;
    PT_CU(cudaDeviceSynchronize());
    const int n = f->width * f->height;
    const size_t bytes = static_cast<size_t>(n) * sizeof(float4);
    if (fresh) {
        PT_CU(cudaMemcpy(host, f->fresh, bytes, host_ptr ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
        return PT_OK;
    }
    k_film_mean<<<(n + 255) / 256, 256>>>(static_cast<const float4*>(f->sum), static_cast<const float4*>(f->comp),
                                          static_cast<float4*>(f->resolve), n);
    PT_CU(cudaGetLastError());
    PT_CU(cudaMemcpy(host, f->resolve, bytes, host_ptr ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
    return PT_OK;
}

void integrator_free(pt_integrator* integ) {
    Wavefront* wf = integ->wf;
    if (!wf) return;
    if (wf->device >= 0) cudaSetDevice(wf->device);
    if (wf->graph) cudaGraphExecDestroy(wf->graph);
    if (wf->arena) cudaFree(wf->arena);
    if (wf->own_stream) cudaStreamDestroy(wf->own_stream);
    delete wf;
    integ->wf = nullptr;
}

// Integrator::launch (Part_2/src/integrators/path.cu:244-255).
// Sizes the integrator's wavefront for `total` samples per pixel and fills the
// launch parameters (P, built byte-wise with zeroed padding because its bytes
// key the graph cache).  budget > 0 overrides the scene's paths-in-flight.
int prepare_wave(pt_integrator* integ, pt_film* film, pt_scene* s, const pt_scene_params* prm, int64_t total,
                 int64_t budget_override, WaveParams& P, int& lanes_out) {
    if (!s->dev.uploaded) { set_error("scene not uploaded: call pt_scene_upload first"); return PT_ERR_STATE; }
    if (film->width != prm->width || film->height != prm->height) { set_error("film size does not match params"); return PT_ERR_INVALID; }
    if (prm->width <= 0 || prm->height <= 0 || prm->sample_per_frame <= 0 || prm->max_depth < 0) {
        set_error("invalid scene params"); return PT_ERR_INVALID;
    }
    if (film->device != s->dev.device) { set_error("film and scene live on different devices"); return PT_ERR_INVALID; }
    if (total < 1) { set_error("sample count must be positive"); return PT_ERR_INVALID; }
    if (!integ->wf) integ->wf = new Wavefront();
    Wavefront& wf = *integ->wf;
    const int npix = prm->width * prm->height;
    const int n_slots = 2 + static_cast<int>(s->host.punctual.size());
    const pt_render_settings& rs = s->host.settings;
    // samples per pixel in flight per pass: as many of the launch's as the path
    // budget holds (a guide's per-path records cap it lower)
    GuideState* gs = wf.guide;
    const bool guided = gs && gs->mode != 0;
    int64_t budget = budget_override > 0 ? budget_override
                   : (rs.paths_in_flight > 0 ? rs.paths_in_flight : kDefaultPathsInFlight);
    if (guided) budget = std::min<int64_t>(budget, gs->mode == PT_GUIDE_TRAIN ? kTrainingPathsInFlight
                                                                              : kGuidedPathsInFlight);
    int lanes = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(total, budget / npix)));
    // fewer samples in flight when the device cannot hold the path slots
    // (results do not depend on the pass size)
    int rc_alloc = wavefront_prepare(wf, s->dev.device, npix * lanes, n_slots);
    while (rc_alloc == PT_ERR_NOMEM && lanes > 1) {
        lanes /= 2;
        rc_alloc = wavefront_prepare(wf, s->dev.device, npix * lanes, n_slots);
    }
    if (rc_alloc) return rc_alloc;
    const int npath = npix * lanes;
    std::memset(&P, 0, sizeof(P));
    std::memcpy(&P, &wf.base, sizeof(P));
    const DeviceScene view = device_view(s);
    std::memcpy(&P.scene, &view, sizeof(DeviceScene));
    P.cam = prm->camera;
    P.width = prm->width; P.height = prm->height; P.npix = npix; P.npath = npath;
    P.spf = prm->sample_per_frame;
    P.max_depth = prm->max_depth;
    P.sampler_type = prm->sampler_type;
    P.arg_rtl = rs.arg_order == PT_ARGS_RTL ? 1 : 0;
    P.flags = rs.flags;
    P.pcg_seed = rs.pcg_seed;
    P.n_slots = n_slots;
    P.f_sum = static_cast<float4*>(film->sum);
    P.f_comp = static_cast<float4*>(film->comp);
    P.f_batch = static_cast<float4*>(film->batch);
    P.f_new = static_cast<float4*>(film->fresh);
    if (guided) {
        if (gs->device != s->dev.device) { set_error("guide and scene live on different devices"); return PT_ERR_INVALID; }
        if (int rc = guide_prepare_work(*gs, npath, prm->max_depth, gs->mode == PT_GUIDE_TRAIN)) return rc;
        P.gmix = gs->mix;
        P.galpha = gs->alpha;
        P.grec = gs->mode == PT_GUIDE_TRAIN ? gs->rec : nullptr;
    }
    // traversal shape: the settings' (the tuner's), 128 threads and 64 entries
    // by default; a stack no deeper than the tree falls back to 64 entries
    P.trace_block = rs.trace_block ? rs.trace_block : 128;
    P.stack_depth = rs.stack_depth ? rs.stack_depth : kStackDepth;
    if (P.stack_depth <= static_cast<int>(s->tables.bvh_depth)) P.stack_depth = kStackDepth;
    lanes_out = lanes;
    return PT_OK;
}

int integrator_launch(pt_integrator* integ, pt_film* film, pt_scene* s, const pt_scene_params* prm, int nframes,
                      void* stream) {
    if (nframes < 1) { set_error("frame count must be positive"); return PT_ERR_INVALID; }
    const int64_t total = static_cast<int64_t>(prm->sample_per_frame) * nframes;
    WaveParams P;
    int lanes = 1;
    if (int rc = prepare_wave(integ, film, s, prm, total, 0, P, lanes)) return rc;
    Wavefront& wf = *integ->wf;
    GuideState* gs = wf.guide;
    const pt_render_settings& rs = s->host.settings;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : wf.own_stream;
    k_begin<<<1, 1, 0, st>>>(P.pass, s->frame_count);
    PT_CU(cudaGetLastError());
    const bool timing = (rs.flags & PT_FLAG_STAGE_TIMING) != 0;
    const bool use_graph = !timing && !(rs.flags & PT_FLAG_NO_GRAPH);
    if (timing) {
        std::vector<StageEvent> ev;
        cudaEvent_t t0, t1;
        PT_CU(cudaEventCreate(&t0));
        PT_CU(cudaEventCreate(&t1));
        PT_CU(cudaEventRecord(t0, st));
        int rc = enqueue_batch(wf, P, total, st, &ev, gs);
        PT_CU(cudaEventRecord(t1, st));
        PT_CU(cudaEventSynchronize(t1));
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t0, t1);
        wf.total_ms += ms;
        for (StageEvent& e : ev) {
            float m = 0.0f;
            cudaEventElapsedTime(&m, e.a, e.b);
            wf.stage_ms[e.kind] += m;
            if (e.kind == 0) wf.extend_launches++;
            cudaEventDestroy(e.a);
            cudaEventDestroy(e.b);
        }
        cudaEventDestroy(t0);
        cudaEventDestroy(t1);
        if (rc) return rc;
    } else if (use_graph) {
        // everything the captured launches bake in: the parameters, the stream,
        // the frame count and the guide's training settings
        struct GuideKey {
            const void* params; const void* feat; float lr, lr_half_life, lr_floor, ema;
            int paths_per_step; uint32_t samples_per_step; int infer;
        } gk{};
        if (gs) gk = GuideKey{gs->params, gs->feat, gs->lr, gs->lr_half_life, gs->lr_floor, gs->net.ema,
                              gs->paths_per_step, gs->samples_per_step, gs->infer};
        std::vector<unsigned char> key(sizeof(WaveParams) + sizeof(cudaStream_t) + sizeof(int) + sizeof(GuideKey));
        std::memcpy(key.data(), &P, sizeof(WaveParams));
        std::memcpy(key.data() + sizeof(WaveParams), &st, sizeof(cudaStream_t));
        std::memcpy(key.data() + sizeof(WaveParams) + sizeof(cudaStream_t), &nframes, sizeof(int));
        std::memcpy(key.data() + sizeof(WaveParams) + sizeof(cudaStream_t) + sizeof(int), &gk, sizeof(GuideKey));
        if (!wf.graph || key != wf.graph_key) {
            if (wf.graph) { cudaGraphExecDestroy(wf.graph); wf.graph = nullptr; }
            cudaGraph_t g = nullptr;
            PT_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
            const int rc = enqueue_batch(wf, P, total, st, nullptr, gs);
            const cudaError_t ec = cudaStreamEndCapture(st, &g);
            if (rc) { if (g) cudaGraphDestroy(g); return rc; }
            if (ec != cudaSuccess) { set_error(std::string("graph capture failed: ") + cudaGetErrorString(ec)); return PT_ERR_CUDA; }
            const cudaError_t ei = cudaGraphInstantiate(&wf.graph, g, 0);
            cudaGraphDestroy(g);
            if (ei != cudaSuccess) { wf.graph = nullptr; set_error(std::string("graph instantiate failed: ") + cudaGetErrorString(ei)); return PT_ERR_CUDA; }
            wf.graph_key = key;
        }
        PT_CU(cudaGraphLaunch(wf.graph, st));
    } else {
        if (int rc = enqueue_batch(wf, P, total, st, nullptr, gs)) return rc;
    }
    // k_begin + per pass (raygen; extend, shade front, shade back, shadow per bounce, no back at the last; finalize)
    const uint64_t passes = static_cast<uint64_t>((total + lanes - 1) / lanes);
    if (!timing) wf.extend_launches += passes * static_cast<uint64_t>(P.max_depth);
    wf.kernel_launches += 1 + passes * (1 + 4 * static_cast<uint64_t>(P.max_depth));
    if (P.gmix)
        wf.kernel_launches += passes * ((wf.guide->infer == PT_GUIDE_INFER_FUSED ? 1 : 3) * P.max_depth +
                                        (P.grec ? 5 + 4 * guide_minibatches(int64_t(P.npix) * lanes, wf.guide->paths_per_step) : 0));
    return PT_OK;
}

int integrator_check(pt_integrator* integ, bool sync) {
    Wavefront* wf = integ->wf;
    if (!wf || wf->device < 0) return PT_OK;
    if (int rc = ensure_device(wf->device)) return rc;
    if (sync) PT_CU(cudaDeviceSynchronize());
    uint32_t err = 0;
    PT_CU(cudaMemcpy(&err, wf->base.err, 4, cudaMemcpyDeviceToHost));
    if (err) {
        std::string m = "device error word 0x" + std::to_string(err) + ":";
        if (err & kErrStackOverflow) m += " traversal stack overflow;";
        if (err & kErrQueueOverflow) m += " queue overflow;";
        if (err & kErrGuideTimeout) m += " guide network wait timed out;";
        set_error(m);
        PT_CU(cudaMemset(wf->base.err, 0, 4));
        return PT_ERR_DEVICE;
    }
    return PT_OK;
}

int integrator_stats(const pt_integrator* integ, pt_render_stats* out) {
    std::memset(out, 0, sizeof(*out));
    const Wavefront* wf = integ->wf;
    if (!wf || wf->device < 0) return PT_OK;
    if (int rc = ensure_device(wf->device)) return rc;
    unsigned long long st[kStatCount];
    PT_CU(cudaMemcpy(st, wf->base.stats, sizeof(st), cudaMemcpyDeviceToHost));
    out->camera_rays = st[kStatCameraRays];
    out->extension_rays = st[kStatExtRays];
    out->shadow_rays = st[kStatShadowRays];
    out->node_visits = st[kStatNodes];
    out->triangle_tests = st[kStatTris];
    out->shadow_node_visits = st[kStatShadowNodes];
    out->shadow_triangle_tests = st[kStatShadowTris];
    out->paths = st[kStatPaths];
    out->extend_launches = wf->extend_launches;
    out->extend_ms = wf->stage_ms[0];
    out->shade_ms = wf->stage_ms[1];
    out->shadow_ms = wf->stage_ms[2];
    out->other_ms = wf->stage_ms[3];
    out->guide_ms = wf->stage_ms[4];
    out->total_ms = wf->total_ms;
    out->kernel_launches = wf->kernel_launches;
    return PT_OK;
}

int integrator_reset_stats(pt_integrator* integ) {
    Wavefront* wf = integ->wf;
    if (!wf || wf->device < 0) return PT_OK;
    if (int rc = ensure_device(wf->device)) return rc;
    PT_CU(cudaMemset(wf->base.stats, 0, kStatCount * 8));
    for (double& d : wf->stage_ms) d = 0.0;
    wf->total_ms = 0.0;
    wf->extend_launches = 0;
    wf->kernel_launches = 0;
    return PT_OK;
}

// ---- diagnostics ----
int trace_rays(pt_scene* s, const float* rays, uint32_t n, pt_hit* hits, uint8_t* occl, bool any, bool device_ptrs) {
    if (!s->dev.uploaded) { set_error("scene not uploaded"); return PT_ERR_STATE; }
    if (int rc = ensure_device(s->dev.device)) return rc;
    if (n == 0) return PT_OK;
    const float* d_rays = rays;
    void* d_out = any ? static_cast<void*>(occl) : static_cast<void*>(hits);
    void* tmp_rays = nullptr;
    void* tmp_out = nullptr;
    uint32_t* d_err = nullptr;
    const size_t out_bytes = any ? n : static_cast<size_t>(n) * sizeof(pt_hit);
    auto cleanup = [&] { if (tmp_rays) cudaFree(tmp_rays); if (tmp_out) cudaFree(tmp_out); if (d_err) cudaFree(d_err); };
    if (!device_ptrs) {
        if (cudaMalloc(&tmp_rays, static_cast<size_t>(n) * 32) != cudaSuccess ||
            cudaMalloc(&tmp_out, out_bytes) != cudaSuccess) {
            cudaGetLastError(); cleanup(); set_error("cannot allocate ray buffers"); return PT_ERR_NOMEM;
        }
        if (cudaMemcpy(tmp_rays, rays, static_cast<size_t>(n) * 32, cudaMemcpyHostToDevice) != cudaSuccess) {
            cleanup(); set_error("ray upload failed"); return PT_ERR_CUDA;
        }
        d_rays = static_cast<const float*>(tmp_rays);
        d_out = tmp_out;
    }
    if (cudaMalloc(&d_err, 4) != cudaSuccess || cudaMemset(d_err, 0, 4) != cudaSuccess) {
        cudaGetLastError(); cleanup(); set_error("cannot allocate error word"); return PT_ERR_NOMEM;
    }
    const DeviceScene v = device_view(s);
    const int wt = (s->host.settings.flags & PT_FLAG_WATERTIGHT) ? 1 : 0;
    const int blocks = static_cast<int>(std::min<uint32_t>((n + 127) / 128, 148u * 16u));
    k_trace_rays<<<blocks, 128>>>(v, d_rays, n, any ? nullptr : static_cast<pt_hit*>(d_out),
                                  any ? static_cast<uint8_t*>(d_out) : nullptr, any ? 1 : 0, wt, d_err);
    cudaError_t e = cudaDeviceSynchronize();
    uint32_t err = 0;
    if (e == cudaSuccess) e = cudaMemcpy(&err, d_err, 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && !device_ptrs)
        e = cudaMemcpy(any ? static_cast<void*>(occl) : static_cast<void*>(hits), d_out, out_bytes, cudaMemcpyDeviceToHost);
    cleanup();
    if (e != cudaSuccess) { set_error(std::string("trace failed: ") + cudaGetErrorString(e)); return PT_ERR_CUDA; }
    if (err) { set_error("traversal stack overflow"); return PT_ERR_DEVICE; }
    return PT_OK;
}

// Display tone mapping of the reference's preview (Part_2/preview/
// tone_mapping.frag:12-29): 1 - exp(-c * 2^exposure) per channel, then the
// sRGB transfer curve, written as 8-bit unorm (round to nearest, as the
// display framebuffer stores it), alpha 255.
__global__ void k_tonemap(const float4* __restrict__ in, uchar4* __restrict__ out, uint32_t n, float scale) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = in[i];
        auto enc = [&](float v) -> unsigned char {
            const float t = 1.0f - expf(-v * scale);
            const float e = t <= 0.0031308f ? 12.92f * t : 1.055f * powf(t, 1.0f / 2.4f) - 0.055f;
            return static_cast<unsigned char>(__float2int_rn(fminf(fmaxf(e, 0.0f), 1.0f) * 255.0f));
        };
        out[i] = make_uchar4(enc(c.x), enc(c.y), enc(c.z), 255);
    }
}

int tonemap(const float* rgba, int w, int h, float exposure, uint8_t* out, bool device_ptrs, int device) {
    if (int rc = ensure_device(device)) return rc;
    const size_t n = static_cast<size_t>(w) * h;
    if (n == 0) return PT_OK;
    const float scale = std::exp2(exposure);
    const int grid = static_cast<int>(std::min<size_t>((n + 255) / 256, 148 * 16));
    if (device_ptrs) {
        k_tonemap<<<grid, 256>>>(reinterpret_cast<const float4*>(rgba), reinterpret_cast<uchar4*>(out),
                                 static_cast<uint32_t>(n), scale);
        PT_CU(cudaGetLastError());
        PT_CU(cudaDeviceSynchronize());
        return PT_OK;
    }
    float4* din = nullptr;
    uchar4* dout = nullptr;
    PT_CU(cudaMalloc(&din, n * sizeof(float4)));
    if (cudaMalloc(&dout, n * sizeof(uchar4)) != cudaSuccess) {
        cudaFree(din); cudaGetLastError(); set_error("tone map: allocation failed"); return PT_ERR_NOMEM;
    }
    cudaError_t e = cudaMemcpy(din, rgba, n * sizeof(float4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_tonemap<<<grid, 256>>>(din, dout, static_cast<uint32_t>(n), scale);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, dout, n * sizeof(uchar4), cudaMemcpyDeviceToHost);
    cudaFree(din);
    cudaFree(dout);
    if (e != cudaSuccess) { set_error(std::string("tone map: ") + cudaGetErrorString(e)); return PT_ERR_CUDA; }
    return PT_OK;
}

int sampler_stream(int type, int w, int h, uint32_t frame, int spf, int sif, uint32_t ndims, uint32_t seed,
                   int device, float* out_host) {
    if (int rc = ensure_device(device)) return rc;
    const size_t bytes = static_cast<size_t>(w) * h * ndims * sizeof(float);
    if (bytes == 0) return PT_OK;
    float* d = nullptr;
    PT_CU(cudaMalloc(&d, bytes));
    k_sampler_stream<<<std::min((w * h + 255) / 256, 148 * 8), 256>>>(type, w, h, frame, spf, sif, ndims, seed, d);
    cudaError_t e = cudaMemcpy(out_host, d, bytes, cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) { set_error(std::string("sampler stream failed: ") + cudaGetErrorString(e)); return PT_ERR_CUDA; }
    return PT_OK;
}

int bsdf_eval(pt_scene* s, const float* in, uint32_t n, float* out_host) {
    if (!s->dev.uploaded) { set_error("scene not uploaded"); return PT_ERR_STATE; }
    if (int rc = ensure_device(s->dev.device)) return rc;
    if (n == 0) return PT_OK;
    float *din = nullptr, *dout = nullptr;
    PT_CU(cudaMalloc(&din, static_cast<size_t>(n) * 13 * 4));
    if (cudaMalloc(&dout, static_cast<size_t>(n) * 4 * 4) != cudaSuccess) { cudaFree(din); cudaGetLastError(); set_error("alloc failed"); return PT_ERR_NOMEM; }
    cudaError_t e = cudaMemcpy(din, in, static_cast<size_t>(n) * 13 * 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        k_bsdf_eval<<<std::min<uint32_t>((n + 127) / 128, 1184u), 128>>>(
            static_cast<const pt_material*>(s->dev.materials), static_cast<uint32_t>(s->host.materials.size()), din, n, dout);
        e = cudaMemcpy(out_host, dout, static_cast<size_t>(n) * 16, cudaMemcpyDeviceToHost);
    }
    cudaFree(din);
    cudaFree(dout);
    if (e != cudaSuccess) { set_error(std::string("bsdf eval failed: ") + cudaGetErrorString(e)); return PT_ERR_CUDA; }
    return PT_OK;
}

}  // namespace ptb

namespace ptb {

int current_device(int* dev) {
    PT_CU(cudaGetDevice(dev));
    return PT_OK;
}

int device_sync(int device) {
    if (int rc = ensure_device(device)) return rc;
    PT_CU(cudaDeviceSynchronize());
    return PT_OK;
}

}  // namespace ptb

// ---------------------------------------------------------------------------
// Guide handles
// ---------------------------------------------------------------------------
struct pt_guide {
    ptb::GuideState g;
};

namespace ptb {
inline const GuideState& guide_state(const pt_guide* h) { return h->g; }
}  // namespace ptb

#include "batch.cuh"

namespace ptb {

// 4 warps; its dynamic shared memory (weights + 4 output tiles) stays under
// the 48 KB that needs no opt-in.
constexpr int kGEvalSmem = kGSmemW * 2 + 4 * 16 * kGOutPad * 4;
static_assert(kGEvalSmem <= 48 * 1024, "guide eval shared memory");
__global__ void __launch_bounds__(128) k_guide_eval(GuideNet net, const float* qd, uint32_t n, float* out) {
    extern __shared__ __align__(16) unsigned char g_smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(g_smem);
    float* srow = reinterpret_cast<float*>(g_smem + kGSmemW * sizeof(__nv_bfloat16));
    load_weights_smem(net, sw);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    float* my = srow + warp * 16 * kGOutPad;
    const uint32_t tiles = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * 4 + warp; tile < tiles; tile += gridDim.x * 4) {
        auto pos = [&](uint32_t r) {
            return r < n ? guide_normalise(net, mk(qd[6 * r], qd[6 * r + 1], qd[6 * r + 2])) : mk(0.5f);
        };
        float o[6][4];
        warp_forward(net, sw, pos(tile * 16 + g), pos(tile * 16 + g + 8), o);
#pragma unroll
        for (int nt = 0; nt < 6; ++nt) {
            my[g * kGOutPad + nt * 8 + 2 * c] = o[nt][0];
            my[g * kGOutPad + nt * 8 + 2 * c + 1] = o[nt][1];
            my[(g + 8) * kGOutPad + nt * 8 + 2 * c] = o[nt][2];
            my[(g + 8) * kGOutPad + nt * 8 + 2 * c + 1] = o[nt][3];
        }
        __syncwarp();
        if (lane < 16 && tile * 16 + lane < n) {
            const uint32_t r = tile * 16 + lane;
            alignas(16) float mix[kGMix];
            mixture_record(my + lane * kGOutPad, mix);
            out[r] = mix_pdf(mix, normalize(mk(qd[6 * r + 3], qd[6 * r + 4], qd[6 * r + 5])));
        }
        __syncwarp();
    }
}

int guide_create(pt_scene* s, uint32_t seed, pt_guide** out) {
    if (!s->dev.uploaded) { set_error("guide: scene not uploaded"); return PT_ERR_STATE; }
    pt_guide* h = new pt_guide();
    const int rc = guide_init(h->g, s->dev.device, s->tables.root_lo, s->tables.root_hi, seed);
    if (rc) { guide_free(h->g); delete h; return rc; }
    *out = h;
    return PT_OK;
}

void guide_destroy(pt_guide* h) {
    guide_free(h->g);
    delete h;
}

void guide_set_lr(pt_guide* h, float lr) { h->g.lr = lr; }
int guide_set_schedule(pt_guide* h, float ema, float lr_half_life, float lr_floor) {
    GuideNet& n = h->g.net;
    if (ema > 0.0f && n.ema == 0.0f) {
        // averaging starts from the current parameters
        if (int rc = ensure_device(h->g.device)) return rc;
        const size_t ng = static_cast<size_t>(kGLevels) * kGTable;
        PT_CU(cudaDeviceSynchronize());
        PT_CU(cudaMemcpy(n.grid_ema, n.grid_master, ng * sizeof(float2), cudaMemcpyDeviceToDevice));
        PT_CU(cudaMemcpy(n.grid_inf, n.grid, ng * sizeof(uint2), cudaMemcpyDeviceToDevice));
        PT_CU(cudaMemcpy(n.w_ema, n.w_master, kGWeights * sizeof(float), cudaMemcpyDeviceToDevice));
        PT_CU(cudaMemcpy(n.w_inf, n.w, kGWeights * sizeof(__nv_bfloat16), cudaMemcpyDeviceToDevice));
    }
    n.ema = ema;
    h->g.lr_half_life = lr_half_life;
    h->g.lr_floor = lr_floor;
    return PT_OK;
}
void guide_set_alpha(pt_guide* h, float alpha) { h->g.alpha = alpha; }
void guide_set_inference(pt_guide* h, int kind) { h->g.infer = kind == PT_GUIDE_INFER_DEFAULT ? kGuideInferDefault : kind; }
void guide_set_training(pt_guide* h, int paths_per_step, uint32_t samples_per_step) {
    h->g.paths_per_step = paths_per_step > 0 ? paths_per_step : kGuideMinibatchPaths;
    h->g.samples_per_step = samples_per_step;
}

int guide_info(const pt_guide* h, uint32_t* steps, uint32_t* samples) {
    uint32_t c[2] = {0, 0};
    if (int rc = ensure_device(h->g.device)) return rc;
    PT_CU(cudaDeviceSynchronize());
    if (h->g.step) PT_CU(cudaMemcpy(&c[1], h->g.step, 4, cudaMemcpyDeviceToHost));
    if (h->g.counters) PT_CU(cudaMemcpy(&c[0], h->g.counters, 4, cudaMemcpyDeviceToHost));
    if (steps) *steps = c[1];
    if (samples) *samples = c[0];
    return PT_OK;
}

int guide_loss(const pt_guide* h, float* loss) {
    if (int rc = ensure_device(h->g.device)) return rc;
    PT_CU(cudaDeviceSynchronize());
    float l[3] = {0, 0, 0};
    if (h->g.net.loss) PT_CU(cudaMemcpy(l, h->g.net.loss, sizeof(l), cudaMemcpyDeviceToHost));
    *loss = l[2];
    return PT_OK;
}

int integrator_set_guide(pt_integrator* integ, pt_guide* h, int mode) {
    if (!integ->wf) integ->wf = new Wavefront();
    integ->wf->guide = h ? &h->g : nullptr;
    if (h) h->g.mode = mode;
    if (integ->wf->graph) { cudaGraphExecDestroy(integ->wf->graph); integ->wf->graph = nullptr; integ->wf->graph_key.clear(); }
    return PT_OK;
}

int guide_get_params(const pt_guide* h, float* weights, float* grid, float* meta) {
    if (int rc = ensure_device(h->g.device)) return rc;
    PT_CU(cudaDeviceSynchronize());
    const GuideNet net = guide_infer_view(h->g.net);
    std::vector<__nv_bfloat16> wb(kGWeights);
    PT_CU(cudaMemcpy(wb.data(), net.w, kGWeights * sizeof(__nv_bfloat16), cudaMemcpyDeviceToHost));
    for (int i = 0; i < kGWeights; ++i) weights[i] = __bfloat162float(wb[i]);
    if (grid) {
        const size_t ng = static_cast<size_t>(kGLevels) * kGTable;
        std::vector<__half2> gh(2 * ng);
        PT_CU(cudaMemcpy(gh.data(), net.grid, ng * sizeof(uint2), cudaMemcpyDeviceToHost));
        for (size_t i = 0; i < ng; ++i) {
            const float2 v = __half22float2(gh[2 * i]);
            grid[2 * i] = v.x;
            grid[2 * i + 1] = v.y;
        }
    }
    if (meta) {
        for (int a = 0; a < 3; ++a) { meta[a] = h->g.net.lo[a]; meta[3 + a] = h->g.net.inv_ext[a]; }
        for (int l = 0; l < kGLevels; ++l) meta[6 + l] = h->g.net.scale[l];
        meta[6 + kGLevels] = static_cast<float>(h->g.net.dense_limit);
    }
    return PT_OK;
}

int guide_backward(pt_guide* h, const float* samples, uint32_t n, float* wgrad, float* ggrad) {
    if (n > static_cast<uint32_t>(kGTrainRows)) {
        set_error("guide backward: at most " + std::to_string(kGTrainRows) + " samples");
        return PT_ERR_INVALID;
    }
    if (int rc = ensure_device(h->g.device)) return rc;
    GuideSample* ds = nullptr;
    uint32_t* dn = nullptr;
    void* store = nullptr;   // the row store and the partial sums of the weight gradient
    PT_CU(cudaMalloc(&ds, std::max<size_t>(n, 1) * sizeof(GuideSample)));
    if (cudaMalloc(&dn, 4) != cudaSuccess ||
        cudaMalloc(&store, kGRowStoreElems * sizeof(__nv_bfloat16) +
                               static_cast<size_t>(kGDwChunks) * kGWeights * sizeof(float)) != cudaSuccess) {
        cudaFree(ds); cudaFree(dn); cudaGetLastError(); set_error("alloc"); return PT_ERR_NOMEM;
    }
    __nv_bfloat16* rows = static_cast<__nv_bfloat16*>(store);
    float* partial = reinterpret_cast<float*>(rows + kGRowStoreElems);
    const size_t ng = static_cast<size_t>(kGLevels) * kGTable;
    cudaError_t e = cudaMemcpy(ds, samples, static_cast<size_t>(n) * sizeof(GuideSample), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(dn, &n, 4, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(h->g.net.w_grad, 0, kGWeights * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(h->g.net.grid_grad, 0, ng * 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) {
        GuideNet net = h->g.net;
        net.loss_fix = nullptr;   // leave the training-loss record alone
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->g.device);
        const uint32_t cap = guide_step_cap(0u);
        k_guide_train<<<sms, 32 * kGTrainWarps, kGTrainSmem>>>(net, ds, dn, n, 0, 1, cap, rows);
        k_guide_dw<<<dim3(kGDwChunks, 4), 128>>>(dn, n, 0, 1, cap, rows, partial);
        k_guide_dw_reduce<<<(kGWeights + 255) / 256, 256>>>(dn, n, 0, 1, cap, partial, net.w_grad);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaDeviceSynchronize();
    }
    // gradients come back as floats (fixed point on the device)
    if (e == cudaSuccess) {
        std::vector<unsigned long long> wg(kGWeights);
        e = cudaMemcpy(wg.data(), h->g.net.w_grad, kGWeights * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
        for (int i = 0; i < kGWeights && e == cudaSuccess; ++i) wgrad[i] = g_unfix(wg[i]);
    }
    if (e == cudaSuccess && ggrad) {
        std::vector<unsigned long long> gg(ng * 2);
        e = cudaMemcpy(gg.data(), h->g.net.grid_grad, ng * 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
        for (size_t i = 0; i < ng * 2 && e == cudaSuccess; ++i) ggrad[i] = g_unfix(gg[i]);
    }
    // leave the optimiser state as it was
    cudaMemset(h->g.net.w_grad, 0, kGWeights * sizeof(unsigned long long));
    cudaMemset(h->g.net.grid_grad, 0, ng * 2 * sizeof(unsigned long long));
    cudaFree(ds);
    cudaFree(dn);
    cudaFree(store);
    if (e != cudaSuccess) { set_error(std::string("guide backward: ") + cudaGetErrorString(e)); return PT_ERR_CUDA; }
    return PT_OK;
}

// q(dir | pos) of query r from its mixture record (split inference kinds).
__global__ void __launch_bounds__(256) k_guide_mix_pdf(const float* __restrict__ mix, const float* __restrict__ qd,
                                                       uint32_t n, float* __restrict__ out) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x)
        out[r] = mix_pdf(mix + static_cast<size_t>(r) * kGMix, normalize(mk(qd[6 * r + 3], qd[6 * r + 4], qd[6 * r + 5])));
}

int guide_eval(pt_guide* h, const float* qd, uint32_t n, float* out) {
    if (int rc = ensure_device(h->g.device)) return rc;
    if (n == 0) return PT_OK;
    GuideState g = h->g;
    g.net = guide_infer_view(h->g.net);
    const bool split = g.infer != PT_GUIDE_INFER_FUSED;
    int sms = 0;
    PT_CU(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g.device));
    // queries, densities, and for the split kinds the feature tiles, the
    // mixture records and an error word: one allocation
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_q = al(static_cast<size_t>(n) * 24), b_out = al(static_cast<size_t>(n) * 4);
    const size_t b_feat = split ? al(static_cast<size_t>(guide_feat_rows(n)) * kGIn * 2) : 0;
    const size_t b_mix = split ? al(static_cast<size_t>(n) * kGMix * 4) : 0;
    char* buf = nullptr;
    PT_CU(cudaMalloc(&buf, b_q + b_out + b_feat + b_mix + 256));
    float* dq = reinterpret_cast<float*>(buf);
    float* dout = reinterpret_cast<float*>(buf + b_q);
    unsigned char* feat = reinterpret_cast<unsigned char*>(buf + b_q + b_out);
    float* mix = reinterpret_cast<float*>(buf + b_q + b_out + b_feat);
    uint32_t* derr = reinterpret_cast<uint32_t*>(buf + b_q + b_out + b_feat + b_mix);
    cudaError_t e = cudaMemcpy(dq, qd, static_cast<size_t>(n) * 24, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(derr, 0, 4);
    if (e == cudaSuccess) {
        if (!split) {
            k_guide_eval<<<sms, 128, kGEvalSmem>>>(g.net, dq, n, dout);
        } else {
            if (g.net.quad) k_guide_quad<<<sms * 2, 256>>>(g.net);
            k_guide_encode<<<sms * 8, 256>>>(g.net, nullptr, 0, 0u, nullptr, nullptr, nullptr, dq, n, feat);
            if (g.infer == PT_GUIDE_INFER_SPLIT_MMA)
                k_guide_mlp_mma<<<sms * kGInferBlocksPerSm, 32 * kGInferWarps, kGInferSmem>>>(g.net, nullptr, 0, 0u, n,
                                                                                          feat, mix);
            else
                k_guide_mlp_tc<<<sms * kGTcBlocksPerSm, kGTcThreads, kGTcSmem>>>(g.net, nullptr, 0, 0u, n, feat, mix,
                                                                               derr);
            k_guide_mix_pdf<<<sms * 4, 256>>>(mix, dq, n, dout);
        }
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpy(out, dout, static_cast<size_t>(n) * 4, cudaMemcpyDeviceToHost);
    }
    uint32_t err = 0;
    if (e == cudaSuccess && split) e = cudaMemcpy(&err, derr, 4, cudaMemcpyDeviceToHost);
    cudaFree(buf);
    if (e != cudaSuccess) { set_error(std::string("guide eval: ") + cudaGetErrorString(e)); return PT_ERR_CUDA; }
    if (err) { set_error("guide eval: the network's tensor-core wait timed out"); return PT_ERR_DEVICE; }
    return PT_OK;
}

}  // namespace ptb
