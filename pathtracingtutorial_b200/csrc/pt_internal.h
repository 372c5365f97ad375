// pt_internal.h -- shared host/device definitions of the B200 path tracer.
//
// Vector math, the device scene view handed to every kernel by value, and the
// traversal layout of the BVH.  Shading math follows the reference formulas;
// the traversal/intersection arithmetic is written with explicitly rounded
// operations (x_add/x_sub/x_mul) so that no FMA contraction can change a bit:
// hit triangle ids must equal those of the reference's IEEE host build.
#pragma once

#include <stdint.h>
#include <float.h>
#include <math.h>
#include <string.h>

#include <vector_types.h>

#include "../../include/pt_b200.h"

#ifdef __CUDACC__
#  define PT_HD __host__ __device__ __forceinline__
#  define PT_DEV __device__ __forceinline__
#else
#  define PT_HD inline
#  define PT_DEV inline
#endif

namespace ptb {

constexpr float kPi     = 3.14159265358979323846f;
constexpr float kInvPi  = 0.31830988618379067154f;
constexpr float kInv2Pi = 0.15915494309189533577f;
constexpr float kTwoPi  = 6.28318530717958647692f;

// Traversal stack bound.  The reference uses 32 entries with no overflow check
// (Part_2/src/accel/bvh_traversal.cuh:14,52,107); this stack holds only deferred
// far children, so it needs at most (tree depth) entries.  Scenes whose BVH is
// deeper than this are rejected at build time, and the kernels still guard.
constexpr int kStackDepth = 64;
// Default path slots of the wavefront (pt_render_settings.paths_in_flight = 0):
// about 260 B of path state each with two light slots (35 GB of the B200's
// 180 GB; a pass allocates only what its pixels x samples need, and halves
// itself when the device cannot hold it).  Larger passes amortise the short
// launches of the deep bounces: on the 1080p 256-spp workload 2^25 / 2^26 /
// 2^27 slots render at 1621 / 1684 / 1719 Mrays/s.  A guide that samples
// adds its mixture per path (160 B; 10.7 GB at 2^26 paths).
constexpr int64_t kDefaultPathsInFlight = int64_t(1) << 27;
constexpr int64_t kGuidedPathsInFlight = int64_t(1) << 26;
// While a guide trains, passes stay small: every pass ends with optimiser
// steps, so smaller passes mean more steps per sample.
constexpr int64_t kTrainingPathsInFlight = int64_t(1) << 20;

// Device error word bits.
enum : uint32_t {
    kErrStackOverflow = 1u << 0,
    kErrQueueOverflow = 1u << 1,
    kErrNanRadiance   = 1u << 2,
    kErrGuideTimeout  = 1u << 3,   // a tensor-core wait of the guide's network gave up
};

// ---------------------------------------------------------------------------
// Explicitly rounded float ops (never contracted into FMA).
// ---------------------------------------------------------------------------
#if defined(__CUDA_ARCH__)
PT_HD uint32_t __float_as_uint_hd(float f) { return __float_as_uint(f); }
PT_HD float __uint_as_float_hd(uint32_t u) { return __uint_as_float(u); }
#else
PT_HD uint32_t __float_as_uint_hd(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
PT_HD float __uint_as_float_hd(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
#endif

#if defined(__CUDA_ARCH__)
PT_HD float x_add(float a, float b) { return __fadd_rn(a, b); }
PT_HD float x_sub(float a, float b) { return __fsub_rn(a, b); }
PT_HD float x_mul(float a, float b) { return __fmul_rn(a, b); }
PT_HD float x_rcp(float a) { return __frcp_rn(a); }
PT_HD float x_div(float a, float b) { return __fdiv_rn(a, b); }
PT_HD double xd_mul(double a, double b) { return __dmul_rn(a, b); }
PT_HD double xd_sub(double a, double b) { return __dsub_rn(a, b); }
#else
PT_HD float x_add(float a, float b) { return a + b; }
PT_HD float x_sub(float a, float b) { return a - b; }
PT_HD float x_mul(float a, float b) { return a * b; }
PT_HD float x_rcp(float a) { return 1.0f / a; }
PT_HD float x_div(float a, float b) { return a / b; }
PT_HD double xd_mul(double a, double b) { return a * b; }
PT_HD double xd_sub(double a, double b) { return a - b; }
#endif

// ---------------------------------------------------------------------------
// f3: plain three-float vector used by the kernels.
// ---------------------------------------------------------------------------
struct f3 { float x, y, z; };

PT_HD f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
PT_HD f3 mk(float s) { return mk(s, s, s); }
PT_HD f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
PT_HD f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
PT_HD f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
PT_HD f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
PT_HD f3 operator*(f3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
PT_HD f3 operator*(float s, f3 a) { return mk(a.x * s, a.y * s, a.z * s); }
PT_HD f3 operator/(f3 a, float s) { return mk(a.x / s, a.y / s, a.z / s); }
PT_HD f3& operator+=(f3& a, f3 b) { a = a + b; return a; }
PT_HD f3& operator*=(f3& a, f3 b) { a = a * b; return a; }
PT_HD f3& operator*=(f3& a, float s) { a = a * s; return a; }
PT_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
PT_HD f3 cross(f3 a, f3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
PT_HD float length(f3 a) { return sqrtf(dot(a, a)); }
// vec3::normalize (Part_2/src/math/vecmath.h:45): zero stays zero.
PT_HD f3 normalize(f3 a) { float l = length(a); return l > 0.0f ? a / l : mk(0.0f); }
PT_HD bool is_zero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
PT_HD f3 reflect(f3 i, f3 n) { return i - 2.0f * dot(i, n) * n; }
PT_HD float max3(f3 a) { return fmaxf(fmaxf(a.x, a.y), a.z); }
PT_HD float luminance(f3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }
PT_HD f3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

// Orthonormal basis from a normal (Frame, Part_2/src/math/frame.h:18-23).
struct Frame {
    f3 t, b, n;
};
PT_HD Frame make_frame(f3 n) {
    f3 helper = fabsf(n.x) > 0.999f ? mk(0.0f, 0.0f, 1.0f) : mk(1.0f, 0.0f, 0.0f);
    Frame f;
    f.n = n;
    f.t = normalize(cross(n, helper));
    f.b = normalize(cross(n, f.t));
    return f;
}
PT_HD f3 to_world(const Frame& f, f3 v) { return v.x * f.t + v.y * f.b + v.z * f.n; }
PT_HD f3 to_local(const Frame& f, f3 v) { return mk(dot(v, f.t), dot(v, f.b), dot(v, f.n)); }

// ---------------------------------------------------------------------------
// Traversal layout.
//
// The reference tree (binary, DFS order, 32-byte nodes) is re-laid out so that
// every inner node carries the boxes of BOTH children (64 bytes, four 16-byte
// vector loads).  Child refs: bit 31 set = leaf whose first triangle record is
// (ref & 0x7fffffff); otherwise the index of an inner node.  meta packs the
// child-order rule of the reference (parent's max-extent axis and whether the
// left child's centroid is below the right's, bvh_traversal.cuh:81-92).
// ---------------------------------------------------------------------------
constexpr uint32_t kLeafBit = 0x80000000u;

struct alignas(16) InnerNode {
    float c0lo[3]; float c0hi_x;
    float c0hi_yz[2]; float c1lo_xy[2];
    float c1lo_z; float c1hi[3];
    uint32_t ref0, ref1, meta, pad;   // meta: bits 0-1 axis, bit 2 "left centroid < right centroid"
};
static_assert(sizeof(InnerNode) == 64, "InnerNode must be 64 bytes");

// Triangle record in BVH leaf order: v0 and the two edges precomputed exactly
// as the reference computes them per test (v1 - v0, v2 - v0).  w of the third
// vector: bit 0 = last triangle of its leaf.
struct alignas(16) TriRecord {
    float v0[3]; float e1x;
    float e1yz[2]; float e2xy[2];
    float e2z; uint32_t flags; uint32_t pad[2];
};
static_assert(sizeof(TriRecord) == 48, "TriRecord must be 48 bytes");

// ---------------------------------------------------------------------------
// Device scene view (DeviceSceneView + DeviceLightView,
// Part_2/src/scene/device_scene.h:29-67), passed by value.
// ---------------------------------------------------------------------------
struct DeviceScene {
    const InnerNode*  inner;
    const TriRecord*  tris;
    float             root_lo[3];
    float             root_hi[3];
    uint32_t          root_ref;        // kLeafBit|first for a leaf root, else 0
    uint32_t          num_faces;

    const pt_vertex*   vertices;
    const pt_face*     faces;          // BVH order
    const pt_material* materials;
    uint32_t           num_materials;

    // lights
    const pt_emissive_ref* emissive;
    uint32_t               num_emissive;
    const float*           tri_light_pmf;   // per face
    const pt_alias_entry*  tri_alias;
    const float*           env_pmf;
    const pt_alias_entry*  env_alias;
    uint32_t               num_env_texels;
    int32_t                env_w, env_h;
    unsigned long long     env_tex;         // cudaTextureObject_t (0 = none)
    const pt_punctual_light* punctual;
    uint32_t               num_punctual;
    // material textures (float4, bilinear, normalized coordinates)
    const unsigned long long* textures;     // cudaTextureObject_t per texture (0 = no image)
    uint32_t               num_textures;
};

// Ray as stored in queues: origin (w unused) and direction (w = tmax for shadow rays).
struct alignas(16) RayO { float x, y, z, w; };

}  // namespace ptb
