// guide.cuh -- learned path guiding (no reference counterpart; included by
// integrator.cu).
//
// A position-conditioned directional distribution q(w | x) is learned online
// from the tracer's own samples and mixed with BSDF sampling by one-sample MIS:
// with probability alpha the direction is drawn from q, otherwise from the
// BSDF's sampler (density pB), and the plain integrator's weight f / pdf is
// scaled by pB / (alpha q + (1 - alpha) pB), so the estimator keeps the
// expectation of the BSDF-only integrator wherever pB > 0 -- also where the
// BSDF's pdf is not its sampler's density.  Light samples and emitter hits
// keep the plain integrator's MIS weights.  Vertices that can produce delta
// samples (roughness < 0.01) are never guided.
//
// Network: multi-resolution hash-grid encoding of the position (16 levels x 2
// features, 2^19 FP16 entries per level, trilinear) -> 3 hidden layers of 64
// (ReLU) -> 40 outputs = 8 von Mises-Fisher lobes x (mean direction 3,
// concentration 1, mixture logit 1).  BF16 weights, FP32 accumulation on the
// tensor cores (mma.sync m16n8k16): each warp carries 16 queries through all
// layers in registers (an accumulator fragment pair is the next layer's A
// fragment), weights sit in shared memory with padded rows.
//
// Training minimises the KL divergence from the normalised cosine-weighted
// incident radiance to q with the one-sample estimate
// -L_in(w) |cos| / p(w) * log q(w | x)  per recorded path vertex, in
// minibatches interleaved over the whole image; the backward pass runs on the
// tensor cores too (dX = dY W per warp tile in the forward/backward kernel,
// dW = dY^T X as a split-K GEMM over the step's rows in k_guide_dw), and Adam
// updates FP32 master copies.  Training is deterministic: the samples are
// stored in path order (count, scan, write), the weight gradient is summed in
// fixed row chunks in a fixed order, and the hash-grid gradient is scattered
// in 64-bit fixed point (units of 2^-40) with integer atomics, whose result
// does not depend on the order in which they land.

#include <cuda_bf16.h>
#include <cuda_fp16.h>

namespace ptb {

constexpr int kGLevels = 16;
constexpr int kGFeat = 2;
constexpr int kGLog2T = 19;
constexpr int kGTable = 1 << kGLog2T;
constexpr int kGIn = kGLevels * kGFeat;   // 32
constexpr int kGHid = 64;
constexpr int kGLobes = 8;
constexpr int kGOut = 40;                 // used outputs
constexpr int kGOutPad = 48;              // 6 n-tiles of 8
constexpr int kGMix = 40;                 // floats per mixture record: 8 x (kappa mu xyz, log factor) + 8 weights
constexpr float kGuideAlpha = 0.5f;        // default probability of sampling the mixture
constexpr int kGuideMinibatchPaths = 1 << 15;
// Training samples per optimiser step at most (an evenly spread subset of the
// step's share of a pass).  On the hidden-light room (1024 x 1024, 64 training
// spp) all samples (about 10^5 a step) cost 3.0 s of training and gave relMSE
// 0.00214 at 256 guided spp; 65,536 a step cost 2.25 s for 0.00233; 32,768
// cost 2.0 s for 0.0034.
constexpr uint32_t kGuideStepSamples = 65536;
// Parameter averaging factor per optimiser step unless pt_guide_set_schedule
// sets another.  Measured on the hidden-light room (1024 x 1024, 64 training
// spp, time to relMSE 1e-3 against the FP64 crop, six network seeds each):
// no averaging 7.21 s (relMSE x spp after training 0.65, sd 0.09), 0.99 6.89
// s (0.62, sd 0.14), 0.995 6.61 s (0.58, sd 0.05), 0.998 7.40 s (0.71, three
// seeds); a halving learning rate (every 512 steps) 7.81 s.
constexpr float kGuideEma = 0.995f;
// Inference kind used unless pt_guide_set_inference chooses another.  Network
// stage time of a 64-spp guided render of the hidden-light room at 1024 x 1024:
// fused 124.7 ms, encoding + mma.sync MLP 114.6 ms, encoding + tcgen05 MLP
// 98.2 ms (with the exactly rounded exponentials and logarithms in the
// mixture records and without the dense levels' four-corner table: 160.5 /
// 152.0 / 114.6 ms).
constexpr int kGuideInferDefault = PT_GUIDE_INFER_SPLIT_TC;

// Optimiser steps per training pass of `paths` paths: one per
// `paths_per_step` paths (2^15 by default, about 10^5 samples), 1 .. 32.
inline int guide_minibatches(int64_t paths, int64_t paths_per_step = kGuideMinibatchPaths) {
    return static_cast<int>(std::min<int64_t>(32, std::max<int64_t>(1, paths / std::max<int64_t>(1, paths_per_step))));
}

// layer l: out x in, row-major, rows padded to in + 8 bf16 in shared memory
__host__ __device__ constexpr int g_in(int l) { return l == 0 ? kGIn : kGHid; }
__host__ __device__ constexpr int g_out(int l) { return l == 3 ? kGOutPad : kGHid; }
__host__ __device__ constexpr int g_woff(int l) {   // offset of layer l in the packed (unpadded) weights
    return l == 0 ? 0 : (l == 1 ? kGHid * kGIn : (l == 2 ? kGHid * kGIn + kGHid * kGHid : kGHid * kGIn + 2 * kGHid * kGHid));
}
constexpr int kGWeights = kGHid * kGIn + 2 * kGHid * kGHid + kGOutPad * kGHid;   // 13312
__host__ __device__ constexpr int g_sld(int l) { return g_in(l) + 8; }               // padded smem row
__host__ __device__ constexpr int g_soff(int l) {
    return l == 0 ? 0 : (l == 1 ? kGHid * g_sld(0) : (l == 2 ? kGHid * g_sld(0) + kGHid * g_sld(1)
                                                              : kGHid * g_sld(0) + 2 * kGHid * g_sld(1)));
}
constexpr int kGSmemW = kGHid * (kGIn + 8) + 2 * kGHid * (kGHid + 8) + kGOutPad * (kGHid + 8);   // bf16 elements

struct GuideNet {
    uint2*          grid;        // kGLevels * kGTable FP16 pairs (inference copy): entry e holds the two
                                 // features of e and of (e + 1) mod kGTable, the corner one step along x
    float2*         grid_master; // FP32 master
    unsigned long long* grid_grad;   // 2 per entry, fixed point (kGFix)
    float2*         grid_m;
    float2*         grid_v;
    __nv_bfloat16*  w;           // kGWeights (inference copy), layer-packed [out][in]
    float*          w_master;
    unsigned long long* w_grad;  // kGWeights, fixed point (kGFix)
    float*          w_m;
    float*          w_v;
    float           lo[3];       // scene bounds (positions mapped to [0,1]^3)
    float           inv_ext[3];
    float           scale[kGLevels];
    uint32_t        dense_limit; // levels with (res+1)^3 <= table use direct indexing
    // Four-corner table of the dense levels for the encoding kernel: entry
    // x + y res + z res^2 of level l (at quad + quad_off[l]) holds the FP16
    // feature pairs of corners (x, y), (x + 1, y), (x, y + 1), (x + 1, y + 1)
    // of layer z, 16 bytes, made from the pair table before each inference
    // (k_guide_quad); null: the encoding reads the pair table.
    uint4*          quad;
    uint32_t        quad_off[kGLevels];
    float*          loss;        // [2] mean loss of the last pass
    unsigned long long* loss_fix;    // [0] sum of w (-log q) (kGLossFix units), [1] samples
    // Parameter averaging (ema > 0): renders sample with copies made from an
    // exponential moving average of the parameters, updated after every
    // optimiser step, while training runs on the parameters themselves.
    float           ema;         // averaging factor (0: off)
    float2*         grid_ema;    // averages (FP32)
    float*          w_ema;
    uint2*          grid_inf;    // FP16 pair table and BF16 weights made from the averages
    __nv_bfloat16*  w_inf;
};

// The network as the renders' inference kernels read it: the averaged copies
// when averaging is on, else the parameters the training kernels use.
__host__ __device__ inline GuideNet guide_infer_view(const GuideNet& n) {
    GuideNet v = n;
    if (n.ema > 0.0f) { v.grid = n.grid_inf; v.w = n.w_inf; }
    return v;
}

// Fixed-point gradient sums: a contribution x is added as round(x * 2^40)
// (clamped to +-2^20, far above any gradient of a mean loss), so a sum holds
// up to +-2^23 with a resolution of 2^-40.  Loss sums use 2^-20 units.
constexpr float kGFix = 1099511627776.0f;              // 2^40
constexpr double kGFixInv = 1.0 / 1099511627776.0;
constexpr float kGLossFix = 1048576.0f;                // 2^20
__host__ __device__ __forceinline__ float g_unfix(unsigned long long v) {
    return static_cast<float>(static_cast<double>(static_cast<long long>(v)) * kGFixInv);
}
#if defined(__CUDACC__)
__device__ __forceinline__ unsigned long long g_fix(float x) {
    x = fminf(fmaxf(x, -1048576.0f), 1048576.0f);
    return static_cast<unsigned long long>(__float2ll_rn(x * kGFix));
}
#endif

// ---------------------------------------------------------------------------
// mma helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<const uint32_t*>(&v);
}
__device__ __forceinline__ void mma_bf16(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Y(16 x OUT) = X(16 x IN) W^T for one warp; X given as A fragments per k-tile,
// W in shared memory ([out][in], padded rows).  acc[nt][4] = C fragments.
template <int IN, int OUT>
__device__ __forceinline__ void warp_layer(const uint32_t (&a)[IN / 16][4], const __nv_bfloat16* W,
                                           float (&acc)[OUT / 8][4]) {
    constexpr int LD = IN + 8;
    const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
#pragma unroll
    for (int nt = 0; nt < OUT / 8; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
        const __nv_bfloat16* row = W + (nt * 8 + g) * LD + 2 * c;
#pragma unroll
        for (int kt = 0; kt < IN / 16; ++kt) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(row + kt * 16);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + kt * 16 + 8);
            mma_bf16(acc[nt], a[kt], b0, b1);
        }
    }
}

// C fragments (with ReLU) -> A fragments of the next layer.
template <int N>
__device__ __forceinline__ void relu_to_a(const float (&acc)[N / 8][4], uint32_t (&a)[N / 16][4]) {
#pragma unroll
    for (int kt = 0; kt < N / 16; ++kt) {
        a[kt][0] = pack_bf16(fmaxf(acc[2 * kt][0], 0.0f), fmaxf(acc[2 * kt][1], 0.0f));
        a[kt][1] = pack_bf16(fmaxf(acc[2 * kt][2], 0.0f), fmaxf(acc[2 * kt][3], 0.0f));
        a[kt][2] = pack_bf16(fmaxf(acc[2 * kt + 1][0], 0.0f), fmaxf(acc[2 * kt + 1][1], 0.0f));
        a[kt][3] = pack_bf16(fmaxf(acc[2 * kt + 1][2], 0.0f), fmaxf(acc[2 * kt + 1][3], 0.0f));
    }
}

// ---------------------------------------------------------------------------
// Hash-grid encoding
// ---------------------------------------------------------------------------
// Corner (x, y, z) of a level: x + y res + z res^2 on the dense levels, and
// x + (y P1 xor z P2) on the hashed ones -- x is added outside the hash, so
// the two corners of a cell edge along x are neighbouring table entries (one
// 32-byte sector holds eight) and a cell's eight corners touch about four
// sectors instead of eight.
__device__ __forceinline__ uint32_t grid_index(const GuideNet& net, int level, uint32_t x, uint32_t y, uint32_t z) {
    const uint32_t res = static_cast<uint32_t>(net.scale[level]) + 2u;
    if (static_cast<uint32_t>(level) < net.dense_limit) return (x + y * res + z * res * res) & (kGTable - 1);
    return (x + ((y * 2654435761u) ^ (z * 805459861u))) & (kGTable - 1);
}

// Trilinear features of one level at normalised position p.  (Gathers that
// bypass L1, ld.global.cg, made the encoding kernel 1.3x slower: 18 % of its
// gathers hit in L1.)
__device__ __forceinline__ float2 encode_level(const GuideNet& net, int level, f3 p) {
    const float s = net.scale[level];
    const float fx = p.x * s + 0.5f, fy = p.y * s + 0.5f, fz = p.z * s + 0.5f;
    const float bx = floorf(fx), by = floorf(fy), bz = floorf(fz);
    const float tx = fx - bx, ty = fy - by, tz = fz - bz;
    const uint32_t ix = static_cast<uint32_t>(bx), iy = static_cast<uint32_t>(by), iz = static_cast<uint32_t>(bz);
    const uint2* tab = net.grid + static_cast<size_t>(level) * kGTable;
    float2 r = make_float2(0.0f, 0.0f);
    // one 8-byte load per cell edge along x: both corners of the edge
#pragma unroll
    for (int e = 0; e < 4; ++e) {
        const uint32_t cy = e & 1, cz = e >> 1;
        const uint2 pr = __ldg(tab + grid_index(net, level, ix, iy + cy, iz + cz));
        const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&pr.x));
        const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&pr.y));
        const float w0 = (1.0f - tx) * (cy ? ty : 1.0f - ty) * (cz ? tz : 1.0f - tz);
        const float w1 = tx * (cy ? ty : 1.0f - ty) * (cz ? tz : 1.0f - tz);
        r.x += w0 * f0.x;
        r.y += w0 * f0.y;
        r.x += w1 * f1.x;
        r.y += w1 * f1.y;
    }
    return r;
}

__device__ __forceinline__ f3 guide_normalise(const GuideNet& net, f3 x) {
    return mk(fminf(fmaxf((x.x - net.lo[0]) * net.inv_ext[0], 0.0f), 1.0f),
              fminf(fmaxf((x.y - net.lo[1]) * net.inv_ext[1], 0.0f), 1.0f),
              fminf(fmaxf((x.z - net.lo[2]) * net.inv_ext[2], 0.0f), 1.0f));
}

// A fragments of the encoded inputs for this warp's rows g and g+8.
__device__ __forceinline__ void encode_a(const GuideNet& net, f3 p0, f3 p1, uint32_t (&a)[2][4]) {
    const int c = threadIdx.x & 3;
#pragma unroll
    for (int kt = 0; kt < 2; ++kt) {
        const int la = 8 * kt + c, lb = 8 * kt + 4 + c;
        const float2 e0a = encode_level(net, la, p0), e1a = encode_level(net, la, p1);
        const float2 e0b = encode_level(net, lb, p0), e1b = encode_level(net, lb, p1);
        a[kt][0] = pack_bf16(e0a.x, e0a.y);
        a[kt][1] = pack_bf16(e1a.x, e1a.y);
        a[kt][2] = pack_bf16(e0b.x, e0b.y);
        a[kt][3] = pack_bf16(e1b.x, e1b.y);
    }
}

__device__ __forceinline__ void load_weights_smem(const GuideNet& net, __nv_bfloat16* sw) {
    for (int l = 0; l < 4; ++l) {
        const int in = g_in(l), out = g_out(l), ld = g_sld(l);
        for (int i = threadIdx.x; i < out * in; i += blockDim.x) {
            const int o = i / in, k = i % in;
            sw[g_soff(l) + o * ld + k] = net.w[g_woff(l) + i];
        }
    }
    __syncthreads();
}

// Forward of one warp's 16 rows; leaves the (linear) outputs in out[6][4].
__device__ __forceinline__ void warp_forward(const GuideNet& net, const __nv_bfloat16* sw, f3 p0, f3 p1,
                                             float (&out)[6][4]) {
    uint32_t a0[2][4];
    encode_a(net, p0, p1, a0);
    float h[8][4];
    uint32_t a[4][4];
    warp_layer<kGIn, kGHid>(a0, sw + g_soff(0), h);
    relu_to_a<kGHid>(h, a);
    warp_layer<kGHid, kGHid>(a, sw + g_soff(1), h);
    relu_to_a<kGHid>(h, a);
    warp_layer<kGHid, kGHid>(a, sw + g_soff(2), h);
    relu_to_a<kGHid>(h, a);
    warp_layer<kGHid, kGOutPad>(a, sw + g_soff(3), out);
}

// ---------------------------------------------------------------------------
// vMF mixture: raw outputs -> (mu, kappa) x 8, weights x 8
// ---------------------------------------------------------------------------
__device__ __forceinline__ float softplusf(float x) { return x > 15.0f ? x : log1pf(expf(x)); }

__device__ __forceinline__ void raw_to_mixture(const float* raw, float* mix) {
    float mx = -1e30f;
    for (int k = 0; k < kGLobes; ++k) mx = fmaxf(mx, raw[5 * k + 4]);
    float sum = 0.0f;
    for (int k = 0; k < kGLobes; ++k) {
        f3 m = mk(raw[5 * k], raw[5 * k + 1], raw[5 * k + 2]);
        const float l = length(m);
        m = l > 1e-12f ? m / l : mk(0.0f, 0.0f, 1.0f);
        mix[4 * k] = m.x; mix[4 * k + 1] = m.y; mix[4 * k + 2] = m.z;
        mix[4 * k + 3] = fminf(softplusf(raw[5 * k + 3]) + 1e-3f, 5e3f);
        const float e = expf(raw[5 * k + 4] - mx);
        mix[32 + k] = e;
        sum += e;
    }
    for (int k = 0; k < kGLobes; ++k) mix[32 + k] /= sum;
}

// vMF density on the sphere for cos(angle to the mean) c.
__device__ __forceinline__ float vmf_pdf(float kappa, float c) {
    if (kappa < 1e-4f) return 0.25f * kInvPi;
    return kappa / (kTwoPi * (1.0f - expf(-2.0f * kappa))) * expf(kappa * (c - 1.0f));
}

// The mixture as the shading kernels read it (kGMix floats per queue entry):
// lobe k as float4(kappa_k mu_k, b_k) with b_k = log(pi_k kappa_k /
// (2 pi (1 - e^{-2 kappa_k}))) - kappa_k, then the eight weights pi_k.  Then
// pi_k vMF_k(w) = exp(kappa_k mu_k . w + b_k): one exponential per lobe.
// The same function as raw_to_mixture followed by the record's algebra, with
// the hardware's approximate exponential and logarithm: log pi_k = (logit_k
// - max) - log(sum), one logarithm per row; the normalisation factor as
// log(kappa / (1 - e^{-2 kappa})) - log(2 pi).  About a quarter of the
// instructions of the exactly rounded library functions; the densities agree
// with the FP64 oracle to about 1e-6 relative.
__device__ __forceinline__ void mixture_record(const float* raw, float* rec) {
    float mx = -1e30f;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) mx = fmaxf(mx, raw[5 * k + 4]);
    float e[kGLobes];
    float sum = 0.0f;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) {
        e[k] = __expf(raw[5 * k + 4] - mx);
        sum += e[k];
    }
    const float inv_sum = 1.0f / sum, log_sum = __logf(sum);
    constexpr float kLog2Pi = 1.83787706640934548356f;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) {
        const float mxx = raw[5 * k], myy = raw[5 * k + 1], mzz = raw[5 * k + 2];
        const float l2 = mxx * mxx + myy * myy + mzz * mzz;
        const float r = raw[5 * k + 3];
        const float sp = r > 15.0f ? r : __logf(1.0f + __expf(r));
        const float kap = fminf(sp + 1e-3f, 5e3f);   // >= 1e-3
        if (l2 > 1e-24f) {
            const float s = kap * rsqrtf(l2);
            rec[4 * k] = s * mxx;
            rec[4 * k + 1] = s * myy;
            rec[4 * k + 2] = s * mzz;
        } else {
            rec[4 * k] = 0.0f;
            rec[4 * k + 1] = 0.0f;
            rec[4 * k + 2] = kap;
        }
        rec[4 * k + 3] = (raw[5 * k + 4] - mx) - log_sum + __logf(__fdividef(kap, 1.0f - __expf(-2.0f * kap))) -
                         kLog2Pi - kap;
        rec[32 + k] = e[k] * inv_sum;
    }
}

// q(w) = sum_k exp(kappa_k mu_k . w + b_k), with the hardware exponential
// (relative error about 1e-6 at the exponents met here).
__device__ __forceinline__ float mix_pdf(const float* rec, f3 w) {
    const float4* r4 = reinterpret_cast<const float4*>(rec);
    float q = 0.0f;
#pragma unroll
    for (int k = 0; k < kGLobes; ++k) {
        const float4 l = r4[k];
        q += __expf(fmaf(l.x, w.x, fmaf(l.y, w.y, fmaf(l.z, w.z, l.w))));
    }
    return q;
}

__device__ __forceinline__ f3 mix_sample(const float* rec, float u0, float u1, float u2) {
    int k = 0;
    float acc = rec[32];
    while (k < kGLobes - 1 && u0 >= acc) { ++k; acc += rec[32 + k]; }
    const float4 l = reinterpret_cast<const float4*>(rec)[k];
    const f3 km = mk(l.x, l.y, l.z);
    const float kappa = length(km);
    const f3 mu = km / kappa;
    const float c = fminf(fmaxf(1.0f + __logf(u1 + (1.0f - u1) * __expf(-2.0f * kappa)) / kappa, -1.0f), 1.0f);
    const float s = sqrtf(fmaxf(0.0f, 1.0f - c * c));
    const float phi = kTwoPi * u2;
    const Frame fr = make_frame(mu);
    return normalize(to_world(fr, mk(s * cosf(phi), s * sinf(phi), c)));
}

// ---------------------------------------------------------------------------
// Inference over a ray queue: position = hit point of queue entry i.
// ---------------------------------------------------------------------------
// 4 warps share one copy of the weights in shared memory; 4 blocks per SM
// (up to 128 registers a thread).  8-warp blocks at 4 per SM left too little
// of the SM's unified L1/shared storage for the L1 cache that serves the
// hash-grid gathers and ran 15 % slower; 5 blocks at 69 registers ran 10 %
// slower.
constexpr int kGInferWarps = 4;
constexpr int kGInferBlocksPerSm = 4;
__global__ void __launch_bounds__(32 * kGInferWarps, kGInferBlocksPerSm)
k_guide_infer(GuideNet net, const uint32_t* counts, int q, uint32_t cap,
                                                     const float4* ray_o, const float4* ray_d, const float4* hit,
                                                     float* mix_out) {
    extern __shared__ __align__(16) unsigned char g_smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(g_smem);
    float* srow = reinterpret_cast<float*>(g_smem + kGSmemW * sizeof(__nv_bfloat16));   // per warp 16 x 48
    load_weights_smem(net, sw);
    const uint32_t n = min(counts[q], cap);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    float* my = srow + warp * 16 * kGOutPad;
    const uint32_t tiles = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * (blockDim.x >> 5) + warp; tile < tiles; tile += gridDim.x * (blockDim.x >> 5)) {
        const uint32_t r0 = tile * 16 + g, r1 = r0 + 8;
        auto pos = [&](uint32_t r) {
            if (r >= n) return mk(0.5f);
            const float4 o = ray_o[r], d = ray_d[r], h = hit[r];
            const float t = __float_as_int(h.y) >= 0 ? h.x : 0.0f;
            return guide_normalise(net, mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z));
        };
        float out[6][4];
        warp_forward(net, sw, pos(r0), pos(r1), out);
#pragma unroll
        for (int nt = 0; nt < 6; ++nt) {
            my[g * kGOutPad + nt * 8 + 2 * c] = out[nt][0];
            my[g * kGOutPad + nt * 8 + 2 * c + 1] = out[nt][1];
            my[(g + 8) * kGOutPad + nt * 8 + 2 * c] = out[nt][2];
            my[(g + 8) * kGOutPad + nt * 8 + 2 * c + 1] = out[nt][3];
        }
        __syncwarp();
        if (lane < 16) {
            const uint32_t r = tile * 16 + lane;
            if (r < n) {
                float mix[kGMix];
                mixture_record(my + lane * kGOutPad, mix);
                float4* dst = reinterpret_cast<float4*>(mix_out + static_cast<size_t>(r) * kGMix);
#pragma unroll
                for (int k = 0; k < kGMix / 4; ++k) dst[k] = make_float4(mix[4 * k], mix[4 * k + 1], mix[4 * k + 2], mix[4 * k + 3]);
            }
        }
        __syncwarp();
    }
}

}  // namespace ptb

namespace ptb {

// ---------------------------------------------------------------------------
// Training
// ---------------------------------------------------------------------------
// One training sample: normalised position (w = weight L_in / p), direction.
struct GuideSample { float4 pos_w; float4 dir; };

// d(-w log q(dir)) / d(raw outputs) for one row (raw: 48 floats, out: 48 floats).
__device__ float mixture_grad(const float* raw, f3 dir, float w, float* d) {
    float mix[kGMix];
    raw_to_mixture(raw, mix);
    float v[kGLobes];
    float q = 0.0f;
    for (int k = 0; k < kGLobes; ++k) {
        const float c = mix[4 * k] * dir.x + mix[4 * k + 1] * dir.y + mix[4 * k + 2] * dir.z;
        v[k] = vmf_pdf(mix[4 * k + 3], c);
        q += mix[32 + k] * v[k];
    }
    q = fmaxf(q, 1e-12f);
    const float gq = -w / q;
    for (int k = 0; k < kGLobes; ++k) {
        const float pi = mix[32 + k], kap = mix[4 * k + 3];
        const f3 mu = mk(mix[4 * k], mix[4 * k + 1], mix[4 * k + 2]);
        const float c = dot(mu, dir);
        // mixture logit
        d[5 * k + 4] = -w * pi * (v[k] / q - 1.0f);
        // concentration: d log v / d kappa = 1/kappa - 2/(e^{2kappa} - 1) + c - 1
        const float dl = (kap > 1e-3f ? 1.0f / kap - 2.0f / expm1f(fminf(2.0f * kap, 80.0f)) : 1.0f) + c - 1.0f;
        const float r = raw[5 * k + 3];
        const float sig = 1.0f / (1.0f + expf(-r));
        d[5 * k + 3] = kap >= 5e3f ? 0.0f : gq * pi * v[k] * dl * sig;
        // mean direction through the normalisation
        const f3 m = mk(raw[5 * k], raw[5 * k + 1], raw[5 * k + 2]);
        const float ml = fmaxf(length(m), 1e-12f);
        const f3 dm = (dir - c * mu) * (gq * pi * kap * v[k] / ml);
        d[5 * k] = dm.x; d[5 * k + 1] = dm.y; d[5 * k + 2] = dm.z;
    }
    for (int j = kGOut; j < kGOutPad; ++j) d[j] = 0.0f;
    return q;
}

// Per-warp shared scratch for the backward pass (bf16):
//   XT0 [32][16], HT1..3 [64][16]      inputs of layers 0..3, transposed
//   DY  [16][64+8]                      row-major upstream gradient
//   DYT [64][16+8]                      transposed upstream gradient
// plus a float [16][48] tile for the outputs.
constexpr int kGWarpScratch = (kGIn * 16 + 3 * kGHid * 16) * 2 + 16 * (kGHid + 8) * 2 + kGHid * (16 + 8) * 2 +
                              16 * kGOutPad * 4;

// store 16 rows of A-fragment data (row-major 16 x K, bf16 pairs) transposed into T[K][16]
template <int K>
__device__ __forceinline__ void store_t(const uint32_t (&a)[K / 16][4], __nv_bfloat16* T) {
    const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
#pragma unroll
    for (int kt = 0; kt < K / 16; ++kt) {
        const __nv_bfloat162 v0 = *reinterpret_cast<const __nv_bfloat162*>(&a[kt][0]);
        const __nv_bfloat162 v1 = *reinterpret_cast<const __nv_bfloat162*>(&a[kt][1]);
        const __nv_bfloat162 v2 = *reinterpret_cast<const __nv_bfloat162*>(&a[kt][2]);
        const __nv_bfloat162 v3 = *reinterpret_cast<const __nv_bfloat162*>(&a[kt][3]);
        const int k0 = kt * 16 + 2 * c;
        T[(k0) * 16 + g] = v0.x;     T[(k0 + 1) * 16 + g] = v0.y;
        T[(k0) * 16 + g + 8] = v1.x; T[(k0 + 1) * 16 + g + 8] = v1.y;
        T[(k0 + 8) * 16 + g] = v2.x; T[(k0 + 9) * 16 + g] = v2.y;
        T[(k0 + 8) * 16 + g + 8] = v3.x; T[(k0 + 9) * 16 + g + 8] = v3.y;
    }
}

// The weight gradient dW_l = DY_l^T X_l is a GEMM over the minibatch's rows;
// the forward/backward kernel stores each layer's input X_l and upstream
// gradient DY_l transposed ([column][row], rows contiguous, bf16) in global
// memory, and k_guide_dw sums them in fixed row chunks (deterministic, no
// atomics).  Row block: kGTrainRows rows per matrix.
constexpr int kGTrainRows = 1 << 17;      // rows (training samples) of one optimiser step at most
constexpr int kGDwChunk = 512;            // rows per partial sum of k_guide_dw
constexpr int kGDwChunks = kGTrainRows / kGDwChunk;
// bf16 element offsets of X_l ([IN_l][R]) and DY_l ([OUT_l][R]) in the row store
__host__ __device__ constexpr size_t g_rx(int l) {
    return static_cast<size_t>(l == 0 ? 0 : kGIn + (l - 1) * kGHid) * kGTrainRows;
}
__host__ __device__ constexpr size_t g_rdy(int l) {
    return static_cast<size_t>(kGIn + 3 * kGHid + (l == 3 ? 0 : kGOutPad + (2 - l) * kGHid)) * kGTrainRows;
}
constexpr size_t kGRowStoreElems = static_cast<size_t>(kGIn + 3 * kGHid + kGOutPad + 3 * kGHid) * kGTrainRows;

// Copy a warp's transposed [N][16] tile (row stride `ld` bf16) to columns
// r0 .. r0 + 15 of a [N][kGTrainRows] matrix: two 16-byte stores per row.
template <int N>
__device__ __forceinline__ void store_rows(const __nv_bfloat16* T, int ld, __nv_bfloat16* dst, uint32_t r0) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = lane; k < 2 * N; k += 32) {
        const int row = k >> 1, half = k & 1;
        const uint4 v = *reinterpret_cast<const uint4*>(T + row * ld + 8 * half);
        *reinterpret_cast<uint4*>(dst + static_cast<size_t>(row) * kGTrainRows + r0 + 8 * half) = v;
    }
}

// dX(16 x IN) = DY(16 x OUT) . W(OUT x IN), with W^T in shared memory ([in][out], padded rows).
template <int OUT, int IN>
__device__ __forceinline__ void back_dx(const __nv_bfloat16* DY, const __nv_bfloat16* WT, float (&acc)[IN / 8][4]) {
    const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    uint32_t a[OUT / 16][4];
#pragma unroll
    for (int kt = 0; kt < OUT / 16; ++kt) {
        const __nv_bfloat16* r0 = DY + g * (kGHid + 8) + kt * 16 + 2 * c;
        const __nv_bfloat16* r1 = DY + (g + 8) * (kGHid + 8) + kt * 16 + 2 * c;
        a[kt][0] = *reinterpret_cast<const uint32_t*>(r0);
        a[kt][1] = *reinterpret_cast<const uint32_t*>(r1);
        a[kt][2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
        a[kt][3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
    }
#pragma unroll
    for (int nt = 0; nt < IN / 8; ++nt) {
        acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
        const __nv_bfloat16* row = WT + (nt * 8 + g) * (OUT + 8) + 2 * c;
#pragma unroll
        for (int kt = 0; kt < OUT / 16; ++kt) {
            const uint32_t b0 = *reinterpret_cast<const uint32_t*>(row + kt * 16);
            const uint32_t b1 = *reinterpret_cast<const uint32_t*>(row + kt * 16 + 8);
            mma_bf16(acc[nt], a[kt], b0, b1);
        }
    }
}

// write a C-fragment tile (16 x N, optionally masked by a ReLU input held as
// transposed bf16 HT[N][16]) as the next upstream gradient: DY row-major and DYT
template <int N>
__device__ __forceinline__ void store_dy(const float (&acc)[N / 8][4], const __nv_bfloat16* HT, __nv_bfloat16* DY,
                                         __nv_bfloat16* DYT) {
    const int lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
#pragma unroll
    for (int nt = 0; nt < N / 8; ++nt) {
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int row = g + (e >= 2 ? 8 : 0), col = nt * 8 + 2 * c + (e & 1);
            float v = acc[nt][e];
            if (HT && __bfloat162float(HT[col * 16 + row]) <= 0.0f) v = 0.0f;
            const __nv_bfloat16 b = __float2bfloat16_rn(v);
            DY[row * (kGHid + 8) + col] = b;
            DYT[col * 24 + row] = b;
        }
    }
}

// Minibatch mb of nmb over the first n samples takes samples mb, mb + S,
// mb + 2 S, ... with the stride S = nmb: the samples are collected in path
// (pixel) order, so interleaving gives every optimiser step samples from the
// whole image instead of one band of rows.  With a cap of `step_cap` samples
// per step (0 = none) the stride grows to nmb * ceil(n / (nmb * step_cap)),
// so a step takes an evenly spread subset and the samples between are skipped.
__host__ __device__ __forceinline__ uint32_t minibatch_stride(uint32_t n, int nmb, uint32_t step_cap) {
    if (step_cap == 0u) return static_cast<uint32_t>(nmb);
    const uint64_t per = static_cast<uint64_t>(nmb) * step_cap;
    const uint64_t k = (static_cast<uint64_t>(n) + per - 1u) / per;
    return static_cast<uint32_t>(nmb) * static_cast<uint32_t>(k > 1u ? k : 1u);
}
// The per-step sample cap the kernels use: the caller's, within the row store.
__host__ __device__ __forceinline__ uint32_t guide_step_cap(uint32_t samples_per_step) {
    return (samples_per_step == 0u || samples_per_step > static_cast<uint32_t>(kGTrainRows)) ? kGTrainRows
                                                                                           : samples_per_step;
}
__host__ __device__ __forceinline__ uint32_t minibatch_size(uint32_t n, int mb, int nmb, uint32_t step_cap) {
    const uint32_t s = minibatch_stride(n, nmb, step_cap);
    return n > static_cast<uint32_t>(mb) ? (n - static_cast<uint32_t>(mb) + s - 1u) / s : 0u;
}

// Optimiser steps taken for the first mb minibatches (the empty ones take none).
__host__ __device__ __forceinline__ uint32_t steps_before(uint32_t n, int mb, int nmb) {
    uint32_t k = 0;
    for (int i = 0; i < mb; ++i) k += n > static_cast<uint32_t>(i) ? 1u : 0u;
    return k;
}

// Forward and backward of minibatch mb (of nmb) of the collected samples:
// the loss gradient of every row, the hash-grid gradient (fixed-point
// atomics), and each layer's input and upstream gradient in the row store
// for k_guide_dw.  CTAs of kGTrainWarps warps share one copy of both weight
// layouts (one CTA per SM).
constexpr int kGTrainWarps = 8;
__global__ void __launch_bounds__(32 * kGTrainWarps) k_guide_train(GuideNet net, const GuideSample* __restrict__ samples_all,
                                                     const uint32_t* count, uint32_t cap, int mb, int nmb,
                                                     uint32_t step_cap, __nv_bfloat16* __restrict__ rows) {
    const uint32_t total = min(*count, cap);
    const uint32_t n = minibatch_size(total, mb, nmb, step_cap);
    if (n == 0u) return;
    // row r of this minibatch is sample mb + r * stride
    const GuideSample* __restrict__ samples = samples_all + mb;
    const uint32_t sstride = minibatch_stride(total, nmb, step_cap);
    const float inv_n = 1.0f / static_cast<float>(n);
    extern __shared__ __align__(16) unsigned char g_smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(g_smem);                       // W  [out][in+8]
    __nv_bfloat16* swt = sw + kGSmemW;                                                 // WT [in][out+8]
    unsigned char* scratch0 = reinterpret_cast<unsigned char*>(swt + kGSmemW + 64);
    load_weights_smem(net, sw);
    // transposed weights: layer l, WT[in][out] with row length out + 8
    for (int l = 0; l < 4; ++l) {
        const int in = g_in(l), out = g_out(l);
        const int woff = l == 0 ? 0 : (l == 1 ? kGIn * (kGHid + 8) : (l == 2 ? kGIn * (kGHid + 8) + kGHid * (kGHid + 8)
                                                                             : kGIn * (kGHid + 8) + 2 * kGHid * (kGHid + 8)));
        for (int i = threadIdx.x; i < out * in; i += blockDim.x) {
            const int o = i / in, k = i % in;
            swt[woff + k * (out + 8) + o] = net.w[g_woff(l) + i];
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    unsigned char* my = scratch0 + warp * kGWarpScratch;
    __nv_bfloat16* XT0 = reinterpret_cast<__nv_bfloat16*>(my);
    __nv_bfloat16* HT1 = XT0 + kGIn * 16;
    __nv_bfloat16* HT2 = HT1 + kGHid * 16;
    __nv_bfloat16* HT3 = HT2 + kGHid * 16;
    __nv_bfloat16* DY = HT3 + kGHid * 16;
    __nv_bfloat16* DYT = DY + 16 * (kGHid + 8);
    float* OUT = reinterpret_cast<float*>(DYT + kGHid * 24);
    const __nv_bfloat16* WT0 = swt;
    const __nv_bfloat16* WT1 = swt + kGIn * (kGHid + 8);
    const __nv_bfloat16* WT2 = WT1 + kGHid * (kGHid + 8);
    const __nv_bfloat16* WT3 = WT2 + kGHid * (kGHid + 8);
    const uint32_t tiles = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * kGTrainWarps + warp; tile < tiles; tile += gridDim.x * kGTrainWarps) {
        const uint32_t r0 = tile * 16 + g, r1 = r0 + 8;
        const GuideSample s0 = r0 < n ? samples[static_cast<size_t>(r0) * sstride]
                                      : GuideSample{make_float4(0.5f, 0.5f, 0.5f, 0.0f), make_float4(0, 0, 1, 0)};
        const GuideSample s1 = r1 < n ? samples[static_cast<size_t>(r1) * sstride]
                                      : GuideSample{make_float4(0.5f, 0.5f, 0.5f, 0.0f), make_float4(0, 0, 1, 0)};
        const f3 p0 = mk(s0.pos_w.x, s0.pos_w.y, s0.pos_w.z), p1 = mk(s1.pos_w.x, s1.pos_w.y, s1.pos_w.z);
        // forward, keeping every layer's input
        uint32_t a0[2][4];
        encode_a(net, p0, p1, a0);
        store_t<kGIn>(a0, XT0);
        float h[8][4];
        uint32_t a[4][4];
        warp_layer<kGIn, kGHid>(a0, sw + g_soff(0), h);
        relu_to_a<kGHid>(h, a);
        store_t<kGHid>(a, HT1);
        warp_layer<kGHid, kGHid>(a, sw + g_soff(1), h);
        relu_to_a<kGHid>(h, a);
        store_t<kGHid>(a, HT2);
        warp_layer<kGHid, kGHid>(a, sw + g_soff(2), h);
        relu_to_a<kGHid>(h, a);
        store_t<kGHid>(a, HT3);
        float out[6][4];
        warp_layer<kGHid, kGOutPad>(a, sw + g_soff(3), out);
#pragma unroll
        for (int nt = 0; nt < 6; ++nt) {
            OUT[g * kGOutPad + nt * 8 + 2 * c] = out[nt][0];
            OUT[g * kGOutPad + nt * 8 + 2 * c + 1] = out[nt][1];
            OUT[(g + 8) * kGOutPad + nt * 8 + 2 * c] = out[nt][2];
            OUT[(g + 8) * kGOutPad + nt * 8 + 2 * c + 1] = out[nt][3];
        }
        __syncwarp();
        // loss gradient per row (lanes 0..15), scaled by 1/n
        float row_loss = 0.0f;
        if (lane < 16) {
            const uint32_t r = tile * 16 + lane;
            float d[kGOutPad];
            if (r < n) {
                const GuideSample s = samples[static_cast<size_t>(r) * sstride];
                const float q = mixture_grad(OUT + lane * kGOutPad, mk(s.dir.x, s.dir.y, s.dir.z), s.pos_w.w * inv_n, d);
                row_loss = -s.pos_w.w * logf(q);
            } else {
                for (int j = 0; j < kGOutPad; ++j) d[j] = 0.0f;
            }
            for (int j = 0; j < kGOutPad; ++j) {
                const __nv_bfloat16 b = __float2bfloat16_rn(d[j]);
                DY[lane * (kGHid + 8) + j] = b;
                DYT[j * 24 + lane] = b;
            }
        }
        if (net.loss_fix) {
            unsigned long long lf = lane < 16 ? static_cast<unsigned long long>(
                                                    __float2ll_rn(fminf(fmaxf(row_loss, -1e12f), 1e12f) * kGLossFix))
                                              : 0ull;
            for (int o = 16; o > 0; o >>= 1) lf += __shfl_xor_sync(0xffffffffu, lf, o);
            if (lane == 0) {
                atomicAdd(net.loss_fix, lf);
                atomicAdd(net.loss_fix + 1, static_cast<unsigned long long>(min(16u, n - tile * 16)));
            }
        }
        __syncwarp();
        // layer 3 (48 x 64)
        store_rows<kGOutPad>(DYT, 24, rows + g_rdy(3), tile * 16);
        store_rows<kGHid>(HT3, 16, rows + g_rx(3), tile * 16);
        float dh[8][4];
        back_dx<kGOutPad, kGHid>(DY, WT3, dh);
        __syncwarp();
        store_dy<kGHid>(dh, HT3, DY, DYT);
        __syncwarp();
        // layer 2
        store_rows<kGHid>(DYT, 24, rows + g_rdy(2), tile * 16);
        store_rows<kGHid>(HT2, 16, rows + g_rx(2), tile * 16);
        back_dx<kGHid, kGHid>(DY, WT2, dh);
        __syncwarp();
        store_dy<kGHid>(dh, HT2, DY, DYT);
        __syncwarp();
        // layer 1
        store_rows<kGHid>(DYT, 24, rows + g_rdy(1), tile * 16);
        store_rows<kGHid>(HT1, 16, rows + g_rx(1), tile * 16);
        back_dx<kGHid, kGHid>(DY, WT1, dh);
        __syncwarp();
        store_dy<kGHid>(dh, HT1, DY, DYT);
        __syncwarp();
        // layer 0: dW0 and the gradient of the encoding
        store_rows<kGHid>(DYT, 24, rows + g_rdy(0), tile * 16);
        store_rows<kGIn>(XT0, 16, rows + g_rx(0), tile * 16);
        float dx[4][4];
        back_dx<kGHid, kGIn>(DY, WT0, dx);
        __syncwarp();
        // scatter the input gradient to the hash grid (levels c, 4+c, 8+c, 12+c)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
            const int level = nt * 4 + c;
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                const uint32_t r = half ? r1 : r0;
                if (r >= n) continue;
                const f3 p = half ? p1 : p0;
                const float gx = dx[nt][2 * half], gy = dx[nt][2 * half + 1];
                const float sc = net.scale[level];
                const float fx = p.x * sc + 0.5f, fy = p.y * sc + 0.5f, fz = p.z * sc + 0.5f;
                const float bx = floorf(fx), by = floorf(fy), bz = floorf(fz);
                const float tx = fx - bx, ty = fy - by, tz = fz - bz;
                const uint32_t ix = static_cast<uint32_t>(bx), iy = static_cast<uint32_t>(by), iz = static_cast<uint32_t>(bz);
                unsigned long long* gg = net.grid_grad + static_cast<size_t>(level) * kGTable * 2;
                for (int cidx = 0; cidx < 8; ++cidx) {
                    const uint32_t cx = cidx & 1, cy = (cidx >> 1) & 1, cz = (cidx >> 2) & 1;
                    const float w = (cx ? tx : 1.0f - tx) * (cy ? ty : 1.0f - ty) * (cz ? tz : 1.0f - tz);
                    const uint32_t e = grid_index(net, level, ix + cx, iy + cy, iz + cz);
                    atomicAdd(&gg[2 * e], g_fix(w * gx));
                    atomicAdd(&gg[2 * e + 1], g_fix(w * gy));
                }
            }
        }
        __syncwarp();
    }
}

// dW_l = DY_l^T X_l over the minibatch's rows: block (chunk, l) sums rows
// chunk * kGDwChunk .. + kGDwChunk (up to the tile-padded row count) of layer
// l into partial[chunk][l's weights]; warp w takes output rows 16 w .. 16 w
// + 15 (every column) on mma.sync m16n8k16, rows as the reduction dimension.
__global__ void __launch_bounds__(128) k_guide_dw(const uint32_t* count, uint32_t cap, int mb, int nmb,
                                                  uint32_t step_cap, const __nv_bfloat16* __restrict__ rows,
                                                  float* __restrict__ partial) {
    const uint32_t n = minibatch_size(min(*count, cap), mb, nmb, step_cap);
    const uint32_t rpad = (n + 15u) & ~15u;
    const uint32_t k0 = blockIdx.x * kGDwChunk;
    if (k0 >= rpad) return;
    const uint32_t k1 = min(rpad, k0 + kGDwChunk);
    const int l = blockIdx.y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    const int out = g_out(l), in = g_in(l);
    if (warp * 16 >= out) return;
    const __nv_bfloat16* dy = rows + g_rdy(l) + static_cast<size_t>(warp * 16) * kGTrainRows;
    const __nv_bfloat16* x = rows + g_rx(l);
    float acc[8][4];
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.0f;
    for (uint32_t k = k0; k < k1; k += 16) {
        uint32_t a[4];
        const __nv_bfloat16* r0 = dy + static_cast<size_t>(g) * kGTrainRows + k + 2 * c;
        const __nv_bfloat16* r1 = r0 + static_cast<size_t>(8) * kGTrainRows;
        a[0] = *reinterpret_cast<const uint32_t*>(r0);
        a[1] = *reinterpret_cast<const uint32_t*>(r1);
        a[2] = *reinterpret_cast<const uint32_t*>(r0 + 8);
        a[3] = *reinterpret_cast<const uint32_t*>(r1 + 8);
#pragma unroll
        for (int nt = 0; nt < 8; ++nt) {
            if (nt * 8 >= in) break;
            const __nv_bfloat16* xb = x + static_cast<size_t>(nt * 8 + g) * kGTrainRows + k + 2 * c;
            mma_bf16(acc[nt], a, *reinterpret_cast<const uint32_t*>(xb), *reinterpret_cast<const uint32_t*>(xb + 8));
        }
    }
    float* dst = partial + static_cast<size_t>(blockIdx.x) * kGWeights + g_woff(l);
    const int m0 = warp * 16 + g;
#pragma unroll
    for (int nt = 0; nt < 8; ++nt) {
        if (nt * 8 >= in) break;
        const int n0 = nt * 8 + 2 * c;
        dst[m0 * in + n0] = acc[nt][0];
        dst[m0 * in + n0 + 1] = acc[nt][1];
        dst[(m0 + 8) * in + n0] = acc[nt][2];
        dst[(m0 + 8) * in + n0 + 1] = acc[nt][3];
    }
}

// Sums the partials of k_guide_dw in chunk order into the weight gradient
// (fixed point, as the optimiser reads it).
__global__ void k_guide_dw_reduce(const uint32_t* count, uint32_t cap, int mb, int nmb, uint32_t step_cap,
                                  const float* __restrict__ partial, unsigned long long* w_grad) {
    const uint32_t n = minibatch_size(min(*count, cap), mb, nmb, step_cap);
    const uint32_t chunks = (((n + 15u) & ~15u) + kGDwChunk - 1u) / kGDwChunk;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kGWeights; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (uint32_t ch = 0; ch < chunks; ++ch) s += partial[static_cast<size_t>(ch) * kGWeights + i];
        if (chunks) w_grad[i] += g_fix(s);
    }
}

// Adam on the MLP weights (FP32 master -> BF16 copy) and the hash grid
// (FP32 master -> FP16 copy); gradients are cleared.
// dynamic shared memory of the two network kernels (4 warps per CTA)
constexpr int kGInferSmem = kGSmemW * 2 + kGInferWarps * 16 * kGOutPad * 4;
constexpr int kGTrainSmem = (2 * kGSmemW + 64) * 2 + kGTrainWarps * kGWarpScratch;
static_assert(kGTrainSmem <= 227 * 1024, "training kernel shared memory");
static_assert(((2 * kGSmemW + 64) * 2) % 16 == 0 && kGWarpScratch % 16 == 0, "shared memory carve alignment");

// Host-side state of one guide: the network, its optimiser state and the
// buffers the wavefront fills (mixtures per queue entry, training records and
// samples).  Owned by pt_guide.
struct GuideState {
    int          device = -1;
    GuideNet     net{};
    void*        params = nullptr;    // grid + weights + Adam state (one allocation)
    size_t       param_bytes = 0;
    void*        work = nullptr;      // mixtures, records, samples, counters
    size_t       work_bytes = 0;
    int          npix = 0, depth = 0;
    float*       mix = nullptr;
    float4*      rec = nullptr;
    GuideSample* samples = nullptr;
    uint32_t     sample_cap = 0;
    uint32_t*    counters = nullptr;  // [0] samples collected in the current pass (work buffer)
    uint32_t*    scan_counts = nullptr;   // training samples per path (npix + 1)
    uint32_t*    scan_offsets = nullptr;  // their exclusive prefix sums
    void*        scan_tmp = nullptr;      // the scan's temporary storage
    size_t       scan_tmp_bytes = 0;
    __nv_bfloat16* rows = nullptr;    // training row store (kGRowStoreElems) for the weight gradient
    float*       partial = nullptr;   // k_guide_dw's partial sums (kGDwChunks x kGWeights)
    uint32_t*    step = nullptr;      // optimiser steps taken (with the parameters: survives work resizes)
    unsigned char* feat = nullptr;    // encoded features of one queue (split inference kinds), 8 KB per 128 entries
    int          infer = kGuideInferDefault;   // PT_GUIDE_INFER_*
    int          mode = 0;            // 0 off, PT_GUIDE_USE, PT_GUIDE_TRAIN
    float        lr = 1e-2f;
    float        lr_half_life = 0.0f;  // optimiser steps per halving of the learning rate (0: constant)
    float        lr_floor = 0.1f;      // the learning rate stays above this fraction of lr
    float        alpha = kGuideAlpha;
    int          paths_per_step = kGuideMinibatchPaths;   // optimiser steps: one per this many paths of a pass
    uint32_t     samples_per_step = kGuideStepSamples;    // cap of training samples per step (0 = all)
};

// After a pass's minibatches: advance the step counter by the steps taken
// and empty the sample buffer.
__global__ void k_guide_step(uint32_t* sample_count, uint32_t* step, float* loss, unsigned long long* loss_fix,
                             uint32_t cap, int nmb) {
    *step += steps_before(min(*sample_count, cap), nmb, nmb);
    *sample_count = 0u;
    if (loss_fix[1] > 0ull)
        loss[2] = static_cast<float>(static_cast<double>(static_cast<long long>(loss_fix[0])) / kGLossFix /
                                     static_cast<double>(loss_fix[1]));
    loss_fix[0] = 0ull;
    loss_fix[1] = 0ull;
}

// Adam step for minibatch mb (skipped when it is empty); the step number is
// the counter plus the non-empty minibatches before it, plus one.
__global__ void k_guide_adam(GuideNet net, const uint32_t* count, uint32_t cap, int mb, int nmb, const uint32_t* step,
                             float lr_w, float lr_g, float b1, float b2, float eps, float lr_half_life, float lr_floor) {
    const uint32_t n = min(*count, cap);
    if (n <= static_cast<uint32_t>(mb)) return;
    const float t = static_cast<float>(*step + steps_before(n, mb, nmb) + 1u);
    const float bc1 = 1.0f - powf(b1, t), bc2 = 1.0f - powf(b2, t);
    if (lr_half_life > 0.0f) {   // learning rate halving every lr_half_life steps, down to lr_floor of it
        const float f = fmaxf(lr_floor, exp2f(-t / lr_half_life));
        lr_w *= f;
        lr_g *= f;
    }
    const float ea = net.ema, eb = 1.0f - net.ema;
    const size_t nw = kGWeights;
    const size_t ng = static_cast<size_t>(kGLevels) * kGTable;
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < nw + ng;
         i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        if (i < nw) {
            const float gr = g_unfix(net.w_grad[i]);
            const float m = b1 * net.w_m[i] + (1.0f - b1) * gr;
            const float v = b2 * net.w_v[i] + (1.0f - b2) * gr * gr;
            net.w_m[i] = m; net.w_v[i] = v; net.w_grad[i] = 0ull;
            const float p = net.w_master[i] - lr_w * (m / bc1) / (sqrtf(v / bc2) + eps);
            net.w_master[i] = p;
            net.w[i] = __float2bfloat16_rn(p);
            if (ea > 0.0f) {
                const float e = ea * net.w_ema[i] + eb * p;
                net.w_ema[i] = e;
                net.w_inf[i] = __float2bfloat16_rn(e);
            }
        } else {
            const size_t j = i - nw;
            const ulonglong2 gi = reinterpret_cast<const ulonglong2*>(net.grid_grad)[j];
            if (gi.x == 0ull && gi.y == 0ull && net.grid_m[j].x == 0.0f && net.grid_m[j].y == 0.0f) continue;
            const float2 gr = make_float2(g_unfix(gi.x), g_unfix(gi.y));
            float2 m = net.grid_m[j], v = net.grid_v[j], p = net.grid_master[j];
            m.x = b1 * m.x + (1.0f - b1) * gr.x; m.y = b1 * m.y + (1.0f - b1) * gr.y;
            v.x = b2 * v.x + (1.0f - b2) * gr.x * gr.x; v.y = b2 * v.y + (1.0f - b2) * gr.y * gr.y;
            p.x -= lr_g * (m.x / bc1) / (sqrtf(v.x / bc2) + eps);
            p.y -= lr_g * (m.y / bc1) / (sqrtf(v.y / bc2) + eps);
            net.grid_m[j] = m; net.grid_v[j] = v; net.grid_master[j] = p;
            reinterpret_cast<ulonglong2*>(net.grid_grad)[j] = make_ulonglong2(0ull, 0ull);
            // the FP16 pair table: this entry's own slot and the neighbour slot of the entry before it
            const __half2 hp = __floats2half2_rn(p.x, p.y);
            const size_t prev = (j & ~static_cast<size_t>(kGTable - 1)) | ((j + kGTable - 1) & (kGTable - 1));
            reinterpret_cast<__half2*>(net.grid + j)[0] = hp;
            reinterpret_cast<__half2*>(net.grid + prev)[1] = hp;
            if (ea > 0.0f) {
                float2 e = net.grid_ema[j];
                e.x = ea * e.x + eb * p.x;
                e.y = ea * e.y + eb * p.y;
                net.grid_ema[j] = e;
                const __half2 he = __floats2half2_rn(e.x, e.y);
                reinterpret_cast<__half2*>(net.grid_inf + j)[0] = he;
                reinterpret_cast<__half2*>(net.grid_inf + prev)[1] = he;
            }
        }
    }
}

}  // namespace ptb
