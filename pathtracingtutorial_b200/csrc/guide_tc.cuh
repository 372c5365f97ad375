// guide_tc.cuh -- guide inference split in two kernels (included by
// integrator.cu after guide.cuh; no reference counterpart).
//
// k_guide_infer (guide.cuh) encodes and evaluates 16 queries
// per warp: at 16 warps per SM (register-limited by the MLP fragments) the
// 64 dependent hash-grid gathers of a query are latency-bound.  Here the
// encoding runs on its own at full occupancy (one thread per query and
// level, four independent 8-byte gathers each) and writes the features in
// the tensor core's operand layout, 128-query tiles of 8 KB; the network then
// runs per 128-query tile on tcgen05 (k_guide_mlp_tc: features moved by the
// bulk-copy engine, weights resident in shared memory, accumulators in
// tensor memory, one row per thread for the ReLU and mixture epilogues) or,
// for comparison, on mma.sync (k_guide_mlp_mma).  All three give the same
// mixture records up to FP32 accumulation order.

namespace ptb {

constexpr int kGTcRows = 128;                              // queries per tile (the MMA's M)
constexpr int kGFeatTileBytes = kGTcRows * kGIn * 2;       // 8 KB of BF16 features per tile

// Byte offset of element (r, k) of a K-major BF16 operand with K columns in
// the tensor core's canonical layout without swizzling: 8 x 8 core matrices
// (8 rows of 16 bytes, 128 contiguous bytes); core matrices adjacent along K
// are 128 bytes apart (the descriptor's leading-dimension offset), 8-row
// groups K * 16 bytes apart (its stride offset).
__host__ __device__ constexpr uint32_t umma_off(uint32_t r, uint32_t k, uint32_t K) {
    return (r >> 3) * (K * 16u) + (k >> 3) * 128u + (r & 7u) * 16u + (k & 7u) * 2u;
}

// Feature rows of a queue of n entries: whole tiles.
__host__ __device__ __forceinline__ uint32_t guide_feat_rows(uint32_t n) {
    return (n + kGTcRows - 1u) / kGTcRows * kGTcRows;
}

// Entries of a dense level's four-corner table: res^3 plus one layer (res^2),
// so that a cell in the last layer (a position at the top of the unit cube,
// where floor(scale * p + 0.5) can reach res - 1) reads the same pair-table
// entries as encode_level does (the index wraps on into the next layers
// there, as the dense index arithmetic does).
__host__ __device__ inline uint32_t guide_quad_level_entries(uint32_t res) { return res * res * res + res * res; }

// The four-corner table of the dense levels from the pair table `net.grid`.
__global__ void __launch_bounds__(256) k_guide_quad(GuideNet net) {
    for (uint32_t l = 0; l < net.dense_limit; ++l) {
        const uint32_t res = static_cast<uint32_t>(net.scale[l]) + 2u;
        const uint32_t n = guide_quad_level_entries(res);
        const uint2* tab = net.grid + static_cast<size_t>(l) * kGTable;
        uint4* dst = net.quad + net.quad_off[l];
        for (uint32_t e = blockIdx.x * blockDim.x + threadIdx.x; e < n; e += gridDim.x * blockDim.x) {
            const uint2 a = tab[e & (kGTable - 1)], b = tab[(e + res) & (kGTable - 1)];
            dst[e] = make_uint4(a.x, a.y, b.x, b.y);
        }
    }
}

// encode_level for a dense level from the four-corner table: two 16-byte
// gathers (layers z and z + 1) instead of four 8-byte ones, the same
// products summed in the same order.
__device__ __forceinline__ float2 encode_level_quad(const GuideNet& net, int level, f3 p) {
    const float s = net.scale[level];
    const float fx = p.x * s + 0.5f, fy = p.y * s + 0.5f, fz = p.z * s + 0.5f;
    const float bx = floorf(fx), by = floorf(fy), bz = floorf(fz);
    const float tx = fx - bx, ty = fy - by, tz = fz - bz;
    const uint32_t ix = static_cast<uint32_t>(bx), iy = static_cast<uint32_t>(by), iz = static_cast<uint32_t>(bz);
    const uint32_t res = static_cast<uint32_t>(s) + 2u;
    const uint4* tab = net.quad + net.quad_off[level];
    const uint32_t e0 = ix + iy * res + iz * res * res;
    float2 r = make_float2(0.0f, 0.0f);
#pragma unroll
    for (int cz = 0; cz < 2; ++cz) {
        const uint4 qd = __ldg(tab + e0 + static_cast<uint32_t>(cz) * res * res);
#pragma unroll
        for (int cy = 0; cy < 2; ++cy) {
            const uint32_t u0 = cy ? qd.z : qd.x, u1 = cy ? qd.w : qd.y;
            const float2 f0 = __half22float2(*reinterpret_cast<const __half2*>(&u0));
            const float2 f1 = __half22float2(*reinterpret_cast<const __half2*>(&u1));
            const float w0 = (1.0f - tx) * (cy ? ty : 1.0f - ty) * (cz ? tz : 1.0f - tz);
            const float w1 = tx * (cy ? ty : 1.0f - ty) * (cz ? tz : 1.0f - tz);
            r.x += w0 * f0.x;
            r.y += w0 * f0.y;
            r.x += w1 * f1.x;
            r.y += w1 * f1.y;
        }
    }
    return r;
}

// ---------------------------------------------------------------------------
// Encoding: thread (row r, level l); 16 lanes per query, 2 queries per warp.
// Rows between n and the end of the last tile get zero features.  Positions
// come from the queue (hit point of ray r) or, when qd is given, from qd[6 r].
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256) k_guide_encode(GuideNet net, const uint32_t* counts, int q, uint32_t cap,
                                                      const float4* __restrict__ ray_o,
                                                      const float4* __restrict__ ray_d,
                                                      const float4* __restrict__ hit, const float* __restrict__ qd,
                                                      uint32_t qn, unsigned char* __restrict__ feat) {
    const uint32_t n = qd ? qn : min(counts[q], cap);
    const uint32_t items = guide_feat_rows(n) * static_cast<uint32_t>(kGLevels);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < items; i += gridDim.x * blockDim.x) {
        const uint32_t r = i / kGLevels;
        const int level = static_cast<int>(i % kGLevels);
        float2 e = make_float2(0.0f, 0.0f);
        if (r < n) {
            f3 x;
            if (qd) {
                x = mk(qd[6 * static_cast<size_t>(r)], qd[6 * static_cast<size_t>(r) + 1], qd[6 * static_cast<size_t>(r) + 2]);
            } else {
                const float4 o = ray_o[r], d = ray_d[r], h = hit[r];
                const float t = __float_as_int(h.y) >= 0 ? h.x : 0.0f;
                x = mk(o.x + t * d.x, o.y + t * d.y, o.z + t * d.z);
            }
            const f3 pn = guide_normalise(net, x);
            e = (net.quad && static_cast<uint32_t>(level) < net.dense_limit) ? encode_level_quad(net, level, pn)
                                                                             : encode_level(net, level, pn);
        }
        unsigned char* tile = feat + static_cast<size_t>(r / kGTcRows) * kGFeatTileBytes;
        *reinterpret_cast<uint32_t*>(tile + umma_off(r % kGTcRows, 2u * level, kGIn)) = pack_bf16(e.x, e.y);
    }
}

// Mixture record of row r (raw: 48 network outputs) into out (kGMix floats).
__device__ __forceinline__ void store_mixture(const float* raw, float* out) {
    alignas(16) float rec[kGMix];
    mixture_record(raw, rec);
    float4* dst = reinterpret_cast<float4*>(out);
#pragma unroll
    for (int k = 0; k < kGMix / 4; ++k) dst[k] = make_float4(rec[4 * k], rec[4 * k + 1], rec[4 * k + 2], rec[4 * k + 3]);
}

// ---------------------------------------------------------------------------
// The network on mma.sync m16n8k16 over encoded features (comparison path):
// the same warp tiles as the fused kernel, A fragments read from the tiles.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * kGInferWarps, kGInferBlocksPerSm)
k_guide_mlp_mma(GuideNet net, const uint32_t* counts, int q, uint32_t cap, uint32_t qn,
                const unsigned char* __restrict__ feat, float* __restrict__ mix_out) {
    extern __shared__ __align__(16) unsigned char g_smem[];
    __nv_bfloat16* sw = reinterpret_cast<__nv_bfloat16*>(g_smem);
    float* srow = reinterpret_cast<float*>(g_smem + kGSmemW * sizeof(__nv_bfloat16));
    load_weights_smem(net, sw);
    const uint32_t n = counts ? min(counts[q], cap) : qn;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, c = lane & 3;
    float* my = srow + warp * 16 * kGOutPad;
    const uint32_t tiles = (n + 15) / 16;
    for (uint32_t tile = blockIdx.x * (blockDim.x >> 5) + warp; tile < tiles; tile += gridDim.x * (blockDim.x >> 5)) {
        const uint32_t r0 = tile * 16 + g;
        const unsigned char* ft = feat + static_cast<size_t>(r0 / kGTcRows) * kGFeatTileBytes;
        const uint32_t rr = r0 % kGTcRows;   // rows rr and rr + 8 lie in the same 128-row tile
        uint32_t a0[2][4];
#pragma unroll
        for (int kt = 0; kt < 2; ++kt) {
            a0[kt][0] = *reinterpret_cast<const uint32_t*>(ft + umma_off(rr, kt * 16 + 2 * c, kGIn));
            a0[kt][1] = *reinterpret_cast<const uint32_t*>(ft + umma_off(rr + 8, kt * 16 + 2 * c, kGIn));
            a0[kt][2] = *reinterpret_cast<const uint32_t*>(ft + umma_off(rr, kt * 16 + 8 + 2 * c, kGIn));
            a0[kt][3] = *reinterpret_cast<const uint32_t*>(ft + umma_off(rr + 8, kt * 16 + 8 + 2 * c, kGIn));
        }
        float h[8][4];
        uint32_t a[4][4];
        warp_layer<kGIn, kGHid>(a0, sw + g_soff(0), h);
        relu_to_a<kGHid>(h, a);
        warp_layer<kGHid, kGHid>(a, sw + g_soff(1), h);
        relu_to_a<kGHid>(h, a);
        warp_layer<kGHid, kGHid>(a, sw + g_soff(2), h);
        relu_to_a<kGHid>(h, a);
        float out[6][4];
        warp_layer<kGHid, kGOutPad>(a, sw + g_soff(3), out);
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
            if (r < n) store_mixture(my + lane * kGOutPad, mix_out + static_cast<size_t>(r) * kGMix);
        }
        __syncwarp();
    }
}

// ---------------------------------------------------------------------------
// tcgen05 building blocks (inline PTX, sm_100a)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy writes to shared memory -> visible to the tensor core / bulk copies
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n.reg .pred p;\n"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        "selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0u;
}
// Bounded wait for the phase with the given parity: false after about a
// second (2^31 SM clocks) without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
    const long long t0 = clock64();
    while (!mbar_try_wait(bar, parity)) {
        if (clock64() - t0 > (1ll << 31)) return false;
    }
    return true;
}
// Bulk copy (no tensor map) global -> shared, completion counted in bytes on bar.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_addr(dst)),
                 "l"(src), "r"(bytes), "r"(smem_addr(bar))
                 : "memory");
}

// Shared-memory operand descriptor, canonical K-major layout without
// swizzling: start address, leading-dimension offset (between core matrices
// along K), stride offset (between 8-row groups), all in 16-byte units; the
// fixed version field (bits 46-48 = 1); swizzle mode 0.
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return static_cast<uint64_t>((saddr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
           (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\n"
        "setp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}
// Arrives once on bar when every tcgen05.mma issued so far by this thread has completed.
__device__ __forceinline__ void umma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}
// 32 lanes x 32 columns (32-bit): this thread's lane, columns col .. col + 31.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]),
          "=r"(v[16]), "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
          "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&v)[16]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
          "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// ---------------------------------------------------------------------------
// The network on tcgen05.  A CTA holds one copy of the four weight matrices
// (B operands, 26 KB of shared memory) and runs kGTcGroups independent tile
// groups of 4 warps; a group takes one 128-query tile at a time through the
// four layers.  Per group: the feature tile (A of layer 0, 8 KB, refilled by
// the bulk-copy engine while layers 1-3 run), the hidden tile (A of layers
// 1-3, 16 KB), two mbarriers and 64 tensor-memory columns of FP32
// accumulators with row i in lane i, so thread i of the group (its warp i / 32
// reads lanes 32 (i / 32) ..) owns query row i through the ReLU epilogues and
// the mixture record.  While one group's warps run an epilogue, the tensor
// core serves the others.  The output layer's rows are reordered (the eight
// logits first, then each lobe's mean and concentration) so that the mixture
// epilogue streams its row out of tensor memory in 8-column pieces.
// 2 CTAs of 3 groups per SM: 24 warps, 2 x 100 KB of shared memory, 2 x 256
// tensor-memory columns, at most 85 registers a thread.
// ---------------------------------------------------------------------------
constexpr int kGTcGroups = 3;
constexpr int kGTcThreads = 128 * kGTcGroups;
constexpr int kGTcBlocksPerSm = 2;
constexpr uint32_t kGTcCols = 256;                                 // tensor-memory columns allocated (power of 2)
static_assert(64 * kGTcGroups <= static_cast<int>(kGTcCols), "accumulator columns");
__host__ __device__ constexpr int g_tc_woff(int l) {              // byte offset of layer l's B operand
    return l == 0 ? 0 : (l == 1 ? kGHid * kGIn * 2 : (l == 2 ? kGHid * kGIn * 2 + kGHid * kGHid * 2
                                                              : kGHid * kGIn * 2 + 2 * kGHid * kGHid * 2));
}
constexpr int kGTcW = g_tc_woff(3) + kGOutPad * kGHid * 2;        // 26,624 bytes of weights
constexpr int kGTcGroupBytes = kGFeatTileBytes + kGTcRows * kGHid * 2;   // feature + hidden tile: 24 KB
constexpr int kGTcBar = kGTcW + kGTcGroups * kGTcGroupBytes;      // barriers, TMEM address
constexpr int kGTcSmem = kGTcBar + 16 * kGTcGroups + 16;
static_assert((kGTcSmem + 1024) * kGTcBlocksPerSm <= 228 * 1024, "tcgen05 MLP occupancy");
static_assert(kGTcCols * kGTcBlocksPerSm <= 512, "tensor memory of the resident CTAs");
static_assert(kGTcW % 16 == 0 && kGTcGroupBytes % 16 == 0 && kGTcBar % 8 == 0, "operand alignment");

// Output row of the network that feeds accumulator column o: logits first
// (column k = logit of lobe k), then lobe k's mean xyz and concentration in
// columns 8 + 4 k .. 8 + 4 k + 3, then the padding rows.
__host__ __device__ constexpr int g_tc_out_row(int o) {
    return o < kGLobes ? 5 * o + 4 : (o < kGLobes + 4 * kGLobes ? 5 * ((o - kGLobes) / 4) + (o - kGLobes) % 4 : o);
}

// Issue the K / 16 MMAs of one layer: D[128 x N] = A[128 x K] B[N x K]^T.
template <int K, int N>
__device__ __forceinline__ void tc_layer(uint32_t tmem, uint32_t a_saddr, uint32_t b_saddr) {
    constexpr uint32_t idesc = umma_idesc_bf16(kGTcRows, N);
#pragma unroll
    for (int s = 0; s < K / 16; ++s) {
        const uint64_t ad = umma_desc(a_saddr + s * 256u, 128u, K * 16u);
        const uint64_t bd = umma_desc(b_saddr + s * 256u, 128u, K * 16u);
        umma_bf16(tmem, ad, bd, idesc, s > 0 ? 1u : 0u);
    }
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
                 : "r"(taddr));
}

// Accumulator row (64 columns) of this thread -> ReLU -> BF16 row of the hidden tile.
__device__ __forceinline__ void tc_relu_to_hidden(uint32_t tmem_row, unsigned char* H, uint32_t row) {
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        uint32_t v[32];
        tmem_ld32(tmem_row + 32u * half, v);
        tmem_wait_ld();
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            uint4 w;
            w.x = pack_bf16(fmaxf(__uint_as_float(v[8 * j]), 0.0f), fmaxf(__uint_as_float(v[8 * j + 1]), 0.0f));
            w.y = pack_bf16(fmaxf(__uint_as_float(v[8 * j + 2]), 0.0f), fmaxf(__uint_as_float(v[8 * j + 3]), 0.0f));
            w.z = pack_bf16(fmaxf(__uint_as_float(v[8 * j + 4]), 0.0f), fmaxf(__uint_as_float(v[8 * j + 5]), 0.0f));
            w.w = pack_bf16(fmaxf(__uint_as_float(v[8 * j + 6]), 0.0f), fmaxf(__uint_as_float(v[8 * j + 7]), 0.0f));
            *reinterpret_cast<uint4*>(H + umma_off(row, 32u * half + 8u * j, kGHid)) = w;
        }
    }
}

// One lobe's record (mixture_record's algebra) from its four accumulator
// columns: float4(kappa mu, b) with b = log pi - kappa + log(kappa / (2 pi (1 - e^{-2 kappa}))).
__device__ __forceinline__ float4 tc_lobe_record(const uint32_t* v, float log_pi) {
    const float mxx = __uint_as_float(v[0]), myy = __uint_as_float(v[1]), mzz = __uint_as_float(v[2]);
    const float r = __uint_as_float(v[3]);
    const float l2 = mxx * mxx + myy * myy + mzz * mzz;
    const float sp = r > 15.0f ? r : __logf(1.0f + __expf(r));
    const float kap = fminf(sp + 1e-3f, 5e3f);
    constexpr float kLog2Pi = 1.83787706640934548356f;
    const float b = log_pi + __logf(__fdividef(kap, 1.0f - __expf(-2.0f * kap))) - kLog2Pi - kap;
    if (l2 > 1e-24f) {
        const float sc = kap * rsqrtf(l2);
        return make_float4(sc * mxx, sc * myy, sc * mzz, b);
    }
    return make_float4(0.0f, 0.0f, kap, b);
}

// Group-wide barrier over the group's 128 threads (named barrier 1 + g, an
// immediate, so that the kernel reserves barriers 0-3 only) with an AND vote.
template <int Id>
__device__ __forceinline__ bool bar_red_and(bool v) {
    uint32_t out;
    asm volatile(
        "{\n.reg .pred p, q;\n"
        "setp.ne.u32 p, %1, 0;\n"
        "bar.red.and.pred q, %2, 128, p;\n"
        "selp.u32 %0, 1, 0, q;\n}"
        : "=r"(out)
        : "r"(v ? 1u : 0u), "n"(Id)
        : "memory");
    return out != 0u;
}
__device__ __forceinline__ bool group_sync_and(int g, bool v) {
    static_assert(kGTcGroups == 3, "one named barrier per group");
    return g == 0 ? bar_red_and<1>(v) : (g == 1 ? bar_red_and<2>(v) : bar_red_and<3>(v));
}

__global__ void __launch_bounds__(kGTcThreads, kGTcBlocksPerSm)
k_guide_mlp_tc(GuideNet net, const uint32_t* counts, int q, uint32_t cap, uint32_t qn,
               const unsigned char* __restrict__ feat, float* __restrict__ mix_out, uint32_t* err) {
    extern __shared__ __align__(1024) unsigned char tc_smem[];
    const uint32_t n = counts ? min(counts[q], cap) : qn;
    const uint32_t tiles = (n + kGTcRows - 1) / kGTcRows;
    if (blockIdx.x * kGTcGroups >= tiles) return;   // uniform: before any barrier or allocation
    const int tid = threadIdx.x, warp = tid >> 5;
    const int grp = warp >> 2, gtid = tid & 127, gwarp = warp & 3;
    uint64_t* bar_feat = reinterpret_cast<uint64_t*>(tc_smem + kGTcBar) + 2 * grp;
    uint64_t* bar_mma = bar_feat + 1;
    uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + kGTcBar + 16 * kGTcGroups);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tmem_slot)),
                     "r"(kGTcCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (gtid == 0) {
        mbar_init(bar_feat, 1);
        mbar_init(bar_mma, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // weights -> the canonical operand layout, 16 bytes (8 inputs of one output) at a time;
    // the output layer's rows in accumulator-column order
#pragma unroll
    for (int l = 0; l < 4; ++l) {
        const int in = g_in(l), chunks = g_out(l) * in / 8;
        for (int c = tid; c < chunks; c += kGTcThreads) {
            const int o = c / (in / 8), j = c % (in / 8);
            const int src = l == 3 ? g_tc_out_row(o) : o;
            const uint4 v = *reinterpret_cast<const uint4*>(net.w + g_woff(l) + src * in + j * 8);
            *reinterpret_cast<uint4*>(tc_smem + g_tc_woff(l) + umma_off(o, 8 * j, in)) = v;
        }
    }
    fence_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + 64u * grp;                                  // this group's columns
    const uint32_t tmem_row = tmem + (static_cast<uint32_t>(32 * gwarp) << 16);   // this warp's lane quadrant
    const uint32_t s_base = smem_addr(tc_smem);
    unsigned char* F = tc_smem + kGTcW + grp * kGTcGroupBytes;
    unsigned char* H = F + kGFeatTileBytes;
    const uint32_t sF = smem_addr(F), sH = smem_addr(H);
    const uint32_t tstride = gridDim.x * kGTcGroups;
    uint32_t feat_phase = 0, mma_phase = 0;
    bool ok = true;
    uint32_t tile = blockIdx.x * kGTcGroups + grp;
    if (gtid == 0 && tile < tiles)
        bulk_load(F, feat + static_cast<size_t>(tile) * kGFeatTileBytes, kGFeatTileBytes, bar_feat);
    // Every decision to stop is taken on a group-wide vote, so the group's
    // threads leave the loop together and meet the same barriers.
    for (; tile < tiles; tile += tstride) {
        // layer 0 once the features have landed
        ok = group_sync_and(grp, mbar_wait(bar_feat, feat_phase));
        feat_phase ^= 1u;
        if (!ok) break;
        if (gtid == 0) {
            tc_fence_after();
            tc_layer<kGIn, kGHid>(tmem, sF, s_base + g_tc_woff(0));
            umma_commit(bar_mma);
        }
        // layers 0..2: wait, ReLU into the hidden tile, next layer
#pragma unroll 1
        for (int l = 0; l < 3; ++l) {
            ok = __all_sync(0xffffffffu, mbar_wait(bar_mma, mma_phase));   // tcgen05.ld wants whole warps
            mma_phase ^= 1u;
            tc_fence_after();
            if (l == 0 && gtid == 0 && ok && tile + tstride < tiles)   // the feature tile is free again
                bulk_load(F, feat + static_cast<size_t>(tile + tstride) * kGFeatTileBytes, kGFeatTileBytes, bar_feat);
            if (ok) tc_relu_to_hidden(tmem_row, H, static_cast<uint32_t>(gtid));
            fence_async_smem();
            tc_fence_before();
            ok = group_sync_and(grp, ok);
            if (!ok) break;
            if (gtid == 0) {
                tc_fence_after();
                if (l < 2) tc_layer<kGHid, kGHid>(tmem, sH, s_base + g_tc_woff(l + 1));
                else tc_layer<kGHid, kGOutPad>(tmem, sH, s_base + g_tc_woff(3));
                umma_commit(bar_mma);
            }
        }
        if (!ok) break;
        ok = __all_sync(0xffffffffu, mbar_wait(bar_mma, mma_phase));
        mma_phase ^= 1u;
        tc_fence_after();
        const uint32_t r = tile * kGTcRows + static_cast<uint32_t>(gtid);
        float4* dst = reinterpret_cast<float4*>(mix_out + static_cast<size_t>(r) * kGMix);
        if (ok) {
            // mixture record, streamed: logits (8 columns), then two lobes (8 columns) at a time
            uint32_t lg[8];
            tmem_ld8(tmem_row, lg);
            tmem_wait_ld();
            float mx = -1e30f;
#pragma unroll
            for (int k = 0; k < kGLobes; ++k) mx = fmaxf(mx, __uint_as_float(lg[k]));
            float e[kGLobes], sum = 0.0f;
#pragma unroll
            for (int k = 0; k < kGLobes; ++k) {
                e[k] = __expf(__uint_as_float(lg[k]) - mx);
                sum += e[k];
            }
            const float log_sum = __logf(sum), inv_sum = 1.0f / sum;
#pragma unroll
            for (int h = 0; h < 4; ++h) {   // lobes 2h, 2h + 1: columns 8 + 8h .. 8 + 8h + 7
                uint32_t v[8];
                tmem_ld8(tmem_row + 8u + 8u * h, v);
                tmem_wait_ld();
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int lobe = 2 * h + k;
                    const float4 rec = tc_lobe_record(v + 4 * k, (__uint_as_float(lg[lobe]) - mx) - log_sum);
                    if (r < n) dst[lobe] = rec;
                }
            }
            if (r < n) {
                dst[8] = make_float4(e[0] * inv_sum, e[1] * inv_sum, e[2] * inv_sum, e[3] * inv_sum);
                dst[9] = make_float4(e[4] * inv_sum, e[5] * inv_sum, e[6] * inv_sum, e[7] * inv_sum);
            }
        }
        // every thread has its row out of tensor memory before the group's next MMAs
        tc_fence_before();
        ok = group_sync_and(grp, ok);
        if (!ok) break;
    }
    if (!ok) {
        if (gtid == 0) atomicOr(err, kErrGuideTimeout);
        // let whatever is still in flight finish (bounded) before the memory goes
        mbar_wait(bar_mma, mma_phase);
        mbar_wait(bar_feat, feat_phase);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(*tmem_slot), "r"(kGTcCols)
                     : "memory");
}

}  // namespace ptb
