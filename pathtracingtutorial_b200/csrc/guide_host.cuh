// guide_host.cuh -- host side of the learned guide: allocation, initialisation
// and the wavefront buffers it needs (included by integrator.cu after guide.cuh).
#pragma once

#include <cmath>
#include <random>
#include <string>
#include <vector>

namespace ptb {

inline bool guide_cuda_ok(cudaError_t e, const char* what) {
    if (e == cudaSuccess) return true;
    set_error(std::string("guide: ") + what + ": " + cudaGetErrorString(e));
    return false;
}

inline void guide_free(GuideState& g) {
    if (g.device >= 0) cudaSetDevice(g.device);
    if (g.params) cudaFree(g.params);
    if (g.work) cudaFree(g.work);
    g.params = g.work = nullptr;
    g.rows = nullptr;
    g.partial = nullptr;
    g.feat = nullptr;
    g.step = g.counters = nullptr;
    g.param_bytes = g.work_bytes = 0;
    g.npix = g.depth = 0;
}

// Network over the box [lo, hi] (cubic cells: the longest extent sets the
// scale), hash-grid resolutions 16 .. 2048 in geometric steps, He-uniform
// weights from `seed`, features uniform in +-1e-4.
inline int guide_init(GuideState& g, int device, const float lo[3], const float hi[3], uint32_t seed) {
    g.device = device;
    if (!guide_cuda_ok(cudaSetDevice(device), "cudaSetDevice")) return PT_ERR_CUDA;
    float ext = 1e-6f;
    for (int a = 0; a < 3; ++a) ext = fmaxf(ext, hi[a] - lo[a]);
    ext *= 1.02f;
    for (int a = 0; a < 3; ++a) {
        g.net.lo[a] = 0.5f * (lo[a] + hi[a]) - 0.5f * ext;
        g.net.inv_ext[a] = 1.0f / ext;
    }
    const double b = std::exp(std::log(2048.0 / 16.0) / (kGLevels - 1));
    g.net.dense_limit = 0;
    for (int l = 0; l < kGLevels; ++l) {
        g.net.scale[l] = static_cast<float>(16.0 * std::pow(b, l));
        const double r = std::floor(g.net.scale[l]) + 2.0;
        if (r * r * r <= static_cast<double>(kGTable) && g.net.dense_limit == static_cast<uint32_t>(l)) g.net.dense_limit = l + 1;
    }
    const size_t ng = static_cast<size_t>(kGLevels) * kGTable;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t off_master = al(ng * sizeof(uint2));
    const size_t off_grad = off_master + al(ng * sizeof(float2));       // 2 x u64 per entry
    const size_t off_m = off_grad + al(ng * 2 * sizeof(unsigned long long));
    const size_t off_v = off_m + al(ng * sizeof(float2));
    const size_t off_w = off_v + al(ng * sizeof(float2));
    const size_t off_wm = off_w + al(kGWeights * sizeof(__nv_bfloat16));
    const size_t wf = al(kGWeights * sizeof(float));
    const size_t off_wg = off_wm + wf;                                    // u64 per weight
    const size_t wg = al(kGWeights * sizeof(unsigned long long));
    const size_t off_step = off_wg + wg + 2 * wf;
    // parameter averages and the copies made from them
    const size_t off_gema = off_step + 256;
    const size_t off_ginf = off_gema + al(ng * sizeof(float2));
    const size_t off_wema = off_ginf + al(ng * sizeof(uint2));
    const size_t off_winf = off_wema + wf;
    const size_t off_quad = off_winf + al(kGWeights * sizeof(__nv_bfloat16));
    uint32_t quad_entries = 0;
    for (uint32_t l = 0; l < g.net.dense_limit; ++l) {
        const uint32_t res = static_cast<uint32_t>(g.net.scale[l]) + 2u;
        g.net.quad_off[l] = quad_entries;
        quad_entries += guide_quad_level_entries(res);
    }
    const size_t total = off_quad + al(static_cast<size_t>(quad_entries) * sizeof(uint4));
    if (!guide_cuda_ok(cudaMalloc(&g.params, total), "parameter allocation")) return PT_ERR_NOMEM;
    g.param_bytes = total;
    char* base = static_cast<char*>(g.params);
    g.net.grid = reinterpret_cast<uint2*>(base);
    g.net.grid_master = reinterpret_cast<float2*>(base + off_master);
    g.net.grid_grad = reinterpret_cast<unsigned long long*>(base + off_grad);
    g.net.grid_m = reinterpret_cast<float2*>(base + off_m);
    g.net.grid_v = reinterpret_cast<float2*>(base + off_v);
    g.net.w = reinterpret_cast<__nv_bfloat16*>(base + off_w);
    g.net.w_master = reinterpret_cast<float*>(base + off_wm);
    g.net.w_grad = reinterpret_cast<unsigned long long*>(base + off_wg);
    g.net.w_m = reinterpret_cast<float*>(base + off_wg + wg);
    g.net.w_v = reinterpret_cast<float*>(base + off_wg + wg + wf);
    g.step = reinterpret_cast<uint32_t*>(base + off_step);
    g.net.loss = reinterpret_cast<float*>(base + off_step + 16);
    g.net.loss_fix = reinterpret_cast<unsigned long long*>(base + off_step + 32);
    g.net.ema = kGuideEma;
    g.net.grid_ema = reinterpret_cast<float2*>(base + off_gema);
    g.net.grid_inf = reinterpret_cast<uint2*>(base + off_ginf);
    g.net.w_ema = reinterpret_cast<float*>(base + off_wema);
    g.net.w_inf = reinterpret_cast<__nv_bfloat16*>(base + off_winf);
    g.net.quad = quad_entries ? reinterpret_cast<uint4*>(base + off_quad) : nullptr;
    // host-side initial values
    std::mt19937 rng(seed);
    std::vector<float> gm(2 * ng);
    std::uniform_real_distribution<float> uf(-1e-4f, 1e-4f);
    for (float& x : gm) x = uf(rng);
    std::vector<__half2> gh(2 * ng);   // the pair table (see GuideNet::grid)
    for (size_t i = 0; i < ng; ++i) {
        const size_t next = (i & ~static_cast<size_t>(kGTable - 1)) | ((i + 1) & (kGTable - 1));
        gh[2 * i] = __floats2half2_rn(gm[2 * i], gm[2 * i + 1]);
        gh[2 * i + 1] = __floats2half2_rn(gm[2 * next], gm[2 * next + 1]);
    }
    std::vector<float> w(kGWeights);
    std::vector<__nv_bfloat16> wb(kGWeights);
    for (int l = 0; l < 4; ++l) {
        const float lim = std::sqrt(6.0f / g_in(l)) * (l == 3 ? 0.1f : 1.0f);
        std::uniform_real_distribution<float> uw(-lim, lim);
        for (int i = 0; i < g_out(l) * g_in(l); ++i) {
            float v = uw(rng);
            if (l == 3 && i / g_in(l) >= kGOut) v = 0.0f;   // padded outputs
            w[g_woff(l) + i] = v;
        }
    }
    for (int i = 0; i < kGWeights; ++i) wb[i] = __float2bfloat16_rn(w[i]);
    bool ok = guide_cuda_ok(cudaMemcpy(g.net.grid, gh.data(), ng * sizeof(uint2), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemcpy(g.net.grid_master, gm.data(), ng * sizeof(float2), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemset(g.net.grid_grad, 0, off_w - off_grad), "clear") &&
              guide_cuda_ok(cudaMemcpy(g.net.w, wb.data(), kGWeights * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemcpy(g.net.w_master, w.data(), kGWeights * sizeof(float), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemset(g.net.w_grad, 0, wg + 2 * wf), "clear") &&
              guide_cuda_ok(cudaMemset(g.step, 0, 256), "clear") &&
              guide_cuda_ok(cudaMemcpy(g.net.grid_inf, gh.data(), ng * sizeof(uint2), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemcpy(g.net.grid_ema, gm.data(), ng * sizeof(float2), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemcpy(g.net.w_inf, wb.data(), kGWeights * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaMemcpy(g.net.w_ema, w.data(), kGWeights * sizeof(float), cudaMemcpyHostToDevice), "upload") &&
              guide_cuda_ok(cudaFuncSetAttribute(k_guide_train, cudaFuncAttributeMaxDynamicSharedMemorySize, kGTrainSmem), "smem") &&
              guide_cuda_ok(cudaFuncSetAttribute(k_guide_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, kGInferSmem), "smem") &&
              guide_cuda_ok(cudaFuncSetAttribute(k_guide_mlp_mma, cudaFuncAttributeMaxDynamicSharedMemorySize, kGInferSmem), "smem") &&
              guide_cuda_ok(cudaFuncSetAttribute(k_guide_mlp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, kGTcSmem), "smem");
    return ok ? PT_OK : PT_ERR_CUDA;
}

// Mixture buffer (one per queue entry), training records (depth x npix x 64 B),
// training samples and counters, sized for npix paths and max_depth bounces.
// Work buffers for passes of `npix` paths: the mixtures always, the training
// records and samples only when `records` (training) -- a guide that only
// samples can then run passes as large as the plain integrator's.
inline int guide_prepare_work(GuideState& g, int npix, int depth, bool records) {
    if (g.work && g.npix == npix && g.depth == depth && (g.rec != nullptr || !records)) return PT_OK;
    if (!guide_cuda_ok(cudaSetDevice(g.device), "cudaSetDevice")) return PT_ERR_CUDA;
    if (g.work) { cudaFree(g.work); g.work = nullptr; }
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t P = static_cast<size_t>(npix), D = static_cast<size_t>(std::max(depth, 1));
    const size_t cap = records ? std::min<size_t>(P * D, size_t(1) << 24) : 0;
    const size_t b_mix = al(P * kGMix * sizeof(float));
    const size_t b_feat = al(static_cast<size_t>(guide_feat_rows(static_cast<uint32_t>(P))) * kGIn * sizeof(__nv_bfloat16));
    const size_t b_rec = records ? al(D * P * 4 * sizeof(float4)) : 0;
    const size_t b_smp = al(cap * sizeof(GuideSample));
    size_t scan_tmp = 0;
    if (records &&
        !guide_cuda_ok(cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp, static_cast<uint32_t*>(nullptr),
                                                     static_cast<uint32_t*>(nullptr), static_cast<int>(P + 1)),
                       "scan size"))
        return PT_ERR_CUDA;
    const size_t b_scan = records ? 2 * al((P + 1) * sizeof(uint32_t)) + al(scan_tmp) : 0;
    const size_t b_rows = records ? al(kGRowStoreElems * sizeof(__nv_bfloat16)) : 0;
    const size_t b_part = records ? al(static_cast<size_t>(kGDwChunks) * kGWeights * sizeof(float)) : 0;
    const size_t total = b_mix + b_rec + b_smp + b_scan + b_rows + b_part + 256 + b_feat;
    if (!guide_cuda_ok(cudaMalloc(&g.work, total), "work allocation")) return PT_ERR_NOMEM;
    g.work_bytes = total;
    char* base = static_cast<char*>(g.work);
    g.mix = reinterpret_cast<float*>(base);
    g.rec = records ? reinterpret_cast<float4*>(base + b_mix) : nullptr;
    g.samples = records ? reinterpret_cast<GuideSample*>(base + b_mix + b_rec) : nullptr;
    g.counters = reinterpret_cast<uint32_t*>(base + b_mix + b_rec + b_smp + b_scan + b_rows + b_part);
    g.rows = records ? reinterpret_cast<__nv_bfloat16*>(base + b_mix + b_rec + b_smp + b_scan) : nullptr;
    g.partial = records ? reinterpret_cast<float*>(base + b_mix + b_rec + b_smp + b_scan + b_rows) : nullptr;
    g.scan_counts = records ? reinterpret_cast<uint32_t*>(base + b_mix + b_rec + b_smp) : nullptr;
    g.scan_offsets = records ? reinterpret_cast<uint32_t*>(base + b_mix + b_rec + b_smp + al((P + 1) * 4)) : nullptr;
    g.scan_tmp = records ? base + b_mix + b_rec + b_smp + 2 * al((P + 1) * 4) : nullptr;
    g.scan_tmp_bytes = records ? scan_tmp : 0;
    g.feat = reinterpret_cast<unsigned char*>(base + b_mix + b_rec + b_smp + b_scan + b_rows + b_part + 256);
    g.sample_cap = static_cast<uint32_t>(cap);
    g.npix = npix;
    g.depth = depth;
    const bool ok = (b_rec == 0 || guide_cuda_ok(cudaMemset(g.rec, 0, b_rec), "clear")) &&
                    guide_cuda_ok(cudaMemset(g.counters, 0, 256), "clear");
    return ok ? PT_OK : PT_ERR_CUDA;
}

}  // namespace ptb
