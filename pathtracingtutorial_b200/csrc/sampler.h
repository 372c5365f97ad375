// sampler.h -- per-path sample streams (host + device), bit-exact with the reference.
//
// Sobol: padded Owen-scrambled sampler of Part_2/src/samplers/sobol.cuh:94-117.
// Per dimension: seed = dimension hash of (px, py, dim) (sobol.cuh:77-85), the
// sample index is Owen-scrambled with it (shuffle), taken through the base-2
// van der Corput radical inverse, and Owen-scrambled again with a hash of the
// seed.  Written here in closed form: scramble(v, s) = rev(hash(rev(v), s)), so
// rev(scramble(idx, s2)) over rev(...) collapses to two hash applications and
// three bit reversals.  The hash constants define the sequence and must be the
// reference's (sobol.cuh:48-75).
//
// PCG: the reference's PCG-RXS-M-XS style step (Part_2/src/samplers/pcg.cuh:11-16)
// and pixel/frame/sample seeding (pcg.cuh:18-27), plus an optional user seed
// that is added to the pre-hash seed (0 = the reference's stream).
#pragma once

#include "pt_internal.h"

namespace ptb {

PT_HD uint32_t bit_reverse(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __brev(x);
#else
    x = ((x >> 1) & 0x55555555u) | ((x & 0x55555555u) << 1);
    x = ((x >> 2) & 0x33333333u) | ((x & 0x33333333u) << 2);
    x = ((x >> 4) & 0x0F0F0F0Fu) | ((x & 0x0F0F0F0Fu) << 4);
    x = ((x >> 8) & 0x00FF00FFu) | ((x & 0x00FF00FFu) << 8);
    return (x >> 16) | (x << 16);
#endif
}

// Avalanche mix (xorshift-multiply rounds).
PT_HD uint32_t mix32(uint32_t x) {
    x ^= x >> 17; x ^= x * 0xed5ad4bbu;
    x ^= x >> 11; x ^= x * 0xac4c1b51u;
    x ^= x >> 15; x ^= x * 0x31848babu;
    x ^= x >> 14;
    return x;
}

// Laine-Karras style nested-uniform hash on a bit-reversed value.
PT_HD uint32_t lk_hash(uint32_t x, uint32_t seed) {
    x += seed;
    x ^= x * 0x6c50b47cu;
    x ^= x * 0xb82f1e52u;
    x ^= x * 0xc7afe638u;
    x ^= x * 0x8d22f6e6u;
    return x;
}

PT_HD uint32_t pixel_dim_seed(int px, int py, uint32_t dim) {
    uint32_t h = mix32(static_cast<uint32_t>(px) + 0x9e3779b9u);
    h ^= static_cast<uint32_t>(py) + 0x9e3779b9u + (h << 6) + (h >> 2);
    h = mix32(h);
    h ^= dim + 0x9e3779b9u + (h << 6) + (h >> 2);
    return mix32(h);
}

PT_HD float u32_to_unit(uint32_t v) {
    // v * 2^-32 (exact scaling after the round-to-nearest conversion)
    return static_cast<float>(v) * 2.3283064365386963e-10f;
}

// One Sobol draw: dimension `dim` of sample `sample_index` for pixel (px, py).
PT_HD float sobol_draw(int px, int py, uint32_t sample_index, uint32_t dim) {
    const uint32_t seed = pixel_dim_seed(px, py, dim);
    const uint32_t shuffled = bit_reverse(lk_hash(bit_reverse(sample_index), seed));
    const uint32_t value = bit_reverse(lk_hash(shuffled, mix32(seed)));
    return fminf(u32_to_unit(value), 0.99999994f);
}

PT_HD uint32_t pcg_seed(int x, int y, uint32_t frame, uint32_t sample, uint32_t user_seed) {
    uint32_t s = static_cast<uint32_t>(x) * 1973u + static_cast<uint32_t>(y) * 9277u +
                 frame * 26699u + sample * 12149u + user_seed * 0x9e3779b1u;
    s = s * 747796405u + 2891336453u;
    return s | 1u;
}

PT_HD float pcg_draw(uint32_t& state) {
    const uint32_t old = state;
    state = old * 747796405u + 2891336453u;
    const uint32_t word = ((old >> ((old >> 28u) + 4u)) ^ old) * 277803737u;
    // may return exactly 1.0f, as the reference does
    return u32_to_unit((word >> 22u) ^ word);
}

// Per-path sampler state.  For Sobol `s` is the next dimension; for PCG it is
// the generator state.
struct PathRng {
    int      type;
    int      px, py;
    uint32_t sample_index;
    uint32_t s;
};

PT_HD float rng_next(PathRng& r) {
    if (r.type == PT_SAMPLER_SOBOL) {
        float v = sobol_draw(r.px, r.py, r.sample_index, r.s);
        r.s += 1u;
        return v;
    }
    return pcg_draw(r.s);
}

// Two draws that the reference takes inside one argument list; `rtl` selects
// which argument receives the first draw.
PT_HD void rng_pair(PathRng& r, int rtl, float& first_arg, float& second_arg) {
    const float a = rng_next(r);
    const float b = rng_next(r);
    if (rtl) { second_arg = a; first_arg = b; }
    else     { first_arg = a; second_arg = b; }
}

}  // namespace ptb
