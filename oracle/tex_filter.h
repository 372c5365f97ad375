// tex_filter.h -- host emulation of a CUDA float4 texture fetch with
// normalized coordinates, wrap addressing and bilinear filtering (interpolation
// weights in 9-bit fixed point with 8 fractional bits, as the CUDA texture unit
// stores them).  TEST INFRASTRUCTURE shared by the oracle and the reference
// harness so both see the same environment radiance.
#pragma once

#include <vector_functions.h>
#include <vector_types.h>

#include <cmath>
#include <cstddef>

struct HostTexture {
    const float* rgba;   // width * height * 4
    int width, height;
};

struct HostSurface {
    float4* data;        // width * height
    int width, height;
};

inline int ptref_wrap(int i, int n) {
    int r = i % n;
    return r < 0 ? r + n : r;
}

// Bilinear fetch with normalized coordinates and wrap addressing.
inline float4 ptref_tex_fetch(const HostTexture* t, float u, float v) {
    const float x = (u - std::floor(u)) * static_cast<float>(t->width) - 0.5f;
    const float y = (v - std::floor(v)) * static_cast<float>(t->height) - 0.5f;
    const float fx = std::floor(x), fy = std::floor(y);
    // 9-bit fixed point weights with 8 fractional bits
    const float a = std::nearbyint((x - fx) * 256.0f) / 256.0f;
    const float b = std::nearbyint((y - fy) * 256.0f) / 256.0f;
    const int i0 = ptref_wrap(static_cast<int>(fx), t->width), i1 = ptref_wrap(static_cast<int>(fx) + 1, t->width);
    const int j0 = ptref_wrap(static_cast<int>(fy), t->height), j1 = ptref_wrap(static_cast<int>(fy) + 1, t->height);
    const float* p00 = t->rgba + (static_cast<size_t>(j0) * t->width + i0) * 4;
    const float* p10 = t->rgba + (static_cast<size_t>(j0) * t->width + i1) * 4;
    const float* p01 = t->rgba + (static_cast<size_t>(j1) * t->width + i0) * 4;
    const float* p11 = t->rgba + (static_cast<size_t>(j1) * t->width + i1) * 4;
    float r[4];
    for (int c = 0; c < 4; ++c)
        r[c] = (1.0f - a) * (1.0f - b) * p00[c] + a * (1.0f - b) * p10[c] + (1.0f - a) * b * p01[c] + a * b * p11[c];
    return make_float4(r[0], r[1], r[2], r[3]);
}
