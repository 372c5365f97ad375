// ref_shim.h -- host stand-ins for the CUDA built-ins used by the reference's
// device code, so that the reference's own integrator
// (Part_2/src/integrators/path.cu up to PathIntegrator::launch) compiles and
// runs as plain C++ on the CPU.  TEST INFRASTRUCTURE: only the tests, the
// smoke check and bench.py's CPU-baseline leg use what is built from it.
//
// Provided here:
//   * blockIdx / threadIdx / blockDim as thread-local variables (the harness
//     sets them per pixel exactly as a 16x16 launch would);
//   * tex2D<float4> over a host texture: normalized coordinates, wrap
//     addressing, bilinear filtering with 8-bit fractional weights, which is
//     the CUDA texture-unit contract the reference configures
//     (Part_2/src/cuda/cuda_texture.cu:56-61);
//   * surf2Dread / surf2Dwrite over a host float4 surface;
//   * the two helpers the reference defines only under __CUDACC__
//     (make_float4(vec3, float), vecmath.h:111-114; sampleHDR /
//     sampleEnvironmentRadiance, envmap.h:34-46) -- defined in the harness
//     after the reference's vecmath/envmap headers are seen.
#pragma once

#include <cuda_runtime.h>
#include <vector_functions.h>

#include <cmath>
#include <cstdint>

extern thread_local uint3 blockIdx;
extern thread_local uint3 threadIdx;
extern thread_local dim3  blockDim;

#include "tex_filter.h"

template <typename T>
T tex2D(cudaTextureObject_t tex, float u, float v);

template <>
inline float4 tex2D<float4>(cudaTextureObject_t tex, float u, float v) {
    return ptref_tex_fetch(reinterpret_cast<const HostTexture*>(static_cast<uintptr_t>(tex)), u, v);
}

template <typename T>
inline void surf2Dwrite(T value, cudaSurfaceObject_t surf, int byte_x, int y) {
    HostSurface* s = reinterpret_cast<HostSurface*>(static_cast<uintptr_t>(surf));
    if (s) s->data[static_cast<size_t>(y) * s->width + byte_x / static_cast<int>(sizeof(T))] = value;
}

template <typename T>
inline void surf2Dread(T* out, cudaSurfaceObject_t surf, int byte_x, int y) {
    HostSurface* s = reinterpret_cast<HostSurface*>(static_cast<uintptr_t>(surf));
    *out = s ? s->data[static_cast<size_t>(y) * s->width + byte_x / static_cast<int>(sizeof(T))] : T{};
}
