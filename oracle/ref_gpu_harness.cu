// ref_gpu_harness.cu -- C entry points that drive the REFERENCE's own CUDA
// integrator, built for sm_100a from the reference tree (never copied here).
// TEST INFRASTRUCTURE: built into oracle/_ref/libptref_gpu.so by
// oracle/Makefile; only tests load it.  Nothing in the library links it.
//
// What runs on the GPU is the reference's code, unchanged and through its own
// plugin interface:
//   DeviceScene::uploadFrom / view / buildParams   Part_2/src/scene/device_scene.cu:8-69
//   CudaTexture (env map)                          Part_2/src/cuda/cuda_texture.cu:37-62
//   Film::init / clear / downloadAccumulated       Part_2/src/film/film.cu:8-59
//   PathIntegrator::launch -> kernelPathTrace      Part_2/src/integrators/path.cu:207-255
// and the host prep of SceneManager::buildAccel (scene_manager.cpp:28-41).
// The frame loop is Renderer::renderBatch (Part_2/src/renderer.cu:20-46):
// launch on the legacy default stream, then frameCount++.
#include <cuda_runtime.h>

#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>

#include "pt.h"
#include "accel/bvh_builder.h"
#include "camera/camera.h"
#include "film/film.h"
#include "integrators/path_integrator.h"
#include "lights/light_sampler.h"
#include "scene/device_scene.h"
#include "scene/scene.h"

using namespace pt;

namespace {

struct Quiet {
    std::streambuf* o;
    std::streambuf* e;
    std::ostringstream sink;
    Quiet() : o(std::cout.rdbuf(sink.rdbuf())), e(std::cerr.rdbuf(sink.rdbuf())) {}
    ~Quiet() { std::cout.rdbuf(o); std::cerr.rdbuf(e); }
};

struct RefGpu {
    HostScene host;
    DeviceScene dev;
    Film film;
    PathIntegrator integrator;
};

}  // namespace

extern "C" {

// A material texture as passed in: RGBA floats and GL wrap modes (the
// layout of oracle_texture in pt_oracle.h).
struct RefTexture { const float* rgba; int32_t width, height, wrap_s, wrap_t; };

int refgpu_create_textured(const void* verts, uint32_t nv, const void* faces, uint32_t nf, const void* mats,
                           uint32_t nm, const float* env, int ew, int eh, const void* camera, const int32_t* settings,
                           const void* textures, uint32_t ntex, int device, void** out);

// settings = {targetSamples, samplePerFrame, maxDepth, samplerType}.
// Scene prep is SceneManager::buildAccel's; the upload is DeviceScene::uploadFrom.
int refgpu_create(const void* verts, uint32_t nv, const void* faces, uint32_t nf, const void* mats, uint32_t nm,
                  const float* env, int ew, int eh, const void* camera, const int32_t* settings, int device,
                  void** out) {
    return refgpu_create_textured(verts, nv, faces, nf, mats, nm, env, ew, eh, camera, settings, nullptr, 0, device,
                                  out);
}

// The same with material textures (HostScene::textures, uploaded by
// DeviceScene::uploadFrom as CudaTextures, device_scene.cu:29-41).
int refgpu_create_textured(const void* verts, uint32_t nv, const void* faces, uint32_t nf, const void* mats,
                           uint32_t nm, const float* env, int ew, int eh, const void* camera, const int32_t* settings,
                           const void* textures, uint32_t ntex, int device, void** out) {
    if (cudaSetDevice(device) != cudaSuccess) return 1;
    Quiet quiet;
    RefGpu* r = new RefGpu();
    HostScene& hs = r->host;
    hs.vertices.resize(nv);
    if (nv) std::memcpy(hs.vertices.data(), verts, sizeof(Vertex) * nv);
    hs.faces.resize(nf);
    if (nf) std::memcpy(hs.faces.data(), faces, sizeof(TriangleFace) * nf);
    hs.materials.resize(nm);
    if (nm) std::memcpy(static_cast<void*>(hs.materials.data()), mats, sizeof(Material) * nm);
    if (env && ew > 0 && eh > 0) {
        hs.hdrImage.width = ew;
        hs.hdrImage.height = eh;
        hs.hdrImage.channel = 4;
        hs.hdrImage.data.assign(env, env + static_cast<size_t>(ew) * eh * 4);
    }
    const RefTexture* tx = static_cast<const RefTexture*>(textures);
    for (uint32_t k = 0; k < ntex; ++k) {
        Image img;
        img.width = tx[k].width;
        img.height = tx[k].height;
        img.channel = 4;
        img.wrapS = tx[k].wrap_s;
        img.wrapT = tx[k].wrap_t;
        if (tx[k].rgba && tx[k].width > 0 && tx[k].height > 0)
            img.data.assign(tx[k].rgba, tx[k].rgba + static_cast<size_t>(tx[k].width) * tx[k].height * 4);
        else
            img.channel = 0;   // no image: CudaTexture creates no texture for it
        hs.textures.push_back(std::move(img));
    }
    std::memcpy(static_cast<void*>(&hs.camera), camera, sizeof(Camera));
    hs.settings.targetSamples = settings[0];
    hs.settings.samplePerFrame = settings[1];
    hs.settings.maxDepth = settings[2];
    hs.settings.samplerType = settings[3];
    if (!hs.faces.empty()) {
        BVHBuilder builder;
        hs.bvh = builder.build(hs.vertices, hs.faces, 0, static_cast<uint32_t>(hs.faces.size()));
    }
    buildEmissiveTriangleSampler(hs.vertices, hs.faces, hs.materials, hs.lightSampler);
    buildEnvironmentSampler(hs.hdrImage, hs.lightSampler);
    r->dev.uploadFrom(hs);
    r->film.init(hs.camera.width, hs.camera.height);
    r->film.clear();
    if (cudaDeviceSynchronize() != cudaSuccess) { delete r; return 2; }
    *out = r;
    return 0;
}

// Renderer::resetAccumulation: frameCount = 0 and a cleared film.
int refgpu_reset(void* h) {
    RefGpu* r = static_cast<RefGpu*>(h);
    r->dev.frameCount = 0;
    r->film.clear();
    return cudaDeviceSynchronize() == cudaSuccess ? 0 : 1;
}

// `frames` calls of Renderer::renderBatch's body.  times[0] = device time of
// the whole loop (CUDA events on the legacy default stream, as renderBatch
// records them), times[1] = host wall time of the loop incl. the final sync.
int refgpu_render(void* h, int frames, double* times) {
    RefGpu* r = static_cast<RefGpu*>(h);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const auto t0 = std::chrono::steady_clock::now();
    cudaEventRecord(e0);
    for (int k = 0; k < frames; ++k) {
        const DeviceSceneView view = r->dev.view();
        const SceneParams params = r->dev.buildParams();
        r->integrator.launch(r->film.newSurface(), r->film.accSurface(), view, params);
        r->dev.frameCount++;
    }
    cudaEventRecord(e1);
    const cudaError_t err = cudaEventSynchronize(e1);
    const auto t1 = std::chrono::steady_clock::now();
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    times[0] = ms;
    times[1] = std::chrono::duration<double, std::milli>(t1 - t0).count();
    return err == cudaSuccess ? 0 : 1;
}

int refgpu_download(void* h, float* rgba) {
    static_cast<RefGpu*>(h)->film.downloadAccumulated(rgba);
    return 0;
}

uint32_t refgpu_frame_count(void* h) { return static_cast<RefGpu*>(h)->dev.frameCount; }

void refgpu_destroy(void* h) { delete static_cast<RefGpu*>(h); }

}  // extern "C"
