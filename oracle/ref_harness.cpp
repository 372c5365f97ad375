// ref_harness.cpp -- C entry points over the REFERENCE's own code, compiled
// for the host from the reference tree (never copied into this repository).
// TEST INFRASTRUCTURE: built into oracle/_ref/libptref.so by oracle/Makefile;
// used by the tests to pin the oracle, by tests/golden/make_golden.py to write
// fixtures, and by bench.py's reference (CPU baseline) arm.  Nothing in the
// library links or loads it.
//
// What runs here is the reference's code:
//   SceneLoader::load                 Part_2/src/scene/scene_loader.cpp:278-292
//   BVHBuilder::build                 Part_2/src/accel/bvh_builder.cpp:56-90
//   buildEmissiveTriangleSampler /
//   buildEnvironmentSampler           Part_2/src/lights/light_sampler.cpp:57-149
//   buildCameraFrame                  Part_2/src/camera/camera.h:36-51
//   Sampler (Sobol / PCG)             Part_2/src/samplers/sampler.cuh:10-36
//   intersectScene / occludedScene    Part_2/src/accel/bvh_traversal.cuh:43-133
//   kernelPathTrace / pathTrace       Part_2/src/integrators/path.cu:62-242
// with blockIdx/threadIdx, textures and surfaces supplied by ref_shim.h.
#include "ref_shim.h"

thread_local uint3 blockIdx;
thread_local uint3 threadIdx;
thread_local dim3  blockDim;

#include <atomic>
#include <chrono>
#include <cstring>
#include <iostream>
#include <sstream>
#include <thread>
#include <vector>

#include "pt.h"
#include "math/vecmath.h"
#include "lights/envmap.h"

namespace pt {
// Host definitions of the two helpers the reference defines only for nvcc
// (vecmath.h:111-114, envmap.h:36-46), with the same formulas.
inline float4 make_float4(const vec3& v, float w) { return ::make_float4(v.x, v.y, v.z, w); }
inline vec3 sampleHDR(cudaTextureObject_t tex, const vec3& d) {
    if (tex == 0) return vec3(0.0f);
    vec2 uv = sampleSphericalMap(d);
    float4 c = tex2D<float4>(tex, uv.x, uv.y);
    return {c.x, c.y, c.z};
}
inline vec3 sampleEnvironmentRadiance(cudaTextureObject_t tex, const vec3& d) { return sampleHDR(tex, d) * TwoPi; }
}  // namespace pt

#include "accel/bvh_traversal.cuh"

struct RefRayCount { uint64_t closest = 0, any = 0; };
static thread_local RefRayCount tl_rays;

namespace pt {
// Counting forwards to the reference's traversal: every ray the integrator
// traces passes through one of these two calls.
inline SurfaceInteraction ptref_intersect(const Ray& r, const BVHNode* n, const Vertex* v, const TriangleFace* f) {
    ++tl_rays.closest;
    return intersectScene(r, n, v, f);
}
inline bool ptref_occluded(const Ray& r, const BVHNode* n, const Vertex* v, const TriangleFace* f, float tmax) {
    ++tl_rays.any;
    return occludedScene(r, n, v, f, tmax);
}
}  // namespace pt

#define intersectScene ptref_intersect
#define occludedScene ptref_occluded
#include "path_head.inc"   // Part_2/src/integrators/path.cu without PathIntegrator::launch
#undef intersectScene
#undef occludedScene

#include "accel/bvh_builder.h"
#include "camera/camera.h"
#include "lights/light_sampler.h"
#include "scene/scene.h"
#include "scene/scene_loader.h"
#include "io/image_io.h"
#include "stb/stb_image.h"

using namespace pt;

namespace {

void set_pixel_indices(int x, int y) {
    blockDim = dim3(BlockSizeX, BlockSizeY, 1);
    blockIdx = make_uint3(static_cast<unsigned>(x / BlockSizeX), static_cast<unsigned>(y / BlockSizeY), 0);
    threadIdx = make_uint3(static_cast<unsigned>(x % BlockSizeX), static_cast<unsigned>(y % BlockSizeY), 0);
}

struct Silence {
    std::streambuf* o;
    std::streambuf* e;
    std::ostringstream sink;
    Silence() : o(std::cout.rdbuf(sink.rdbuf())), e(std::cerr.rdbuf(sink.rdbuf())) {}
    ~Silence() { std::cout.rdbuf(o); std::cerr.rdbuf(e); }
};

HostScene g_loaded;

// Prep exactly as SceneManager::buildAccel (Part_2/src/scene/scene_manager.cpp:28-41).
void build_like_scene_manager(HostScene& hs) {
    if (!hs.faces.empty()) {
        BVHBuilder builder;
        hs.bvh = builder.build(hs.vertices, hs.faces, 0, static_cast<uint32_t>(hs.faces.size()));
    }
    buildEmissiveTriangleSampler(hs.vertices, hs.faces, hs.materials, hs.lightSampler);
    buildEnvironmentSampler(hs.hdrImage, hs.lightSampler);
}

HostScene scene_from_arrays(const void* verts, uint32_t nv, const void* faces, uint32_t nf, const void* mats,
                            uint32_t nm, const float* env, int ew, int eh, const void* lights, uint32_t nl) {
    HostScene hs;
    hs.vertices.resize(nv);
    if (nv) std::memcpy(hs.vertices.data(), verts, sizeof(Vertex) * nv);
    hs.faces.resize(nf);
    if (nf) std::memcpy(hs.faces.data(), faces, sizeof(TriangleFace) * nf);
    hs.materials.resize(nm);
    if (nm) std::memcpy(static_cast<void*>(hs.materials.data()), mats, sizeof(Material) * nm);
    hs.punctualLights.resize(nl);
    if (nl) std::memcpy(static_cast<void*>(hs.punctualLights.data()), lights, sizeof(PunctualLight) * nl);
    if (env && ew > 0 && eh > 0) {
        hs.hdrImage.width = ew;
        hs.hdrImage.height = eh;
        hs.hdrImage.channel = 4;
        hs.hdrImage.data.assign(env, env + static_cast<size_t>(ew) * eh * 4);
    }
    return hs;
}

}  // namespace

extern "C" {

// Sizes and field offsets of the reference structs, for layout checks.
int ref_struct_layout(int64_t* out, int cap) {
    const int64_t v[] = {
        sizeof(Vertex), offsetof(Vertex, position), offsetof(Vertex, normal), offsetof(Vertex, uv),
        offsetof(Vertex, tangent),
        sizeof(TriangleFace), offsetof(TriangleFace, materialID),
        sizeof(Material), offsetof(Material, baseColor), offsetof(Material, metallic),
        offsetof(Material, roughness), offsetof(Material, specularTint), offsetof(Material, anisotropic),
        offsetof(Material, sheen), offsetof(Material, sheenTint), offsetof(Material, clearcoat),
        offsetof(Material, clearcoatRoughness), offsetof(Material, specTrans), offsetof(Material, ior),
        offsetof(Material, subsurface), offsetof(Material, specularFactor), offsetof(Material, specularColorR),
        offsetof(Material, specularColorG), offsetof(Material, specularColorB),
        offsetof(Material, anisotropyRotation), offsetof(Material, normalScale), offsetof(Material, emissive),
        offsetof(Material, emissiveStrength), offsetof(Material, alphaCutoff), offsetof(Material, alphaMode),
        offsetof(Material, baseAlpha), offsetof(Material, doubleSided), offsetof(Material, sheenColorR),
        offsetof(Material, sheenColorG), offsetof(Material, sheenColorB), offsetof(Material, occlusionStrength),
        offsetof(Material, thicknessFactor), offsetof(Material, attenuationDistance), offsetof(Material, attColorR),
        offsetof(Material, attColorG), offsetof(Material, attColorB), offsetof(Material, uvOffsetX),
        offsetof(Material, uvOffsetY), offsetof(Material, uvScaleX), offsetof(Material, uvScaleY),
        offsetof(Material, uvRotation), offsetof(Material, baseColorTexId),
        offsetof(Material, metallicRoughnessTexId), offsetof(Material, normalTexId),
        offsetof(Material, emissiveTexId), offsetof(Material, occlusionTexId), offsetof(Material, clearcoatTexId),
        offsetof(Material, clearcoatRoughnessTexId), offsetof(Material, clearcoatNormalTexId),
        offsetof(Material, transmissionTexId), offsetof(Material, sheenColorTexId),
        offsetof(Material, sheenRoughnessTexId),
        sizeof(Camera), offsetof(Camera, position), offsetof(Camera, lookAt), offsetof(Camera, up),
        offsetof(Camera, fov), offsetof(Camera, aperture), offsetof(Camera, focalDistance),
        offsetof(Camera, width), offsetof(Camera, height),
        sizeof(CameraFrame), sizeof(SceneParams),
        sizeof(PunctualLight), offsetof(PunctualLight, position), offsetof(PunctualLight, range),
        offsetof(PunctualLight, color), offsetof(PunctualLight, intensity), offsetof(PunctualLight, direction),
        offsetof(PunctualLight, innerCone), offsetof(PunctualLight, outerCone), offsetof(PunctualLight, type),
        sizeof(BVHNode), sizeof(AliasEntry), sizeof(EmissiveTriangleRef),
    };
    const int n = static_cast<int>(sizeof(v) / sizeof(v[0]));
    if (cap < n) return -n;
    for (int i = 0; i < n; ++i) out[i] = v[i];
    return n;
}

// SceneLoader::load; counts = {nv, nf, nm, nlights, env_w, env_h}; settings = {spp, spf, maxDepth, sampler}.
int ref_load_json(const char* path, uint32_t* counts, void* camera_out, int32_t* settings) {
    Silence quiet;
    g_loaded = HostScene{};
    if (!SceneLoader::load(path, g_loaded)) return 1;
    counts[0] = static_cast<uint32_t>(g_loaded.vertices.size());
    counts[1] = static_cast<uint32_t>(g_loaded.faces.size());
    counts[2] = static_cast<uint32_t>(g_loaded.materials.size());
    counts[3] = static_cast<uint32_t>(g_loaded.punctualLights.size());
    counts[4] = static_cast<uint32_t>(g_loaded.hdrImage.channel == 4 ? g_loaded.hdrImage.width : 0);
    counts[5] = static_cast<uint32_t>(g_loaded.hdrImage.channel == 4 ? g_loaded.hdrImage.height : 0);
    std::memcpy(camera_out, &g_loaded.camera, sizeof(Camera));
    settings[0] = g_loaded.settings.targetSamples;
    settings[1] = g_loaded.settings.samplePerFrame;
    settings[2] = g_loaded.settings.maxDepth;
    settings[3] = g_loaded.settings.samplerType;
    return 0;
}

// ImageIO::write (Part_2/src/io/image_io.cpp:79-121) of a w x h RGBA image.
int ref_write_image(const char* path, const float* rgba, int w, int h, int flip_y) {
    Silence quiet;
    Image img;
    img.width = w;
    img.height = h;
    img.channel = 4;
    img.data.assign(rgba, rgba + static_cast<size_t>(w) * h * 4);
    return ImageIO::write(img, path, flip_y != 0) ? 0 : 1;
}

// Material textures of the last loaded scene: count, then per texture its size,
// wrap modes and RGBA floats (HostScene::textures as the reference's loaders fill it).
uint32_t ref_loaded_texture_count() { return static_cast<uint32_t>(g_loaded.textures.size()); }
int ref_loaded_texture(uint32_t i, int32_t* info, float* rgba) {
    if (i >= g_loaded.textures.size()) return 1;
    const Image& t = g_loaded.textures[i];
    info[0] = t.width;
    info[1] = t.height;
    info[2] = t.channel;
    info[3] = t.wrapS;
    info[4] = t.wrapT;
    if (rgba && !t.data.empty()) std::memcpy(rgba, t.data.data(), t.data.size() * sizeof(float));
    return 0;
}

// The reference's image decoder as its glTF loader calls it (stb_image from
// its 3rdparty tree, four channels forced, gltf_loader.cpp:21-39).
int ref_decode_image(const unsigned char* bytes, int size, unsigned char* rgba, int cap, int32_t* w, int32_t* h) {
    int ww = 0, hh = 0, comp = 0;
    unsigned char* data = stbi_load_from_memory(bytes, size, &ww, &hh, &comp, 4);
    if (!data) return 1;
    *w = ww;
    *h = hh;
    const int n = ww * hh * 4;
    if (rgba && cap >= n) std::memcpy(rgba, data, static_cast<size_t>(n));
    stbi_image_free(data);
    return 0;
}

int ref_loaded_arrays(void* verts, void* faces, void* mats, void* lights, float* env) {
    if (!g_loaded.vertices.empty()) std::memcpy(verts, g_loaded.vertices.data(), sizeof(Vertex) * g_loaded.vertices.size());
    if (!g_loaded.faces.empty()) std::memcpy(faces, g_loaded.faces.data(), sizeof(TriangleFace) * g_loaded.faces.size());
    if (!g_loaded.materials.empty()) std::memcpy(mats, static_cast<const void*>(g_loaded.materials.data()), sizeof(Material) * g_loaded.materials.size());
    if (!g_loaded.punctualLights.empty()) std::memcpy(lights, static_cast<const void*>(g_loaded.punctualLights.data()), sizeof(PunctualLight) * g_loaded.punctualLights.size());
    if (env && g_loaded.hdrImage.channel == 4) std::memcpy(env, g_loaded.hdrImage.data.data(), g_loaded.hdrImage.data.size() * sizeof(float));
    return 0;
}

// buildAccel on raw arrays.  faces is permuted in place into BVH order.
// sizes_out = {nodes, emissive, env_texels, env_w, env_h}.
int ref_build(const void* verts, uint32_t nv, void* faces, uint32_t nf, const void* mats, uint32_t nm,
              const float* env, int ew, int eh, void* nodes_out, uint32_t cap_nodes, void* emissive_out,
              float* tri_pmf_out, void* tri_alias_out, float* env_pmf_out, void* env_alias_out, uint32_t* sizes_out) {
    HostScene hs = scene_from_arrays(verts, nv, faces, nf, mats, nm, env, ew, eh, nullptr, 0);
    build_like_scene_manager(hs);
    if (hs.bvh.nodes.size() > cap_nodes) return 2;
    if (nf) std::memcpy(faces, hs.faces.data(), sizeof(TriangleFace) * nf);
    if (!hs.bvh.nodes.empty()) std::memcpy(nodes_out, hs.bvh.nodes.data(), sizeof(BVHNode) * hs.bvh.nodes.size());
    const HostLightSampler& ls = hs.lightSampler;
    if (emissive_out && !ls.emissiveTriangles.empty())
        std::memcpy(emissive_out, ls.emissiveTriangles.data(), sizeof(EmissiveTriangleRef) * ls.emissiveTriangles.size());
    if (tri_pmf_out && !ls.triangleSelectionPmf.empty())
        std::memcpy(tri_pmf_out, ls.triangleSelectionPmf.data(), sizeof(float) * ls.triangleSelectionPmf.size());
    if (tri_alias_out && !ls.triangleAlias.empty())
        std::memcpy(tri_alias_out, ls.triangleAlias.data(), sizeof(AliasEntry) * ls.triangleAlias.size());
    if (env_pmf_out && !ls.envPmf.empty()) std::memcpy(env_pmf_out, ls.envPmf.data(), sizeof(float) * ls.envPmf.size());
    if (env_alias_out && !ls.envAlias.empty())
        std::memcpy(env_alias_out, ls.envAlias.data(), sizeof(AliasEntry) * ls.envAlias.size());
    sizes_out[0] = static_cast<uint32_t>(hs.bvh.nodes.size());
    sizes_out[1] = static_cast<uint32_t>(ls.emissiveTriangles.size());
    sizes_out[2] = static_cast<uint32_t>(ls.envPmf.size());
    sizes_out[3] = static_cast<uint32_t>(ls.envWidth);
    sizes_out[4] = static_cast<uint32_t>(ls.envHeight);
    return 0;
}

int ref_camera_frame(const void* cam, void* out) {
    Camera c;
    std::memcpy(static_cast<void*>(&c), cam, sizeof(Camera));
    const CameraFrame f = buildCameraFrame(c);
    std::memcpy(out, &f, sizeof(CameraFrame));
    return 0;
}

// The reference's sampler stream for every pixel of a w x h launch.
int ref_sampler_stream(int type, int w, int h, uint32_t frame, int spf, int sif, uint32_t ndims, float* out) {
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            set_pixel_indices(x, y);
            Sampler s;
            if (type == 1) s.initSobol(type, x, y, frame * static_cast<uint32_t>(spf) + static_cast<uint32_t>(sif));
            else s.initPCG(type, frame, static_cast<unsigned>(sif));
            float* o = out + (static_cast<size_t>(y) * w + x) * ndims;
            for (uint32_t k = 0; k < ndims; ++k) o[k] = s.get1D();
        }
    return 0;
}

// Rays: n x 8 floats (o, -, d, tmax); direction used as given (no renormalisation).
int ref_trace(const void* nodes, const void* verts, const void* faces, const float* rays, uint32_t n, int any,
              float* hits_out, uint8_t* occl_out) {
    const BVHNode* N = static_cast<const BVHNode*>(nodes);
    const Vertex* V = static_cast<const Vertex*>(verts);
    const TriangleFace* F = static_cast<const TriangleFace*>(faces);
    for (uint32_t i = 0; i < n; ++i) {
        const float* r = rays + static_cast<size_t>(i) * 8;
        Ray ray;
        ray.origin = vec3(r[0], r[1], r[2]);
        ray.direction = vec3(r[4], r[5], r[6]);
        if (any) {
            occl_out[i] = occludedScene(ray, N, V, F, r[7]) ? 1 : 0;
        } else {
            const SurfaceInteraction si = intersectScene(ray, N, V, F);
            float* h = hits_out + static_cast<size_t>(i) * 4;
            h[0] = si.distance;
            int32_t prim = si.hit ? si.primitiveId : -1;
            std::memcpy(&h[1], &prim, 4);
            h[2] = si.hit ? si.baryU : 0.0f;
            h[3] = si.hit ? si.baryV : 0.0f;
        }
    }
    return 0;
}

// Runs kernelPathTrace for every pixel of rows row0, row0+row_step, ... for
// frames [first_frame, first_frame + num_frames).  The scene arrays are raw
// (pre-BVH); they are built exactly as SceneManager::buildAccel does.
// settings = {spp, samplePerFrame, maxDepth, samplerType}.
// out_acc / out_new: w*h*4 floats (the reference's two film surfaces).
// stats_out = {closest rays, shadow rays, paths, render seconds}.
int ref_render(const void* verts, uint32_t nv, const void* faces, uint32_t nf, const void* mats, uint32_t nm,
               const float* env, int ew, int eh, const void* lights, uint32_t nl, const void* camera,
               const int32_t* settings, uint32_t first_frame, uint32_t num_frames, int row0, int row_step,
               int nthreads, float* out_acc, float* out_new, double* stats_out) {
    HostScene hs = scene_from_arrays(verts, nv, faces, nf, mats, nm, env, ew, eh, lights, nl);
    std::memcpy(static_cast<void*>(&hs.camera), camera, sizeof(Camera));
    build_like_scene_manager(hs);
    const int w = hs.camera.width, h = hs.camera.height;
    HostTexture tex{hs.hdrImage.data.data(), hs.hdrImage.width, hs.hdrImage.height};
    d_params = SceneParams{};
    d_params.camera = buildCameraFrame(hs.camera);
    d_params.width = w;
    d_params.height = h;
    d_params.samplePerFrame = settings[1];
    d_params.targetSamples = settings[0];
    d_params.maxDepth = settings[2];
    d_params.samplerType = settings[3];
    DeviceSceneView view{};
    view.vertices = hs.vertices.data();
    view.numVertices = static_cast<uint32_t>(hs.vertices.size());
    view.faces = hs.faces.data();
    view.numFaces = static_cast<uint32_t>(hs.faces.size());
    view.materials = hs.materials.data();
    view.numMaterials = static_cast<uint32_t>(hs.materials.size());
    view.bvhNodes = hs.bvh.nodes.data();
    view.numBvhNodes = static_cast<uint32_t>(hs.bvh.nodes.size());
    view.textures = nullptr;
    view.numTextures = 0;
    const HostLightSampler& ls = hs.lightSampler;
    view.lights.emissiveTriangles = ls.emissiveTriangles.empty() ? nullptr : ls.emissiveTriangles.data();
    view.lights.numEmissiveTriangles = static_cast<uint32_t>(ls.emissiveTriangles.size());
    view.lights.triangleLightPmf = ls.triangleSelectionPmf.empty() ? nullptr : ls.triangleSelectionPmf.data();
    view.lights.triangleAlias = ls.triangleAlias.empty() ? nullptr : ls.triangleAlias.data();
    view.lights.envPmf = ls.envPmf.empty() ? nullptr : ls.envPmf.data();
    view.lights.envAlias = ls.envAlias.empty() ? nullptr : ls.envAlias.data();
    view.lights.numEnvTexels = static_cast<uint32_t>(ls.envPmf.size());
    view.lights.envWidth = ls.envWidth;
    view.lights.envHeight = ls.envHeight;
    view.lights.hdrTex = hs.hdrImage.channel == 4 ? static_cast<cudaTextureObject_t>(reinterpret_cast<uintptr_t>(&tex)) : 0;
    view.lights.punctualLights = hs.punctualLights.empty() ? nullptr : hs.punctualLights.data();
    view.lights.numPunctualLights = static_cast<uint32_t>(hs.punctualLights.size());
    std::vector<float4> acc(static_cast<size_t>(w) * h, make_float4(0, 0, 0, 0));
    std::vector<float4> fresh(static_cast<size_t>(w) * h, make_float4(0, 0, 0, 0));
    HostSurface s_new{fresh.data(), w, h}, s_acc{acc.data(), w, h};
    const cudaSurfaceObject_t surf_new = static_cast<cudaSurfaceObject_t>(reinterpret_cast<uintptr_t>(&s_new));
    const cudaSurfaceObject_t surf_acc = static_cast<cudaSurfaceObject_t>(reinterpret_cast<uintptr_t>(&s_acc));
    if (nthreads <= 0) nthreads = static_cast<int>(std::max(1u, std::thread::hardware_concurrency()));
    if (row_step <= 0) row_step = 1;
    std::vector<int> rows;
    for (int y = row0; y < h; y += row_step) rows.push_back(y);
    std::atomic<uint64_t> closest{0}, any{0};
    const auto t0 = std::chrono::steady_clock::now();
    for (uint32_t f = first_frame; f < first_frame + num_frames; ++f) {
        view.frameCount = f;
        std::vector<std::thread> pool;
        for (int t = 0; t < nthreads; ++t) {
            pool.emplace_back([&, t] {
                tl_rays = RefRayCount{};
                for (size_t k = static_cast<size_t>(t); k < rows.size(); k += static_cast<size_t>(nthreads)) {
                    const int y = rows[k];
                    for (int x = 0; x < w; ++x) {
                        set_pixel_indices(x, y);
                        kernelPathTrace(surf_new, surf_acc, view);
                    }
                }
                closest += tl_rays.closest;
                any += tl_rays.any;
            });
        }
        for (auto& th : pool) th.join();
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (out_acc) std::memcpy(out_acc, acc.data(), acc.size() * sizeof(float4));
    if (out_new) std::memcpy(out_new, fresh.data(), fresh.size() * sizeof(float4));
    stats_out[0] = static_cast<double>(closest.load());
    stats_out[1] = static_cast<double>(any.load());
    stats_out[2] = static_cast<double>(rows.size()) * w * settings[1] * num_frames;
    stats_out[3] = secs;
    return 0;
}

}  // extern "C"
