// engine.h -- host-side objects behind the C ABI (scene, film, integrator).
#pragma once

#include <cstdint>
#include <memory>
#include <new>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "pt_internal.h"

namespace ptb {

// Thread-local error text for pt_last_error().
void set_error(const std::string& msg);
const std::string& get_error();

// ---- host scene (HostScene, Part_2/src/scene/scene.h:24-35) ----
// A material texture as the reference keeps it (Image, Part_2/src/io/image_io.h,
// filled by loadTextures, gltf_loader.cpp:112-147): float RGBA texels (8-bit
// values / 255, no colour decoding) and the glTF sampler's GL wrap modes.
struct HostTextureImage {
    int32_t width = 0, height = 0;
    int32_t wrap_s = 10497, wrap_t = 10497;    // GL_REPEAT
    std::vector<float> rgba;                    // width * height * 4
};

struct HostScene {
    std::vector<pt_vertex>         vertices;
    std::vector<pt_face>           faces;
    std::vector<pt_material>       materials;
    std::vector<HostTextureImage>  textures;
    std::vector<pt_punctual_light> punctual;
    pt_camera                      camera{};
    std::vector<float>             env_rgba;   // env_w * env_h * 4
    int32_t                        env_w = 0, env_h = 0;
    pt_render_settings             settings{};
    std::string                    output_file = "output.hdr";
};

// Allocator whose resize() leaves new elements default-initialised (plain
// records: uninitialised), for large arrays that are written in full right
// after they are sized.
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U> struct rebind { using other = NoInitAlloc<U>; };
    NoInitAlloc() = default;
    template <class U> NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
    template <class U> void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
        ::new (static_cast<void*>(p)) U;
    }
    template <class U, class... A> void construct(U* p, A&&... a) {
        ::new (static_cast<void*>(p)) U(std::forward<A>(a)...);
    }
};

// Prep results (SceneManager::buildAccel, Part_2/src/scene/scene_manager.cpp:28-41).
struct SceneTables {
    bool built = false;
    std::vector<pt_bvh_node>     bvh;           // reference layout, DFS order
    uint32_t                     bvh_depth = 0; // edges on the longest root-leaf path
    std::vector<pt_emissive_ref> emissive;
    std::vector<float>           tri_pmf;       // per face
    std::vector<pt_alias_entry>  tri_alias;
    std::vector<float>           env_pmf;
    std::vector<pt_alias_entry>  env_alias;
    int32_t                      env_w = 0, env_h = 0;
    // traversal layout
    std::vector<InnerNode, NoInitAlloc<InnerNode>> inner;   // every record written by its builder
    std::vector<TriRecord, NoInitAlloc<TriRecord>> tris;
    float                        root_lo[3] = {0, 0, 0}, root_hi[3] = {0, 0, 0};
    uint32_t                     root_ref = 0;
    uint32_t                     num_leaves = 0;
};

// Device copies (DeviceScene, Part_2/src/scene/device_scene.h:71-97).
struct DeviceSceneBuffers {
    int      device = -1;
    bool     uploaded = false;
    void*    inner = nullptr;
    void*    tris = nullptr;
    void*    vertices = nullptr;
    void*    faces = nullptr;
    void*    materials = nullptr;
    void*    emissive = nullptr;
    void*    tri_pmf = nullptr;
    void*    tri_alias = nullptr;
    void*    env_pmf = nullptr;
    void*    env_alias = nullptr;
    void*    punctual = nullptr;
    void*    env_array = nullptr;          // cudaArray_t
    unsigned long long env_tex = 0;        // cudaTextureObject_t
    std::vector<void*> tex_arrays;         // per material texture: cudaArray_t (null when empty)
    std::vector<unsigned long long> tex_objs;   // cudaTextureObject_t (0 when empty)
    void*    tex_table = nullptr;          // device copy of tex_objs
    std::vector<size_t> tex_sizes;         // texels per uploaded texture
    std::vector<int32_t> tex_wraps;        // its wrap modes (s << 16 ^ t)
    uint64_t bytes = 0;
    size_t   sizes[11] = {};               // bytes of the buffers above, in declaration order
    int      env_w = 0, env_h = 0;
};

// Default render settings (RenderSettings defaults, scene.h:16-22).
pt_render_settings default_settings();
pt_camera default_camera();
pt_material default_material();

// ---- host prep ----
// Camera basis (buildCameraFrame, Part_2/src/camera/camera.h:36-51).
pt_camera_frame camera_frame(const pt_camera& cam);
// SAH BVH; reorders `faces`; returns false with an error on invalid input.
bool build_bvh(const std::vector<pt_vertex>& vertices, std::vector<pt_face>& faces,
               std::vector<pt_bvh_node>& nodes, uint32_t& depth);
// Vose alias table with the reference's FIFO discipline.
std::vector<pt_alias_entry> build_alias_table(const std::vector<float>& weights);
void build_emissive_tables(const HostScene& hs, SceneTables& t);
void build_env_tables(const HostScene& hs, SceneTables& t);
bool build_traversal_layout(const HostScene& hs, SceneTables& t);
bool nodes_from_traversal_layout(const SceneTables& t, std::vector<pt_bvh_node>& nodes);
// Quad -> 2 triangles (shapes::buildQuad, Part_2/src/geometry/shapes.cpp:5-22).
void add_quad(const float a[3], const float b[3], const float c[3], const float d[3], int mat,
              std::vector<pt_vertex>& verts, std::vector<pt_face>& faces);
// Scene JSON (SceneLoader::loadFromJson, Part_2/src/scene/scene_loader.cpp:240-276).
bool load_json_scene(const std::string& path, HostScene& hs);
bool load_hdr(const std::string& path, std::vector<float>& rgba, int32_t& w, int32_t& h);
bool write_hdr(const std::string& path, const float* rgba, int32_t w, int32_t h, bool flip_y);
// Radiance RGBE .hdr reader (as ImageIO::load, Part_2/src/io/image_io.cpp:19-49).
bool load_hdr(const std::string& path, std::vector<float>& rgba, int32_t& w, int32_t& h);
// Wavefront OBJ (MeshLoader::loadObj, Part_2/src/io/mesh_loader.cpp:23-112).
bool load_obj(const std::string& path, int mat, const float xform[16],
              std::vector<pt_vertex>& verts, std::vector<pt_face>& faces);

}  // namespace ptb

// Opaque C handles.
struct pt_scene {
    ptb::HostScene          host;
    ptb::SceneTables        tables;
    ptb::DeviceSceneBuffers dev;
    uint32_t                frame_count = 0;   // DeviceScene::frameCount
    std::vector<void*>      pinned;            // host arrays page-locked for uploads
};

struct pt_film {
    int32_t width = 0, height = 0, device = 0;
    void*   sum = nullptr;     // float4: rgb sum, w = sample count
    void*   comp = nullptr;    // float4: Neumaier compensation
    void*   batch = nullptr;   // float4: sum of the current launch
    void*   fresh = nullptr;   // float4: mean of the last launch ("new" surface)
    void*   resolve = nullptr; // float4: download staging
};

namespace ptb { struct Wavefront; }

struct pt_integrator {
    std::string      name = "Path";
    ptb::Wavefront*  wf = nullptr;
};
