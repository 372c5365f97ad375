// capi.cpp -- the extern "C" boundary (include/pt_b200.h).
//
// Mirrors the reference's host flow SceneManager::load -> buildAccel ->
// uploadToDevice -> Renderer::renderAll -> download
// (Part_2/src/main.cpp:69-78,148-149), but every entry point returns a status
// code instead of exiting, and the library owns all device memory.
#include <chrono>
#include <cmath>
#include <algorithm>
#include <cctype>
#include <cstring>
#include <exception>
#include <mutex>
#include <new>
#include <string>
#include <unordered_map>
#include <vector>

#include "device_api.h"
#include "engine.h"
#include "image_decode.h"

namespace ptb {

static thread_local std::string g_error;
void set_error(const std::string& msg) { g_error = msg; }
const std::string& get_error() { return g_error; }

}  // namespace ptb

using namespace ptb;

#define PT_GUARD_BEGIN try {
#define PT_GUARD_END                                                   \
    }                                                                  \
    catch (const std::bad_alloc&) { set_error("host allocation failed"); return PT_ERR_NOMEM; } \
    catch (const std::exception& e) { set_error(e.what()); return PT_ERR_INVALID; }

#define PT_REQUIRE(cond, msg) do { if (!(cond)) { set_error(msg); return PT_ERR_INVALID; } } while (0)

namespace {

// Per-scene render state reused by pt_render (film + integrator).
// pt_render keeps a film per scene and ONE integrator per device for all
// scenes: the integrator's wavefront state is sized for the largest pass
// (up to 2^25 paths, several GB), so one per scene would run a process that
// renders many scenes out of device memory.  pt_render calls are serialised
// by g_render_mu (each is synchronous anyway).
struct RenderCache {
    pt_film* film = nullptr;
};

std::mutex g_cache_mu;
std::mutex g_render_mu;
std::unordered_map<pt_scene*, RenderCache>& caches() {
    static std::unordered_map<pt_scene*, RenderCache> m;
    return m;
}
std::unordered_map<int, pt_integrator*>& device_integrators() {
    static std::unordered_map<int, pt_integrator*> m;
    return m;
}

void drop_cache(pt_scene* s) {
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto it = caches().find(s);
    if (it == caches().end()) return;
    if (it->second.film) { film_free(it->second.film); delete it->second.film; }
    caches().erase(it);
}

template <typename T>
int copy_out(const std::vector<T>& v, T* out, uint32_t cap) {
    PT_REQUIRE(out || v.empty(), "null output");
    PT_REQUIRE(cap >= v.size(), "output capacity too small");
    if (!v.empty()) std::memcpy(out, v.data(), v.size() * sizeof(T));
    return PT_OK;
}

void invalidate_build(pt_scene* s) {
    unpin_host_arrays(s);
    s->tables = SceneTables{};
    if (s->dev.uploaded || s->dev.device >= 0) free_scene_device(s);
}

}  // namespace

extern "C" {

const char* pt_last_error(void) { return get_error().c_str(); }
const char* pt_version(void) { return "pt_b200 1.0 (sm_100a wavefront path tracer)"; }

int pt_build_camera_frame(const pt_camera* cam, pt_camera_frame* out) {
    PT_REQUIRE(cam && out, "null argument");
    *out = camera_frame(*cam);
    return PT_OK;
}

int pt_scene_load_json(const char* path, pt_scene** out) {
    PT_REQUIRE(path && out, "null argument");
    PT_GUARD_BEGIN
    pt_scene* s = new pt_scene();
    s->host.camera = default_camera();
    s->host.settings = default_settings();
    if (!load_json_scene(path, s->host)) {
        const std::string msg = get_error();
        delete s;
        set_error(msg);
        return PT_ERR_IO;
    }
    *out = s;
    return PT_OK;
    PT_GUARD_END
}

int pt_scene_create(const pt_vertex* vertices, uint32_t num_vertices, const pt_face* faces, uint32_t num_faces,
                    const pt_material* materials, uint32_t num_materials, const pt_camera* camera,
                    const float* env_rgba, int32_t env_width, int32_t env_height, pt_scene** out) {
    PT_REQUIRE(out, "null output handle");
    PT_REQUIRE(num_vertices == 0 || vertices, "vertices is null");
    PT_REQUIRE(num_faces == 0 || faces, "faces is null");
    PT_REQUIRE(num_materials == 0 || materials, "materials is null");
    PT_REQUIRE(env_width >= 0 && env_height >= 0, "negative environment size");
    PT_REQUIRE((env_width == 0) == (env_height == 0), "environment width and height must both be zero or positive");
    PT_REQUIRE(env_width == 0 || env_rgba, "environment data is null");
    PT_GUARD_BEGIN
    pt_scene* s = new pt_scene();
    s->host.vertices.assign(vertices, vertices + num_vertices);
    s->host.faces.assign(faces, faces + num_faces);
    s->host.materials.assign(materials, materials + num_materials);
    if (s->host.materials.empty()) s->host.materials.push_back(default_material());
    s->host.camera = camera ? *camera : default_camera();
    s->host.settings = default_settings();
    if (env_width > 0) {
        s->host.env_w = env_width;
        s->host.env_h = env_height;
        s->host.env_rgba.assign(env_rgba, env_rgba + static_cast<size_t>(env_width) * env_height * 4);
    }
    *out = s;
    return PT_OK;
    PT_GUARD_END
}

int pt_scene_destroy(pt_scene* scene) {
    if (!scene) return PT_OK;
    drop_cache(scene);
    batch_forget_scene(scene);
    free_scene_device(scene);
    unpin_host_arrays(scene);
    delete scene;
    return PT_OK;
}

int pt_scene_set_punctual_lights(pt_scene* s, const pt_punctual_light* lights, uint32_t n) {
    PT_REQUIRE(s && (n == 0 || lights), "null argument");
    PT_REQUIRE(n <= 64, "at most 64 punctual lights are supported");
    s->host.punctual.assign(lights, lights + n);
    if (s->dev.uploaded) free_scene_device(s);
    return PT_OK;
}

int pt_scene_add_texture(pt_scene* s, const float* rgba, int32_t width, int32_t height, int32_t wrap_s,
                         int32_t wrap_t, int32_t* out_index) {
    PT_REQUIRE(s && out_index, "null argument");
    PT_REQUIRE((width > 0 && height > 0 && rgba) || (width == 0 && height == 0),
               "texture size must be positive (or 0 x 0 for a texture without an image)");
    PT_REQUIRE(static_cast<uint64_t>(width) * height <= (uint64_t(1) << 28), "texture too large");
    PT_GUARD_BEGIN
    HostTextureImage t;
    t.width = width;
    t.height = height;
    t.wrap_s = wrap_s;
    t.wrap_t = wrap_t;
    if (width > 0) t.rgba.assign(rgba, rgba + static_cast<size_t>(width) * height * 4);
    s->host.textures.push_back(std::move(t));
    *out_index = static_cast<int32_t>(s->host.textures.size() - 1);
    if (s->dev.uploaded) free_scene_device(s);
    return PT_OK;
    PT_GUARD_END
}

int pt_scene_get_texture(const pt_scene* s, int32_t index, float* rgba, uint64_t cap_floats, int32_t* width,
                         int32_t* height, int32_t* wrap_s, int32_t* wrap_t) {
    PT_REQUIRE(s && width && height, "null argument");
    PT_REQUIRE(index >= 0 && static_cast<size_t>(index) < s->host.textures.size(), "texture index out of range");
    const HostTextureImage& t = s->host.textures[static_cast<size_t>(index)];
    *width = t.width;
    *height = t.height;
    if (wrap_s) *wrap_s = t.wrap_s;
    if (wrap_t) *wrap_t = t.wrap_t;
    if (rgba) {
        PT_REQUIRE(cap_floats >= t.rgba.size(), "output capacity too small");
        std::memcpy(rgba, t.rgba.data(), t.rgba.size() * sizeof(float));
    }
    return PT_OK;
}

int pt_decode_image(const uint8_t* bytes, uint64_t size, uint8_t* rgba8, uint64_t cap, int32_t* width,
                    int32_t* height) {
    PT_REQUIRE(bytes && width && height, "null argument");
    PT_GUARD_BEGIN
    DecodedImage img;
    std::string err;
    if (!decode_image(bytes, static_cast<size_t>(size), img, err)) { set_error(err); return PT_ERR_IO; }
    *width = img.width;
    *height = img.height;
    if (rgba8) {
        PT_REQUIRE(cap >= img.rgba.size(), "output capacity too small");
        std::memcpy(rgba8, img.rgba.data(), img.rgba.size());
    }
    return PT_OK;
    PT_GUARD_END
}

int pt_scene_set_render_settings(pt_scene* s, const pt_render_settings* st) {
    PT_REQUIRE(s && st, "null argument");
    PT_REQUIRE(st->sample_per_frame > 0, "sample_per_frame must be positive");
    PT_REQUIRE(st->max_depth >= 0, "max_depth must be non-negative");
    PT_REQUIRE(st->sampler_type == PT_SAMPLER_PCG || st->sampler_type == PT_SAMPLER_SOBOL, "unknown sampler");
    PT_REQUIRE(st->arg_order == PT_ARGS_LTR || st->arg_order == PT_ARGS_RTL, "unknown arg order");
    PT_REQUIRE(st->trace_block == 0 || st->trace_block == 64 || st->trace_block == 128 || st->trace_block == 256,
               "trace_block must be 0, 64, 128 or 256");
    PT_REQUIRE(st->stack_depth == 0 || st->stack_depth == 32 || st->stack_depth == 64, "stack_depth must be 0, 32 or 64");
    s->host.settings = *st;
    return PT_OK;
}

int pt_scene_get_render_settings(const pt_scene* s, pt_render_settings* st) {
    PT_REQUIRE(s && st, "null argument");
    *st = s->host.settings;
    return PT_OK;
}

int pt_scene_set_camera(pt_scene* s, const pt_camera* cam) {
    PT_REQUIRE(s && cam, "null argument");
    PT_REQUIRE(cam->width > 0 && cam->height > 0, "camera resolution must be positive");
    s->host.camera = *cam;
    return PT_OK;
}

int pt_scene_get_camera(const pt_scene* s, pt_camera* cam) {
    PT_REQUIRE(s && cam, "null argument");
    *cam = s->host.camera;
    return PT_OK;
}

int pt_scene_build_accel(pt_scene* s) {
    PT_REQUIRE(s, "null scene");
    PT_GUARD_BEGIN
    if (s->tables.built) return PT_OK;   // faces are already in BVH order
    const HostScene& h = s->host;
    for (size_t i = 0; i < h.faces.size(); ++i) {
        const pt_face& f = h.faces[i];
        if (f.material_id < 0 || f.material_id >= static_cast<int>(h.materials.size())) {
            set_error("face " + std::to_string(i) + " has material id " + std::to_string(f.material_id) +
                      " outside [0, " + std::to_string(h.materials.size()) + ")");
            return PT_ERR_INVALID;
        }
    }
    invalidate_build(s);
    SceneTables& t = s->tables;
    if (!build_bvh(s->host.vertices, s->host.faces, t.bvh, t.bvh_depth)) return PT_ERR_INVALID;
    if (t.bvh_depth >= static_cast<uint32_t>(kStackDepth)) {
        set_error("BVH depth " + std::to_string(t.bvh_depth) + " exceeds the traversal stack (" +
                  std::to_string(kStackDepth) + ")");
        return PT_ERR_INVALID;
    }
    build_emissive_tables(s->host, t);
    build_env_tables(s->host, t);
    if (!build_traversal_layout(s->host, t)) return PT_ERR_INVALID;
    t.built = true;
    return PT_OK;
    PT_GUARD_END
}

int pt_scene_build_accel_device(pt_scene* s, int32_t device, const pt_build_options* options,
                                pt_build_stats* stats) {
    PT_REQUIRE(s, "null scene");
    PT_REQUIRE(device >= 0, "device must be >= 0");
    const pt_build_options o = options ? *options : pt_build_options{};
    PT_REQUIRE(o.max_leaf <= 64, "max_leaf must be at most 64");
    PT_REQUIRE(o.treelet_leaves <= 7, "treelet_leaves must be at most 7");
    PT_REQUIRE(o.passes <= 8, "passes must be at most 8");
    PT_REQUIRE(o.traversal_cost >= 0.0f && o.traversal_cost <= 16.0f, "traversal_cost must be in [0, 16]");
    PT_GUARD_BEGIN
    invalidate_build(s);
    const uint32_t leaf = o.max_leaf ? o.max_leaf : 8u;
    const int treelet = o.treelet_leaves == 0 ? 7 : (o.treelet_leaves < 3 ? 0 : static_cast<int>(o.treelet_leaves));
    // defaults measured on the 2M-triangle icosphere field and the 20M-triangle
    // scene: three passes, a node visit costed as one triangle test
    const int passes = o.passes ? static_cast<int>(o.passes) : 3;
    const float ct = o.traversal_cost > 0.0f ? o.traversal_cost : 1.0f;
    const int rc = build_accel_device(s, device, leaf, treelet, passes, ct, stats);
    if (rc != PT_OK) s->tables = SceneTables{};
    else if (stats) stats->max_leaf = leaf;
    return rc;
    PT_GUARD_END
}

int pt_scene_upload(pt_scene* s, int32_t device) {
    PT_REQUIRE(s, "null scene");
    PT_REQUIRE(device >= 0, "device must be >= 0");
    PT_GUARD_BEGIN
    return upload_scene(s, device);
    PT_GUARD_END
}

int pt_scene_info_get(const pt_scene* s, pt_scene_info* info) {
    PT_REQUIRE(s && info, "null argument");
    std::memset(info, 0, sizeof(*info));
    info->num_vertices = static_cast<uint32_t>(s->host.vertices.size());
    info->num_faces = static_cast<uint32_t>(s->host.faces.size());
    info->num_materials = static_cast<uint32_t>(s->host.materials.size());
    info->num_bvh_nodes = static_cast<uint32_t>(
        s->tables.bvh.empty() && s->tables.built ? s->tables.inner.size() + s->tables.num_leaves : s->tables.bvh.size());
    info->num_emissive_triangles = static_cast<uint32_t>(s->tables.emissive.size());
    info->num_punctual_lights = static_cast<uint32_t>(s->host.punctual.size());
    info->env_width = s->host.env_w;
    info->env_height = s->host.env_h;
    info->bvh_max_depth = s->tables.bvh_depth;
    info->num_inner_nodes = static_cast<uint32_t>(s->tables.inner.size());
    info->num_leaves = s->tables.num_leaves;
    info->frame_count = s->frame_count;
    info->device_bytes = s->dev.bytes;
    info->num_textures = static_cast<uint32_t>(s->host.textures.size());
    return PT_OK;
}

int pt_scene_build_params(const pt_scene* s, pt_scene_params* out) {
    PT_REQUIRE(s && out, "null argument");
    std::memset(out, 0, sizeof(*out));
    out->camera = camera_frame(s->host.camera);
    out->width = s->host.camera.width;
    out->height = s->host.camera.height;
    out->sample_per_frame = s->host.settings.sample_per_frame;
    out->target_samples = s->host.settings.spp;
    out->max_depth = s->host.settings.max_depth;
    out->sampler_type = s->host.settings.sampler_type;
    return PT_OK;
}

int pt_scene_get_vertices(const pt_scene* s, pt_vertex* out, uint32_t cap) {
    PT_REQUIRE(s, "null scene");
    return copy_out(s->host.vertices, out, cap);
}
int pt_scene_get_faces(const pt_scene* s, pt_face* out, uint32_t cap) {
    PT_REQUIRE(s, "null scene");
    return copy_out(s->host.faces, out, cap);
}
int pt_scene_get_materials(const pt_scene* s, pt_material* out, uint32_t cap) {
    PT_REQUIRE(s, "null scene");
    return copy_out(s->host.materials, out, cap);
}
int pt_scene_get_punctual_lights(const pt_scene* s, pt_punctual_light* out, uint32_t cap) {
    PT_REQUIRE(s, "null scene");
    return copy_out(s->host.punctual, out, cap);
}
int pt_scene_get_bvh(const pt_scene* s, pt_bvh_node* out, uint32_t cap) {
    PT_REQUIRE(s, "null scene");
    PT_GUARD_BEGIN
    if (s->tables.bvh.empty() && s->tables.built) {   // built on the device: derive from the traversal layout
        std::vector<pt_bvh_node> nodes;
        if (!nodes_from_traversal_layout(s->tables, nodes)) return PT_ERR_INVALID;
        return copy_out(nodes, out, cap);
    }
    return copy_out(s->tables.bvh, out, cap);
    PT_GUARD_END
}
int pt_scene_get_traversal(const pt_scene* s, void* inner, uint32_t cap_inner, void* tris, uint32_t cap_tris,
                           uint32_t* root_ref) {
    PT_REQUIRE(s, "null scene");
    PT_REQUIRE(s->tables.built, "scene not built");
    if (inner) {
        PT_REQUIRE(cap_inner >= s->tables.inner.size(), "inner capacity too small");
        if (!s->tables.inner.empty())
            std::memcpy(inner, s->tables.inner.data(), s->tables.inner.size() * sizeof(InnerNode));
    }
    if (tris) {
        PT_REQUIRE(cap_tris >= s->tables.tris.size(), "triangle capacity too small");
        if (!s->tables.tris.empty()) std::memcpy(tris, s->tables.tris.data(), s->tables.tris.size() * sizeof(TriRecord));
    }
    if (root_ref) *root_ref = s->tables.root_ref;
    return PT_OK;
}
int pt_scene_get_emissive(const pt_scene* s, pt_emissive_ref* refs, uint32_t cap_refs, float* face_pmf,
                          uint32_t cap_pmf, pt_alias_entry* alias, uint32_t cap_alias) {
    PT_REQUIRE(s, "null scene");
    if (int rc = copy_out(s->tables.emissive, refs, cap_refs)) return rc;
    if (int rc = copy_out(s->tables.tri_pmf, face_pmf, cap_pmf)) return rc;
    return copy_out(s->tables.tri_alias, alias, cap_alias);
}
int pt_scene_get_env_tables(const pt_scene* s, float* pmf, pt_alias_entry* alias, uint32_t cap) {
    PT_REQUIRE(s, "null scene");
    if (int rc = copy_out(s->tables.env_pmf, pmf, cap)) return rc;
    return copy_out(s->tables.env_alias, alias, cap);
}

// ---- film ----
int pt_film_create(int32_t width, int32_t height, int32_t device, pt_film** out) {
    PT_REQUIRE(out && width > 0 && height > 0 && device >= 0, "invalid film arguments");
    PT_GUARD_BEGIN
    pt_film* f = new pt_film();
    f->width = width; f->height = height; f->device = device;
    if (int rc = film_alloc(f)) { film_free(f); delete f; return rc; }
    *out = f;
    return PT_OK;
    PT_GUARD_END
}
int pt_film_destroy(pt_film* f) {
    if (!f) return PT_OK;
    film_free(f);
    delete f;
    return PT_OK;
}
int pt_film_clear(pt_film* f) {
    PT_REQUIRE(f, "null film");
    return film_clear(f);
}
int pt_film_download(const pt_film* f, float* host_rgba) {
    PT_REQUIRE(f && host_rgba, "null argument");
    return film_download(f, host_rgba, false, true);
}
int pt_write_hdr(const char* path, const float* rgba, int32_t w, int32_t h, int32_t flip_y) {
    PT_REQUIRE(path && rgba, "null argument");
    PT_REQUIRE(w > 0 && h > 0, "image size must be positive");
    PT_GUARD_BEGIN
    return write_hdr(path, rgba, w, h, flip_y != 0) ? PT_OK : PT_ERR_IO;
    PT_GUARD_END
}
int pt_read_hdr(const char* path, float* rgba, uint64_t cap, int32_t* w, int32_t* h) {
    PT_REQUIRE(path && w && h, "null argument");
    PT_GUARD_BEGIN
    std::vector<float> px;
    int32_t ww = 0, hh = 0;
    if (!load_hdr(path, px, ww, hh)) return PT_ERR_IO;
    *w = ww;
    *h = hh;
    if (rgba) {
        PT_REQUIRE(cap >= px.size(), "output capacity too small");
        std::memcpy(rgba, px.data(), px.size() * sizeof(float));
    }
    return PT_OK;
    PT_GUARD_END
}
int pt_film_download_to(const pt_film* f, float* dst, int32_t dst_is_device) {
    PT_REQUIRE(f && dst, "null argument");
    return film_download(f, dst, false, dst_is_device == 0);
}
int pt_film_download_new(const pt_film* f, float* host_rgba) {
    PT_REQUIRE(f && host_rgba, "null argument");
    return film_download(f, host_rgba, true, true);
}

// ---- integrator ----
int pt_integrator_create(const char* name, pt_integrator** out) {
    PT_REQUIRE(out, "null output handle");
    const std::string n = name ? name : "path";
    std::string low = n;
    std::transform(low.begin(), low.end(), low.begin(), [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
    if (low != "path") { set_error("unknown integrator '" + n + "' (available: path)"); return PT_ERR_INVALID; }
    PT_GUARD_BEGIN
    *out = new pt_integrator();
    return PT_OK;
    PT_GUARD_END
}
int pt_integrator_destroy(pt_integrator* integ) {
    if (!integ) return PT_OK;
    integrator_free(integ);
    delete integ;
    return PT_OK;
}
const char* pt_integrator_name(const pt_integrator* integ) { return integ ? integ->name.c_str() : ""; }

int pt_integrator_launch(pt_integrator* integ, pt_film* film, pt_scene* s, const pt_scene_params* params,
                         void* stream) {
    PT_REQUIRE(integ && film && s && params, "null argument");
    PT_GUARD_BEGIN
    return integrator_launch(integ, film, s, params, 1, stream);
    PT_GUARD_END
}
int pt_integrator_stats(const pt_integrator* integ, pt_render_stats* out) {
    PT_REQUIRE(integ && out, "null argument");
    return integrator_stats(integ, out);
}
int pt_integrator_reset_stats(pt_integrator* integ) {
    PT_REQUIRE(integ, "null argument");
    return integrator_reset_stats(integ);
}

// ---- renderer ----
int pt_renderer_render_batch(pt_integrator* integ, pt_film* film, pt_scene* s, void* stream) {
    return pt_renderer_render_frames(integ, film, s, 1, stream);
}
int pt_renderer_render_frames(pt_integrator* integ, pt_film* film, pt_scene* s, uint32_t frames, void* stream) {
    PT_REQUIRE(integ && film && s, "null argument");
    PT_REQUIRE(frames >= 1 && frames <= (1u << 20), "frame count out of range");
    pt_scene_params prm;
    pt_scene_build_params(s, &prm);
    PT_GUARD_BEGIN
    if (int rc = integrator_launch(integ, film, s, &prm, static_cast<int>(frames), stream)) return rc;
    PT_GUARD_END
    s->frame_count += frames;
    return PT_OK;
}
int pt_renderer_reset_accumulation(pt_film* film, pt_scene* s) {
    PT_REQUIRE(film && s, "null argument");
    s->frame_count = 0;
    return film_clear(film);
}

int pt_scene_set_frame_count(pt_scene* s, uint32_t frame_count) {
    PT_REQUIRE(s, "null scene");
    s->frame_count = frame_count;
    return PT_OK;
}

int pt_render(pt_scene* s, int32_t spp, float* out_rgba, int32_t out_is_device, pt_render_stats* stats) {
    PT_REQUIRE(s && out_rgba, "null argument");
    PT_REQUIRE(spp > 0, "spp must be positive");
    PT_GUARD_BEGIN
    if (!s->tables.built) {
        if (int rc = pt_scene_build_accel(s)) return rc;
    }
    if (!s->dev.uploaded) {
        int dev = 0;
        if (int rc = current_device(&dev)) return rc;
        if (int rc = upload_scene(s, dev)) return rc;
    }
    const int dev = s->dev.device;
    const int w = s->host.camera.width, h = s->host.camera.height;
    PT_REQUIRE(w > 0 && h > 0, "camera resolution must be positive");
    std::lock_guard<std::mutex> render_lock(g_render_mu);
    RenderCache rcache;
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        rcache = caches()[s];
    }
    if (rcache.film && (rcache.film->width != w || rcache.film->height != h || rcache.film->device != dev)) {
        film_free(rcache.film); delete rcache.film; rcache.film = nullptr;
    }
    if (!rcache.film) {
        if (int rc = pt_film_create(w, h, dev, &rcache.film)) return rc;
    }
    {
        std::lock_guard<std::mutex> lk(g_cache_mu);
        caches()[s] = rcache;
    }
    pt_integrator*& integ = device_integrators()[dev];
    if (!integ) {
        if (int rc = pt_integrator_create("path", &integ)) return rc;
    }
    if (int rc = pt_renderer_reset_accumulation(rcache.film, s)) return rc;
    pt_integrator_reset_stats(integ);
    const int spf = s->host.settings.sample_per_frame;
    // Renderer::renderAll: whole batches until frameCount * spf >= spp, here
    // all of them in one launch (the same samples, in the same order)
    const int64_t frames = (static_cast<int64_t>(spp) + spf - 1) / spf;
    if (int rc = pt_renderer_render_frames(integ, rcache.film, s, static_cast<uint32_t>(frames), nullptr)) return rc;
    if (int rc = integrator_check(integ, true)) return rc;
    if (int rc = film_download(rcache.film, out_rgba, false, out_is_device == 0)) return rc;
    if (stats) integrator_stats(integ, stats);
    return device_sync(dev);
    PT_GUARD_END
}

// ---- autotuner ----
namespace {

std::mutex g_tune_mu;
std::unordered_map<std::string, pt_tune_report>& tune_cache() {
    static std::unordered_map<std::string, pt_tune_report> c;
    return c;
}

int log2_floor(uint64_t v) { int b = 0; while (v > 1) { v >>= 1; ++b; } return b; }

// device : triangles : pixels : depth : sampler : environment : textures : shallow tree
std::string tune_class(const pt_scene* s) {
    const HostScene& h = s->host;
    return std::to_string(s->dev.device) + ":" + std::to_string(log2_floor(h.faces.size())) + ":" +
           std::to_string(log2_floor(uint64_t(h.camera.width) * uint64_t(h.camera.height))) + ":" +
           std::to_string(h.settings.max_depth) + ":" + std::to_string(h.settings.sampler_type) + ":" +
           std::to_string(h.env_w > 0 ? 1 : 0) + ":" + std::to_string(h.textures.empty() ? 0 : 1) + ":" +
           std::to_string(s->tables.bvh_depth < 32 ? 1 : 0);
}

// One calibration render of `spp` samples per pixel with the scene's current
// settings, through pt_render's film and integrator: wall milliseconds of the
// second of two runs (the first captures its graph and sizes its arena).
int calibration_ms(pt_scene* s, int spp, float* ms) {
    const int w = s->host.camera.width, h = s->host.camera.height;
    std::vector<float> img(static_cast<size_t>(w) * h * 4);
    for (int rep = 0; rep < 2; ++rep) {
        const auto t0 = std::chrono::steady_clock::now();
        if (int rc = pt_render(s, spp, img.data(), 0, nullptr)) return rc;
        *ms = static_cast<float>(std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
    return PT_OK;
}

}  // namespace

int pt_autotune(pt_scene* s, int32_t calib_spp, pt_tune_report* report) {
    PT_REQUIRE(s && report, "null argument");
    PT_REQUIRE(calib_spp >= 0, "calib_spp must not be negative");
    PT_GUARD_BEGIN
    std::memset(report, 0, sizeof(*report));
    if (!s->tables.built) {
        if (int rc = pt_scene_build_accel(s)) return rc;
    }
    if (!s->dev.uploaded) {
        int dev = 0;
        if (int rc = current_device(&dev)) return rc;
        if (int rc = upload_scene(s, dev)) return rc;
    }
    const std::string key = tune_class(s);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = tune_cache().find(key);
        if (it != tune_cache().end()) {
            *report = it->second;
            report->cached = 1;
            s->host.settings.paths_in_flight = report->paths_in_flight;
            s->host.settings.trace_block = report->trace_block;
            s->host.settings.stack_depth = report->stack_depth;
            return PT_OK;
        }
    }
    const uint64_t npix = uint64_t(s->host.camera.width) * uint64_t(s->host.camera.height);
    PT_REQUIRE(npix > 0, "camera resolution must be positive");
    int spp = calib_spp;
    if (spp == 0) spp = static_cast<int>(std::min<uint64_t>(256, std::max<uint64_t>(8, ((1ull << 27) + npix - 1) / npix)));
    report->calib_spp = spp;
    const pt_render_settings saved = s->host.settings;
    pt_render_settings best = saved;
    best.paths_in_flight = saved.paths_in_flight > 0 ? saved.paths_in_flight : (1 << 27);
    best.trace_block = 128;
    best.stack_depth = 64;
    float best_ms = 1e30f;
    auto attempt = [&](int pif, int block, int depth) -> int {
        if (report->candidates >= PT_TUNE_MAX_CANDIDATES) return PT_OK;
        for (int k = 0; k < report->candidates; ++k)
            if (report->cand_paths[k] == pif && report->cand_block[k] == block && report->cand_depth[k] == depth)
                return PT_OK;
        s->host.settings = saved;
        s->host.settings.paths_in_flight = pif;
        s->host.settings.trace_block = block;
        s->host.settings.stack_depth = depth;
        float ms = 0.0f;
        if (int rc = calibration_ms(s, spp, &ms)) { s->host.settings = saved; return rc; }
        const int k = report->candidates++;
        report->cand_paths[k] = pif;
        report->cand_block[k] = block;
        report->cand_depth[k] = depth;
        report->cand_ms[k] = ms;
        if (k == 0) report->default_ms = ms;
        if (ms < best_ms) { best_ms = ms; best = s->host.settings; }
        return PT_OK;
    };
    // 1) stack depth, 2) block size, 3) queue capacity -- each at the best so far
    const int pif0 = best.paths_in_flight;
    if (int rc = attempt(pif0, 128, 64)) return rc;
    if (s->tables.bvh_depth < 32)
        if (int rc = attempt(pif0, 128, 32)) return rc;
    const int depth = best.stack_depth;
    for (int block : {64, 256})
        if (int rc = attempt(pif0, block, depth)) return rc;
    const int block = best.trace_block;
    for (int lg = 24; lg <= 27; ++lg) {
        const int pif = 1 << lg;
        if (static_cast<uint64_t>(pif) < npix) continue;
        if (int rc = attempt(pif, block, depth)) return rc;
    }
    s->host.settings = saved;
    s->host.settings.paths_in_flight = best.paths_in_flight;
    s->host.settings.trace_block = best.trace_block;
    s->host.settings.stack_depth = best.stack_depth;
    report->paths_in_flight = best.paths_in_flight;
    report->trace_block = best.trace_block;
    report->stack_depth = best.stack_depth;
    report->best_ms = best_ms;
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_cache()[key] = *report;
    return PT_OK;
    PT_GUARD_END
}

int pt_render_batch(const pt_batch_item* items, uint32_t n, int32_t out_is_device, pt_batch_config* cfg,
                    pt_render_stats* stats) {
    PT_REQUIRE(n == 0 || items, "null items");
    PT_GUARD_BEGIN
    return render_batch(items, n, out_is_device, cfg, stats);
    PT_GUARD_END
}

// ---- learned guiding ----
int pt_guide_create(pt_scene* scene, uint32_t seed, pt_guide** out) {
    PT_REQUIRE(scene && out, "null argument");
    PT_GUARD_BEGIN
    return guide_create(scene, seed, out);
    PT_GUARD_END
}
int pt_guide_destroy(pt_guide* guide) {
    if (guide) guide_destroy(guide);
    return PT_OK;
}
int pt_guide_set_learning_rate(pt_guide* guide, float lr) {
    PT_REQUIRE(guide && lr > 0.0f, "invalid argument");
    guide_set_lr(guide, lr);
    return PT_OK;
}
int pt_guide_set_schedule(pt_guide* guide, float ema, float lr_half_life, float lr_floor) {
    PT_REQUIRE(guide && ema >= 0.0f && ema < 1.0f && lr_half_life >= 0.0f && lr_floor >= 0.0f && lr_floor <= 1.0f,
               "invalid argument");
    return guide_set_schedule(guide, ema, lr_half_life, lr_floor);
}
int pt_guide_set_alpha(pt_guide* guide, float alpha) {
    PT_REQUIRE(guide && alpha > 0.0f && alpha < 1.0f, "alpha must be in (0, 1)");
    guide_set_alpha(guide, alpha);
    return PT_OK;
}
int pt_guide_set_training(pt_guide* guide, int32_t paths_per_step, uint32_t samples_per_step) {
    PT_REQUIRE(guide && paths_per_step >= 0, "invalid argument");
    guide_set_training(guide, paths_per_step, samples_per_step);
    return PT_OK;
}
int pt_guide_set_inference(pt_guide* guide, int32_t kind) {
    PT_REQUIRE(guide && kind >= PT_GUIDE_INFER_DEFAULT && kind <= PT_GUIDE_INFER_SPLIT_TC, "unknown inference kind");
    guide_set_inference(guide, kind);
    return PT_OK;
}
int pt_guide_info(const pt_guide* guide, uint32_t* steps, uint32_t* last_samples) {
    PT_REQUIRE(guide, "null guide");
    return guide_info(guide, steps, last_samples);
}
int pt_guide_loss(const pt_guide* guide, float* loss) {
    PT_REQUIRE(guide && loss, "null argument");
    return guide_loss(guide, loss);
}
int pt_integrator_set_guide(pt_integrator* integ, pt_guide* guide, int32_t mode) {
    PT_REQUIRE(integ, "null integrator");
    PT_REQUIRE(mode == PT_GUIDE_OFF || mode == PT_GUIDE_USE || mode == PT_GUIDE_TRAIN, "unknown guide mode");
    PT_REQUIRE(guide || mode == PT_GUIDE_OFF, "a guide is required for this mode");
    return integrator_set_guide(integ, mode == PT_GUIDE_OFF ? nullptr : guide, mode);
}
int pt_guide_eval(pt_guide* guide, const float* pos_dir, uint32_t n, float* out_pdf) {
    PT_REQUIRE(guide && (n == 0 || (pos_dir && out_pdf)), "null argument");
    return guide_eval(guide, pos_dir, n, out_pdf);
}

int pt_guide_get_params(const pt_guide* guide, float* weights, float* grid, float* meta) {
    PT_REQUIRE(guide && weights, "null argument");
    return guide_get_params(guide, weights, grid, meta);
}
int pt_guide_backward(pt_guide* guide, const float* samples, uint32_t n, float* weight_grad, float* grid_grad) {
    PT_REQUIRE(guide && weight_grad && (n == 0 || samples), "null argument");
    return guide_backward(guide, samples, n, weight_grad, grid_grad);
}

// ---- diagnostics ----
int pt_trace_closest(pt_scene* s, const float* rays, uint32_t n, pt_hit* hits, int32_t ptrs_are_device) {
    PT_REQUIRE(s && (n == 0 || (rays && hits)), "null argument");
    return trace_rays(s, rays, n, hits, nullptr, false, ptrs_are_device != 0);
}
int pt_trace_any(pt_scene* s, const float* rays, uint32_t n, uint8_t* occluded, int32_t ptrs_are_device) {
    PT_REQUIRE(s && (n == 0 || (rays && occluded)), "null argument");
    return trace_rays(s, rays, n, nullptr, occluded, true, ptrs_are_device != 0);
}
int pt_sampler_stream(int32_t sampler_type, int32_t width, int32_t height, uint32_t frame_count,
                      int32_t sample_per_frame, int32_t sample_in_frame, uint32_t ndims, uint32_t pcg_seed,
                      int32_t device, float* out_host) {
    PT_REQUIRE(out_host, "null output");
    PT_REQUIRE(width > 0 && height > 0 && sample_per_frame > 0 && ndims > 0, "invalid sizes");
    PT_REQUIRE(sampler_type == PT_SAMPLER_PCG || sampler_type == PT_SAMPLER_SOBOL, "unknown sampler");
    return sampler_stream(sampler_type, width, height, frame_count, sample_per_frame, sample_in_frame, ndims,
                          pcg_seed, device, out_host);
}
int pt_bsdf_eval(pt_scene* s, const float* in, uint32_t n, float* out_host) {
    PT_REQUIRE(s && (n == 0 || (in && out_host)), "null argument");
    return bsdf_eval(s, in, n, out_host);
}
int pt_tonemap(const float* rgba, int32_t width, int32_t height, float exposure, uint8_t* out_rgba8,
               int32_t ptrs_are_device, int32_t device) {
    PT_REQUIRE(width >= 0 && height >= 0, "invalid sizes");
    PT_REQUIRE((width == 0 || height == 0) || (rgba && out_rgba8), "null argument");
    PT_REQUIRE(std::isfinite(exposure), "exposure must be finite");
    return tonemap(rgba, width, height, exposure, out_rgba8, ptrs_are_device != 0, device);
}

}  // extern "C"
