/*
 * pt_b200.h -- C ABI of the B200 path tracer (libpt_b200.so).
 *
 * This is the drop-in boundary for the per-pixel path-tracing integrator of
 * Neroued/PathTracingTutorial Part_2.  Every entry point returns an int status
 * (PT_OK == 0); on failure pt_last_error() returns a thread-local message.
 * No entry point exits the process (the reference's CUDA_CHECK calls exit(1),
 * Part_2/src/cuda/check.h:6-24).
 *
 * Structs below are byte-for-byte layout-compatible with the reference's host
 * structs so that arrays built for the reference can be passed unchanged:
 *   pt_vertex          <-> pt::Vertex          Part_2/src/geometry/vertex.h:10-15   (64 B)
 *   pt_face            <-> pt::TriangleFace    Part_2/src/geometry/vertex.h:17-20   (16 B)
 *   pt_material        <-> pt::Material        Part_2/src/materials/material.h:8-75 (256 B)
 *   pt_camera          <-> pt::Camera          Part_2/src/camera/camera.h:12-21     (80 B)
 *   pt_camera_frame    <-> pt::CameraFrame     Part_2/src/camera/camera.h:25-34     (64 B)
 *   pt_scene_params    <-> pt::SceneParams     Part_2/src/scene/device_scene.h:19-27 (88 B)
 *   pt_punctual_light  <-> pt::PunctualLight   Part_2/src/lights/punctual_light.h:14-25 (112 B)
 *   pt_bvh_node        <-> pt::BVHNode         Part_2/src/accel/bvh_common.h:16-27  (32 B)
 *   pt_alias_entry     <-> pt::AliasEntry      Part_2/src/lights/light_sampler.h:20-23 (8 B)
 *   pt_emissive_ref    <-> pt::EmissiveTriangleRef Part_2/src/lights/light_sampler.h:13-18 (16 B)
 *
 * Ownership: the library owns every device allocation; the caller owns host
 * buffers it passes in.  A scene is thread-compatible, not thread-safe.
 */
#ifndef PT_B200_H
#define PT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define PT_OK            0
#define PT_ERR_INVALID   1  /* bad argument or unsupported input            */
#define PT_ERR_IO        2  /* file missing, unreadable or malformed          */
#define PT_ERR_CUDA      3  /* a CUDA runtime call failed                     */
#define PT_ERR_STATE     4  /* call order violated (e.g. render before build) */
#define PT_ERR_DEVICE    5  /* a kernel reported an error word (see message)  */
#define PT_ERR_NOMEM     6  /* host or device allocation failed               */

/* ---- samplers (Part_2/src/scene/device_scene.h:17) ---- */
#define PT_SAMPLER_PCG   0
#define PT_SAMPLER_SOBOL 1

/* ---- render flags ---- */
#define PT_FLAG_WATERTIGHT     1  /* watertight triangle test instead of the reference's Moller-Trumbore */
#define PT_FLAG_STAGE_TIMING   2  /* record CUDA events around every stage launch                       */
#define PT_FLAG_NO_GRAPH       4  /* launch stages directly instead of replaying a captured CUDA graph   */
#define PT_FLAG_COUNT_TRAVERSAL 8 /* count node visits / triangle tests (device counters)               */

/* ---- argument-order of paired sampler draws ----
 * The reference draws two sampler dimensions inside one call's argument list
 * (e.g. Part_2/src/integrators/direct_lighting.cuh:63-64,69-70,137-138 and
 * Part_2/src/materials/disney_bsdf.cuh:350,354,362,368).  C++ leaves the order
 * unspecified; the two compilers of the reference differ.  PT_ARGS_LTR draws the
 * first argument first, PT_ARGS_RTL draws the second argument first. */
#define PT_ARGS_LTR 0
#define PT_ARGS_RTL 1

/* ---- layout-compatible scene structs ---- */
typedef struct pt_vertex {
    float position[3]; float _pad0;
    float normal[3];   float _pad1;
    float uv[2];       float _pad2[2];
    float tangent[4];               /* xyz = tangent, w = handedness */
} pt_vertex;

typedef struct pt_face {
    uint32_t v0, v1, v2;
    int32_t  material_id;
} pt_face;

typedef struct pt_material {
    float   base_color[3]; float _pad0;                                  /*   0 */
    float   metallic, roughness, specular_tint, anisotropic;             /*  16 */
    float   sheen, sheen_tint, clearcoat, clearcoat_roughness;           /*  32 */
    float   spec_trans, ior, subsurface, specular_factor;                /*  48 */
    float   specular_color_r, specular_color_g, specular_color_b,
            anisotropy_rotation;                                         /*  64 */
    float   normal_scale; float _pad1[3];                                /*  80 */
    float   emissive[3]; float _pad2;                                    /*  96 */
    float   emissive_strength, alpha_cutoff; int32_t alpha_mode;
    float   base_alpha;                                                  /* 112 */
    int32_t double_sided; float sheen_color_r, sheen_color_g,
            sheen_color_b;                                               /* 128 */
    float   occlusion_strength, thickness_factor, attenuation_distance,
            att_color_r;                                                 /* 144 */
    float   att_color_g, att_color_b, uv_offset_x, uv_offset_y;          /* 160 */
    float   uv_scale_x, uv_scale_y, uv_rotation, _pad3;                  /* 176 */
    float   _pad4; int32_t base_color_tex, metallic_roughness_tex,
            normal_tex;                                                  /* 192 */
    int32_t emissive_tex, occlusion_tex, clearcoat_tex,
            clearcoat_roughness_tex;                                     /* 208 */
    int32_t clearcoat_normal_tex, transmission_tex, sheen_color_tex,
            sheen_roughness_tex;                                         /* 224 */
    int32_t _pad5; int32_t _pad6[3];                                     /* 240 */
} pt_material;

typedef struct pt_camera {
    float   position[3]; float _pad0;
    float   look_at[3];  float _pad1;
    float   up[3];       float _pad2;
    float   fov, aperture, focal_distance;
    int32_t width, height;
    int32_t _pad3[3];
} pt_camera;

typedef struct pt_camera_frame {
    float position[3], forward[3], right[3], up[3];
    float tan_half_fov, aspect, aperture, focal_distance;
} pt_camera_frame;

typedef struct pt_scene_params {
    pt_camera_frame camera;
    int32_t width, height, sample_per_frame, target_samples, max_depth, sampler_type;
} pt_scene_params;

typedef struct pt_punctual_light {
    float   position[3]; float _pad0;
    float   range; float _pad1[3];
    float   color[3]; float _pad2;
    float   intensity; float _pad3[3];
    float   direction[3]; float _pad4;
    float   inner_cone, outer_cone;     /* cosines */
    int32_t type;                       /* 0 point, 1 directional, 2 spot */
    float   _pad5, _pad6; float _pad7[3];
} pt_punctual_light;

typedef struct pt_bvh_node {
    float    bmin[3]; uint32_t data0;   /* leaf: first | 0x80000000, inner: left  */
    float    bmax[3]; uint32_t data1;   /* leaf: count,             inner: right */
} pt_bvh_node;

typedef struct pt_alias_entry { float prob; uint32_t alias; } pt_alias_entry;

typedef struct pt_emissive_ref {
    uint32_t triangle_index; float selection_pmf; float cdf; float _pad;
} pt_emissive_ref;

/* ---- render settings (RenderSettings, Part_2/src/scene/scene.h:16-22) ---- */
typedef struct pt_render_settings {
    int32_t  spp;               /* targetSamples                                  */
    int32_t  sample_per_frame;  /* samples per launch (batch)                     */
    int32_t  max_depth;
    int32_t  sampler_type;      /* PT_SAMPLER_*                                   */
    uint32_t pcg_seed;          /* added knob; 0 reproduces the reference seeding */
    int32_t  arg_order;         /* PT_ARGS_*                                      */
    int32_t  flags;             /* PT_FLAG_*                                      */
    int32_t  paths_in_flight;   /* added: wavefront path slots (0 = 2^27); samples of a
                                   frame run concurrently while they fit.  Results do
                                   not depend on it. */
    int32_t  trace_block;       /* added: threads per block of the traversal kernels,
                                   64, 128 or 256 (0 = 128) */
    int32_t  stack_depth;       /* added: traversal stack entries, 32 or 64 (0 = 64); a
                                   value not above the tree's depth is raised to 64.
                                   pt_autotune sets these three.  Results do not
                                   depend on them. */
} pt_render_settings;

typedef struct pt_scene_info {
    uint32_t num_vertices, num_faces, num_materials, num_bvh_nodes;
    uint32_t num_emissive_triangles, num_punctual_lights;
    int32_t  env_width, env_height;
    uint32_t bvh_max_depth, num_inner_nodes, num_leaves;
    uint32_t frame_count;
    uint64_t device_bytes;
    uint32_t num_textures;           /* material textures (HostScene::textures) */
    uint32_t _pad;
} pt_scene_info;

typedef struct pt_render_stats {
    uint64_t camera_rays, extension_rays, shadow_rays;  /* rays traced          */
    uint64_t node_visits, triangle_tests;               /* closest-hit only     */
    uint64_t shadow_node_visits, shadow_triangle_tests;
    uint64_t paths;                                      /* camera samples       */
    uint64_t extend_launches;
    double   extend_ms, shade_ms, shadow_ms, other_ms;   /* with PT_FLAG_STAGE_TIMING */
    double   total_ms;
    uint64_t kernel_launches;                            /* this library's kernels launched */
    double   guide_ms;          /* guiding network (inference, training) with PT_FLAG_STAGE_TIMING */
} pt_render_stats;

typedef struct pt_hit {
    float   t;          /* FLT_MAX on miss (SurfaceInteraction::distance)     */
    int32_t prim;       /* -1 on miss; index into the BVH-ordered face array  */
    float   u, v;       /* barycentrics of the closest hit                    */
} pt_hit;

typedef struct pt_scene      pt_scene;
typedef struct pt_film       pt_film;
typedef struct pt_integrator pt_integrator;

/* ---- errors / version ---- */
const char* pt_last_error(void);
const char* pt_version(void);

/* ---- camera (buildCameraFrame, Part_2/src/camera/camera.h:36-51) ---- */
int pt_build_camera_frame(const pt_camera* cam, pt_camera_frame* out);

/* ---- scene: load / create (SceneLoader::load, Part_2/src/scene/scene_loader.cpp:240-292) ---- */
int pt_scene_load_json(const char* path, pt_scene** out);
int pt_scene_create(const pt_vertex* vertices, uint32_t num_vertices,
                    const pt_face* faces, uint32_t num_faces,
                    const pt_material* materials, uint32_t num_materials,
                    const pt_camera* camera,
                    const float* env_rgba, int32_t env_width, int32_t env_height,
                    pt_scene** out);
int pt_scene_destroy(pt_scene* scene);
int pt_scene_set_punctual_lights(pt_scene* scene, const pt_punctual_light* lights, uint32_t n);
/* Material textures (HostScene::textures, Part_2/src/scene/scene.h:24-35; the
 * reference fills them from glTF images, gltf_loader.cpp:112-147, and uploads
 * each as a CudaTexture, cuda/cuda_texture.cu:37-62): width * height RGBA
 * floats (8-bit images as value / 255, no colour decoding -- base colour and
 * sheen colour texels are raised to 2.2 when sampled), GL wrap modes (10497
 * repeat, 33071 clamp to edge, 33648 mirrored repeat), bilinear filtering and
 * normalized coordinates on the device.  A material's *_tex fields index this
 * list.  pt_scene_add_texture appends one (out_index = its index; 0 x 0 with
 * rgba null adds a texture without an image, as a glTF texture without a
 * source becomes; lookups skip it); pt_scene_get_texture reads one back (rgba
 * may be null). */
int pt_scene_add_texture(pt_scene* scene, const float* rgba, int32_t width, int32_t height, int32_t wrap_s,
                         int32_t wrap_t, int32_t* out_index);
int pt_scene_get_texture(const pt_scene* scene, int32_t index, float* rgba, uint64_t cap_floats, int32_t* width,
                         int32_t* height, int32_t* wrap_s, int32_t* wrap_t);
/* PNG or baseline JPEG bytes -> 8-bit RGBA (grey, grey + alpha and RGB
 * expanded as the reference's stb_image call with four channels does,
 * gltf_loader.cpp:21-39).  With rgba8 null only the size is reported. */
int pt_decode_image(const uint8_t* bytes, uint64_t size, uint8_t* rgba8, uint64_t cap, int32_t* width,
                    int32_t* height);
int pt_scene_set_render_settings(pt_scene* scene, const pt_render_settings* s);   /* setSpp/setSampler/setMaxDepth */
int pt_scene_get_render_settings(const pt_scene* scene, pt_render_settings* s);
int pt_scene_set_camera(pt_scene* scene, const pt_camera* cam);                   /* SceneManager::updateCamera */
int pt_scene_get_camera(const pt_scene* scene, pt_camera* cam);

/* ---- scene: prep (SceneManager::buildAccel, Part_2/src/scene/scene_manager.cpp:28-41) ----
 * SAH BVH (reorders faces: triangle ids are BVH-ordered face indices), emissive
 * triangle and environment alias tables, and the device node layout.  Host only. */
int pt_scene_build_accel(pt_scene* scene);

/* The same prep with the BVH built on `device` instead of by the reference's
 * host builder (BVHBuilder::build, Part_2/src/accel/bvh_builder.cpp:56-221):
 * a linear BVH over 63-bit Morton codes (Karras radix tree); then, in
 * `passes` bottom-up passes (0 = 3), every inner node's treelet of
 * `treelet_leaves` leaves (0 = 7, 1-2 = off) is re-topologised to its least
 * SAH cost (Karras and Aila's treelet restructuring); subtrees become leaves
 * by the reference's two rules: at most 3 faces (fewer than its LeafThreshold
 * of 4), or at most `max_leaf` faces (0 = 8) where the SAH cost model (a
 * node visit costs `traversal_cost` triangle tests; 0 = 1.0, which traces
 * faster here than the reference's 0.5) prefers a leaf (max_leaf below 3 also
 * caps the first rule).  Faces are reordered into the tree's depth-first order as
 * pt_scene_build_accel reorders them; light and environment tables are then
 * built on the host, and the tree is walked on the host before it is accepted
 * (PT_ERR_DEVICE if malformed).  Closest-hit distances equal those of the
 * host-built tree; triangle ids, the light table order and hence the images'
 * sample streams differ from the reference's.  Deterministic: the same scene
 * and options give the same tree.  PT_ERR_INVALID when a face indexes a
 * missing vertex or material or the tree is deeper than the traversal stack
 * (64).  `options` and `stats` may be null. */
typedef struct pt_build_options {
    uint32_t max_leaf;        /* 0 = 8, at most 64             */
    uint32_t treelet_leaves;  /* 0 = 7, 1-2 = no restructuring */
    uint32_t passes;          /* 0 = 3, at most 8              */
    float    traversal_cost;  /* SAH cost of a node visit in triangle tests; 0 = 1.0 (the reference: 0.5) */
} pt_build_options;
typedef struct pt_build_stats {
    double   total_ms;      /* the whole call, host wall time                 */
    double   upload_ms;     /* vertices and faces to the device (CUDA events)  */
    double   device_ms;     /* boxes, codes, sort, tree, treelets, emission    */
    double   download_ms;   /* nodes, triangle records, reordered faces back   */
    double   tables_ms;     /* tree check, emissive and environment tables    */
    double   setup_ms;      /* device arena, stream and events                */
    uint32_t inner_nodes, leaves, depth, max_leaf;
} pt_build_stats;
int pt_scene_build_accel_device(pt_scene* scene, int32_t device, const pt_build_options* options,
                                pt_build_stats* stats);
/* ---- scene: upload (SceneManager::uploadToDevice / DeviceScene::uploadFrom,
 *      Part_2/src/scene/device_scene.cu:8-57) ---- */
int pt_scene_upload(pt_scene* scene, int32_t device);
int pt_scene_info_get(const pt_scene* scene, pt_scene_info* info);
int pt_scene_build_params(const pt_scene* scene, pt_scene_params* out);           /* DeviceScene::buildParams */
/* Read back host-side prep results (arrays sized from pt_scene_info). */
int pt_scene_get_vertices(const pt_scene* scene, pt_vertex* out, uint32_t cap);
int pt_scene_get_faces(const pt_scene* scene, pt_face* out, uint32_t cap);
int pt_scene_get_materials(const pt_scene* scene, pt_material* out, uint32_t cap);
int pt_scene_get_punctual_lights(const pt_scene* scene, pt_punctual_light* out, uint32_t cap);
int pt_scene_get_bvh(const pt_scene* scene, pt_bvh_node* out, uint32_t cap);
int pt_scene_get_emissive(const pt_scene* scene, pt_emissive_ref* refs, uint32_t cap_refs,
                          float* face_pmf, uint32_t cap_pmf,
                          pt_alias_entry* alias, uint32_t cap_alias);
int pt_scene_get_env_tables(const pt_scene* scene, float* pmf, pt_alias_entry* alias, uint32_t cap);
/* The device node layout as built (either builder): `inner` receives
 * num_inner_nodes records of 64 bytes (child 0 box lo xyz, hi xyz, child 1 box
 * lo xyz, hi xyz, ref0, ref1, meta, pad; ref bit 31 = leaf starting at that
 * triangle record, meta bits 0-1 = split axis, bit 2 = child 0's centre below
 * child 1's), `tris` num_faces records of 48 bytes (v0, v1 - v0, v2 - v0,
 * flags: bit 0 = last of its leaf, 2 pad words); root_ref = kLeafBit|first for
 * a one-leaf tree, else 0.  For tests and tools; either pointer may be null. */
int pt_scene_get_traversal(const pt_scene* scene, void* inner, uint32_t cap_inner, void* tris, uint32_t cap_tris,
                           uint32_t* root_ref);

/* ---- images (ImageIO, Part_2/src/io/image_io.cpp) ----
 * pt_write_hdr: ImageIO::write for .hdr (lines 79-121): w x h RGBA floats,
 * rows swapped when flip_y (the reference's default), written as the
 * reference's stb_image_write v1.16 writes them (RLE RGBE), byte for byte.
 * pt_read_hdr: a Radiance .hdr (flat or RLE) into RGBA floats (alpha 1);
 * with rgba null it only reports the size. */
int pt_write_hdr(const char* path, const float* rgba, int32_t width, int32_t height, int32_t flip_y);
int pt_read_hdr(const char* path, float* rgba, uint64_t cap_floats, int32_t* width, int32_t* height);

/* ---- film (Film, Part_2/src/film/film.h:9-40) ----
 * Per pixel: compensated FP32 sum (Neumaier), compensation, sample count, and
 * the mean of the last launch (the reference's "new" surface). */
int pt_film_create(int32_t width, int32_t height, int32_t device, pt_film** out);
int pt_film_destroy(pt_film* film);
int pt_film_clear(pt_film* film);
int pt_film_download(const pt_film* film, float* host_rgba);       /* Film::downloadAccumulated */
int pt_film_download_new(const pt_film* film, float* host_rgba);   /* the last launch's mean     */
/* Film::downloadAccumulated into a host or (dst_is_device) device buffer of the film's device. */
int pt_film_download_to(const pt_film* film, float* dst_rgba, int32_t dst_is_device);

/* ---- integrator plugin (Integrator, Part_2/src/integrators/integrator.h:10-20) ---- */
int         pt_integrator_create(const char* name, pt_integrator** out);          /* "path" */
int         pt_integrator_destroy(pt_integrator* integ);
const char* pt_integrator_name(const pt_integrator* integ);                       /* "Path" */
/* Integrator::launch: trace params->sample_per_frame samples per pixel with the
 * scene's current frame count and fold them into the film.  Asynchronous on
 * `stream` (a cudaStream_t; NULL = the integrator's own stream). */
int pt_integrator_launch(pt_integrator* integ, pt_film* film, pt_scene* scene,
                         const pt_scene_params* params, void* stream);
int pt_integrator_stats(const pt_integrator* integ, pt_render_stats* out);
int pt_integrator_reset_stats(pt_integrator* integ);

/* ---- renderer (Renderer, Part_2/src/renderer.h:17-55) ---- */
int pt_renderer_render_batch(pt_integrator* integ, pt_film* film, pt_scene* scene, void* stream); /* renderBatch */
/* Added: `frames` consecutive renderBatch calls in one launch (one CUDA graph);
 * identical film, frame counter and "new" image (the last frame's). */
int pt_renderer_render_frames(pt_integrator* integ, pt_film* film, pt_scene* scene, uint32_t frames,
                              void* stream);
int pt_renderer_reset_accumulation(pt_film* film, pt_scene* scene);                               /* resetAccumulation */
/* Frame counter that drives sample indices (DeviceScene::frameCount, device_scene.h:97). */
int pt_scene_set_frame_count(pt_scene* scene, uint32_t frame_count);
/* render(scene, spp) -> HDR image: build (if needed), upload (if needed), render
 * spp samples per pixel, write width*height*4 floats (RGBA, row y at y*width*4).
 * Keeps a film per scene and one integrator per device shared by all scenes;
 * concurrent pt_render calls are serialised. */
int pt_render(pt_scene* scene, int32_t spp, float* out_rgba, int32_t out_is_device,
              pt_render_stats* stats);

/* ---- autotuner (no reference counterpart: the reference has fixed launch
 *      shapes).  Times calibration renders of the scene (the pt_render path,
 *      the scene's own settings otherwise) and picks, by coordinate descent,
 *      the traversal stack depth (64, and 32 when the tree is shallower), the
 *      traversal kernels' block size (64, 128, 256) and the wavefront's queue
 *      capacity (paths in flight: 2^24 .. 2^27, as the device holds them).
 *      The choice is written into the scene's render settings (trace_block,
 *      stack_depth, paths_in_flight), so pt_render and pt_render_batch use it,
 *      and cached per device and scene class (triangles, pixels and depth,
 *      each by its power of two; sampler; environment; textures): a later
 *      call for a scene of the same class applies it without timing
 *      (cached = 1).  calib_spp: samples per pixel of a calibration render
 *      (0: enough to fill the largest queue once, at most 256).  Images do not
 *      depend on any of the tuned values. */
#define PT_TUNE_MAX_CANDIDATES 16
typedef struct pt_tune_report {
    int32_t paths_in_flight, trace_block, stack_depth;   /* the choice            */
    int32_t cached;                                      /* 1: from the cache      */
    int32_t calib_spp;                                   /* per calibration render */
    int32_t candidates;                                  /* configurations timed   */
    float   best_ms, default_ms;                         /* the choice, the defaults */
    int32_t cand_paths[PT_TUNE_MAX_CANDIDATES];
    int32_t cand_block[PT_TUNE_MAX_CANDIDATES];
    int32_t cand_depth[PT_TUNE_MAX_CANDIDATES];
    float   cand_ms[PT_TUNE_MAX_CANDIDATES];
} pt_tune_report;
int pt_autotune(pt_scene* scene, int32_t calib_spp, pt_tune_report* report);

/* ---- batched rendering (no reference counterpart: the reference renders one
 *      scene per process).  Many scenes of uneven size and sample budget are
 *      rendered by ONE persistent kernel launch captured in a CUDA graph; launch
 *      shape and chunking come from the built-in autotuner unless fixed in cfg. */
typedef struct pt_guide pt_guide;
typedef struct pt_batch_item {
    pt_scene* scene;        /* built and uploaded; all items on one device          */
    int32_t   spp;          /* samples per pixel for this item                       */
    int32_t   max_depth;    /* < 0: the scene's setting                              */
    uint32_t  first_frame;  /* frame index of the first sample (sample offset)       */
    int32_t   _pad;
    float*    out_rgba;     /* width*height*4 floats (host, or device, 16 B aligned) */
    const pt_camera* camera;/* NULL: the scene's camera; else this item's camera and
                               resolution (many cameras of one scene in one batch)   */
    pt_guide* guide;        /* NULL: BSDF sampling; else sample with this trained
                               guide (wavefront mode only; the guide is only read)  */
} pt_batch_item;

typedef struct pt_batch_config {
    int32_t block_size;     /* 64, 128 or 256 (0: autotune / default)   */
    int32_t blocks_per_sm;  /* 0: occupancy maximum                     */
    int32_t chunk_spp;      /* samples per work unit (0: default)       */
    int32_t autotune;       /* 1: time candidate shapes (cached per batch class) */
    float   tuned_ms;       /* out: calibration time of the chosen shape */
    int32_t mode;           /* PT_BATCH_AUTO / _PERSISTENT / _WAVEFRONT; out: the mode used */
    int32_t paths_in_flight;/* wavefront mode: path slots shared by all items (0: 2^27) */
    int32_t _pad;
} pt_batch_config;
/* Batch modes.  PERSISTENT: one persistent kernel traces whole paths of all
 * items (dynamic work fetch).  WAVEFRONT: every item runs the wavefront
 * integrator on its share of the path slots, the items as parallel branches
 * of one CUDA graph.  AUTO: the autotuner times both on a calibration batch. */
#define PT_BATCH_AUTO       0
#define PT_BATCH_PERSISTENT 1
#define PT_BATCH_WAVEFRONT  2

int pt_render_batch(const pt_batch_item* items, uint32_t n, int32_t out_is_device, pt_batch_config* cfg,
                    pt_render_stats* stats);

/* ---- learned path guiding (no reference counterpart).  A hash-grid + MLP
 *      network (BF16 tensor-core kernels) learns the incident radiance per
 *      position online from the integrator's own samples; while attached, the
 *      integrator draws directions from it or the BSDF by one-sample MIS
 *      (mixture probability 0.5), which keeps the estimator's expectation.
 *      Vertices with delta lobes (roughness < 0.01) are never guided. */
#define PT_GUIDE_OFF   0
#define PT_GUIDE_USE   1   /* sample with the network, do not train      */
#define PT_GUIDE_TRAIN 2   /* sample with it and train after every pass  */
int pt_guide_create(pt_scene* scene, uint32_t seed, pt_guide** out);   /* scene must be uploaded */
int pt_guide_destroy(pt_guide* guide);
int pt_guide_set_learning_rate(pt_guide* guide, float lr);
/* Training schedule.  ema > 0: renders sample with a copy of the network made
 * from an exponential moving average of its parameters (factor ema per
 * optimiser step; 0.995 by default), updated after every step, while training
 * continues on the parameters themselves (0: off; averaging switched on later
 * starts from the current parameters).  lr_half_life > 0: the learning rate
 * halves every lr_half_life optimiser steps, down to lr_floor times its set
 * value (0: constant, the default). */
int pt_guide_set_schedule(pt_guide* guide, float ema, float lr_half_life, float lr_floor);
/* probability of drawing the continuation from the network (default 0.5) */
int pt_guide_set_alpha(pt_guide* guide, float alpha);
/* online training: one optimiser step per `paths_per_step` paths of a pass
   (0 = 32768; at most 32 steps per pass), each on at most `samples_per_step`
   training samples spread evenly over the pass's (0 or more than 131072:
   131072, the most one step takes).  The defaults are 32768 and 65536. */
int pt_guide_set_training(pt_guide* guide, int32_t paths_per_step, uint32_t samples_per_step);
/* How the network is evaluated while rendering (and by pt_guide_eval); all
 * kinds give the same densities up to FP32 accumulation order.
 *   FUSED      one kernel: hash-grid encoding and the MLP on mma.sync, 16
 *              queries per warp;
 *   SPLIT_MMA  the encoding as its own kernel (one thread per query and level),
 *              then the MLP on mma.sync;
 *   SPLIT_TC   the encoding kernel, then the MLP on the tcgen05 tensor cores
 *              (128-query tiles, accumulators in tensor memory).
 * 0 selects the library default. */
#define PT_GUIDE_INFER_DEFAULT   0
#define PT_GUIDE_INFER_FUSED     1
#define PT_GUIDE_INFER_SPLIT_MMA 2
#define PT_GUIDE_INFER_SPLIT_TC  3
int pt_guide_set_inference(pt_guide* guide, int32_t kind);
/* steps taken and samples used by the last step (synchronises the device) */
int pt_guide_info(const pt_guide* guide, uint32_t* steps, uint32_t* last_samples);
/* mean training loss -w log q(dir | pos) over the last training pass (synchronises) */
int pt_guide_loss(const pt_guide* guide, float* loss);
int pt_integrator_set_guide(pt_integrator* integ, pt_guide* guide, int32_t mode);
/* Evaluate the learned directional density q(dir | pos) for n queries
 * (pos[3], dir[3] floats each) -> out[n].  Diagnostic / checkpoint check. */
int pt_guide_eval(pt_guide* guide, const float* pos_dir, uint32_t n, float* out_pdf);
/* Parameters as the renders' inference kernels use them (the averaged copy
 * while averaging is on, see pt_guide_set_schedule): weights (13312 floats: layers 32->64,
 * 64->64, 64->64, 64->48 row-major [out][in], BF16 values) and, if grid is not
 * NULL, the hash grid (16 levels x 2^19 entries x 2 features, FP16 values);
 * meta = {lo[3], inv_extent[3], scale[16], dense_limit}. */
int pt_guide_get_params(const pt_guide* guide, float* weights, float* grid, float* meta);
/* One backward pass (no optimiser step) over n samples given as n x 8 floats
 * (normalised position[3], weight, direction[3], 0); returns the weight
 * gradient (13312 floats) and, if grid_grad is not NULL, the hash-grid
 * gradient (16 x 2^19 x 2 floats), both at the parameters training runs on
 * (those pt_guide_get_params returns once averaging is off). */
int pt_guide_backward(pt_guide* guide, const float* samples, uint32_t n, float* weight_grad, float* grid_grad);

/* ---- diagnostics used by the parity tests (same kernels as the render path) ---- */
/* rays: n x 8 floats (ox, oy, oz, unused, dx, dy, dz, tmax).  tmax only used by trace_any. */
int pt_trace_closest(pt_scene* scene, const float* rays, uint32_t n, pt_hit* hits,
                     int32_t ptrs_are_device);
int pt_trace_any(pt_scene* scene, const float* rays, uint32_t n, uint8_t* occluded,
                 int32_t ptrs_are_device);
/* Added, no reference counterpart: pt_trace_closest for HOST rays and hits
 * that allocates nothing, for callers that cannot allocate device memory (a
 * host whose own pool allocator owns the device, or code where a cudaMalloc
 * is not allowed).  Rays and hits pass through a fixed file-scope device
 * array of PT_STATIC_TRACE_MAX_RAYS rays (3 MiB, held on every device that
 * loads the library until exit); n above that is rejected with
 * PT_ERR_INVALID.  The work runs on the calling thread's per-thread default
 * stream and the call returns once it is done.  Calls on one device share the
 * array and must not overlap; the first call on a device looks up the
 * array's address (and may load the module), so make it before any stream
 * capture on that device.  Resetting the device between calls is not
 * supported (the looked-up address belongs to the old context). */
#define PT_STATIC_TRACE_MAX_RAYS 65536
int pt_trace_closest_static(pt_scene* scene, const float* rays, uint32_t n, pt_hit* hits);
/* Sampler streams: out[(y*width + x)*ndims + k] = dimension k of pixel (x,y) for the
 * sample with (frame_count, sample_in_frame) as the render kernel draws it. */
int pt_sampler_stream(int32_t sampler_type, int32_t width, int32_t height,
                      uint32_t frame_count, int32_t sample_per_frame, int32_t sample_in_frame,
                      uint32_t ndims, uint32_t pcg_seed, int32_t device, float* out_host);
/* BSDF table: for n (material index, wo, wi, n, t) records evaluate the device
 * Disney BSDF.  in: n x 13 floats (mat, wo[3], wi[3], N[3], T[3]); out: n x 4 (f.rgb, pdf). */
int pt_bsdf_eval(pt_scene* scene, const float* in, uint32_t n, float* out_host);
/* Display tone mapping of the reference's preview shader
 * (Part_2/preview/tone_mapping.frag:12-29, drawn there through OpenGL; here a
 * headless buffer): c' = 1 - exp(-c * 2^exposure) per channel, sRGB transfer
 * curve, 8-bit unorm.  rgba: width*height*4 floats (A ignored); out_rgba8:
 * width*height*4 bytes (A = 255); host or device pointers.  The preview's
 * default exposure is -2.8. */
int pt_tonemap(const float* rgba, int32_t width, int32_t height, float exposure, uint8_t* out_rgba8,
               int32_t ptrs_are_device, int32_t device);

#ifdef __cplusplus
}
#endif
#endif /* PT_B200_H */
