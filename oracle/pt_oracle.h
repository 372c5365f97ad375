// pt_oracle.h -- TEST INFRASTRUCTURE.  C interface of the CPU oracle
// (liboracle.so): a restatement of the reference's path-tracing hot path used
// only by tests, the smoke check and bench.py's CPU-baseline leg, never by the
// library.
//
// Precision 32 restates the reference's FP32 arithmetic operation by operation
// (no contraction), so that on the same host it reproduces the reference's
// IEEE host build bit for bit; precision 64 evaluates the same estimator in
// double and is the radiance judge for the GPU renders.
#pragma once

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_scene {
    const void*  vertices;  uint32_t num_vertices;     /* pt_vertex (64 B)                */
    const void*  faces;     uint32_t num_faces;        /* pt_face, BVH order              */
    const void*  materials; uint32_t num_materials;    /* pt_material (256 B)             */
    const void*  nodes;     uint32_t num_nodes;        /* pt_bvh_node (32 B), DFS order   */
    const void*  emissive;  uint32_t num_emissive;     /* pt_emissive_ref                 */
    const float* tri_pmf;                              /* per face                        */
    const void*  tri_alias;                            /* pt_alias_entry per emissive     */
    const float* env_rgba;  int32_t env_w, env_h;      /* environment image (texture)     */
    const float* env_pmf;   const void* env_alias;     /* environment tables or NULL      */
    uint32_t     num_env_texels; int32_t env_tw, env_th;
    const void*  punctual;  uint32_t num_punctual;     /* pt_punctual_light (112 B)       */
    const void*  camera_frame;                         /* pt_camera_frame (64 B)          */
    int32_t      width, height;
    const void*  textures;  uint32_t num_textures;     /* oracle_texture per material texture */
} oracle_scene;

/* a material texture: width * height RGBA floats, GL wrap modes of its sampler */
typedef struct oracle_texture {
    const float* rgba;
    int32_t width, height, wrap_s, wrap_t;
} oracle_texture;

typedef struct oracle_render_args {
    int32_t  sample_per_frame, max_depth, sampler_type, arg_rtl;
    uint32_t pcg_seed;
    uint32_t first_frame, num_frames;
    int32_t  row0, row_step, threads;
    int32_t  precision;         /* 32 or 64 */
    int32_t  col0, col1;        /* pixel columns [col0, col1) (col1 0 = width)  */
    int32_t  row_end;           /* rows row0, row0 + row_step, ... below row_end (0 = height) */
    int32_t  watertight;        /* 1: the watertight triangle and box tests (added mode) */
    int32_t  _pad;
} oracle_render_args;

typedef struct oracle_counters {
    uint64_t closest_rays, shadow_rays, node_pops, tri_tests, shadow_node_pops, shadow_tri_tests, paths;
    double   seconds;
} oracle_counters;

int oracle_build_bvh(const void* vertices, uint32_t nv, void* faces_inout, uint32_t nf, void* nodes_out,
                     uint32_t cap, uint32_t* num_nodes, uint32_t* depth);
int oracle_alias_table(const float* weights, uint32_t n, void* out);
int oracle_emissive_tables(const void* vertices, const void* faces, uint32_t nf, const void* materials, uint32_t nm,
                           void* refs_out, float* pmf_out, void* alias_out, uint32_t* count);
int oracle_env_tables(const float* rgba, int32_t w, int32_t h, float* pmf_out, void* alias_out);
int oracle_camera_frame(const void* camera, void* out);
int oracle_sampler_stream(int32_t type, int32_t w, int32_t h, uint32_t frame, int32_t spf, int32_t sif,
                          uint32_t ndims, uint32_t pcg_seed, float* out);
/* rays: n x 8 floats (o, -, d, tmax).  hits: n x 4 (t, prim bits, u, v). */
int oracle_trace(const void* nodes, const void* vertices, const void* faces, const float* rays, uint32_t n,
                 int32_t any, float* hits_out, uint8_t* occl_out, oracle_counters* counters);
/* the same with watertight = 1: Woop et al.'s triangle test on the shared
 * vertices and the widened box exit (an added mode, not the reference's) */
int oracle_trace_mode(const void* nodes, const void* vertices, const void* faces, const float* rays, uint32_t n,
                      int32_t any, int32_t watertight, float* hits_out, uint8_t* occl_out,
                      oracle_counters* counters);
/* precision 32: out_f32 = the reference's accumulated film (w*h*4, running mean).
 * precision 64: out_mean / out_var = per-pixel mean and sample variance of the
 * clamped per-sample radiance (w*h*3 doubles each). */
int oracle_render(const oracle_scene* scene, const oracle_render_args* args, float* out_f32, double* out_mean,
                  double* out_var, oracle_counters* counters);
/* in: n x 13 floats (material, wo, wi, N, T); out: n x 4 (f*|N.L| rgb, pdf) in FP32 */
int oracle_bsdf_eval(const void* materials, uint32_t nm, const float* in, uint32_t n, float* out);

#ifdef __cplusplus
}
#endif
