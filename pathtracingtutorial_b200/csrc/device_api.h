// device_api.h -- host functions implemented in integrator.cu (CUDA side),
// called by the C ABI layer in capi.cpp.
#pragma once

#include "engine.h"

namespace ptb {

DeviceScene device_view(const pt_scene* s);
void free_scene_device(pt_scene* s);
void unpin_host_arrays(pt_scene* s);
int  upload_scene(pt_scene* s, int device);
int  build_accel_device(pt_scene* s, int device, uint32_t max_leaf, int treelet, int passes, float ct,
                         pt_build_stats* stats);

int  film_alloc(pt_film* f);
void film_free(pt_film* f);
int  film_clear(pt_film* f);
int  film_download(const pt_film* f, float* dst, bool fresh, bool host_ptr);

void integrator_free(pt_integrator* integ);
int  integrator_launch(pt_integrator* integ, pt_film* film, pt_scene* s, const pt_scene_params* prm, int nframes,
                       void* stream);
int  integrator_check(pt_integrator* integ, bool sync);
int  integrator_stats(const pt_integrator* integ, pt_render_stats* out);
int  integrator_reset_stats(pt_integrator* integ);

int  trace_rays(pt_scene* s, const float* rays, uint32_t n, pt_hit* hits, uint8_t* occl, bool any, bool device_ptrs);
int  sampler_stream(int type, int w, int h, uint32_t frame, int spf, int sif, uint32_t ndims, uint32_t seed,
                    int device, float* out_host);
int  bsdf_eval(pt_scene* s, const float* in, uint32_t n, float* out_host);
int  tonemap(const float* rgba, int w, int h, float exposure, uint8_t* out, bool device_ptrs, int device);
int  render_batch(const pt_batch_item* in, uint32_t n, int out_is_device, pt_batch_config* cfg, pt_render_stats* stats);
void batch_forget_scene(const pt_scene* s);
int  guide_create(pt_scene* s, uint32_t seed, pt_guide** out);
void guide_destroy(pt_guide* g);
void guide_set_lr(pt_guide* g, float lr);
int  guide_set_schedule(pt_guide* g, float ema, float lr_half_life, float lr_floor);
void guide_set_alpha(pt_guide* g, float alpha);
void guide_set_training(pt_guide* g, int paths_per_step, uint32_t samples_per_step);
void guide_set_inference(pt_guide* g, int kind);
int  guide_info(const pt_guide* g, uint32_t* steps, uint32_t* samples);
int  guide_loss(const pt_guide* g, float* loss);
int  integrator_set_guide(pt_integrator* integ, pt_guide* g, int mode);
int  guide_eval(pt_guide* g, const float* qd, uint32_t n, float* out);
int  guide_get_params(const pt_guide* g, float* weights, float* grid, float* meta);
int  guide_backward(pt_guide* g, const float* samples, uint32_t n, float* wgrad, float* ggrad);
int  current_device(int* dev);
int  device_sync(int device);

}  // namespace ptb
