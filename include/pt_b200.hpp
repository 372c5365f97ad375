// pt_b200.hpp -- C++ host API over the C ABI (pt_b200.h), with the class
// names and call flow of the reference's renderer so that a caller of
// Neroued/PathTracingTutorial Part_2 can switch with minimal edits:
//
//   pt::SceneManager  load / buildAccel / uploadToDevice / setSpp / setSampler
//                     (Part_2/src/scene/scene_manager.h:11-45)
//   pt::Integrator    launch(film, scene, params) / name()
//                     (Part_2/src/integrators/integrator.h:10-20)
//   pt::PathIntegrator                    (Part_2/src/integrators/path_integrator.h:7-15)
//   pt::Renderer      renderBatch / renderAll / downloadCurrentImage /
//                     resetAccumulation / currentSpp / isComplete
//                     (Part_2/src/renderer.h:17-55)
//   pt::render(scene, spp) -> RGBA float image
//
// Differences from the reference: errors throw pt::Error (carrying the C
// status and pt_last_error()) instead of exiting the process; launches take an
// optional cudaStream_t.  Header only; link libpt_b200.so.
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "pt_b200.h"

namespace pt {

class Error : public std::runtime_error {
public:
    Error(int code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int code() const { return code_; }

private:
    int code_;
};

inline void check(int rc) {
    if (rc != PT_OK) throw Error(rc, pt_last_error());
}

class SceneManager {
public:
    SceneManager() = default;
    ~SceneManager() { if (s_) pt_scene_destroy(s_); }
    SceneManager(const SceneManager&) = delete;
    SceneManager& operator=(const SceneManager&) = delete;

    void load(const std::string& path) { reset(); check(pt_scene_load_json(path.c_str(), &s_)); }
    void create(const std::vector<pt_vertex>& v, const std::vector<pt_face>& f, const std::vector<pt_material>& m,
                const pt_camera& cam, const std::vector<float>& env_rgba = {}, int env_w = 0, int env_h = 0) {
        reset();
        check(pt_scene_create(v.data(), static_cast<uint32_t>(v.size()), f.data(), static_cast<uint32_t>(f.size()),
                              m.data(), static_cast<uint32_t>(m.size()), &cam,
                              env_rgba.empty() ? nullptr : env_rgba.data(), env_w, env_h, &s_));
    }
    void buildAccel() { check(pt_scene_build_accel(s_)); }
    void uploadToDevice(int device = 0) { check(pt_scene_upload(s_, device)); }

    void setSpp(int spp) { auto s = settings(); s.spp = spp; check(pt_scene_set_render_settings(s_, &s)); }
    void setMaxDepth(int d) { auto s = settings(); s.max_depth = d; check(pt_scene_set_render_settings(s_, &s)); }
    void setSampler(int type) { auto s = settings(); s.sampler_type = type; check(pt_scene_set_render_settings(s_, &s)); }
    void updateCamera(const pt_camera& cam) { check(pt_scene_set_camera(s_, &cam)); }
    pt_camera camera() const { pt_camera c; check(pt_scene_get_camera(s_, &c)); return c; }
    pt_render_settings settings() const { pt_render_settings s; check(pt_scene_get_render_settings(s_, &s)); return s; }
    void setSettings(const pt_render_settings& s) { check(pt_scene_set_render_settings(s_, &s)); }
    pt_scene_info info() const { pt_scene_info i; check(pt_scene_info_get(s_, &i)); return i; }
    pt_scene_params buildParams() const { pt_scene_params p; check(pt_scene_build_params(s_, &p)); return p; }
    pt_scene* handle() const { return s_; }

private:
    void reset() { if (s_) { pt_scene_destroy(s_); s_ = nullptr; } }
    pt_scene* s_ = nullptr;
};

class Film {
public:
    Film(int w, int h, int device = 0) { check(pt_film_create(w, h, device, &f_)); }
    ~Film() { pt_film_destroy(f_); }
    Film(const Film&) = delete;
    Film& operator=(const Film&) = delete;
    void clear() { check(pt_film_clear(f_)); }
    void downloadAccumulated(float* host_rgba) const { check(pt_film_download(f_, host_rgba)); }
    pt_film* handle() const { return f_; }

private:
    pt_film* f_ = nullptr;
};

class Integrator {
public:
    virtual ~Integrator() = default;
    virtual void launch(Film& film, SceneManager& scene, const pt_scene_params& params, void* stream = nullptr) = 0;
    virtual const char* name() const = 0;
};

class PathIntegrator : public Integrator {
public:
    PathIntegrator() { check(pt_integrator_create("path", &i_)); }
    ~PathIntegrator() override { pt_integrator_destroy(i_); }
    void launch(Film& film, SceneManager& scene, const pt_scene_params& params, void* stream = nullptr) override {
        check(pt_integrator_launch(i_, film.handle(), scene.handle(), &params, stream));
    }
    const char* name() const override { return pt_integrator_name(i_); }
    pt_render_stats stats() const { pt_render_stats s; check(pt_integrator_stats(i_, &s)); return s; }
    pt_integrator* handle() const { return i_; }

private:
    pt_integrator* i_ = nullptr;
};

class Renderer {
public:
    Renderer(SceneManager& scene, std::unique_ptr<Integrator> integrator, int device = 0)
        : scene_(scene), integrator_(std::move(integrator)) {
        const pt_camera c = scene_.camera();
        film_ = std::make_unique<Film>(c.width, c.height, device);
    }
    // Renderer::renderBatch (renderer.cu:20-45): one launch of samplePerFrame spp.
    uint32_t renderBatch(void* stream = nullptr) {
        const pt_scene_params p = scene_.buildParams();
        integrator_->launch(*film_, scene_, p, stream);
        check(pt_scene_set_frame_count(scene_.handle(), scene_.info().frame_count + 1));
        return currentSpp();
    }
    // Renderer::renderAll; with this library's path integrator the remaining
    // frames run as one launch (pt_renderer_render_frames, same result).
    void renderAll(void* stream = nullptr) {
        if (auto* pi = dynamic_cast<PathIntegrator*>(integrator_.get())) {
            const uint32_t spf = static_cast<uint32_t>(scene_.settings().sample_per_frame);
            const uint32_t cur = currentSpp(), tgt = targetSpp();
            if (cur < tgt)
                check(pt_renderer_render_frames(pi->handle(), film_->handle(), scene_.handle(),
                                                (tgt - cur + spf - 1) / spf, stream));
            return;
        }
        while (!isComplete()) renderBatch(stream);
    }
    uint32_t currentSpp() const { return scene_.info().frame_count * scene_.settings().sample_per_frame; }
    uint32_t targetSpp() const { return static_cast<uint32_t>(scene_.settings().spp); }
    bool isComplete() const { return currentSpp() >= targetSpp(); }
    void resetAccumulation() { check(pt_renderer_reset_accumulation(film_->handle(), scene_.handle())); }
    void downloadCurrentImage(std::vector<float>& buf) const {
        buf.resize(static_cast<size_t>(film_->handle() ? scene_.camera().width : 0) * scene_.camera().height * 4);
        film_->downloadAccumulated(buf.data());
    }
    Film& film() { return *film_; }
    Integrator& integrator() { return *integrator_; }

private:
    SceneManager& scene_;
    std::unique_ptr<Integrator> integrator_;
    std::unique_ptr<Film> film_;
};

// render(scene, spp) -> HDR image (width * height RGBA floats).
inline std::vector<float> render(SceneManager& scene, int spp, pt_render_stats* stats = nullptr) {
    const pt_camera c = scene.camera();
    std::vector<float> img(static_cast<size_t>(c.width) * c.height * 4);
    check(pt_render(scene.handle(), spp, img.data(), 0, stats));
    return img;
}

}  // namespace pt
