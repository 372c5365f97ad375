"""The C++ host API (include/pt_b200.hpp) compiles against the C ABI, links the
library, and runs: host-only calls on any machine, a render on a GPU."""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "pathtracingtutorial_b200")

PROGRAM = r"""
#include "pt_b200.hpp"
#include <cstdio>
#include <cstring>
int main(int argc, char** argv) {
    pt::SceneManager scene;
    std::vector<pt_vertex> v(4);
    const float p[4][3] = {{-1, 0, 1}, {1, 0, 1}, {1, 0, -1}, {-1, 0, -1}};
    for (int i = 0; i < 4; ++i) { std::memset(&v[i], 0, sizeof(pt_vertex)); for (int k = 0; k < 3; ++k) v[i].position[k] = p[i][k]; v[i].normal[1] = 1; }
    std::vector<pt_face> f = {{0, 1, 2, 0}, {0, 2, 3, 0}};
    pt_material m; std::memset(&m, 0, sizeof m);
    m.base_color[0] = m.base_color[1] = m.base_color[2] = 0.5f; m.roughness = 1; m.ior = 1.5f; m.specular_factor = 1;
    m.specular_color_r = m.specular_color_g = m.specular_color_b = 1; m.emissive_strength = 1; m.attenuation_distance = 1e30f;
    pt_camera c; std::memset(&c, 0, sizeof c);
    c.position[1] = 2; c.position[2] = 3; c.up[1] = 1; c.fov = 60; c.focal_distance = 1; c.width = 32; c.height = 24;
    std::vector<float> env(8 * 4 * 4, 1.0f);
    scene.create(v, f, {m}, c, env, 8, 4);
    scene.setSpp(8);
    scene.buildAccel();
    const pt_scene_info info = scene.info();
    std::printf("faces %u nodes %u\n", info.num_faces, info.num_bvh_nodes);
    try { scene.setSettings([&]{ auto s = scene.settings(); s.sample_per_frame = 0; return s; }()); return 3; }
    catch (const pt::Error& e) { std::printf("error ok %d\n", e.code()); }
    if (argc > 1 && std::strcmp(argv[1], "--render") == 0) {
        scene.uploadToDevice(0);
        pt::Renderer r(scene, std::make_unique<pt::PathIntegrator>());
        r.renderAll();
        std::vector<float> img;
        r.downloadCurrentImage(img);
        double s = 0; for (size_t i = 0; i < img.size(); i += 4) s += img[i];
        std::printf("spp %u mean %.4f name %s\n", r.currentSpp(), s / (img.size() / 4), r.integrator().name());
        if (!(s > 0)) return 4;
    }
    return 0;
}
"""


def _build(tmp_path):
    src = tmp_path / "api.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "api"
    subprocess.run(["g++", "-std=c++17", "-O1", str(src), "-I", os.path.join(ROOT, "include"), "-L", LIBDIR,
                    "-lpt_b200", f"-Wl,-rpath,{LIBDIR}", "-o", str(exe)], check=True)
    return str(exe)


def test_cpp_api_host_calls(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout
    assert "faces 2 nodes 1" in out and "error ok 1" in out


@pytest.mark.gpu
def test_cpp_api_render(tmp_path):
    exe = _build(tmp_path)
    out = subprocess.run([exe, "--render"], capture_output=True, text=True, check=True).stdout
    assert "spp 8" in out and "name Path" in out
