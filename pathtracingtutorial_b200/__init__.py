"""pathtracingtutorial_b200 -- B200-native path tracer behind the reference's plugin API.

Host-side mirror of Neroued/PathTracingTutorial Part_2's rendering interface
over the C ABI of libpt_b200.so (include/pt_b200.h):

  SceneManager   load / buildAccel / uploadToDevice / setSpp / setSampler
                 (Part_2/src/scene/scene_manager.h:11-45)
  PathIntegrator launch(film, scene, params) / name()   (Part_2/src/integrators/integrator.h:10-20,
                 path_integrator.h:7-15)
  Film           clear / download_accumulated            (Part_2/src/film/film.h:9-40)
  Renderer       render_batch / render_all / save_image / download_current_image /
                 run_convergence_benchmark / reset_accumulation (Part_2/src/renderer.h:17-55)
  render(scene, spp) -> HDR image (H, W, 4) float32

Every compute call runs on the GPU through the CUDA library; there is no CPU
fallback -- the library raises when it is missing.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import time
from dataclasses import dataclass

import numpy as np

from . import _ffi
from ._ffi import (ALIAS_DTYPE, BVH_NODE_DTYPE, CAMERA_DTYPE, EMISSIVE_DTYPE, FACE_DTYPE, HIT_DTYPE,
                   MATERIAL_DTYPE, PUNCTUAL_DTYPE, VERTEX_DTYPE, PTError, check, lib, ptr)
from ._ffi import SAMPLER_PCG, SAMPLER_SOBOL, FLAG_WATERTIGHT, FLAG_STAGE_TIMING, FLAG_NO_GRAPH, \
    FLAG_COUNT_TRAVERSAL, ARGS_LTR, ARGS_RTL

__all__ = ["SceneManager", "PathIntegrator", "Film", "Renderer", "render", "default_material", "make_camera",
           "trace_closest", "trace_any", "sampler_stream", "bsdf_eval", "write_hdr", "read_hdr", "tonemap", "decode_image",
           "compute_rmse", "rmse_to_db", "PTError", "VERTEX_DTYPE", "FACE_DTYPE", "MATERIAL_DTYPE",
           "CAMERA_DTYPE", "PUNCTUAL_DTYPE", "BVH_NODE_DTYPE", "SAMPLER_PCG", "SAMPLER_SOBOL",
           "FLAG_WATERTIGHT", "FLAG_STAGE_TIMING", "FLAG_NO_GRAPH", "FLAG_COUNT_TRAVERSAL",
           "ARGS_LTR", "ARGS_RTL"]

# Order in which nvcc's device code evaluates the two sampler draws that the
# reference takes inside one argument list; the kernels default to it so that
# they consume dimensions as the reference's GPU build does.
DEVICE_ARG_ORDER = ARGS_LTR


def default_material(**kw) -> np.ndarray:
    """One Material with the reference's defaults (Part_2/src/materials/material.h:8-75)."""
    m = np.zeros((), MATERIAL_DTYPE)
    m["base_color"] = (0.8, 0.8, 0.8)
    m["roughness"] = 0.5
    m["sheen_tint"] = 0.5
    m["clearcoat_roughness"] = 0.03
    m["ior"] = 1.5
    m["specular_factor"] = 1.0
    m["specular_color_r"] = m["specular_color_g"] = m["specular_color_b"] = 1.0
    m["normal_scale"] = 1.0
    m["emissive_strength"] = 1.0
    m["base_alpha"] = 1.0
    m["sheen_color_r"] = m["sheen_color_g"] = m["sheen_color_b"] = 1.0
    m["occlusion_strength"] = 1.0
    m["attenuation_distance"] = 1e30
    m["att_color_r"] = m["att_color_g"] = m["att_color_b"] = 1.0
    m["uv_scale_x"] = m["uv_scale_y"] = 1.0
    for k in ("base_color_tex", "metallic_roughness_tex", "normal_tex", "emissive_tex", "occlusion_tex",
              "clearcoat_tex", "clearcoat_roughness_tex", "clearcoat_normal_tex", "transmission_tex",
              "sheen_color_tex", "sheen_roughness_tex"):
        m[k] = -1
    for k, v in kw.items():
        m[k] = v
    return m


def make_camera(position=(0, 0, 4), look_at=(0, 0, 0), up=(0, 1, 0), fov=90.0, aperture=0.0,
                focal_distance=10.0, width=1600, height=1600) -> np.ndarray:
    """Camera with the reference's defaults (Part_2/src/camera/camera.h:12-21)."""
    c = np.zeros((), CAMERA_DTYPE)
    c["position"], c["look_at"], c["up"] = position, look_at, up
    c["fov"], c["aperture"], c["focal_distance"] = fov, aperture, focal_distance
    c["width"], c["height"] = width, height
    return c


class SceneManager:
    """Scene handle: load or create, buildAccel (host prep), uploadToDevice."""

    def __init__(self, handle: C.c_void_p):
        self._h = handle

    # -- construction --
    @classmethod
    def load(cls, path: str) -> "SceneManager":
        h = C.c_void_p()
        check(lib().pt_scene_load_json(os.fsencode(path), C.byref(h)))
        return cls(h)

    @classmethod
    def from_arrays(cls, vertices: np.ndarray, faces: np.ndarray, materials: np.ndarray,
                    camera: np.ndarray | None = None, env_rgba: np.ndarray | None = None) -> "SceneManager":
        v = np.ascontiguousarray(vertices, dtype=VERTEX_DTYPE)
        f = np.ascontiguousarray(faces, dtype=FACE_DTYPE)
        m = np.ascontiguousarray(np.atleast_1d(materials), dtype=MATERIAL_DTYPE)
        cam = None if camera is None else np.ascontiguousarray(camera, dtype=CAMERA_DTYPE)
        env = None
        ew = eh = 0
        if env_rgba is not None:
            env = np.ascontiguousarray(env_rgba, dtype=np.float32)
            if env.ndim != 3 or env.shape[2] != 4:
                raise ValueError("env_rgba must be (H, W, 4)")
            eh, ew = env.shape[:2]
        h = C.c_void_p()
        check(lib().pt_scene_create(ptr(v), len(v), ptr(f), len(f), ptr(m), len(m),
                                    ptr(cam) if cam is not None else None, ptr(env) if env is not None else None,
                                    ew, eh, C.byref(h)))
        return cls(h)

    def close(self) -> None:
        if self._h:
            lib().pt_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    # -- settings (SceneManager::setSpp / setSampler / setMaxDepth) --
    def settings(self) -> _ffi.RenderSettings:
        s = _ffi.RenderSettings()
        check(lib().pt_scene_get_render_settings(self._h, C.byref(s)))
        return s

    def update_settings(self, **kw) -> None:
        s = self.settings()
        for k, v in kw.items():
            setattr(s, k, int(v))
        check(lib().pt_scene_set_render_settings(self._h, C.byref(s)))

    def set_spp(self, spp: int) -> None:
        self.update_settings(spp=spp)

    def set_sampler(self, sampler: int | str) -> None:
        if isinstance(sampler, str):
            sampler = {"pcg": SAMPLER_PCG, "sobol": SAMPLER_SOBOL}[sampler]
        self.update_settings(sampler_type=sampler)

    def set_max_depth(self, depth: int) -> None:
        self.update_settings(max_depth=depth)

    @property
    def camera(self) -> np.ndarray:
        c = np.zeros((), CAMERA_DTYPE)
        check(lib().pt_scene_get_camera(self._h, ptr(c)))
        return c

    def set_frame_count(self, n: int) -> None:
        check(lib().pt_scene_set_frame_count(self._h, int(n)))

    def update_camera(self, cam: np.ndarray) -> None:
        c = np.ascontiguousarray(cam, dtype=CAMERA_DTYPE)
        check(lib().pt_scene_set_camera(self._h, ptr(c)))

    def add_texture(self, rgba: np.ndarray, wrap_s: int = 10497, wrap_t: int = 10497) -> int:
        """Append a material texture ((H, W, 4) float texels; GL wrap modes) and
        return its index for the materials' *_tex fields."""
        a = np.ascontiguousarray(rgba, np.float32)
        if a.ndim != 3 or a.shape[2] != 4:
            raise ValueError("texture must be (H, W, 4)")
        idx = C.c_int32()
        check(lib().pt_scene_add_texture(self._h, ptr(a) if a.size else None, a.shape[1], a.shape[0], int(wrap_s),
                                         int(wrap_t), C.byref(idx)))
        return idx.value

    def texture(self, index: int) -> dict:
        """Material texture `index`: {"rgba": (H, W, 4) float32, "wrap_s", "wrap_t"}."""
        w, h, ws, wt = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        check(lib().pt_scene_get_texture(self._h, int(index), None, 0, C.byref(w), C.byref(h), C.byref(ws),
                                         C.byref(wt)))
        out = np.zeros((h.value, w.value, 4), np.float32)
        if out.size:
            check(lib().pt_scene_get_texture(self._h, int(index), ptr(out), out.size, C.byref(w), C.byref(h), None,
                                             None))
        return {"rgba": out, "wrap_s": ws.value, "wrap_t": wt.value}

    def set_punctual_lights(self, lights: np.ndarray) -> None:
        L = np.ascontiguousarray(lights, dtype=PUNCTUAL_DTYPE)
        check(lib().pt_scene_set_punctual_lights(self._h, ptr(L), len(L)))

    # -- prep / upload --
    def build_accel(self, builder: str = "host", device: int = 0, max_leaf: int = 0,
                    treelet: int = 0, passes: int = 0, traversal_cost: float = 0.0) -> dict | None:
        """SceneManager::buildAccel.  builder="host" is the reference's SAH
        build (node for node); builder="device" builds a linear BVH on
        `device`, re-topologises its treelets of `treelet` leaves (0 = 7, 1 =
        off) in `passes` passes (0 = 3) and collapses leaves by the SAH (a node
        visit costs `traversal_cost` triangle tests, 0 = 1.0), and returns its
        timings and sizes."""
        if builder == "host":
            check(lib().pt_scene_build_accel(self._h))
            return None
        if builder != "device":
            raise ValueError(f"unknown builder {builder!r} (host or device)")
        st = _ffi.BuildStats()
        opt = _ffi.BuildOptions(max_leaf, treelet, passes, traversal_cost)
        check(lib().pt_scene_build_accel_device(self._h, device, C.byref(opt), C.byref(st)))
        return st.as_dict()

    def autotune(self, calib_spp: int = 0) -> dict:
        """pt_autotune: time calibration renders and keep the fastest traversal
        stack depth, traversal block size and queue capacity in this scene's
        settings (cached per device and scene class).  Returns the report."""
        r = _ffi.TuneReport()
        check(lib().pt_autotune(self._h, int(calib_spp), C.byref(r)))
        return r.as_dict()

    def upload_to_device(self, device: int = 0) -> None:
        check(lib().pt_scene_upload(self._h, device))

    def info(self) -> dict:
        i = _ffi.SceneInfo()
        check(lib().pt_scene_info_get(self._h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in i._fields_}

    def build_params(self) -> _ffi.SceneParams:
        p = _ffi.SceneParams()
        check(lib().pt_scene_build_params(self._h, C.byref(p)))
        return p

    # -- read back prep results --
    def vertices(self) -> np.ndarray:
        out = np.zeros(self.info()["num_vertices"], VERTEX_DTYPE)
        check(lib().pt_scene_get_vertices(self._h, ptr(out), len(out)))
        return out

    def faces(self) -> np.ndarray:
        out = np.zeros(self.info()["num_faces"], FACE_DTYPE)
        check(lib().pt_scene_get_faces(self._h, ptr(out), len(out)))
        return out

    def materials(self) -> np.ndarray:
        out = np.zeros(self.info()["num_materials"], MATERIAL_DTYPE)
        check(lib().pt_scene_get_materials(self._h, ptr(out), len(out)))
        return out

    def punctual_lights(self) -> np.ndarray:
        out = np.zeros(self.info()["num_punctual_lights"], PUNCTUAL_DTYPE)
        check(lib().pt_scene_get_punctual_lights(self._h, ptr(out), len(out)))
        return out

    def bvh_nodes(self) -> np.ndarray:
        out = np.zeros(self.info()["num_bvh_nodes"], BVH_NODE_DTYPE)
        check(lib().pt_scene_get_bvh(self._h, ptr(out), len(out)))
        return out

    def traversal_layout(self) -> tuple[np.ndarray, np.ndarray, int]:
        """(inner nodes as uint32[n, 16], triangle records as uint32[m, 12],
        root_ref): the device node layout, bit for bit."""
        info = self.info()
        inner = np.zeros((info["num_inner_nodes"], 16), np.uint32)
        tris = np.zeros((info["num_faces"], 12), np.uint32)
        root = C.c_uint32(0)
        check(lib().pt_scene_get_traversal(self._h, ptr(inner), len(inner), ptr(tris), len(tris), C.byref(root)))
        return inner, tris, int(root.value)

    def emissive_tables(self) -> tuple[np.ndarray, np.ndarray, np.ndarray]:
        info = self.info()
        refs = np.zeros(info["num_emissive_triangles"], EMISSIVE_DTYPE)
        pmf = np.zeros(info["num_faces"] if info["num_bvh_nodes"] else 0, np.float32)
        alias = np.zeros(info["num_emissive_triangles"], ALIAS_DTYPE)
        check(lib().pt_scene_get_emissive(self._h, ptr(refs), len(refs), ptr(pmf), len(pmf), ptr(alias), len(alias)))
        return refs, pmf, alias

    def env_tables(self) -> tuple[np.ndarray, np.ndarray]:
        info = self.info()
        n = info["env_width"] * info["env_height"]
        pmf = np.zeros(n, np.float32)
        alias = np.zeros(n, ALIAS_DTYPE)
        rc = lib().pt_scene_get_env_tables(self._h, ptr(pmf), ptr(alias), n)
        check(rc)
        return pmf, alias


class Film:
    """Device film: compensated accumulation + the last launch's mean."""

    def __init__(self, width: int, height: int, device: int = 0):
        self.width, self.height, self.device = width, height, device
        h = C.c_void_p()
        check(lib().pt_film_create(width, height, device, C.byref(h)))
        self._h = h

    def clear(self) -> None:
        check(lib().pt_film_clear(self._h))

    def download_accumulated(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float32)
        check(lib().pt_film_download(self._h, ptr(out)))
        return out

    def download_new(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float32)
        check(lib().pt_film_download_new(self._h, ptr(out)))
        return out

    def close(self) -> None:
        if self._h:
            lib().pt_film_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PathIntegrator:
    """The "Path" integrator plugin (Integrator::launch / name)."""

    def __init__(self):
        h = C.c_void_p()
        check(lib().pt_integrator_create(b"path", C.byref(h)))
        self._h = h

    def name(self) -> str:
        return lib().pt_integrator_name(self._h).decode()

    def launch(self, film: Film, scene: SceneManager, params: _ffi.SceneParams, stream: int | None = None) -> None:
        check(lib().pt_integrator_launch(self._h, film._h, scene.handle, C.byref(params),
                                         C.c_void_p(stream) if stream else None))

    def stats(self) -> dict:
        s = _ffi.RenderStats()
        check(lib().pt_integrator_stats(self._h, C.byref(s)))
        return s.as_dict()

    def reset_stats(self) -> None:
        check(lib().pt_integrator_reset_stats(self._h))

    def close(self) -> None:
        if self._h:
            lib().pt_integrator_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Renderer:
    """Batch loop over the integrator (Renderer, Part_2/src/renderer.h:17-55)."""

    def __init__(self, scene: SceneManager, integrator: PathIntegrator | None = None, device: int = 0,
                 stream: int | None = None):
        self.scene = scene
        self.integrator = integrator or PathIntegrator()
        cam = scene.camera
        self.film = Film(int(cam["width"]), int(cam["height"]), device)
        self.stream = stream
        self.last_batch_ms = 0.0

    def render_batch(self) -> int:
        t0 = time.perf_counter()
        check(lib().pt_renderer_render_batch(self.integrator._h, self.film._h, self.scene.handle,
                                             C.c_void_p(self.stream) if self.stream else None))
        self.last_batch_ms = (time.perf_counter() - t0) * 1e3
        return self.current_spp()

    def render_frames(self, frames: int) -> int:
        """`frames` renderBatch calls in one launch (same result as calling
        render_batch that many times)."""
        t0 = time.perf_counter()
        check(lib().pt_renderer_render_frames(self.integrator._h, self.film._h, self.scene.handle, int(frames),
                                              C.c_void_p(self.stream) if self.stream else None))
        self.last_batch_ms = (time.perf_counter() - t0) * 1e3
        return self.current_spp()

    def current_spp(self) -> int:
        return self.scene.info()["frame_count"] * self.scene.settings().sample_per_frame

    def target_spp(self) -> int:
        return self.scene.settings().spp

    def is_complete(self) -> bool:
        return self.current_spp() >= self.target_spp()

    def render_all(self) -> None:
        spf = self.scene.settings().sample_per_frame
        left = -(-(self.target_spp() - self.current_spp()) // spf)
        if left > 0:
            self.render_frames(left)
        self.synchronize()

    def synchronize(self) -> None:
        import torch  # noqa: plumbing only
        if torch.cuda.is_available():
            torch.cuda.synchronize(self.film.device)

    def reset_accumulation(self) -> None:
        check(lib().pt_renderer_reset_accumulation(self.film._h, self.scene.handle))

    def download_current_image(self) -> np.ndarray:
        return self.film.download_accumulated()

    def save_image(self, path: str) -> None:
        write_hdr(path, self.download_current_image())

    def run_convergence_benchmark(self, ref: np.ndarray, checkpoints: list[int]) -> list[dict]:
        """RMSE / PSNR at spp checkpoints (Renderer::runConvergenceBenchmark, renderer.cu:138-173)."""
        self.reset_accumulation()
        out = []
        nxt = 0
        t0 = time.perf_counter()
        while nxt < len(checkpoints):
            spp = self.render_batch()
            if spp >= checkpoints[nxt]:
                img = self.download_current_image()
                ms = (time.perf_counter() - t0) * 1e3
                rmse = compute_rmse(img, ref)
                out.append({"spp": spp, "rmse": rmse, "psnr": rmse_to_db(rmse), "time_ms": ms})
                nxt += 1
        return out


def render(scene: SceneManager, spp: int, stats: bool = False):
    """render(scene, spp) -> HDR image (H, W, 4) float32 (and the render stats)."""
    cam = scene.camera
    out = np.zeros((int(cam["height"]), int(cam["width"]), 4), np.float32)
    st = _ffi.RenderStats()
    check(lib().pt_render(scene.handle, int(spp), ptr(out), 0, C.byref(st)))
    return (out, st.as_dict()) if stats else out


class Guide:
    """Learned directional guide (hash grid + MLP + 8-lobe vMF mixture) for one scene."""

    OFF, USE, TRAIN = _ffi.GUIDE_OFF, _ffi.GUIDE_USE, _ffi.GUIDE_TRAIN
    # how the network is evaluated (pt_guide_set_inference)
    INFER_DEFAULT, INFER_FUSED, INFER_SPLIT_MMA, INFER_SPLIT_TC = (
        _ffi.GUIDE_INFER_DEFAULT, _ffi.GUIDE_INFER_FUSED, _ffi.GUIDE_INFER_SPLIT_MMA, _ffi.GUIDE_INFER_SPLIT_TC)
    STEP_SAMPLES = 65536   # the library's default cap of training samples per optimiser step

    def __init__(self, scene: SceneManager, seed: int = 1, lr: float | None = None, alpha: float | None = None,
                 paths_per_step: int | None = None, samples_per_step: int | None = None,
                 inference: int | None = None):
        h = C.c_void_p()
        check(lib().pt_guide_create(scene.handle, seed, C.byref(h)))
        self._h = h
        if inference is not None:
            self.set_inference(inference)
        if lr is not None:
            check(lib().pt_guide_set_learning_rate(self._h, float(lr)))
        if alpha is not None:
            self.set_alpha(alpha)
        if paths_per_step is not None or samples_per_step is not None:
            self.set_training(paths_per_step or 0,
                              self.STEP_SAMPLES if samples_per_step is None else samples_per_step)

    def set_alpha(self, alpha: float) -> None:
        """Probability of drawing a continuation from the network (one-sample MIS)."""
        check(lib().pt_guide_set_alpha(self._h, float(alpha)))

    def set_schedule(self, ema: float = 0.0, lr_half_life: float = 0.0, lr_floor: float = 0.1) -> None:
        """Parameter averaging for the renders (ema: factor per optimiser step,
        0 = off) and learning-rate halving every lr_half_life steps down to
        lr_floor of the set rate (0 = constant)."""
        check(lib().pt_guide_set_schedule(self._h, float(ema), float(lr_half_life), float(lr_floor)))

    def set_inference(self, kind: int) -> None:
        """Network evaluation kernels: INFER_FUSED (encoding and MLP in one
        mma.sync kernel), INFER_SPLIT_MMA / INFER_SPLIT_TC (encoding kernel,
        then the MLP on mma.sync / on the tcgen05 tensor cores)."""
        check(lib().pt_guide_set_inference(self._h, int(kind)))

    def set_training(self, paths_per_step: int = 0, samples_per_step: int = 65536) -> None:
        """Online training: one optimiser step per `paths_per_step` paths of a
        pass (0 = 32768), each on at most `samples_per_step` samples (0 = the
        most a step takes, 131072; 65536 is the library's default)."""
        check(lib().pt_guide_set_training(self._h, int(paths_per_step), int(samples_per_step)))

    def attach(self, integrator: PathIntegrator, mode: int) -> None:
        check(lib().pt_integrator_set_guide(integrator._h, self._h if mode else None, mode))

    def info(self) -> dict:
        steps, samples = C.c_uint32(), C.c_uint32()
        check(lib().pt_guide_info(self._h, C.byref(steps), C.byref(samples)))
        return {"steps": steps.value, "last_samples": samples.value}

    def loss(self) -> float:
        """Mean training loss -w log q(dir | pos) of the last training pass."""
        v = C.c_float()
        check(lib().pt_guide_loss(self._h, C.byref(v)))
        return v.value

    def pdf(self, pos: np.ndarray, dirs: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(np.concatenate([np.asarray(pos, np.float32).reshape(-1, 3),
                                                 np.asarray(dirs, np.float32).reshape(-1, 3)], 1))
        out = np.zeros(len(q), np.float32)
        check(lib().pt_guide_eval(self._h, ptr(q), len(q), ptr(out)))
        return out

    N_WEIGHTS = 13312
    GRID_SHAPE = (16, 1 << 19, 2)

    def params(self, with_grid: bool = True) -> dict:
        """The network as the kernels use it: BF16 weights and FP16 grid values
        widened to float32, plus the position normalisation and level scales."""
        w = np.zeros(self.N_WEIGHTS, np.float32)
        grid = np.zeros(self.GRID_SHAPE, np.float32) if with_grid else None
        meta = np.zeros(6 + 16 + 1, np.float32)
        check(lib().pt_guide_get_params(self._h, ptr(w), ptr(grid) if with_grid else None, ptr(meta)))
        return {"weights": w, "grid": grid, "lo": meta[0:3].copy(), "inv_extent": meta[3:6].copy(),
                "scale": meta[6:22].copy(), "dense_limit": int(meta[22])}

    def backward(self, pos01: np.ndarray, weight: np.ndarray, dirs: np.ndarray, with_grid: bool = True):
        """Gradient of mean(-weight * log q(dir | pos)) over the given samples
        (positions already normalised to [0,1]^3), computed by the training
        kernel without an optimiser step.  Returns (weight_grad, grid_grad)."""
        n = len(weight)
        s = np.zeros((n, 8), np.float32)
        s[:, 0:3] = np.asarray(pos01, np.float32).reshape(-1, 3)
        s[:, 3] = np.asarray(weight, np.float32)
        s[:, 4:7] = np.asarray(dirs, np.float32).reshape(-1, 3)
        gw = np.zeros(self.N_WEIGHTS, np.float32)
        gg = np.zeros(self.GRID_SHAPE, np.float32) if with_grid else None
        check(lib().pt_guide_backward(self._h, ptr(s), n, ptr(gw), ptr(gg) if with_grid else None))
        return gw, gg

    def close(self) -> None:
        if self._h:
            lib().pt_guide_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def render_guided(scene: SceneManager, train_spp: int, spp: int, guide: Guide | None = None, seed: int = 1,
                  device: int = 0, stream: int | None = None, first_frame: int = 0):
    """Train a guide online for train_spp samples per pixel (those samples are
    discarded), then render spp samples per pixel sampling with it.
    Returns (image, guide, render stats)."""
    g = guide or Guide(scene, seed)
    r = Renderer(scene, device=device, stream=stream)
    spf = scene.settings().sample_per_frame
    g.attach(r.integrator, Guide.TRAIN)
    r.reset_accumulation()
    scene.set_frame_count(first_frame + 100000)   # training samples are independent of the image's
    if train_spp > 0:
        r.render_frames((train_spp + spf - 1) // spf)
    g.attach(r.integrator, Guide.USE)
    r.reset_accumulation()
    scene.set_frame_count(first_frame)
    r.integrator.reset_stats()
    r.render_frames((spp + spf - 1) // spf)
    r.synchronize()
    img = r.download_current_image()
    return img, g, r.integrator.stats()


BATCH_AUTO, BATCH_PERSISTENT, BATCH_WAVEFRONT = _ffi.BATCH_AUTO, _ffi.BATCH_PERSISTENT, _ffi.BATCH_WAVEFRONT


def render_batch(items, block_size: int = 0, blocks_per_sm: int = 0, chunk_spp: int = 0, autotune: bool = True,
                 mode: int = BATCH_AUTO, paths_in_flight: int = 0):
    """Render [(scene, spp[, first_frame[, camera[, guide]]])...] in one graph
    launch: one persistent kernel over all items, or every item's wavefront as
    a parallel graph branch (mode; AUTO lets the autotuner time both).  An
    item's camera (a make_camera array; None: the scene's) sets its view and
    resolution, so many cameras of one scene share its device data; an item
    with a trained Guide samples with it (wavefront mode).
    Returns (list of (H, W, 4) images, stats dict, config dict)."""
    n = len(items)
    arr = (_ffi.BatchItem * n)()
    outs = []
    keep = []
    for k, it in enumerate(items):
        scene, spp = it[0], it[1]
        first = it[2] if len(it) > 2 else 0
        icam = it[3] if len(it) > 3 else None
        guide = it[4] if len(it) > 4 else None
        cam = scene.camera if icam is None else icam
        img = np.zeros((int(cam["height"]), int(cam["width"]), 4), np.float32)
        outs.append(img)
        arr[k].scene = scene.handle
        arr[k].spp = int(spp)
        arr[k].max_depth = -1
        arr[k].first_frame = int(first)
        arr[k].out_rgba = img.ctypes.data
        if icam is not None:
            c = np.ascontiguousarray(icam, CAMERA_DTYPE)
            keep.append(c)
            arr[k].camera = c.ctypes.data
        if guide is not None:
            arr[k].guide = guide._h
    cfg = _ffi.BatchConfig(block_size, blocks_per_sm, chunk_spp, 1 if autotune else 0, 0.0, int(mode),
                           int(paths_in_flight), 0)
    st = _ffi.RenderStats()
    check(lib().pt_render_batch(arr, n, 0, C.byref(cfg), C.byref(st)))
    return outs, st.as_dict(), {"block_size": cfg.block_size, "blocks_per_sm": cfg.blocks_per_sm,
                                "chunk_spp": cfg.chunk_spp, "tuned_ms": cfg.tuned_ms, "mode": cfg.mode,
                                "paths_in_flight": cfg.paths_in_flight}


# ---- diagnostics over the same kernels ----
def trace_closest(scene: SceneManager, origins: np.ndarray, dirs: np.ndarray) -> np.ndarray:
    rays = _pack_rays(origins, dirs, None)
    hits = np.zeros(len(rays), HIT_DTYPE)
    check(lib().pt_trace_closest(scene.handle, ptr(rays), len(rays), ptr(hits), 0))
    return hits


STATIC_TRACE_MAX_RAYS = 65536


def trace_closest_static(scene: SceneManager, origins: np.ndarray, dirs: np.ndarray) -> np.ndarray:
    """trace_closest through the allocation-free entry point (at most
    STATIC_TRACE_MAX_RAYS rays per call)."""
    rays = _pack_rays(origins, dirs, None)
    hits = np.zeros(len(rays), HIT_DTYPE)
    check(lib().pt_trace_closest_static(scene.handle, ptr(rays), len(rays), ptr(hits)))
    return hits


def trace_any(scene: SceneManager, origins: np.ndarray, dirs: np.ndarray, tmax: np.ndarray) -> np.ndarray:
    rays = _pack_rays(origins, dirs, tmax)
    occ = np.zeros(len(rays), np.uint8)
    check(lib().pt_trace_any(scene.handle, ptr(rays), len(rays), ptr(occ), 0))
    return occ.astype(bool)


def _pack_rays(o: np.ndarray, d: np.ndarray, tmax: np.ndarray | None) -> np.ndarray:
    o = np.asarray(o, np.float32).reshape(-1, 3)
    d = np.asarray(d, np.float32).reshape(-1, 3)
    r = np.zeros((len(o), 8), np.float32)
    r[:, 0:3] = o
    r[:, 4:7] = d
    r[:, 7] = np.float32(np.finfo(np.float32).max) if tmax is None else np.asarray(tmax, np.float32)
    return np.ascontiguousarray(r)


def sampler_stream(sampler: int, width: int, height: int, frame: int, spf: int, sample_in_frame: int,
                   ndims: int, pcg_seed: int = 0, device: int = 0) -> np.ndarray:
    out = np.zeros((height, width, ndims), np.float32)
    check(lib().pt_sampler_stream(sampler, width, height, frame, spf, sample_in_frame, ndims, pcg_seed, device,
                                  ptr(out)))
    return out


def bsdf_eval(scene: SceneManager, records: np.ndarray) -> np.ndarray:
    """records: (n, 13) = material index, wo, wi, N, T.  Returns (n, 4) = f*|N.L| rgb, pdf."""
    rec = np.ascontiguousarray(records, np.float32)
    out = np.zeros((len(rec), 4), np.float32)
    check(lib().pt_bsdf_eval(scene.handle, ptr(rec), len(rec), ptr(out)))
    return out


def tonemap(img: np.ndarray, exposure: float = -2.8, device: int = 0) -> np.ndarray:
    """Display image of the reference's preview tone mapping
    (Part_2/preview/tone_mapping.frag:12-29) computed on the GPU:
    (H, W, 4) float radiance -> (H, W, 4) uint8 sRGB, alpha 255."""
    a = np.ascontiguousarray(img, np.float32)
    h, w = a.shape[0], a.shape[1]
    if a.shape[2] == 3:
        a = np.ascontiguousarray(np.concatenate([a, np.ones((h, w, 1), np.float32)], 2))
    out = np.zeros((h, w, 4), np.uint8)
    check(lib().pt_tonemap(ptr(a), w, h, float(exposure), ptr(out), 0, device))
    return out


def decode_image(data: bytes) -> np.ndarray:
    """PNG or baseline JPEG bytes -> (H, W, 4) uint8 RGBA (the library's decoder)."""
    buf = np.frombuffer(bytes(data), np.uint8)
    w, h = C.c_int32(), C.c_int32()
    check(lib().pt_decode_image(ptr(buf), len(buf), None, 0, C.byref(w), C.byref(h)))
    out = np.zeros((h.value, w.value, 4), np.uint8)
    check(lib().pt_decode_image(ptr(buf), len(buf), ptr(out), out.size, C.byref(w), C.byref(h)))
    return out


# ---- quality metrics (Part_2/src/film/quality_metrics.h:20-39) ----
def compute_rmse(img: np.ndarray, ref: np.ndarray, channels: int = 3) -> float:
    d = img[..., :channels].astype(np.float64) - ref[..., :channels].astype(np.float64)
    return float(np.sqrt(np.mean(d * d))) if d.size else 0.0


def rmse_to_db(rmse: float) -> float:
    return 100.0 if rmse <= 0.0 else -20.0 * math.log10(rmse)


# ---- Radiance RGBE files ----
def write_hdr(path: str, img: np.ndarray, flip_y: bool = True) -> None:
    """ImageIO::write for .hdr: (H, W, 3|4) float radiance as run-length coded
    RGBE, rows flipped by default, byte for byte as the reference writes it."""
    a = np.asarray(img, np.float32)
    h, w = a.shape[:2]
    rgba = np.ones((h, w, 4), np.float32)
    rgba[..., :3] = a[..., :3]
    check(lib().pt_write_hdr(os.fsencode(path), ptr(rgba), w, h, 1 if flip_y else 0))


def read_hdr(path: str) -> np.ndarray:
    """A Radiance .hdr (flat or run-length coded) -> (H, W, 4) float32, alpha 1."""
    w, h = C.c_int32(), C.c_int32()
    check(lib().pt_read_hdr(os.fsencode(path), None, 0, C.byref(w), C.byref(h)))
    out = np.zeros((h.value, w.value, 4), np.float32)
    check(lib().pt_read_hdr(os.fsencode(path), ptr(out), out.size, C.byref(w), C.byref(h)))
    return out
