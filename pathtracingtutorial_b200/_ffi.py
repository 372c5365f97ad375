"""ctypes binding of libpt_b200.so (declarations in include/pt_b200.h).

The numpy dtypes below are byte-compatible with the reference's host structs
(Vertex 64 B, TriangleFace 16 B, Material 256 B, Camera 80 B, ...), so arrays
laid out for the reference can be handed to the library unchanged.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpt_b200.so")

PT_OK, PT_ERR_INVALID, PT_ERR_IO, PT_ERR_CUDA, PT_ERR_STATE, PT_ERR_DEVICE, PT_ERR_NOMEM = range(7)
SAMPLER_PCG, SAMPLER_SOBOL = 0, 1
FLAG_WATERTIGHT, FLAG_STAGE_TIMING, FLAG_NO_GRAPH, FLAG_COUNT_TRAVERSAL = 1, 2, 4, 8
ARGS_LTR, ARGS_RTL = 0, 1
GUIDE_OFF, GUIDE_USE, GUIDE_TRAIN = 0, 1, 2
GUIDE_INFER_DEFAULT, GUIDE_INFER_FUSED, GUIDE_INFER_SPLIT_MMA, GUIDE_INFER_SPLIT_TC = 0, 1, 2, 3

VERTEX_DTYPE = np.dtype([("position", "<f4", 3), ("_pad0", "<f4"), ("normal", "<f4", 3), ("_pad1", "<f4"),
                         ("uv", "<f4", 2), ("_pad2", "<f4", 2), ("tangent", "<f4", 4)])
FACE_DTYPE = np.dtype([("v0", "<u4"), ("v1", "<u4"), ("v2", "<u4"), ("material_id", "<i4")])
MATERIAL_DTYPE = np.dtype({
    "names": ["base_color", "metallic", "roughness", "specular_tint", "anisotropic", "sheen", "sheen_tint",
              "clearcoat", "clearcoat_roughness", "spec_trans", "ior", "subsurface", "specular_factor",
              "specular_color_r", "specular_color_g", "specular_color_b", "anisotropy_rotation", "normal_scale",
              "emissive", "emissive_strength", "alpha_cutoff", "alpha_mode", "base_alpha", "double_sided",
              "sheen_color_r", "sheen_color_g", "sheen_color_b", "occlusion_strength", "thickness_factor",
              "attenuation_distance", "att_color_r", "att_color_g", "att_color_b", "uv_offset_x", "uv_offset_y",
              "uv_scale_x", "uv_scale_y", "uv_rotation", "base_color_tex", "metallic_roughness_tex", "normal_tex",
              "emissive_tex", "occlusion_tex", "clearcoat_tex", "clearcoat_roughness_tex", "clearcoat_normal_tex",
              "transmission_tex", "sheen_color_tex", "sheen_roughness_tex"],
    "formats": [("<f4", 3)] + ["<f4"] * 17 + [("<f4", 3), "<f4", "<f4", "<i4", "<f4", "<i4"] + ["<f4"] * 14 + ["<i4"] * 11,
    "offsets": [0, 16, 20, 24, 28, 32, 36, 40, 44, 48, 52, 56, 60, 64, 68, 72, 76, 80,
                96, 112, 116, 120, 124, 128, 132, 136, 140, 144, 148, 152, 156, 160, 164, 168, 172,
                176, 180, 184, 196, 200, 204, 208, 212, 216, 220, 224, 228, 232, 236],
    "itemsize": 256,
})
CAMERA_DTYPE = np.dtype({"names": ["position", "look_at", "up", "fov", "aperture", "focal_distance", "width", "height"],
                         "formats": [("<f4", 3), ("<f4", 3), ("<f4", 3), "<f4", "<f4", "<f4", "<i4", "<i4"],
                         "offsets": [0, 16, 32, 48, 52, 56, 60, 64], "itemsize": 80})
PUNCTUAL_DTYPE = np.dtype({"names": ["position", "range", "color", "intensity", "direction", "inner_cone",
                                     "outer_cone", "type"],
                           "formats": [("<f4", 3), "<f4", ("<f4", 3), "<f4", ("<f4", 3), "<f4", "<f4", "<i4"],
                           "offsets": [0, 16, 32, 48, 64, 80, 84, 88], "itemsize": 112})
BVH_NODE_DTYPE = np.dtype([("bmin", "<f4", 3), ("data0", "<u4"), ("bmax", "<f4", 3), ("data1", "<u4")])
ALIAS_DTYPE = np.dtype([("prob", "<f4"), ("alias", "<u4")])
EMISSIVE_DTYPE = np.dtype([("triangle_index", "<u4"), ("selection_pmf", "<f4"), ("cdf", "<f4"), ("_pad", "<f4")])
HIT_DTYPE = np.dtype([("t", "<f4"), ("prim", "<i4"), ("u", "<f4"), ("v", "<f4")])

assert VERTEX_DTYPE.itemsize == 64 and FACE_DTYPE.itemsize == 16 and MATERIAL_DTYPE.itemsize == 256
assert CAMERA_DTYPE.itemsize == 80 and PUNCTUAL_DTYPE.itemsize == 112 and BVH_NODE_DTYPE.itemsize == 32


class CameraFrame(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3), ("right", C.c_float * 3),
                ("up", C.c_float * 3), ("tan_half_fov", C.c_float), ("aspect", C.c_float),
                ("aperture", C.c_float), ("focal_distance", C.c_float)]


class SceneParams(C.Structure):
    _fields_ = [("camera", CameraFrame), ("width", C.c_int32), ("height", C.c_int32),
                ("sample_per_frame", C.c_int32), ("target_samples", C.c_int32), ("max_depth", C.c_int32),
                ("sampler_type", C.c_int32)]


class RenderSettings(C.Structure):
    _fields_ = [("spp", C.c_int32), ("sample_per_frame", C.c_int32), ("max_depth", C.c_int32),
                ("sampler_type", C.c_int32), ("pcg_seed", C.c_uint32), ("arg_order", C.c_int32),
                ("flags", C.c_int32), ("paths_in_flight", C.c_int32), ("trace_block", C.c_int32),
                ("stack_depth", C.c_int32)]


class BuildOptions(C.Structure):
    _fields_ = [("max_leaf", C.c_uint32), ("treelet_leaves", C.c_uint32), ("passes", C.c_uint32),
                ("traversal_cost", C.c_float)]


class BuildStats(C.Structure):
    _fields_ = [("total_ms", C.c_double), ("upload_ms", C.c_double), ("device_ms", C.c_double),
                ("download_ms", C.c_double), ("tables_ms", C.c_double), ("setup_ms", C.c_double),
                ("inner_nodes", C.c_uint32),
                ("leaves", C.c_uint32), ("depth", C.c_uint32), ("max_leaf", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


assert C.sizeof(BuildStats) == 64


class SceneInfo(C.Structure):
    _fields_ = [("num_vertices", C.c_uint32), ("num_faces", C.c_uint32), ("num_materials", C.c_uint32),
                ("num_bvh_nodes", C.c_uint32), ("num_emissive_triangles", C.c_uint32),
                ("num_punctual_lights", C.c_uint32), ("env_width", C.c_int32), ("env_height", C.c_int32),
                ("bvh_max_depth", C.c_uint32), ("num_inner_nodes", C.c_uint32), ("num_leaves", C.c_uint32),
                ("frame_count", C.c_uint32), ("device_bytes", C.c_uint64), ("num_textures", C.c_uint32),
                ("_pad", C.c_uint32)]


class TuneReport(C.Structure):
    _fields_ = [("paths_in_flight", C.c_int32), ("trace_block", C.c_int32), ("stack_depth", C.c_int32),
                ("cached", C.c_int32), ("calib_spp", C.c_int32), ("candidates", C.c_int32),
                ("best_ms", C.c_float), ("default_ms", C.c_float),
                ("cand_paths", C.c_int32 * 16), ("cand_block", C.c_int32 * 16), ("cand_depth", C.c_int32 * 16),
                ("cand_ms", C.c_float * 16)]

    def as_dict(self) -> dict:
        n = self.candidates
        return {"paths_in_flight": self.paths_in_flight, "trace_block": self.trace_block,
                "stack_depth": self.stack_depth, "cached": bool(self.cached), "calib_spp": self.calib_spp,
                "best_ms": self.best_ms, "default_ms": self.default_ms,
                "candidates": [{"paths_in_flight": self.cand_paths[k], "trace_block": self.cand_block[k],
                                "stack_depth": self.cand_depth[k], "ms": self.cand_ms[k]}
                               for k in range(n)]}


class RenderStats(C.Structure):
    _fields_ = [("camera_rays", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("node_visits", C.c_uint64), ("triangle_tests", C.c_uint64),
                ("shadow_node_visits", C.c_uint64), ("shadow_triangle_tests", C.c_uint64),
                ("paths", C.c_uint64), ("extend_launches", C.c_uint64),
                ("extend_ms", C.c_double), ("shade_ms", C.c_double), ("shadow_ms", C.c_double),
                ("other_ms", C.c_double), ("total_ms", C.c_double), ("kernel_launches", C.c_uint64),
                ("guide_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("spp", C.c_int32), ("max_depth", C.c_int32), ("first_frame", C.c_uint32),
                ("_pad", C.c_int32), ("out_rgba", C.c_void_p), ("camera", C.c_void_p), ("guide", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("block_size", C.c_int32), ("blocks_per_sm", C.c_int32), ("chunk_spp", C.c_int32),
                ("autotune", C.c_int32), ("tuned_ms", C.c_float), ("mode", C.c_int32),
                ("paths_in_flight", C.c_int32), ("_pad", C.c_int32)]


BATCH_AUTO, BATCH_PERSISTENT, BATCH_WAVEFRONT = 0, 1, 2


assert C.sizeof(SceneParams) == 88 and C.sizeof(CameraFrame) == 64 and C.sizeof(BatchItem) == 48

# (name, restype, argtypes) for every entry point declared in include/pt_b200.h
_P = C.c_void_p
_SIGS = [
    ("pt_last_error", C.c_char_p, []),
    ("pt_version", C.c_char_p, []),
    ("pt_build_camera_frame", C.c_int, [_P, C.POINTER(CameraFrame)]),
    ("pt_scene_load_json", C.c_int, [C.c_char_p, C.POINTER(_P)]),
    ("pt_scene_create", C.c_int, [_P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32, _P, _P, C.c_int32, C.c_int32,
                                  C.POINTER(_P)]),
    ("pt_scene_destroy", C.c_int, [_P]),
    ("pt_scene_set_punctual_lights", C.c_int, [_P, _P, C.c_uint32]),
    ("pt_scene_add_texture", C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.POINTER(C.c_int32)]),
    ("pt_scene_get_texture", C.c_int, [_P, C.c_int32, _P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                       C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("pt_decode_image", C.c_int, [_P, C.c_uint64, _P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("pt_scene_set_render_settings", C.c_int, [_P, C.POINTER(RenderSettings)]),
    ("pt_scene_get_render_settings", C.c_int, [_P, C.POINTER(RenderSettings)]),
    ("pt_scene_set_camera", C.c_int, [_P, _P]),
    ("pt_scene_get_camera", C.c_int, [_P, _P]),
    ("pt_scene_build_accel", C.c_int, [_P]),
    ("pt_scene_build_accel_device", C.c_int, [_P, C.c_int32, C.POINTER(BuildOptions), C.POINTER(BuildStats)]),
    ("pt_scene_get_traversal", C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, C.POINTER(C.c_uint32)]),
    ("pt_scene_upload", C.c_int, [_P, C.c_int32]),
    ("pt_scene_info_get", C.c_int, [_P, C.POINTER(SceneInfo)]),
    ("pt_scene_build_params", C.c_int, [_P, C.POINTER(SceneParams)]),
    ("pt_scene_get_vertices", C.c_int, [_P, _P, C.c_uint32]),
    ("pt_scene_get_faces", C.c_int, [_P, _P, C.c_uint32]),
    ("pt_scene_get_materials", C.c_int, [_P, _P, C.c_uint32]),
    ("pt_scene_get_punctual_lights", C.c_int, [_P, _P, C.c_uint32]),
    ("pt_scene_get_bvh", C.c_int, [_P, _P, C.c_uint32]),
    ("pt_scene_get_emissive", C.c_int, [_P, _P, C.c_uint32, _P, C.c_uint32, _P, C.c_uint32]),
    ("pt_scene_get_env_tables", C.c_int, [_P, _P, _P, C.c_uint32]),
    ("pt_film_create", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.POINTER(_P)]),
    ("pt_film_destroy", C.c_int, [_P]),
    ("pt_film_clear", C.c_int, [_P]),
    ("pt_film_download", C.c_int, [_P, _P]),
    ("pt_film_download_to", C.c_int, [_P, _P, C.c_int32]),
    ("pt_write_hdr", C.c_int, [C.c_char_p, _P, C.c_int32, C.c_int32, C.c_int32]),
    ("pt_read_hdr", C.c_int, [C.c_char_p, _P, C.c_uint64, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    ("pt_film_download_new", C.c_int, [_P, _P]),
    ("pt_integrator_create", C.c_int, [C.c_char_p, C.POINTER(_P)]),
    ("pt_integrator_destroy", C.c_int, [_P]),
    ("pt_integrator_name", C.c_char_p, [_P]),
    ("pt_integrator_launch", C.c_int, [_P, _P, _P, C.POINTER(SceneParams), _P]),
    ("pt_integrator_stats", C.c_int, [_P, C.POINTER(RenderStats)]),
    ("pt_integrator_reset_stats", C.c_int, [_P]),
    ("pt_renderer_render_batch", C.c_int, [_P, _P, _P, _P]),
    ("pt_renderer_render_frames", C.c_int, [_P, _P, _P, C.c_uint32, _P]),
    ("pt_renderer_reset_accumulation", C.c_int, [_P, _P]),
    ("pt_scene_set_frame_count", C.c_int, [_P, C.c_uint32]),
    ("pt_render", C.c_int, [_P, C.c_int32, _P, C.c_int32, C.POINTER(RenderStats)]),
    ("pt_render_batch", C.c_int, [_P, C.c_uint32, C.c_int32, C.POINTER(BatchConfig), C.POINTER(RenderStats)]),
    ("pt_autotune", C.c_int, [_P, C.c_int32, C.POINTER(TuneReport)]),
    ("pt_guide_create", C.c_int, [_P, C.c_uint32, C.POINTER(_P)]),
    ("pt_guide_destroy", C.c_int, [_P]),
    ("pt_guide_set_learning_rate", C.c_int, [_P, C.c_float]),
    ("pt_guide_set_alpha", C.c_int, [_P, C.c_float]),
    ("pt_guide_set_training", C.c_int, [_P, C.c_int32, C.c_uint32]),
    ("pt_guide_set_inference", C.c_int, [_P, C.c_int32]),
    ("pt_guide_set_schedule", C.c_int, [_P, C.c_float, C.c_float, C.c_float]),
    ("pt_guide_info", C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    ("pt_guide_loss", C.c_int, [_P, C.POINTER(C.c_float)]),
    ("pt_integrator_set_guide", C.c_int, [_P, _P, C.c_int32]),
    ("pt_guide_eval", C.c_int, [_P, _P, C.c_uint32, _P]),
    ("pt_guide_get_params", C.c_int, [_P, _P, _P, _P]),
    ("pt_guide_backward", C.c_int, [_P, _P, C.c_uint32, _P, _P]),
    ("pt_trace_closest", C.c_int, [_P, _P, C.c_uint32, _P, C.c_int32]),
    ("pt_trace_any", C.c_int, [_P, _P, C.c_uint32, _P, C.c_int32]),
    ("pt_trace_closest_static", C.c_int, [_P, _P, C.c_uint32, _P]),
    ("pt_sampler_stream", C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_uint32, C.c_int32, C.c_int32,
                                    C.c_uint32, C.c_uint32, C.c_int32, _P]),
    ("pt_bsdf_eval", C.c_int, [_P, _P, C.c_uint32, _P]),
    ("pt_tonemap", C.c_int, [_P, C.c_int32, C.c_int32, C.c_float, _P, C.c_int32, C.c_int32]),
]
EXPORTED = [name for name, _, _ in _SIGS]

_lib = None


class PTError(RuntimeError):
    """Raised when a C entry point returns a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[pt status {code}] {msg}")
        self.code = code


def lib() -> C.CDLL:
    """Load libpt_b200.so (fails loudly when it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m pathtracingtutorial_b200.build` "
                              f"(or __graft_entry__.build())")
        L = C.CDLL(LIB_PATH)
        for name, res, args in _SIGS:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != PT_OK:
        raise PTError(code, lib().pt_last_error().decode(errors="replace"))


def ptr(a: np.ndarray | None) -> C.c_void_p | None:
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return C.c_void_p(a.ctypes.data)
