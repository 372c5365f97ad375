"""TEST INFRASTRUCTURE: Python access to the CPU oracle (liboracle.so), to the
reference's own host-compiled code (_ref/libptref.so) and to the reference's
own CUDA integrator built for sm_100a (_ref/libptref_gpu.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.  `Oracle` is the restatement (oracle/pt_oracle.cpp); `RefHarness`
runs the reference's code and exists only where oracle/_ref was built (it is
built from the reference tree in the development container and travels with
the repository snapshot as a binary).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libptref.so")
REF_GPU_SO = os.path.join(HERE, "_ref", "libptref_gpu.so")

VERTEX = np.dtype([("position", "<f4", 3), ("_pad0", "<f4"), ("normal", "<f4", 3), ("_pad1", "<f4"),
                   ("uv", "<f4", 2), ("_pad2", "<f4", 2), ("tangent", "<f4", 4)])
FACE = np.dtype([("v0", "<u4"), ("v1", "<u4"), ("v2", "<u4"), ("material_id", "<i4")])
NODE = np.dtype([("bmin", "<f4", 3), ("data0", "<u4"), ("bmax", "<f4", 3), ("data1", "<u4")])
ALIAS = np.dtype([("prob", "<f4"), ("alias", "<u4")])
EMREF = np.dtype([("triangle_index", "<u4"), ("selection_pmf", "<f4"), ("cdf", "<f4"), ("_pad", "<f4")])


class Scene(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("num_vertices", C.c_uint32), ("faces", C.c_void_p),
                ("num_faces", C.c_uint32), ("materials", C.c_void_p), ("num_materials", C.c_uint32),
                ("nodes", C.c_void_p), ("num_nodes", C.c_uint32), ("emissive", C.c_void_p),
                ("num_emissive", C.c_uint32), ("tri_pmf", C.c_void_p), ("tri_alias", C.c_void_p),
                ("env_rgba", C.c_void_p), ("env_w", C.c_int32), ("env_h", C.c_int32), ("env_pmf", C.c_void_p),
                ("env_alias", C.c_void_p), ("num_env_texels", C.c_uint32), ("env_tw", C.c_int32),
                ("env_th", C.c_int32), ("punctual", C.c_void_p), ("num_punctual", C.c_uint32),
                ("camera_frame", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32),
                ("textures", C.c_void_p), ("num_textures", C.c_uint32)]


class OTex(C.Structure):
    _fields_ = [("rgba", C.c_void_p), ("width", C.c_int32), ("height", C.c_int32), ("wrap_s", C.c_int32),
                ("wrap_t", C.c_int32)]


class RenderArgs(C.Structure):
    _fields_ = [("sample_per_frame", C.c_int32), ("max_depth", C.c_int32), ("sampler_type", C.c_int32),
                ("arg_rtl", C.c_int32), ("pcg_seed", C.c_uint32), ("first_frame", C.c_uint32),
                ("num_frames", C.c_uint32), ("row0", C.c_int32), ("row_step", C.c_int32), ("threads", C.c_int32),
                ("precision", C.c_int32), ("col0", C.c_int32), ("col1", C.c_int32),
                ("row_end", C.c_int32), ("watertight", C.c_int32), ("_pad", C.c_int32)]


class Counters(C.Structure):
    _fields_ = [("closest_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("node_pops", C.c_uint64),
                ("tri_tests", C.c_uint64), ("shadow_node_pops", C.c_uint64), ("shadow_tri_tests", C.c_uint64),
                ("paths", C.c_uint64), ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


def _p(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return C.c_void_p(a.ctypes.data)


def reference_dir() -> str | None:
    """The reference tree oracle/Makefile would build from (PT_REF_DIR, else
    its default search), or None when there is none."""
    r = subprocess.run(["make", "-s", "-C", HERE, "ref-dir"], capture_output=True, text=True)
    path = r.stdout.strip()
    return path if r.returncode == 0 and path else None


def build(ref: bool | None = None) -> None:
    """Compile liboracle.so and, with ref (default: when a reference tree is
    found), the reference's host and GPU builds under _ref/."""
    if ref is None:
        ref = reference_dir() is not None
    targets = ["oracle", "ref", "ref-gpu"] if ref else ["oracle"]
    r = subprocess.run(["make", "-C", HERE, "-j8", *targets], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")


class Prepared:
    """Scene prepared with the oracle's own builder (BVH order, light tables)."""

    def __init__(self, vertices, faces, materials, nodes, depth, em_refs, tri_pmf, tri_alias, env, env_pmf,
                 env_alias, camera_frame, width, height, punctual=None, textures=None):
        if np.asarray(materials).dtype.itemsize != 256:
            raise ValueError("materials must be 256-byte records (pt_material)")
        self.vertices, self.faces, self.materials, self.nodes, self.depth = vertices, faces, materials, nodes, depth
        self.em_refs, self.tri_pmf, self.tri_alias = em_refs, tri_pmf, tri_alias
        self.env, self.env_pmf, self.env_alias = env, env_pmf, env_alias
        self.camera_frame, self.width, self.height = camera_frame, width, height
        self.punctual = punctual
        # material textures: [{"rgba": (H, W, 4) float32, "wrap_s": gl, "wrap_t": gl}, ...]
        self.textures = [dict(t, rgba=np.ascontiguousarray(t["rgba"], np.float32)) for t in (textures or [])]
        self._tex_table = None

    def struct(self) -> Scene:
        s = Scene()
        s.vertices, s.num_vertices = _p(self.vertices), len(self.vertices)
        s.faces, s.num_faces = _p(self.faces), len(self.faces)
        s.materials, s.num_materials = _p(self.materials), len(self.materials)
        s.nodes, s.num_nodes = _p(self.nodes), len(self.nodes)
        s.emissive, s.num_emissive = _p(self.em_refs), len(self.em_refs)
        s.tri_pmf, s.tri_alias = _p(self.tri_pmf), _p(self.tri_alias)
        if self.env is not None:
            s.env_rgba, s.env_h, s.env_w = _p(self.env), self.env.shape[0], self.env.shape[1]
        if self.env_pmf is not None and len(self.env_pmf):
            s.env_pmf, s.env_alias, s.num_env_texels = _p(self.env_pmf), _p(self.env_alias), len(self.env_pmf)
            s.env_tw, s.env_th = self.env.shape[1], self.env.shape[0]
        if self.punctual is not None and len(self.punctual):
            s.punctual, s.num_punctual = _p(self.punctual), len(self.punctual)
        s.camera_frame = _p(self.camera_frame)
        s.width, s.height = self.width, self.height
        if self.textures:
            tab = (OTex * len(self.textures))()
            for k, t in enumerate(self.textures):
                a = t["rgba"]
                tab[k] = OTex(a.ctypes.data if a.size else None, a.shape[1], a.shape[0],
                              int(t.get("wrap_s", 10497)), int(t.get("wrap_t", 10497)))
            self._tex_table = tab
            s.textures, s.num_textures = C.cast(tab, C.c_void_p), len(self.textures)
        return s


class Oracle:
    def __init__(self):
        if not os.path.exists(ORACLE_SO):
            build()
        self.L = C.CDLL(ORACLE_SO)

    def build_bvh(self, vertices, faces):
        v = np.ascontiguousarray(vertices, VERTEX)
        f = np.ascontiguousarray(faces, FACE).copy()
        nodes = np.zeros(max(1, 2 * len(f)), NODE)
        nn, depth = C.c_uint32(), C.c_uint32()
        rc = self.L.oracle_build_bvh(_p(v), C.c_uint32(len(v)), _p(f), C.c_uint32(len(f)), _p(nodes),
                                     C.c_uint32(len(nodes)), C.byref(nn), C.byref(depth))
        assert rc == 0, rc
        return nodes[:nn.value].copy(), f, depth.value

    def alias_table(self, weights):
        w = np.ascontiguousarray(weights, np.float32)
        out = np.zeros(len(w), ALIAS)
        rc = self.L.oracle_alias_table(_p(w), C.c_uint32(len(w)), _p(out))
        return out if rc == 0 else np.zeros(0, ALIAS)

    def emissive_tables(self, vertices, faces, materials):
        f = np.ascontiguousarray(faces, FACE)
        refs = np.zeros(len(f), EMREF)
        pmf = np.zeros(len(f), np.float32)
        alias = np.zeros(len(f), ALIAS)
        cnt = C.c_uint32()
        m = np.ascontiguousarray(materials)
        self.L.oracle_emissive_tables(_p(np.ascontiguousarray(vertices, VERTEX)), _p(f), C.c_uint32(len(f)), _p(m),
                                      C.c_uint32(len(m)), _p(refs), _p(pmf), _p(alias), C.byref(cnt))
        return refs[:cnt.value].copy(), pmf, alias[:cnt.value].copy()

    def env_tables(self, env):
        if env is None:
            return np.zeros(0, np.float32), np.zeros(0, ALIAS)
        e = np.ascontiguousarray(env, np.float32)
        h, w = e.shape[:2]
        pmf = np.zeros(w * h, np.float32)
        alias = np.zeros(w * h, ALIAS)
        rc = self.L.oracle_env_tables(_p(e), C.c_int32(w), C.c_int32(h), _p(pmf), _p(alias))
        if rc != 0:
            return np.zeros(0, np.float32), np.zeros(0, ALIAS)
        return pmf, alias

    def camera_frame(self, camera):
        out = np.zeros(16, np.float32)
        self.L.oracle_camera_frame(_p(np.ascontiguousarray(camera)), _p(out))
        return out

    def sampler_stream(self, sampler, w, h, frame, spf, sif, ndims, pcg_seed=0):
        out = np.zeros((h, w, ndims), np.float32)
        self.L.oracle_sampler_stream(C.c_int32(sampler), C.c_int32(w), C.c_int32(h), C.c_uint32(frame),
                                     C.c_int32(spf), C.c_int32(sif), C.c_uint32(ndims), C.c_uint32(pcg_seed), _p(out))
        return out

    def trace(self, nodes, vertices, faces, rays, any_hit=False, watertight=False):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        hits = np.zeros((n, 4), np.float32)
        occ = np.zeros(n, np.uint8)
        cnt = Counters()
        self.L.oracle_trace_mode(_p(nodes), _p(np.ascontiguousarray(vertices, VERTEX)),
                                 _p(np.ascontiguousarray(faces, FACE)), _p(rays), C.c_uint32(n),
                                 C.c_int32(1 if any_hit else 0), C.c_int32(1 if watertight else 0), _p(hits), _p(occ),
                                 C.byref(cnt))
        return (occ.astype(bool) if any_hit else hits), cnt.as_dict()

    def bsdf_eval(self, materials, records):
        rec = np.ascontiguousarray(records, np.float32)
        out = np.zeros((len(rec), 4), np.float32)
        m = np.ascontiguousarray(materials)
        self.L.oracle_bsdf_eval(_p(m), C.c_uint32(len(m)), _p(rec), C.c_uint32(len(rec)), _p(out))
        return out

    def prepare(self, sa) -> Prepared:
        """Build a SceneArrays (pathtracingtutorial_b200.scenes) with the oracle's own prep."""
        if np.asarray(sa.materials).dtype.itemsize != 256:
            raise ValueError("materials must be 256-byte records (pt_material)")
        nodes, faces, depth = self.build_bvh(sa.vertices, sa.faces)
        refs, pmf, alias = self.emissive_tables(sa.vertices, faces, sa.materials)
        env_pmf, env_alias = self.env_tables(sa.env)
        cf = self.camera_frame(sa.camera)
        env = None if sa.env is None else np.ascontiguousarray(sa.env, np.float32)
        punct = getattr(sa, "punctual", None)
        return Prepared(np.ascontiguousarray(sa.vertices, VERTEX), faces, np.ascontiguousarray(sa.materials), nodes,
                        depth, refs, pmf, alias, env, env_pmf, env_alias, cf, int(sa.camera["width"]),
                        int(sa.camera["height"]), punct, getattr(sa, "textures", None))

    def render(self, prep: Prepared, spf, max_depth, sampler, frames, first_frame=0, precision=64, rtl=1,
               pcg_seed=0, row0=0, row_step=1, threads=0, crop=None, watertight=False):
        """precision 32: the reference's film (H, W, 4).  precision 64: (mean, var) of shape (H, W, 3).
        crop = (x0, y0, x1, y1) renders only those pixels (the rest stay zero)."""
        sc = prep.struct()
        x0, y0, x1, y1 = crop if crop is not None else (0, row0, 0, 0)
        a = RenderArgs(spf, max_depth, sampler, rtl, pcg_seed, first_frame, frames, y0, row_step, threads,
                       precision, x0, x1, y1, 1 if watertight else 0, 0)
        cnt = Counters()
        h, w = prep.height, prep.width
        if precision == 32:
            out = np.zeros((h, w, 4), np.float32)
            self.L.oracle_render(C.byref(sc), C.byref(a), _p(out), None, None, C.byref(cnt))
            return out, cnt.as_dict()
        mean = np.zeros((h, w, 3), np.float64)
        var = np.zeros((h, w, 3), np.float64)
        self.L.oracle_render(C.byref(sc), C.byref(a), None, _p(mean), _p(var), C.byref(cnt))
        return (mean, var), cnt.as_dict()


class RefHarness:
    """The reference's own code, host compiled (requires oracle/_ref/libptref.so)."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_SO)

    def __init__(self):
        self.L = C.CDLL(REF_SO)

    def layout(self):
        out = np.zeros(256, np.int64)
        n = self.L.ref_struct_layout(_p(out), C.c_int(256))
        return out[:n]

    def write_image(self, path, rgba, flip_y=True):
        """ImageIO::write of an (H, W, 4) float image."""
        a = np.ascontiguousarray(rgba, np.float32)
        rc = self.L.ref_write_image(os.fsencode(path), _p(a), C.c_int(a.shape[1]), C.c_int(a.shape[0]),
                                    C.c_int(1 if flip_y else 0))
        if rc != 0:
            raise RuntimeError(f"reference writer failed on {path}")

    def load_json(self, path):
        counts = np.zeros(6, np.uint32)
        cam = np.zeros(80, np.uint8)
        settings = np.zeros(4, np.int32)
        rc = self.L.ref_load_json(os.fsencode(path), _p(counts), _p(cam), _p(settings))
        if rc != 0:
            raise RuntimeError(f"reference loader failed on {path}")
        nv, nf, nm, nl, ew, eh = (int(x) for x in counts)
        v = np.zeros(nv, VERTEX)
        f = np.zeros(nf, FACE)
        m = np.zeros(nm * 256, np.uint8)
        lights = np.zeros(nl * 112, np.uint8)
        env = np.zeros((eh, ew, 4), np.float32) if ew else None
        self.L.ref_loaded_arrays(_p(v), _p(f), _p(m), _p(lights), _p(env) if env is not None else None)
        return {"vertices": v, "faces": f, "materials": m, "lights": lights, "env": env, "camera": cam,
                "settings": settings}

    def loaded_textures(self):
        """Material textures of the last load_json: [{"rgba": (H, W, 4), "wrap_s", "wrap_t"}]."""
        self.L.ref_loaded_texture_count.restype = C.c_uint32
        out = []
        for i in range(int(self.L.ref_loaded_texture_count())):
            info = np.zeros(5, np.int32)
            self.L.ref_loaded_texture(C.c_uint32(i), _p(info), None)
            rgba = np.zeros((max(int(info[1]), 0), max(int(info[0]), 0), 4), np.float32)
            if rgba.size:
                self.L.ref_loaded_texture(C.c_uint32(i), _p(info), _p(rgba))
            out.append({"rgba": rgba, "wrap_s": int(info[3]), "wrap_t": int(info[4]), "channel": int(info[2])})
        return out

    def decode_image(self, data: bytes):
        """The reference's stb_image decode with four channels forced -> (H, W, 4) uint8."""
        buf = np.frombuffer(bytes(data), np.uint8)
        w, h = C.c_int32(), C.c_int32()
        if self.L.ref_decode_image(_p(buf), C.c_int(len(buf)), None, C.c_int(0), C.byref(w), C.byref(h)) != 0:
            raise RuntimeError("reference decoder rejected the image")
        out = np.zeros((h.value, w.value, 4), np.uint8)
        self.L.ref_decode_image(_p(buf), C.c_int(len(buf)), _p(out), C.c_int(out.size), C.byref(w), C.byref(h))
        return out

    def build(self, vertices, faces, materials, env=None):
        v = np.ascontiguousarray(vertices, VERTEX)
        f = np.ascontiguousarray(faces, FACE).copy()
        m = np.ascontiguousarray(materials)
        nm = m.nbytes // 256
        ew, eh = (env.shape[1], env.shape[0]) if env is not None else (0, 0)
        e = np.ascontiguousarray(env, np.float32) if env is not None else None
        nodes = np.zeros(max(1, 2 * len(f)), NODE)
        em = np.zeros(max(1, len(f)), EMREF)
        tp = np.zeros(max(1, len(f)), np.float32)
        ta = np.zeros(max(1, len(f)), ALIAS)
        ep = np.zeros(max(1, ew * eh), np.float32)
        ea = np.zeros(max(1, ew * eh), ALIAS)
        sizes = np.zeros(5, np.uint32)
        rc = self.L.ref_build(_p(v), C.c_uint32(len(v)), _p(f), C.c_uint32(len(f)), _p(m), C.c_uint32(nm), _p(e),
                              C.c_int(ew), C.c_int(eh), _p(nodes), C.c_uint32(len(nodes)), _p(em), _p(tp), _p(ta),
                              _p(ep), _p(ea), _p(sizes))
        assert rc == 0, rc
        n_nodes, n_em, n_env = int(sizes[0]), int(sizes[1]), int(sizes[2])
        return {"nodes": nodes[:n_nodes].copy(), "faces": f, "emissive": em[:n_em].copy(),
                "tri_pmf": tp[:len(f)].copy(), "tri_alias": ta[:n_em].copy(), "env_pmf": ep[:n_env].copy(),
                "env_alias": ea[:n_env].copy()}

    def camera_frame(self, camera):
        out = np.zeros(16, np.float32)
        self.L.ref_camera_frame(_p(np.ascontiguousarray(camera)), _p(out))
        return out

    def sampler_stream(self, sampler, w, h, frame, spf, sif, ndims):
        out = np.zeros((h, w, ndims), np.float32)
        self.L.ref_sampler_stream(C.c_int(sampler), C.c_int(w), C.c_int(h), C.c_uint32(frame), C.c_int(spf),
                                  C.c_int(sif), C.c_uint32(ndims), _p(out))
        return out

    def trace(self, nodes, vertices, faces, rays, any_hit=False):
        rays = np.ascontiguousarray(rays, np.float32)
        n = len(rays)
        hits = np.zeros((n, 4), np.float32)
        occ = np.zeros(n, np.uint8)
        self.L.ref_trace(_p(nodes), _p(np.ascontiguousarray(vertices, VERTEX)), _p(np.ascontiguousarray(faces, FACE)),
                         _p(rays), C.c_uint32(n), C.c_int(1 if any_hit else 0), _p(hits), _p(occ))
        return occ.astype(bool) if any_hit else hits

    def render(self, vertices, faces, materials, camera, settings, env=None, lights=None, first_frame=0,
               num_frames=1, row0=0, row_step=1, threads=0):
        """kernelPathTrace over the selected rows.  Returns (acc, new, stats)."""
        v = np.ascontiguousarray(vertices, VERTEX)
        f = np.ascontiguousarray(faces, FACE)
        m = np.ascontiguousarray(materials)
        nm = m.nbytes // 256
        cam = np.ascontiguousarray(camera)
        w = int(np.frombuffer(cam.tobytes()[60:64], np.int32)[0])
        h = int(np.frombuffer(cam.tobytes()[64:68], np.int32)[0])
        ew, eh = (env.shape[1], env.shape[0]) if env is not None else (0, 0)
        e = np.ascontiguousarray(env, np.float32) if env is not None else None
        L = np.ascontiguousarray(lights) if lights is not None else None
        nl = 0 if L is None else L.nbytes // 112
        st = np.ascontiguousarray(settings, np.int32)
        acc = np.zeros((h, w, 4), np.float32)
        new = np.zeros((h, w, 4), np.float32)
        stats = np.zeros(4, np.float64)
        self.L.ref_render(_p(v), C.c_uint32(len(v)), _p(f), C.c_uint32(len(f)), _p(m), C.c_uint32(nm), _p(e),
                          C.c_int(ew), C.c_int(eh), _p(L), C.c_uint32(nl), _p(cam), _p(st), C.c_uint32(first_frame),
                          C.c_uint32(num_frames), C.c_int(row0), C.c_int(row_step), C.c_int(threads), _p(acc),
                          _p(new), _p(stats))
        return acc, new, {"closest_rays": stats[0], "shadow_rays": stats[1], "paths": stats[2], "seconds": stats[3]}


class RefGpu:
    """The reference's own CUDA path tracer (kernelPathTrace through
    PathIntegrator::launch, DeviceScene, Film), built unchanged for sm_100a
    (requires oracle/_ref/libptref_gpu.so).  One instance = one scene."""

    @staticmethod
    def available() -> bool:
        return os.path.exists(REF_GPU_SO)

    def __init__(self, sa, device: int = 0):
        self.L = C.CDLL(REF_GPU_SO)
        self.L.refgpu_frame_count.restype = C.c_uint32
        v = np.ascontiguousarray(sa.vertices)
        f = np.ascontiguousarray(sa.faces)
        m = np.ascontiguousarray(sa.materials)
        cam = np.ascontiguousarray(sa.camera)
        self.width = int(np.frombuffer(cam.tobytes()[60:64], np.int32)[0])
        self.height = int(np.frombuffer(cam.tobytes()[64:68], np.int32)[0])
        env = None if sa.env is None else np.ascontiguousarray(sa.env, np.float32)
        ew, eh = (env.shape[1], env.shape[0]) if env is not None else (0, 0)
        st = np.array([sa.spp, sa.sample_per_frame, sa.max_depth, sa.sampler], np.int32)
        h = C.c_void_p()
        texs = [dict(t, rgba=np.ascontiguousarray(t["rgba"], np.float32)) for t in getattr(sa, "textures", [])]
        tab = (OTex * max(1, len(texs)))()
        for k, t in enumerate(texs):
            a = t["rgba"]
            tab[k] = OTex(a.ctypes.data if a.size else None, a.shape[1], a.shape[0], int(t.get("wrap_s", 10497)),
                          int(t.get("wrap_t", 10497)))
        rc = self.L.refgpu_create_textured(_p(v), C.c_uint32(len(v)), _p(f), C.c_uint32(len(f)), _p(m),
                                           C.c_uint32(m.nbytes // 256), _p(env), C.c_int(ew), C.c_int(eh), _p(cam),
                                           _p(st), C.cast(tab, C.c_void_p), C.c_uint32(len(texs)), C.c_int(device),
                                           C.byref(h))
        if rc != 0:
            raise RuntimeError(f"reference GPU scene setup failed ({rc})")
        self._h = h

    def reset(self) -> None:
        """Renderer::resetAccumulation: frame 0, cleared film."""
        if self.L.refgpu_reset(self._h) != 0:
            raise RuntimeError("reference GPU reset failed")

    def render(self, frames: int) -> tuple[float, float]:
        """`frames` renderBatch calls; returns (device ms, wall ms) of the loop."""
        t = np.zeros(2, np.float64)
        if self.L.refgpu_render(self._h, C.c_int(frames), _p(t)) != 0:
            raise RuntimeError("reference GPU render failed")
        return float(t[0]), float(t[1])

    def image(self) -> np.ndarray:
        out = np.zeros((self.height, self.width, 4), np.float32)
        self.L.refgpu_download(self._h, _p(out))
        return out

    def close(self) -> None:
        if self._h:
            self.L.refgpu_destroy(self._h)
            self._h = None


def tonemap_ref(img, exposure=-2.8):
    """The reference preview's display mapping (Part_2/preview/tone_mapping.frag:12-29)
    in float64: 1 - exp(-c * 2^exposure), linear_to_srgb per channel (:12-19),
    then 8-bit unorm with round to nearest.  Returns (H, W, 4) uint8, alpha 255."""
    c = np.asarray(img, np.float64)[..., :3]
    t = 1.0 - np.exp(-c * 2.0 ** exposure)
    e = np.where(t <= 0.0031308, 12.92 * t, 1.055 * np.power(np.maximum(t, 0.0), 1.0 / 2.4) - 0.055)
    out = np.full(c.shape[:2] + (4,), 255, np.uint8)
    out[..., :3] = np.rint(np.clip(e, 0.0, 1.0) * 255.0).astype(np.uint8)
    return out
