"""Seeded procedural scenes for the benchmark workloads.

All scenes are returned as plain arrays in the reference's struct layouts
(VERTEX_DTYPE / FACE_DTYPE / MATERIAL_DTYPE / CAMERA_DTYPE) plus render
settings, so the same input feeds the GPU library, the oracle and the
reference's own host code.  The reference measures on no public data set;
these generators produce the workload shapes named for each configuration.

  cornell_box()      36 triangles, 512x512, 64 spp, depth 8, PCG
  icosphere_field()  400 displaced subdivision-4 icospheres on a ground quad
                     (2,048,002 triangles), Disney materials, synthetic HDR sky
                     with a 5e4-peak sun lobe, 1920x1080, 256 spp, depth 16, Sobol
  hidden_light_room() 10 x 10 x 4 m room, 300 tessellated boxes (~200k triangles),
                     0.5 x 0.5 light of radiance 200 behind a wall with a 0.3 m gap
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from ._ffi import FACE_DTYPE, MATERIAL_DTYPE, SAMPLER_PCG, SAMPLER_SOBOL, VERTEX_DTYPE
from . import default_material, make_camera


@dataclass
class SceneArrays:
    name: str
    vertices: np.ndarray
    faces: np.ndarray
    materials: np.ndarray
    camera: np.ndarray
    env: np.ndarray | None = None
    spp: int = 64
    sample_per_frame: int = 4
    max_depth: int = 8
    sampler: int = SAMPLER_SOBOL
    pcg_seed: int = 0
    meta: dict = field(default_factory=dict)
    # material textures: [{"rgba": (H, W, 4) float32 texels, "wrap_s": GL mode, "wrap_t": GL mode}]
    textures: list = field(default_factory=list)

    def scene(self):
        """A SceneManager with these arrays and render settings (not yet built)."""
        from . import SceneManager
        s = SceneManager.from_arrays(self.vertices, self.faces, self.materials, self.camera, self.env)
        for t in self.textures:
            s.add_texture(t["rgba"], t.get("wrap_s", 10497), t.get("wrap_t", 10497))
        s.update_settings(spp=self.spp, sample_per_frame=self.sample_per_frame, max_depth=self.max_depth,
                          sampler_type=self.sampler, pcg_seed=self.pcg_seed)
        return s

    def save(self, path: str) -> None:
        """Binary dump read by the oracle's reference harness (oracle/ref_harness.cpp)."""
        with open(path, "wb") as f:
            hdr = np.array([0x50544231, len(self.vertices), len(self.faces), len(self.materials),
                            0 if self.env is None else self.env.shape[1],
                            0 if self.env is None else self.env.shape[0],
                            self.spp, self.sample_per_frame, self.max_depth, self.sampler, self.pcg_seed, 0],
                           np.uint32)
            f.write(hdr.tobytes())
            f.write(np.ascontiguousarray(self.camera).tobytes())
            f.write(np.ascontiguousarray(self.vertices).tobytes())
            f.write(np.ascontiguousarray(self.faces).tobytes())
            f.write(np.ascontiguousarray(self.materials).tobytes())
            if self.env is not None:
                f.write(np.ascontiguousarray(self.env, np.float32).tobytes())


# ---------------------------------------------------------------------------
# geometry helpers
# ---------------------------------------------------------------------------
def _vertices(pos: np.ndarray, nrm: np.ndarray, uv: np.ndarray | None = None,
              tangent: np.ndarray | None = None) -> np.ndarray:
    v = np.zeros(len(pos), VERTEX_DTYPE)
    v["position"] = pos
    v["normal"] = nrm
    if uv is not None:
        v["uv"] = uv
    if tangent is not None:
        v["tangent"] = tangent
    return v


def _faces(tri: np.ndarray, mat) -> np.ndarray:
    f = np.zeros(len(tri), FACE_DTYPE)
    f["v0"], f["v1"], f["v2"] = tri[:, 0], tri[:, 1], tri[:, 2]
    f["material_id"] = mat
    return f


def _materials(items) -> np.ndarray:
    """List of 0-d material records -> MATERIAL_DTYPE array (np.stack would drop the padding)."""
    out = np.zeros(len(items), MATERIAL_DTYPE)
    for i, m in enumerate(items):
        out[i] = m
    return out


def _normalize(v: np.ndarray) -> np.ndarray:
    n = np.linalg.norm(v, axis=-1, keepdims=True)
    return v / np.where(n > 0, n, 1)


def quad(a, b, c, d, mat: int, subdiv: int = 1):
    """Quad a-b-c-d split into subdiv x subdiv cells of two triangles each
    (subdiv=1 gives the reference's buildQuad triangles (0,1,2), (0,2,3))."""
    a, b, c, d = (np.asarray(x, np.float64) for x in (a, b, c, d))
    n = _normalize(np.cross(b - a, c - a))
    t = _normalize(b - a)
    k = subdiv
    s, r = np.meshgrid(np.linspace(0, 1, k + 1), np.linspace(0, 1, k + 1), indexing="xy")
    s, r = s.ravel(), r.ravel()
    # bilinear patch: s along a->b, r along a->d
    pos = ((1 - s) * (1 - r))[:, None] * a + (s * (1 - r))[:, None] * b + (s * r)[:, None] * c + ((1 - s) * r)[:, None] * d
    uv = np.stack([s, r], 1)
    idx = np.arange((k + 1) * (k + 1)).reshape(k + 1, k + 1)
    p0, p1 = idx[:-1, :-1].ravel(), idx[:-1, 1:].ravel()
    p2, p3 = idx[1:, 1:].ravel(), idx[1:, :-1].ravel()
    tri = np.concatenate([np.stack([p0, p1, p2], 1), np.stack([p0, p2, p3], 1)])
    tri = tri.reshape(2, -1, 3).transpose(1, 0, 2).reshape(-1, 3)
    tan = np.concatenate([np.broadcast_to(t, (len(pos), 3)), np.ones((len(pos), 1))], 1)
    return pos.astype(np.float32), np.broadcast_to(n, pos.shape).astype(np.float32), uv.astype(np.float32), \
        tan.astype(np.float32), tri, mat


def box(center, size, yaw: float, mat: int, subdiv: int = 1):
    """Axis-aligned (then yawed) box as 6 outward-facing quads."""
    cx, cy, cz = center
    sx, sy, sz = (s * 0.5 for s in size)
    corners = np.array([[-sx, -sy, -sz], [sx, -sy, -sz], [sx, sy, -sz], [-sx, sy, -sz],
                        [-sx, -sy, sz], [sx, -sy, sz], [sx, sy, sz], [-sx, sy, sz]], np.float64)
    cyw, syw = np.cos(yaw), np.sin(yaw)
    rot = np.array([[cyw, 0, syw], [0, 1, 0], [-syw, 0, cyw]])
    corners = corners @ rot.T + np.array([cx, cy, cz])
    faces = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (3, 7, 6, 2), (0, 4, 7, 3), (1, 2, 6, 5)]
    return [quad(corners[a], corners[b], corners[c], corners[d], mat, subdiv) for a, b, c, d in faces]


class _Builder:
    def __init__(self):
        self.pos, self.nrm, self.uv, self.tan, self.tri, self.mat = [], [], [], [], [], []
        self.nv = 0

    def add(self, part):
        pos, nrm, uv, tan, tri, mat = part
        self.pos.append(pos); self.nrm.append(nrm); self.uv.append(uv); self.tan.append(tan)
        self.tri.append(tri + self.nv)
        self.mat.append(np.broadcast_to(np.asarray(mat, np.int32), (len(tri),)))
        self.nv += len(pos)

    def arrays(self):
        v = _vertices(np.concatenate(self.pos), np.concatenate(self.nrm), np.concatenate(self.uv),
                      np.concatenate(self.tan))
        f = _faces(np.concatenate(self.tri).astype(np.uint32), np.concatenate(self.mat))
        return v, f


# ---------------------------------------------------------------------------
# Cornell box: 36 triangles
# ---------------------------------------------------------------------------
def cornell_box(width: int = 512, height: int = 512, spp: int = 64, max_depth: int = 8,
                pcg_seed: int = 1) -> SceneArrays:
    """5 diffuse walls (white 0.73, red 0.65, green 0.12 dominant channels), a tall
    mirror box (metallic 1, roughness 0 -> clamped to 0.001, a delta surface), a
    short diffuse box and a 0.25 x 0.25 light of radiance (17, 12, 4)."""
    mats = _materials([
        default_material(base_color=(0.73, 0.73, 0.73), roughness=1.0),              # 0 white
        default_material(base_color=(0.65, 0.05, 0.05), roughness=1.0),              # 1 red
        default_material(base_color=(0.12, 0.45, 0.15), roughness=1.0),              # 2 green
        default_material(base_color=(1.0, 1.0, 1.0), metallic=1.0, roughness=0.0),   # 3 mirror
        default_material(base_color=(1.0, 1.0, 1.0), emissive=(17.0, 12.0, 4.0), emissive_strength=1.0),  # 4 light
    ])
    b = _Builder()
    L, H = 0.5, 1.0
    b.add(quad((-L, 0, L), (L, 0, L), (L, 0, -L), (-L, 0, -L), 0))          # floor
    b.add(quad((-L, H, L), (-L, H, -L), (L, H, -L), (L, H, L), 0))          # ceiling
    b.add(quad((-L, 0, -L), (L, 0, -L), (L, H, -L), (-L, H, -L), 0))        # back
    b.add(quad((-L, 0, L), (-L, 0, -L), (-L, H, -L), (-L, H, L), 1))        # left (red)
    b.add(quad((L, 0, -L), (L, 0, L), (L, H, L), (L, H, -L), 2))            # right (green)
    for part in box((-0.17, 0.3, -0.15), (0.28, 0.6, 0.28), np.radians(17.0), 3):
        b.add(part)
    for part in box((0.18, 0.15, 0.16), (0.28, 0.3, 0.28), np.radians(-18.0), 0):
        b.add(part)
    s = 0.125
    b.add(quad((-s, H - 1e-3, -s), (s, H - 1e-3, -s), (s, H - 1e-3, s), (-s, H - 1e-3, s), 4))
    v, f = b.arrays()
    assert len(f) == 36
    cam = make_camera(position=(0.0, 0.5, 1.95), look_at=(0.0, 0.5, 0.0), up=(0, 1, 0), fov=40.0,
                      width=width, height=height)
    return SceneArrays("cornell_box_36tri", v, f, mats, cam, None, spp=spp, sample_per_frame=4,
                       max_depth=max_depth, sampler=SAMPLER_PCG, pcg_seed=pcg_seed,
                       meta={"triangles": 36})


# ---------------------------------------------------------------------------
# Textured Cornell box
# ---------------------------------------------------------------------------
def procedural_textures(seed: int = 5, size: int = 64):
    """Four material textures as float RGBA arrays (glTF texels are 8-bit
    values / 255): a coloured checker whose alpha holds a disc cut-out
    (REPEAT), a metallic-roughness map (G roughness, B metallic; CLAMP), a
    tangent-space bump normal map (REPEAT) and a value-noise map used for the
    clearcoat, transmission and sheen channels (MIRRORED_REPEAT)."""
    rng = np.random.default_rng(seed)
    n = size
    y, x = (np.mgrid[0:n, 0:n] + 0.5) / n
    chk = ((np.floor(x * 8) + np.floor(y * 8)) % 2)[..., None]
    col = np.where(chk > 0, np.array([0.85, 0.75, 0.3]), np.array([0.2, 0.45, 0.8]))
    alpha = (((x - 0.5) ** 2 + (y - 0.5) ** 2) > 0.12).astype(np.float64)
    base = np.concatenate([col, alpha[..., None]], -1)
    mr = np.stack([np.zeros_like(x), 0.2 + 0.8 * x, (y > 0.5).astype(np.float64), np.ones_like(x)], -1)
    hx, hy = np.sin(x * 6 * np.pi), np.sin(y * 6 * np.pi)
    nrm = np.stack([-0.4 * np.cos(x * 6 * np.pi) * hy, -0.4 * hx * np.cos(y * 6 * np.pi), np.ones_like(x)], -1)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    nmap = np.concatenate([0.5 * (nrm + 1.0), np.ones_like(x)[..., None]], -1)
    noise = rng.uniform(0, 1, (n // 8 + 1, n // 8 + 1))
    noise = np.kron(noise, np.ones((8, 8)))[:n, :n]
    misc = np.stack([noise, 1.0 - noise, 0.5 * noise + 0.25, noise], -1)

    def q8(a):   # 8-bit texels as glTF images store them
        return (np.round(np.clip(a, 0, 1) * 255.0) / 255.0).astype(np.float32)
    return [{"rgba": q8(base), "wrap_s": 10497, "wrap_t": 10497},
            {"rgba": q8(mr), "wrap_s": 33071, "wrap_t": 33071},
            {"rgba": q8(nmap), "wrap_s": 10497, "wrap_t": 10497},
            {"rgba": q8(misc), "wrap_s": 33648, "wrap_t": 33648}]


def textured_cornell(width: int = 128, height: int = 128, spp: int = 16, max_depth: int = 8,
                     sampler: int = SAMPLER_PCG, pcg_seed: int = 1) -> SceneArrays:
    """The Cornell box with material textures on every path of the textured
    shading: a checker base colour on the floor (KHR_texture_transform scale,
    rotation and offset), a normal map and metallic-roughness map on the back
    wall, clearcoat / sheen / transmission maps on the short box, an
    alpha-MASK cut-out panel and an alpha-BLEND panel (baseAlpha 0.6 times the
    texture's alpha) standing in the room."""
    sa = cornell_box(width=width, height=height, spp=spp, max_depth=max_depth, pcg_seed=pcg_seed)
    sa.sampler = sampler
    mats = list(sa.materials)
    floor = default_material(base_color=(0.9, 0.9, 0.9), roughness=0.8, base_color_tex=0,
                             uv_scale_x=3.0, uv_scale_y=2.0, uv_rotation=0.35, uv_offset_x=0.1)
    back = default_material(base_color=(0.8, 0.8, 0.8), roughness=1.0, metallic=1.0, normal_tex=2,
                            normal_scale=1.5, metallic_roughness_tex=1)
    short_box = default_material(base_color=(0.7, 0.6, 0.5), roughness=0.4, clearcoat=1.0, clearcoat_tex=3,
                                 clearcoat_roughness=0.5, clearcoat_roughness_tex=3, sheen=1.0, sheen_roughness_tex=3,
                                 sheen_color_tex=0, spec_trans=0.5, transmission_tex=3)
    mask = default_material(base_color=(0.9, 0.3, 0.3), roughness=0.6, base_color_tex=0, alpha_mode=1,
                            alpha_cutoff=0.5, double_sided=1)
    blend = default_material(base_color=(0.3, 0.9, 0.4), roughness=0.5, base_color_tex=0, alpha_mode=2,
                             base_alpha=0.6, double_sided=1)
    first = len(mats)
    mats += [floor, back, short_box, mask, blend]
    m = _materials(mats)
    f = sa.faces.copy()
    f["material_id"][0:2] = first          # floor
    f["material_id"][4:6] = first + 1      # back wall
    f["material_id"][22:34] = first + 2    # short box (the second box)
    b = _Builder()
    b.add(quad((-0.35, 0.05, 0.25), (-0.05, 0.05, 0.25), (-0.05, 0.45, 0.25), (-0.35, 0.45, 0.25), first + 3))
    b.add(quad((0.05, 0.35, 0.3), (0.4, 0.35, 0.3), (0.4, 0.7, 0.3), (0.05, 0.7, 0.3), first + 4))
    pv, pf = b.arrays()
    pf["v0"] += len(sa.vertices); pf["v1"] += len(sa.vertices); pf["v2"] += len(sa.vertices)
    sa.vertices = np.concatenate([sa.vertices, pv])
    sa.faces = np.concatenate([f, pf])
    sa.materials = m
    sa.textures = procedural_textures()
    sa.name = f"textured_cornell_{len(sa.faces)}tri"
    sa.meta = {"triangles": int(len(sa.faces)), "textures": len(sa.textures)}
    return sa


# ---------------------------------------------------------------------------
# Icosphere field
# ---------------------------------------------------------------------------
def icosphere(subdiv: int):
    t = (1.0 + 5 ** 0.5) / 2.0
    verts = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
             (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    faces = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
             (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
             (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)]
    v = _normalize(np.array(verts, np.float64))
    f = np.array(faces, np.int64)
    for _ in range(subdiv):
        edges = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        key = np.sort(edges, 1)
        uniq, inv = np.unique(key, axis=0, return_inverse=True)
        mids = _normalize(0.5 * (v[uniq[:, 0]] + v[uniq[:, 1]]))
        base = len(v)
        v = np.concatenate([v, mids])
        m = inv.reshape(3, -1).T + base      # midpoints of edges (01, 12, 20)
        a, b_, c = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([a, m01, m20], 1), np.stack([b_, m12, m01], 1),
                            np.stack([c, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    return v, f


def _vertex_normals(pos: np.ndarray, tri: np.ndarray) -> np.ndarray:
    fn = np.cross(pos[tri[:, 1]] - pos[tri[:, 0]], pos[tri[:, 2]] - pos[tri[:, 0]])
    n = np.zeros_like(pos)
    for k in range(3):
        for c in range(3):
            n[:, c] += np.bincount(tri[:, k], weights=fn[:, c], minlength=len(pos))
    return _normalize(n)


def sky_env(width: int = 2048, height: int = 1024, sun_peak: float = 5e4, sun_sigma_deg: float = 0.5,
            sun_elev_deg: float = 35.0, sun_azim_deg: float = 40.0) -> np.ndarray:
    """Sky gradient + Gaussian sun lobe, (H, W, 4) float32, equirectangular in the
    reference's mapping (v = 0 is +y, direction = (cos phi sin th, cos th, sin phi sin th))."""
    u = (np.arange(width) + 0.5) / width
    v = (np.arange(height) + 0.5) / height
    phi = (u - 0.5) * 2 * np.pi
    th = v * np.pi
    d = np.stack([np.cos(phi)[None, :] * np.sin(th)[:, None], np.broadcast_to(np.cos(th)[:, None], (height, width)),
                  np.sin(phi)[None, :] * np.sin(th)[:, None]], -1)
    y = d[..., 1]
    zen = np.array([0.25, 0.45, 1.0])
    hor = np.array([0.9, 0.95, 1.0])
    gnd = np.array([0.18, 0.16, 0.14])
    t = np.clip(y, 0, 1)[..., None] ** 0.5
    sky = np.where(y[..., None] >= 0, hor * (1 - t) + zen * t, gnd * np.clip(1 + y, 0.2, 1)[..., None])
    el, az = np.radians(sun_elev_deg), np.radians(sun_azim_deg)
    sd = np.array([np.cos(az) * np.cos(el), np.sin(el), np.sin(az) * np.cos(el)])
    ang = np.arccos(np.clip(d @ sd, -1, 1))
    sig = np.radians(sun_sigma_deg)
    sun = sun_peak * np.exp(-0.5 * (ang / sig) ** 2)
    rgb = sky * 1.5 + sun[..., None] * np.array([1.0, 0.95, 0.85])
    out = np.ones((height, width, 4), np.float32)
    out[..., :3] = rgb
    return out


def icosphere_field(n_spheres: int = 400, subdiv: int = 4, width: int = 1920, height: int = 1080,
                    spp: int = 256, max_depth: int = 16, seed: int = 7, env_size=(2048, 1024)) -> SceneArrays:
    rng = np.random.default_rng(seed)
    base_v, base_f = icosphere(subdiv)
    nv, nf = len(base_v), len(base_f)
    radius = np.exp(rng.uniform(np.log(0.05), np.log(2.0), n_spheres))
    extent = 22.0
    cx = rng.uniform(-extent, extent, n_spheres)
    cz = rng.uniform(-extent, extent * 0.6, n_spheres)
    # displacement: sum of 4 random plane waves on the unit sphere, amplitude 5 % of radius
    kdir = _normalize(rng.normal(size=(n_spheres, 4, 3)))
    kfreq = rng.uniform(2.0, 6.0, (n_spheres, 4, 1))
    kph = rng.uniform(0, 2 * np.pi, (n_spheres, 4))
    waves = np.sin(np.einsum("vc,skc->svk", base_v, kdir * kfreq) + kph[:, None, :]).mean(-1)  # (S, V)
    disp = 1.0 + 0.05 * waves
    pos = base_v[None] * (radius[:, None, None] * disp[..., None])
    pos += np.stack([cx, radius, cz], 1)[:, None, :]
    pos = pos.reshape(-1, 3)
    tri = (base_f[None] + (np.arange(n_spheres) * nv)[:, None, None]).reshape(-1, 3)
    nrm = _vertex_normals(pos, tri)
    uv = np.zeros((len(pos), 2))
    mats = [default_material(base_color=(0.5, 0.5, 0.5), roughness=0.8)]   # ground
    for i in range(n_spheres):
        mats.append(default_material(base_color=tuple(rng.uniform(0, 1, 3)), metallic=rng.uniform(0, 1),
                                     roughness=rng.uniform(0.05, 1.0), clearcoat=rng.uniform(0, 1)))
    mats = _materials(mats)
    sph_mat = np.repeat(np.arange(1, n_spheres + 1, dtype=np.int32), nf)
    G = 200.0
    g = quad((-G, 0, G), (G, 0, G), (G, 0, -G), (-G, 0, -G), 0)
    b = _Builder()
    b.add((pos.astype(np.float32), nrm.astype(np.float32), uv.astype(np.float32),
           np.zeros((len(pos), 4), np.float32), tri, sph_mat))
    b.add(g)
    v, f = b.arrays()
    env = sky_env(*env_size) if env_size is not None else None
    cam = make_camera(position=(0.0, 7.0, 32.0), look_at=(0.0, 0.5, 0.0), fov=50.0, width=width, height=height)
    return SceneArrays(f"icosphere_field_{len(f)}tri", v, f, mats, cam, env, spp=spp, sample_per_frame=4,
                       max_depth=max_depth, sampler=SAMPLER_SOBOL,
                       meta={"triangles": int(len(f)), "spheres": n_spheres, "subdiv": subdiv})


def uneven_batch(n_scenes: int = 64, seed: int = 3, env_size=(1024, 512), max_depth: int = 12,
                 tri_range=(1_000, 2_000_000)):
    """Uneven batch: scenes generated like icosphere_field with triangle counts
    log-uniform in tri_range, resolutions drawn from {256^2, 512^2, 1024^2,
    1280x720}, spp uniform in 16..512, depth 12.  One shared sky (env_size)."""
    rng = np.random.default_rng(seed)
    env = sky_env(*env_size)
    res = [(256, 256), (512, 512), (1024, 1024), (1280, 720)]
    out = []
    for k in range(n_scenes):
        target = float(np.exp(rng.uniform(np.log(tri_range[0]), np.log(tri_range[1]))))
        sub = next(s for s in (1, 2, 3, 4) if target / (20 * 4 ** s) <= 400 or s == 4)
        n_sph = max(1, int(round(target / (20 * 4 ** sub))))
        w, h = res[int(rng.integers(0, len(res)))]
        spp = int(rng.integers(16, 513))
        sa = icosphere_field(n_spheres=n_sph, subdiv=sub, width=w, height=h, spp=spp, max_depth=max_depth,
                             seed=int(rng.integers(0, 2 ** 31)), env_size=None)
        sa.env = env
        sa.name = f"batch{k:02d}_{len(sa.faces)}tri_{w}x{h}_{spp}spp"
        out.append(sa)
    return out


# ---------------------------------------------------------------------------
# Hidden-light room
# ---------------------------------------------------------------------------
def hidden_light_room(n_boxes: int = 300, box_subdiv: int = 7, width: int = 1024, height: int = 1024,
                      spp: int = 1024, max_depth: int = 16, seed: int = 11) -> SceneArrays:
    rng = np.random.default_rng(seed)
    mats = _materials([
        default_material(base_color=(0.7, 0.7, 0.7), roughness=1.0),                 # 0 walls
        default_material(base_color=(0.6, 0.5, 0.4), roughness=0.6),                 # 1 furniture
        default_material(base_color=(1, 1, 1), emissive=(200.0, 200.0, 200.0)),     # 2 light
        default_material(base_color=(0.5, 0.6, 0.7), roughness=0.3, metallic=0.5),  # 3 furniture 2
    ])
    b = _Builder()
    X, Z, Y = 5.0, 5.0, 4.0
    ws = 40
    b.add(quad((-X, 0, Z), (X, 0, Z), (X, 0, -Z), (-X, 0, -Z), 0, ws))       # floor
    b.add(quad((-X, Y, Z), (-X, Y, -Z), (X, Y, -Z), (X, Y, Z), 0, ws))       # ceiling
    b.add(quad((-X, 0, -Z), (X, 0, -Z), (X, Y, -Z), (-X, Y, -Z), 0, ws))     # back
    b.add(quad((-X, 0, Z), (-X, 0, -Z), (-X, Y, -Z), (-X, Y, Z), 0, ws))     # left
    b.add(quad((X, 0, -Z), (X, 0, Z), (X, Y, Z), (X, Y, -Z), 0, ws))         # right
    b.add(quad((X, 0, Z), (-X, 0, Z), (-X, Y, Z), (X, Y, Z), 0, ws))         # front
    # partition wall at x = 3.7 leaving a 0.3 m gap under the ceiling
    wx, gap = 3.7, 0.3
    b.add(quad((wx, 0, -Z), (wx, 0, Z), (wx, Y - gap, Z), (wx, Y - gap, -Z), 0, ws))
    b.add(quad((wx, 0, Z), (wx, 0, -Z), (wx, Y - gap, -Z), (wx, Y - gap, Z), 0, ws))
    # light on the ceiling behind the wall, facing down
    ly = Y - 1e-3
    b.add(quad((4.1, ly, -0.25), (4.6, ly, -0.25), (4.6, ly, 0.25), (4.1, ly, 0.25), 2))
    for _ in range(n_boxes):
        size = rng.uniform([0.2, 0.2, 0.2], [1.2, 1.5, 1.2])
        c = (rng.uniform(-X + 0.7, wx - 0.7), size[1] * 0.5 + rng.choice([0.0, rng.uniform(0, 1.5)]),
             rng.uniform(-Z + 0.7, Z - 0.7))
        for part in box(c, size, rng.uniform(0, np.pi), int(rng.choice([1, 3])), box_subdiv):
            b.add(part)
    v, f = b.arrays()
    cam = make_camera(position=(-4.6, 1.7, 4.6), look_at=(1.0, 1.2, -1.0), fov=70.0, width=width, height=height)
    return SceneArrays(f"hidden_light_room_{len(f)}tri", v, f, mats, cam, None, spp=spp, sample_per_frame=4,
                       max_depth=max_depth, sampler=SAMPLER_SOBOL, meta={"triangles": int(len(f))})


# ---------------------------------------------------------------------------
# Combined large case
# ---------------------------------------------------------------------------
def large_scene(n_spheres: int = 3500, subdiv: int = 4, n_tets: int = 500_000, n_lights: int = 32,
                n_cameras: int = 16, width: int = 1920, height: int = 1080, spp: int = 512, max_depth: int = 16,
                seed: int = 13, env_size=(2048, 1024)):
    """About 20M triangles flattened from displaced icospheres (as in
    icosphere_field, spread over a larger field) and random tetrahedral
    clutter, Disney materials as in icosphere_field, the synthetic sky, and
    n_lights small emissive quads; n_cameras views on a ring around the field.
    Returns (SceneArrays, list of cameras)."""
    rng = np.random.default_rng(seed)
    field = icosphere_field(n_spheres=n_spheres, subdiv=subdiv, width=width, height=height, spp=spp,
                            max_depth=max_depth, seed=seed, env_size=env_size)
    # spread the spheres: the field generator places them in a 44 x 35 area
    v = field.vertices.copy()
    f = field.faces.copy()
    mats = list(field.materials)
    # tetrahedral clutter: 4 triangles each, edge 0.05 .. 0.6, on the ground
    c = np.stack([rng.uniform(-60, 60, n_tets), np.zeros(n_tets), rng.uniform(-60, 60, n_tets)], 1)
    size = np.exp(rng.uniform(np.log(0.05), np.log(0.6), n_tets))[:, None]
    corners = rng.normal(size=(n_tets, 4, 3))
    corners /= np.linalg.norm(corners, axis=2, keepdims=True)
    corners[..., 1] = np.abs(corners[..., 1])
    tv = (c[:, None, :] + corners * size[:, :, None]).reshape(-1, 3)
    tt = np.array([[0, 1, 2], [0, 3, 1], [0, 2, 3], [1, 3, 2]])
    ttri = (tt[None] + (np.arange(n_tets) * 4)[:, None, None]).reshape(-1, 3)
    tn = _vertex_normals(tv, ttri)
    n_tm = 64
    for _ in range(n_tm):
        mats.append(default_material(base_color=tuple(rng.uniform(0, 1, 3)), metallic=rng.uniform(0, 1),
                                     roughness=rng.uniform(0.05, 1.0), clearcoat=rng.uniform(0, 1)))
    tmat = np.repeat(len(field.materials) + rng.integers(0, n_tm, n_tets).astype(np.int32), 4)
    # small area lights above the field
    light_mat = len(mats)
    mats.append(default_material(base_color=(1, 1, 1), emissive=(40.0, 36.0, 30.0)))
    b = _Builder()
    b.add((tv.astype(np.float32), tn.astype(np.float32), np.zeros((len(tv), 2), np.float32),
           np.zeros((len(tv), 4), np.float32), ttri, tmat))
    for _ in range(n_lights):
        x, z, y, s = rng.uniform(-40, 40), rng.uniform(-40, 40), rng.uniform(6, 12), rng.uniform(0.2, 0.5)
        b.add(quad((x - s, y, z + s), (x + s, y, z + s), (x + s, y, z - s), (x - s, y, z - s), light_mat))
    cv, cf = b.arrays()
    cf["v0"] += len(v); cf["v1"] += len(v); cf["v2"] += len(v)
    v = np.concatenate([v, cv])
    f = np.concatenate([f, cf])
    mats = _materials(mats)
    cams = []
    for k in range(n_cameras):
        a = 2 * np.pi * k / n_cameras
        cams.append(make_camera(position=(48 * np.cos(a), 6.0 + 4.0 * (k % 3), 48 * np.sin(a)),
                                look_at=(0.0, 1.0, 0.0), fov=45.0, width=width, height=height))
    sa = SceneArrays(f"large_scene_{len(f)}tri", v, f, mats, cams[0], field.env, spp=spp, sample_per_frame=4,
                     max_depth=max_depth, sampler=SAMPLER_SOBOL, meta={"triangles": int(len(f))})
    return sa, cams
