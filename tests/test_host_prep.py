"""Host side of the library (no GPU): the C ABI loads and exports every declared
symbol, the structs are layout-identical to the reference's, and host prep
(SAH BVH, light tables, camera frame, scene I/O) equals the reference's
golden vectors bit for bit.  Error paths return status codes."""
import ctypes as C
import json
import os
import re

import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import _ffi, scenes

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
G = np.load(os.path.join(HERE, "golden", "reference_vectors.npz"))


def bits(a):
    return np.ascontiguousarray(a).view(np.uint8)


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "pt_b200.h")).read()
    declared = set(re.findall(r"^\s*(?:int|const char\*)\s+(pt_\w+)\s*\(", header, re.M))
    assert len(declared) >= 40
    lib = C.CDLL(_ffi.LIB_PATH)
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert declared == set(_ffi.EXPORTED), set(_ffi.EXPORTED) ^ declared


def test_struct_layouts_match_reference(ref):
    lay = ref.layout()
    assert lay[0] == 64 and list(lay[1:5]) == [0, 16, 32, 48]                      # Vertex
    assert lay[5] == 16 and lay[6] == 12                                           # TriangleFace
    mat = lay[7:7 + 50]
    ours = [256] + [pt.MATERIAL_DTYPE.fields[k][1] for k in pt.MATERIAL_DTYPE.names]
    assert list(mat) == ours                                                       # Material
    cam = lay[57:66]
    assert list(cam) == [80] + [pt.CAMERA_DTYPE.fields[k][1] for k in pt.CAMERA_DTYPE.names]
    assert lay[66] == 64 and lay[67] == 88                                         # CameraFrame, SceneParams
    pl = lay[68:77]
    assert list(pl) == [112] + [pt.PUNCTUAL_DTYPE.fields[k][1] for k in pt.PUNCTUAL_DTYPE.names]
    assert list(lay[77:80]) == [32, 8, 16]                                         # BVHNode, AliasEntry, EmissiveTriangleRef


def _scene_from_golden(tag, env=None):
    s = pt.SceneManager.from_arrays(G[f"{tag}_vertices"], G[f"{tag}_faces_in"], G[f"{tag}_materials"],
                                    None, env)
    s.build_accel()
    return s


@pytest.mark.parametrize("tag", ["rand", "cornell"])
def test_library_bvh_equals_reference(tag):
    s = _scene_from_golden(tag)
    assert np.array_equal(bits(s.bvh_nodes()), bits(G[f"{tag}_nodes"]))
    assert np.array_equal(bits(s.faces()), bits(G[f"{tag}_faces"]))
    refs, pmf, alias = s.emissive_tables()
    assert np.array_equal(bits(refs), bits(G[f"{tag}_emissive"]))
    assert np.array_equal(bits(pmf), bits(G[f"{tag}_tri_pmf"]))
    assert np.array_equal(bits(alias), bits(G[f"{tag}_tri_alias"]))


def test_library_env_tables_equal_reference():
    s = _scene_from_golden("cornell", G["env_image"])
    pmf, alias = s.env_tables()
    assert np.array_equal(pmf.view(np.uint32), G["env_pmf"].view(np.uint32))
    assert np.array_equal(bits(alias), bits(G["env_alias"]))


def test_library_camera_frames_equal_reference():
    for cam, want in zip(G["cameras"], G["camera_frames"]):
        c = np.frombuffer(cam.tobytes(), pt.CAMERA_DTYPE)[0]
        f = _ffi.CameraFrame()
        _ffi.check(pt.lib().pt_build_camera_frame(_ffi.ptr(np.ascontiguousarray(c)), C.byref(f)))
        assert np.array_equal(np.frombuffer(bytes(f), np.float32).view(np.uint32), want.view(np.uint32))


def test_large_scene_bvh_matches_oracle(oracle):
    """A 2,048,002-triangle scene: the parallel builder equals the oracle's serial restatement."""
    sa = scenes.icosphere_field()
    s = sa.scene()
    s.build_accel()
    nodes, faces, depth = oracle.build_bvh(sa.vertices, sa.faces)
    assert np.array_equal(bits(s.bvh_nodes()), bits(nodes))
    assert np.array_equal(bits(s.faces()), bits(faces))
    assert s.info()["bvh_max_depth"] == depth


def test_traversal_layout_counts():
    s = _scene_from_golden("rand")
    info = s.info()
    assert info["num_inner_nodes"] + info["num_leaves"] == info["num_bvh_nodes"]
    assert info["num_leaves"] == info["num_inner_nodes"] + 1


def _write_scene(tmp_path, obj):
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(obj))
    return str(p)


def test_json_scene_format(tmp_path):
    env = scenes.sky_env(32, 16, sun_peak=50.0, sun_sigma_deg=5.0)
    pt.write_hdr(str(tmp_path / "sky.hdr"), env, flip_y=False)
    obj = {
        "camera": {"position": [0, 1, 5], "lookAt": [0, 0.5, 0], "up": [0, 1, 0], "fov": 50,
                   "aperture": 0.05, "focalDistance": 4.5, "resolution": [320, 200]},
        "render": {"spp": 32, "samplePerFrame": 2, "maxDepth": 6, "sampler": "pcg", "output": "x.hdr"},
        "environment": {"file": "sky.hdr"},
        "materials": {"zeta": {"baseColor": [0.2, 0.3, 0.4]}, "alpha": {"metallic": 1, "roughness": 0.2},
                      "lamp": {"emissive": [1, 1, 1], "emissiveStrength": 10, "doubleSided": True}},
        "lights": [{"type": "point", "position": [0, 3, 0], "intensity": 5},
                   {"type": "spot", "position": [1, 3, 0], "direction": [0, -1, 0], "innerCone": 0.2,
                    "outerCone": 0.5}, {"type": "directional", "direction": [0, -1, 0.2]}],
        "objects": [{"type": "quad", "vertices": [[-1, 0, 1], [1, 0, 1], [1, 0, -1], [-1, 0, -1]], "material": "zeta"},
                    {"type": "quad", "vertices": [[-1, 2, 1], [1, 2, 1], [1, 2, -1], [-1, 2, -1]], "material": "lamp"},
                    {"type": "quad", "vertices": [[-1, 0, -1], [1, 0, -1], [1, 2, -1], [-1, 2, -1]], "material": 1}],
    }
    s = pt.SceneManager.load(_write_scene(tmp_path, obj))
    info = s.info()
    assert info["num_faces"] == 6 and info["num_vertices"] == 12 and info["num_materials"] == 3
    assert info["num_punctual_lights"] == 3 and info["env_width"] == 32 and info["env_height"] == 16
    m = s.materials()
    # materials are indexed in sorted-key order: alpha, lamp, zeta
    assert m[0]["metallic"] == 1.0 and m[1]["double_sided"] == 1 and np.allclose(m[2]["base_color"], [0.2, 0.3, 0.4])
    f = s.faces()
    assert list(f["material_id"]) == [2, 2, 1, 1, 1, 1]
    cam = s.camera
    assert cam["width"] == 320 and cam["height"] == 200 and abs(cam["aperture"] - 0.05) < 1e-7
    st = s.settings()
    assert (st.spp, st.sample_per_frame, st.max_depth, st.sampler_type) == (32, 2, 6, pt.SAMPLER_PCG)
    s.build_accel()
    assert s.info()["num_emissive_triangles"] == 4   # material 1 is "lamp" in sorted order


def test_json_auto_camera_and_default_material(tmp_path):
    obj = {"objects": [{"type": "quad", "vertices": [[-1, 0, 1], [1, 0, 1], [1, 0, -1], [-1, 0, -1]],
                        "material": "missing"}]}
    s = pt.SceneManager.load(_write_scene(tmp_path, obj))
    assert s.info()["num_materials"] == 1
    cam = s.camera
    assert cam["position"][2] > 0 and np.allclose(cam["look_at"], [0, 0, 0])


def test_obj_mesh_object(tmp_path):
    (tmp_path / "tri.obj").write_text("v 0 0 0\nv 1 0 0\nv 0 1 0\nv 1 1 0\nvn 0 0 1\nf 1//1 2//1 3//1\nf 2 4 3\n")
    obj = {"materials": {"m": {}}, "objects": [{"type": "mesh", "file": "tri.obj", "material": "m",
                                                "transform": {"translate": [0, 0, -2], "scale": 2.0}}]}
    s = pt.SceneManager.load(_write_scene(tmp_path, obj))
    v = s.vertices()
    assert s.info()["num_faces"] == 2
    assert np.allclose(v["position"][1], [2, 0, -2])


@pytest.mark.parametrize("text,code", [("{", _ffi.PT_ERR_IO), ('{"objects": [{"type": "gltf", "file": "x.glb"}]}', _ffi.PT_ERR_IO),
                                       ('{"camera": {"position": [0, 1]}}', _ffi.PT_ERR_IO)])
def test_json_errors_return_status(tmp_path, text, code):
    p = tmp_path / "bad.json"
    p.write_text(text)
    with pytest.raises(pt.PTError) as e:
        pt.SceneManager.load(str(p))
    assert e.value.code == code


def test_missing_file_and_bad_arguments(tmp_path):
    with pytest.raises(pt.PTError) as e:
        pt.SceneManager.load(str(tmp_path / "nope.json"))
    assert e.value.code == _ffi.PT_ERR_IO
    sa = scenes.cornell_box(width=8, height=8)
    f = sa.faces.copy()
    f["material_id"][3] = 99
    s = pt.SceneManager.from_arrays(sa.vertices, f, sa.materials, sa.camera)
    with pytest.raises(pt.PTError) as e:
        s.build_accel()
    assert e.value.code == _ffi.PT_ERR_INVALID and "material id" in str(e.value)
    f = sa.faces.copy()
    f["v1"][0] = 10 ** 6
    s = pt.SceneManager.from_arrays(sa.vertices, f, sa.materials, sa.camera)
    with pytest.raises(pt.PTError):
        s.build_accel()
    s = sa.scene()
    with pytest.raises(pt.PTError) as e:
        s.update_settings(sample_per_frame=0)
    assert e.value.code == _ffi.PT_ERR_INVALID
    with pytest.raises(pt.PTError) as e:
        s.upload_to_device(0)   # not built yet
    assert e.value.code == _ffi.PT_ERR_STATE


def test_empty_scene_builds():
    s = pt.SceneManager.from_arrays(np.zeros(0, pt.VERTEX_DTYPE), np.zeros(0, pt.FACE_DTYPE),
                                    np.zeros(0, pt.MATERIAL_DTYPE), pt.make_camera(width=4, height=4))
    s.build_accel()
    assert s.info()["num_bvh_nodes"] == 0


def test_degenerate_coincident_triangles_make_one_leaf(oracle):
    v = np.zeros(3 * 40, pt.VERTEX_DTYPE)
    v["position"][0::3] = (0, 0, 0)
    v["position"][1::3] = (1, 0, 0)
    v["position"][2::3] = (0, 1, 0)
    f = np.zeros(40, pt.FACE_DTYPE)
    f["v0"], f["v1"], f["v2"] = np.arange(0, 120, 3), np.arange(1, 120, 3), np.arange(2, 120, 3)
    s = pt.SceneManager.from_arrays(v, f, pt.default_material()[None], pt.make_camera(width=4, height=4))
    s.build_accel()
    nodes = s.bvh_nodes()
    assert len(nodes) == 1 and nodes[0]["data1"] == 40
    on, of, _ = oracle.build_bvh(v, f)
    assert np.array_equal(bits(on), bits(nodes))


def test_hdr_roundtrip(tmp_path):
    img = np.random.default_rng(0).uniform(0, 100, (8, 12, 4)).astype(np.float32)
    pt.write_hdr(str(tmp_path / "a.hdr"), img, flip_y=False)
    back = pt.read_hdr(str(tmp_path / "a.hdr"))
    # RGBE keeps 8 mantissa bits relative to the pixel's largest channel
    tol = img[..., :3].max(axis=2, keepdims=True) / 128.0
    assert np.all(np.abs(back[..., :3] - img[..., :3]) <= tol)
    # the library's reader decodes the file written here identically
    s = pt.SceneManager.from_arrays(np.zeros(0, pt.VERTEX_DTYPE), np.zeros(0, pt.FACE_DTYPE),
                                    pt.default_material()[None], pt.make_camera(width=4, height=4))
    obj = {"environment": {"file": "a.hdr"}, "materials": {"m": {}}}
    (tmp_path / "s.json").write_text(json.dumps(obj))
    s = pt.SceneManager.load(str(tmp_path / "s.json"))
    assert s.info()["env_width"] == 12 and s.info()["env_height"] == 8


def test_large_scene_generator_small():
    """The combined large case generator at small counts: spheres + clutter +
    light quads flattened into one scene, one camera per view, emissive
    tables hold exactly the light quads' triangles."""
    sa, cams = scenes.large_scene(n_spheres=20, subdiv=2, n_tets=500, n_lights=5, n_cameras=3, width=64,
                                  height=32, env_size=(64, 32))
    assert len(sa.faces) == 20 * 320 + 2 + 500 * 4 + 5 * 2
    assert len(cams) == 3 and all(int(c["width"]) == 64 for c in cams)
    assert int(sa.faces["v0"].max()) < len(sa.vertices) and int(sa.faces["material_id"].max()) < len(sa.materials)
    s = sa.scene()
    s.build_accel()
    info = s.info()
    assert info["num_faces"] == len(sa.faces)
    assert info["num_emissive_triangles"] == 10


def test_tonemap_oracle_known_values():
    """The tone-map restatement at points worked by hand from the preview
    shader (tone_mapping.frag:12-29): black, the linear sRGB segment, c = 1 at
    exposure 0 (1 - 1/e -> sRGB 0.8165 -> 208), saturation."""
    import math
    from oracle.pyoracle import tonemap_ref
    img = np.array([[[0.0, 1e-4, 1.0, 1], [1e9, 1e9, 1e9, 1]]], np.float32)
    out = tonemap_ref(img, 0.0)
    t = 1 - math.exp(-1e-4)
    assert out[0, 0, 0] == 0 and out[0, 0, 1] == round(12.92 * t * 255)
    assert out[0, 0, 2] == round((1.055 * (1 - math.exp(-1.0)) ** (1 / 2.4) - 0.055) * 255) == 208
    assert (out[0, 1, :3] == 255).all() and (out[..., 3] == 255).all()


@pytest.mark.parametrize("shape,flip", [((13, 40), True), ((13, 40), False), ((6, 5), True), ((3, 300), False),
                                        ((2, 129), True)])
def test_hdr_writer_bytes_match_reference_writer(ref, tmp_path, shape, flip):
    """pt_write_hdr against the reference's ImageIO::write (its vendored
    stb_image_write, built from its tree): identical files, for run-length
    coded rows (width >= 8: runs, literal stretches longer than 128, runs
    longer than 127) and flat rows (width < 8), zeros, tiny values and both
    row orders; and the file reads back to the RGBE-quantised image."""
    h, w = shape
    rng = np.random.default_rng(h * 1000 + w)
    img = np.ones((h, w, 4), np.float32)
    img[..., :3] = rng.lognormal(0.0, 2.0, (h, w, 3)).astype(np.float32)
    img[0, : w // 2, :3] = 0.25                        # a run
    img[h - 1, :, :3] = 0.0                            # a zero row
    img[h // 2, : min(w, 4), :3] = 1e-35               # below the RGBE floor
    ours, theirs = tmp_path / "ours.hdr", tmp_path / "ref.hdr"
    pt.write_hdr(str(ours), img, flip_y=flip)
    ref.write_image(str(theirs), img, flip_y=flip)
    assert ours.read_bytes() == theirs.read_bytes()
    back = pt.read_hdr(str(ours))
    if flip:
        back = back[::-1]
    err = np.abs(back[..., :3] - img[..., :3])            # RGBE keeps 8 bits below each pixel's largest channel
    assert np.all(err <= img[..., :3].max(axis=2, keepdims=True) / 128 + 1e-30)
