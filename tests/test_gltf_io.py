"""glTF 2.0 import against the reference's own loader (GltfSceneLoader through
SceneLoader::load, compiled from the reference tree into oracle/_ref).

A synthetic glTF is written three ways (.gltf with an external .bin, .gltf
with a data: URI, .glb): an interleaved indexed mesh with normals, uvs and
tangents, a non-indexed mesh without normals (normals generated), 8- and
32-bit index primitives, a primitive without a material, node matrices and
TRS with a non-uniform scale, a perspective camera, KHR_lights_punctual
lights, and materials using the metal-rough factors, emissive strength, ior,
transmission, clearcoat, sheen, specular, volume and anisotropy extensions and
the three alpha modes.  Loaded directly (.gltf/.glb path) and as an object of
a JSON scene (with a transform and materialOverrides), every vertex, face,
material, light and the camera must equal the reference's bit for bit.
"""
import base64
import json
import struct

import numpy as np
import pytest

import pathtracingtutorial_b200 as pt


def _mesh_data():
    rng = np.random.default_rng(4)
    # mesh A: 6 vertices, interleaved position/normal/uv/tangent (48-byte stride), u16 indices
    pa = rng.uniform(-1, 1, (6, 3)).astype(np.float32)
    na = rng.normal(size=(6, 3)).astype(np.float32)
    na /= np.linalg.norm(na, axis=1, keepdims=True)
    ua = rng.uniform(0, 1, (6, 2)).astype(np.float32)
    ta = np.concatenate([rng.normal(size=(6, 3)), np.where(rng.uniform(size=(6, 1)) < 0.5, -1.0, 1.0)], 1).astype(np.float32)
    inter = np.concatenate([pa, na, ua, ta], 1).astype(np.float32)    # 12 floats = 48 bytes
    ia = np.array([0, 1, 2, 2, 1, 3, 3, 4, 5, 5, 4, 0], np.uint16)
    # mesh B: 9 vertices, positions only, no indices
    pb = rng.uniform(-2, 2, (9, 3)).astype(np.float32)
    # mesh C: 4 vertices, two primitives with u8 and u32 indices
    pc = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0.5]], np.float32)
    nc = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    i8 = np.array([0, 1, 2], np.uint8)
    i32 = np.array([0, 2, 3], np.uint32)
    return inter, ia, pb, pc, nc, i8, i32


def _gltf(buffer_uri=None):
    inter, ia, pb, pc, nc, i8, i32 = _mesh_data()
    blobs, views = [], []

    def add(arr, stride=None):
        off = sum(len(b) for b in blobs)
        pad = (-off) % 4
        if pad:
            blobs.append(b"\0" * pad)
            off += pad
        data = arr.tobytes()
        blobs.append(data)
        v = {"buffer": 0, "byteOffset": off, "byteLength": len(data)}
        if stride:
            v["byteStride"] = stride
        views.append(v)
        return len(views) - 1

    v_inter = add(inter, 48)
    v_ia = add(ia)
    v_pb = add(pb)
    v_pc = add(pc)
    v_nc = add(nc)
    v_i8 = add(i8)
    v_i32 = add(i32)
    acc = [
        {"bufferView": v_inter, "byteOffset": 0, "componentType": 5126, "count": 6, "type": "VEC3"},    # 0 pos
        {"bufferView": v_inter, "byteOffset": 12, "componentType": 5126, "count": 6, "type": "VEC3"},   # 1 nrm
        {"bufferView": v_inter, "byteOffset": 24, "componentType": 5126, "count": 6, "type": "VEC2"},   # 2 uv
        {"bufferView": v_inter, "byteOffset": 32, "componentType": 5126, "count": 6, "type": "VEC4"},   # 3 tan
        {"bufferView": v_ia, "componentType": 5123, "count": 12, "type": "SCALAR"},                    # 4
        {"bufferView": v_pb, "componentType": 5126, "count": 9, "type": "VEC3"},                       # 5
        {"bufferView": v_pc, "componentType": 5126, "count": 4, "type": "VEC3"},                       # 6
        {"bufferView": v_nc, "componentType": 5126, "count": 4, "type": "VEC3"},                       # 7
        {"bufferView": v_i8, "componentType": 5121, "count": 3, "type": "SCALAR"},                     # 8
        {"bufferView": v_i32, "componentType": 5125, "count": 3, "type": "SCALAR"},                    # 9
    ]
    blob = b"".join(blobs)
    mats = [
        {"name": "full", "pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.2, 0.3, 0.8], "metallicFactor": 0.25,
                                                  "roughnessFactor": 0.4},
         "emissiveFactor": [0.5, 0.25, 0.0], "doubleSided": True,
         "extensions": {"KHR_materials_emissive_strength": {"emissiveStrength": 7.5},
                        "KHR_materials_ior": {"ior": 1.33},
                        "KHR_materials_transmission": {"transmissionFactor": 0.6},
                        "KHR_materials_clearcoat": {"clearcoatFactor": 0.7, "clearcoatRoughnessFactor": 0.15},
                        "KHR_materials_sheen": {"sheenRoughnessFactor": 0.3, "sheenColorFactor": [0.1, 0.2, 0.9]},
                        "KHR_materials_specular": {"specularFactor": 0.45, "specularColorFactor": [0.8, 0.7, 0.6]},
                        "KHR_materials_volume": {"thicknessFactor": 0.02, "attenuationDistance": 3.5,
                                                 "attenuationColor": [0.9, 0.5, 0.4]},
                        "KHR_materials_anisotropy": {"anisotropyStrength": 0.55, "anisotropyRotation": 1.1}}},
        {"name": "masked", "alphaMode": "MASK", "alphaCutoff": 0.35},
        {"name": "blend", "alphaMode": "BLEND", "pbrMetallicRoughness": {"metallicFactor": 0}},
        {"name": "plain"},
    ]
    meshes = [
        {"primitives": [{"attributes": {"POSITION": 0, "NORMAL": 1, "TEXCOORD_0": 2, "TANGENT": 3}, "indices": 4,
                         "material": 0}]},
        {"primitives": [{"attributes": {"POSITION": 5}, "material": 1, "mode": 4}]},
        {"primitives": [{"attributes": {"POSITION": 6, "NORMAL": 7}, "indices": 8, "material": 2},
                        {"attributes": {"POSITION": 6}, "indices": 9},
                        {"attributes": {"POSITION": 6}, "indices": 9, "material": 3, "mode": 1}]},
    ]
    s2 = 0.5 ** 0.5
    nodes = [
        {"name": "root", "translation": [0.5, -1.0, 2.0], "rotation": [0.0, s2, 0.0, s2], "scale": [1.0, 2.0, 0.5],
         "children": [1, 2, 3, 4]},
        {"mesh": 0},
        {"mesh": 1, "matrix": [1, 0, 0, 0, 0, 0, 1, 0, 0, -1, 0, 0, 3, 0.5, -2, 1]},
        {"mesh": 2, "translation": [0, 0, -1], "children": [5, 6]},
        {"camera": 0, "translation": [0, 1, 6], "extensions": {"KHR_lights_punctual": {"light": 0}}},
        {"extensions": {"KHR_lights_punctual": {"light": 1}}, "rotation": [0.3826834, 0, 0, 0.9238795]},
        {"extensions": {"KHR_lights_punctual": {"light": 2}}, "translation": [1, 2, 3]},
    ]
    g = {
        "asset": {"version": "2.0"},
        "scene": 0,
        "scenes": [{"nodes": [0]}],
        "nodes": nodes,
        "meshes": meshes,
        "materials": mats,
        "accessors": acc,
        "bufferViews": views,
        "buffers": [{"byteLength": len(blob)}],
        "cameras": [{"type": "perspective", "perspective": {"yfov": 0.7, "aspectRatio": 1.5, "znear": 0.1}}],
        "extensionsUsed": ["KHR_lights_punctual"],
        "extensions": {"KHR_lights_punctual": {"lights": [
            {"type": "point", "color": [1.0, 0.5, 0.25], "intensity": 20.0, "range": 15.0},
            {"type": "spot", "intensity": 5.0, "spot": {"innerConeAngle": 0.2, "outerConeAngle": 0.6}},
            {"type": "directional", "color": [0.3, 0.3, 1.0], "intensity": 2.0}]}},
    }
    if buffer_uri is not None:
        g["buffers"][0]["uri"] = buffer_uri
    return g, blob


def _write(tmp_path, kind):
    g, blob = _gltf()
    if kind == "bin":
        (tmp_path / "m.bin").write_bytes(blob)
        g["buffers"][0]["uri"] = "m.bin"
        path = tmp_path / "m.gltf"
        path.write_text(json.dumps(g))
    elif kind == "datauri":
        g["buffers"][0]["uri"] = "data:application/octet-stream;base64," + base64.b64encode(blob).decode()
        path = tmp_path / "m.gltf"
        path.write_text(json.dumps(g))
    else:
        js = json.dumps(g).encode()
        js += b" " * ((-len(js)) % 4)
        bb = blob + b"\0" * ((-len(blob)) % 4)
        out = struct.pack("<III", 0x46546C67, 2, 12 + 8 + len(js) + 8 + len(bb))
        out += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(bb), 0x004E4942) + bb
        path = tmp_path / "m.glb"
        path.write_bytes(out)
    return path


def _ours(path):
    s = pt.SceneManager.load(str(path))
    info = s.info()
    return s, {"vertices": s.vertices(), "faces": s.faces(), "materials": s.materials(), "camera": s.camera,
               "n_lights": info["num_punctual_lights"], "lights": s.punctual_lights()}


def _same(ours, ref):
    assert len(ours["vertices"]) == len(ref["vertices"]) > 0
    for k in ("position", "normal", "uv", "tangent"):     # not the padding words (the reference copies
        a = np.ascontiguousarray(ours["vertices"][k])      # a temporary's into them)
        b = np.ascontiguousarray(ref["vertices"][k])
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
    assert np.array_equal(ours["faces"].view(np.uint32), ref["faces"].view(np.uint32))
    rm = ref["materials"].view(pt.MATERIAL_DTYPE)
    assert len(rm) == len(ours["materials"])
    for k in pt.MATERIAL_DTYPE.names:
        if not k.startswith("_"):
            a, b = np.ascontiguousarray(ours["materials"][k]), np.ascontiguousarray(rm[k])
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
    assert ours["n_lights"] == len(ref["lights"]) // 112
    rl = ref["lights"].view(pt.PUNCTUAL_DTYPE)
    for k in ("position", "range", "color", "intensity", "direction", "inner_cone", "outer_cone", "type"):
        a, b = np.ascontiguousarray(ours["lights"][k]), np.ascontiguousarray(rl[k])
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
    rc = ref["camera"].view(pt.CAMERA_DTYPE)[0]
    for k in pt.CAMERA_DTYPE.names:
        if not k.startswith("_"):
            a, b = np.ascontiguousarray(ours["camera"][k]), np.ascontiguousarray(rc[k])
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k


@pytest.mark.parametrize("kind", ["bin", "datauri", "glb"])
def test_gltf_file_matches_reference_loader(ref, tmp_path, kind):
    path = _write(tmp_path, kind)
    _, ours = _ours(path)
    _same(ours, ref.load_json(str(path)))
    assert ours["n_lights"] == 3


def test_gltf_object_in_json_scene_matches_reference_loader(ref, tmp_path):
    _write(tmp_path, "bin")
    scene = {
        "camera": {"position": [0, 1, 8], "lookAt": [0, 0, 0], "up": [0, 1, 0], "fov": 40, "resolution": [64, 48]},
        "materials": {"a": {"baseColor": [0.5, 0.5, 0.5]}, "b": {"emissive": [4, 4, 4]}},
        "objects": [
            {"type": "quad", "vertices": [[-1, 0, -1], [1, 0, -1], [1, 0, 1], [-1, 0, 1]], "material": "a"},
            {"type": "gltf", "file": "m.gltf",
             "transform": {"translate": [1, 2, 3], "rotate": {"axis": [0, 1, 1], "angle": 30}, "scale": 1.5},
             "materialOverrides": {"masked": {"roughness": 0.9, "baseColor": [0.1, 0.9, 0.1]},
                                   "plain": {"emissive": [1, 2, 3], "emissiveStrength": 2.0}}},
        ],
    }
    p = tmp_path / "scene.json"
    p.write_text(json.dumps(scene))
    _, ours = _ours(p)
    r = ref.load_json(str(p))
    _same(ours, r)
    assert ours["n_lights"] == 3       # the glTF's lights; no default lights, no camera from the glTF


def test_gltf_scene_renders_after_device_and_host_builds(tmp_path):
    s = pt.SceneManager.load(str(_write(tmp_path, "glb")))
    s.build_accel()
    assert s.info()["num_faces"] == 4 + 3 + 1 + 1


def test_gltf_with_a_missing_image_file_is_an_error(tmp_path):
    """Textures load (tests/test_textures.py); an image file that is not
    there fails the load with the file named."""
    g, blob = _gltf()
    g["images"] = [{"uri": "x.png"}]
    g["textures"] = [{"source": 0}]
    (tmp_path / "m.bin").write_bytes(blob)
    g["buffers"][0]["uri"] = "m.bin"
    p = tmp_path / "t.gltf"
    p.write_text(json.dumps(g))
    with pytest.raises(pt.PTError, match="x.png"):
        pt.SceneManager.load(str(p))


def _write_big_glb(path, sa):
    """One mesh of the scene's triangles (positions, normals, uvs, u32 indices) as a .glb."""
    v, f = sa.vertices, sa.faces
    pos = np.ascontiguousarray(v["position"], np.float32)
    nrm = np.ascontiguousarray(v["normal"], np.float32)
    uv = np.ascontiguousarray(v["uv"], np.float32)
    idx = np.ascontiguousarray(np.stack([f["v0"], f["v1"], f["v2"]], 1).astype(np.uint32))
    parts = [pos.tobytes(), nrm.tobytes(), uv.tobytes(), idx.tobytes()]
    offs = np.cumsum([0] + [len(p) for p in parts])[:-1]
    views = [{"buffer": 0, "byteOffset": int(o), "byteLength": len(p)} for o, p in zip(offs, parts)]
    acc = [{"bufferView": 0, "componentType": 5126, "count": len(pos), "type": "VEC3"},
           {"bufferView": 1, "componentType": 5126, "count": len(pos), "type": "VEC3"},
           {"bufferView": 2, "componentType": 5126, "count": len(pos), "type": "VEC2"},
           {"bufferView": 3, "componentType": 5125, "count": idx.size, "type": "SCALAR"}]
    blob = b"".join(parts)
    g = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0]}],
         "nodes": [{"mesh": 0, "scale": [1.0, 1.0, 1.0]}],
         "meshes": [{"primitives": [{"attributes": {"POSITION": 0, "NORMAL": 1, "TEXCOORD_0": 2}, "indices": 3,
                                     "material": 0}]}],
         "materials": [{"name": "m", "pbrMetallicRoughness": {"baseColorFactor": [0.7, 0.7, 0.7, 1.0]}}],
         "accessors": acc, "bufferViews": views, "buffers": [{"byteLength": len(blob)}]}
    js = json.dumps(g).encode()
    js += b" " * ((-len(js)) % 4)
    blob += b"\0" * ((-len(blob)) % 4)
    out = struct.pack("<III", 0x46546C67, 2, 12 + 8 + len(js) + 8 + len(blob))
    out += struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(blob), 0x004E4942) + blob
    path.write_bytes(out)


def test_gltf_load_speed_against_reference_loader(ref, tmp_path):
    """A 524,802-triangle .glb (the icosphere field at 100 spheres) loaded by
    both loaders on the host: the same arrays, and one JSON line with the
    wall times (best of two)."""
    import time
    from pathtracingtutorial_b200 import scenes
    sa = scenes.icosphere_field(n_spheres=100, subdiv=4, width=64, height=36, env_size=(16, 8))
    p = tmp_path / "big.glb"
    _write_big_glb(p, sa)
    t_ours, t_ref = [], []
    for _ in range(2):
        t0 = time.perf_counter()
        s = pt.SceneManager.load(str(p))
        t_ours.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        r = ref.load_json(str(p))
        t_ref.append(time.perf_counter() - t0)
    v = s.vertices()
    assert len(s.faces()) == len(sa.faces) and np.array_equal(s.faces().view(np.uint32), r["faces"].view(np.uint32))
    assert np.array_equal(np.ascontiguousarray(v["position"]).view(np.uint32),
                          np.ascontiguousarray(r["vertices"]["position"]).view(np.uint32))
    print(json.dumps({"workload": f"glb of {len(sa.faces)} triangles", "ours_ms": round(min(t_ours) * 1e3, 1),
                      "reference_loader_ms": round(min(t_ref) * 1e3, 1),
                      "speedup": round(min(t_ref) / min(t_ours), 2)}))
