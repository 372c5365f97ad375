"""Textured materials: image decoding, glTF texture loading and textured shading.

CPU (against the reference's own code, compiled from its tree into oracle/_ref):
  * PNG decoding equals the reference's stb_image decode with four channels
    (Part_2/src/io/gltf_loader.cpp:21-39) byte for byte, for every colour type
    and bit depth, tRNS, and Adam7 interlacing; baseline JPEG (4:4:4, 4:2:2,
    4:2:0, grey) within a few levels (decoders round the IDCT and the chroma
    upsampling differently), progressive JPEG rejected;
  * a glTF with embedded (bufferView), data-URI and external images loads to
    the same textures (texels as value / 255, sampler wrap modes) and the same
    materials (texture indices, KHR_texture_transform, normal scale,
    occlusion strength) as the reference's loader (loadTextures and
    loadMaterials, gltf_loader.cpp:112-347).

GPU: a textured Cornell box (base colour with a uv transform, normal map,
metallic-roughness, clearcoat / sheen / transmission maps, alpha MASK and
BLEND panels; REPEAT, CLAMP and MIRROR samplers) rendered by pt_render
against the FP64 oracle on the same sample streams, and against the
reference's own CUDA integrator built for sm_100a
(Part_2/src/materials/disney_bsdf.cuh:79-116, shading_utils.cuh:17-68,
integrators/path.cu:84-158, cuda/cuda_texture.cu:37-62).
"""
import base64
import io
import json
import struct
import zlib

import numpy as np
import pytest

import pathtracingtutorial_b200 as pt
from pathtracingtutorial_b200 import scenes

PIL = pytest.importorskip("PIL.Image")


# ---------------------------------------------------------------------------
# image files
# ---------------------------------------------------------------------------
def _png(img, **kw):
    b = io.BytesIO()
    img.save(b, format="PNG", **kw)
    return b.getvalue()


def _jpeg(img, **kw):
    b = io.BytesIO()
    img.save(b, format="JPEG", **kw)
    return b.getvalue()


def _png_chunk(t, data):
    return struct.pack(">I", len(data)) + t + data + struct.pack(">I", zlib.crc32(t + data) & 0xffffffff)


def _interlaced_png(rgba):
    """An Adam7-interlaced RGBA8 PNG written from the specification (every
    scanline with a filter chosen by its index, so all five are exercised)."""
    h, w = rgba.shape[:2]
    passes = [(0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2)]
    raw = bytearray()
    for x0, y0, dx, dy in passes:
        sub = rgba[y0::dy, x0::dx]
        if sub.size == 0:
            continue
        prev = np.zeros(sub.shape[1] * 4, np.int32)
        for j, row in enumerate(sub.reshape(sub.shape[0], -1).astype(np.int32)):
            f = j % 5
            a = np.concatenate([np.zeros(4, np.int32), row[:-4]])
            c = np.concatenate([np.zeros(4, np.int32), prev[:-4]])
            if f == 0:
                out = row
            elif f == 1:
                out = row - a
            elif f == 2:
                out = row - prev
            elif f == 3:
                out = row - (a + prev) // 2
            else:
                p = a + prev - c
                pa, pb, pc = np.abs(p - a), np.abs(p - prev), np.abs(p - c)
                pred = np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, prev, c))
                out = row - pred
            raw += bytes([f]) + (out & 255).astype(np.uint8).tobytes()
            prev = row
    ihdr = struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 1)
    return (b"\x89PNG\r\n\x1a\n" + _png_chunk(b"IHDR", ihdr) + _png_chunk(b"IDAT", zlib.compress(bytes(raw))) +
            _png_chunk(b"IEND", b""))


def _images():
    rng = np.random.default_rng(12)
    H, W = 21, 34
    rgba = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
    out = {
        "rgba8": _png(PIL.fromarray(rgba, "RGBA")),
        "rgb8": _png(PIL.fromarray(rgba[..., :3], "RGB")),
        "grey8": _png(PIL.fromarray(rgba[..., 0], "L")),
        "grey_alpha8": _png(PIL.fromarray(rgba[..., :2], "LA")),
        "grey1": _png(PIL.fromarray(rgba[..., 0] > 127)),
        "palette4": _png(PIL.fromarray(rgba[..., :3], "RGB").convert("P", palette=PIL.ADAPTIVE, colors=12), bits=4),
        "palette8_trns": _png(PIL.fromarray(rgba, "RGBA").convert("P", palette=PIL.ADAPTIVE, colors=200)),
        "grey16": _png(PIL.fromarray(rgba[..., 0].astype(np.uint16) * 257)),
        "interlaced_rgba8": _interlaced_png(rgba),
    }
    yy, xx = np.mgrid[0:48, 0:72]
    smooth = np.stack([128 + 100 * np.sin(xx / 7.0), 128 + 100 * np.cos(yy / 5.0),
                       128 + 90 * np.sin((xx + yy) / 9.0)], -1).astype(np.uint8)
    jpegs = {
        "jpeg444": _jpeg(PIL.fromarray(smooth, "RGB"), quality=92, subsampling=0),
        "jpeg422": _jpeg(PIL.fromarray(smooth, "RGB"), quality=85, subsampling=1),
        "jpeg420": _jpeg(PIL.fromarray(smooth, "RGB"), quality=80, subsampling=2),
        "jpeg_grey": _jpeg(PIL.fromarray(smooth[..., 1], "L"), quality=90),
    }
    return out, jpegs


def test_png_decoding_equals_reference_decoder(ref):
    pngs, _ = _images()
    for name, data in pngs.items():
        ours = pt.decode_image(data)
        theirs = ref.decode_image(data)
        assert ours.shape == theirs.shape, name
        assert np.array_equal(ours, theirs), (name, np.abs(ours.astype(int) - theirs).max())


def test_jpeg_decoding_close_to_reference_decoder(ref):
    """Within 4 levels of the reference's decoder and of libjpeg (through
    PIL).  The reference's decoder upsamples horizontally subsampled chroma
    (4:2:2) differently in the last two columns (libjpeg and this decoder
    agree there), so those columns are compared with libjpeg only."""
    _, jpegs = _images()
    for name, data in jpegs.items():
        ours = pt.decode_image(data).astype(int)
        theirs = ref.decode_image(data).astype(int)
        libjpeg = np.asarray(PIL.open(io.BytesIO(data)).convert("RGB")).astype(int)
        assert ours.shape == theirs.shape, name
        cols = slice(0, ours.shape[1] - 2) if name == "jpeg422" else slice(None)
        d = np.abs(ours - theirs)[:, cols]
        assert d.max() <= 4 and d.mean() < 0.5, (name, d.max(), d.mean())
        dl = np.abs(ours[..., :3] - libjpeg)
        assert dl.max() <= 4 and dl.mean() < 0.5, (name, dl.max(), dl.mean())
        assert (ours[..., 3] == 255).all()


def test_jpeg_rejections():
    yy, xx = np.mgrid[0:40, 0:56]
    img = np.stack([xx * 4, yy * 6, (xx + yy) * 2], -1).astype(np.uint8)
    with pytest.raises(pt.PTError, match="progressive"):
        pt.decode_image(_jpeg(PIL.fromarray(img, "RGB"), progressive=True))
    with pytest.raises(pt.PTError):
        pt.decode_image(b"GIF89a" + bytes(32))


# ---------------------------------------------------------------------------
# glTF with textures
# ---------------------------------------------------------------------------
def _textured_gltf(tmp_path, kind):
    pngs, jpegs = _images()
    quad_p = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0]], np.float32)
    quad_n = np.tile(np.array([[0, 0, 1]], np.float32), (4, 1))
    quad_uv = np.array([[0, 0], [2, 0], [2, 1.5], [0, 1.5]], np.float32)
    quad_t = np.tile(np.array([[1, 0, 0, 1]], np.float32), (4, 1))
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint16)
    blobs, views = [], []

    def add(data):
        off = sum(len(b) for b in blobs)
        pad = (-off) % 4
        if pad:
            blobs.append(b"\0" * pad)
            off += pad
        blobs.append(data)
        views.append({"buffer": 0, "byteOffset": off, "byteLength": len(data)})
        return len(views) - 1

    acc = []
    for arr, typ, comp in ((quad_p, "VEC3", 5126), (quad_n, "VEC3", 5126), (quad_uv, "VEC2", 5126),
                           (quad_t, "VEC4", 5126), (idx, "SCALAR", 5123)):
        acc.append({"bufferView": add(arr.tobytes()), "componentType": comp, "count": len(arr), "type": typ})
    images = []
    (tmp_path / "external.png").write_bytes(pngs["rgb8"])
    for k, data in enumerate([pngs["rgba8"], jpegs["jpeg420"], pngs["grey_alpha8"], pngs["palette8_trns"]]):
        if kind == "glb" or k == 1:
            images.append({"bufferView": add(data), "mimeType": "image/png" if data[:4] == b"\x89PNG" else "image/jpeg"})
        else:
            images.append({"uri": "data:application/octet-stream;base64," + base64.b64encode(data).decode()})
    images.append({"uri": "external.png"})
    samplers = [{"wrapS": 33071, "wrapT": 33648}, {}]
    textures = [{"source": 0, "sampler": 0}, {"source": 1, "sampler": 1}, {"source": 2}, {"source": 3, "sampler": 0},
                {"source": 4}, {"sampler": 1}]
    materials = [
        {"pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.8, 0.7, 0.75],
                                  "baseColorTexture": {"index": 0, "extensions": {"KHR_texture_transform": {
                                      "offset": [0.25, -0.5], "scale": [2.0, 3.0], "rotation": 0.4}}},
                                  "metallicRoughnessTexture": {"index": 1}, "metallicFactor": 0.3},
         "normalTexture": {"index": 2, "scale": 0.7}, "occlusionTexture": {"index": 3, "strength": 0.5},
         "emissiveTexture": {"index": 4}, "alphaMode": "MASK", "alphaCutoff": 0.3},
        {"pbrMetallicRoughness": {"baseColorTexture": {"index": 3}}, "alphaMode": "BLEND", "doubleSided": True,
         "extensions": {"KHR_materials_clearcoat": {"clearcoatFactor": 0.5, "clearcoatTexture": {"index": 1},
                                                    "clearcoatRoughnessTexture": {"index": 2},
                                                    "clearcoatNormalTexture": {"index": 4}},
                        "KHR_materials_sheen": {"sheenColorFactor": [1, 0.5, 0.2], "sheenColorTexture": {"index": 0},
                                                "sheenRoughnessTexture": {"index": 1}},
                        "KHR_materials_transmission": {"transmissionFactor": 0.4, "transmissionTexture": {"index": 5}}}},
    ]
    prims = [{"attributes": {"POSITION": 0, "NORMAL": 1, "TEXCOORD_0": 2, "TANGENT": 3}, "indices": 4, "material": m}
             for m in (0, 1)]
    doc = {"asset": {"version": "2.0"}, "scene": 0, "scenes": [{"nodes": [0, 1]}],
           "nodes": [{"mesh": 0}, {"mesh": 1, "translation": [0, 0, -1]}],
           "meshes": [{"primitives": [prims[0]]}, {"primitives": [prims[1]]}],
           "accessors": acc, "bufferViews": views, "images": images, "samplers": samplers, "textures": textures,
           "materials": materials}
    binary = b"".join(blobs)
    binary += b"\0" * ((-len(binary)) % 4)
    if kind == "glb":
        doc["buffers"] = [{"byteLength": len(binary)}]
        js = json.dumps(doc).encode()
        js += b" " * ((-len(js)) % 4)
        body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(binary), 0x004E4942) + binary
        path = tmp_path / "textured.glb"
        path.write_bytes(struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body)
    else:
        (tmp_path / "textured.bin").write_bytes(binary)
        doc["buffers"] = [{"byteLength": len(binary), "uri": "textured.bin"}]
        path = tmp_path / "textured.gltf"
        path.write_text(json.dumps(doc))
    return path


@pytest.mark.parametrize("kind", ["glb", "gltf"])
def test_gltf_textures_match_reference_loader(ref, tmp_path, kind):
    path = _textured_gltf(tmp_path, kind)
    s = pt.SceneManager.load(str(path))
    theirs = ref.load_json(str(path))
    ref_tex = ref.loaded_textures()
    assert s.info()["num_textures"] == len(ref_tex) == 6
    for k, rt in enumerate(ref_tex):
        ours = s.texture(k)
        assert (ours["wrap_s"], ours["wrap_t"]) == (rt["wrap_s"], rt["wrap_t"]), k
        assert ours["rgba"].shape == rt["rgba"].shape, k
        if k == 1:   # the JPEG (4:2:0): within a few levels of the reference's decoder
            assert np.abs(ours["rgba"] - rt["rgba"]).max() <= 4.0 / 255.0 + 1e-6
        else:
            assert np.array_equal(ours["rgba"], rt["rgba"]), k
    assert ref_tex[5]["rgba"].size == 0     # a texture without a source image stays empty
    m = s.materials()
    assert np.array_equal(m.view(np.uint8), theirs["materials"].view(np.uint8))
    assert m["base_color_tex"][0] == 0 and m["uv_rotation"][0] == np.float32(0.4)
    assert m["transmission_tex"][1] == 5 and m["clearcoat_normal_tex"][1] == 4


def test_gltf_bad_image_is_an_error(tmp_path):
    path = _textured_gltf(tmp_path, "gltf")
    doc = json.loads(path.read_text())
    doc["images"][0] = {"uri": "data:application/octet-stream;base64," + base64.b64encode(b"not an image").decode()}
    path.write_text(json.dumps(doc))
    with pytest.raises(pt.PTError, match="image 0"):
        pt.SceneManager.load(str(path))


def test_textured_scene_round_trips_through_the_c_abi():
    sa = scenes.textured_cornell(width=16, height=16)
    s = sa.scene()
    assert s.info()["num_textures"] == len(sa.textures) == 4
    for k, t in enumerate(sa.textures):
        got = s.texture(k)
        assert np.array_equal(got["rgba"], t["rgba"]) and got["wrap_s"] == t["wrap_s"]


# ---------------------------------------------------------------------------
# GPU renders
# ---------------------------------------------------------------------------
def _correlated(img, mean):
    img = img[..., :3].astype(np.float64)
    rel = np.abs(img - mean) / np.maximum(np.abs(mean), 1e-3)
    return float(np.median(rel)), float(np.mean((img - mean) ** 2 / (mean ** 2 + 1e-2)))


@pytest.mark.gpu
@pytest.mark.parametrize("sampler", [pt.SAMPLER_PCG, pt.SAMPLER_SOBOL])
def test_textured_render_correlated_with_fp64_oracle(oracle, sampler):
    sa = scenes.textured_cornell(width=96, height=96, spp=16, sampler=sampler)
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    img = pt.render(s, sa.spp)
    prep = oracle.prepare(sa)
    (mean, _), _ = oracle.render(prep, sa.sample_per_frame, sa.max_depth, sa.sampler, frames=sa.spp // 4,
                                 precision=64, rtl=pt.DEVICE_ARG_ORDER, pcg_seed=sa.pcg_seed)
    med, rmse = _correlated(img, mean)
    assert med < 1e-4, med
    assert rmse < 1e-3, rmse
    # the textures matter: the same scene without them renders differently
    plain = scenes.textured_cornell(width=96, height=96, spp=16, sampler=sampler)
    plain.textures = []
    (mean0, _), _ = oracle.render(oracle.prepare(plain), 4, sa.max_depth, sa.sampler, frames=sa.spp // 4,
                                  precision=64, rtl=pt.DEVICE_ARG_ORDER, pcg_seed=sa.pcg_seed)
    assert _correlated(img, mean0)[1] > 20 * rmse


@pytest.mark.gpu
def test_textured_render_correlated_with_reference_gpu_build(oracle):
    from oracle.pyoracle import RefGpu
    if not RefGpu.available():
        pytest.skip("the reference's GPU build (oracle/_ref/libptref_gpu.so) is not built")
    sa = scenes.textured_cornell(width=96, height=96, spp=16, sampler=pt.SAMPLER_SOBOL)
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    img = pt.render(s, sa.spp)
    r = RefGpu(sa)
    try:
        r.reset()
        r.render(sa.spp // sa.sample_per_frame)
        theirs = r.image()
    finally:
        r.close()
    med, rmse = _correlated(img, theirs[..., :3].astype(np.float64))
    assert med < 1e-4, med
    assert rmse < 1e-3, rmse


@pytest.mark.gpu
def test_textured_batch_items_use_wavefront_mode_and_match_render():
    sa = scenes.textured_cornell(width=48, height=40, spp=8)
    s = sa.scene()
    s.build_accel()
    s.upload_to_device(0)
    imgs, _, cfg = pt.render_batch([(s, sa.spp)])
    assert cfg["mode"] == pt.BATCH_WAVEFRONT
    assert np.array_equal(imgs[0], pt.render(s, sa.spp))
    with pytest.raises(pt.PTError, match="wavefront"):
        pt.render_batch([(s, sa.spp)], mode=pt.BATCH_PERSISTENT)


@pytest.mark.gpu
def test_textured_gltf_file_renders_like_the_oracle(oracle, tmp_path):
    """A textured .glb through pt_scene_load_json: the loaded arrays and
    textures, rendered on the GPU, correlate with the FP64 oracle given the
    same arrays."""
    path = _textured_gltf(tmp_path, "glb")
    s = pt.SceneManager.load(str(path))
    cam = pt.make_camera(position=(0.5, 0.5, 2.2), look_at=(0.5, 0.5, 0), fov=60.0, width=48, height=48)
    v, f, m = s.vertices(), s.faces(), s.materials()
    tex = [s.texture(k) for k in range(s.info()["num_textures"])]
    sa = scenes.SceneArrays("textured_glb", v, f, m, cam, scenes.sky_env(64, 32), spp=8, sample_per_frame=4,
                            max_depth=6, sampler=pt.SAMPLER_SOBOL, textures=tex)
    t = sa.scene()
    t.build_accel()
    t.upload_to_device(0)
    img = pt.render(t, sa.spp)
    (mean, _), _ = oracle.render(oracle.prepare(sa), 4, sa.max_depth, sa.sampler, frames=2, precision=64,
                                 rtl=pt.DEVICE_ARG_ORDER)
    med, rmse = _correlated(img, mean)
    assert med < 1e-4, med
    assert rmse < 1e-3, rmse
