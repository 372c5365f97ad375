// image_decode.h -- PNG and baseline JPEG decoding into 8-bit RGBA, for the
// textures of glTF materials.
//
// The reference decodes glTF images with its vendored stb_image, forcing four
// channels (Part_2/src/io/gltf_loader.cpp:21-39): grey becomes (g, g, g, 255),
// grey + alpha (g, g, g, a), RGB (r, g, b, 255).  These decoders produce the
// same channel layout from their own implementations of the formats' public
// specifications (PNG: W3C / ISO 15948, inflate through zlib; JPEG: ITU-T
// T.81 baseline and extended sequential Huffman, JFIF colour).  PNG output is
// exact; JPEG output follows the specification's IDCT and colour transform,
// which decoders implement with different roundings (a level or two apart).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

namespace ptb {

struct DecodedImage {
    int width = 0, height = 0;
    std::vector<uint8_t> rgba;   // width * height * 4
};

bool decode_png(const uint8_t* data, size_t size, DecodedImage& out, std::string& err);
bool decode_jpeg(const uint8_t* data, size_t size, DecodedImage& out, std::string& err);
// By signature: PNG (89 50 4E 47 ...) or JPEG (FF D8).
bool decode_image(const uint8_t* data, size_t size, DecodedImage& out, std::string& err);

}  // namespace ptb
