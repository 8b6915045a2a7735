// Host texture prep (texture_prep.cpp): data sizes and the BC block encoder.
#pragma once
#include <cstdint>

namespace cn {

// Bytes of a texture's data for its format and size; 0 when invalid (unknown
// format, zero or oversize extent, BC extents not multiples of 4).
uint64_t texture_bytes(uint32_t format, uint32_t width, uint32_t height);
// RGBA8 texels -> BC1 (RGB), BC4 (R), BC5 (R, G) or BC7 (RGBA) blocks; false
// if the format is not a BC format or the size is invalid.
bool texture_encode(uint32_t format, const uint8_t* rgba, uint32_t width, uint32_t height, uint8_t* out);
// One 4x4 block of RGBA8 texels (row-major) -> one 16-byte BC7 block
// (bc7_encode.cpp).
void encode_bc7_block(const uint8_t px[16][4], uint8_t out[16]);
// RGBA float texels -> BC6H unsigned blocks (RGB; alpha is dropped); false
// for another format or an invalid size.
bool texture_encode_float(uint32_t format, const float* rgba, uint32_t width, uint32_t height, uint8_t* out);
// One 4x4 block of RGBA floats (row-major) -> one 16-byte BC6H unsigned
// block (bc6h_encode.cpp).
void encode_bc6h_block(const float px[16][4], uint8_t out[16]);

}  // namespace cn
