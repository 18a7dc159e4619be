// DDS container header for block-compressed textures (host code).
//
// The reference's example CLI writes its output with the `ddsfile` crate
// (compressor/src/main.rs:313-353): a DX10-extended DDS header for one 2D
// texture with a DXGI format per variant (:343-353) and straight alpha. This
// writes the same container as the Microsoft DDS specification defines it:
//   "DDS " magic, DDS_HEADER (124 bytes), DDS_HEADER_DXT10 (20 bytes),
// followed by the caller's block data (all mip levels, largest first).
#include <cstdint>
#include <cstring>

#include "../../include/bc_capi.h"

namespace {

void put32(uint8_t* p, uint32_t v) {
    p[0] = (uint8_t)v;
    p[1] = (uint8_t)(v >> 8);
    p[2] = (uint8_t)(v >> 16);
    p[3] = (uint8_t)(v >> 24);
}

// DXGI_FORMAT values (dxgiformat.h).
uint32_t dxgi_format(int variant, int srgb) {
    switch (variant) {
        case BC_VARIANT_BC1: return srgb ? 72u : 71u;   // BC1_UNORM_SRGB / BC1_UNORM
        case BC_VARIANT_BC2: return srgb ? 75u : 74u;   // BC2_UNORM_SRGB / BC2_UNORM
        case BC_VARIANT_BC3: return srgb ? 78u : 77u;   // BC3_UNORM_SRGB / BC3_UNORM
        case BC_VARIANT_BC4: return 80u;                // BC4_UNORM
        case BC_VARIANT_BC5: return 83u;                // BC5_UNORM
        case BC_VARIANT_BC6H: return 95u;               // BC6H_UF16
        case BC_VARIANT_BC7: return srgb ? 99u : 98u;   // BC7_UNORM_SRGB / BC7_UNORM
        default: return 0u;
    }
}

}  // namespace

extern "C" uint32_t bc_dds_dxgi_format(int variant, int srgb) { return dxgi_format(variant, srgb); }

extern "C" int bc_dds_header(int variant, uint32_t width, uint32_t height, uint32_t mip_levels, int srgb,
                             uint8_t* out, size_t out_len) {
    if (!out) return BC_ERR_NULL;
    uint32_t fmt = dxgi_format(variant, srgb);
    if (fmt == 0) return BC_ERR_VARIANT;
    if (width == 0 || height == 0 || mip_levels == 0 || mip_levels > 32) return BC_ERR_DIMS;
    if (out_len < BC_DDS_HEADER_BYTES) return BC_ERR_DST_SIZE;
    std::memset(out, 0, BC_DDS_HEADER_BYTES);
    const uint32_t DDSD_CAPS = 0x1, DDSD_HEIGHT = 0x2, DDSD_WIDTH = 0x4, DDSD_PIXELFORMAT = 0x1000,
                   DDSD_MIPMAPCOUNT = 0x20000, DDSD_LINEARSIZE = 0x80000;
    const uint32_t DDSCAPS_COMPLEX = 0x8, DDSCAPS_TEXTURE = 0x1000, DDSCAPS_MIPMAP = 0x400000;
    const uint32_t bytes_per_block = (variant == BC_VARIANT_BC1 || variant == BC_VARIANT_BC4) ? 8u : 16u;
    const uint64_t top = (uint64_t)((width + 3) / 4) * ((height + 3) / 4) * bytes_per_block;
    std::memcpy(out, "DDS ", 4);
    uint8_t* h = out + 4;
    put32(h + 0, 124);  // dwSize
    put32(h + 4, DDSD_CAPS | DDSD_HEIGHT | DDSD_WIDTH | DDSD_PIXELFORMAT | DDSD_MIPMAPCOUNT | DDSD_LINEARSIZE);
    put32(h + 8, height);
    put32(h + 12, width);
    put32(h + 16, top > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)top);  // dwPitchOrLinearSize: top level bytes
    put32(h + 20, 0);                                                   // dwDepth
    put32(h + 24, mip_levels);                                          // dwMipMapCount
    // dwReserved1[11] stay zero; DDS_PIXELFORMAT at h + 72
    put32(h + 72, 32);          // ddspf.dwSize
    put32(h + 76, 0x4);         // DDPF_FOURCC
    std::memcpy(h + 80, "DX10", 4);
    put32(h + 104, DDSCAPS_TEXTURE | (mip_levels > 1 ? DDSCAPS_COMPLEX | DDSCAPS_MIPMAP : 0u));
    // DDS_HEADER_DXT10 at offset 128
    uint8_t* x = out + 128;
    put32(x + 0, fmt);   // dxgiFormat
    put32(x + 4, 3);     // D3D10_RESOURCE_DIMENSION_TEXTURE2D
    put32(x + 8, 0);     // miscFlag
    put32(x + 12, 1);    // arraySize
    put32(x + 16, 1);    // miscFlags2: DDS_ALPHA_MODE_STRAIGHT
    return BC_OK;
}
