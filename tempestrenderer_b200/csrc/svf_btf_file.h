// svf_btf_file.h - the factored BTF file formats LoadBTF reads (DFMF, FMF0,
// FMF1; src/image/btf.cc:389-1028), parsed in place on the host.
#pragma once

#include <stddef.h>
#include <stdint.h>
#include <vector>

namespace svf
{

struct BtfFile
{
    uint32_t format = 0;            // 0 DFMF, 1 FMF0, 2 FMF1
    uint32_t version = 0;           // BTFCommonHeader::Version
    uint32_t width = 0, height = 0, light_count = 0, channels = 3;
    uint32_t data_size = 0;         // 2, 4 or 8 bytes per plane element
    uint32_t color_model = 0;       // DFMF: 0 or 11
    uint32_t drr = 0;               // FMF1: DynamicRangeReduction
    uint32_t cosine_flag = 0;
    std::vector<float> lights_parabolic;   // [L][2]
    // Channel c's planes inside the file: U_c row lv starts at byte
    // u_off[c] + lv * u_row[c] * data_size (k[c] elements), SxV_c row `col` at
    // sxv_off[c] + col * sxv_row[c] * data_size.  u_bytes / sxv_bytes: the
    // plane's extent from u_off / sxv_off (FMF: one shared extent).
    uint32_t k[3] = {};
    uint64_t u_off[3] = {}, sxv_off[3] = {}, u_row[3] = {}, sxv_row[3] = {};
    uint64_t u_bytes[3] = {}, sxv_bytes[3] = {};
};

// Parses a whole file image; false with a message in `err` when LoadBTF would
// reject it, or when it holds what the decode does not support (a channel count
// other than 3, a plane of 0 components, an element size other than 2, 4, 8).
bool parse_btf(const uint8_t* data, size_t size, BtfFile& out, char* err, size_t err_len);

} // namespace svf
