// svf_btf_file.cpp - host parser of the factored BTF files LoadBTF reads
// (src/image/btf.cc:389-1028): the same fields in the same order, the same
// consistency checks, and the light directions derived as LoadBTF derives them
// (SphereToCartesianCoordinates, then CartesianToParabolicCoordinates).  The
// planes are not copied: their byte ranges in the file image are recorded for
// the upload.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>

#include "svf_btf_file.h"
#include "svf_layout.h"

namespace svf
{

namespace
{

// Sequential reader over the file image with bounds checks.
struct Reader
{
    const uint8_t* p;
    size_t size, pos = 0;
    bool ok = true;

    bool take(void* dst, size_t n)
    {
        if(!ok || n > size - pos)
        {
            ok = false;
            return false;
        }
        if(dst)
            std::memcpy(dst, p + pos, n);
        pos += n;
        return true;
    }
    uint32_t u32()
    {
        uint32_t v = 0;
        take(&v, 4);
        return v;
    }
    uint8_t u8()
    {
        uint8_t v = 0;
        take(&v, 1);
        return v;
    }
    float f32()
    {
        float v = 0.0f;
        take(&v, 4);
        return v;
    }
    // skips n bytes; false when they are not there
    bool skip(uint64_t n)
    {
        if(!ok || n > size - pos)
        {
            ok = false;
            return false;
        }
        pos += (size_t)n;
        return true;
    }
};

bool failf(char* err, size_t len, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(err, len, fmt, ap);
    va_end(ap);
    return false;
}

constexpr uint32_t kHeaderBytes = 264;   // BTFCommonHeader (btf.hh:48-57)

} // namespace

bool parse_btf(const uint8_t* data, size_t size, BtfFile& b, char* err, size_t err_len)
{
    b = BtfFile{};
    Reader r{ data, size };
    if(r.u8() != '!' || !r.ok)
        return failf(err, err_len, "unsupported BTF format (no '!' marker)");
    char sig[4];
    if(!r.take(sig, 4))
        return failf(err, err_len, "truncated BTF signature");
    const char* expected;
    if(!std::memcmp(sig, "DFMF", 4))
    {
        b.format = 0;
        expected = "08FC";
    }
    else if(!std::memcmp(sig, "FMF0", 4))
    {
        b.format = 1;
        expected = "6FC";
    }
    else if(!std::memcmp(sig, "FMF1", 4))
    {
        b.format = 2;
        expected = "2FCE";
    }
    else
        return failf(err, err_len, "unsupported BTF signature '%.4s' (DFMF, FMF0 and FMF1 are read)", sig);
    for(const char* e = expected; *e; ++e)
        if(r.u8() != (uint8_t)*e || !r.ok)
            return failf(err, err_len, "invalid BTF signature");

    // read_common (btf.cc:413-657)
    bool rotations = false;
    if(r.pos < size && data[r.pos] == 'R')
    {
        rotations = true;
        ++r.pos;
    }
    const size_t start = r.pos;
    uint32_t header_size = r.u32();
    b.version = r.u32();
    r.skip(kHeaderBytes - 8);
    if(b.version > 1)
        b.cosine_flag = r.u32();
    if(b.version > 2)
        r.skip(r.u32());   // XML string
    if(b.version > 3)
    {
        b.channels = r.u32();
        for(uint32_t c = 0; c < b.channels && r.ok; ++c)
            r.skip(r.u32());   // channel name
    }
    if(!r.ok)
        return failf(err, err_len, "truncated BTF header");
    if(r.pos - start != header_size)
        return failf(err, err_len, "failed to parse BTF header (size %u, read %zu)", header_size, r.pos - start);
    if(b.channels != 3)
        return failf(err, err_len, "%u channels: the decode reads RGB BTFs (3 channels)", b.channels);

    const uint32_t view_count = r.u32();
    std::vector<float> views;
    std::vector<float> lights;
    for(uint32_t v = 0; v < view_count && r.ok; ++v)
    {
        float theta = r.f32(), phi = r.f32();
        float w[3];
        angles_to_cartesian(theta, phi, w);
        views.insert(views.end(), w, w + 3);
        const uint32_t num_lights = r.u32();
        if(b.light_count == 0)
        {
            b.light_count = num_lights;
            if((uint64_t)num_lights * 8 > size - std::min(size, r.pos))
                return failf(err, err_len, "truncated BTF direction table");
            for(uint32_t l = 0; l < num_lights && r.ok; ++l)
            {
                float lt = r.f32(), lp = r.f32();
                angles_to_cartesian(lt, lp, w);
                lights.insert(lights.end(), w, w + 3);
            }
        }
        else if(num_lights == b.light_count)
            r.skip(8ull * b.light_count);
        else
            return failf(err, err_len, "fixed light hemisphere is only allowed");
    }
    b.width = r.u32();
    b.height = r.u32();
    if(rotations)
        r.skip(36ull * r.u32());   // Matrix3 per rotation
    if(!r.ok)
        return failf(err, err_len, "truncated BTF direction table");
    if(b.light_count < 3 || b.light_count > 160)
        return failf(err, err_len, "%u directions (3..160 supported)", b.light_count);
    if(view_count > b.light_count)
        return failf(err, err_len, "%u views for %u lights: non-bidirectional functions are unsupported", view_count,
                     b.light_count);
    // std::equal(views, views + view_count, lights) (btf.cc:631-635)
    if(std::memcmp(views.data(), lights.data(), sizeof(float) * views.size()) != 0)
        for(size_t i = 0; i < views.size(); ++i)
            if(!(views[i] == lights[i]))
                return failf(err, err_len, "non-bidirectional functions are unsupported");
    b.lights_parabolic.resize(2 * (size_t)b.light_count);
    for(uint32_t l = 0; l < b.light_count; ++l)
    {
        const float* w = &lights[3 * l];
        b.lights_parabolic[2 * l] = w[0] / (w[2] + 1.0f);
        b.lights_parabolic[2 * l + 1] = w[1] / (w[2] + 1.0f);
    }
    const uint64_t rows = (uint64_t)b.light_count * b.light_count, cols = (uint64_t)b.width * b.height;
    if(cols == 0)
        return failf(err, err_len, "BTF of %ux%u texels", b.width, b.height);

    if(b.format == 0)
    {
        // DFMF (btf.cc:660-843)
        r.u32();   // num_components (the per-channel counts follow)
        b.color_model = r.u32();
        r.skip(12 + 36);   // ColorMean, ColorTransform
        for(uint32_t c = 0; c < 3 && r.ok; ++c)
        {
            const uint32_t scalar_size = r.u8();
            if(b.data_size == 0)
                b.data_size = scalar_size;
            else if(b.data_size != scalar_size)
                return failf(err, err_len, "different sized channels are not supported");
            const uint32_t K = r.u32();
            const uint32_t num_row = r.u32(), num_column = r.u32();
            if(!r.ok)
                break;
            if(num_row != rows)
                return failf(err, err_len, "invalid BTF row count %u (expected %llu)", num_row,
                             (unsigned long long)rows);
            if(num_column != cols)
                return failf(err, err_len, "invalid BTF column count %u (expected %llu)", num_column,
                             (unsigned long long)cols);
            if(b.data_size != 2 && b.data_size != 4 && b.data_size != 8)
                return failf(err, err_len, "unsupported element size %u", b.data_size);
            if(K == 0)
                return failf(err, err_len, "channel %u has no components", c);
            r.skip((uint64_t)K * b.data_size);   // singular values (already in SxV)
            b.k[c] = K;
            b.u_row[c] = K;
            b.sxv_row[c] = K;
            b.u_off[c] = r.pos;
            b.u_bytes[c] = rows * K * b.data_size;
            r.skip(b.u_bytes[c]);
            b.sxv_off[c] = r.pos;
            b.sxv_bytes[c] = cols * K * b.data_size;
            r.skip(b.sxv_bytes[c]);
        }
        if(!r.ok)
            return failf(err, err_len, "failed to parse BTF file (truncated planes)");
        if(b.color_model != 0 && b.color_model != 11)
            return failf(err, err_len, "unsupported colour model %u", b.color_model);
    }
    else
    {
        // FMF0 / FMF1 (btf.cc:844-957)
        if(b.format == 2)
        {
            const uint32_t hv = r.u8();
            if(hv >= 1)
                b.drr = r.u32();
            if(hv >= 2)
            {
                const uint32_t hw = r.u32(), hh = r.u32();
                if(hw && hh)
                    r.skip(2ull * hw * hh);
            }
            if(hv >= 3)
                return failf(err, err_len, "unsupported BTF header version %u", hv);
        }
        const uint32_t nc0 = r.u32();
        b.data_size = r.u8();
        const uint32_t nc1 = r.u32();
        const uint32_t K = std::max(1u, std::min(nc0, nc1));
        const uint32_t row_count = r.u32(), column_count = r.u32();
        if(!r.ok)
            return failf(err, err_len, "failed to parse BTF file (truncated)");
        if(b.data_size != 2 && b.data_size != 4 && b.data_size != 8)
            return failf(err, err_len, "unsupported element size %u", b.data_size);
        r.skip((uint64_t)K * b.data_size);   // singular values
        if(row_count != rows * 3)
            return failf(err, err_len, "invalid BTF row count %u (expected %llu)", row_count,
                         (unsigned long long)(rows * 3));
        if(column_count != cols)
            return failf(err, err_len, "invalid BTF column count %u (expected %llu)", column_count,
                         (unsigned long long)cols);
        const uint64_t u0 = r.pos, ub = (uint64_t)row_count * K * b.data_size;
        r.skip(ub);
        const uint64_t s0 = r.pos, sb = cols * K * b.data_size;
        r.skip(sb);
        if(!r.ok)
            return failf(err, err_len, "failed to parse BTF file (truncated planes)");
        // U rows interleaved by channel: row lv*3 + c (UElementStride = 3 * DataSize)
        for(uint32_t c = 0; c < 3; ++c)
        {
            b.k[c] = K;
            b.u_off[c] = u0 + (uint64_t)c * K * b.data_size;
            b.u_row[c] = 3ull * K;
            b.u_bytes[c] = ub - (uint64_t)c * K * b.data_size;
            b.sxv_off[c] = s0;
            b.sxv_row[c] = K;
            b.sxv_bytes[c] = sb;
        }
    }
    if(r.pos != size)
        return failf(err, err_len, "additional data that cannot be parsed available (%zu bytes)", size - r.pos);
    return true;
}

} // namespace svf
