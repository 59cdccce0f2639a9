// svf_exr.cpp - OpenEXR images of the fitted maps, as svbrdffit writes them
// (svbrdf-fitting.cc:713-735 through SaveEXRImage, src/image/exr-image.cc) and
// svbrdf-error-tool reads them (LoadEXRImage).
//
// Written from the OpenEXR file layout (magic 20000630, version 2, a header of
// attributes, a scanline offset table, one uncompressed scanline per chunk):
// FLOAT channels named R, G, B, A (the first 1..4), image row y stored as
// scanline height-1-y with increasing-y line order -- the reference saves the
// maps flipped that way and flips them back on load.  The reader takes what the
// reference writes (uncompressed FLOAT or HALF scanlines, channels R/G/B/A in
// any order) and rejects compressed or tiled files.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/svf.h"

namespace svf
{
svf_status host_fail(svf_status s, const char* fmt, ...);
}

namespace
{

using svf::host_fail;

void put_bytes(std::string& o, const void* p, size_t n) { o.append(static_cast<const char*>(p), n); }
void put_i32(std::string& o, int32_t v) { put_bytes(o, &v, 4); }
void put_f32(std::string& o, float v) { put_bytes(o, &v, 4); }
void put_attr(std::string& o, const char* name, const char* type, const std::string& value)
{
    o += name;
    o += '\0';
    o += type;
    o += '\0';
    put_i32(o, (int32_t)value.size());
    o += value;
}

float half_to_float(uint16_t h)
{
    const uint32_t sign = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1f, m = h & 0x3ff;
    uint32_t bits;
    if(e == 0)
    {
        const float f = (float)m * (1.0f / 16777216.0f);
        return sign ? -f : f;
    }
    if(e == 31)
        bits = sign | 0x7f800000u | (m << 13);
    else
        bits = sign | ((e + 112u) << 23) | (m << 13);
    float f;
    std::memcpy(&f, &bits, 4);
    return f;
}

struct In
{
    const uint8_t* p;
    size_t n, pos = 0;
    bool ok = true;
    bool get(void* d, size_t k)
    {
        if(!ok || k > n - pos)
            return ok = false;
        std::memcpy(d, p + pos, k);
        pos += k;
        return true;
    }
    std::string str()
    {
        std::string s;
        while(ok && pos < n && p[pos])
            s += (char)p[pos++];
        if(pos >= n)
            ok = false;
        else
            ++pos;
        return s;
    }
};

} // namespace

extern "C" {

svf_status svf_exr_write(const char* path, uint32_t width, uint32_t height, uint32_t channels, const float* data)
{
    if(!path || !data || width == 0 || height == 0 || channels < 1 || channels > 4)
        return host_fail(SVF_EINVAL, "svf_exr_write: null path/data, empty image or %u channels (1..4)", channels);
    if(width > (1u << 30) / channels || height > (1u << 30))
        return host_fail(SVF_EINVAL, "svf_exr_write: image too large");
    // channels in the header's alphabetical order, each with its source index
    const char* names = "RGBA";
    std::vector<int> order;
    for(char c : std::string("ABGR"))
        for(uint32_t i = 0; i < channels; ++i)
            if(names[i] == c)
                order.push_back((int)i);
    std::string hdr;
    const uint32_t magic = 20000630u, version = 2u;
    put_bytes(hdr, &magic, 4);
    put_bytes(hdr, &version, 4);
    std::string chlist;
    for(int i : order)
    {
        chlist += names[i];
        chlist += '\0';
        put_i32(chlist, 2);                 // FLOAT
        chlist.append(4, '\0');             // pLinear, reserved
        put_i32(chlist, 1);                 // xSampling
        put_i32(chlist, 1);                 // ySampling
    }
    chlist += '\0';
    put_attr(hdr, "channels", "chlist", chlist);
    put_attr(hdr, "compression", "compression", std::string(1, '\0'));
    std::string box;
    put_i32(box, 0);
    put_i32(box, 0);
    put_i32(box, (int32_t)width - 1);
    put_i32(box, (int32_t)height - 1);
    put_attr(hdr, "dataWindow", "box2i", box);
    put_attr(hdr, "displayWindow", "box2i", box);
    put_attr(hdr, "lineOrder", "lineOrder", std::string(1, '\0'));
    std::string f;
    put_f32(f, 1.0f);
    put_attr(hdr, "pixelAspectRatio", "float", f);
    std::string v2;
    put_f32(v2, 0.0f);
    put_f32(v2, 0.0f);
    put_attr(hdr, "screenWindowCenter", "v2f", v2);
    put_attr(hdr, "screenWindowWidth", "float", f);
    hdr += '\0';

    const uint64_t line_bytes = (uint64_t)width * channels * 4;
    const uint64_t chunk_bytes = 8 + line_bytes;
    std::string table;
    const uint64_t first = hdr.size() + 8ull * height;
    for(uint32_t s = 0; s < height; ++s)
    {
        const uint64_t off = first + s * chunk_bytes;
        put_bytes(table, &off, 8);
    }
    FILE* fp = std::fopen(path, "wb");
    if(!fp)
        return host_fail(SVF_EINVAL, "svf_exr_write: cannot create %s", path);
    bool ok = std::fwrite(hdr.data(), 1, hdr.size(), fp) == hdr.size() &&
              std::fwrite(table.data(), 1, table.size(), fp) == table.size();
    std::vector<float> line((size_t)width * channels);
    for(uint32_t s = 0; s < height && ok; ++s)
    {
        // scanline s holds image row height-1-s
        const float* row = data + (uint64_t)(height - 1 - s) * width * channels;
        size_t k = 0;
        for(int i : order)
            for(uint32_t x = 0; x < width; ++x)
                line[k++] = row[(uint64_t)x * channels + i];
        const int32_t y = (int32_t)s, size = (int32_t)line_bytes;
        ok = std::fwrite(&y, 4, 1, fp) == 1 && std::fwrite(&size, 4, 1, fp) == 1 &&
             std::fwrite(line.data(), 4, line.size(), fp) == line.size();
    }
    ok = (std::fclose(fp) == 0) && ok;
    if(!ok)
        return host_fail(SVF_EINVAL, "svf_exr_write: write to %s failed", path);
    return SVF_OK;
}

svf_status svf_exr_read(const char* path, uint32_t* width, uint32_t* height, uint32_t* channels, float* data,
                        size_t capacity)
{
    if(!path || !width || !height || !channels)
        return host_fail(SVF_EINVAL, "svf_exr_read: null argument");
    FILE* fp = std::fopen(path, "rb");
    if(!fp)
        return host_fail(SVF_EINVAL, "svf_exr_read: cannot open %s", path);
    std::vector<uint8_t> file;
    uint8_t buf[1 << 16];
    size_t got;
    while((got = std::fread(buf, 1, sizeof(buf), fp)) > 0)
        file.insert(file.end(), buf, buf + got);
    std::fclose(fp);
    In r{ file.data(), file.size() };
    uint32_t magic = 0, version = 0;
    r.get(&magic, 4);
    r.get(&version, 4);
    if(!r.ok || magic != 20000630u)
        return host_fail(SVF_EINVAL, "svf_exr_read: %s is not an OpenEXR file", path);
    if((version & 0xff) != 2 || (version & ~0x4ffu) != 0 || (version & 0x200u))
        return host_fail(SVF_EINVAL, "svf_exr_read: %s: only single-part scanline images are read", path);
    struct Chan
    {
        std::string name;
        int32_t type;
    };
    std::vector<Chan> chans;
    int compression = -1, line_order = 0;
    int32_t box[4] = { 0, 0, -1, -1 };
    for(;;)
    {
        std::string name = r.str();
        if(!r.ok)
            return host_fail(SVF_EINVAL, "svf_exr_read: %s: truncated header", path);
        if(name.empty())
            break;
        std::string type = r.str();
        int32_t size = 0;
        r.get(&size, 4);
        if(!r.ok || size < 0 || (size_t)size > r.n - r.pos)
            return host_fail(SVF_EINVAL, "svf_exr_read: %s: truncated header", path);
        In a{ r.p + r.pos, (size_t)size };
        if(name == "channels")
        {
            for(;;)
            {
                std::string cn = a.str();
                if(!a.ok || cn.empty())
                    break;
                int32_t t = 0, xs = 0, ys = 0;
                uint8_t pad[4];
                a.get(&t, 4);
                a.get(pad, 4);
                a.get(&xs, 4);
                a.get(&ys, 4);
                if(xs != 1 || ys != 1)
                    return host_fail(SVF_EINVAL, "svf_exr_read: %s: subsampled channels are not read", path);
                chans.push_back({ cn, t });
            }
        }
        else if(name == "compression" && size >= 1)
            compression = a.p[0];
        else if(name == "dataWindow" && size >= 16)
            std::memcpy(box, a.p, 16);
        else if(name == "lineOrder" && size >= 1)
            line_order = a.p[0];
        r.pos += (size_t)size;
    }
    if(compression != 0)
        return host_fail(SVF_EINVAL, "svf_exr_read: %s: compression %d (only uncompressed files are read)", path,
                         compression);
    const int64_t w = (int64_t)box[2] - box[0] + 1, h = (int64_t)box[3] - box[1] + 1;
    if(w <= 0 || h <= 0 || chans.empty() || chans.size() > 4 || w > (1 << 28) || h > (1 << 28))
        return host_fail(SVF_EINVAL, "svf_exr_read: %s: bad data window or %zu channels", path, chans.size());
    int remap[4];
    for(size_t i = 0; i < chans.size(); ++i)
    {
        const std::string& n = chans[i].name;
        if(n.size() != 1 || !std::strchr("RGBA", n[0]))
            return host_fail(SVF_EINVAL, "svf_exr_read: %s: channel '%s' (R, G, B, A are read)", path, n.c_str());
        remap[i] = (int)(std::strchr("RGBA", n[0]) - "RGBA");
        if(remap[i] >= (int)chans.size())
            return host_fail(SVF_EINVAL, "svf_exr_read: %s: channel %s without the ones before it", path, n.c_str());
        if(chans[i].type != 1 && chans[i].type != 2)
            return host_fail(SVF_EINVAL, "svf_exr_read: %s: pixel type %d (HALF or FLOAT are read)", path,
                             chans[i].type);
    }
    *width = (uint32_t)w;
    *height = (uint32_t)h;
    *channels = (uint32_t)chans.size();
    const uint64_t need = (uint64_t)w * h * chans.size();
    if(!data)
        return SVF_OK;
    if(capacity < need)
        return host_fail(SVF_EINVAL, "svf_exr_read: %s: %llu floats needed, %zu given", path,
                         (unsigned long long)need, capacity);
    std::vector<uint64_t> offsets((size_t)h);
    if(!r.get(offsets.data(), 8 * (size_t)h))
        return host_fail(SVF_EINVAL, "svf_exr_read: %s: truncated offset table", path);
    uint64_t line_bytes = 0;
    for(auto& c : chans)
        line_bytes += (uint64_t)w * (c.type == 1 ? 2 : 4);
    for(int64_t k = 0; k < h; ++k)
    {
        In c{ file.data(), file.size(), (size_t)offsets[(size_t)k] };
        int32_t y = 0, size = 0;
        c.get(&y, 4);
        c.get(&size, 4);
        const int64_t s = (int64_t)y - box[1];
        if(!c.ok || s < 0 || s >= h || (uint64_t)size != line_bytes || line_bytes > c.n - c.pos)
            return host_fail(SVF_EINVAL, "svf_exr_read: %s: bad scanline chunk %lld", path, (long long)k);
        // increasing-y files hold image row h-1-s in scanline s (the reference's flip)
        const int64_t row = line_order == 0 ? h - 1 - s : s;
        const uint8_t* src = c.p + c.pos;
        for(size_t i = 0; i < chans.size(); ++i)
        {
            for(int64_t x = 0; x < w; ++x)
            {
                float v;
                if(chans[i].type == 1)
                {
                    uint16_t hv;
                    std::memcpy(&hv, src + 2 * x, 2);
                    v = half_to_float(hv);
                }
                else
                    std::memcpy(&v, src + 4 * x, 4);
                data[((uint64_t)row * w + x) * chans.size() + remap[i]] = v;
            }
            src += (uint64_t)w * (chans[i].type == 1 ? 2 : 4);
        }
    }
    return SVF_OK;
}

svf_status svf_maps_write_exr(const char* prefix, uint32_t width, uint32_t height, const svf_maps* maps)
{
    if(!prefix || !maps)
        return host_fail(SVF_EINVAL, "svf_maps_write_exr: null prefix/maps");
    struct Item
    {
        const char* suffix;
        const float* data;
        uint32_t channels;
    } items[] = { { "_albedo.exr", maps->diffuse, 3 },   { "_specular.exr", maps->specular, 3 },
                  { "_sggx_scale.exr", maps->sigma, 2 }, { "_sggx_basis.exr", maps->basis, 4 },
                  { "_rmse.exr", maps->rmse, 1 } };
    for(const Item& it : items)
    {
        if(!it.data)
            continue;
        const std::string path = std::string(prefix) + it.suffix;
        const svf_status s = svf_exr_write(path.c_str(), width, height, it.channels, it.data);
        if(s != SVF_OK)
            return s;
    }
    return SVF_OK;
}

} // extern "C"
