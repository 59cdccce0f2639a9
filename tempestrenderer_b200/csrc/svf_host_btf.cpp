// svf_host_btf.cpp - factored BTF files on the device (svf_btf_*: parse, upload,
// decode, fit), the error tool (svf_error_maps), rendering a BTF from maps
// (svf_render_btf, svf_params_from_maps) and the neighbourhood refit.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/svf.h"
#include "svf_host.h"
#include "svf_internal.h"
#include "svf_btf_file.h"
#include "svf_layout.h"

using namespace svfh;

// A factored BTF resident on one device: its planes (DFMF: the three channels'
// U planes back to back, then the SxV planes; FMF: the channel-interleaved U
// and the shared SxV) and the parsed header.
struct svf_btf
{
    int device = 0;
    svf::BtfFile f;
    DevBuf u, sxv;
    const void* u_ptr[3] = {};
    const void* sxv_ptr[3] = {};
};

namespace
{

void btf_info(const svf::BtfFile& f, svf_btf_info* info, float* lp)
{
    if(info)
    {
        *info = svf_btf_info{};
        info->format = f.format;
        info->width = f.width;
        info->height = f.height;
        info->light_count = f.light_count;
        info->data_size = f.data_size;
        info->color_model = f.color_model;
        info->dynamic_range_reduction = f.drr;
        info->cosine_flag = f.cosine_flag;
        info->version = f.version;
        for(int c = 0; c < 3; ++c)
            info->components[c] = f.k[c];
    }
    if(lp)
        std::memcpy(lp, f.lights_parabolic.data(), sizeof(float) * f.lights_parabolic.size());
}

svf::BtfDecodeArgs btf_args(const svf_btf* b, uint64_t first, uint64_t count, uint32_t type, void* out)
{
    svf::BtfDecodeArgs a{};
    for(int c = 0; c < 3; ++c)
    {
        a.u[c] = b->u_ptr[c];
        a.sxv[c] = b->sxv_ptr[c];
        a.k[c] = b->f.k[c];
        a.u_row[c] = b->f.u_row[c];
        a.sxv_row[c] = b->f.sxv_row[c];
    }
    a.data_size = b->f.data_size;
    a.color_model = b->f.color_model;
    a.drr = b->f.drr;
    a.width = b->f.width;
    a.height = b->f.height;
    a.N = b->f.light_count * b->f.light_count;
    a.first = first;
    a.count = count;
    a.out_type = type;
    a.out = out;
    return a;
}

svf_status check_btf(svf_ctx* ctx, const svf_btf* btf)
{
    SVF_TRY(check_ctx(ctx));
    if(!btf)
        return fail(SVF_EINVAL, "null BTF");
    if(btf->device != ctx->device)
        return fail(SVF_EINVAL, "the BTF lives on device %d, the context on %d", btf->device, ctx->device);
    return SVF_OK;
}

} // namespace

extern "C" {

svf_status svf_btf_probe(const void* file, size_t size, svf_btf_info* info, float* lights_parabolic)
{
    if(!file)
        return fail(SVF_EINVAL, "null file image");
    svf::BtfFile f;
    char err[256];
    if(!svf::parse_btf(static_cast<const uint8_t*>(file), size, f, err, sizeof(err)))
        return fail(SVF_EINVAL, "%s", err);
    btf_info(f, info, lights_parabolic);
    return SVF_OK;
}

svf_status svf_btf_load(svf_ctx* ctx, const void* file, size_t size, svf_btf** out)
{
    SVF_TRY(check_ctx(ctx));
    if(!file || !out)
        return fail(SVF_EINVAL, "null file image/output");
    *out = nullptr;
    std::unique_ptr<svf_btf> b(new(std::nothrow) svf_btf);
    if(!b)
        return fail(SVF_ENOMEM, "BTF allocation failed");
    char err[256];
    if(!svf::parse_btf(static_cast<const uint8_t*>(file), size, b->f, err, sizeof(err)))
        return fail(SVF_EINVAL, "%s", err);
    b->device = ctx->device;
    const svf::BtfFile& f = b->f;
    const char* src = static_cast<const char*>(file);
    if(f.format == 0)
    {
        // three plane pairs, each copied to its place in one allocation
        uint64_t ub = 0, sb = 0;
        for(int c = 0; c < 3; ++c)
        {
            ub += round_up(f.u_bytes[c], 256);
            sb += round_up(f.sxv_bytes[c], 256);
        }
        SVF_TRY(b->u.ensure(ub));
        SVF_TRY(b->sxv.ensure(sb));
        uint64_t uo = 0, so = 0;
        for(int c = 0; c < 3; ++c)
        {
            char* ud = b->u.as<char>() + uo;
            char* sd = b->sxv.as<char>() + so;
            SVF_CUDA(cudaMemcpyAsync(ud, src + f.u_off[c], f.u_bytes[c], cudaMemcpyHostToDevice, ctx->stream));
            SVF_CUDA(cudaMemcpyAsync(sd, src + f.sxv_off[c], f.sxv_bytes[c], cudaMemcpyHostToDevice, ctx->stream));
            b->u_ptr[c] = ud;
            b->sxv_ptr[c] = sd;
            uo += round_up(f.u_bytes[c], 256);
            so += round_up(f.sxv_bytes[c], 256);
        }
    }
    else
    {
        SVF_TRY(b->u.ensure(f.u_bytes[0]));
        SVF_TRY(b->sxv.ensure(f.sxv_bytes[0]));
        SVF_CUDA(cudaMemcpyAsync(b->u.p, src + f.u_off[0], f.u_bytes[0], cudaMemcpyHostToDevice, ctx->stream));
        SVF_CUDA(cudaMemcpyAsync(b->sxv.p, src + f.sxv_off[0], f.sxv_bytes[0], cudaMemcpyHostToDevice,
                                 ctx->stream));
        for(int c = 0; c < 3; ++c)
        {
            b->u_ptr[c] = b->u.as<char>() + (f.u_off[c] - f.u_off[0]);
            b->sxv_ptr[c] = b->sxv.p;
        }
    }
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = b.release();
    return SVF_OK;
}

svf_status svf_btf_load_file(svf_ctx* ctx, const char* path, svf_btf** out)
{
    if(!path)
        return fail(SVF_EINVAL, "null path");
    std::ifstream fs(path, std::ios::binary);
    if(!fs)
        return fail(SVF_EINVAL, "failed to open BTF file %s", path);
    std::vector<char> data((std::istreambuf_iterator<char>(fs)), std::istreambuf_iterator<char>());
    if(!fs.good() && !fs.eof())
        return fail(SVF_EINVAL, "failed to read BTF file %s", path);
    return svf_btf_load(ctx, data.data(), data.size(), out);
}

svf_status svf_btf_get_info(const svf_btf* btf, svf_btf_info* info, float* lights_parabolic)
{
    if(!btf)
        return fail(SVF_EINVAL, "null BTF");
    btf_info(btf->f, info, lights_parabolic);
    return SVF_OK;
}

svf_status svf_btf_decode(svf_ctx* ctx, const svf_btf* btf, uint64_t first, uint64_t count, uint32_t sample_type,
                          void* samples)
{
    SVF_TRY(check_btf(ctx, btf));
    const uint64_t T = (uint64_t)btf->f.width * btf->f.height;
    if(!samples || first > T || count > T - first)
        return fail(SVF_EINVAL, "null samples or texels [%llu, %llu) outside the BTF's %llu",
                    (unsigned long long)first, (unsigned long long)(first + count), (unsigned long long)T);
    if(sample_type != SVF_SAMPLES_F32 && sample_type != SVF_SAMPLES_F16)
        return fail(SVF_EINVAL, "unknown sample_type %u", sample_type);
    if(count == 0)
        return SVF_OK;
    const uint64_t N = (uint64_t)btf->f.light_count * btf->f.light_count;
    const size_t texel_bytes = (sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * N;
    bool out_dev = false;
    SVF_TRY(buffer_location(samples, "samples", &out_dev));
    if(out_dev)
    {
        SVF_CUDA(svf::launch_btf_decode(btf_args(btf, first, count, sample_type, samples), ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
        return SVF_OK;
    }
    // host output: decode chunks on the device and copy them out
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(count, (size_t(1) << 30) / texel_bytes));
    DevBuf buf;
    SVF_TRY(buf.ensure(texel_bytes * chunk));
    for(uint64_t c0 = 0; c0 < count; c0 += chunk)
    {
        const uint64_t n = std::min(chunk, count - c0);
        SVF_CUDA(svf::launch_btf_decode(btf_args(btf, first + c0, n, sample_type, buf.p), ctx->stream));
        SVF_CUDA(cudaMemcpyAsync(static_cast<char*>(samples) + c0 * texel_bytes, buf.p, texel_bytes * n,
                                 cudaMemcpyDeviceToHost, ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return SVF_OK;
}

svf_status svf_fit_btf(svf_ctx* ctx, const svf_btf* btf, const svf_layout_desc* mesh, const svf_fit_options* opts,
                       const svf_maps* maps, svf_run_stats* run)
{
    SVF_TRY(check_btf(ctx, btf));
    if(!opts || !maps)
        return fail(SVF_EINVAL, "null options/maps");
    const svf::BtfFile& f = btf->f;
    const uint32_t L = f.light_count;
    svf_layout_desc desc{ f.lights_parabolic.data(), L, nullptr, 0, nullptr, nullptr, 0 };
    if(mesh)
    {
        if(mesh->light_count != L)
            return fail(SVF_EINVAL, "the mesh has %u directions, the BTF %u", mesh->light_count, L);
        desc.triangles = mesh->triangles;
        desc.triangle_count = mesh->triangle_count;
        desc.edges = mesh->edges;
        desc.edge_angles = mesh->edge_angles;
        desc.edge_count = mesh->edge_count;
    }
    const uint64_t T = (uint64_t)f.width * f.height, N = (uint64_t)L * L;
    const size_t texel_bytes = sizeof(float) * 3 * N;
    size_t free_b = 0, total_b = 0;
    SVF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    // the decoded chunk takes a quarter of the free memory; the fit's own
    // buffers grow within the rest
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(T, free_b / 4 / texel_bytes));
    DevBuf& buf = ctx->btf_decoded;   // (kept: a fresh 10 GB buffer per call costs more than the decode)
    SVF_TRY(buf.ensure(texel_bytes * chunk));
    const uint32_t kout = (opts->lsq.flags & SVF_LSQ_RGB) ? 12 : 7;
    svf_run_stats all{};
    bool partial = false;
    for(uint64_t c0 = 0; c0 < T; c0 += chunk)
    {
        const uint64_t n = std::min(chunk, T - c0);
        SVF_CUDA(svf::launch_btf_decode(btf_args(btf, c0, n, SVF_SAMPLES_F32, buf.p), ctx->stream));
        const svf_btf_view v{ buf.p, SVF_SAMPLES_F32, (uint32_t)n, 1, &desc };
        svf_fit_options o = *opts;
        if(o.init_params)
            o.init_params += kout * c0;
        auto off = [&](float* p, uint64_t k) { return p ? p + k * c0 : nullptr; };
        svf_maps m{ off(maps->diffuse, 3), off(maps->specular, 3), off(maps->sigma, 2), off(maps->basis, 4),
                    off(maps->rmse, 1), off(maps->params, kout), off(maps->init, kout),
                    maps->stats ? maps->stats + c0 : nullptr, off(maps->ndf, svf::kNdfTexels) };
        svf_run_stats rs{};
        const svf_status st = svf_fit_texels(ctx, &v, &o, &m, &rs);
        if(st == SVF_EPARTIAL)
            partial = true;
        else if(st != SVF_OK)
            return st;
        all.texels += rs.texels;
        all.iterations += rs.iterations;
        all.jacobians += rs.jacobians;
        all.residuals += rs.residuals;
        all.failed_texels += rs.failed_texels;
        all.ms_total += rs.ms_total;
        all.ms_luminance += rs.ms_luminance;
        all.ms_init += rs.ms_init;
        all.ms_fit += rs.ms_fit;
        all.ms_copy += rs.ms_copy;
        all.ms_ndf += rs.ms_ndf;
        all.lm_threads = rs.lm_threads;
        all.lm_slots = rs.lm_slots;
    }
    if(run)
        *run = all;
    if(partial)
        return fail(SVF_EPARTIAL, "%llu texels did not produce a finite fit", (unsigned long long)all.failed_texels);
    return SVF_OK;
}

svf_status svf_error_maps(svf_ctx* ctx, const svf_btf* btf, const svf_svbrdf_maps* maps, uint32_t x0, uint32_t y0,
                          uint32_t method, uint32_t color, float* rmse, float* psnr)
{
    SVF_TRY(check_btf(ctx, btf));
    if(!maps || !rmse || !psnr || !maps->diffuse || !maps->specular || !maps->sigma || !maps->basis)
        return fail(SVF_EINVAL, "null maps/outputs");
    if(method != SVF_ERROR_PAIRWISE && method != SVF_ERROR_MAX_VIEW)
        return fail(SVF_EINVAL, "unknown method %u", method);
    if(maps->sigma_channels != 2 && maps->sigma_channels != 3)
        return fail(SVF_EINVAL, "sigma_channels %u (2 or 3)", maps->sigma_channels);
    const svf::BtfFile& f = btf->f;
    const uint32_t w = maps->width, h = maps->height;
    if(w == 0 || h == 0 || x0 >= f.width || y0 >= f.height || w > f.width - x0 || h > f.height - y0)
        return fail(SVF_EINVAL, "maps of %ux%u at (%u, %u) outside the %ux%u BTF", w, h, x0, y0, f.width, f.height);
    Layout* lay = nullptr;
    SVF_TRY(get_layout(ctx, f.lights_parabolic.data(), f.light_count, &lay));
    const uint64_t N = (uint64_t)f.light_count * f.light_count;
    const size_t row_bytes = sizeof(float) * 3 * N * f.width;
    size_t free_b = 0, total_b = 0;
    SVF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const uint32_t rows = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(h, free_b / 4 / row_bytes));
    const uint32_t nout = color ? 3 : 1;
    const uint32_t sc = maps->sigma_channels;
    DevBuf samples, md, out;
    SVF_TRY(samples.ensure(row_bytes * rows));
    const uint64_t rt = (uint64_t)rows * w;
    SVF_TRY(md.ensure(sizeof(float) * rt * (3 + 3 + sc + 4)));
    SVF_TRY(out.ensure(sizeof(float) * rt * 2 * nout));
    float* d_diff = md.as<float>();
    float* d_spec = d_diff + 3 * rt;
    float* d_sig = d_spec + 3 * rt;
    float* d_basis = d_sig + sc * rt;
    float* d_rmse = out.as<float>();
    float* d_psnr = d_rmse + nout * rt;
    for(uint32_t r0 = 0; r0 < h; r0 += rows)
    {
        const uint32_t nr = std::min(rows, h - r0);
        const uint64_t n = (uint64_t)nr * w, m0 = (uint64_t)r0 * w;
        SVF_CUDA(svf::launch_btf_decode(btf_args(btf, (uint64_t)(y0 + r0) * f.width, (uint64_t)nr * f.width,
                                                 SVF_SAMPLES_F32, samples.p),
                                        ctx->stream));
        SVF_TRY(to_device(ctx, d_diff, maps->diffuse + 3 * m0, sizeof(float) * 3 * n));
        SVF_TRY(to_device(ctx, d_spec, maps->specular + 3 * m0, sizeof(float) * 3 * n));
        SVF_TRY(to_device(ctx, d_sig, maps->sigma + sc * m0, sizeof(float) * sc * n));
        SVF_TRY(to_device(ctx, d_basis, maps->basis + 4 * m0, sizeof(float) * 4 * n));
        svf::ErrorArgs a{};
        a.samples = samples.p;
        a.sample_type = SVF_SAMPLES_F32;
        a.L = f.light_count;
        a.N = (uint32_t)N;
        a.geo = lay->geo.as<float>();
        a.count = n;
        a.region_w = w;
        a.row_texels = f.width;
        a.x0 = x0;
        a.diffuse = d_diff;
        a.specular = d_spec;
        a.sigma = d_sig;
        a.basis = d_basis;
        a.sigma_channels = sc;
        a.method = method;
        a.color = color ? 1u : 0u;
        a.rmse = d_rmse;
        a.psnr = d_psnr;
        SVF_CUDA(svf::launch_error(a, ctx->stream));
        SVF_CUDA(cudaMemcpyAsync(rmse + nout * m0, d_rmse, sizeof(float) * nout * n, cudaMemcpyDefault, ctx->stream));
        SVF_CUDA(cudaMemcpyAsync(psnr + nout * m0, d_psnr, sizeof(float) * nout * n, cudaMemcpyDefault, ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return SVF_OK;
}

svf_status svf_render_btf(svf_ctx* ctx, const float* lp, uint32_t L, const svf_svbrdf_maps* maps, float fresnel,
                          uint32_t sample_type, void* samples)
{
    SVF_TRY(check_ctx(ctx));
    if(!lp || !maps || !samples || !maps->diffuse || !maps->specular || !maps->sigma || !maps->basis)
        return fail(SVF_EINVAL, "null lights/maps/samples");
    if(maps->sigma_channels != 2 && maps->sigma_channels != 3)
        return fail(SVF_EINVAL, "sigma_channels %u (2 or 3)", maps->sigma_channels);
    if(sample_type != SVF_SAMPLES_F32 && sample_type != SVF_SAMPLES_F16)
        return fail(SVF_EINVAL, "unknown sample_type %u", sample_type);
    if(!(fresnel >= 1.0f))
        return fail(SVF_EINVAL, "refractive index %g (>= 1)", fresnel);
    Layout* lay = nullptr;
    SVF_TRY(get_layout(ctx, lp, L, &lay));
    const uint64_t T = (uint64_t)maps->width * maps->height, N = (uint64_t)L * L;
    const uint32_t sc = maps->sigma_channels;
    const size_t texel_bytes = (sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * N;
    bool out_dev = false;
    SVF_TRY(buffer_location(samples, "samples", &out_dev));
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(T, (size_t(1) << 30) / texel_bytes));
    DevBuf md, buf;
    SVF_TRY(md.ensure(sizeof(float) * chunk * (3 + 3 + sc + 4)));
    if(!out_dev)
        SVF_TRY(buf.ensure(texel_bytes * chunk));
    float* d_diff = md.as<float>();
    float* d_spec = d_diff + 3 * chunk;
    float* d_sig = d_spec + 3 * chunk;
    float* d_basis = d_sig + sc * chunk;
    for(uint64_t c0 = 0; c0 < T; c0 += chunk)
    {
        const uint64_t n = std::min(chunk, T - c0);
        SVF_TRY(to_device(ctx, d_diff, maps->diffuse + 3 * c0, sizeof(float) * 3 * n));
        SVF_TRY(to_device(ctx, d_spec, maps->specular + 3 * c0, sizeof(float) * 3 * n));
        SVF_TRY(to_device(ctx, d_sig, maps->sigma + sc * c0, sizeof(float) * sc * n));
        SVF_TRY(to_device(ctx, d_basis, maps->basis + 4 * c0, sizeof(float) * 4 * n));
        void* out = out_dev ? static_cast<char*>(samples) + c0 * texel_bytes : buf.p;
        svf::RenderArgs a{ L, lay->geo.as<float>(), n, d_diff, d_spec, d_sig, d_basis, sc, fresnel, sample_type, out };
        SVF_CUDA(svf::launch_render(a, ctx->stream));
        if(!out_dev)
            SVF_CUDA(cudaMemcpyAsync(static_cast<char*>(samples) + c0 * texel_bytes, buf.p, texel_bytes * n,
                                     cudaMemcpyDeviceToHost, ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return SVF_OK;
}

svf_status svf_params_from_maps(const svf_svbrdf_maps* maps, float* params, float* colour)
{
    if(!maps || !params || !maps->diffuse || !maps->specular || !maps->sigma || !maps->basis)
        return fail(SVF_EINVAL, "null maps/params");
    if(maps->sigma_channels != 2 && maps->sigma_channels != 3)
        return fail(SVF_EINVAL, "sigma_channels %u (2 or 3)", maps->sigma_channels);
    const uint64_t T = (uint64_t)maps->width * maps->height;
    const uint32_t sc = maps->sigma_channels;
    for(uint64_t t = 0; t < T; ++t)
    {
        const float* d = maps->diffuse + 3 * t;
        const float* sp = maps->specular + 3 * t;
        const float* sg = maps->sigma + sc * t;
        float* p = params + 7 * t;
        // RGBToLuminance (spectrum.hh:328-331)
        const float kd = 0.2126f * d[0] + 0.7152f * d[1] + 0.0722f * d[2];
        const float ks = 0.2126f * sp[0] + 0.7152f * sp[1] + 0.0722f * sp[2];
        p[0] = sc == 3 ? sg[0] / sg[2] : sg[0];
        p[1] = sc == 3 ? sg[1] / sg[2] : sg[1];
        p[2] = ks;
        p[3] = kd;
        svf::quaternion_to_euler(maps->basis + 4 * t, p + 4);
        if(colour)
            for(int c = 0; c < 3; ++c)
                colour[3 * t + c] = sp[c] / ks;   // avg_spec = Specular / specular (pipeline.cc:669)
    }
    return SVF_OK;
}

svf_status svf_refit_neighborhood(svf_ctx* ctx, const svf_btf_view* btf, const svf_lsq_options* lsq,
                                  const float* params_in, const float* rmse_in, const svf_maps* out,
                                  svf_run_stats* run)
{
    SVF_TRY(check_ctx(ctx));
    if(!btf || !btf->samples || !btf->layout || !params_in || !rmse_in || !out)
        return fail(SVF_EINVAL, "null btf/params/rmse/outputs");
    svf_lsq_options o;
    svf_lsq_options_default(&o);
    if(lsq)
        o = *lsq;
    SVF_TRY(check_options(&o));
    if(o.flags & SVF_LSQ_RGB)
        return fail(SVF_EINVAL, "the neighbourhood refit fits the luminance model (no SVF_LSQ_RGB)");
    if(btf->sample_type != SVF_SAMPLES_F32 && btf->sample_type != SVF_SAMPLES_F16)
        return fail(SVF_EINVAL, "unknown sample_type %u", btf->sample_type);
    const svf_layout_desc* desc = btf->layout;
    Layout* lay = nullptr;
    SVF_TRY(get_layout(ctx, desc->lights_parabolic, desc->light_count, &lay));
    const uint32_t L = lay->L, N = L * L, W = btf->width, H = btf->height;
    const uint64_t T = (uint64_t)W * H, stride = round_up(N, 8);
    if(T == 0)
        return SVF_OK;
    const size_t texel_bytes = (btf->sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * (size_t)N;
    bool on_device = false;
    SVF_TRY(buffer_location(btf->samples, "samples", &on_device));
    size_t free_b = 0, total_b = 0;
    SVF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per_texel = sizeof(float) * (stride + 3 + 9 * (7 + 7 + 1) + 7 + 1 + 12) + 9 * sizeof(svf_texel_stats) +
                             (on_device ? 0 : texel_bytes);
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>({ T, (free_b / 2) / per_texel, 1ull << 22 }));
    DevBuf all, cand, stage;
    SVF_TRY(all.ensure(sizeof(float) * 8 * T));
    float* d_params = all.as<float>();
    float* d_rmse = d_params + 7 * T;
    SVF_TRY(to_device(ctx, d_params, params_in, sizeof(float) * 7 * T));
    SVF_TRY(to_device(ctx, d_rmse, rmse_in, sizeof(float) * T));
    SVF_TRY(ctx->lum.ensure(sizeof(float) * stride * chunk));
    SVF_TRY(ctx->avg.ensure(sizeof(float) * 3 * chunk));
    SVF_TRY(cand.ensure(sizeof(float) * 9 * chunk * 15 + sizeof(svf_texel_stats) * 9 * chunk));
    float* c_init = cand.as<float>();
    float* c_out = c_init + 63 * chunk;
    float* c_rmse = c_out + 63 * chunk;
    svf_texel_stats* c_stats = reinterpret_cast<svf_texel_stats*>(c_rmse + 9 * chunk);
    SVF_TRY(ctx->maps_buf.ensure(sizeof(float) * (12 + 7 + 1 + 1) * chunk));
    float* mb = ctx->maps_buf.as<float>();
    float* sel_params = mb + 12 * chunk;
    float* sel_rmse = sel_params + 7 * chunk;
    float* dummy_rmse = sel_rmse + chunk;
    if(!on_device)
        SVF_TRY(stage.ensure(texel_bytes * chunk));
    svf_run_stats all_stats{};
    std::vector<svf_texel_stats> hs;
    SVF_TRY(zero_error_flags(ctx));
    for(uint64_t c0 = 0; c0 < T; c0 += chunk)
    {
        const uint64_t n = std::min(chunk, T - c0);
        const void* samples = static_cast<const char*>(btf->samples) + c0 * texel_bytes;
        if(!on_device)
        {
            SVF_CUDA(cudaMemcpyAsync(stage.p, samples, texel_bytes * n, cudaMemcpyHostToDevice, ctx->stream));
            samples = stage.p;
        }
        SVF_CUDA(svf::launch_luminance(samples, btf->sample_type, n, N, ctx->lum.as<float>(), stride,
                                       ctx->avg.as<float>(), nullptr, nullptr, nullptr, ctx->stream));
        SVF_CUDA(svf::launch_refit_gather(d_params, c0, n, W, H, c_init, ctx->stream));
        // nine candidate fits per texel in one launch: segment k holds candidate k
        // of every texel, all reading the texels' own slabs
        svf::LmSegment seg[9];
        for(int k = 0; k < 9; ++k)
            seg[k] = svf::LmSegment{ (uint32_t)(k * n), L, stride, ctx->lum.as<float>(), lay->geo.as<float>() };
        if(9 * n > 0xffffffffull)
            return fail(SVF_EINVAL, "internal: refit chunk too large");
        LmRun r{ nullptr, stride, c_init, c_out, c_rmse, c_stats, nullptr, nullptr, nullptr, nullptr, nullptr, 9 * n,
                 seg, 9, lay->all_up, false };
        SVF_TRY(run_lm(ctx, lay, &o, r));
        SVF_CUDA(svf::launch_refit_select(d_params, d_rmse, c0, n, W, H, c_out, c_rmse, sel_params, sel_rmse, nullptr,
                                          ctx->stream));
        // the maps of the selected parameters (a pass without iterations)
        svf_lsq_options o0 = o;
        o0.max_iterations = 0;
        o0.restarts = 0;
        LmRun m{ ctx->lum.as<float>(), stride, sel_params, sel_params, dummy_rmse, nullptr,
                 ctx->avg.as<float>(), mb, mb + 3 * n, mb + 6 * n, mb + 8 * n, n };
        // out == init is safe: each texel reads its parameters before writing them
        SVF_TRY(launch_lm(ctx, lay, &o0, m, lm_choice(lay, stride, false)));
        auto put = [&](void* dst, const void* src, size_t bytes) -> svf_status {
            if(dst)
                SVF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
            return SVF_OK;
        };
        SVF_TRY(put(out->params ? out->params + 7 * c0 : nullptr, sel_params, sizeof(float) * 7 * n));
        SVF_TRY(put(out->rmse ? out->rmse + c0 : nullptr, sel_rmse, sizeof(float) * n));
        SVF_TRY(put(out->diffuse ? out->diffuse + 3 * c0 : nullptr, mb, sizeof(float) * 3 * n));
        SVF_TRY(put(out->specular ? out->specular + 3 * c0 : nullptr, mb + 3 * n, sizeof(float) * 3 * n));
        SVF_TRY(put(out->sigma ? out->sigma + 2 * c0 : nullptr, mb + 6 * n, sizeof(float) * 2 * n));
        SVF_TRY(put(out->basis ? out->basis + 4 * c0 : nullptr, mb + 8 * n, sizeof(float) * 4 * n));
        hs.resize(9 * n);
        SVF_CUDA(cudaMemcpyAsync(hs.data(), c_stats, sizeof(svf_texel_stats) * 9 * n, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
        all_stats.texels += n;
        for(const auto& st : hs)
        {
            all_stats.iterations += st.iterations;
            all_stats.jacobians += st.jacobians;
            all_stats.residuals += st.residuals;
        }
    }
    SVF_TRY(read_error_flag(ctx));
    if(run)
        *run = all_stats;
    return SVF_OK;
}

void svf_btf_destroy(svf_btf* btf)
{
    if(!btf)
        return;
    cudaSetDevice(btf->device);
    cudaDeviceSynchronize();
    delete btf;
}

} // extern "C"
