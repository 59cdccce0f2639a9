// svf_host_ms.cpp - the pseudo-volume multi-scattering BRDF (svbrdffit -m):
// svf_render_btf_ms, and the LM driver of the SVF_LSQ_MULTI_SCATTERING fit
// (svf_lsq_fit_batch / svf_lsq_fit_sggx), whose kernels are in svf_ms.cu.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/svf.h"
#include "svf_host.h"
#include "svf_internal.h"

using namespace svfh;

namespace svfh
{

// The SVF_LSQ_MULTI_SCATTERING fit of T texels: luminance slices lum
// ([T][stride], device), initial guesses init ([T][7], device); out, rmse and
// stats (device) as svf_lsq_fit_batch returns them.  The reference's
// LevenbergMarquardtCurveFit runs for all texels of a batch in lock step, one
// iteration per round of launches (svf_ms.cu); the host reads, once a round,
// how many texels are still fitting.
svf_status run_ms_fit(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const float* lum, uint64_t stride,
                      uint64_t T, const float* init, float* out, float* rmse, svf_texel_stats* stats)
{
    const uint64_t N = (uint64_t)lay->L * lay->L;
    // a batch's device memory: the 14 perturbed evaluations and the residual of
    // every pair, the LM state and the list; batches of at most 512 MB
    const uint64_t per = N * (14 + 1) * sizeof(float) + sizeof(svf::MsTexel) + sizeof(uint32_t);
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(T, (uint64_t(512) << 20) / per));
    DevBuf st, res, fev, list, counts;
    SVF_TRY(st.ensure(sizeof(svf::MsTexel) * chunk));
    SVF_TRY(res.ensure(sizeof(float) * N * chunk));
    SVF_TRY(fev.ensure(sizeof(float) * N * 14 * chunk));
    SVF_TRY(list.ensure(sizeof(uint32_t) * chunk));
    SVF_TRY(counts.ensure(sizeof(uint32_t) * 4));
    for(uint64_t first = 0; first < T; first += chunk)
    {
        const uint64_t n = std::min(chunk, T - first);
        svf::MsFitArgs a{};
        a.L = lay->L;
        a.geo = lay->geo.as<float>();
        a.bounces = o->multi_scattering_bounces;
        a.texels = n;
        a.lum = lum + first * stride;
        a.lum_stride = stride;
        a.st = st.as<svf::MsTexel>();
        a.res = res.as<float>();
        a.fev = fev.as<float>();
        a.list = list.as<uint32_t>();
        a.counts = counts.as<uint32_t>();
        a.max_iter = o->max_iterations;
        a.mse_target = o->mse_target;
        a.eps = o->break_on_small_step;
        const uint32_t nn = (uint32_t)n;
        // the first residual and Jacobian at the initial guesses, then the damping
        SVF_CUDA(svf::launch_ms_setup(a, init + 7 * first, ctx->stream));
        SVF_CUDA(svf::launch_ms_eval(a, svf::kMsEvalCurrent, nn, nullptr, ctx->stream));
        SVF_CUDA(svf::launch_ms_eval(a, svf::kMsEvalJacobian, nn, nullptr, ctx->stream));
        SVF_CUDA(svf::launch_ms_control(a, svf::kMsStageStart, ctx->stream));
        // every round takes each texel that is not done one LM iteration further,
        // so max_iterations + 1 rounds end every fit
        for(uint64_t round = 0; round <= (uint64_t)o->max_iterations; ++round)
        {
            SVF_CUDA(cudaMemsetAsync(counts.p, 0, sizeof(uint32_t) * 4, ctx->stream));
            SVF_CUDA(svf::launch_ms_control(a, svf::kMsStageStep, ctx->stream));
            uint32_t c[4] = {};
            SVF_CUDA(cudaMemcpyAsync(c, counts.p, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
            SVF_CUDA(cudaStreamSynchronize(ctx->stream));
            if(c[2] == 0)
                break;
            if(c[0] == 0)
                continue;
            SVF_CUDA(svf::launch_ms_eval(a, svf::kMsEvalTrial, c[0], nullptr, ctx->stream));
            SVF_CUDA(svf::launch_ms_control(a, svf::kMsStageGain, ctx->stream));
            // the accepted points (at most c[0]): the kernels read their number
            SVF_CUDA(svf::launch_ms_eval(a, svf::kMsEvalJacobian, c[0], a.counts + 1, ctx->stream));
            SVF_CUDA(svf::launch_ms_control(a, svf::kMsStageDamping, ctx->stream));
        }
        SVF_CUDA(svf::launch_ms_finish(a, init + 7 * first, out + 7 * first, rmse + first,
                                       stats ? stats + first : nullptr, ctx->stream));
    }
    return SVF_OK;
}

} // namespace svfh

extern "C" {

svf_status svf_render_btf_ms(svf_ctx* ctx, const float* lp, uint32_t L, const svf_svbrdf_maps* maps, uint32_t bounces,
                             uint32_t samples, uint32_t seed, uint32_t sample_type, void* samples_out)
{
    SVF_TRY(check_ctx(ctx));
    if(!lp || !maps || !samples_out || !maps->diffuse || !maps->specular || !maps->sigma || !maps->basis)
        return fail(SVF_EINVAL, "null lights/maps/samples");
    if(maps->sigma_channels != 2 && maps->sigma_channels != 3)
        return fail(SVF_EINVAL, "sigma_channels %u (2 or 3)", maps->sigma_channels);
    if(sample_type != SVF_SAMPLES_F32 && sample_type != SVF_SAMPLES_F16)
        return fail(SVF_EINVAL, "unknown sample_type %u", sample_type);
    if(samples == 0 || samples > 65536 || bounces > 1024)
        return fail(SVF_EINVAL, "samples %u (1 to 65536) / bounces %u (at most 1024)", samples, bounces);
    Layout* lay = nullptr;
    SVF_TRY(get_layout(ctx, lp, L, &lay));
    const uint64_t T = (uint64_t)maps->width * maps->height, N = (uint64_t)L * L;
    const uint32_t sc = maps->sigma_channels;
    const size_t texel_bytes = (sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * N;
    bool out_dev = false;
    SVF_TRY(buffer_location(samples_out, "samples", &out_dev));
    const uint64_t chunk = std::max<uint64_t>(1, std::min<uint64_t>(T, (size_t(1) << 28) / texel_bytes));
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
        void* out = out_dev ? static_cast<char*>(samples_out) + c0 * texel_bytes : buf.p;
        svf::MsRenderArgs a{ L, lay->geo.as<float>(), n, d_diff, d_spec, d_sig, d_basis, sc, bounces, samples, seed,
                             sample_type, out };
        SVF_CUDA(svf::launch_ms_render(a, ctx->stream));
        if(!out_dev)
            SVF_CUDA(cudaMemcpyAsync(static_cast<char*>(samples_out) + c0 * texel_bytes, buf.p, texel_bytes * n,
                                     cudaMemcpyDeviceToHost, ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return SVF_OK;
}

} // extern "C"
