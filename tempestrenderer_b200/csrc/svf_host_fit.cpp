// svf_host_fit.cpp - the fit pipeline of svf_fit_texels (one BTF) and
// svf_fit_btfs (several in one persistent LM launch), and svf_synth_btf.
//   luminance_kernel     samples -> luminance slices [T][Kp] + average chromaticity
//   ndf_tc_kernel        NDF rows = slices x NDF operator^T, tcgen05 (default init)
//   init_finish_kernel   NDF -> initial parameters                  (default init)
//   lm_fit_kernel        persistent LM over all texels + output maps
// Host buffers are staged in chunks through the device.
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

extern "C" {

svf_status svf_fit_texels(svf_ctx* ctx, const svf_btf_view* btf, const svf_fit_options* opts, const svf_maps* maps,
                          svf_run_stats* run)
{
    SVF_TRY(check_ctx(ctx));
    if(!btf || !opts || !maps || !btf->layout || !btf->samples)
        return fail(SVF_EINVAL, "null btf/options/maps/layout/samples");
    SVF_TRY(check_options(&opts->lsq));
    if(btf->sample_type != SVF_SAMPLES_F32 && btf->sample_type != SVF_SAMPLES_F16)
        return fail(SVF_EINVAL, "unknown sample_type %u", btf->sample_type);
    if(opts->init_mode != SVF_INIT_DEFAULT && opts->init_mode != SVF_INIT_GIVEN && opts->init_mode != SVF_INIT_MLP)
        return fail(SVF_EINVAL, "unknown init_mode %u", opts->init_mode);
    if(opts->init_mode == SVF_INIT_MLP && !opts->mlp)
        return fail(SVF_EINVAL, "SVF_INIT_MLP needs a model (svf_fit_options::mlp)");
    if(opts->init_mode == SVF_INIT_GIVEN && !opts->init_params)
        return fail(SVF_EINVAL, "SVF_INIT_GIVEN needs init_params");
    const uint64_t T = (uint64_t)btf->width * btf->height;
    if(T == 0)
        return SVF_OK;
    if(T > 0xffffffffull)
        return fail(SVF_EINVAL, "too many texels");
    const svf_layout_desc* desc = btf->layout;
    Layout* lay = nullptr;
    SVF_TRY(get_layout(ctx, desc->lights_parabolic, desc->light_count, &lay));
    const uint32_t L = lay->L, N = L * L;
    const uint64_t stride = round_up(N, 8);
    const svf::InitLayout* init_lay = nullptr;
    if(opts->init_mode == SVF_INIT_DEFAULT)
        SVF_TRY(prepare_init(ctx, lay, desc, &init_lay));
    const svf_mlp* mlp = opts->init_mode == SVF_INIT_MLP ? opts->mlp : nullptr;
    if(mlp && (mlp->L != L || std::memcmp(mlp->lp.data(), lay->lp.data(), sizeof(float) * 2 * L) != 0))
        return fail(SVF_EINVAL, "the model was trained for another direction layout");
    if(mlp && mlp->device != ctx->device)
        return fail(SVF_EINVAL, "the model lives on device %d, the context on %d", mlp->device, ctx->device);

    const size_t elem = btf->sample_type == SVF_SAMPLES_F16 ? 2 : 4;
    const size_t texel_bytes = elem * 3 * (size_t)N;
    bool samples_on_device = false;
    SVF_TRY(buffer_location(btf->samples, "samples", &samples_on_device));
    const bool default_init = opts->init_mode == SVF_INIT_DEFAULT;
    if(maps->ndf && !default_init)
        return fail(SVF_EINVAL, "the NDF map exists only with the default initial guess");
    const uint32_t ndf_ld = default_init ? init_lay->ndf_rows_pad : 0;
    // the RGB fit: FP16 RGB slabs, 12 floats of parameters per texel
    const bool rgb = (opts->lsq.flags & SVF_LSQ_RGB) != 0;
    const uint64_t stride3 = round_up(3ull * N, 8);
    const uint64_t kout = rgb ? 12 : 7;
    // the learned guess's fallback to the default guess (selected texels only)
    const bool fallback = mlp && opts->mlp_fallback > 0.0f;
    if(opts->mlp_fallback != 0.0f && (!mlp || rgb || !(opts->mlp_fallback > 0.0f)))
        return fail(SVF_EINVAL, "mlp_fallback needs SVF_INIT_MLP, the luminance fit and a positive threshold");
    if(fallback)
        SVF_TRY(prepare_init(ctx, lay, desc, &init_lay));
    const uint32_t fb_ld = fallback ? init_lay->ndf_rows_pad : 0;

    // Chunking.  Device-resident samples: as few chunks as the device memory
    // allows.  Host samples: a pipeline of chunks, each copied host -> device on
    // the copy stream into one of two staging buffers while the compute stream
    // fits the previous chunk; a staging buffer is free again once the
    // luminance kernel has read it.
    size_t free_b = 0, total_b = 0;
    SVF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t per_texel = sizeof(float) * (stride + 3 + 2 * kout + 7 + 1 + 12) + (rgb ? 2 * stride3 : 0) +
                             (mlp ? sizeof(float) * (svf::kMlpInputs + 2 * svf::kMlpHidden + svf::kMlpOutputs) : 0) +
                             (default_init ? 2 * 2 * stride + sizeof(float) * ndf_ld : 0) +
                             (fallback ? sizeof(float) * (stride + fb_ld + 3 + 7 + 7 + 1 + 12 + 1) + 2 * 2 * stride +
                                             sizeof(svf_texel_stats)
                                       : 0) +
                             (maps->ndf ? sizeof(float) * svf::kNdfTexels : 0) +
                             (samples_on_device ? 0 : 2 * texel_bytes);
    uint64_t chunk = std::max<uint64_t>(1, (uint64_t)(0.5 * (double)free_b / (double)per_texel));
    if(!samples_on_device)
        chunk = std::min<uint64_t>(chunk, std::max<uint64_t>(8192, (T + 7) / 8));
    chunk = std::min<uint64_t>(chunk, T);
    chunk = std::min<uint64_t>(chunk, 65535ull * 128);   // the NDF GEMM's grid rows of 128 texels
    const uint64_t n_chunks = (T + chunk - 1) / chunk;

    SVF_TRY(ctx->lum.ensure(sizeof(float) * stride * chunk));
    SVF_TRY(ctx->avg.ensure(sizeof(float) * 3 * chunk));
    SVF_TRY(ctx->init.ensure(sizeof(float) * 7 * chunk));
    SVF_TRY(ctx->out.ensure(sizeof(float) * kout * chunk));
    if(rgb)
    {
        SVF_TRY(ctx->rgb16.ensure(2 * stride3 * chunk));
        SVF_TRY(ctx->init_rgb.ensure(sizeof(float) * 12 * chunk));
    }
    SVF_TRY(ctx->rmse.ensure(sizeof(float) * chunk));
    SVF_TRY(ctx->stats.ensure(sizeof(svf_texel_stats) * T));
    SVF_TRY(ctx->maps_buf.ensure(sizeof(float) * 12 * chunk));
    if(default_init)
    {
        SVF_TRY(ctx->lum_hi.ensure(2 * stride * chunk));
        SVF_TRY(ctx->lum_lo.ensure(2 * stride * chunk));
        SVF_TRY(ctx->ndf.ensure(sizeof(float) * ndf_ld * chunk));
    }
    if(maps->ndf)
        SVF_TRY(ctx->ndf_tex.ensure(sizeof(float) * svf::kNdfTexels * chunk));
    if(mlp)
    {
        SVF_TRY(ctx->mlp_x.ensure(sizeof(float) * svf::kMlpInputs * chunk));
        SVF_TRY(ctx->mlp_h1.ensure(sizeof(float) * svf::kMlpHidden * chunk));
        SVF_TRY(ctx->mlp_h2.ensure(sizeof(float) * svf::kMlpHidden * chunk));
        SVF_TRY(ctx->mlp_y.ensure(sizeof(float) * svf::kMlpOutputs * chunk));
    }
    if(fallback)
    {
        SVF_TRY(ctx->fb_idx.ensure(sizeof(uint32_t) * (chunk + 4)));
        SVF_TRY(ctx->fb_lum.ensure(sizeof(float) * stride * chunk));
        SVF_TRY(ctx->fb_hi.ensure(2 * stride * chunk));
        SVF_TRY(ctx->fb_lo.ensure(2 * stride * chunk));
        SVF_TRY(ctx->fb_ndf.ensure(sizeof(float) * fb_ld * chunk));
        SVF_TRY(ctx->fb_small.ensure((sizeof(float) * (3 + 7 + 7 + 1 + 12) + sizeof(svf_texel_stats)) * chunk));
    }
    uint64_t fallback_texels = 0;
    DevBuf* staging[2] = { &ctx->samples, &ctx->samples2 };
    if(!samples_on_device)
    {
        SVF_TRY(ctx->samples.ensure(texel_bytes * chunk));
        if(n_chunks > 1)
            SVF_TRY(ctx->samples2.ensure(texel_bytes * chunk));
    }
    // per chunk: copy start/end (copy stream), then lum, init, LM, outputs, NDF GEMM end (compute stream)
    constexpr int kEv = 8;
    while(ctx->chunk_ev.size() < kEv * n_chunks)
    {
        cudaEvent_t e;
        SVF_CUDA(cudaEventCreate(&e));
        ctx->chunk_ev.push_back(e);
    }
    auto ev = [&](uint64_t c, int k) { return ctx->chunk_ev[kEv * c + (uint64_t)k]; };
    // inside a graph capture a timing event must be an external record node
    bool capturing = false;
    auto mark = [&](cudaEvent_t e, cudaStream_t st) {
        return cudaEventRecordWithFlags(e, st, capturing ? cudaEventRecordExternal : cudaEventRecordDefault);
    };

    // host -> device copy of chunk c into staging buffer c % 2
    auto issue_copy = [&](uint64_t c) -> svf_status {
        const uint64_t c0 = c * chunk, n = std::min<uint64_t>(chunk, T - c0);
        const int buf = (int)(c & 1);
        if(c >= 2)
            SVF_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->freed[buf], 0));
        SVF_CUDA(cudaEventRecord(ev(c, 0), ctx->copy_stream));
        SVF_CUDA(cudaMemcpyAsync(staging[buf]->p, static_cast<const char*>(btf->samples) + c0 * texel_bytes,
                                 texel_bytes * n, cudaMemcpyHostToDevice, ctx->copy_stream));
        SVF_CUDA(cudaEventRecord(ev(c, 1), ctx->copy_stream));
        SVF_CUDA(cudaEventRecord(ctx->copied[buf], ctx->copy_stream));
        return SVF_OK;
    };

    // Everything the call puts on the streams; run directly, or recorded once
    // into a CUDA graph and replayed (below).
    auto enqueue = [&]() -> svf_status {
    SVF_TRY(zero_error_flags(ctx));
    if(!samples_on_device)
    {
        // the compute stream's earlier work (a previous call) is done with the
        // staging buffers before the first copies overwrite them
        SVF_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
        SVF_CUDA(cudaStreamWaitEvent(ctx->copy_stream, ctx->ev[0], 0));
        SVF_TRY(issue_copy(0));
        if(n_chunks > 1)
            SVF_TRY(issue_copy(1));
    }
    for(uint64_t c = 0; c < n_chunks; ++c)
    {
        const uint64_t c0 = c * chunk, n = std::min<uint64_t>(chunk, T - c0);
        const void* samples = static_cast<const char*>(btf->samples) + c0 * texel_bytes;
        const int buf = (int)(c & 1);
        if(!samples_on_device)
        {
            SVF_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->copied[buf], 0));
            samples = staging[buf]->p;
        }
        SVF_CUDA(mark(ev(c, 2), ctx->stream));
        // the average chromaticity only colours the diffuse / specular maps and starts the RGB fit
        const bool chroma = rgb || maps->diffuse || maps->specular;
        SVF_CUDA(svf::launch_luminance(samples, btf->sample_type, n, N, ctx->lum.as<float>(), stride,
                                       chroma ? ctx->avg.as<float>() : nullptr, default_init ? ctx->lum_hi.p : nullptr,
                                       default_init ? ctx->lum_lo.p : nullptr,
                                       default_init ? init_lay->col_pos : nullptr, ctx->stream,
                                       rgb ? ctx->rgb16.p : nullptr, stride3,
                                       lum_features(mlp, ctx->mlp_x.as<float>(), true)));
        // the learned guess's inputs, read before the staging buffer is handed back
        SVF_CUDA(rgb_features(mlp, samples, btf->sample_type, N, n, ctx->mlp_x.as<float>(), true, ctx->stream));
        if(!samples_on_device)
        {
            SVF_CUDA(cudaEventRecord(ctx->freed[buf], ctx->stream));
            if(c + 2 < n_chunks)
                SVF_TRY(issue_copy(c + 2));
        }
        SVF_CUDA(mark(ev(c, 3), ctx->stream));
        if(default_init)
        {
            cudaError_t e = launch_ndf(*init_lay, ctx->lum_hi.p, ctx->lum_lo.p, n, stride, ctx->ndf.as<float>(),
                                       ndf_ld, ctx->error.as<uint32_t>() + 2, ctx->stream);
            if(e != cudaSuccess)
                return fail(SVF_ECUDA, "NDF GEMM launch: %s", cudaGetErrorString(e));
            SVF_CUDA(mark(ev(c, 7), ctx->stream));
            SVF_CUDA(svf::launch_init_finish(*init_lay, ctx->ndf.as<float>(), ndf_ld, n, ctx->init.as<float>(),
                                             nullptr, maps->ndf ? ctx->ndf_tex.as<float>() : nullptr, ctx->stream));
        }
        else if(mlp)
        {
            // the learned initial guess from the chunk's features
            SVF_TRY(mlp_infer(ctx, mlp, ctx->mlp_x.as<float>(), n, ctx->mlp_h1.as<float>(), ctx->mlp_h2.as<float>(),
                              ctx->mlp_y.as<float>()));
            SVF_CUDA(svf::mlp_finish(ctx->mlp_y.as<float>(), n, mlp->d_ymean.as<float>(), mlp->d_ystd.as<float>(),
                                     ctx->init.as<float>(), ctx->stream));
        }
        else
            SVF_TRY(to_device(ctx, rgb ? ctx->init_rgb.p : ctx->init.p, opts->init_params + kout * c0,
                              sizeof(float) * kout * n));
        if(rgb && (default_init || mlp))
        {
            // the RGB fit starts where the luminance fit from the default guess
            // ends, coloured by the average chromaticity (svbrdffit's own maps):
            // its accepted steps only lower that RGB residual
            LmRun lr{ ctx->lum.p, stride, ctx->init.as<float>(), ctx->out.as<float>(), ctx->rmse.as<float>(),
                      ctx->stats.as<svf_texel_stats>() + c0, nullptr, nullptr, nullptr, nullptr, nullptr, n };
            lr.damping = initial_damping(*opts);
            SVF_TRY(run_lm(ctx, lay, &opts->lsq, lr));
            SVF_CUDA(svf::launch_rgb_init(ctx->out.as<float>(), ctx->avg.as<float>(), n, ctx->init_rgb.as<float>(),
                                          ctx->stream));
        }
        const float* init_used = rgb ? ctx->init_rgb.as<float>() : ctx->init.as<float>();
        SVF_CUDA(mark(ev(c, 4), ctx->stream));
        float* mb = ctx->maps_buf.as<float>();
        LmRun r{ rgb ? (const void*)ctx->rgb16.p : (const void*)ctx->lum.p, rgb ? stride3 : stride, init_used,
                 ctx->out.as<float>(), ctx->rmse.as<float>(), ctx->stats.as<svf_texel_stats>() + c0,
                 ctx->avg.as<float>(), mb, mb + 3 * n, mb + 6 * n, mb + 8 * n, n };
        r.rgb = rgb;
        // (the RGB fit chained from the luminance fit starts with the reference's damping)
        r.damping = rgb && (default_init || mlp) ? 1.0f : initial_damping(*opts);
        SVF_TRY(run_lm(ctx, lay, &opts->lsq, r));
        if(fallback)
        {
            // texels whose relative RMSE is above the threshold are fitted from
            // the default guess too (their slabs gathered) and keep the lower RMSE
            uint32_t* idx = ctx->fb_idx.as<uint32_t>();
            uint32_t* count = idx + chunk;   // [0] selected, [1] replaced
            SVF_CUDA(cudaMemsetAsync(count, 0, 2 * sizeof(uint32_t), ctx->stream));
            SVF_CUDA(svf::launch_fallback_select(ctx->lum.as<float>(), stride, N, ctx->rmse.as<float>(), n,
                                                 opts->mlp_fallback, idx, count, ctx->stream));
            uint32_t m = 0;
            SVF_CUDA(cudaMemcpyAsync(&m, count, sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
            SVF_CUDA(cudaStreamSynchronize(ctx->stream));
            if(m)
            {
                float* g = ctx->fb_small.as<float>();
                float* g_avg = g;
                float* g_init = g_avg + 3 * (uint64_t)m;
                float* g_out = g_init + 7 * (uint64_t)m;
                float* g_rmse = g_out + 7 * (uint64_t)m;
                float* g_maps = g_rmse + m;
                svf_texel_stats* g_stats = reinterpret_cast<svf_texel_stats*>(g_maps + 12 * (uint64_t)m);
                SVF_CUDA(svf::launch_gather_slabs(ctx->lum.as<float>(), stride, chroma ? ctx->avg.as<float>() : nullptr,
                                                  idx, m, ctx->fb_lum.as<float>(), g_avg, ctx->stream));
                SVF_CUDA(svf::launch_split_bf16_permuted(ctx->fb_lum.as<float>(), m, stride, N, init_lay->col_of,
                                                         ctx->fb_hi.p, ctx->fb_lo.p, ctx->stream));
                cudaError_t e = launch_ndf(*init_lay, ctx->fb_hi.p, ctx->fb_lo.p, m, stride, ctx->fb_ndf.as<float>(),
                                           fb_ld, ctx->error.as<uint32_t>() + 2, ctx->stream);
                if(e != cudaSuccess)
                    return fail(SVF_ECUDA, "NDF GEMM launch: %s", cudaGetErrorString(e));
                SVF_CUDA(svf::launch_init_finish(*init_lay, ctx->fb_ndf.as<float>(), fb_ld, m, g_init, nullptr,
                                                 nullptr, ctx->stream));
                LmRun gr{ ctx->fb_lum.p, stride, g_init, g_out, g_rmse, g_stats, chroma ? g_avg : nullptr, g_maps,
                          g_maps + 3 * m, g_maps + 6 * m, g_maps + 8 * m, m };
                SVF_TRY(run_lm(ctx, lay, &opts->lsq, gr));
                SVF_CUDA(svf::launch_fallback_merge(idx, m, g_out, g_rmse, g_stats, g_maps, g_init, n,
                                                    ctx->out.as<float>(), ctx->rmse.as<float>(),
                                                    ctx->stats.as<svf_texel_stats>() + c0, mb, ctx->init.as<float>(),
                                                    count + 1, ctx->stream));
                fallback_texels += m;
            }
        }
        SVF_CUDA(mark(ev(c, 5), ctx->stream));
        // outputs (into host or device buffers of the caller)
        auto put = [&](void* dst, const void* src, size_t bytes) -> svf_status {
            if(dst)
                SVF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
            return SVF_OK;
        };
        SVF_TRY(put(maps->diffuse ? maps->diffuse + 3 * c0 : nullptr, mb, sizeof(float) * 3 * n));
        SVF_TRY(put(maps->specular ? maps->specular + 3 * c0 : nullptr, mb + 3 * n, sizeof(float) * 3 * n));
        SVF_TRY(put(maps->sigma ? maps->sigma + 2 * c0 : nullptr, mb + 6 * n, sizeof(float) * 2 * n));
        SVF_TRY(put(maps->basis ? maps->basis + 4 * c0 : nullptr, mb + 8 * n, sizeof(float) * 4 * n));
        SVF_TRY(put(maps->rmse ? maps->rmse + c0 : nullptr, ctx->rmse.p, sizeof(float) * n));
        SVF_TRY(put(maps->params ? maps->params + kout * c0 : nullptr, ctx->out.p, sizeof(float) * kout * n));
        SVF_TRY(put(maps->init ? maps->init + kout * c0 : nullptr, init_used, sizeof(float) * kout * n));
        SVF_TRY(put(maps->ndf ? maps->ndf + (uint64_t)svf::kNdfTexels * c0 : nullptr, ctx->ndf_tex.p,
                    sizeof(float) * svf::kNdfTexels * n));
        SVF_CUDA(mark(ev(c, 6), ctx->stream));
    }
    return SVF_OK;
    };

    // CUDA graph.  A call that repeats the previous call exactly (the same
    // device-resident samples, sizes, options, initial parameters and output
    // buffers, all on the device or in pinned host memory; one chunk; no
    // device buffer reallocated since) is recorded into a graph on its second
    // occurrence and replayed from then on: its launches, copies and events
    // go to the GPU as one graph launch.
    uint32_t graph_mode = 0;   // svf_run_stats::graph
    auto reachable = [&](const void* p) {
        if(!p)
            return true;
        cudaPointerAttributes at;
        if(cudaPointerGetAttributes(&at, p) != cudaSuccess)
        {
            cudaGetLastError();
            return false;
        }
        return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged || at.type == cudaMemoryTypeHost;
    };
    bool eligible = samples_on_device && n_chunks == 1 && !fallback && reachable(opts->init_params) &&
                    reachable(maps->diffuse) && reachable(maps->specular) && reachable(maps->sigma) &&
                    reachable(maps->basis) && reachable(maps->rmse) && reachable(maps->params) &&
                    reachable(maps->init) && reachable(maps->ndf);
    if(eligible && (!rgb || default_init || mlp) && !lay->tuned && T >= 4096)
        SVF_TRY(tune_lm(ctx, lay, &opts->lsq));   // the autotuner synchronises: never inside a capture
    std::vector<uint64_t> key;
    if(eligible)
    {
        auto u = [&](const void* p) { key.push_back((uint64_t)(uintptr_t)p); };
        u(btf->samples);
        u(lay);
        u(init_lay);
        u(opts->init_params);
        u(mlp);
        key.push_back(mlp ? (uint64_t)mlp->step : 0);
        {
            const float dmp = initial_damping(*opts);
            uint32_t bits;
            std::memcpy(&bits, &dmp, 4);
            key.push_back(bits);
        }
        u(maps->diffuse);
        u(maps->specular);
        u(maps->sigma);
        u(maps->basis);
        u(maps->rmse);
        u(maps->params);
        u(maps->init);
        u(maps->ndf);
        key.insert(key.end(), { (uint64_t)btf->sample_type, T, (uint64_t)opts->init_mode,
                                (uint64_t)opts->lsq.max_iterations, (uint64_t)opts->lsq.flags,
                                (uint64_t)opts->lsq.restarts, g_buffer_gen.load(),
                                (uint64_t)(lay->tuned ? lay->choice.threads * 16 + lay->choice.slots : 0) });
        uint64_t bits[3];
        std::memcpy(&bits[0], &opts->lsq.mse_target, 8);
        std::memcpy(&bits[1], &opts->lsq.break_on_small_step, 8);
        const double fr = opts->lsq.fresnel;
        std::memcpy(&bits[2], &fr, 8);
        key.insert(key.end(), bits, bits + 3);
    }
    if(eligible && ctx->graph_exec && key == ctx->graph_key)
    {
        SVF_CUDA(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
        graph_mode = 2;
    }
    else if(eligible && key == ctx->pending_key)
    {
        if(ctx->graph_exec)
        {
            cudaGraphExecDestroy(ctx->graph_exec);
            ctx->graph_exec = nullptr;
            ctx->graph_key.clear();
        }
        cudaGraph_t graph = nullptr;
        bool captured = false;
        if(cudaStreamBeginCapture(ctx->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess)
        {
            capturing = true;
            const svf_status st_enq = enqueue();
            capturing = false;
            const cudaError_t e_end = cudaStreamEndCapture(ctx->stream, &graph);
            if(st_enq == SVF_OK && e_end == cudaSuccess && graph &&
               cudaGraphInstantiate(&ctx->graph_exec, graph, 0) == cudaSuccess)
                captured = true;
            if(graph)
                cudaGraphDestroy(graph);
        }
        cudaGetLastError();
        if(captured)
        {
            ctx->graph_key = key;
            SVF_CUDA(cudaGraphLaunch(ctx->graph_exec, ctx->stream));
            graph_mode = 1;
        }
        else
        {
            // not capturable here: run the call directly
            ctx->graph_exec = nullptr;
            ctx->pending_key.clear();
            SVF_TRY(enqueue());
        }
    }
    else
    {
        if(eligible)
            ctx->pending_key = key;
        SVF_TRY(enqueue());
    }
    std::vector<svf_texel_stats> st(T);
    SVF_CUDA(cudaMemcpyAsync(st.data(), ctx->stats.p, sizeof(svf_texel_stats) * T, cudaMemcpyDeviceToHost,
                             ctx->stream));
    SVF_TRY(read_error_flag(ctx, default_init || mlp));   // waits for the compute stream
    SVF_CUDA(cudaStreamSynchronize(ctx->copy_stream));
    if(maps->stats)
        SVF_CUDA(cudaMemcpy(maps->stats, st.data(), sizeof(svf_texel_stats) * T, cudaMemcpyDefault));

    svf_run_stats rs{};
    for(auto& x : st)
    {
        rs.iterations += x.iterations;
        rs.jacobians += x.jacobians;
        rs.residuals += x.residuals;
        if(x.status & (SVF_TEXEL_NONFINITE | SVF_TEXEL_TIMEOUT))
            rs.failed_texels++;
    }
    auto span = [&](cudaEvent_t a0, cudaEvent_t a1) -> double {
        float ms = 0.0f;
        return cudaEventElapsedTime(&ms, a0, a1) == cudaSuccess ? (double)ms : 0.0;
    };
    for(uint64_t c = 0; c < n_chunks; ++c)
    {
        if(!samples_on_device)
            rs.ms_copy += span(ev(c, 0), ev(c, 1));
        rs.ms_luminance += span(ev(c, 2), ev(c, 3));
        rs.ms_init += span(ev(c, 3), ev(c, 4));
        if(default_init)
            rs.ms_ndf += span(ev(c, 3), ev(c, 7));
        rs.ms_fit += span(ev(c, 4), ev(c, 5));
        rs.ms_copy += span(ev(c, 5), ev(c, 6));
    }
    if(default_init)
    {
        rs.ndf_tiles = init_lay->nonempty_tiles;
        rs.ndf_tiles_total = init_lay->all_tiles;
    }
    // the whole call: from the first copy (or the first kernel) to the last output
    rs.ms_total = span(samples_on_device ? ev(0, 2) : ev(0, 0), ev(n_chunks - 1, 6));
    cudaGetLastError();
    rs.texels = T;
    rs.graph = graph_mode;
    const svf::LmKernelChoice used = lm_choice(lay, rgb ? stride3 : stride, rgb);
    rs.lm_threads = (uint32_t)used.threads;
    rs.lm_slots = (uint32_t)used.slots;
    rs.fallback_texels = (uint32_t)fallback_texels;
    if(run)
        *run = rs;
    if(rs.failed_texels)
        return fail(SVF_EPARTIAL, "%llu texels did not produce a finite fit", (unsigned long long)rs.failed_texels);
    return SVF_OK;
}

svf_status svf_fit_btfs(svf_ctx* ctx, const svf_btf_view* btfs, uint32_t n_btf, const svf_fit_options* opts,
                        const svf_maps* maps, svf_run_stats* runs, svf_run_stats* total)
{
    SVF_TRY(check_ctx(ctx));
    if(n_btf == 0)
        return SVF_OK;
    if(!btfs || !opts || !maps)
        return fail(SVF_EINVAL, "null btfs/options/maps");
    SVF_TRY(check_options(&opts[0].lsq));

    // per BTF: layout, default-init tables, sizes
    const bool rgb = (opts[0].lsq.flags & SVF_LSQ_RGB) != 0;
    const uint64_t kout = rgb ? 12 : 7;
    struct Item
    {
        Layout* lay = nullptr;
        const svf::InitLayout* init = nullptr;
        uint64_t T = 0, stride = 0, stride3 = 0;
        size_t texel_bytes = 0;
        bool on_device = false, default_init = false;
        const svf_mlp* mlp = nullptr;   // SVF_INIT_MLP
    };
    std::vector<Item> it(n_btf);
    for(uint32_t b = 0; b < n_btf; ++b)
    {
        const svf_btf_view& v = btfs[b];
        const svf_fit_options& o = opts[b];
        if(!v.layout || !v.samples)
            return fail(SVF_EINVAL, "btf %u: null layout/samples", b);
        if(v.sample_type != SVF_SAMPLES_F32 && v.sample_type != SVF_SAMPLES_F16)
            return fail(SVF_EINVAL, "btf %u: unknown sample_type %u", b, v.sample_type);
        if(o.init_mode != SVF_INIT_DEFAULT && o.init_mode != SVF_INIT_GIVEN && o.init_mode != SVF_INIT_MLP)
            return fail(SVF_EINVAL, "btf %u: unknown init_mode %u", b, o.init_mode);
        if(o.init_mode == SVF_INIT_MLP && !o.mlp)
            return fail(SVF_EINVAL, "btf %u: SVF_INIT_MLP needs a model (svf_fit_options::mlp)", b);
        if(o.mlp_fallback != 0.0f)
            return fail(SVF_EINVAL, "btf %u: mlp_fallback is taken by svf_fit_texels only", b);
        if(o.init_mode == SVF_INIT_GIVEN && !o.init_params)
            return fail(SVF_EINVAL, "btf %u: SVF_INIT_GIVEN needs init_params", b);
        const svf_lsq_options &a = o.lsq, &z = opts[0].lsq;
        if(a.max_iterations != z.max_iterations || a.fresnel != z.fresnel || a.flags != z.flags ||
           a.mse_target != z.mse_target || a.break_on_small_step != z.break_on_small_step || a.restarts != z.restarts)
            return fail(SVF_EINVAL, "btf %u: the lsq options must be the same for every BTF of a call", b);
        if(maps[b].ndf && o.init_mode != SVF_INIT_DEFAULT)
            return fail(SVF_EINVAL, "btf %u: the NDF map exists only with the default initial guess", b);
        Item& x = it[b];
        x.T = (uint64_t)v.width * v.height;
        if(x.T > 0xffffffffull)
            return fail(SVF_EINVAL, "btf %u: too many texels", b);
        SVF_TRY(get_layout(ctx, v.layout->lights_parabolic, v.layout->light_count, &x.lay));
        x.stride = round_up((uint64_t)x.lay->L * x.lay->L, 8);
        x.stride3 = round_up(3ull * x.lay->L * x.lay->L, 8);
        x.texel_bytes = (v.sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * (size_t)x.lay->L * x.lay->L;
        SVF_TRY(buffer_location(v.samples, "samples", &x.on_device));
        x.default_init = o.init_mode == SVF_INIT_DEFAULT;
        if(x.default_init)
            SVF_TRY(prepare_init(ctx, x.lay, v.layout, &x.init));
        if(o.init_mode == SVF_INIT_MLP)
        {
            x.mlp = o.mlp;
            if(x.mlp->L != x.lay->L || std::memcmp(x.mlp->lp.data(), x.lay->lp.data(), sizeof(float) * 2 * x.mlp->L))
                return fail(SVF_EINVAL, "btf %u: the model was trained for another direction layout", b);
            if(x.mlp->device != ctx->device)
                return fail(SVF_EINVAL, "btf %u: the model lives on device %d, the context on %d", b, x.mlp->device,
                            ctx->device);
        }
    }
    uint32_t ndf_ld = 0;   // NDF rows per texel (the same for every layout: the 64x64 texture's hemisphere)
    for(auto& x : it)
        if(x.default_init)
            ndf_ld = std::max(ndf_ld, x.init->ndf_rows_pad);

    // Chunks of up to kLmMaxSegments pieces (runs of one BTF's texels) within a
    // device-memory budget; each chunk is one LM launch.
    size_t free_b = 0, total_b = 0;
    SVF_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const size_t budget = free_b / 2;
    auto texel_cost = [&](uint32_t b) -> size_t {
        const Item& x = it[b];
        return sizeof(float) * (x.stride + 3 + 7 + kout + 1 + 12) + sizeof(svf_texel_stats) +
               (rgb ? 2 * x.stride3 + sizeof(float) * 12 : 0) +
               (x.default_init ? 2 * 2 * x.stride + sizeof(float) * ndf_ld : 0) +
               (x.mlp ? sizeof(float) * (svf::kMlpInputs + 2 * svf::kMlpHidden + svf::kMlpOutputs) : 0) +
               (maps[b].ndf ? sizeof(float) * svf::kNdfTexels : 0) + (x.on_device ? 0 : x.texel_bytes);
    };
    struct Piece
    {
        uint32_t b;
        uint64_t first, count, k0;   // texels of BTF b; k0: position in the chunk
        uint64_t off;                // slab offset (floats) in the chunk
        uint64_t off3;               // RGB slab offset (halves) in the chunk
    };
    std::vector<std::vector<Piece>> chunks(1);
    uint64_t chunk_texels = 0, chunk_floats = 0, chunk_halves = 0;
    size_t chunk_bytes = 0;
    const uint64_t max_texels = 65535ull * 128;   // the NDF GEMM's grid rows of 128 texels
    for(uint32_t b = 0; b < n_btf; ++b)
    {
        uint64_t first = 0;
        while(first < it[b].T)
        {
            const size_t cost = texel_cost(b);
            uint64_t room = std::min<uint64_t>((budget - std::min(budget, chunk_bytes)) / cost, max_texels - chunk_texels);
            if(chunks.back().size() >= (size_t)svf::kLmMaxSegments || room == 0)
            {
                if(chunks.back().empty())
                    return fail(SVF_ENOMEM, "btf %u: one texel does not fit in device memory", b);
                chunks.emplace_back();
                chunk_texels = chunk_floats = chunk_halves = 0;
                chunk_bytes = 0;
                continue;
            }
            const uint64_t n = std::min<uint64_t>(room, it[b].T - first);
            chunks.back().push_back(Piece{ b, first, n, chunk_texels, chunk_floats, chunk_halves });
            chunk_texels += n;
            chunk_floats += n * it[b].stride;
            chunk_halves += n * it[b].stride3;
            chunk_bytes += n * cost;
            first += n;
        }
    }
    if(chunks.back().empty())
        chunks.pop_back();

    // buffers for the largest chunk
    uint64_t max_n = 0, max_floats = 0, max_halves = 0, max_mlp = 0;
    size_t max_stage = 0;
    bool any_ndf = false, any_default = false;
    for(auto& ch : chunks)
    {
        uint64_t n = 0, f = 0, h = 0;
        for(auto& p : ch)
        {
            n += p.count;
            f += p.count * it[p.b].stride;
            h += p.count * it[p.b].stride3;
            if(!it[p.b].on_device)
                max_stage = std::max(max_stage, it[p.b].texel_bytes * (size_t)p.count);
            any_ndf = any_ndf || maps[p.b].ndf;
            any_default = any_default || it[p.b].default_init;
            if(it[p.b].mlp)
                max_mlp = std::max(max_mlp, p.count);
        }
        max_n = std::max(max_n, n);
        max_floats = std::max(max_floats, f);
        max_halves = std::max(max_halves, h);
    }
    SVF_TRY(ctx->lum.ensure(sizeof(float) * max_floats));
    SVF_TRY(ctx->avg.ensure(sizeof(float) * 3 * max_n));
    SVF_TRY(ctx->init.ensure(sizeof(float) * 7 * max_n));
    SVF_TRY(ctx->out.ensure(sizeof(float) * kout * max_n));
    if(rgb)
    {
        SVF_TRY(ctx->rgb16.ensure(2 * max_halves));
        SVF_TRY(ctx->init_rgb.ensure(sizeof(float) * 12 * max_n));
    }
    float* init_used = rgb ? ctx->init_rgb.as<float>() : ctx->init.as<float>();
    SVF_TRY(ctx->rmse.ensure(sizeof(float) * max_n));
    SVF_TRY(ctx->stats.ensure(sizeof(svf_texel_stats) * max_n));
    SVF_TRY(ctx->maps_buf.ensure(sizeof(float) * 12 * max_n));
    if(any_default)
    {
        SVF_TRY(ctx->lum_hi.ensure(2 * max_floats));
        SVF_TRY(ctx->lum_lo.ensure(2 * max_floats));
        SVF_TRY(ctx->ndf.ensure(sizeof(float) * ndf_ld * max_n));
    }
    if(any_ndf)
        SVF_TRY(ctx->ndf_tex.ensure(sizeof(float) * svf::kNdfTexels * max_n));
    if(max_stage)
        SVF_TRY(ctx->samples.ensure(max_stage));
    if(max_mlp)
    {
        SVF_TRY(ctx->mlp_x.ensure(sizeof(float) * svf::kMlpInputs * max_mlp));
        SVF_TRY(ctx->mlp_h1.ensure(sizeof(float) * svf::kMlpHidden * max_mlp));
        SVF_TRY(ctx->mlp_h2.ensure(sizeof(float) * svf::kMlpHidden * max_mlp));
        SVF_TRY(ctx->mlp_y.ensure(sizeof(float) * svf::kMlpOutputs * max_mlp));
    }

    std::vector<svf_run_stats> rs(n_btf);
    svf_run_stats all{};
    SVF_TRY(zero_error_flags(ctx));
    SVF_CUDA(cudaEventRecord(ctx->ev[0], ctx->stream));
    float ms = 0.0f;
    for(auto& ch : chunks)
    {
        uint64_t n = 0;
        for(auto& p : ch)
            n += p.count;
        SVF_CUDA(cudaEventRecord(ctx->ev[1], ctx->stream));
        // luminance and initial guess, piece by piece
        for(auto& p : ch)
        {
            const Item& x = it[p.b];
            const svf_btf_view& v = btfs[p.b];
            const void* samples = static_cast<const char*>(v.samples) + p.first * x.texel_bytes;
            if(!x.on_device)
            {
                SVF_CUDA(cudaMemcpyAsync(ctx->samples.p, samples, x.texel_bytes * p.count, cudaMemcpyHostToDevice,
                                         ctx->stream));
                samples = ctx->samples.p;
            }
            const uint32_t L = x.lay->L, N = L * L;
            float* lum = ctx->lum.as<float>() + p.off;
            const bool chroma = rgb || maps[p.b].diffuse || maps[p.b].specular;
            SVF_CUDA(svf::launch_luminance(samples, v.sample_type, p.count, N, lum, x.stride,
                                           chroma ? ctx->avg.as<float>() + 3 * p.k0 : nullptr,
                                           x.default_init ? ctx->lum_hi.as<uint16_t>() + p.off : nullptr,
                                           x.default_init ? ctx->lum_lo.as<uint16_t>() + p.off : nullptr,
                                           x.default_init ? x.init->col_pos : nullptr,
                                           ctx->stream, rgb ? ctx->rgb16.as<uint16_t>() + p.off3 : nullptr,
                                           x.stride3, lum_features(x.mlp, ctx->mlp_x.as<float>(), true)));
            if(x.default_init)
            {
                cudaError_t e = launch_ndf(*x.init, ctx->lum_hi.as<uint16_t>() + p.off,
                                           ctx->lum_lo.as<uint16_t>() + p.off, p.count, x.stride,
                                           ctx->ndf.as<float>() + p.k0 * ndf_ld, ndf_ld,
                                           ctx->error.as<uint32_t>() + 2, ctx->stream);
                if(e != cudaSuccess)
                    return fail(SVF_ECUDA, "NDF GEMM launch: %s", cudaGetErrorString(e));
                SVF_CUDA(svf::launch_init_finish(*x.init, ctx->ndf.as<float>() + p.k0 * ndf_ld, ndf_ld, p.count,
                                                 ctx->init.as<float>() + 7 * p.k0, nullptr,
                                                 maps[p.b].ndf ? ctx->ndf_tex.as<float>() + p.k0 * svf::kNdfTexels
                                                               : nullptr,
                                                 ctx->stream));
            }
            else if(x.mlp)
            {
                SVF_CUDA(rgb_features(x.mlp, samples, v.sample_type, N, p.count, ctx->mlp_x.as<float>(), true,
                                      ctx->stream));
                SVF_TRY(mlp_infer(ctx, x.mlp, ctx->mlp_x.as<float>(), p.count, ctx->mlp_h1.as<float>(),
                                  ctx->mlp_h2.as<float>(), ctx->mlp_y.as<float>()));
                SVF_CUDA(svf::mlp_finish(ctx->mlp_y.as<float>(), p.count, x.mlp->d_ymean.as<float>(),
                                         x.mlp->d_ystd.as<float>(), ctx->init.as<float>() + 7 * p.k0, ctx->stream));
            }
            else
                SVF_TRY(to_device(ctx, init_used + kout * p.k0, opts[p.b].init_params + kout * p.first,
                                  sizeof(float) * kout * p.count));

        }
        // the RGB fit of default-initialised pieces starts from their luminance
        // fit coloured by the average chromaticity (as in svf_fit_texels)
        bool rgb_from_lum = false;
        for(auto& p : ch)
            rgb_from_lum = rgb_from_lum || (rgb && (it[p.b].default_init || it[p.b].mlp));
        if(rgb_from_lum)
        {
            // pieces with given RGB parameters ride along from a zero start
            for(auto& p : ch)
                if(!it[p.b].default_init && !it[p.b].mlp)
                    SVF_CUDA(cudaMemsetAsync(ctx->init.as<float>() + 7 * p.k0, 0, sizeof(float) * 7 * p.count,
                                             ctx->stream));
            svf::LmSegment ls[svf::kLmMaxSegments];
            bool lup = true;
            uint64_t lstride = 0;
            for(size_t i = 0; i < ch.size(); ++i)
            {
                const Item& x = it[ch[i].b];
                ls[i] = svf::LmSegment{ (uint32_t)ch[i].k0, x.lay->L, x.stride, ctx->lum.as<float>() + ch[i].off,
                                        x.lay->geo.as<float>(), initial_damping(opts[ch[i].b]) };
                lup = lup && x.lay->all_up;
                lstride = std::max(lstride, x.stride);
            }
            LmRun lr{ nullptr, lstride, ctx->init.as<float>(), ctx->out.as<float>(), ctx->rmse.as<float>(),
                      ctx->stats.as<svf_texel_stats>(), nullptr, nullptr, nullptr, nullptr, nullptr, n,
                      ls, (uint32_t)ch.size(), lup, false };
            std::vector<Layout*> llays(ch.size());
            for(size_t i = 0; i < ch.size(); ++i)
                llays[i] = it[ch[i].b].lay;
            SVF_TRY(run_lm_segments(ctx, llays.data(), &opts[0].lsq, lr));
            for(auto& p : ch)
                if(it[p.b].default_init || it[p.b].mlp)
                    SVF_CUDA(svf::launch_rgb_init(ctx->out.as<float>() + 7 * p.k0, ctx->avg.as<float>() + 3 * p.k0,
                                                  p.count, init_used + 12 * p.k0, ctx->stream));
        }
        SVF_CUDA(cudaEventRecord(ctx->ev[2], ctx->stream));
        // LM over the pieces, whatever their layouts: one launch per run of pieces
        // whose layouts choose the same kernel configuration
        svf::LmSegment seg[svf::kLmMaxSegments];
        bool all_up = true;
        uint64_t max_stride = 0;
        for(size_t i = 0; i < ch.size(); ++i)
        {
            const Item& x = it[ch[i].b];
            // (the RGB fit chained from the luminance fit starts with the reference's damping)
            const float dmp = rgb && (x.default_init || x.mlp) ? 1.0f : initial_damping(opts[ch[i].b]);
            if(rgb)
                seg[i] = svf::LmSegment{ (uint32_t)ch[i].k0, x.lay->L, x.stride3,
                                         ctx->rgb16.as<uint16_t>() + ch[i].off3, x.lay->geo.as<float>(), dmp };
            else
                seg[i] = svf::LmSegment{ (uint32_t)ch[i].k0, x.lay->L, x.stride, ctx->lum.as<float>() + ch[i].off,
                                         x.lay->geo.as<float>(), dmp };
            all_up = all_up && x.lay->all_up;
            max_stride = std::max(max_stride, rgb ? x.stride3 : x.stride);
        }
        float* mb = ctx->maps_buf.as<float>();
        LmRun r{ nullptr, max_stride, init_used, ctx->out.as<float>(), ctx->rmse.as<float>(),
                 ctx->stats.as<svf_texel_stats>(), ctx->avg.as<float>(), mb, mb + 3 * n, mb + 6 * n, mb + 8 * n, n,
                 seg, (uint32_t)ch.size(), all_up, rgb };
        std::vector<Layout*> lays(ch.size());
        for(size_t i = 0; i < ch.size(); ++i)
            lays[i] = it[ch[i].b].lay;
        SVF_TRY(run_lm_segments(ctx, lays.data(), &opts[0].lsq, r));
        SVF_CUDA(cudaEventRecord(ctx->ev[3], ctx->stream));
        // outputs, piece by piece
        std::vector<svf_texel_stats> st(n);
        SVF_CUDA(cudaMemcpyAsync(st.data(), ctx->stats.p, sizeof(svf_texel_stats) * n, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        for(auto& p : ch)
        {
            const svf_maps& m = maps[p.b];
            auto put = [&](void* dst, const void* src, size_t bytes) -> svf_status {
                if(dst)
                    SVF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
                return SVF_OK;
            };
            const uint64_t k = p.k0, c = p.count, f = p.first;
            SVF_TRY(put(m.diffuse ? m.diffuse + 3 * f : nullptr, mb + 3 * k, sizeof(float) * 3 * c));
            SVF_TRY(put(m.specular ? m.specular + 3 * f : nullptr, mb + 3 * n + 3 * k, sizeof(float) * 3 * c));
            SVF_TRY(put(m.sigma ? m.sigma + 2 * f : nullptr, mb + 6 * n + 2 * k, sizeof(float) * 2 * c));
            SVF_TRY(put(m.basis ? m.basis + 4 * f : nullptr, mb + 8 * n + 4 * k, sizeof(float) * 4 * c));
            SVF_TRY(put(m.rmse ? m.rmse + f : nullptr, ctx->rmse.as<float>() + k, sizeof(float) * c));
            SVF_TRY(put(m.params ? m.params + kout * f : nullptr, ctx->out.as<float>() + kout * k,
                        sizeof(float) * kout * c));
            SVF_TRY(put(m.init ? m.init + kout * f : nullptr, init_used + kout * k, sizeof(float) * kout * c));
            SVF_TRY(put(m.ndf ? m.ndf + (uint64_t)svf::kNdfTexels * f : nullptr,
                        ctx->ndf_tex.as<float>() + (uint64_t)svf::kNdfTexels * k, sizeof(float) * svf::kNdfTexels * c));
        }
        SVF_CUDA(cudaEventRecord(ctx->ev[4], ctx->stream));
        SVF_TRY(read_error_flag(ctx, any_default || max_mlp));   // waits for the chunk
        for(auto& p : ch)
        {
            svf_run_stats& q = rs[p.b];
            q.texels += p.count;
            for(uint64_t i = 0; i < p.count; ++i)
            {
                const svf_texel_stats& x = st[p.k0 + i];
                q.iterations += x.iterations;
                q.jacobians += x.jacobians;
                q.residuals += x.residuals;
                if(x.status & (SVF_TEXEL_NONFINITE | SVF_TEXEL_TIMEOUT))
                    q.failed_texels++;
            }
            if(maps[p.b].stats)
                SVF_CUDA(cudaMemcpy(maps[p.b].stats + p.first, st.data() + p.k0, sizeof(svf_texel_stats) * p.count,
                                    cudaMemcpyDefault));
        }
        SVF_CUDA(cudaEventElapsedTime(&ms, ctx->ev[1], ctx->ev[2]));
        all.ms_init += ms;   // luminance, NDF GEMM and init finish (and any host copies) of the pieces
        SVF_CUDA(cudaEventElapsedTime(&ms, ctx->ev[2], ctx->ev[3]));
        all.ms_fit += ms;
        SVF_CUDA(cudaEventElapsedTime(&ms, ctx->ev[3], ctx->ev[4]));
        all.ms_copy += ms;
    }
    SVF_CUDA(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[4]));
    all.ms_total = ms;
    Layout* big = it[0].lay;
    uint64_t big_stride = rgb ? it[0].stride3 : it[0].stride;
    for(auto& x : it)
        if(x.lay->L > big->L)
        {
            big = x.lay;
            big_stride = rgb ? x.stride3 : x.stride;
        }
    const svf::LmKernelChoice used = lm_choice(big, big_stride, rgb);
    for(auto& q : rs)
    {
        all.texels += q.texels;
        all.iterations += q.iterations;
        all.jacobians += q.jacobians;
        all.residuals += q.residuals;
        all.failed_texels += q.failed_texels;
    }
    all.lm_threads = (uint32_t)used.threads;
    all.lm_slots = (uint32_t)used.slots;
    for(uint32_t b = 0; b < n_btf; ++b)
    {
        rs[b].ms_total = all.ms_total;
        rs[b].ms_init = all.ms_init;
        rs[b].ms_fit = all.ms_fit;
        rs[b].ms_copy = all.ms_copy;
        rs[b].lm_threads = all.lm_threads;
        rs[b].lm_slots = all.lm_slots;
        if(runs)
            runs[b] = rs[b];
    }
    if(total)
        *total = all;
    if(all.failed_texels)
        return fail(SVF_EPARTIAL, "%llu texels did not produce a finite fit", (unsigned long long)all.failed_texels);
    return SVF_OK;
}

svf_status svf_synth_btf(svf_ctx* ctx, uint32_t seed, uint32_t mix, const float* lp, uint32_t L, uint64_t first,
                         uint64_t count, uint32_t sample_type, float noise, void* samples, float* truth)
{
    SVF_TRY(check_ctx(ctx));
    if(!samples || !lp)
        return fail(SVF_EINVAL, "null samples/lights");
    bool samples_dev = false;
    SVF_TRY(buffer_location(samples, "samples", &samples_dev));
    if(!samples_dev)
        return fail(SVF_EINVAL, "samples must be device memory");
    if(mix > 1 || (sample_type != SVF_SAMPLES_F32 && sample_type != SVF_SAMPLES_F16) || L < 1 || L > 160)
        return fail(SVF_EINVAL, "bad mix/sample_type/light_count");
    if(count == 0)
        return SVF_OK;
    DevBuf d_lp;
    SVF_TRY(d_lp.ensure(sizeof(float) * 2 * L));
    SVF_CUDA(cudaMemcpyAsync(d_lp.p, lp, sizeof(float) * 2 * L, cudaMemcpyDefault, ctx->stream));
    const uint64_t step = 1u << 20;
    float* truth_dev = nullptr;
    DevBuf d_truth;
    bool truth_on_device = false;
    SVF_TRY(buffer_location(truth, "truth", &truth_on_device));
    const bool truth_host = truth && !truth_on_device;
    if(truth_host)
    {
        SVF_TRY(d_truth.ensure(sizeof(float) * 16 * std::min<uint64_t>(count, step)));
        truth_dev = d_truth.as<float>();
    }
    const size_t texel_bytes = (sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * (size_t)L * L;
    for(uint64_t c = 0; c < count; c += step)
    {
        uint64_t n = std::min<uint64_t>(step, count - c);
        float* tr = truth ? (truth_host ? truth_dev : truth + 16 * c) : nullptr;
        SVF_CUDA(svf::launch_synth(seed, mix, d_lp.as<float>(), L, first + c, n, sample_type, noise,
                                   static_cast<char*>(samples) + c * texel_bytes, tr, ctx->stream));
        if(truth_host)
            SVF_CUDA(cudaMemcpyAsync(truth + 16 * c, truth_dev, sizeof(float) * 16 * n, cudaMemcpyDeviceToHost,
                                     ctx->stream));
    }
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    return SVF_OK;
}

} // extern "C"
