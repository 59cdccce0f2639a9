// svf_host_lm.cpp - the persistent LM launch (lm_fit_kernel): its argument
// block, the kernel configuration and its autotuner, the held-parameter masks;
// and the LeastSquaresFitSGGX entry points svf_lsq_fit_batch,
// svf_lsq_fit_batch_noalloc and svf_lsq_fit_sggx.
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

namespace svfh
{

// The LM kernel configuration (CTA size and texel slots) of a layout, once:
// by default svf::lm_default_choice's occupancy rule, which ranks the
// configurations as full launches measured on the B200 do.  With SVF_LM_TUNE
// set, a timed probe decides instead: each candidate fits the same seeded
// synthetic probe (32768 texels of the uneven parameter mix, from a perturbed
// ground truth) and is scored by
// model flops per second (the flops per Jacobian and residual pass times the
// passes it ran, over its CUDA-event time).  The first candidate is kept unless
// another is more than 3% faster.  Tuning on a fixed probe, not on the caller's
// texels, keeps every texel of a call on one configuration.  (Within about 3 %
// the probe ranks the top configurations by noise: on ring-81 it preferred 256
// threads x 2 or 3 slots, which full launches measure 5 - 7 % slower than 128 x
// 2.)
svf_status tune_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o)
{
    if(lay->tuned || std::getenv("SVF_LM_KERNEL"))   // (a pinned configuration needs no probe)
        return SVF_OK;
    if(!std::getenv("SVF_LM_TUNE"))
    {
        lay->choice = svf::lm_default_choice(lay->L, round_up((uint64_t)lay->L * lay->L, 8));
        lay->tuned = true;
        return SVF_OK;
    }
    // the plain passes only: the packed pass (one 256-thread CTA per SM at its
    // register count) wins on this short probe but loses on full launches
    // (measured: 59.4 against 52.2 ms for 160000 ring-81 texels), so it is left
    // to SVF_LM_KERNEL
    svf::LmKernelChoice cand[svf::kLmPlainCandidates];
    const int n_cand = svf::lm_candidates(lay->L, cand, svf::kLmPlainCandidates);
    lay->choice = cand[0];
    if(n_cand <= 1)
    {
        lay->tuned = true;
        return SVF_OK;
    }
    const uint32_t L = lay->L, N = L * L;
    // enough texels to keep every slot of every resident CTA busy for many
    // rounds; the samples are rendered and reduced to slabs in chunks
    const uint64_t stride = round_up(N, 8), T = 32768, chunk = 8192;
    DevBuf samples, truth, lum, avg, init, out, rmse, stats;
    SVF_TRY(samples.ensure(sizeof(float) * 3 * N * chunk));
    SVF_TRY(truth.ensure(sizeof(float) * 16 * T));
    SVF_TRY(lum.ensure(sizeof(float) * stride * T));
    SVF_TRY(avg.ensure(sizeof(float) * 3 * T));
    SVF_TRY(init.ensure(sizeof(float) * 7 * T));
    SVF_TRY(out.ensure(sizeof(float) * 7 * T));
    SVF_TRY(rmse.ensure(sizeof(float) * T));
    SVF_TRY(stats.ensure(sizeof(svf_texel_stats) * T));
    DevBuf d_lp;
    SVF_TRY(upload(d_lp, lay->lp));
    for(uint64_t c0 = 0; c0 < T; c0 += chunk)
    {
        SVF_CUDA(svf::launch_synth(0x5EEDu, 1, d_lp.as<float>(), L, c0, chunk, SVF_SAMPLES_F32, 0.01f, samples.p,
                                   truth.as<float>() + 16 * c0, ctx->stream));
        SVF_CUDA(svf::launch_luminance(samples.p, SVF_SAMPLES_F32, chunk, N, lum.as<float>() + stride * c0, stride,
                                       avg.as<float>() + 3 * c0, nullptr, nullptr, nullptr, ctx->stream));
    }
    std::vector<float> tr(16 * T), in(7 * T);
    SVF_CUDA(cudaMemcpyAsync(tr.data(), truth.p, sizeof(float) * 16 * T, cudaMemcpyDeviceToHost, ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    for(uint64_t t = 0; t < T; ++t)
    {
        const float* q = &tr[16 * t];   // kd[3], ks[3], sigma[2], quat[4], euler[3], kind
        const float lw[3] = { 0.2126f, 0.7152f, 0.0722f };
        const float wob = 1.0f + 0.15f * (float)((int)(t % 7) - 3) / 3.0f;
        float* p = &in[7 * t];
        p[0] = q[6] * wob;
        p[1] = q[7] / wob;
        p[2] = (lw[0] * q[3] + lw[1] * q[4] + lw[2] * q[5]) * wob;
        p[3] = (lw[0] * q[0] + lw[1] * q[1] + lw[2] * q[2]) / wob;
        p[4] = q[12] + 0.1f;
        p[5] = q[13] - 0.1f;
        p[6] = q[14] + 0.1f;
    }
    SVF_CUDA(cudaMemcpyAsync(init.p, in.data(), sizeof(float) * 7 * T, cudaMemcpyHostToDevice, ctx->stream));
    LmRun r{ lum.as<float>(), stride, init.as<float>(), out.as<float>(), rmse.as<float>(),
             stats.as<svf_texel_stats>(), nullptr, nullptr, nullptr, nullptr, nullptr, T };
    // warm-up (module load, attribute set-up) on a small slice
    LmRun warm = r;
    warm.texels = 256;
    // candidates that do not fit on an SM (shared memory at large L) drop out
    int n_fit = 0;
    for(int c = 0; c < n_cand; ++c)
        if(svf::lm_max_ctas_per_sm(L, stride, cand[c]) > 0)
            cand[n_fit++] = cand[c];
    if(n_fit == 0)
        return fail(SVF_EINVAL, "no LM kernel configuration fits on an SM for L = %u", L);
    lay->choice = cand[0];
    if(n_fit == 1)
    {
        lay->tuned = true;
        return SVF_OK;
    }
    for(int c = 0; c < n_fit; ++c)
        SVF_TRY(launch_lm(ctx, lay, o, warm, cand[c]));
    double best_rate = 0.0, first_rate = 0.0;
    int best = 0;
    std::vector<svf_texel_stats> st(T);
    std::vector<double> rates(n_fit, 0.0);
    // two rounds, the second in reverse order, each candidate scored by its
    // better round (the order of launches does not favour a candidate)
    for(int k = 0; k < 2 * n_fit; ++k)
    {
        const int c = k < n_fit ? k : 2 * n_fit - 1 - k;
        SVF_CUDA(cudaEventRecord(ctx->ev[6], ctx->stream));
        SVF_TRY(launch_lm(ctx, lay, o, r, cand[c]));
        SVF_CUDA(cudaEventRecord(ctx->ev[7], ctx->stream));
        SVF_CUDA(cudaMemcpyAsync(st.data(), stats.p, sizeof(svf_texel_stats) * T, cudaMemcpyDeviceToHost,
                                 ctx->stream));
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
        float ms = 0.0f;
        SVF_CUDA(cudaEventElapsedTime(&ms, ctx->ev[6], ctx->ev[7]));
        double flops = 0.0;
        for(auto& s : st)
            flops += (double)N * (169.0 * s.jacobians + 33.0 * s.residuals);
        const double rate = flops / std::max(1e-3, (double)ms);
        if(getenv("SVF_DEBUG"))
            fprintf(stderr, "svf: LM tune L=%u threads=%d slots=%d pass=%d: %.3f ms, %.2f TFLOP/s (model)\n", L,
                    cand[c].threads, cand[c].slots, cand[c].pass, ms, rate * 1e-9);
        rates[c] = std::max(rates[c], rate);
    }
    first_rate = rates[0];
    for(int c = 0; c < n_fit; ++c)
        if(rates[c] > best_rate)
        {
            best_rate = rates[c];
            best = c;
        }
    lay->choice = best_rate > 1.03 * first_rate ? cand[best] : cand[0];
    lay->tuned = true;
    // the probe's launches write only the LM word
    SVF_TRY(read_error_flag(ctx));
    SVF_CUDA(cudaMemsetAsync(ctx->error.p, 0, sizeof(uint32_t), ctx->stream));
    return SVF_OK;
}

// The LM configuration of a run: the autotuned one for the luminance fit, the
// first that fits for the RGB fit (its slabs differ from the probe's).
svf::LmKernelChoice lm_choice(Layout* lay, uint64_t stride, bool rgb)
{
    // SVF_LM_KERNEL=threads,slots,pass pins one candidate of svf::lm_candidates
    // (for tests and measurements); others are ignored
    if(const char* e = std::getenv("SVF_LM_KERNEL"))
    {
        svf::LmKernelChoice c{ 0, 0, 0 };
        if(std::sscanf(e, "%d,%d,%d", &c.threads, &c.slots, &c.pass) == 3)
        {
            svf::LmKernelChoice cand[svf::kLmCandidates];
            const int n = svf::lm_candidates(lay->L, cand, svf::kLmCandidates);
            for(int i = 0; i < n; ++i)
                if(cand[i].threads == c.threads && cand[i].slots == c.slots && cand[i].pass == c.pass &&
                   svf::lm_max_ctas_per_sm(lay->L, stride, c, rgb) > 0)
                    return c;
        }
    }
    if(rgb)
        return svf::lm_default_choice(lay->L, stride, true);
    return lay->tuned ? lay->choice : svf::lm_default_choice(lay->L, stride);
}

svf_status run_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const LmRun& r)
{
    if(!r.rgb && !lay->tuned && r.texels >= 4096)
        SVF_TRY(tune_lm(ctx, lay, o));
    return launch_lm(ctx, lay, o, r, lm_choice(lay, r.stride, r.rgb));
}

// Consecutive segments whose layouts choose the same kernel configuration
// share a launch, so that every texel is fitted by the configuration of its own
// layout's single fit: a texel's result depends on the number of worker warps
// through the order of its reductions, and this keeps a batch bit-identical to
// fitting its BTFs one by one.
svf_status run_lm_segments(svf_ctx* ctx, Layout* const* lays, const svf_lsq_options* o, const LmRun& r)
{
    const uint32_t n = r.n_seg;
    std::vector<svf::LmKernelChoice> ch(n);
    for(uint32_t i = 0; i < n; ++i)
    {
        if(!r.rgb && !lays[i]->tuned && r.texels >= 4096)
            SVF_TRY(tune_lm(ctx, lays[i], o));
        ch[i] = lm_choice(lays[i], r.seg[i].stride, r.rgb);
    }
    for(uint32_t a = 0; a < n;)
    {
        uint32_t b = a + 1;
        while(b < n && ch[b].threads == ch[a].threads && ch[b].slots == ch[a].slots && ch[b].pass == ch[a].pass)
            ++b;
        LmRun rr = r;
        rr.seg = r.seg + a;
        rr.n_seg = b - a;
        rr.base = r.seg[a].first;
        rr.texels = (b < n ? (uint64_t)r.seg[b].first : r.texels) - r.seg[a].first;
        rr.all_up = true;
        Layout* big = lays[a];
        for(uint32_t i = a; i < b; ++i)
        {
            rr.all_up = rr.all_up && lays[i]->all_up;
            if(lays[i]->L > big->L)
                big = lays[i];
        }
        if(rr.texels > 0)
            SVF_TRY(launch_lm(ctx, big, o, rr, ch[a]));
        a = b;
    }
    return SVF_OK;
}

// The parameters LM holds: the diffuse albedo (at 0) without SVF_LSQ_DIFFUSE,
// the Euler angles with SVF_LSQ_DISABLE_DIRECTION_FITTING (the luminance fit).
void lm_masks(const svf_lsq_options* o, svf::LmConfig& cfg)
{
    cfg.fixed_mask = cfg.zero_mask = 0;
    if(o->flags & SVF_LSQ_RGB)
        return;
    if(!(o->flags & SVF_LSQ_DIFFUSE))
        cfg.fixed_mask = cfg.zero_mask = 1u << 3;
    if(o->flags & SVF_LSQ_DISABLE_DIRECTION_FITTING)
        cfg.fixed_mask |= 0x70u;
}

// Fault injection for the tests of the bounded slab wait, read from the
// environment at each launch: SVF_FAULT_SKIP_SLAB_COPY=<texel> leaves that
// texel's slab copy unissued (its wait runs out: SVF_ETIMEOUT, the texel's status
// SVF_TEXEL_TIMEOUT), SVF_FAULT_WAIT_SPINS=<n> shortens the wait's bound.  No
// GPU fault is involved: the wait is on a barrier that nothing completes.
void lm_fault_injection(svf::LmArgs& a)
{
    a.fault_skip_texel = svf::kLmNoFault;
    a.wait_spins = 0;
    if(const char* e = std::getenv("SVF_FAULT_SKIP_SLAB_COPY"))
        a.fault_skip_texel = (uint32_t)std::strtoul(e, nullptr, 10);
    if(const char* e = std::getenv("SVF_FAULT_WAIT_SPINS"))
        a.wait_spins = (uint32_t)std::strtoul(e, nullptr, 10);
}

svf_status launch_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const LmRun& r, svf::LmKernelChoice c)
{
    svf::LmArgs a{};
    if(r.n_seg == 0)
    {
        a.seg[0] = svf::LmSegment{ 0, lay->L, r.stride, r.lum, lay->geo.as<float>(), r.damping };
        a.n_seg = 1;
        a.L = lay->L;
        a.lum_stride = r.stride;
        a.all_up = lay->all_up ? 1u : 0u;
    }
    else
    {
        if(r.n_seg > (uint32_t)svf::kLmMaxSegments)
            return fail(SVF_EINVAL, "internal: %u LM segments", r.n_seg);
        a.n_seg = r.n_seg;
        for(uint32_t i = 0; i < r.n_seg; ++i)
        {
            a.seg[i] = r.seg[i];
            a.L = std::max(a.L, r.seg[i].L);
            a.lum_stride = std::max<uint64_t>(a.lum_stride, r.seg[i].stride);
        }
        a.all_up = r.all_up ? 1u : 0u;
    }
    a.init = r.init;
    a.out = r.out;
    a.rmse = r.rmse;
    a.stats = r.stats;
    a.avg_chroma = r.avg;
    a.map_diffuse = r.diffuse;
    a.map_specular = r.specular;
    a.map_sigma = r.sigma;
    a.map_basis = r.basis;
    a.texels = (uint32_t)r.texels;
    a.texel_base = r.base;
    a.cfg.max_iter = o->max_iterations;
    a.cfg.mse_target = o->mse_target;
    a.cfg.eps = o->break_on_small_step;
    a.cfg.fresnel = o->fresnel;
    a.cfg.restarts = o->restarts;
    a.cfg.step_per_param = (o->flags & SVF_LSQ_STEP_PER_PARAMETER) ? 1u : 0u;
    a.cfg.row_fit = (o->flags & SVF_LSQ_FIT_TOP) ? 1u : 0u;
    lm_masks(o, a.cfg);
    SVF_TRY(ctx->counter.ensure(16));
    SVF_TRY(ctx->error.ensure(16));
    a.work_counter = ctx->counter.as<uint32_t>();
    a.error_flag = ctx->error.as<uint32_t>();
    lm_fault_injection(a);
    SVF_CUDA(cudaMemsetAsync(ctx->counter.p, 0, 16, ctx->stream));   // the error words are zeroed per call
    a.rgb = r.rgb ? 1u : 0u;
    int per_sm = svf::lm_max_ctas_per_sm(a.L, a.lum_stride, c, r.rgb);
    if(per_sm <= 0)
        return fail(SVF_EINVAL, "the LM kernel (%d threads) does not fit on an SM for L = %u", c.threads, a.L);
    uint64_t grid = std::min<uint64_t>((uint64_t)per_sm * ctx->sms, r.texels);
    SVF_CUDA(svf::launch_lm_fit(a, c, (int)std::max<uint64_t>(grid, 1), ctx->stream));
    return SVF_OK;
}

} // namespace svfh

extern "C" {

svf_status svf_lsq_fit_batch(svf_ctx* ctx, const float* lp, uint32_t L, const float* lum, uint64_t lum_stride,
                             uint32_t texels, const svf_lsq_options* opts, const float* init, float* out, float* rmse,
                             svf_texel_stats* stats)
{
    SVF_TRY(check_ctx(ctx));
    SVF_TRY(check_options(opts, true, true));
    if(opts->flags & SVF_LSQ_RGB)
        return fail(SVF_EINVAL, "the RGB fit (SVF_LSQ_RGB) takes RGB samples: use svf_fit_texels");
    if(!lum || !init || !out || !rmse)
        return fail(SVF_EINVAL, "null lum/init/out/rmse");
    const uint32_t N = L * L;
    if(lum_stride < N)
        return fail(SVF_EINVAL, "lum_stride %llu < L*L = %u", (unsigned long long)lum_stride, N);
    if(texels == 0)
        return SVF_OK;
    Layout* lay = nullptr;
    SVF_TRY(get_layout(ctx, lp, L, &lay));
    const uint64_t stride = round_up(N, 8);
    const uint64_t T = texels;
    SVF_TRY(ctx->lum.ensure(sizeof(float) * stride * T));
    SVF_TRY(ctx->init.ensure(sizeof(float) * 7 * T));
    SVF_TRY(ctx->out.ensure(sizeof(float) * 7 * T));
    SVF_TRY(ctx->rmse.ensure(sizeof(float) * T));
    SVF_TRY(ctx->stats.ensure(sizeof(svf_texel_stats) * T));
    SVF_CUDA(cudaMemcpy2DAsync(ctx->lum.p, sizeof(float) * stride, lum, sizeof(float) * lum_stride, sizeof(float) * N, T,
                               cudaMemcpyDefault, ctx->stream));
    SVF_TRY(to_device(ctx, ctx->init.p, init, sizeof(float) * 7 * T));
    LmRun r{ ctx->lum.as<float>(), stride, ctx->init.as<float>(), ctx->out.as<float>(), ctx->rmse.as<float>(),
             ctx->stats.as<svf_texel_stats>(), nullptr, nullptr, nullptr, nullptr, nullptr, T };
    SVF_TRY(zero_error_flags(ctx));
    const uint32_t n = opts->downsample_light_view;
    DevBuf d_pairs, d_sub;
    if(opts->flags & SVF_LSQ_MULTI_SCATTERING)
        SVF_TRY(run_ms_fit(ctx, lay, opts, ctx->lum.as<float>(), stride, T, ctx->init.as<float>(),
                           ctx->out.as<float>(), ctx->rmse.as<float>(), ctx->stats.as<svf_texel_stats>()));
    else if(opts->flags & SVF_LSQ_FIT_TOP)
    {
        // the top-most view's row (svbrdf-lsq-fitting-setup.cc:291-305: the first
        // direction of least parabolic length, from 1 down)
        uint32_t top = 0;
        float len = 1.0f;
        for(uint32_t v = 0; v < L; ++v)
        {
            const float px = lay->lp[2 * v], py = lay->lp[2 * v + 1];
            const float cur = std::sqrt(px * px + py * py);
            if(cur < len)
            {
                len = cur;
                top = v;
            }
        }
        std::vector<uint32_t> pairs(L);
        for(uint32_t l = 0; l < L; ++l)
            pairs[l] = top * L + l;
        const uint64_t rstride = round_up(L, 8);
        SVF_TRY(upload(d_pairs, pairs));
        SVF_TRY(d_sub.ensure(sizeof(float) * rstride * T));
        SVF_CUDA(svf::launch_gather_pairs(ctx->lum.as<float>(), stride, d_pairs.as<uint32_t>(), L, T,
                                          d_sub.as<float>(), rstride, ctx->stream));
        LmRun rr = r;
        rr.lum = d_sub.p;
        rr.stride = rstride;
        // the row pass (one instance: 256 threads, 2 slots)
        SVF_TRY(launch_lm(ctx, lay, opts, rr, svf::LmKernelChoice{ 256, 2, 3 }));
        svf_lsq_options full = *opts;
        full.flags &= ~SVF_LSQ_FIT_TOP;
        full.max_iterations = 0;
        full.fresnel = 1.0f;
        LmRun rf = r;
        rf.init = ctx->out.as<float>();
        rf.stats = nullptr;
        SVF_TRY(launch_lm(ctx, lay, &full, rf, lm_choice(lay, stride, false)));
    }
    else if(n >= 2 && n < L)
    {
        // DownsampleLightView: the n x n pairs of the kept directions, fitted on
        // their own layout (svbrdf-lsq-fitting-setup.cc:314-330)
        std::vector<uint32_t> idx(n);
        if(!svf::downsample_light_view(L, n, idx.data()))
            return fail(SVF_EINVAL, "downsample_light_view %u of %u directions: no draw", n, L);
        std::vector<float> sub_lp(2 * (size_t)n);
        std::vector<uint32_t> pairs((size_t)n * n);
        for(uint32_t k = 0; k < n; ++k)
        {
            sub_lp[2 * k] = lay->lp[2 * idx[k]];
            sub_lp[2 * k + 1] = lay->lp[2 * idx[k] + 1];
            for(uint32_t l = 0; l < n; ++l)
                pairs[(size_t)k * n + l] = idx[k] * L + idx[l];
        }
        Layout* sub = nullptr;
        SVF_TRY(get_layout(ctx, sub_lp.data(), n, &sub));
        const uint64_t sstride = round_up((uint64_t)n * n, 8);
        SVF_TRY(upload(d_pairs, pairs));
        SVF_TRY(d_sub.ensure(sizeof(float) * sstride * T));
        SVF_CUDA(svf::launch_gather_pairs(ctx->lum.as<float>(), stride, d_pairs.as<uint32_t>(), n * n, T,
                                          d_sub.as<float>(), sstride, ctx->stream));
        LmRun rs = r;
        rs.lum = d_sub.p;
        rs.stride = sstride;
        SVF_TRY(run_lm(ctx, sub, opts, rs));
        // the RMSE the reference reports: all L x L pairs at the fitted parameters,
        // Fresnel 1 (svbrdf-lsq-fitting-setup.cc:403-421)
        svf_lsq_options full = *opts;
        full.max_iterations = 0;
        full.fresnel = 1.0f;
        LmRun rf = r;
        rf.init = ctx->out.as<float>();
        rf.stats = nullptr;
        SVF_TRY(launch_lm(ctx, lay, &full, rf, lm_choice(lay, stride, false)));
    }
    else
        SVF_TRY(run_lm(ctx, lay, opts, r));
    SVF_CUDA(cudaMemcpyAsync(out, ctx->out.p, sizeof(float) * 7 * T, cudaMemcpyDefault, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(rmse, ctx->rmse.p, sizeof(float) * T, cudaMemcpyDefault, ctx->stream));
    if(stats)
        SVF_CUDA(cudaMemcpyAsync(stats, ctx->stats.p, sizeof(svf_texel_stats) * T, cudaMemcpyDefault, ctx->stream));
    SVF_TRY(read_error_flag(ctx));
    if(stats)
    {
        std::vector<svf_texel_stats> st(T);
        if(is_device_pointer(stats))
            SVF_CUDA(cudaMemcpy(st.data(), stats, sizeof(svf_texel_stats) * T, cudaMemcpyDeviceToHost));
        else
            std::memcpy(st.data(), stats, sizeof(svf_texel_stats) * T);
        for(auto& s : st)
            if(s.status & (SVF_TEXEL_NONFINITE | SVF_TEXEL_TIMEOUT))
                return fail(SVF_EPARTIAL, "some texels did not produce a finite fit");
    }
    return SVF_OK;
}

svf_status svf_lsq_fit_batch_noalloc(const float* lp, uint32_t L, const float* lum, uint64_t lum_stride,
                                     uint32_t texels, const svf_lsq_options* opts, const float* init, float* out,
                                     float* rmse, svf_texel_stats* stats, void* stream)
{
    // Nothing here allocates: the checks read pointer attributes, errors go to the
    // fixed per-thread message buffer, the work runs in the static scratch array.
    SVF_TRY(check_options(opts));
    if(opts->flags & SVF_LSQ_RGB)
        return fail(SVF_EINVAL, "the RGB fit (SVF_LSQ_RGB) takes RGB samples: use svf_fit_texels");
    if(L < 3 || L > 160)
        return fail(SVF_EINVAL, "light_count must be in [3, 160], got %u", L);
    const uint64_t N = (uint64_t)L * L;
    if(lum_stride < N)
        return fail(SVF_EINVAL, "lum_stride %llu < L*L = %llu", (unsigned long long)lum_stride, (unsigned long long)N);
    if(texels == 0)
        return SVF_OK;
    const uint64_t slab = round_up(N, 8);
    if((uint64_t)texels * slab > SVF_NOALLOC_MAX_SLAB_FLOATS)
        return fail(SVF_EINVAL,
                    "svf_lsq_fit_batch_noalloc: %u texels of %u directions need %llu slab floats, more than the "
                    "static scratch holds (SVF_NOALLOC_MAX_SLAB_FLOATS = %u, i.e. at most %llu texels here); "
                    "split the batch",
                    texels, L, (unsigned long long)((uint64_t)texels * slab), SVF_NOALLOC_MAX_SLAB_FLOATS,
                    (unsigned long long)(SVF_NOALLOC_MAX_SLAB_FLOATS / slab));
    // device memory of the current device only: a buffer of another GPU (or
    // managed memory) would make the kernels read or write a peer's memory
    int dev = -1;
    SVF_CUDA(cudaGetDevice(&dev));
    const void* must_be_device[] = { lp, lum, init, out, rmse, stats };
    for(int i = 0; i < 6; ++i)
    {
        const void* p = must_be_device[i];
        if(!p && i == 5)
            break;   // stats may be NULL
        if(!is_device_pointer_on(p, dev))
            return fail(SVF_EINVAL,
                        "svf_lsq_fit_batch_noalloc: every buffer must be device memory of the current device "
                        "(device %d; not NULL, not host, managed or another GPU's memory)",
                        dev);
    }
    svf::LmConfig cfg;
    cfg.max_iter = opts->max_iterations;
    cfg.mse_target = opts->mse_target;
    cfg.eps = opts->break_on_small_step;
    cfg.fresnel = opts->fresnel;
    cfg.restarts = opts->restarts;
    cfg.step_per_param = (opts->flags & SVF_LSQ_STEP_PER_PARAMETER) ? 1u : 0u;
    cfg.row_fit = 0;
    lm_masks(opts, cfg);
    if(opts->downsample_light_view || (opts->flags & SVF_LSQ_FIT_TOP))
        return fail(SVF_EINVAL, "svf_lsq_fit_batch_noalloc: no downsampling or top-view fit");
    uint32_t flags[2] = { 0, 0 };
    SVF_CUDA(svf::launch_lm_fit_noalloc(lp, L, lum, lum_stride, texels, cfg, init, out, rmse, stats,
                                        static_cast<cudaStream_t>(stream), flags));
    if(flags[0])
        return fail(SVF_ETIMEOUT, "a bounded device wait expired (a texel slab did not arrive)");
    // the status contract of svf_lsq_fit_batch
    if(flags[1])
        return fail(SVF_EPARTIAL, "some texels did not produce a finite fit");
    return SVF_OK;
}

svf_status svf_lsq_fit_sggx(svf_ctx* ctx, const float* lp, uint32_t L, const float* lum, const svf_lsq_options* opts,
                            const float init[7], float out[7], float* rmse, svf_texel_stats* stats)
{
    svf_texel_stats st{};
    svf_status s = svf_lsq_fit_batch(ctx, lp, L, lum, (uint64_t)L * L, 1, opts, init, out, rmse, &st);
    if(stats)
        *stats = st;
    return s;
}

} // extern "C"
