// svf_host_mlp.cpp - the learned initial guess: the model object, its
// half-vector bins and features, training (tensor-core forward and backward,
// Adam), inference, save and load (svf_mlp_*).
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

// The half-vector bins of a model's direction layout: h = normalize(w_i + w_o)
// of every pair, in parabolic coordinates, on an 8 x 8 grid over the square
// that holds them all.
void mlp_bins(svf_mlp* mlp)
{
    using namespace svf;
    const uint32_t L = mlp->L, N = L * L;
    std::vector<float> w(3 * (size_t)L), hx(N), hy(N);
    for(uint32_t d = 0; d < L; ++d)
        parabolic_to_cartesian_ref(mlp->lp[2 * d], mlp->lp[2 * d + 1], &w[3 * d]);
    float r = 1e-6f;
    for(uint32_t i = 0; i < L; ++i)
        for(uint32_t o = 0; o < L; ++o)
        {
            float h[3] = { w[3 * i] + w[3 * o], w[3 * i + 1] + w[3 * o + 1], w[3 * i + 2] + w[3 * o + 2] };
            const float n = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
            const uint32_t k = i * L + o;
            if(!(n > 1e-6f))
            {
                hx[k] = hy[k] = 1e30f;   // opposite directions: no half vector
                continue;
            }
            for(float& c : h)
                c /= n;
            const float z = 1.0f + std::max(h[2], -0.999f);
            hx[k] = h[0] / z;
            hy[k] = h[1] / z;
            if(hx[k] < 1e29f)
                r = std::max(r, std::max(std::fabs(hx[k]), std::fabs(hy[k])));
        }
    const int G = 8;   // kMlpBins = G * G
    std::vector<uint32_t> bin(N, (uint32_t)kMlpBins);
    std::vector<uint32_t> count(kMlpBins + 1, 0);
    for(uint32_t k = 0; k < N; ++k)
    {
        if(hx[k] > 1e29f)
            continue;
        const int bx = std::min(G - 1, (int)((hx[k] + r) / (2.0f * r) * G));
        const int by = std::min(G - 1, (int)((hy[k] + r) / (2.0f * r) * G));
        bin[k] = (uint32_t)(by * G + bx);   // hx, hy >= -r: bx, by >= 0
        ++count[bin[k]];
    }
    mlp->start.assign(kMlpBins + 1, 0);
    for(int b = 0; b < kMlpBins; ++b)
        mlp->start[b + 1] = mlp->start[b] + count[b];
    mlp->order.assign(mlp->start[kMlpBins], 0);
    std::vector<uint32_t> fill(mlp->start.begin(), mlp->start.end() - 1);
    for(uint32_t k = 0; k < N; ++k)
        if(bin[k] < (uint32_t)kMlpBins)
            mlp->order[fill[bin[k]]++] = k;
    mlp->bin_w.assign(kMlpBins, 0.0f);
    for(int b = 0; b < kMlpBins; ++b)
        mlp->bin_w[b] = count[b] ? 1.0f / (float)count[b] : 0.0f;
    // 16-bit positions: a model's layout has at most 160 directions (25600 pairs)
    mlp->pos.assign(N, 0);
    uint32_t next = mlp->start[kMlpBins];
    for(uint32_t k = 0; k < mlp->start[kMlpBins]; ++k)
        mlp->pos[mlp->order[k]] = (uint16_t)k;
    for(uint32_t k = 0; k < N; ++k)
        if(bin[k] == (uint32_t)kMlpBins)
            mlp->pos[k] = (uint16_t)next++;
    for(int j = 0; j < kMlpPairs; ++j)
        mlp->pair_pos[j] = mlp->pos[mlp->pairs[j]];
}

// Uploads the host-side tables of a model and zeroes its optimiser state.
svf_status mlp_upload(svf_ctx* ctx, svf_mlp* mlp, const std::vector<float>& w)
{
    using namespace svf;
    mlp_bins(mlp);
    SVF_TRY(mlp->d_pos.ensure(sizeof(uint16_t) * std::max<size_t>(1, mlp->pos.size())));
    SVF_TRY(mlp->d_pair_pos.ensure(sizeof(mlp->pair_pos)));
    SVF_TRY(mlp->d_start.ensure(sizeof(uint32_t) * mlp->start.size()));
    SVF_TRY(mlp->d_binw.ensure(sizeof(float) * mlp->bin_w.size()));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_pos.p, mlp->pos.data(), sizeof(uint16_t) * mlp->pos.size(),
                             cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_pair_pos.p, mlp->pair_pos, sizeof(mlp->pair_pos), cudaMemcpyHostToDevice,
                             ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_start.p, mlp->start.data(), sizeof(uint32_t) * mlp->start.size(),
                             cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_binw.p, mlp->bin_w.data(), sizeof(float) * mlp->bin_w.size(),
                             cudaMemcpyHostToDevice, ctx->stream));
    SVF_TRY(mlp->w.ensure(sizeof(float) * kMlpParams));
    SVF_TRY(mlp->g.ensure(sizeof(float) * kMlpParams));
    SVF_TRY(mlp->m.ensure(sizeof(float) * kMlpParams));
    SVF_TRY(mlp->v.ensure(sizeof(float) * kMlpParams));
    SVF_TRY(mlp->tc_hi.ensure(2 * kMlpTcWeights));
    SVF_TRY(mlp->tc_lo.ensure(2 * kMlpTcWeights));
    SVF_TRY(mlp->d_pairs.ensure(sizeof(uint32_t) * kMlpPairs));
    SVF_TRY(mlp->d_xmean.ensure(sizeof(float) * kMlpInputs));
    SVF_TRY(mlp->d_xrstd.ensure(sizeof(float) * kMlpInputs));
    SVF_TRY(mlp->d_ymean.ensure(sizeof(float) * kMlpOutputs));
    SVF_TRY(mlp->d_ystd.ensure(sizeof(float) * kMlpOutputs));
    SVF_CUDA(cudaMemcpyAsync(mlp->w.p, w.data(), sizeof(float) * kMlpParams, cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemsetAsync(mlp->m.p, 0, sizeof(float) * kMlpParams, ctx->stream));
    SVF_CUDA(cudaMemsetAsync(mlp->v.p, 0, sizeof(float) * kMlpParams, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_pairs.p, mlp->pairs, sizeof(mlp->pairs), cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_xmean.p, mlp->xmean, sizeof(mlp->xmean), cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_xrstd.p, mlp->xrstd, sizeof(mlp->xrstd), cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_ymean.p, mlp->ymean, sizeof(mlp->ymean), cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(mlp->d_ystd.p, mlp->ystd, sizeof(mlp->ystd), cudaMemcpyHostToDevice, ctx->stream));
    SVF_CUDA(svf::mlp_pack_weights(mlp->w.as<float>(), mlp->tc_hi.p, mlp->tc_lo.p, ctx->stream));
    mlp->step = 0;
    return SVF_OK;
}

// Training forward pass (FP32) of `rows` normalised inputs X [rows][96] -> Y
// [rows][8]; the hidden activations H1, H2 and their pre-activations Z1, Z2 are
// [rows][256].
svf_status mlp_forward(svf_ctx* ctx, const svf_mlp* mlp, const float* X, int rows, float* Z1, float* H1, float* Z2,
                       float* H2, float* Y)
{
    using namespace svf;
    const float* w = mlp->w.as<float>();
    const int block = 1 << 20;   // rows per launch (the GEMM grid's y extent)
    for(int r0 = 0; r0 < rows; r0 += block)
    {
        const int r = std::min(block, rows - r0);
        const size_t h = (size_t)r0 * kMlpHidden;
        SVF_CUDA(mlp_gemm(false, true, r, kMlpHidden, kMlpInputs, X + (size_t)r0 * kMlpInputs, kMlpInputs,
                          w + kMlpW1, kMlpInputs, H1 + h, kMlpHidden, w + kMlpB1, 1, Z1 ? Z1 + h : nullptr, nullptr,
                          ctx->stream));
        SVF_CUDA(mlp_gemm(false, true, r, kMlpHidden, kMlpHidden, H1 + h, kMlpHidden, w + kMlpW2, kMlpHidden,
                          H2 + h, kMlpHidden, w + kMlpB2, 1, Z2 ? Z2 + h : nullptr, nullptr, ctx->stream));
        SVF_CUDA(mlp_gemm(false, true, r, kMlpOutputs, kMlpHidden, H2 + h, kMlpHidden, w + kMlpW3, kMlpHidden,
                          Y + (size_t)r0 * kMlpOutputs, kMlpOutputs, w + kMlpB3, 0, nullptr, nullptr, ctx->stream));
    }
    return SVF_OK;
}

// Inference of `rows` normalised inputs X [rows][96] -> Y [rows][8] on the
// tensor cores; C, act: scratch of [rows][256] floats each.  A bounded wait that
// expires in a GEMM raises error word 2.
svf_status mlp_infer(svf_ctx* ctx, const svf_mlp* mlp, const float* X, uint64_t rows, float* C, float* act, float* Y)
{
    using namespace svf;
    const uint64_t block = 1ull << 20;   // rows per pass (within the GEMM grid's y extent)
    for(uint64_t r0 = 0; r0 < rows; r0 += block)
    {
        const uint64_t r = std::min(block, rows - r0);
        const cudaError_t e = mlp_forward_tc(X + r0 * kMlpInputs, r, mlp->tc_hi.p, mlp->tc_lo.p, mlp->w.as<float>(),
                                             C + r0 * kMlpHidden, act + r0 * kMlpHidden, Y + r0 * kMlpOutputs,
                                             ctx->error.as<uint32_t>() + 2, ctx->stream);
        if(e != cudaSuccess)
            return fail(SVF_ECUDA, "MLP inference launch: %s", cudaGetErrorString(e));
    }
    return SVF_OK;
}

// Features [n][96] of n texels, normalised with the model's statistics when
// `normalise`.  The bin features come out of the luminance pass (lum_features
// gives its arguments; none for a model of another feature set or without a
// model); the RGB-pair features are read from the samples (rgb_features, which
// does nothing for a bins model).
svf::LumFeatures lum_features(const svf_mlp* mlp, float* X, bool normalise)
{
    svf::LumFeatures f;
    if(!mlp || mlp->features != SVF_MLP_FEATURES_BINS)
        return f;
    f.pos = mlp->d_pos.as<uint16_t>();
    f.start = mlp->d_start.as<uint32_t>();
    f.bin_w = mlp->d_binw.as<float>();
    f.pair_pos = mlp->d_pair_pos.as<uint16_t>();
    f.mean = normalise ? mlp->d_xmean.as<float>() : nullptr;
    f.rstd = normalise ? mlp->d_xrstd.as<float>() : nullptr;
    f.X = X;
    return f;
}

cudaError_t rgb_features(const svf_mlp* mlp, const void* samples, uint32_t sample_type, uint32_t N, uint64_t n,
                         float* X, bool normalise, cudaStream_t stream)
{
    if(!mlp || mlp->features != SVF_MLP_FEATURES_PAIRS_RGB)
        return cudaSuccess;
    return svf::mlp_features_rgb(samples, sample_type, n, N, mlp->d_pairs.as<uint32_t>(),
                                 normalise ? mlp->d_xmean.as<float>() : nullptr,
                                 normalise ? mlp->d_xrstd.as<float>() : nullptr, X, stream);
}

// Scratch of one training step for `rows` rows (in the context).
struct MlpScratch
{
    DevBuf z1, h1, z2, h2, y, dy, dh2, dh1, dsum, loss;
};

// One optimiser step on normalised X [rows][96], T [rows][8]: forward, MSE
// gradient, backward into mlp->g, Adam (or SGD); adds the loss to *loss_dev.
svf_status mlp_train_step(svf_ctx* ctx, svf_mlp* mlp, MlpScratch& s, const float* X, const float* T, int rows,
                          float lr, bool sgd)
{
    using namespace svf;
    const size_t hr = (size_t)rows * kMlpHidden;
    SVF_TRY(s.z1.ensure(sizeof(float) * hr));
    SVF_TRY(s.h1.ensure(sizeof(float) * hr));
    SVF_TRY(s.z2.ensure(sizeof(float) * hr));
    SVF_TRY(s.h2.ensure(sizeof(float) * hr));
    SVF_TRY(s.dh2.ensure(sizeof(float) * hr));
    SVF_TRY(s.dh1.ensure(sizeof(float) * hr));
    SVF_TRY(s.y.ensure(sizeof(float) * rows * kMlpOutputs));
    SVF_TRY(s.dy.ensure(sizeof(float) * rows * kMlpOutputs));
    SVF_TRY(s.dsum.ensure(sizeof(double) * kMlpHidden));
    SVF_TRY(s.loss.ensure(sizeof(double)));
    float *z1 = s.z1.as<float>(), *h1 = s.h1.as<float>(), *z2 = s.z2.as<float>(), *h2 = s.h2.as<float>();
    float *y = s.y.as<float>(), *dy = s.dy.as<float>(), *dh2 = s.dh2.as<float>(), *dh1 = s.dh1.as<float>();
    float* w = mlp->w.as<float>();
    float* g = mlp->g.as<float>();
    SVF_TRY(mlp_forward(ctx, mlp, X, rows, z1, h1, z2, h2, y));
    SVF_CUDA(mlp_mse_grad(y, T, rows, kMlpOutputs, dy, s.loss.as<double>(), ctx->stream));
    // layer 3
    SVF_CUDA(mlp_gemm(true, false, kMlpOutputs, kMlpHidden, rows, dy, kMlpOutputs, h2, kMlpHidden,
                      g + kMlpW3, kMlpHidden, nullptr, 0, nullptr, nullptr, ctx->stream));
    SVF_CUDA(mlp_colsum(dy, rows, kMlpOutputs, s.dsum.as<double>(), nullptr, ctx->stream));
    SVF_CUDA(mlp_to_float(s.dsum.as<double>(), kMlpOutputs, 1.0f, g + kMlpB3, ctx->stream));
    SVF_CUDA(mlp_gemm(false, false, rows, kMlpHidden, kMlpOutputs, dy, kMlpOutputs, w + kMlpW3, kMlpHidden,
                      dh2, kMlpHidden, nullptr, 2, nullptr, z2, ctx->stream));
    // layer 2
    SVF_CUDA(mlp_gemm(true, false, kMlpHidden, kMlpHidden, rows, dh2, kMlpHidden, h1, kMlpHidden,
                      g + kMlpW2, kMlpHidden, nullptr, 0, nullptr, nullptr, ctx->stream));
    SVF_CUDA(mlp_colsum(dh2, rows, kMlpHidden, s.dsum.as<double>(), nullptr, ctx->stream));
    SVF_CUDA(mlp_to_float(s.dsum.as<double>(), kMlpHidden, 1.0f, g + kMlpB2, ctx->stream));
    SVF_CUDA(mlp_gemm(false, false, rows, kMlpHidden, kMlpHidden, dh2, kMlpHidden, w + kMlpW2, kMlpHidden,
                      dh1, kMlpHidden, nullptr, 2, nullptr, z1, ctx->stream));
    // layer 1
    SVF_CUDA(mlp_gemm(true, false, kMlpHidden, kMlpInputs, rows, dh1, kMlpHidden, X, kMlpInputs, g + kMlpW1,
                      kMlpInputs, nullptr, 0, nullptr, nullptr, ctx->stream));
    SVF_CUDA(mlp_colsum(dh1, rows, kMlpHidden, s.dsum.as<double>(), nullptr, ctx->stream));
    SVF_CUDA(mlp_to_float(s.dsum.as<double>(), kMlpHidden, 1.0f, g + kMlpB1, ctx->stream));
    ++mlp->step;
    SVF_CUDA(mlp_adam(w, g, mlp->m.as<float>(), mlp->v.as<float>(), kMlpParams, lr, mlp->step, sgd, ctx->stream));
    return SVF_OK;
}

} // namespace svfh

namespace
{

uint64_t splitmix64(uint64_t& x)
{
    uint64_t z = (x += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

double uniform01(uint64_t& x) { return (double)(splitmix64(x) >> 11) * (1.0 / 9007199254740992.0); }

// 32 direction pairs (sample indices light * L + view): 16 near-mirror pairs
// (the view closest to the light reflected about +z; parabolic (x, y) -> (-x,
// -y)) over randomly drawn lights, then 16 distinct random pairs.
void choose_pairs(const float* lp, uint32_t L, uint64_t seed, uint32_t* pairs)
{
    uint64_t r = seed ^ 0x5f3759dfull;
    const uint32_t N = L * L;
    int k = 0;
    auto taken = [&](uint32_t p) { return std::find(pairs, pairs + k, p) != pairs + k; };
    for(int tries = 0; k < svf::kMlpPairs / 2 && tries < 1000; ++tries)
    {
        const uint32_t i = (uint32_t)(splitmix64(r) % L);
        uint32_t best = 0;
        float bd = 1e30f;
        for(uint32_t o = 0; o < L; ++o)
        {
            const float dx = lp[2 * o] + lp[2 * i], dy = lp[2 * o + 1] + lp[2 * i + 1];
            if(dx * dx + dy * dy < bd)
            {
                bd = dx * dx + dy * dy;
                best = o;
            }
        }
        const uint32_t p = i * L + best;
        if(!taken(p))
            pairs[k++] = p;
    }
    while(k < svf::kMlpPairs)
    {
        const uint32_t p = (uint32_t)(splitmix64(r) % N);
        if(!taken(p) || N <= (uint32_t)k)
            pairs[k++] = p;
    }
}

svf_status check_mlp(svf_ctx* ctx, const svf_mlp* mlp)
{
    SVF_TRY(check_ctx(ctx));
    if(!mlp)
        return fail(SVF_EINVAL, "null model");
    if(mlp->device != ctx->device)
        return fail(SVF_EINVAL, "the model lives on device %d, the context on %d", mlp->device, ctx->device);
    return SVF_OK;
}

constexpr char kMlpMagic[8] = { 'S', 'V', 'F', 'M', 'L', 'P', '0', '2' };

size_t mlp_blob_bytes(uint32_t L)
{
    return sizeof(kMlpMagic) + 3 * sizeof(uint32_t) + sizeof(float) * 2 * L + sizeof(uint32_t) * svf::kMlpPairs +
           sizeof(float) * 2 * (svf::kMlpInputs + svf::kMlpOutputs) + sizeof(float) * svf::kMlpParams;
}

} // namespace

extern "C" {

void svf_mlp_train_options_default(svf_mlp_train_options* o)
{
    if(!o)
        return;
    o->texels = 1u << 20;
    o->seed = 12345;
    o->mix = 1;
    o->epochs = 48;
    o->batch = 4096;
    o->lr = 2e-3f;
    o->max_iterations = 1024;
    o->features = SVF_MLP_FEATURES_BINS;
}

svf_status svf_mlp_train(svf_ctx* ctx, const float* lp, uint32_t L, const svf_mlp_train_options* opts, svf_mlp** out,
                         float* final_loss)
{
    using namespace svf;
    SVF_TRY(check_ctx(ctx));
    if(!out || !lp)
        return fail(SVF_EINVAL, "null output/lights");
    *out = nullptr;
    svf_mlp_train_options o;
    svf_mlp_train_options_default(&o);
    if(opts)
        o = *opts;
    if(L < 3 || L > 160)
        return fail(SVF_EINVAL, "light_count %u outside 3..160", L);
    if(o.texels < 256 || o.texels > (1u << 24) || o.batch < 16 || o.batch > (1u << 16) || o.epochs < 1 ||
       o.epochs > 1000 || !(o.lr > 0.0f) || o.mix > 1 || o.features > SVF_MLP_FEATURES_BINS)
        return fail(SVF_EINVAL, "bad training options (texels 256..2^24, batch 16..65536, epochs 1..1000, lr > 0, "
                                "features 0..1)");
    std::unique_ptr<svf_mlp> mlp(new(std::nothrow) svf_mlp);
    if(!mlp)
        return fail(SVF_ENOMEM, "model allocation failed");
    mlp->device = ctx->device;
    mlp->L = L;
    mlp->features = o.features;
    mlp->lp.resize(2 * (size_t)L);
    SVF_CUDA(cudaMemcpy(mlp->lp.data(), lp, sizeof(float) * 2 * L, cudaMemcpyDefault));
    choose_pairs(mlp->lp.data(), L, o.seed, mlp->pairs);
    // Glorot-uniform weights, zero biases (statistics are filled in below)
    std::vector<float> w(kMlpParams, 0.0f);
    uint64_t r = o.seed * 0x2545f4914f6cdd1dull + 7;
    auto glorot = [&](size_t off, int fan_out, int fan_in) {
        const double a = std::sqrt(6.0 / (fan_in + fan_out));
        for(size_t i = 0; i < (size_t)fan_out * fan_in; ++i)
            w[off + i] = (float)((2.0 * uniform01(r) - 1.0) * a);
    };
    glorot(kMlpW1, kMlpHidden, kMlpInputs);
    glorot(kMlpW2, kMlpHidden, kMlpHidden);
    glorot(kMlpW3, kMlpOutputs, kMlpHidden);
    SVF_TRY(mlp_upload(ctx, mlp.get(), w));

    // training data: synthetic texels fitted by the plain LM from the default guess
    const uint32_t N = L * L, T = o.texels;
    const size_t texel_bytes = sizeof(float) * 3 * (size_t)N;
    const uint32_t gen = (uint32_t)std::max<size_t>(256, std::min<size_t>(65536, (size_t(2) << 30) / texel_bytes));
    const uint64_t stride = round_up(N, 8);
    DevBuf samples, params, X, Y, lum;
    SVF_TRY(samples.ensure(texel_bytes * std::min(gen, T)));
    SVF_TRY(lum.ensure(sizeof(float) * stride * std::min(gen, T)));
    SVF_TRY(params.ensure(sizeof(float) * 7 * std::min(gen, T)));
    SVF_TRY(X.ensure(sizeof(float) * kMlpInputs * (size_t)T));
    SVF_TRY(Y.ensure(sizeof(float) * kMlpOutputs * (size_t)T));
    const svf_layout_desc desc{ mlp->lp.data(), L, nullptr, 0, nullptr, nullptr, 0 };
    svf_fit_options fo{};
    svf_lsq_options_default(&fo.lsq);
    fo.lsq.max_iterations = o.max_iterations;
    fo.init_mode = SVF_INIT_DEFAULT;
    for(uint32_t c0 = 0; c0 < T; c0 += gen)
    {
        const uint32_t n = std::min(gen, T - c0);
        SVF_TRY(svf_synth_btf(ctx, o.seed, o.mix, mlp->lp.data(), L, c0, n, SVF_SAMPLES_F32, 0.0f, samples.p,
                              nullptr));
        const svf_btf_view v{ samples.p, SVF_SAMPLES_F32, n, 1, &desc };
        svf_maps m{};
        m.params = params.as<float>();
        const svf_status st = svf_fit_texels(ctx, &v, &fo, &m, nullptr);
        if(st != SVF_OK && st != SVF_EPARTIAL)
            return st;
        float* Xc = X.as<float>() + (size_t)kMlpInputs * c0;
        SVF_CUDA(launch_luminance(samples.p, SVF_SAMPLES_F32, n, N, lum.as<float>(), stride, nullptr, nullptr,
                                  nullptr, nullptr, ctx->stream, nullptr, 0, lum_features(mlp.get(), Xc, false)));
        SVF_CUDA(rgb_features(mlp.get(), samples.p, SVF_SAMPLES_F32, N, n, Xc, false, ctx->stream));
        SVF_CUDA(mlp_targets(params.as<float>(), n, Y.as<float>() + (size_t)kMlpOutputs * c0, ctx->stream));
    }
    samples.reset();
    lum.reset();
    // input statistics on the device, target statistics (finite rows only) on the host
    DevBuf sums;
    SVF_TRY(sums.ensure(sizeof(double) * 2 * kMlpInputs));
    SVF_CUDA(mlp_colsum(X.as<float>(), (int)T, kMlpInputs, sums.as<double>(), sums.as<double>() + kMlpInputs,
                        ctx->stream));
    std::vector<double> hs(2 * kMlpInputs);
    std::vector<float> hy((size_t)kMlpOutputs * T);
    SVF_CUDA(cudaMemcpyAsync(hs.data(), sums.p, sizeof(double) * 2 * kMlpInputs, cudaMemcpyDeviceToHost, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(hy.data(), Y.p, sizeof(float) * hy.size(), cudaMemcpyDeviceToHost, ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    for(int f = 0; f < kMlpInputs; ++f)
    {
        const double mean = hs[f] / T, var = std::max(0.0, hs[kMlpInputs + f] / T - mean * mean);
        mlp->xmean[f] = (float)mean;
        mlp->xrstd[f] = var > 1e-12 ? (float)(1.0 / std::sqrt(var)) : 1.0f;
    }
    std::vector<uint32_t> valid;
    valid.reserve(T);
    double ys[kMlpOutputs] = {}, ys2[kMlpOutputs] = {};
    for(uint32_t t = 0; t < T; ++t)
    {
        const float* y = hy.data() + (size_t)kMlpOutputs * t;
        bool ok = true;
        for(int k = 0; k < kMlpOutputs; ++k)
            ok = ok && std::isfinite(y[k]);
        if(!ok)
            continue;
        valid.push_back(t);
        for(int k = 0; k < kMlpOutputs; ++k)
        {
            ys[k] += y[k];
            ys2[k] += (double)y[k] * y[k];
        }
    }
    if(valid.size() < o.batch)
        return fail(SVF_EINVAL, "only %zu of %u training texels have a finite fit", valid.size(), T);
    for(int k = 0; k < kMlpOutputs; ++k)
    {
        const double mean = ys[k] / valid.size(), var = std::max(0.0, ys2[k] / valid.size() - mean * mean);
        mlp->ymean[k] = (float)mean;
        mlp->ystd[k] = var > 1e-12 ? (float)std::sqrt(var) : 1.0f;
    }
    for(uint32_t t : valid)
        for(int k = 0; k < kMlpOutputs; ++k)
        {
            float& y = hy[(size_t)kMlpOutputs * t + k];
            y = (y - mlp->ymean[k]) / mlp->ystd[k];
        }
    SVF_CUDA(cudaMemcpyAsync(Y.p, hy.data(), sizeof(float) * hy.size(), cudaMemcpyHostToDevice, ctx->stream));
    // (hy stays alive until the stream is synchronised below)

    SVF_TRY(mlp_upload(ctx, mlp.get(), w));   // with the statistics
    SVF_CUDA(mlp_normalize(X.as<float>(), (int)T, kMlpInputs, mlp->d_xmean.as<float>(), mlp->d_xrstd.as<float>(),
                           ctx->stream));

    // epochs of shuffled minibatches, Adam with a cosine-decayed step size
    const uint32_t V = (uint32_t)valid.size(), B = o.batch;
    const uint32_t per_epoch = (V + B - 1) / B;
    const uint64_t total_steps = (uint64_t)per_epoch * o.epochs;
    DevBuf idx, Xb, Yb;
    SVF_TRY(idx.ensure(sizeof(uint32_t) * V));
    SVF_TRY(Xb.ensure(sizeof(float) * kMlpInputs * B));
    SVF_TRY(Yb.ensure(sizeof(float) * kMlpOutputs * B));
    MlpScratch scratch;
    std::vector<uint32_t> perm(valid);
    uint64_t done = 0;
    for(uint32_t e = 0; e < o.epochs; ++e)
    {
        for(uint32_t i = V - 1; i > 0; --i)
            std::swap(perm[i], perm[splitmix64(r) % (i + 1)]);
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));   // the previous epoch's indices are consumed
        SVF_CUDA(cudaMemcpyAsync(idx.p, perm.data(), sizeof(uint32_t) * V, cudaMemcpyHostToDevice, ctx->stream));
        if(e + 1 == o.epochs)
        {
            SVF_TRY(scratch.loss.ensure(sizeof(double)));
            SVF_CUDA(cudaMemsetAsync(scratch.loss.p, 0, sizeof(double), ctx->stream));
        }
        for(uint32_t b0 = 0; b0 < V; b0 += B, ++done)
        {
            const int rows = (int)std::min(B, V - b0);
            SVF_CUDA(mlp_gather_rows(X.as<float>(), kMlpInputs, Y.as<float>(), kMlpOutputs, idx.as<uint32_t>() + b0,
                                     rows, Xb.as<float>(), Yb.as<float>(), ctx->stream));
            const double f = 0.5 * (1.0 + std::cos(3.14159265358979 * (double)done / (double)total_steps));
            SVF_TRY(mlp_train_step(ctx, mlp.get(), scratch, Xb.as<float>(), Yb.as<float>(), rows,
                                   (float)(o.lr * (0.05 + 0.95 * f)), false));
        }
    }
    SVF_CUDA(mlp_pack_weights(mlp->w.as<float>(), mlp->tc_hi.p, mlp->tc_lo.p, ctx->stream));
    double loss = 0.0;
    SVF_CUDA(cudaMemcpyAsync(&loss, scratch.loss.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    if(final_loss)
        *final_loss = (float)(loss / per_epoch);
    if(!std::isfinite(loss))
        return fail(SVF_ECUDA, "training diverged (non-finite loss)");
    *out = mlp.release();
    return SVF_OK;
}

svf_status svf_mlp_predict(svf_ctx* ctx, const svf_mlp* mlp, const void* samples, uint32_t sample_type,
                           uint32_t texels, float* params, float* features)
{
    using namespace svf;
    SVF_TRY(check_mlp(ctx, mlp));
    if(!samples || !params)
        return fail(SVF_EINVAL, "null samples/params");
    if(sample_type != SVF_SAMPLES_F32 && sample_type != SVF_SAMPLES_F16)
        return fail(SVF_EINVAL, "unknown sample_type %u", sample_type);
    const uint32_t N = mlp->L * mlp->L;
    const size_t texel_bytes = (sample_type == SVF_SAMPLES_F16 ? 2 : 4) * 3 * (size_t)N;
    bool on_device = false;
    SVF_TRY(buffer_location(samples, "samples", &on_device));
    const uint32_t chunk = 65536;
    const uint32_t c = std::min(chunk, texels);
    const uint64_t stride = round_up(N, 8);
    DevBuf staged, x, h1, h2, y, p, lum;
    SVF_TRY(zero_error_flags(ctx));
    if(!on_device)
        SVF_TRY(staged.ensure(texel_bytes * c));
    SVF_TRY(lum.ensure(sizeof(float) * stride * c));
    SVF_TRY(x.ensure(sizeof(float) * kMlpInputs * c));
    SVF_TRY(h1.ensure(sizeof(float) * kMlpHidden * c));
    SVF_TRY(h2.ensure(sizeof(float) * kMlpHidden * c));
    SVF_TRY(y.ensure(sizeof(float) * kMlpOutputs * c));
    SVF_TRY(p.ensure(sizeof(float) * 7 * c));
    for(uint32_t c0 = 0; c0 < texels; c0 += chunk)
    {
        const uint32_t n = std::min(chunk, texels - c0);
        const void* s = static_cast<const char*>(samples) + c0 * texel_bytes;
        if(!on_device)
        {
            SVF_CUDA(cudaMemcpyAsync(staged.p, s, texel_bytes * n, cudaMemcpyHostToDevice, ctx->stream));
            s = staged.p;
        }
        SVF_CUDA(launch_luminance(s, sample_type, n, N, lum.as<float>(), stride, nullptr, nullptr, nullptr, nullptr,
                                  ctx->stream, nullptr, 0, lum_features(mlp, x.as<float>(), true)));
        SVF_CUDA(rgb_features(mlp, s, sample_type, N, n, x.as<float>(), true, ctx->stream));
        SVF_TRY(mlp_infer(ctx, mlp, x.as<float>(), n, h1.as<float>(), h2.as<float>(), y.as<float>()));
        SVF_CUDA(mlp_finish(y.as<float>(), n, mlp->d_ymean.as<float>(), mlp->d_ystd.as<float>(), p.as<float>(),
                            ctx->stream));
        SVF_CUDA(cudaMemcpyAsync(params + (size_t)7 * c0, p.p, sizeof(float) * 7 * n, cudaMemcpyDefault,
                                 ctx->stream));
        if(features)
            SVF_CUDA(cudaMemcpyAsync(features + (size_t)kMlpInputs * c0, x.p, sizeof(float) * kMlpInputs * n,
                                     cudaMemcpyDefault, ctx->stream));
        // staged, x and p are reused by the next chunk
        SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    return read_error_flag(ctx, true);
}

svf_status svf_mlp_step(svf_ctx* ctx, svf_mlp* mlp, const float* features, const float* targets, uint32_t rows,
                        float lr, uint32_t sgd, float* loss)
{
    using namespace svf;
    SVF_TRY(check_mlp(ctx, mlp));
    if(!features || !targets || rows == 0 || rows > (1u << 20))
        return fail(SVF_EINVAL, "null features/targets or rows outside 1..2^20");
    DevBuf X, Y;
    SVF_TRY(X.ensure(sizeof(float) * kMlpInputs * rows));
    SVF_TRY(Y.ensure(sizeof(float) * kMlpOutputs * rows));
    SVF_CUDA(cudaMemcpyAsync(X.p, features, sizeof(float) * kMlpInputs * rows, cudaMemcpyDefault, ctx->stream));
    SVF_CUDA(cudaMemcpyAsync(Y.p, targets, sizeof(float) * kMlpOutputs * rows, cudaMemcpyDefault, ctx->stream));
    MlpScratch s;
    SVF_TRY(s.loss.ensure(sizeof(double)));
    SVF_CUDA(cudaMemsetAsync(s.loss.p, 0, sizeof(double), ctx->stream));
    SVF_TRY(mlp_train_step(ctx, mlp, s, X.as<float>(), Y.as<float>(), (int)rows, lr, sgd != 0));
    SVF_CUDA(mlp_pack_weights(mlp->w.as<float>(), mlp->tc_hi.p, mlp->tc_lo.p, ctx->stream));
    double l = 0.0;
    SVF_CUDA(cudaMemcpyAsync(&l, s.loss.p, sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    if(loss)
        *loss = (float)l;
    return SVF_OK;
}

svf_status svf_mlp_save(const svf_mlp* mlp, void* buf, size_t* size)
{
    using namespace svf;
    if(!mlp || !size)
        return fail(SVF_EINVAL, "null model/size");
    const size_t need = mlp_blob_bytes(mlp->L);
    if(!buf)
    {
        *size = need;
        return SVF_OK;
    }
    if(*size < need)
    {
        *size = need;
        return fail(SVF_EINVAL, "buffer of %zu bytes, %zu needed", *size, need);
    }
    *size = need;
    SVF_CUDA(cudaSetDevice(mlp->device));
    char* c = static_cast<char*>(buf);
    auto put = [&](const void* src, size_t n) {
        std::memcpy(c, src, n);
        c += n;
    };
    const uint32_t hdr[3] = { mlp->L, (uint32_t)kMlpParams, mlp->features };
    put(kMlpMagic, sizeof(kMlpMagic));
    put(hdr, sizeof(hdr));
    put(mlp->lp.data(), sizeof(float) * 2 * mlp->L);
    put(mlp->pairs, sizeof(mlp->pairs));
    put(mlp->xmean, sizeof(mlp->xmean));
    put(mlp->xrstd, sizeof(mlp->xrstd));
    put(mlp->ymean, sizeof(mlp->ymean));
    put(mlp->ystd, sizeof(mlp->ystd));
    // every function that changes the weights synchronises its stream before returning
    SVF_CUDA(cudaMemcpy(c, mlp->w.p, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    return SVF_OK;
}

svf_status svf_mlp_load(svf_ctx* ctx, const void* buf, size_t size, svf_mlp** out)
{
    using namespace svf;
    SVF_TRY(check_ctx(ctx));
    if(!buf || !out)
        return fail(SVF_EINVAL, "null buffer/output");
    *out = nullptr;
    const char* c = static_cast<const char*>(buf);
    uint32_t hdr[3];
    if(size < sizeof(kMlpMagic) + sizeof(hdr) || std::memcmp(c, kMlpMagic, sizeof(kMlpMagic)) != 0)
        return fail(SVF_EINVAL, "not a model (bad magic)");
    std::memcpy(hdr, c + sizeof(kMlpMagic), sizeof(hdr));
    if(hdr[0] < 3 || hdr[0] > 160 || hdr[1] != kMlpParams || hdr[2] > SVF_MLP_FEATURES_BINS ||
       size != mlp_blob_bytes(hdr[0]))
        return fail(SVF_EINVAL, "model header: L %u, %u parameters, %zu bytes (expected %zu parameters)", hdr[0],
                    hdr[1], size, (size_t)kMlpParams);
    std::unique_ptr<svf_mlp> mlp(new(std::nothrow) svf_mlp);
    if(!mlp)
        return fail(SVF_ENOMEM, "model allocation failed");
    mlp->device = ctx->device;
    mlp->L = hdr[0];
    mlp->features = hdr[2];
    mlp->lp.resize(2 * (size_t)mlp->L);
    c += sizeof(kMlpMagic) + sizeof(hdr);
    auto get = [&](void* dst, size_t n) {
        std::memcpy(dst, c, n);
        c += n;
    };
    get(mlp->lp.data(), sizeof(float) * 2 * mlp->L);
    get(mlp->pairs, sizeof(mlp->pairs));
    get(mlp->xmean, sizeof(mlp->xmean));
    get(mlp->xrstd, sizeof(mlp->xrstd));
    get(mlp->ymean, sizeof(mlp->ymean));
    get(mlp->ystd, sizeof(mlp->ystd));
    for(uint32_t p : mlp->pairs)
        if(p >= mlp->L * mlp->L)
            return fail(SVF_EINVAL, "model pair index %u outside the %u samples", p, mlp->L * mlp->L);
    std::vector<float> w(kMlpParams);
    get(w.data(), sizeof(float) * kMlpParams);
    SVF_TRY(mlp_upload(ctx, mlp.get(), w));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = mlp.release();
    return SVF_OK;
}

void svf_mlp_destroy(svf_mlp* mlp)
{
    if(!mlp)
        return;
    cudaSetDevice(mlp->device);
    cudaDeviceSynchronize();
    delete mlp;
}

} // extern "C"
