// svf_host.cpp - the C ABI of libsvf.so (include/svf.h): contexts, direction
// layouts, buffer staging and the launch sequence of a fit.
//
// A fit of texels runs as one stream of kernels:
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
#include "svf_internal.h"
#include "svf_btf_file.h"
#include "svf_layout.h"

namespace
{

// The calling thread's last error message, in a fixed buffer so that reporting
// an error (out-of-memory included) allocates nothing.
thread_local char g_last_error[512];

svf_status fail(svf_status s, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return s;
}

} // namespace

// The last-error reporting for the library's other host files.
namespace svf
{
svf_status host_fail(svf_status s, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return s;
}
} // namespace svf

namespace
{

#define SVF_CUDA(call)                                                                                     \
    do                                                                                                     \
    {                                                                                                      \
        cudaError_t e__ = (call);                                                                          \
        if(e__ != cudaSuccess)                                                                             \
            return fail(e__ == cudaErrorMemoryAllocation ? SVF_ENOMEM : SVF_ECUDA, "%s failed: %s (%s:%d)", \
                        #call, cudaGetErrorString(e__), __FILE__, __LINE__);                               \
    } while(0)

#define SVF_TRY(expr)                 \
    do                                \
    {                                 \
        svf_status s__ = (expr);      \
        if(s__ != SVF_OK)             \
            return s__;               \
    } while(0)

// A grow-only device allocation.
// Bumped whenever a device buffer is (re)allocated: a captured CUDA graph
// holds buffer addresses and is replayed only while this has not changed.
std::atomic<uint64_t> g_buffer_gen{ 1 };

struct DevBuf
{
    void* p = nullptr;
    size_t n = 0;
    svf_status ensure(size_t bytes)
    {
        if(bytes <= n)
            return SVF_OK;
        g_buffer_gen.fetch_add(1);
        if(p)
            cudaFree(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMalloc(&p, bytes);
        if(e != cudaSuccess)
        {
            cudaGetLastError();
            return fail(SVF_ENOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
        }
        n = bytes;
        return SVF_OK;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(p); }
    void reset()
    {
        if(p)
            cudaFree(p);
        p = nullptr;
        n = 0;
    }
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf()
    {
        if(p)
            cudaFree(p);
    }
};

struct PinnedBuf
{
    void* p = nullptr;
    size_t n = 0;
    svf_status ensure(size_t bytes)
    {
        if(bytes <= n)
            return SVF_OK;
        if(p)
            cudaFreeHost(p);
        p = nullptr;
        n = 0;
        cudaError_t e = cudaMallocHost(&p, bytes);
        if(e != cudaSuccess)
        {
            cudaGetLastError();
            return fail(SVF_ENOMEM, "cudaMallocHost(%zu) failed: %s", bytes, cudaGetErrorString(e));
        }
        n = bytes;
        return SVF_OK;
    }
    ~PinnedBuf()
    {
        if(p)
            cudaFreeHost(p);
    }
};

uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull)
{
    const unsigned char* c = static_cast<const unsigned char*>(data);
    for(size_t i = 0; i < bytes; ++i)
    {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

bool is_device_pointer(const void* p)
{
    if(!p)
        return false;
    cudaPointerAttributes a;
    if(cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged;
}

// Plain device memory (not managed, not host) of device `dev`.
bool is_device_pointer_on(const void* p, int dev)
{
    if(!p)
        return false;
    cudaPointerAttributes a;
    if(cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeDevice && a.device == dev;
}

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// Default-init tables of one (direction table, mesh) pair.
struct InitData
{
    svf::InitLayout init{};
    DevBuf op, row_texel, denom_w, pca_cell_id, pca_cell_start, pca_index, pca_frac, pca_dir, proj_dir, proj_frac,
        proj_cell, col_pos, col_of, tile_hi, tile_lo, tile_kb, tile_start;
};

// Interleaves the bits of x and y (x in the even bits).
uint64_t morton2(uint32_t x, uint32_t y)
{
    uint64_t z = 0;
    for(int b = 0; b < 16; ++b)
        z |= (uint64_t)((x >> b) & 1u) << (2 * b) | (uint64_t)((y >> b) & 1u) << (2 * b + 1);
    return z;
}

// The NDF GEMM's column order: pairs lv = view L + light sorted (stably) by the
// Morton code of their half vector's parabolic coordinates on a 256 x 256 grid,
// so that neighbouring columns reach neighbouring NDF texels.
void half_vector_order(const std::vector<float>& lp, uint32_t L, std::vector<uint32_t>& col_of,
                       std::vector<uint16_t>& col_pos)
{
    const uint32_t N = L * L;
    std::vector<float> w(3 * L);
    for(uint32_t d = 0; d < L; ++d)
        svf::parabolic_to_cartesian_ref(lp[2 * d], lp[2 * d + 1], &w[3 * d]);
    std::vector<uint64_t> code(N);
    const auto q = [](double v) { return (uint32_t)std::min(255.0, std::max(0.0, std::floor((v + 1.0) * 128.0))); };
    for(uint32_t v = 0; v < L; ++v)
        for(uint32_t l = 0; l < L; ++l)
        {
            double h[3] = { (double)w[3 * v] + w[3 * l], (double)w[3 * v + 1] + w[3 * l + 1],
                            (double)w[3 * v + 2] + w[3 * l + 2] };
            const double n = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
            double px = 0.0, py = 0.0;
            if(n > 1e-12)
            {
                const double den = 1.0 + h[2] / n;
                if(den > 1e-12)
                {
                    px = h[0] / n / den;
                    py = h[1] / n / den;
                }
            }
            code[v * L + l] = morton2(q(px), q(py));
        }
    col_of.resize(N);
    for(uint32_t k = 0; k < N; ++k)
        col_of[k] = k;
    std::stable_sort(col_of.begin(), col_of.end(), [&](uint32_t a, uint32_t b) { return code[a] < code[b]; });
    col_pos.resize(N);
    for(uint32_t p = 0; p < N; ++p)
        col_pos[col_of[p]] = (uint16_t)p;
}

// Direction layout: LM geometry and, once needed, the default-init tables per
// interpolation mesh (the caller's mesh, or the library's own triangulation).
struct Layout
{
    uint32_t L = 0;
    std::vector<float> lp;
    DevBuf geo;                 // [3][L] Cartesian directions (LM)
    bool all_up = false;        // every direction has z > 0 (LM kernel specialisation)
    std::map<uint64_t, std::unique_ptr<InitData>> inits;
    bool tuned = false;         // LM kernel configuration chosen by the autotuner
    svf::LmKernelChoice choice{ 0, 0 };
};

} // namespace

struct svf_ctx
{
    int device = 0;
    int sms = 0;
    cudaStream_t stream = nullptr;        // compute
    cudaStream_t copy_stream = nullptr;   // host -> device staging of svf_fit_texels
    cudaEvent_t ev[8] = {};
    cudaEvent_t copied[2] = {}, freed[2] = {};   // staging handoff (no timing)
    std::vector<cudaEvent_t> chunk_ev;           // per-chunk phase timing
    // CUDA graph of a repeated svf_fit_texels call (see svf_fit_texels)
    std::vector<uint64_t> graph_key, pending_key;
    cudaGraphExec_t graph_exec = nullptr;
    std::map<uint64_t, std::unique_ptr<Layout>> layouts;
    std::unique_ptr<svf::InitHostTables> tables;
    DevBuf lum, lum_hi, lum_lo, avg, ndf, ndf_tex, init, out, rmse, stats, counter, error, samples, samples2,
        maps_buf, scratch, rgb16, init_rgb, mlp_x, mlp_h1, mlp_h2, mlp_y, fb_idx, fb_lum, fb_hi, fb_lo, fb_ndf,
        fb_small,
        btf_decoded /* svf_fit_btf: the decoded chunk, kept between calls */;
    PinnedBuf pinned;
};

// A learned initial-guess model (svf_mlp_*): FP32 master weights (Adam state
// alongside), the hidden layers' weights split into BF16 hi/lo pairs for the
// tensor-core inference, the normalisation of inputs and
// targets, the 32 direction pairs and the layout it was trained for.
struct svf_mlp
{
    int device = 0;
    uint32_t L = 0;
    uint32_t features = SVF_MLP_FEATURES_BINS;
    std::vector<float> lp;               // [L][2]
    uint32_t pairs[svf::kMlpPairs] = {};
    // half-vector bins of the direction pairs (derived from lp): the pairs of bin
    // b are order[start[b] .. start[b + 1]), their mean is the sum times bin_w[b]
    std::vector<uint32_t> order, start;
    std::vector<float> bin_w;
    // the luminance pass keeps the slab in bin order: pair k at pos[k] (the pairs
    // of bin b at start[b] .. start[b + 1], those with no half vector after
    // them); pair_pos: the single pairs' positions
    std::vector<uint16_t> pos;
    uint16_t pair_pos[svf::kMlpPairs] = {};
    float xmean[svf::kMlpInputs] = {}, xrstd[svf::kMlpInputs] = {};
    float ymean[svf::kMlpOutputs] = {}, ystd[svf::kMlpOutputs] = {};
    // tc_hi, tc_lo: the hidden layers' weights split into BF16 pairs (inference)
    DevBuf w, tc_hi, tc_lo, m, v, g, d_pairs, d_xmean, d_xrstd, d_ymean, d_ystd, d_pos, d_pair_pos, d_start, d_binw;
    int step = 0;
};

namespace
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

svf_status check_ctx(svf_ctx* ctx)
{
    if(!ctx)
        return fail(SVF_EINVAL, "null context");
    cudaError_t e = cudaSetDevice(ctx->device);
    if(e != cudaSuccess)
        return fail(SVF_ECUDA, "cudaSetDevice(%d): %s", ctx->device, cudaGetErrorString(e));
    return SVF_OK;
}

// Initial LM damping relative to the reference's rule for a BTF's fit options:
// the learned guess starts close to a minimum, where the reference's damping
// (sized for its default guess) takes steps below BreakOnSmallStep and stops
// the fit early; it starts lighter unless the caller says otherwise.
constexpr float kMlpInitialDamping = 1e-4f;
float initial_damping(const svf_fit_options& o)
{
    if(o.initial_damping > 0.0f)
        return o.initial_damping;
    return o.init_mode == SVF_INIT_MLP ? kMlpInitialDamping : 1.0f;
}

svf_status check_options(const svf_lsq_options* o, bool downsample_ok = false)
{
    if(!o)
        return fail(SVF_EINVAL, "null options");
    if((o->flags & SVF_LSQ_FIT_TOP) && (!downsample_ok || (o->flags & SVF_LSQ_RGB)))
        return fail(SVF_EINVAL, "SVF_LSQ_FIT_TOP is taken by svf_lsq_fit_sggx / svf_lsq_fit_batch (luminance fit)");
    if(o->downsample_light_view == 1 || (o->downsample_light_view && !downsample_ok) ||
       (o->downsample_light_view && (o->flags & SVF_LSQ_RGB)))
        return fail(SVF_EINVAL, "downsample_light_view %u: 0, or 2 and more with svf_lsq_fit_sggx / svf_lsq_fit_batch",
                    o->downsample_light_view);
    if((o->flags & SVF_LSQ_RGB) && (o->flags & SVF_LSQ_DISABLE_DIRECTION_FITTING || !(o->flags & SVF_LSQ_DIFFUSE)))
        return fail(SVF_EINVAL, "the RGB fit (SVF_LSQ_RGB) fits every parameter, with the diffuse term");
    constexpr uint32_t known = SVF_LSQ_DIFFUSE | SVF_LSQ_RGB | SVF_LSQ_STEP_PER_PARAMETER |
                               SVF_LSQ_DISABLE_DIRECTION_FITTING | SVF_LSQ_FIT_TOP;
    if(o->flags & ~known)
        return fail(SVF_EINVAL, "unknown lsq flags 0x%x", o->flags & ~known);
    if(!(o->fresnel >= 1.0f) || !std::isfinite(o->fresnel))
        return fail(SVF_EINVAL, "fresnel (refractive index) must be >= 1, got %g", o->fresnel);
    if(!(o->mse_target >= 0.0) || !(o->break_on_small_step > 0.0))
        return fail(SVF_EINVAL, "mse_target must be >= 0 and break_on_small_step > 0");
    if(o->restarts > 16)
        return fail(SVF_EINVAL, "restarts must be <= 16, got %u", o->restarts);
    return SVF_OK;
}

svf_status get_layout(svf_ctx* ctx, const float* lp_in, uint32_t L, Layout** out)
{
    if(L < 3 || L > 160)
        return fail(SVF_EINVAL, "light_count must be in [3, 160], got %u", L);
    if(!lp_in)
        return fail(SVF_EINVAL, "null lights_parabolic");
    std::vector<float> lp(2 * L);
    if(is_device_pointer(lp_in))
        SVF_CUDA(cudaMemcpy(lp.data(), lp_in, sizeof(float) * 2 * L, cudaMemcpyDeviceToHost));
    else
        std::memcpy(lp.data(), lp_in, sizeof(float) * 2 * L);
    for(float x : lp)
        if(!std::isfinite(x))
            return fail(SVF_EINVAL, "non-finite direction coordinate");
    uint64_t key = fnv1a(lp.data(), lp.size() * sizeof(float), L);
    auto it = ctx->layouts.find(key);
    if(it == ctx->layouts.end())
    {
        auto lay = std::make_unique<Layout>();
        lay->L = L;
        lay->lp = lp;
        std::vector<float> geo(3 * L);
        for(uint32_t d = 0; d < L; ++d)
        {
            float w[3];
            svf::parabolic_to_cartesian_ref(lp[2 * d], lp[2 * d + 1], w);
            geo[d] = w[0];
            geo[L + d] = w[1];
            geo[2 * L + d] = w[2];
        }
        lay->all_up = true;
        for(uint32_t d = 0; d < L; ++d)
            lay->all_up = lay->all_up && geo[2 * L + d] > 0.0f;
        SVF_TRY(lay->geo.ensure(sizeof(float) * 3 * L));
        SVF_CUDA(cudaMemcpy(lay->geo.p, geo.data(), sizeof(float) * 3 * L, cudaMemcpyHostToDevice));
        it = ctx->layouts.emplace(key, std::move(lay)).first;
    }
    *out = it->second.get();
    return SVF_OK;
}

template <typename T>
svf_status upload(DevBuf& dst, const std::vector<T>& v)
{
    SVF_TRY(dst.ensure(std::max<size_t>(sizeof(T) * v.size(), 16)));
    SVF_CUDA(cudaMemcpy(dst.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return SVF_OK;
}

// Builds (once per mesh) the default-init tables of a layout, with the given
// mesh or the library's own triangulation.
svf_status prepare_init(svf_ctx* ctx, Layout* lay, const svf_layout_desc* desc, const svf::InitLayout** out)
{
    const uint32_t L = lay->L, N = L * L;
    uint64_t key = 0;   // 0: the library's triangulation
    if(desc->triangles)
    {
        if(desc->triangle_count == 0 || !desc->edges || !desc->edge_angles || desc->edge_count == 0)
            return fail(SVF_EINVAL, "a given mesh needs triangles, edges and edge angles");
        key = fnv1a(desc->triangles, sizeof(uint32_t) * 3 * (size_t)desc->triangle_count);
        key = fnv1a(desc->edges, sizeof(uint32_t) * 3 * (size_t)desc->edge_count, key);
        key = fnv1a(desc->edge_angles, sizeof(float) * 2 * (size_t)desc->edge_count, key) | 1u;
    }
    auto found = lay->inits.find(key);
    if(found != lay->inits.end())
    {
        *out = &found->second->init;
        return SVF_OK;
    }
    std::vector<uint32_t> tris, edges;
    std::vector<float> eang;
    if(desc->triangles)
    {
        tris.assign(desc->triangles, desc->triangles + 3 * (size_t)desc->triangle_count);
        edges.assign(desc->edges, desc->edges + 3 * (size_t)desc->edge_count);
        eang.assign(desc->edge_angles, desc->edge_angles + 2 * (size_t)desc->edge_count);
        for(uint32_t v : tris)
            if(v >= L)
                return fail(SVF_EINVAL, "triangle vertex %u out of range", v);
        for(size_t i = 0; i < edges.size(); i += 3)
            if(edges[i] >= L || edges[i + 1] >= L || edges[i + 2] >= desc->triangle_count)
                return fail(SVF_EINVAL, "edge %zu out of range", i / 3);
    }
    else
    {
        if(!svf::delaunay(lay->lp.data(), L, tris))
            return fail(SVF_EINVAL, "Delaunay triangulation of the directions failed");
        svf::boundary_edges(lay->lp.data(), tris, edges, eang);
    }
    if(!ctx->tables)
    {
        ctx->tables = std::make_unique<svf::InitHostTables>();
        svf::build_init_host_tables(*ctx->tables);
    }
    const svf::InitHostTables& t = *ctx->tables;
    auto data = std::make_unique<InitData>();
    InitData* dd = data.get();
    svf::InitLayout& il = dd->init;
    il.L = L;
    il.N = N;
    il.k_pad = (uint32_t)round_up(N, 8);
    il.ndf_rows = (uint32_t)t.ndf_row_texel.size();
    il.ndf_rows_pad = (uint32_t)round_up(il.ndf_rows, 256);
    SVF_TRY(dd->op.ensure(sizeof(float) * il.ndf_rows_pad * (size_t)il.k_pad));
    SVF_CUDA(cudaMemset(dd->op.p, 0, sizeof(float) * il.ndf_rows_pad * (size_t)il.k_pad));
    // operator rows in Morton order of their NDF texel (a 256-row tile is then a
    // compact block of the texture)
    std::vector<uint32_t> row_order(il.ndf_rows);
    for(uint32_t r = 0; r < il.ndf_rows; ++r)
        row_order[r] = r;
    std::stable_sort(row_order.begin(), row_order.end(), [&](uint32_t a, uint32_t b) {
        const int32_t ta = t.ndf_row_texel[a], tb = t.ndf_row_texel[b];
        return morton2((uint32_t)(ta % svf::kNdfRes), (uint32_t)(ta / svf::kNdfRes)) <
               morton2((uint32_t)(tb % svf::kNdfRes), (uint32_t)(tb / svf::kNdfRes));
    });
    std::vector<int32_t> row_texel(il.ndf_rows);
    std::vector<float> row_normal(3 * (size_t)il.ndf_rows);
    for(uint32_t r = 0; r < il.ndf_rows; ++r)
    {
        row_texel[r] = t.ndf_row_texel[row_order[r]];
        for(int c = 0; c < 3; ++c)
            row_normal[3 * r + c] = t.ndf_row_normal[3 * row_order[r] + c];
    }
    SVF_TRY(upload(dd->row_texel, row_texel));
    SVF_TRY(upload(dd->denom_w, t.denom_w));
    SVF_TRY(upload(dd->pca_cell_id, t.pca_cell_id));
    SVF_TRY(upload(dd->pca_cell_start, t.pca_cell_start));
    SVF_TRY(upload(dd->pca_index, t.pca_index));
    SVF_TRY(upload(dd->pca_frac, t.pca_frac));
    SVF_TRY(upload(dd->pca_dir, t.pca_dir));
    SVF_TRY(upload(dd->proj_dir, t.proj_dir));
    SVF_TRY(upload(dd->proj_frac, t.proj_frac));
    SVF_TRY(upload(dd->proj_cell, t.proj_cell));
    il.ndf_op = dd->op.as<float>();
    il.ndf_row_texel = dd->row_texel.as<int32_t>();
    il.denom_w = dd->denom_w.as<float>();
    il.pca_cells = (uint32_t)t.pca_cell_id.size();
    il.pca_cell_id = dd->pca_cell_id.as<int32_t>();
    il.pca_cell_start = dd->pca_cell_start.as<uint32_t>();
    il.pca_index = dd->pca_index.as<uint32_t>();
    il.pca_frac = dd->pca_frac.as<float2>();
    il.pca_dir = dd->pca_dir.as<float4>();
    il.proj_dir = dd->proj_dir.as<float4>();
    il.proj_frac = dd->proj_frac.as<float2>();
    il.proj_cell = dd->proj_cell.as<int32_t>();
    il.rot_s = t.rot_s;
    il.rot_c = t.rot_c;
    il.pdf = t.pdf;
    il.axis_cell = t.axis_cell;
    il.axis_fx1 = t.axis_frac[0];
    il.axis_fy1 = t.axis_frac[1];

    // the NDF operator, built on the device
    DevBuf d_lp, d_tri, d_edges, d_eang, d_dirs, d_normals, d_ltri, d_lbary;
    SVF_TRY(upload(d_lp, lay->lp));
    SVF_TRY(upload(d_tri, tris));
    SVF_TRY(upload(d_edges, edges));
    SVF_TRY(upload(d_eang, eang));
    SVF_TRY(upload(d_dirs, t.ndf_dirs));
    SVF_TRY(upload(d_normals, row_normal));
    SVF_TRY(d_ltri.ensure(sizeof(int32_t) * svf::kNdfSamples));
    SVF_TRY(d_lbary.ensure(sizeof(float) * 3 * svf::kNdfSamples));
    svf::MeshDevice mesh{ d_lp.as<float>(), d_tri.as<uint32_t>(), (uint32_t)(tris.size() / 3), d_edges.as<uint32_t>(),
                          d_eang.as<float>(), (uint32_t)(edges.size() / 3) };
    SVF_CUDA(svf::launch_ndf_operator(il, mesh, d_dirs.as<float>(), d_normals.as<float>(), t.ndf_scale,
                                      d_ltri.as<int32_t>(), d_lbary.as<float>(), ctx->stream));
    // its non-empty 256 x 64 tiles (columns in half-vector order), packed as the
    // BF16 hi/lo split for the tensor-core GEMM
    std::vector<uint32_t> col_of;
    std::vector<uint16_t> col_pos;
    half_vector_order(lay->lp, L, col_of, col_pos);
    SVF_TRY(upload(dd->col_of, col_of));
    SVF_TRY(upload(dd->col_pos, col_pos));
    il.col_of = dd->col_of.as<uint32_t>();
    il.col_pos = dd->col_pos.as<uint16_t>();
    const uint32_t ktiles = (N + 63) / 64, ntiles = il.ndf_rows_pad / 256;
    DevBuf d_flags;
    SVF_TRY(d_flags.ensure(sizeof(uint32_t) * ktiles * ntiles));
    SVF_CUDA(svf::launch_ndf_tile_flags(il.ndf_op, il.k_pad, il.col_of, N, il.ndf_rows_pad, d_flags.as<uint32_t>(),
                                        ctx->stream));
    std::vector<uint32_t> flags(ktiles * ntiles);
    SVF_CUDA(cudaMemcpyAsync(flags.data(), d_flags.p, sizeof(uint32_t) * flags.size(), cudaMemcpyDeviceToHost,
                             ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<uint32_t> tile_n, tile_kb, tile_start(ntiles + 1, 0);
    for(uint32_t n = 0; n < ntiles; ++n)
    {
        tile_start[n] = (uint32_t)tile_kb.size();
        for(uint32_t kb = 0; kb < ktiles; ++kb)
            if(flags[n * ktiles + kb])
            {
                tile_n.push_back(n);
                tile_kb.push_back(kb);
            }
    }
    tile_start[ntiles] = (uint32_t)tile_kb.size();
    il.packed_tiles = (uint32_t)tile_kb.size();
    if(il.packed_tiles == 0)
    {
        // an operator without a non-zero: one zero tile that no row tile lists
        tile_n.push_back(0);
        tile_kb.push_back(0);
    }
    const uint32_t alloc_tiles = (uint32_t)tile_kb.size();
    DevBuf d_tile_n;
    SVF_TRY(upload(d_tile_n, tile_n));
    SVF_TRY(upload(dd->tile_kb, tile_kb));
    SVF_TRY(upload(dd->tile_start, tile_start));
    SVF_TRY(dd->tile_hi.ensure(sizeof(uint16_t) * 256 * 64 * (size_t)alloc_tiles));
    SVF_TRY(dd->tile_lo.ensure(sizeof(uint16_t) * 256 * 64 * (size_t)alloc_tiles));
    if(il.packed_tiles == 0)
    {
        SVF_CUDA(cudaMemsetAsync(dd->tile_hi.p, 0, sizeof(uint16_t) * 256 * 64, ctx->stream));
        SVF_CUDA(cudaMemsetAsync(dd->tile_lo.p, 0, sizeof(uint16_t) * 256 * 64, ctx->stream));
    }
    else
        SVF_CUDA(svf::launch_ndf_tile_pack(il.ndf_op, il.k_pad, il.col_of, N, d_tile_n.as<uint32_t>(),
                                           dd->tile_kb.as<uint32_t>(), il.packed_tiles, dd->tile_hi.p, dd->tile_lo.p,
                                           ctx->stream));
    il.packed_tiles = alloc_tiles;
    il.nonempty_tiles = tile_start[ntiles];
    il.all_tiles = ktiles * ntiles;
    il.tile_hi = dd->tile_hi.p;
    il.tile_lo = dd->tile_lo.p;
    il.tile_kb = dd->tile_kb.as<uint32_t>();
    il.tile_start = dd->tile_start.as<uint32_t>();
    if(getenv("SVF_DEBUG"))
        fprintf(stderr, "svf: NDF operator L=%u: %u of %u tiles non-empty (%.1f%%)\n", L, tile_start[ntiles],
                ktiles * ntiles, 100.0 * tile_start[ntiles] / (ktiles * ntiles));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    *out = &dd->init;
    lay->inits.emplace(key, std::move(data));
    return SVF_OK;
}

// The NDF rows of `texels` luminance splits (columns in the operator's order) on
// the tensor cores, over the operator's non-empty tiles.
cudaError_t launch_ndf(const svf::InitLayout& il, const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda,
                       float* C, uint32_t ldc, uint32_t* error_flag, cudaStream_t stream)
{
    return svf::launch_ndf_tc_tiles(a_hi, a_lo, texels, lda, il.tile_hi, il.tile_lo, il.ndf_rows_pad, il.k_pad, il.N,
                                    C, ldc, error_flag, stream, il.tile_kb, il.tile_start, il.packed_tiles);
}

// Copies `bytes` from src (host or device) to the device buffer dst.
svf_status to_device(svf_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    SVF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
    return SVF_OK;
}

struct LmRun
{
    const void* lum;       // device, padded slabs (FP32 luminance; FP16 RGB for the RGB fit)
    uint64_t stride;       // slab elements
    const float* init;     // device [T][7] ([T][12] RGB)
    float* out;            // device [T][7] ([T][12] RGB)
    float* rmse;           // device [T]
    svf_texel_stats* stats;
    const float* avg;
    float *diffuse, *specular, *sigma, *basis;
    uint64_t texels;
    // several layouts in one launch (svf_fit_btfs): segments replace lum/stride
    // and the layout's table; all_up over all of them
    const svf::LmSegment* seg = nullptr;
    uint32_t n_seg = 0;
    bool all_up = false;
    bool rgb = false;      // the 11-parameter RGB fit
    float damping = 0.0f;  // initial damping scale of a single-segment run (0: the reference's rule)
};

svf_status launch_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const LmRun& r, svf::LmKernelChoice c);
svf_status read_error_flag(svf_ctx* ctx, bool with_ndf = false);

// Autotuner of the LM kernel configuration (CTA size and texel slots), once per
// layout: each candidate fits the same seeded synthetic probe (8192 texels of
// the uneven parameter mix, from a perturbed ground truth) and is scored by
// model flops per second (the flops per Jacobian and residual pass times the
// passes it ran, over its CUDA-event time).  The first candidate is kept unless
// another is more than 3% faster.  Tuning on a fixed probe, not on the caller's
// texels, keeps every texel of a call on one configuration.
svf_status tune_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o)
{
    if(lay->tuned || std::getenv("SVF_LM_KERNEL"))   // (a pinned configuration needs no probe)
        return SVF_OK;
    // the plain passes only: the packed pass (one 256-thread CTA per SM at its
    // register count) wins on this short probe but loses on full launches
    // (measured: 59.4 against 52.2 ms for 160000 ring-81 texels), so it is left
    // to SVF_LM_KERNEL
    svf::LmKernelChoice cand[4];
    const int n_cand = svf::lm_candidates(lay->L, cand, 4);
    lay->choice = cand[0];
    if(n_cand <= 1)
    {
        lay->tuned = true;
        return SVF_OK;
    }
    const uint32_t L = lay->L, N = L * L;
    // enough texels to keep every slot of every resident CTA busy for a while
    const uint64_t stride = round_up(N, 8), T = 8192;
    DevBuf samples, truth, lum, avg, init, out, rmse, stats;
    SVF_TRY(samples.ensure(sizeof(float) * 3 * N * T));
    SVF_TRY(truth.ensure(sizeof(float) * 16 * T));
    SVF_TRY(lum.ensure(sizeof(float) * stride * T));
    SVF_TRY(avg.ensure(sizeof(float) * 3 * T));
    SVF_TRY(init.ensure(sizeof(float) * 7 * T));
    SVF_TRY(out.ensure(sizeof(float) * 7 * T));
    SVF_TRY(rmse.ensure(sizeof(float) * T));
    SVF_TRY(stats.ensure(sizeof(svf_texel_stats) * T));
    DevBuf d_lp;
    SVF_TRY(upload(d_lp, lay->lp));
    SVF_CUDA(svf::launch_synth(0x5EEDu, 1, d_lp.as<float>(), L, 0, T, SVF_SAMPLES_F32, 0.01f, samples.p,
                               truth.as<float>(), ctx->stream));
    SVF_CUDA(svf::launch_luminance(samples.p, SVF_SAMPLES_F32, T, N, lum.as<float>(), stride, avg.as<float>(),
                                   nullptr, nullptr, nullptr, ctx->stream));
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
    for(int c = 0; c < n_fit; ++c)
    {
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
        if(c == 0)
            first_rate = rate;
        if(rate > best_rate)
        {
            best_rate = rate;
            best = c;
        }
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

// Error words: [0] LM kernel, [2] tensor-core GEMMs (NDF operator, MLP).  Zeroed once per call, so that a
// flag raised by any launch of the call is seen.
svf_status zero_error_flags(svf_ctx* ctx)
{
    SVF_TRY(ctx->error.ensure(16));
    SVF_CUDA(cudaMemsetAsync(ctx->error.p, 0, 16, ctx->stream));
    return SVF_OK;
}

svf_status read_error_flag(svf_ctx* ctx, bool with_ndf)
{
    uint32_t flag[3] = {};
    SVF_CUDA(cudaMemcpyAsync(flag, ctx->error.p, sizeof(flag), cudaMemcpyDeviceToHost, ctx->stream));
    SVF_CUDA(cudaStreamSynchronize(ctx->stream));
    if(flag[0])
        return fail(SVF_ETIMEOUT, "a bounded device wait expired (a texel slab did not arrive)");
    if(with_ndf && flag[2])
        return fail(SVF_ETIMEOUT, "a bounded device wait expired in a tensor-core GEMM");
    return SVF_OK;
}

} // namespace

// ============================================================================
// C ABI
// ============================================================================

extern "C" {

uint32_t svf_abi_version(void) { return SVF_ABI_VERSION; }

const char* svf_status_string(svf_status s)
{
    switch(s)
    {
    case SVF_OK: return "ok";
    case SVF_EINVAL: return "invalid argument";
    case SVF_ENOMEM: return "out of memory";
    case SVF_ECUDA: return "CUDA error";
    case SVF_ETIMEOUT: return "bounded device wait expired";
    case SVF_EPARTIAL: return "some texels failed";
    case SVF_ENODEV: return "no sm_100 device";
    }
    return "unknown status";
}

const char* svf_last_error(void) { return g_last_error; }

void svf_lsq_options_default(svf_lsq_options* o)
{
    if(!o)
        return;
    o->max_iterations = 1024;            // CurveFitSteps
    o->fresnel = 1.0f;
    o->flags = SVF_LSQ_DIFFUSE | SVF_LSQ_STEP_PER_PARAMETER;
    o->mse_target = 1e-6;
    o->break_on_small_step = (double)1e-3f;   // settings.BreakOnSmallStep = 1e-3f
    o->restarts = 1;
    o->downsample_light_view = 0;   // DownSampleLightView = ~0u: all directions
}

uint32_t svf_downsample_light_view(uint32_t L, uint32_t n, uint32_t* idx)
{
    if(!idx || !svf::downsample_light_view(L, n, idx))
        return 0;
    return n;
}

svf_status svf_create(int device, svf_ctx** out)
{
    if(!out)
        return fail(SVF_EINVAL, "null output pointer");
    *out = nullptr;
    int count = 0;
    if(cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count)
    {
        cudaGetLastError();
        return fail(SVF_ENODEV, "CUDA device %d not available", device);
    }
    cudaDeviceProp prop;
    if(cudaGetDeviceProperties(&prop, device) != cudaSuccess)
    {
        cudaGetLastError();
        return fail(SVF_ENODEV, "cannot query device %d", device);
    }
    if(prop.major != 10)
        return fail(SVF_ENODEV, "device %d is sm_%d%d; this library is built for sm_100a", device, prop.major,
                    prop.minor);
    std::unique_ptr<svf_ctx> ctx(new(std::nothrow) svf_ctx);
    if(!ctx)
        return fail(SVF_ENOMEM, "context allocation failed");
    ctx->device = device;
    ctx->sms = prop.multiProcessorCount;
    SVF_CUDA(cudaSetDevice(device));
    SVF_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    SVF_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    for(auto& e : ctx->ev)
        SVF_CUDA(cudaEventCreate(&e));
    for(int i = 0; i < 2; ++i)
    {
        SVF_CUDA(cudaEventCreateWithFlags(&ctx->copied[i], cudaEventDisableTiming));
        SVF_CUDA(cudaEventCreateWithFlags(&ctx->freed[i], cudaEventDisableTiming));
    }
    // the LM's work counter and the error words, for the context's lifetime
    SVF_TRY(ctx->counter.ensure(16));
    SVF_TRY(ctx->error.ensure(16));
    *out = ctx.release();
    return SVF_OK;
}

void svf_destroy(svf_ctx* ctx)
{
    if(!ctx)
        return;
    cudaSetDevice(ctx->device);
    if(ctx->stream)
        cudaStreamSynchronize(ctx->stream);
    if(ctx->copy_stream)
        cudaStreamSynchronize(ctx->copy_stream);
    for(auto& e : ctx->ev)
        if(e)
            cudaEventDestroy(e);
    for(int i = 0; i < 2; ++i)
    {
        if(ctx->copied[i])
            cudaEventDestroy(ctx->copied[i]);
        if(ctx->freed[i])
            cudaEventDestroy(ctx->freed[i]);
    }
    for(auto e : ctx->chunk_ev)
        cudaEventDestroy(e);
    if(ctx->graph_exec)
        cudaGraphExecDestroy(ctx->graph_exec);
    if(ctx->copy_stream)
        cudaStreamDestroy(ctx->copy_stream);
    if(ctx->stream)
        cudaStreamDestroy(ctx->stream);
    delete ctx;
}

uint32_t svf_directions_ring81(float* lp)
{
    if(!lp)
        return 0;
    return svf::ring81_directions(lp);
}

uint32_t svf_directions_fibonacci(uint32_t count, float* lp)
{
    if(!lp || count == 0)
        return 0;
    return svf::fibonacci_directions(count, lp);
}

uint32_t svf_layout_triangulate(const float* lp, uint32_t L, uint32_t* triangles, uint32_t* edges, float* edge_angles,
                                uint32_t* edge_count)
{
    if(!lp || L < 3 || !triangles || !edges || !edge_angles || !edge_count)
        return 0;
    std::vector<uint32_t> tris, e;
    std::vector<float> a;
    if(!svf::delaunay(lp, L, tris))
        return 0;
    uint32_t ne = svf::boundary_edges(lp, tris, e, a);
    std::copy(tris.begin(), tris.end(), triangles);
    std::copy(e.begin(), e.end(), edges);
    std::copy(a.begin(), a.end(), edge_angles);
    *edge_count = ne;
    return (uint32_t)(tris.size() / 3);
}

svf_status svf_lsq_fit_batch(svf_ctx* ctx, const float* lp, uint32_t L, const float* lum, uint64_t lum_stride,
                             uint32_t texels, const svf_lsq_options* opts, const float* init, float* out, float* rmse,
                             svf_texel_stats* stats)
{
    SVF_TRY(check_ctx(ctx));
    SVF_TRY(check_options(opts, true));
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
    if(opts->flags & SVF_LSQ_FIT_TOP)
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
        SVF_TRY(launch_lm(ctx, lay, opts, rr, lm_choice(lay, rstride, false)));
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
    const bool samples_on_device = is_device_pointer(btf->samples);
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
        x.on_device = is_device_pointer(v.samples);
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
            Layout* lbig = it[ch[0].b].lay;
            bool lup = true;
            uint64_t lstride = 0;
            for(size_t i = 0; i < ch.size(); ++i)
            {
                const Item& x = it[ch[i].b];
                ls[i] = svf::LmSegment{ (uint32_t)ch[i].k0, x.lay->L, x.stride, ctx->lum.as<float>() + ch[i].off,
                                        x.lay->geo.as<float>(), initial_damping(opts[ch[i].b]) };
                lup = lup && x.lay->all_up;
                lstride = std::max(lstride, x.stride);
                if(x.lay->L > lbig->L)
                    lbig = x.lay;
            }
            LmRun lr{ nullptr, lstride, ctx->init.as<float>(), ctx->out.as<float>(), ctx->rmse.as<float>(),
                      ctx->stats.as<svf_texel_stats>(), nullptr, nullptr, nullptr, nullptr, nullptr, n,
                      ls, (uint32_t)ch.size(), lup, false };
            SVF_TRY(run_lm(ctx, lbig, &opts[0].lsq, lr));
            for(auto& p : ch)
                if(it[p.b].default_init || it[p.b].mlp)
                    SVF_CUDA(svf::launch_rgb_init(ctx->out.as<float>() + 7 * p.k0, ctx->avg.as<float>() + 3 * p.k0,
                                                  p.count, init_used + 12 * p.k0, ctx->stream));
        }
        SVF_CUDA(cudaEventRecord(ctx->ev[2], ctx->stream));
        // one LM launch over the pieces, whatever their layouts
        svf::LmSegment seg[svf::kLmMaxSegments];
        Layout* big = it[ch[0].b].lay;
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
            if(x.lay->L > big->L)
                big = x.lay;
        }
        float* mb = ctx->maps_buf.as<float>();
        LmRun r{ nullptr, max_stride, init_used, ctx->out.as<float>(), ctx->rmse.as<float>(),
                 ctx->stats.as<svf_texel_stats>(), ctx->avg.as<float>(), mb, mb + 3 * n, mb + 6 * n, mb + 8 * n, n,
                 seg, (uint32_t)ch.size(), all_up, rgb };
        SVF_TRY(run_lm(ctx, big, &opts[0].lsq, r));
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
    if(!is_device_pointer(samples))
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
    const bool truth_host = truth && !is_device_pointer(truth);
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

// ---- learned initial guess ------------------------------------------------------

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
    const bool on_device = is_device_pointer(samples);
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

// ---- factored BTF files -------------------------------------------------------------

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
    if(is_device_pointer(samples))
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
    const bool out_dev = is_device_pointer(samples);
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
    const bool on_device = is_device_pointer(btf->samples);
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
