// svf_host.h - what the host files of libsvf.so share: the objects behind the
// C ABI's handles (svf_ctx, svf_mlp), device and pinned buffers, direction
// layouts, error reporting, and the steps of the launch sequence that more
// than one entry point takes.
//   svf_host.cpp       errors, contexts, options, layouts, error words; the ABI's core
//   svf_host_init.cpp  the default-init tables of a layout (NDF operator, PCA and
//                      projection tables, the NDF GEMM's tile lists)
//   svf_host_lm.cpp    the persistent LM launch and its autotuner; svf_lsq_fit_*
//   svf_host_fit.cpp   svf_fit_texels, svf_fit_btfs, svf_synth_btf
//   svf_host_mlp.cpp   the learned initial guess (svf_mlp_*)
//   svf_host_btf.cpp   factored BTF files, error maps, rendering, neighbourhood refit
//   svf_host_ms.cpp    the pseudo-volume multi-scattering BRDF: rendering, the -m fit
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <map>
#include <memory>
#include <vector>

#include "../../include/svf.h"
#include "svf_internal.h"
#include "svf_layout.h"

namespace svfh
{

// Records s and a message as the calling thread's last error (svf_last_error); returns s.
svf_status fail(svf_status s, const char* fmt, ...);

} // namespace svfh

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

namespace svfh
{

// Bumped whenever a device buffer is (re)allocated: a captured CUDA graph
// holds buffer addresses and is replayed only while this has not changed.
extern std::atomic<uint64_t> g_buffer_gen;

// A grow-only device allocation.
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

inline uint64_t fnv1a(const void* data, size_t bytes, uint64_t h = 1469598103934665603ull)
{
    const unsigned char* c = static_cast<const unsigned char*>(data);
    for(size_t i = 0; i < bytes; ++i)
    {
        h ^= c[i];
        h *= 1099511628211ull;
    }
    return h;
}

// Device or managed memory (of any device).
bool is_device_pointer(const void* p);
// Plain device memory (not managed, not host) of device `dev`.
bool is_device_pointer_on(const void* p, int dev);
// Where a caller's buffer that an entry point may hand to its kernels lives:
// *on_device for device memory of the current device or managed memory, false
// for host memory (pageable or pinned); SVF_EINVAL for device memory of
// another GPU, which the kernels on this one must not read or write.
svf_status buffer_location(const void* p, const char* what, bool* on_device);

inline uint64_t round_up(uint64_t x, uint64_t m) { return (x + m - 1) / m * m; }

// Default-init tables of one (direction table, mesh) pair.
struct InitData
{
    svf::InitLayout init{};
    DevBuf op, row_texel, denom_w, pca_cell_id, pca_cell_start, pca_index, pca_frac, pca_dir, proj_dir, proj_frac,
        proj_cell, col_pos, col_of, tile_hi, tile_lo, tile_kb, tile_start;
};

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

} // namespace svfh

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
    std::map<uint64_t, std::unique_ptr<svfh::Layout>> layouts;
    std::unique_ptr<svf::InitHostTables> tables;
    svfh::DevBuf lum, lum_hi, lum_lo, avg, ndf, ndf_tex, init, out, rmse, stats, counter, error, samples, samples2,
        maps_buf, scratch, rgb16, init_rgb, mlp_x, mlp_h1, mlp_h2, mlp_y, fb_idx, fb_lum, fb_hi, fb_lo, fb_ndf,
        fb_small,
        btf_decoded /* svf_fit_btf: the decoded chunk, kept between calls */;
    svfh::PinnedBuf pinned;
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
    svfh::DevBuf w, tc_hi, tc_lo, m, v, g, d_pairs, d_xmean, d_xrstd, d_ymean, d_ystd, d_pos, d_pair_pos, d_start, d_binw;
    int step = 0;
};

namespace svfh
{

// ---- contexts, options, layouts (svf_host.cpp)
svf_status check_ctx(svf_ctx* ctx);
// Initial LM damping relative to the reference's rule for a BTF's fit options.
float initial_damping(const svf_fit_options& o);
// downsample_ok: the entry point takes downsample_light_view and SVF_LSQ_FIT_TOP.
// ms_ok: the entry point takes SVF_LSQ_MULTI_SCATTERING.
svf_status check_options(const svf_lsq_options* o, bool downsample_ok = false, bool ms_ok = false);
svf_status get_layout(svf_ctx* ctx, const float* lp_in, uint32_t L, Layout** out);
// Copies `bytes` from src (host or device) to the device buffer dst.
svf_status to_device(svf_ctx* ctx, void* dst, const void* src, size_t bytes);
svf_status zero_error_flags(svf_ctx* ctx);
svf_status read_error_flag(svf_ctx* ctx, bool with_ndf = false);

template <typename T>
svf_status upload(DevBuf& dst, const std::vector<T>& v)
{
    SVF_TRY(dst.ensure(std::max<size_t>(sizeof(T) * v.size(), 16)));
    SVF_CUDA(cudaMemcpy(dst.p, v.data(), sizeof(T) * v.size(), cudaMemcpyHostToDevice));
    return SVF_OK;
}

// ---- default-init tables (svf_host_init.cpp)
svf_status prepare_init(svf_ctx* ctx, Layout* lay, const svf_layout_desc* desc, const svf::InitLayout** out);
cudaError_t launch_ndf(const svf::InitLayout& il, const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda,
                       float* C, uint32_t ldc, uint32_t* error_flag, cudaStream_t stream);

// ---- the LM (svf_host_lm.cpp)
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
    uint32_t base = 0;     // first texel of the launch (texels are base .. base + texels - 1)
};

svf_status launch_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const LmRun& r, svf::LmKernelChoice c);
svf_status tune_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o);
svf::LmKernelChoice lm_choice(Layout* lay, uint64_t stride, bool rgb);
svf_status run_lm(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const LmRun& r);
// An LM run over r.seg[0 .. r.n_seg), segment i of layout lays[i].
svf_status run_lm_segments(svf_ctx* ctx, Layout* const* lays, const svf_lsq_options* o, const LmRun& r);

// ---- the multi-scattering fit (svf_host_ms.cpp)
svf_status run_ms_fit(svf_ctx* ctx, Layout* lay, const svf_lsq_options* o, const float* lum, uint64_t stride,
                      uint64_t T, const float* init, float* out, float* rmse, svf_texel_stats* stats);

// ---- the learned initial guess (svf_host_mlp.cpp)
svf_status mlp_infer(svf_ctx* ctx, const svf_mlp* mlp, const float* X, uint64_t rows, float* C, float* act, float* Y);
svf::LumFeatures lum_features(const svf_mlp* mlp, float* X, bool normalise);
cudaError_t rgb_features(const svf_mlp* mlp, const void* samples, uint32_t sample_type, uint32_t N, uint64_t n,
                         float* X, bool normalise, cudaStream_t stream);

} // namespace svfh
