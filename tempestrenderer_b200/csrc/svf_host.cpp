// svf_host.cpp - the core of libsvf.so's C ABI (include/svf.h): error
// reporting, contexts, option checks, direction layouts and the error words the
// kernels raise; the other entry points are in svf_host_lm.cpp (LM),
// svf_host_fit.cpp (the fit pipeline), svf_host_mlp.cpp (learned guess) and
// svf_host_btf.cpp (BTF files, error maps, rendering, refit).
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

namespace
{

// The calling thread's last error message, in a fixed buffer so that reporting
// an error (out-of-memory included) allocates nothing.
thread_local char g_last_error[512];

} // namespace

svf_status svfh::fail(svf_status s, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return s;
}

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

namespace svfh
{

// Bumped whenever a device buffer is (re)allocated: a captured CUDA graph
// holds buffer addresses and is replayed only while this has not changed.
std::atomic<uint64_t> g_buffer_gen{ 1 };

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

svf_status buffer_location(const void* p, const char* what, bool* on_device)
{
    *on_device = false;
    if(!p)
        return SVF_OK;
    cudaPointerAttributes a;
    if(cudaPointerGetAttributes(&a, p) != cudaSuccess)
    {
        cudaGetLastError();
        return SVF_OK;   // memory CUDA does not know: pageable host memory
    }
    if(a.type == cudaMemoryTypeManaged)
    {
        *on_device = true;
        return SVF_OK;
    }
    if(a.type != cudaMemoryTypeDevice)
        return SVF_OK;
    int dev = 0;
    SVF_CUDA(cudaGetDevice(&dev));
    if(a.device != dev)
        return fail(SVF_EINVAL, "%s is device memory of GPU %d; the context runs on GPU %d", what, a.device, dev);
    *on_device = true;
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

svf_status check_options(const svf_lsq_options* o, bool downsample_ok, bool ms_ok)
{
    if(!o)
        return fail(SVF_EINVAL, "null options");
    if(o->flags & SVF_LSQ_MULTI_SCATTERING)
    {
        if(!ms_ok)
            return fail(SVF_EINVAL, "SVF_LSQ_MULTI_SCATTERING is taken by svf_lsq_fit_sggx / svf_lsq_fit_batch");
        constexpr uint32_t other = SVF_LSQ_RGB | SVF_LSQ_DISABLE_DIRECTION_FITTING | SVF_LSQ_FIT_TOP;
        if(!(o->flags & SVF_LSQ_DIFFUSE) || (o->flags & other) || o->downsample_light_view)
            return fail(SVF_EINVAL, "SVF_LSQ_MULTI_SCATTERING fits the 7 parameters (SVF_LSQ_DIFFUSE) without "
                                    "other options");
        if(o->multi_scattering_bounces > 1024)
            return fail(SVF_EINVAL, "multi_scattering_bounces %u (at most 1024)", o->multi_scattering_bounces);
    }
    if((o->flags & SVF_LSQ_FIT_TOP) && (!downsample_ok || (o->flags & SVF_LSQ_RGB)))
        return fail(SVF_EINVAL, "SVF_LSQ_FIT_TOP is taken by svf_lsq_fit_sggx / svf_lsq_fit_batch (luminance fit)");
    if(o->downsample_light_view == 1 || (o->downsample_light_view && !downsample_ok) ||
       (o->downsample_light_view && (o->flags & SVF_LSQ_RGB)))
        return fail(SVF_EINVAL, "downsample_light_view %u: 0, or 2 and more with svf_lsq_fit_sggx / svf_lsq_fit_batch",
                    o->downsample_light_view);
    if((o->flags & SVF_LSQ_RGB) && (o->flags & SVF_LSQ_DISABLE_DIRECTION_FITTING || !(o->flags & SVF_LSQ_DIFFUSE)))
        return fail(SVF_EINVAL, "the RGB fit (SVF_LSQ_RGB) fits every parameter, with the diffuse term");
    constexpr uint32_t known = SVF_LSQ_DIFFUSE | SVF_LSQ_RGB | SVF_LSQ_STEP_PER_PARAMETER |
                               SVF_LSQ_DISABLE_DIRECTION_FITTING | SVF_LSQ_FIT_TOP | SVF_LSQ_MULTI_SCATTERING;
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
    if(L < 3 || L > svf::kMaxLayout)
        return fail(SVF_EINVAL, "light_count must be in [3, %u], got %u", svf::kMaxLayout, L);
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

// Copies `bytes` from src (host or device) to the device buffer dst.
svf_status to_device(svf_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    SVF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, ctx->stream));
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
} // namespace svfh

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
    o->multi_scattering_bounces = 2;   // used with SVF_LSQ_MULTI_SCATTERING only
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
} // extern "C"
