// svf_error.cu - the error of fitted SVBRDF maps against a BTF, per texel
// (svbrdf-error-tool, tools/svbrdf-error-tool/svbrdf-error-tool.cc:88-250),
// and the rendered BTF of SVBRDF maps (the same BRDF written out).
//
// For texel t the map values give the material (diffuse and specular RGB, the
// SGGX scales, the basis quaternion; Fresnel 1) and the SGGX surface BRDF is
// evaluated at every (light, view) pair of the BTF's directions (the factored
// form of svf_model.cuh); the residual is BTF - BRDF per channel (color) or of
// the luminance.  Pair-wise: MSE over all L^2 pairs and the peak BTF value;
// max-view: the view whose sum over the lights is largest (per channel), its
// sum / L and its peak.  RMSE = sqrt(MSE), PSNR = 20 log10(peak / RMSE).
//
// One CTA per texel: the direction table in shared memory, threads over pairs
// (max-view: warps over views, lanes over lights), sums in FP64 reduced in a
// fixed order (deterministic).
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "svf_internal.h"
#include "svf_model.cuh"

namespace svf
{

namespace
{

constexpr int kThreads = 256, kWarps = kThreads / 32;

__device__ __forceinline__ void load_rgb(const ErrorArgs& a, uint64_t s, uint32_t lv, float* v)
{
    const uint64_t i = (s * a.N + lv) * 3;
    if(a.sample_type == SVF_SAMPLES_F16)
    {
        const __half* p = static_cast<const __half*>(a.samples) + i;
        v[0] = __half2float(p[0]);
        v[1] = __half2float(p[1]);
        v[2] = __half2float(p[2]);
    }
    else
    {
        const float* p = static_cast<const float*>(a.samples) + i;
        v[0] = p[0];
        v[1] = p[1];
        v[2] = p[2];
    }
}

// RGBToLuminance (spectrum.hh:328-331), products and sums rounded in order
__device__ __forceinline__ float lum(const float* c)
{
    return __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, c[0]), __fmul_rn(0.7152f, c[1])), __fmul_rn(0.0722f, c[2]));
}

__global__ void __launch_bounds__(kThreads) error_kernel(ErrorArgs a)
{
    extern __shared__ float smem[];
    const uint32_t L = a.L;
    DirEntry* tab = reinterpret_cast<DirEntry*>(smem);
    float* dirs = reinterpret_cast<float*>(tab + L);                    // [L][3]
    __shared__ double red_sq[kWarps][3];
    __shared__ float red_mx[kWarps][3];
    __shared__ ParamSet ps;
    const uint64_t t = blockIdx.x;
    const uint64_t ry = t / a.region_w, rx = t - ry * a.region_w;
    const uint64_t s = ry * a.row_texels + a.x0 + rx;   // sample row of the texel
    const uint32_t nch = a.color ? 3 : 1;
    float kd[3], ks[3];
    for(int c = 0; c < 3; ++c)
    {
        kd[c] = a.diffuse[3 * t + c];
        ks[c] = a.specular[3 * t + c];
    }
    if(threadIdx.x == 0)
    {
        float p[12];
        float sx = a.sigma[a.sigma_channels * t], sy = a.sigma[a.sigma_channels * t + 1];
        if(a.sigma_channels == 3)
        {
            const float sz = a.sigma[3 * t + 2];
            sx = sx / sz;
            sy = sy / sz;
        }
        p[6] = sx;
        p[7] = sy;
        for(int k = 0; k < 4; ++k)
            p[8 + k] = a.basis[4 * t + k];
        make_param_set_rgb(p, ps);
    }
    __syncthreads();
    for(uint32_t d = threadIdx.x; d < L; d += kThreads)
    {
        const float wx = a.geo[d], wy = a.geo[L + d], wz = a.geo[2 * L + d];
        make_dir_entry(ps, wx, wy, wz, tab[d]);
        dirs[3 * d] = wx;
        dirs[3 * d + 1] = wy;
        dirs[3 * d + 2] = wz;
    }
    __syncthreads();

    // the residuals of pair (light, view): r[c] and the BTF value b[c]
    auto pair = [&](uint32_t light, uint32_t view, float* r, float* b) {
        float v[3];
        load_rgb(a, s, view * L + light, v);
        const DirEntry& li = tab[light];
        const DirEntry& vo = tab[view];
        const float* wi = dirs + 3 * light;
        const float* wo = dirs + 3 * view;
        const float W0 = wi[0] + wo[0], W1 = wi[1] + wo[1], W2 = wi[2] + wo[2];
        const float g = W0 * W0 + W1 * W1 + W2 * W2;
        const float s0 = li.a[0] + vo.a[0], s1 = li.a[1] + vo.a[1], s2 = li.a[2] + vo.a[2];
        const float Q = ps.u * s0 * s0 + ps.v * s1 * s1 + s2 * s2;
        const float S = li.sp + vo.sp;
        const float QQS = Q * Q * S;
        const float spec = QQS > 0.0f ? ps.kspec * vo.kv * li.up * g * g / QQS : 0.0f;
        const float diff = vo.up * li.kdc;
        float f[3];
        for(int c = 0; c < 3; ++c)
            f[c] = kd[c] * diff + ks[c] * spec;
        if(a.color)
            for(int c = 0; c < 3; ++c)
            {
                b[c] = v[c];
                r[c] = v[c] - f[c];
            }
        else
        {
            b[0] = lum(v);
            r[0] = b[0] - lum(f);
        }
    };

    double sq[3] = { 0.0, 0.0, 0.0 };
    float mx[3] = { 0.0f, 0.0f, 0.0f };
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if(a.method == SVF_ERROR_PAIRWISE)
    {
        for(uint32_t lv = threadIdx.x; lv < L * L; lv += kThreads)
        {
            float r[3], b[3];
            pair(lv % L, lv / L, r, b);
            for(uint32_t c = 0; c < nch; ++c)
            {
                sq[c] += (double)r[c] * r[c];
                mx[c] = fmaxf(mx[c], b[c]);
            }
        }
        for(uint32_t c = 0; c < nch; ++c)
            for(int o = 16; o > 0; o >>= 1)
            {
                sq[c] += __shfl_xor_sync(0xffffffffu, sq[c], o);
                mx[c] = fmaxf(mx[c], __shfl_xor_sync(0xffffffffu, mx[c], o));
            }
    }
    else
    {
        // warps over views; a warp keeps, per channel, its largest view sum
        double best[3] = { -1.0, -1.0, -1.0 };
        float best_mx[3] = { 0.0f, 0.0f, 0.0f };
        for(uint32_t view = warp; view < L; view += kWarps)
        {
            double vs[3] = { 0.0, 0.0, 0.0 };
            float vm[3] = { 0.0f, 0.0f, 0.0f };
            for(uint32_t light = lane; light < L; light += 32)
            {
                float r[3], b[3];
                pair(light, view, r, b);
                for(uint32_t c = 0; c < nch; ++c)
                {
                    vs[c] += (double)r[c] * r[c];
                    vm[c] = fmaxf(vm[c], b[c]);
                }
            }
            for(uint32_t c = 0; c < nch; ++c)
            {
                for(int o = 16; o > 0; o >>= 1)
                {
                    vs[c] += __shfl_xor_sync(0xffffffffu, vs[c], o);
                    vm[c] = fmaxf(vm[c], __shfl_xor_sync(0xffffffffu, vm[c], o));
                }
                if(vs[c] > best[c])
                {
                    best[c] = vs[c];
                    best_mx[c] = vm[c];
                }
            }
        }
        for(uint32_t c = 0; c < nch; ++c)
        {
            sq[c] = best[c];
            mx[c] = best_mx[c];
        }
    }
    if(lane == 0)
        for(uint32_t c = 0; c < nch; ++c)
        {
            red_sq[warp][c] = sq[c];
            red_mx[warp][c] = mx[c];
        }
    __syncthreads();
    if(threadIdx.x == 0)
    {
        for(uint32_t c = 0; c < nch; ++c)
        {
            double tot = red_sq[0][c];
            float peak = red_mx[0][c];
            for(int w = 1; w < kWarps; ++w)
            {
                if(a.method == SVF_ERROR_PAIRWISE)
                {
                    tot += red_sq[w][c];
                    peak = fmaxf(peak, red_mx[w][c]);
                }
                else if(red_sq[w][c] > tot)
                {
                    // views were dealt round robin: warp w held views w, w+8, ...;
                    // equal sums keep the warp seen first
                    tot = red_sq[w][c];
                    peak = red_mx[w][c];
                }
            }
            const double mse = a.method == SVF_ERROR_PAIRWISE ? tot / ((double)L * L) : (tot < 0.0 ? 0.0 : tot / L);
            const float rmse = (float)sqrt(mse);
            a.rmse[nch * t + c] = rmse;
            a.psnr[nch * t + c] = 20.0f * log10f(peak / rmse);
        }
    }
}

} // namespace

// Rendered BTF: texel t's samples [L^2][3] from its map values (the same
// material set-up and BRDF as the error kernel), lv = view * L + light.
__global__ void __launch_bounds__(kThreads) render_kernel(RenderArgs a)
{
    extern __shared__ float smem[];
    const uint32_t L = a.L;
    DirEntry* tab = reinterpret_cast<DirEntry*>(smem);
    float* dirs = reinterpret_cast<float*>(tab + L);
    __shared__ ParamSet ps;
    const uint64_t t = blockIdx.x;
    float kd[3], ks[3];
    for(int c = 0; c < 3; ++c)
    {
        kd[c] = a.diffuse[3 * t + c];
        ks[c] = a.specular[3 * t + c];
    }
    if(threadIdx.x == 0)
    {
        float p[12];
        float sx = a.sigma[a.sigma_channels * t], sy = a.sigma[a.sigma_channels * t + 1];
        if(a.sigma_channels == 3)
        {
            const float sz = a.sigma[3 * t + 2];
            sx = sx / sz;
            sy = sy / sz;
        }
        p[6] = sx;
        p[7] = sy;
        for(int k = 0; k < 4; ++k)
            p[8 + k] = a.basis[4 * t + k];
        make_param_set_rgb(p, ps);
    }
    __syncthreads();
    for(uint32_t d = threadIdx.x; d < L; d += kThreads)
    {
        const float wx = a.geo[d], wy = a.geo[L + d], wz = a.geo[2 * L + d];
        make_dir_entry(ps, wx, wy, wz, tab[d]);
        dirs[3 * d] = wx;
        dirs[3 * d + 1] = wy;
        dirs[3 * d + 2] = wz;
    }
    __syncthreads();
    for(uint32_t lv = threadIdx.x; lv < L * L; lv += kThreads)
    {
        const uint32_t light = lv % L, view = lv / L;
        const DirEntry& li = tab[light];
        const DirEntry& vo = tab[view];
        const float* wi = dirs + 3 * light;
        const float* wo = dirs + 3 * view;
        const float W0 = wi[0] + wo[0], W1 = wi[1] + wo[1], W2 = wi[2] + wo[2];
        const float g = W0 * W0 + W1 * W1 + W2 * W2;
        const float s0 = li.a[0] + vo.a[0], s1 = li.a[1] + vo.a[1], s2 = li.a[2] + vo.a[2];
        const float Q = ps.u * s0 * s0 + ps.v * s1 * s1 + s2 * s2;
        const float S = li.sp + vo.sp;
        const float QQS = Q * Q * S;
        const float F = a.fresnel == 1.0f ? 1.0f : fresnel_factor(a.fresnel, wi, wo);
        const float spec = QQS > 0.0f ? ps.kspec * vo.kv * li.up * F * g * g / QQS : 0.0f;
        const float diff = vo.up * li.kdc;
        const uint64_t o = (t * L * L + lv) * 3;
        for(int c = 0; c < 3; ++c)
        {
            const float f = kd[c] * diff + ks[c] * spec;
            if(a.sample_type == SVF_SAMPLES_F16)
                static_cast<__half*>(a.out)[o + c] = __float2half_rn(f);
            else
                static_cast<float*>(a.out)[o + c] = f;
        }
    }
}

cudaError_t launch_render(const RenderArgs& a, cudaStream_t stream)
{
    if(a.count == 0)
        return cudaSuccess;
    if(a.count > 0x7fffffffull)
        return cudaErrorInvalidValue;
    const size_t smem = (sizeof(DirEntry) + 3 * sizeof(float)) * a.L;
    render_kernel<<<(unsigned)a.count, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_error(const ErrorArgs& a, cudaStream_t stream)
{
    if(a.count == 0)
        return cudaSuccess;
    if(a.count > 0x7fffffffull)
        return cudaErrorInvalidValue;
    const size_t smem = (sizeof(DirEntry) + 3 * sizeof(float)) * a.L;
    error_kernel<<<(unsigned)a.count, kThreads, smem, stream>>>(a);
    return cudaGetLastError();
}

} // namespace svf
