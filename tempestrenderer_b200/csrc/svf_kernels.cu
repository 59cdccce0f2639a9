// svf_kernels.cu - luminance slice, repacking, the synthetic BTF renderer and
// the allocation-free LM entry, for sm_100a.  The LM kernel itself is in
// svf_lm.cu.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>
#include <array>
#include <type_traits>
#include <utility>

#include "svf_internal.h"
#include "svf_model.cuh"

namespace svf
{

namespace
{

// ------------------------------------------------------------------------------
// luminance slice
// ------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ float to_f(T x);
template <>
__device__ __forceinline__ float to_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ float to_f<__half>(__half x) { return __half2float(x); }

constexpr uint32_t kLumThreads = 256;
constexpr uint32_t kLumChunk = 1024;   // pairs per shared-memory chunk (a multiple of kLumThreads)
constexpr int kLumUnroll = 4;          // pairs a thread has in flight on the direct path

// The learned guess's features of one texel from its luminance slab y in bin
// order (shared memory, complete), by a CTA of kLumThreads: each bin's run
// summed by one warp, lane-strided then a fixed butterfly (deterministic), the
// single pairs, log, normalised.  st: the bin starts (shared); v: shared
// scratch of kMlpInputs floats.
__device__ void texel_features(const float* y, const uint32_t* st, const LumFeatures& f, uint64_t t, float* v)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for(int b = warp; b < kMlpBins; b += kLumThreads / 32)
    {
        float s = 0.0f;
        for(uint32_t k = st[b] + lane; k < st[b + 1]; k += 32)
            s += y[k];
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if(lane == 0)
            v[b] = s * f.bin_w[b];
    }
    if(threadIdx.x < kMlpPairs)
        v[kMlpBins + threadIdx.x] = y[f.pair_pos[threadIdx.x]];
    __syncthreads();
    if(threadIdx.x < kMlpInputs)
    {
        const int i = threadIdx.x;
        float x = logf(fmaxf(v[i], 1e-6f));
        if(f.mean)
            x = (x - f.mean[i]) * f.rstd[i];
        f.X[t * kMlpInputs + i] = x;
    }
}

// The luminance pass reads FP16 samples through shared memory (kStaged: chunks
// of kLumChunk pairs, a multiple of kLumThreads so that each thread keeps its
// pairs, double-buffered) and FP32 samples straight into registers, kLumUnroll
// pairs a thread in flight: a warp's direct 2-byte loads carry too few bytes
// to cover the latency, its 4-byte loads enough (measured both ways on both
// types).  With features the slab is kept in shared memory (direct path).
template <typename T, bool kFeat>
struct LumPass
{
    static constexpr bool kStaged = sizeof(T) == 2 && !kFeat;
    static constexpr uint32_t kChunkBytes = kLumChunk * 3 * sizeof(T) + 16;   // + the alignment offset
    __host__ __device__ static size_t smem(uint32_t N)
    {
        return kStaged ? 2 * (size_t)kChunkBytes : (kFeat ? sizeof(float) * N : 0);
    }
    // with the BF16 split: its hi and lo rows after the above, 16-byte aligned
    __host__ __device__ static size_t split_offset(uint32_t N) { return (smem(N) + 15) & ~size_t(15); }
    static size_t smem(uint32_t N, uint64_t lum_stride, bool hilo)
    {
        return hilo ? split_offset(N) + 2 * sizeof(__nv_bfloat16) * lum_stride : smem(N);
    }
};

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(smem_dst)),
                 "l"(gmem_src)
                 : "memory");
}

// Copies the bytes [g0, g1) of the samples (T-aligned) into buf + (g0 & 15), so
// that 16-byte words of global memory land on 16-byte words of shared memory:
// the aligned interior by cp.async, the ragged head and tail (under 16 bytes
// each) element by element.
template <typename T>
__device__ __forceinline__ void stage_bytes(const char* g0, const char* g1, unsigned char* buf)
{
    const uintptr_t a0 = reinterpret_cast<uintptr_t>(g0), a1 = reinterpret_cast<uintptr_t>(g1);
    unsigned char* dst = buf + (a0 & 15u);
    uintptr_t ia = (a0 + 15u) & ~uintptr_t(15), ib = a1 & ~uintptr_t(15);
    if(ia > ib)
        ia = ib = a1;   // inside one 16-byte word: all of it is head
    const uint32_t words = (uint32_t)((ib - ia) / 16);
    for(uint32_t w = threadIdx.x; w < words; w += kLumThreads)
        cp_async16(dst + (ia - a0) + 16 * w, reinterpret_cast<const void*>(ia + 16 * w));
    const uint32_t head = (uint32_t)((ia - a0) / sizeof(T)), tail = (uint32_t)((a1 - ib) / sizeof(T));
    const uint32_t tail0 = (uint32_t)((ib - a0) / sizeof(T));
    if(threadIdx.x < head)
        reinterpret_cast<T*>(dst)[threadIdx.x] = reinterpret_cast<const T*>(g0)[threadIdx.x];
    else if(threadIdx.x >= 32 && threadIdx.x - 32 < tail)
        reinterpret_cast<T*>(dst)[tail0 + threadIdx.x - 32] = reinterpret_cast<const T*>(ib)[threadIdx.x - 32];
}

// One pair of the luminance pass: lum = 0.2126 R + 0.7152 G + 0.0722 B
// (spectrum.hh:328-331, evaluated without fused multiply-adds, as the
// reference's x86-64 build does) and the optional outputs; chromaticity rgb/lum,
// or (1,1,1) when lum <= 1e-6, added to the thread's sums.
template <bool kHiLo, bool kRgb, bool kFeat, bool kChroma>
__device__ __forceinline__ void lum_pair(uint32_t i, float r, float g, float b, uint32_t ypos, uint64_t t,
                                         float* dst, float* y, __half* rgb16, uint64_t rgb_stride,
                                         __nv_bfloat16* sh_hi, __nv_bfloat16* sh_lo, const uint16_t* hilo_pos,
                                         float& ax, float& ay, float& az)
{
    const float l = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, r), __fmul_rn(0.7152f, g)), __fmul_rn(0.0722f, b));
    dst[i] = l;
    if constexpr(kFeat)
        y[ypos] = l;
    if constexpr(kRgb)
    {
        // the RGB fit's slab: the samples in FP16, [L*L][3], 16-byte rows
        __half* o = rgb16 + t * rgb_stride + 3 * (uint64_t)i;
        o[0] = __float2half_rn(r);
        o[1] = __float2half_rn(g);
        o[2] = __float2half_rn(b);
    }
    if constexpr(kHiLo)
    {
        // x = hi + lo to 16 significant bits, for the BF16x3 NDF GEMM, at the
        // pair's column of the operator (shared memory; written out at the end)
        const __nv_bfloat16 h = __float2bfloat16_rn(l);
        const uint32_t p = __ldg(hilo_pos + i);
        sh_hi[p] = h;
        sh_lo[p] = __float2bfloat16_rn(__fsub_rn(l, __bfloat162float(h)));
    }
    if constexpr(kChroma)
    {
        if(l > 1e-6f)
        {
            const float rl = 1.0f / l;
            ax += r * rl;
            ay += g * rl;
            az += b * rl;
        }
        else
        {
            ax += 1.0f;
            ay += 1.0f;
            az += 1.0f;
        }
    }
}

// One CTA of kLumThreads per texel: the luminance slab, and the average
// chromaticity over the pairs.  Thread j takes pairs j, j + 256, ... in that
// order whichever way the samples arrive (LumPass).  With features, the slab
// is also kept in shared memory in bin order and the features are computed
// from it.  The optional outputs are template flags (kHiLo: the BF16 split for
// the NDF GEMM; kRgb: the FP16 RGB slab; kFeat: the features; kChroma: the
// average chromaticity, which only the colour maps and the RGB fit read), so
// that the per-pair loop carries no branches for them.
template <typename T, bool kHiLo, bool kRgb, bool kFeat, bool kChroma>
__global__ void __launch_bounds__(kLumThreads) luminance_kernel(const T* __restrict__ samples, uint32_t N,
                                                                float* __restrict__ lum, uint64_t lum_stride,
                                                                float* __restrict__ avg,
                                                                __nv_bfloat16* __restrict__ lum_hi,
                                                                __nv_bfloat16* __restrict__ lum_lo,
                                                                const uint16_t* __restrict__ hilo_pos,
                                                                __half* __restrict__ rgb16, uint64_t rgb_stride,
                                                                LumFeatures feat)
{
    using S = LumPass<T, kFeat>;
    // staged: [2][kChunkBytes] samples; with features: y [N] in bin order
    extern __shared__ __align__(16) unsigned char smem[];
    float* y = reinterpret_cast<float*>(smem);
    __shared__ uint32_t st[kMlpBins + 1];
    if(kFeat && threadIdx.x <= kMlpBins)
        st[threadIdx.x] = feat.start[threadIdx.x];
    const uint64_t t = blockIdx.x;
    const T* src = samples + t * (uint64_t)N * 3;
    float* dst = lum + t * lum_stride;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    __nv_bfloat16* sh_hi = reinterpret_cast<__nv_bfloat16*>(smem + S::split_offset(N));
    __nv_bfloat16* sh_lo = sh_hi + lum_stride;
    if constexpr(S::kStaged)
    {
        const char* bytes = reinterpret_cast<const char*>(src);
        const uint32_t chunks = (N + kLumChunk - 1) / kLumChunk;
        const auto stage = [&](uint32_t c) {
            const uint32_t p0 = c * kLumChunk, pn = min(kLumChunk, N - p0);
            stage_bytes<T>(bytes + (size_t)p0 * 3 * sizeof(T), bytes + (size_t)(p0 + pn) * 3 * sizeof(T),
                           smem + (c & 1) * S::kChunkBytes);
            asm volatile("cp.async.commit_group;" ::: "memory");
        };
        if(chunks)
            stage(0);
        for(uint32_t c = 0; c < chunks; ++c)
        {
            if(c + 1 < chunks)
            {
                stage(c + 1);
                asm volatile("cp.async.wait_group 1;" ::: "memory");
            }
            else
                asm volatile("cp.async.wait_group 0;" ::: "memory");
            __syncthreads();
            const uint32_t p0 = c * kLumChunk, pn = min(kLumChunk, N - p0);
            const uintptr_t g0 = reinterpret_cast<uintptr_t>(bytes + (size_t)p0 * 3 * sizeof(T));
            const T* cs = reinterpret_cast<const T*>(smem + (c & 1) * S::kChunkBytes + (g0 & 15u));
#pragma unroll 4
            for(uint32_t k = threadIdx.x; k < pn; k += kLumThreads)
                lum_pair<kHiLo, kRgb, kFeat, kChroma>(p0 + k, to_f(cs[3 * k]), to_f(cs[3 * k + 1]),
                                                      to_f(cs[3 * k + 2]), 0, t, dst, y, rgb16, rgb_stride, sh_hi,
                                                      sh_lo, hilo_pos, ax, ay, az);
            __syncthreads();   // the buffer is refilled two chunks on
        }
    }
    else
    {
        for(uint32_t i0 = threadIdx.x; i0 < N; i0 += kLumUnroll * kLumThreads)
        {
            float rr[kLumUnroll], gg[kLumUnroll], bb[kLumUnroll];
            uint32_t pp[kLumUnroll];
#pragma unroll
            for(int u = 0; u < kLumUnroll; ++u)
            {
                const uint32_t i = i0 + u * kLumThreads;
                rr[u] = gg[u] = bb[u] = 0.0f;
                pp[u] = 0;
                if(i < N)
                {
                    rr[u] = to_f(src[3 * i]);
                    gg[u] = to_f(src[3 * i + 1]);
                    bb[u] = to_f(src[3 * i + 2]);
                    if(kFeat)
                        pp[u] = feat.pos[i];
                }
            }
#pragma unroll
            for(int u = 0; u < kLumUnroll; ++u)
            {
                const uint32_t i = i0 + u * kLumThreads;
                if(i >= N)
                    break;
                lum_pair<kHiLo, kRgb, kFeat, kChroma>(i, rr[u], gg[u], bb[u], pp[u], t, dst, y, rgb16, rgb_stride,
                                                      sh_hi, sh_lo, hilo_pos, ax, ay, az);
            }
        }
        if constexpr(kFeat)
            __syncthreads();   // y is complete
    }
    for(uint32_t i = N + threadIdx.x; i < lum_stride; i += blockDim.x)
        dst[i] = 0.0f;
    if constexpr(kHiLo)
    {
        // the split rows, in the operator's column order, out in 16-byte words
        for(uint32_t i = N + threadIdx.x; i < lum_stride; i += blockDim.x)
            sh_hi[i] = sh_lo[i] = __float2bfloat16_rn(0.0f);
        __syncthreads();
        const uint4* sh4 = reinterpret_cast<const uint4*>(sh_hi);
        const uint32_t words = (uint32_t)(lum_stride / 8);
        uint4* gh = reinterpret_cast<uint4*>(lum_hi + t * lum_stride);
        uint4* gl = reinterpret_cast<uint4*>(lum_lo + t * lum_stride);
        for(uint32_t w = threadIdx.x; w < words; w += blockDim.x)
        {
            gh[w] = sh4[w];
            gl[w] = sh4[words + w];
        }
    }
    if constexpr(kChroma)
    {
        __shared__ float red[3][8];
#pragma unroll
        for(int o = 16; o > 0; o >>= 1)
        {
            ax += __shfl_xor_sync(0xffffffffu, ax, o);
            ay += __shfl_xor_sync(0xffffffffu, ay, o);
            az += __shfl_xor_sync(0xffffffffu, az, o);
        }
        const uint32_t warp = threadIdx.x >> 5;
        if((threadIdx.x & 31u) == 0)
        {
            red[0][warp] = ax;
            red[1][warp] = ay;
            red[2][warp] = az;
        }
        __syncthreads();
        if(threadIdx.x < 3)
        {
            float s = 0.0f;
            for(uint32_t w = 0; w < blockDim.x / 32; ++w)
                s += red[threadIdx.x][w];
            // Vector3 / float multiplies by the reciprocal (vector3.hh:185-190)
            avg[3 * t + threadIdx.x] = s * (1.0f / (float)N);
        }
    }
    __shared__ float fv[kMlpInputs];
    if(kFeat)
        texel_features(y, st, feat, t, fv);
}

__global__ void gather_pairs_kernel(const float* __restrict__ src, uint64_t src_stride,
                                    const uint32_t* __restrict__ pairs, uint32_t n_pairs, float* __restrict__ dst,
                                    uint64_t dst_stride)
{
    const uint64_t t = blockIdx.x;
    for(uint32_t j = threadIdx.x; j < dst_stride; j += blockDim.x)
        dst[t * dst_stride + j] = j < n_pairs ? src[t * src_stride + pairs[j]] : 0.0f;
}

__global__ void repack_kernel(const float* __restrict__ src, uint64_t src_stride, uint32_t N, float* __restrict__ dst,
                              uint64_t dst_stride)
{
    const uint64_t t = blockIdx.x;
    for(uint32_t i = threadIdx.x; i < dst_stride; i += blockDim.x)
        dst[t * dst_stride + i] = i < N ? src[t * src_stride + i] : 0.0f;
}

// ------------------------------------------------------------------------------
// synthetic BTF (mirrors svfo_synth_truth / svfo_synth_render of the oracle)
// ------------------------------------------------------------------------------

__device__ __forceinline__ void philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                       uint32_t* out)
{
#pragma unroll
    for(int r = 0; r < 10; ++r)
    {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__device__ __forceinline__ float u01(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float loguni(float a, float b, float u) { return a * expf(u * logf(b / a)); }

struct Truth
{
    float kd[3], ks[3], sigma[2], quat[4], euler[3], kind;
};

__device__ void synth_truth(uint32_t seed, uint32_t mix, uint64_t texel, Truth& t)
{
    uint32_t b0[4], b1[4], b2[4];
    const uint32_t lo = (uint32_t)texel, hi = (uint32_t)(texel >> 32);
    philox(seed, 0x53564631u, lo, hi, 0, 0, b0);
    philox(seed, 0x53564631u, lo, hi, 1, 0, b1);
    philox(seed, 0x53564631u, lo, hi, 2, 0, b2);
    float uk = u01(b0[0]);
    uint32_t kind = 0;
    if(mix == 1)
        kind = uk < 0.2f ? 1u : (uk < 0.3f ? 2u : 0u);
    t.kind = (float)kind;
    for(int c = 0; c < 3; ++c)
        t.kd[c] = 0.8f * u01(b0[1 + c]);
    for(int c = 0; c < 3; ++c)
        t.ks[c] = (kind == 1 ? 0.05f : 1.0f) * u01(b1[c]);
    if(kind == 2)
    {
        float smin = loguni(0.01f, 0.05f, u01(b1[3]));
        float ratio = loguni(8.5f, 16.0f, u01(b2[0]));
        float smax = smin * ratio;
        t.sigma[0] = smax < 0.8f ? smax : 0.8f;
        t.sigma[1] = smin;
    }
    else
    {
        t.sigma[0] = loguni(0.02f, 0.8f, u01(b1[3]));
        t.sigma[1] = loguni(0.02f, 0.8f, u01(b2[0]));
    }
    const float cos30 = 0.866025403784f, two_pi = 6.283185307179586f;
    float nz = 1.0f - u01(b2[1]) * (1.0f - cos30);
    float nr = sqrtf(fmaxf(0.0f, 1.0f - nz * nz));
    float phi = two_pi * u01(b2[2]), psi = two_pi * u01(b2[3]);
    float n[3] = { nr * cosf(phi), nr * sinf(phi), nz };
    float t0[3] = { 1.0f - n[0] * n[0], -n[1] * n[0], -n[2] * n[0] };
    float l0 = sqrtf(t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2]);
    float rl0 = 1.0f / l0;
    t0[0] *= rl0; t0[1] *= rl0; t0[2] *= rl0;
    float b0v[3] = { n[1] * t0[2] - n[2] * t0[1], n[2] * t0[0] - n[0] * t0[2], n[0] * t0[1] - n[1] * t0[0] };
    float cp = cosf(psi), sp = sinf(psi);
    float tt[3] = { t0[0] * cp + b0v[0] * sp, t0[1] * cp + b0v[1] * sp, t0[2] * cp + b0v[2] * sp };
    float bb[3] = { n[1] * tt[2] - n[2] * tt[1], n[2] * tt[0] - n[0] * tt[2], n[0] * tt[1] - n[1] * tt[0] };
    float m00 = tt[0], m01 = tt[1], m02 = tt[2], m10 = bb[0], m11 = bb[1], m12 = bb[2], m20 = n[0], m21 = n[1], m22 = n[2];
    float q[4];
    float tr = m00 + m11 + m22;
    if(tr > 0.0f)
    {
        float s = sqrtf(tr + 1.0f) * 2.0f;
        q[3] = 0.25f * s; q[0] = (m12 - m21) / s; q[1] = (m20 - m02) / s; q[2] = (m01 - m10) / s;
    }
    else if(m00 > m11 && m00 > m22)
    {
        float s = sqrtf(1.0f + m00 - m11 - m22) * 2.0f;
        q[3] = (m12 - m21) / s; q[0] = 0.25f * s; q[1] = (m01 + m10) / s; q[2] = (m02 + m20) / s;
    }
    else if(m11 > m22)
    {
        float s = sqrtf(1.0f + m11 - m00 - m22) * 2.0f;
        q[3] = (m20 - m02) / s; q[0] = (m01 + m10) / s; q[1] = 0.25f * s; q[2] = (m12 + m21) / s;
    }
    else
    {
        float s = sqrtf(1.0f + m22 - m00 - m11) * 2.0f;
        q[3] = (m01 - m10) / s; q[0] = (m02 + m20) / s; q[1] = (m12 + m21) / s; q[2] = 0.25f * s;
    }
    float ql = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for(int i = 0; i < 4; ++i)
        t.quat[i] = q[i] / ql;
    // Matrix3::decompose of ToMatrix3(quat) (matrix3.hh:311-332)
    const float x = t.quat[0], y = t.quat[1], z = t.quat[2], w = t.quat[3];
    float C0[3] = { 1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w) };
    float C1[3] = { 2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w) };
    float C2[3] = { 2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y) };
    float sc0 = sqrtf(C0[0] * C0[0] + C0[1] * C0[1] + C0[2] * C0[2]);
    float sc1 = sqrtf(C1[0] * C1[0] + C1[1] * C1[1] + C1[2] * C1[2]);
    float sc2 = sqrtf(C2[0] * C2[0] + C2[1] * C2[1] + C2[2] * C2[2]);
    float m20d = C2[0] / sc2;
    const float half_pi = kRefPi * 0.5f;
    if(m20d >= 0.9999f)
    {
        t.euler[0] = 0.0f; t.euler[1] = half_pi; t.euler[2] = atan2f(C0[1], C1[1]);
    }
    else if(m20d <= -0.9999f)
    {
        t.euler[0] = 0.0f; t.euler[1] = -half_pi; t.euler[2] = atan2f(C0[1], C1[1]);
    }
    else
    {
        t.euler[0] = atan2f(-C2[1], C2[2]);
        t.euler[1] = asinf(m20d);
        t.euler[2] = atan2f(-C1[0] / sc1, C0[0] / sc0);
    }
}

__device__ __forceinline__ float surface_brdf_rgb(float kd, float ks, float sx, float sy, const float* R, float out_density,
                                                  const float* wi, const float* wo)
{
    // SGGXMicroFlakeSurfaceBRDF in the reference's operation order (Fresnel 1)
    float dot_inc = wi[2], dot_out = wo[2];
    if(dot_inc < 0.0f || dot_out < 0.0f)
        return 0.0f;
    float result = kd * dot_inc * (1.0f / kRefPi);
    if(sx >= 1e-6f && sy >= 1e-6f && out_density >= 1e-6f)
    {
        float h[3] = { wi[0] + wo[0], wi[1] + wo[1], wi[2] + wo[2] };
        float hl = sqrtf(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
        float rh = 1.0f / hl;
        h[0] *= rh; h[1] *= rh; h[2] *= rh;
        float ai[3], ah[3];
        for(int c = 0; c < 3; ++c)
        {
            ai[c] = R[3 * c] * wi[0] + R[3 * c + 1] * wi[1] + R[3 * c + 2] * wi[2];
            ah[c] = R[3 * c] * h[0] + R[3 * c + 1] * h[1] + R[3 * c + 2] * h[2];
        }
        float in_density = sqrtf(sx * sx * ai[0] * ai[0] + sy * sy * ai[1] * ai[1] + ai[2] * ai[2]);
        float u = 1.0f / (sx * sx), v = 1.0f / (sy * sy);
        float det = u * v;
        float ndf = 0.0f;
        if(det >= 1e-6f)
        {
            float den = u * ah[0] * ah[0] + v * ah[1] * ah[1] + ah[2] * ah[2];
            ndf = 0.5f * sqrtf(det) / (kRefPi * den * den);
        }
        float contrib = 1.0f / (out_density + in_density * dot_out / dot_inc);
        result += contrib * ks * ndf * 2.0f / 4.0f;
    }
    return result;
}

// One CTA (256 threads) per texel.
template <typename T>
__global__ void __launch_bounds__(256) synth_kernel(uint32_t seed, uint32_t mix, const float* __restrict__ lp, uint32_t L,
                                                     uint64_t first, float noise, T* __restrict__ samples,
                                                     float* __restrict__ truth)
{
    __shared__ Truth tr;
    __shared__ float R[9];
    __shared__ float w[3][160];
    __shared__ float dens[160];
    const uint64_t texel = first + blockIdx.x;
    if(threadIdx.x == 0)
    {
        synth_truth(seed, mix, texel, tr);
        const float x = tr.quat[0], y = tr.quat[1], z = tr.quat[2], ww = tr.quat[3];
        R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + z * ww); R[2] = 2.0f * (x * z - y * ww);
        R[3] = 2.0f * (x * y - z * ww); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + x * ww);
        R[6] = 2.0f * (x * z + y * ww); R[7] = 2.0f * (y * z - x * ww); R[8] = 1.0f - 2.0f * (x * x + y * y);
        if(truth)
        {
            float* o = truth + 16 * (uint64_t)blockIdx.x;
            for(int i = 0; i < 16; ++i)
                o[i] = (&tr.kd[0])[i];
        }
    }
    __syncthreads();
    for(uint32_t d = threadIdx.x; d < L; d += blockDim.x)
    {
        float wd[3];
        parabolic_to_cartesian(lp[2 * d], lp[2 * d + 1], wd);
        w[0][d] = wd[0]; w[1][d] = wd[1]; w[2][d] = wd[2];
        float a[3];
        for(int c = 0; c < 3; ++c)
            a[c] = R[3 * c] * wd[0] + R[3 * c + 1] * wd[1] + R[3 * c + 2] * wd[2];
        dens[d] = sqrtf(tr.sigma[0] * tr.sigma[0] * a[0] * a[0] + tr.sigma[1] * tr.sigma[1] * a[1] * a[1] + a[2] * a[2]);
    }
    __syncthreads();
    const uint32_t N = L * L;
    T* out = samples + (uint64_t)blockIdx.x * N * 3;
    const uint32_t lo = (uint32_t)texel, hi = (uint32_t)(texel >> 32);
    for(uint32_t lv = threadIdx.x; lv < N; lv += blockDim.x)
    {
        uint32_t v = lv / L, l = lv % L;
        float wi[3] = { w[0][l], w[1][l], w[2][l] };
        float wo[3] = { w[0][v], w[1][v], w[2][v] };
        uint32_t r[4];
        philox(seed, 0x53564631u, lo, hi, 16u + lv, 0u, r);
        float z[4];
        for(int k = 0; k < 2; ++k)
        {
            float ua = (float)((r[2 * k] >> 8) + 1u) * (1.0f / 16777216.0f);
            float ub = u01(r[2 * k + 1]);
            float rad = sqrtf(-2.0f * logf(ua));
            float sn, cs;
            sincosf(6.283185307179586f * ub, &sn, &cs);
            z[2 * k] = rad * cs;
            z[2 * k + 1] = rad * sn;
        }
        for(int c = 0; c < 3; ++c)
        {
            float f = surface_brdf_rgb(tr.kd[c], tr.ks[c], tr.sigma[0], tr.sigma[1], R, dens[v], wi, wo);
            float val = f * (1.0f + noise * z[c]);
            if constexpr(sizeof(T) == 2)
                out[3 * lv + c] = __float2half_rn(val);
            else
                out[3 * lv + c] = val;
        }
    }
}

// ------------------------------------------------------------------------------
// allocation-free LM batch: working memory in one static device array
// ------------------------------------------------------------------------------

// Layout of the static array: luminance slabs, then the direction table, then
// the work counter and the error flag.
constexpr size_t kNoAllocGeoOffset = size_t(SVF_NOALLOC_MAX_SLAB_FLOATS) * sizeof(float);
constexpr size_t kNoAllocFlagOffset = kNoAllocGeoOffset + 3 * 160 * sizeof(float);
static_assert(kNoAllocFlagOffset + 16 <= SVF_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout overflows");

// Direction table [3][L] from parabolic coordinates, with the operation order
// and rounding of ParabolicToCartesianCoordinates (vector3.hh:389-393) that the
// host computes for the other entry points, so both fit identical geometry.
__global__ void geo_from_parabolic_kernel(const float* __restrict__ lp, uint32_t L, float* __restrict__ geo)
{
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if(d >= L)
        return;
    const float px = lp[2 * d], py = lp[2 * d + 1];
    const float len_sq = __fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py));
    const float den = __fadd_rn(len_sq, 1.0f);
    geo[d] = __fdiv_rn(__fmul_rn(2.0f, px), den);
    geo[L + d] = __fdiv_rn(__fmul_rn(2.0f, py), den);
    geo[2 * L + d] = __fdiv_rn(__fsub_rn(1.0f, len_sq), __fadd_rn(1.0f, len_sq));
}

// ORs the texels' "no finite fit" bits (SVF_TEXEL_NONFINITE, SVF_TEXEL_TIMEOUT)
// into *partial, so the host learns of them from one word.
__global__ void partial_scan_kernel(const svf_texel_stats* __restrict__ stats, uint32_t texels, uint32_t* partial)
{
    uint32_t bits = 0;
    for(uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < texels; t += gridDim.x * blockDim.x)
        bits |= stats[t].status & (SVF_TEXEL_NONFINITE | SVF_TEXEL_TIMEOUT);
    bits = __reduce_or_sync(0xffffffffu, bits);
    if(bits && (threadIdx.x & 31u) == 0)
        atomicOr(partial, bits);
}

} // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[SVF_NOALLOC_SCRATCH_BYTES];

namespace
{
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_address[kNoAllocMaxDevices];

// Device address of g_noalloc_scratch on the current device, looked up once per
// device and kept for the life of the process (a cudaDeviceReset of the device
// would leave it stale).  In host code the array's name is only a host-side
// stand-in.
cudaError_t noalloc_scratch_address(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if(e != cudaSuccess)
        return e;
    if(dev < 0 || dev >= kNoAllocMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if(!g_noalloc_address[dev])
    {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if(e != cudaSuccess)
            return e;
        g_noalloc_address[dev] = p;
    }
    *out = g_noalloc_address[dev];
    return cudaSuccess;
}
} // namespace

cudaError_t launch_gather_pairs(const float* src, uint64_t src_stride, const uint32_t* pairs, uint32_t n_pairs,
                                uint64_t texels, float* dst, uint64_t dst_stride, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    if(texels > 0x7fffffffull || dst_stride < n_pairs)
        return cudaErrorInvalidValue;
    gather_pairs_kernel<<<(unsigned)texels, 256, 0, stream>>>(src, src_stride, pairs, n_pairs, dst, dst_stride);
    return cudaGetLastError();
}

cudaError_t launch_lm_fit_noalloc(const float* lights_parabolic, uint32_t L, const float* lum, uint64_t lum_stride,
                                  uint32_t texels, const LmConfig& cfg, const float* init, float* out, float* rmse,
                                  svf_texel_stats* stats, cudaStream_t stream, uint32_t host_flags[2])
{
    void* base = nullptr;
    cudaError_t e = noalloc_scratch_address(&base);
    if(e != cudaSuccess)
        return e;
    unsigned char* scratch = static_cast<unsigned char*>(base);
    float* slabs = reinterpret_cast<float*>(scratch);
    float* geo = reinterpret_cast<float*>(scratch + kNoAllocGeoOffset);
    uint32_t* flags = reinterpret_cast<uint32_t*>(scratch + kNoAllocFlagOffset);
    const uint32_t N = L * L;
    const uint64_t stride = (N + 7u) & ~uint64_t(7);

    // the array keeps the previous call's contents: counter and flag start at 0
    if((e = cudaMemsetAsync(flags, 0, 16, stream)) != cudaSuccess)
        return e;
    geo_from_parabolic_kernel<<<(L + 127) / 128, 128, 0, stream>>>(lights_parabolic, L, geo);
    if((e = cudaGetLastError()) != cudaSuccess)
        return e;
    repack_kernel<<<texels, 256, 0, stream>>>(lum, lum_stride, N, slabs, stride);
    if((e = cudaGetLastError()) != cudaSuccess)
        return e;
    int dev = 0, sms = 0;
    if((e = cudaGetDevice(&dev)) != cudaSuccess ||
       (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    LmArgs a{};
    a.seg[0] = LmSegment{ 0, L, stride, slabs, geo };
    a.n_seg = 1;
    a.L = L;
    a.lum_stride = stride;
    a.init = init;
    a.out = out;
    a.rmse = rmse;
    a.stats = stats;
    a.texels = texels;
    a.cfg = cfg;
    a.work_counter = flags;
    a.error_flag = flags + 1;
    a.fault_skip_texel = kLmNoFault;
    a.wait_spins = 0;
    const LmKernelChoice choice = lm_default_choice(L, stride);
    const int per_sm = lm_max_ctas_per_sm(L, stride, choice);
    if(per_sm <= 0)
        return cudaErrorInvalidConfiguration;
    const uint64_t grid = std::min<uint64_t>((uint64_t)per_sm * sms, texels);
    if((e = launch_lm_fit(a, choice, (int)std::max<uint64_t>(grid, 1), stream)) != cudaSuccess)
        return e;
    if(stats)
    {
        partial_scan_kernel<<<(texels + 255) / 256, 256, 0, stream>>>(stats, texels, flags + 2);
        if((e = cudaGetLastError()) != cudaSuccess)
            return e;
    }
    // flags[1]: a bounded wait expired; flags[2]: texels without a finite fit
    if((e = cudaMemcpyAsync(host_flags, flags + 1, 2 * sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(stream);
}

namespace
{

template <typename T, int... F>
auto luminance_kernel_table(std::integer_sequence<int, F...>)
{
    using K = decltype(&luminance_kernel<T, false, false, false, false>);
    return std::array<K, sizeof...(F)>{ &luminance_kernel<T, (F & 1) != 0, (F & 2) != 0, (F & 4) != 0,
                                                          (F & 8) != 0>... };
}

// The instance for output flags 1 kHiLo | 2 kRgb | 4 kFeat | 8 kChroma
template <typename T>
auto luminance_kernel_of(int flags, const T*)
{
    static const auto table = luminance_kernel_table<T>(std::make_integer_sequence<int, 16>{});
    return table[flags];
}

} // namespace

cudaError_t launch_luminance(const void* samples, uint32_t sample_type, uint64_t texels, uint32_t N, float* lum,
                             uint64_t lum_stride, float* avg, void* lum_hi, void* lum_lo, const uint16_t* hilo_pos,
                             cudaStream_t stream, void* rgb16, uint64_t rgb_stride, const LumFeatures& features)
{
    if(texels == 0)
        return cudaSuccess;
    if((lum_hi == nullptr) != (lum_lo == nullptr) || texels > 0x7fffffffull)
        return cudaErrorInvalidValue;
    // the split: a column table, 16-byte rows and bases
    if(lum_hi && (!hilo_pos || lum_stride % 8 != 0 || (reinterpret_cast<uintptr_t>(lum_hi) & 15u) ||
                  (reinterpret_cast<uintptr_t>(lum_lo) & 15u)))
        return cudaErrorInvalidValue;
    if(features.X && !(features.pos && features.start && features.bin_w && features.pair_pos &&
                       (features.mean == nullptr) == (features.rstd == nullptr) && N <= 65536u))
        return cudaErrorInvalidValue;
    __nv_bfloat16* hi = static_cast<__nv_bfloat16*>(lum_hi);
    __nv_bfloat16* lo = static_cast<__nv_bfloat16*>(lum_lo);
    const auto run = [&](auto kernel, const auto* src) -> cudaError_t {
        using T = std::remove_cv_t<std::remove_pointer_t<decltype(src)>>;
        const bool hl = hi != nullptr;
        const size_t smem = features.X ? LumPass<T, true>::smem(N, lum_stride, hl)
                                       : LumPass<T, false>::smem(N, lum_stride, hl);
        if(smem > 48 * 1024)
        {
            const cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if(e != cudaSuccess)
                return e;
        }
        kernel<<<(unsigned)texels, kLumThreads, smem, stream>>>(src, N, lum, lum_stride, avg, hi, lo, hilo_pos,
                                                                static_cast<__half*>(rgb16), rgb_stride, features);
        return cudaGetLastError();
    };
    const int flags = (hi ? 1 : 0) | (rgb16 ? 2 : 0) | (features.X ? 4 : 0) | (avg ? 8 : 0);
    if(sample_type == SVF_SAMPLES_F16)
        return run(luminance_kernel_of(flags, static_cast<const __half*>(samples)), static_cast<const __half*>(samples));
    return run(luminance_kernel_of(flags, static_cast<const float*>(samples)), static_cast<const float*>(samples));
}

__global__ void rgb_init_kernel(const float* __restrict__ init7, const float* __restrict__ avg, uint64_t texels,
                                float* __restrict__ init12)
{
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(t >= texels)
        return;
    const float* p = init7 + 7 * t;
    const float* a = avg + 3 * t;
    float* o = init12 + 12 * t;
    for(int k = 0; k < 3; ++k)
    {
        o[k] = a[k] * p[3];
        o[3 + k] = a[k] * p[2];
    }
    o[6] = p[0];
    o[7] = p[1];
    // ToQuaternion(euler), quaternion.hh:82-94
    float s1, c1, s2, c2, s3, c3;
    sincosf(0.5f * p[4], &s1, &c1);
    sincosf(0.5f * p[5], &s2, &c2);
    sincosf(0.5f * p[6], &s3, &c3);
    o[8] = s1 * c2 * c3 + c1 * s2 * s3;
    o[9] = -s1 * c2 * s3 + c1 * s2 * c3;
    o[10] = c1 * c2 * s3 + s1 * s2 * c3;
    o[11] = c1 * c2 * c3 - s1 * s2 * s3;
}

cudaError_t launch_rgb_init(const float* init7, const float* avg_chroma, uint64_t texels, float* init12,
                            cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    rgb_init_kernel<<<(unsigned)((texels + 127) / 128), 128, 0, stream>>>(init7, avg_chroma, texels, init12);
    return cudaGetLastError();
}

cudaError_t launch_repack(const float* src, uint64_t src_stride, uint64_t texels, uint32_t N, float* dst,
                          uint64_t dst_stride, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    repack_kernel<<<(unsigned)texels, 256, 0, stream>>>(src, src_stride, N, dst, dst_stride);
    return cudaGetLastError();
}

cudaError_t launch_synth(uint32_t seed, uint32_t mix, const float* lp, uint32_t L, uint64_t first, uint64_t count,
                         uint32_t sample_type, float noise, void* samples, float* truth, cudaStream_t stream)
{
    if(count == 0)
        return cudaSuccess;
    if(sample_type == SVF_SAMPLES_F16)
        synth_kernel<__half><<<(unsigned)count, 256, 0, stream>>>(seed, mix, lp, L, first, noise,
                                                                static_cast<__half*>(samples), truth);
    else
        synth_kernel<float><<<(unsigned)count, 256, 0, stream>>>(seed, mix, lp, L, first, noise,
                                                               static_cast<float*>(samples), truth);
    return cudaGetLastError();
}

// ---- neighbourhood refit (svbrdffit -j, svbrdf-fitting.cc:123-178) ----------------

namespace
{

// Candidate k (0..8, the 3x3 neighbourhood row by row) of texel c0 + i starts
// from the neighbour's parameters; a neighbour outside the image gives the
// texel's own (the candidate is then ignored).
__global__ void refit_gather_kernel(const float* __restrict__ params, uint64_t c0, uint64_t n, uint32_t width,
                                    uint32_t height, float* __restrict__ cand)
{
    const uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(j >= 9 * n)
        return;
    const uint64_t k = j / n, i = j - k * n, t = c0 + i;
    const int64_t y = (int64_t)(t / width), x = (int64_t)(t - (uint64_t)y * width);
    const int64_t ny = y + (int64_t)(k / 3) - 1, nx = x + (int64_t)(k % 3) - 1;
    const bool in = ny >= 0 && ny < height && nx >= 0 && nx < width;
    const uint64_t src = in ? (uint64_t)ny * width + (uint64_t)nx : t;
    for(int p = 0; p < 7; ++p)
        cand[7 * j + p] = params[7 * src + p];
}

// The texel keeps its parameters unless a candidate's RMSE is lower; candidates
// are taken in neighbourhood order with a strict comparison, as the reference's
// loop updates best_rmse.
__global__ void refit_select_kernel(const float* __restrict__ params, const float* __restrict__ rmse, uint64_t c0,
                                    uint64_t n, uint32_t width, uint32_t height, const float* __restrict__ cand_out,
                                    const float* __restrict__ cand_rmse, float* __restrict__ sel_params,
                                    float* __restrict__ sel_rmse, uint32_t* __restrict__ sel_from)
{
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    const uint64_t t = c0 + i;
    const int64_t y = (int64_t)(t / width), x = (int64_t)(t - (uint64_t)y * width);
    float best = rmse[t];
    int from = -1;
    for(int k = 0; k < 9; ++k)
    {
        const int64_t ny = y + k / 3 - 1, nx = x + k % 3 - 1;
        if(ny < 0 || ny >= height || nx < 0 || nx >= width)
            continue;
        const float r = cand_rmse[k * n + i];
        if(r < best)   // (NaN never wins)
        {
            best = r;
            from = k;
        }
    }
    const float* src = from < 0 ? params + 7 * t : cand_out + 7 * ((uint64_t)from * n + i);
    for(int p = 0; p < 7; ++p)
        sel_params[7 * i + p] = src[p];
    sel_rmse[i] = best;
    if(sel_from)
        sel_from[i] = (uint32_t)(from < 0 ? 9 : from);
}

} // namespace

cudaError_t launch_refit_gather(const float* params, uint64_t c0, uint64_t n, uint32_t width, uint32_t height,
                                float* cand, cudaStream_t stream)
{
    if(n == 0)
        return cudaSuccess;
    refit_gather_kernel<<<(unsigned)((9 * n + 255) / 256), 256, 0, stream>>>(params, c0, n, width, height, cand);
    return cudaGetLastError();
}

cudaError_t launch_refit_select(const float* params, const float* rmse, uint64_t c0, uint64_t n, uint32_t width,
                                uint32_t height, const float* cand_out, const float* cand_rmse, float* sel_params,
                                float* sel_rmse, uint32_t* sel_from, cudaStream_t stream)
{
    if(n == 0)
        return cudaSuccess;
    refit_select_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(params, rmse, c0, n, width, height, cand_out,
                                                                       cand_rmse, sel_params, sel_rmse, sel_from);
    return cudaGetLastError();
}

// ---- learned guess: fallback to the default guess ---------------------------------

namespace
{

// Texel t is selected when its RMSE relative to the RMS of its luminance slice
// is above the threshold (one CTA per texel; the order of the selected list
// follows the atomics, which changes nothing: each texel is fitted on its own).
__global__ void __launch_bounds__(256) fallback_select_kernel(const float* __restrict__ lum, uint64_t stride,
                                                              uint32_t N, const float* __restrict__ rmse,
                                                              float threshold, uint32_t* __restrict__ idx,
                                                              uint32_t* __restrict__ count)
{
    const uint64_t t = blockIdx.x;
    const float* y = lum + t * stride;
    double s = 0.0;
    for(uint32_t i = threadIdx.x; i < N; i += blockDim.x)
        s += (double)y[i] * y[i];
    __shared__ double red[8];
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = s;
    __syncthreads();
    if(threadIdx.x == 0)
    {
        double tot = 0.0;
        for(int w = 0; w < (int)(blockDim.x >> 5); ++w)
            tot += red[w];
        const double rms = sqrt(tot / N);
        if(rms > 0.0 && (double)rmse[t] > threshold * rms)
            idx[atomicAdd(count, 1u)] = (uint32_t)t;
    }
}

__global__ void gather_slabs_kernel(const float* __restrict__ lum, uint64_t stride, const float* __restrict__ avg,
                                    const uint32_t* __restrict__ idx, float* __restrict__ g_lum,
                                    float* __restrict__ g_avg)
{
    const uint64_t i = blockIdx.x;
    const uint64_t t = idx[i];
    for(uint64_t k = threadIdx.x; k < stride; k += blockDim.x)
        g_lum[i * stride + k] = lum[t * stride + k];
    if(avg && threadIdx.x < 3)   // the average chromaticity, when it was computed
        g_avg[3 * i + threadIdx.x] = avg[3 * t + threadIdx.x];
}

// The default-guess fit of selected texel i replaces the learned-guess fit of
// texel idx[i] when its RMSE is lower.  Maps: diffuse 3 | specular 3 | sigma 2 |
// basis 4, each a block of n (resp. m) texels.
__global__ void fallback_merge_kernel(const uint32_t* __restrict__ idx, uint32_t m, const float* __restrict__ g_out,
                                      const float* __restrict__ g_rmse, const svf_texel_stats* __restrict__ g_stats,
                                      const float* __restrict__ g_maps, const float* __restrict__ g_init,
                                      uint64_t n, float* __restrict__ out, float* __restrict__ rmse,
                                      svf_texel_stats* __restrict__ stats, float* __restrict__ maps,
                                      float* __restrict__ init, uint32_t* __restrict__ taken)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= m)
        return;
    const uint64_t t = idx[i];
    if(!(g_rmse[i] < rmse[t]))
        return;
    atomicAdd(taken, 1u);
    for(int p = 0; p < 7; ++p)
    {
        out[7 * t + p] = g_out[7 * i + p];
        init[7 * t + p] = g_init[7 * i + p];
    }
    rmse[t] = g_rmse[i];
    if(stats)
        stats[t] = g_stats[i];
    for(int c = 0; c < 3; ++c)
    {
        maps[3 * t + c] = g_maps[3 * i + c];
        maps[3 * n + 3 * t + c] = g_maps[3 * (uint64_t)m + 3 * i + c];
    }
    for(int c = 0; c < 2; ++c)
        maps[6 * n + 2 * t + c] = g_maps[6 * (uint64_t)m + 2 * i + c];
    for(int c = 0; c < 4; ++c)
        maps[8 * n + 4 * t + c] = g_maps[8 * (uint64_t)m + 4 * i + c];
}

} // namespace

cudaError_t launch_fallback_select(const float* lum, uint64_t stride, uint32_t N, const float* rmse, uint64_t n,
                                   float threshold, uint32_t* idx, uint32_t* count, cudaStream_t stream)
{
    if(n == 0)
        return cudaSuccess;
    fallback_select_kernel<<<(unsigned)n, 256, 0, stream>>>(lum, stride, N, rmse, threshold, idx, count);
    return cudaGetLastError();
}

cudaError_t launch_gather_slabs(const float* lum, uint64_t stride, const float* avg, const uint32_t* idx, uint32_t m,
                                float* g_lum, float* g_avg, cudaStream_t stream)
{
    if(m == 0)
        return cudaSuccess;
    gather_slabs_kernel<<<m, 256, 0, stream>>>(lum, stride, avg, idx, g_lum, g_avg);
    return cudaGetLastError();
}

cudaError_t launch_fallback_merge(const uint32_t* idx, uint32_t m, const float* g_out, const float* g_rmse,
                                  const svf_texel_stats* g_stats, const float* g_maps, const float* g_init, uint64_t n,
                                  float* out, float* rmse, svf_texel_stats* stats, float* maps, float* init,
                                  uint32_t* taken, cudaStream_t stream)
{
    if(m == 0)
        return cudaSuccess;
    fallback_merge_kernel<<<(m + 255) / 256, 256, 0, stream>>>(idx, m, g_out, g_rmse, g_stats, g_maps, g_init, n, out,
                                                               rmse, stats, maps, init, taken);
    return cudaGetLastError();
}

} // namespace svf
