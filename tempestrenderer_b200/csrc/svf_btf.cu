// svf_btf.cu - decode of a factored BTF (DFMF / FMF planes resident in HBM)
// into RGB samples [texels][L*L][3], texel-major, as svf_fit_texels reads them.
//
// Reference: BTFEvaluateMatrix (include/tempest/image/btf.hh:608-634) and
// BTFFetchSpectrum (btf.hh:498-556).  Channel c of sample (lv, texel) is
// sum_k U_c[lv][k] * SxV_c[col][k], summed in order k = 0, 1, ... in the
// accumulator type of the plane elements (float for half and float planes,
// double for double planes) with every product rounded before it is added, as
// the reference's x86-64 build evaluates it; then colour model 11 (log-YUV ->
// RGB) and the dynamic range reduction exp(x) - 1e-5.  col is the file column
// of texel y*W + x: LoadBTF flips rows (btf.cc:1000-1022), so it is
// (H - 1 - y)*W + x.
//
// The sums are bit-identical to the reference's; with colour model 11 or DRR
// the exponentials are CUDA's expf (within 2 ulp of libm's), so those samples
// agree to a few ulp.
//
// Work split: a CTA of 128 threads owns 128 consecutive pairs lv (one per
// thread) and TX texels (16 for half planes, whose accumulators then leave room
// for more resident CTAs; 32 for float planes).  Per chunk of 32 components the CTA stages, with
// coalesced loads, the 128 U rows (transposed, padded: a thread reads its pair's
// value conflict-free) and the TX texels' SxV rows (transposed: a thread reads
// TX of them with vector broadcasts) in shared memory.  Half planes accumulate
// with FMAs (a product of two halves is exact in float, so the FMA rounds as the
// reference's separate multiply and add do); float and double planes need the
// separate multiply and add.  Writes: a warp stores 32 consecutive pairs x 3
// channels of one texel at a time (384 contiguous bytes in FP32).  Bound by
// the FP32 pipe for K >= ~20 components, by the HBM write otherwise.
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "svf_internal.h"

namespace svf
{

namespace
{

constexpr int kThreads = 128, kChunk = 32;

__device__ __forceinline__ float elem(const __half* p, uint64_t i) { return __half2float(p[i]); }
__device__ __forceinline__ float elem(const float* p, uint64_t i) { return p[i]; }
__device__ __forceinline__ double elem(const double* p, uint64_t i) { return p[i]; }

// sum + u * v with the product rounded first (no contraction into an FMA,
// which would round once); for half elements the product is exact in float and
// an FMA gives the same result.
template <typename T>
__device__ __forceinline__ float madd(float sum, float u, float v) { return __fadd_rn(sum, __fmul_rn(u, v)); }
template <>
__device__ __forceinline__ float madd<__half>(float sum, float u, float v) { return __fmaf_rn(u, v, sum); }
template <typename T>
__device__ __forceinline__ double madd(double sum, double u, double v) { return __dadd_rn(sum, __dmul_rn(u, v)); }

// The epilogue of a CTA: colour model 11 and DRR, then the TX texels' samples
// of its 128 pairs, a warp storing 32 consecutive pairs x RGB of one texel at
// a time.
template <typename Acc, int TX>
__device__ __forceinline__ void store_texels(const BtfDecodeArgs& a, const Acc (&acc)[3][TX], uint64_t t0,
                                             uint32_t lv0)
{
    __shared__ float s_out[kThreads / 32][96];   // one texel's 32 pairs x RGB per warp
    const uint64_t t_end = a.first + a.count;
    const float eps = 1e-5f;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t lv_w = lv0 + warp * 32;   // the warp's first pair
    const uint32_t nvalid = lv_w >= a.N ? 0u : (a.N - lv_w < 32u ? a.N - lv_w : 32u);
#pragma unroll
    for(int j = 0; j < TX; ++j)
    {
        const uint64_t t = t0 + j;
        if(t >= t_end)
            break;   // (the same for the whole CTA)
        float r = (float)acc[0][j], g = (float)acc[1][j], b = (float)acc[2][j];
        if(a.color_model == 11)
        {
            // btf.hh:522-531 and YUVToRGB (spectrum.hh:344-350): dot products
            // with the conversion's columns, left to right, then a clamp to [0, 1]
            const float Y = __fsub_rn(expf(r), eps);
            const float U = __fadd_rn(__fmul_rn(g, Y), eps);
            const float V = __fadd_rn(__fmul_rn(b, Y), eps);
            float o[3];
            o[0] = __fadd_rn(__fadd_rn(__fmul_rn(Y, 1.0f), __fmul_rn(U, 0.0f)), __fmul_rn(V, 1.13983f));
            o[1] = __fadd_rn(__fadd_rn(__fmul_rn(Y, 1.0f), __fmul_rn(U, -0.39465f)), __fmul_rn(V, -0.5806f));
            o[2] = __fadd_rn(__fadd_rn(__fmul_rn(Y, 1.0f), __fmul_rn(U, 2.03211f)), __fmul_rn(V, 0.0f));
            // Clamp (functions.hh:156-159)
#pragma unroll
            for(int i = 0; i < 3; ++i)
                o[i] = o[i] <= 0.0f ? 0.0f : (o[i] >= 1.0f ? 1.0f : o[i]);
            r = o[0];
            g = o[1];
            b = o[2];
        }
        if(a.drr)
        {
            r = __fsub_rn(expf(r), eps);
            g = __fsub_rn(expf(g), eps);
            b = __fsub_rn(expf(b), eps);
        }
        // the warp's 32 samples are 96 consecutive values: stage them and store
        // them lane-consecutive (each store instruction covers 32 neighbours)
        s_out[warp][3 * lane] = r;
        s_out[warp][3 * lane + 1] = g;
        s_out[warp][3 * lane + 2] = b;
        __syncwarp();
        const uint64_t o = ((t - a.first) * a.N + lv_w) * 3;
        if(a.out_type == SVF_SAMPLES_F16)
        {
            __half* out = static_cast<__half*>(a.out) + o;
            for(uint32_t e = lane; e < 3 * nvalid; e += 32)
                out[e] = __float2half_rn(s_out[warp][e]);
        }
        else
        {
            float* out = static_cast<float*>(a.out) + o;
            for(uint32_t e = lane; e < 3 * nvalid; e += 32)
                out[e] = s_out[warp][e];
        }
        __syncwarp();
    }
}

template <typename T, typename Acc, int TX>
__global__ void __launch_bounds__(kThreads) btf_decode_kernel(BtfDecodeArgs a, uint64_t t_begin)
{
    // rows padded by 4: the staging writes of one warp (32 components of one
    // texel) spread over 8 banks, and rows stay 16-byte aligned for the
    // vector broadcasts of the inner loop
    __shared__ __align__(16) Acc s_sxv[kChunk][TX + 4];
    __shared__ Acc s_u[kChunk][kThreads + 1];
    __shared__ uint64_t s_col[TX];   // file column of each texel (after the row flip)
    const uint32_t lv0 = blockIdx.x * kThreads;
    const uint64_t t0 = t_begin + (uint64_t)blockIdx.y * TX;
    const uint64_t t_end = a.first + a.count;
    if(threadIdx.x < TX)
    {
        const uint64_t t = t0 + threadIdx.x;
        const uint64_t y = t / a.width, x = t - y * a.width;
        s_col[threadIdx.x] = t < t_end ? (a.height - 1 - y) * a.width + x : ~0ull;
    }
    Acc acc[3][TX];
#pragma unroll
    for(int c = 0; c < 3; ++c)
#pragma unroll
        for(int j = 0; j < TX; ++j)
            acc[c][j] = Acc(0);

#pragma unroll
    for(int c = 0; c < 3; ++c)
    {
        const T* U = static_cast<const T*>(a.u[c]);
        const T* S = static_cast<const T*>(a.sxv[c]);
        const uint32_t K = a.k[c];
        for(uint32_t k0 = 0; k0 < K; k0 += kChunk)
        {
            __syncthreads();
            // a warp reads 32 consecutive components of one row per step
            const int kk = threadIdx.x % kChunk, r0 = threadIdx.x / kChunk;
            const bool k_ok = k0 + kk < K;
            for(int j = r0; j < TX; j += kThreads / kChunk)
            {
                const uint64_t col = s_col[j];
                s_sxv[kk][j] = (col != ~0ull && k_ok) ? elem(S, col * a.sxv_row[c] + k0 + kk) : Acc(0);
            }
            {
                const T* up = U + (uint64_t)(lv0 + r0) * a.u_row[c] + k0 + kk;
                const uint64_t step = (uint64_t)(kThreads / kChunk) * a.u_row[c];
                for(int row = r0; row < kThreads; row += kThreads / kChunk, up += step)
                    s_u[kk][row] = (lv0 + row < a.N && k_ok) ? elem(up, 0) : Acc(0);
            }
            __syncthreads();
            const uint32_t n = K - k0 < (uint32_t)kChunk ? K - k0 : (uint32_t)kChunk;
            for(uint32_t kk = 0; kk < n; ++kk)
            {
                const Acc u = s_u[kk][threadIdx.x];
#pragma unroll
                for(int j = 0; j < TX; ++j)
                    acc[c][j] = madd<T>(acc[c][j], u, s_sxv[kk][j]);
            }
        }
    }
    store_texels<Acc, TX>(a, acc, t0, lv0);
}

// 4-byte asynchronous copy global -> shared (cp.async, L1-allocating), the
// bytes past src_bytes (0, 2 or 4) zero-filled.
__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes)
{
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Half planes with 4-byte aligned rows: the same sums as btf_decode_kernel, the
// staging double-buffered so that the next chunk's loads run under this
// chunk's FMAs.  U arrives by cp.async as half2 words (components k, k+1 of a
// pair's row; word rows padded to 130 so that the copies of a warp, two pairs x
// 16 words, hit 32 banks, and a thread's read of its pair is conflict-free);
// SxV through registers, converted to float and transposed as before.  The
// chunk sequence runs over the three channels, each channel's accumulator row
// selected by a compile-time switch.
template <int TX>
__global__ void __launch_bounds__(kThreads) btf_decode_half_async_kernel(BtfDecodeArgs a, uint64_t t_begin)
{
    constexpr int kWords = kChunk / 2, kRowWords = kThreads + 2;
    constexpr int kSx = TX * kChunk / kThreads;   // SxV elements a thread stages per chunk
    static_assert(TX * kChunk % kThreads == 0, "SxV staging split");
    __shared__ uint32_t s_u[2][kWords][kRowWords];
    __shared__ __align__(16) float s_sxv[2][kChunk][TX + 4];
    __shared__ uint64_t s_col[TX];
    const uint32_t lv0 = blockIdx.x * kThreads;
    const uint64_t t0 = t_begin + (uint64_t)blockIdx.y * TX;
    const uint64_t t_end = a.first + a.count;
    if(threadIdx.x < TX)
    {
        const uint64_t t = t0 + threadIdx.x;
        const uint64_t y = t / a.width, x = t - y * a.width;
        s_col[threadIdx.x] = t < t_end ? (a.height - 1 - y) * a.width + x : ~0ull;
    }
    __syncthreads();
    // chunks: (channel, first component)
    uint32_t nq[3];
    for(int c = 0; c < 3; ++c)
        nq[c] = (a.k[c] + kChunk - 1) / kChunk;
    const uint32_t n_chunks = nq[0] + nq[1] + nq[2];
    auto chunk = [&](uint32_t q, int& c, uint32_t& k0) {
        c = q < nq[0] ? 0 : (q < nq[0] + nq[1] ? 1 : 2);
        k0 = (q - (c == 0 ? 0 : (c == 1 ? nq[0] : nq[0] + nq[1]))) * kChunk;
    };
    // U: thread t copies words w = t % 16 of rows t / 16 + 8 i
    const int uw = threadIdx.x % kWords, ur = threadIdx.x / kWords;
    auto issue_u = [&](uint32_t q, int buf) {
        int c;
        uint32_t k0;
        chunk(q, c, k0);
        const __half* U = static_cast<const __half*>(a.u[c]);
        const uint32_t K = a.k[c];
        const uint32_t k = k0 + 2 * uw;
        const uint32_t bytes = k + 1 < K ? 4u : (k < K ? 2u : 0u);
        for(int row = ur; row < kThreads; row += kThreads / kWords)
        {
            const bool ok = lv0 + row < a.N && bytes > 0;
            const __half* src = ok ? U + (uint64_t)(lv0 + row) * a.u_row[c] + k : U;
            cp_async4(&s_u[buf][uw][row], src, ok ? bytes : 0u);
        }
    };
    // SxV: thread t loads component t % 32 of texels t / 32 + 4 i
    const int sk = threadIdx.x % kChunk, sj = threadIdx.x / kChunk;
    float sx[kSx];
    auto load_sx = [&](uint32_t q) {
        int c;
        uint32_t k0;
        chunk(q, c, k0);
        const __half* S = static_cast<const __half*>(a.sxv[c]);
        const bool k_ok = k0 + sk < a.k[c];
#pragma unroll
        for(int i = 0; i < kSx; ++i)
        {
            const uint64_t col = s_col[sj + i * (kThreads / kChunk)];
            sx[i] = (col != ~0ull && k_ok) ? __half2float(S[col * a.sxv_row[c] + k0 + sk]) : 0.0f;
        }
    };
    auto store_sx = [&](int buf) {
#pragma unroll
        for(int i = 0; i < kSx; ++i)
            s_sxv[buf][sk][sj + i * (kThreads / kChunk)] = sx[i];
    };
    float acc[3][TX];
#pragma unroll
    for(int c = 0; c < 3; ++c)
#pragma unroll
        for(int j = 0; j < TX; ++j)
            acc[c][j] = 0.0f;
    auto compute = [&](float (&ac)[TX], int buf, uint32_t n) {
        for(uint32_t kk = 0; kk < n; kk += 2)
        {
            const uint32_t w = s_u[buf][kk >> 1][threadIdx.x];
            const float u0 = __half2float(__ushort_as_half((unsigned short)(w & 0xffffu)));
            const float u1 = __half2float(__ushort_as_half((unsigned short)(w >> 16)));
#pragma unroll
            for(int j = 0; j < TX; ++j)
                ac[j] = __fmaf_rn(u0, s_sxv[buf][kk][j], ac[j]);
            if(kk + 1 < n)
#pragma unroll
                for(int j = 0; j < TX; ++j)
                    ac[j] = __fmaf_rn(u1, s_sxv[buf][kk + 1][j], ac[j]);
        }
    };
    issue_u(0, 0);
    cp_async_commit();
    load_sx(0);
    for(uint32_t q = 0; q < n_chunks; ++q)
    {
        const int buf = q & 1;
        store_sx(buf);
        if(q + 1 < n_chunks)
        {
            issue_u(q + 1, buf ^ 1);
            cp_async_commit();
            load_sx(q + 1);
            cp_async_wait<1>();
        }
        else
            cp_async_wait<0>();
        __syncthreads();
        int c;
        uint32_t k0;
        chunk(q, c, k0);
        const uint32_t n = a.k[c] - k0 < (uint32_t)kChunk ? a.k[c] - k0 : (uint32_t)kChunk;
        if(c == 0)
            compute(acc[0], buf, n);
        else if(c == 1)
            compute(acc[1], buf, n);
        else
            compute(acc[2], buf, n);
        __syncthreads();
    }
    cp_async_wait<0>();   // (no copy outlives the CTA, also when there was no chunk)
    store_texels<float, TX>(a, acc, t0, lv0);
}

template <typename T, typename Acc, int TX>
cudaError_t launch_typed(const BtfDecodeArgs& a, cudaStream_t stream)
{
    const uint64_t per_launch = 65535ull * TX;   // grid.y limit
    for(uint64_t t = a.first; t < a.first + a.count; t += per_launch)
    {
        const uint64_t n = a.first + a.count - t < per_launch ? a.first + a.count - t : per_launch;
        dim3 grid((a.N + kThreads - 1) / kThreads, (unsigned)((n + TX - 1) / TX));
        btf_decode_kernel<T, Acc, TX><<<grid, kThreads, 0, stream>>>(a, t);
        const cudaError_t e = cudaGetLastError();
        if(e != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

} // namespace

cudaError_t launch_btf_decode(const BtfDecodeArgs& a, cudaStream_t stream)
{
    if(a.count == 0)
        return cudaSuccess;
    switch(a.data_size)
    {
    case 2:
    {
        // the asynchronous staging wants every U row 4-byte aligned
        bool aligned = true;
        for(int c = 0; c < 3; ++c)
            aligned = aligned && (a.u_row[c] % 2 == 0) && ((uintptr_t)a.u[c] % 4 == 0);
        if(!aligned)
            return launch_typed<__half, float, 16>(a, stream);
        constexpr int TX = 16;
        const uint64_t per_launch = 65535ull * TX;
        for(uint64_t t = a.first; t < a.first + a.count; t += per_launch)
        {
            const uint64_t n = a.first + a.count - t < per_launch ? a.first + a.count - t : per_launch;
            dim3 grid((a.N + kThreads - 1) / kThreads, (unsigned)((n + TX - 1) / TX));
            btf_decode_half_async_kernel<TX><<<grid, kThreads, 0, stream>>>(a, t);
            const cudaError_t e = cudaGetLastError();
            if(e != cudaSuccess)
                return e;
        }
        return cudaSuccess;
    }
    case 4: return launch_typed<float, float, 32>(a, stream);
    case 8: return launch_typed<double, double, 16>(a, stream);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace svf
