// svf_mlp.cu - the learned initial guess: a small MLP that maps a summary of a
// texel's luminance slab to the luminance fit's parameters, trained on texels
// the plain LM has fitted.  No counterpart in the reference (its only initial
// guess is the NDF -> PCA -> projection pipeline, svbrdf-fitting-pipeline.cc:
// 350-660); LM refinement always follows.
//
//   features  x = (log max(v, 1e-6) - mean) / std, 96 values, one of:
//             32 fixed direction pairs x RGB (SVF_MLP_FEATURES_PAIRS_RGB), or
//             64 half-vector bins (mean luminance of the direction pairs whose
//             half vector falls in the bin) and 32 pairs' luminance
//             (SVF_MLP_FEATURES_BINS)
//   network   96 -> 256 -> 256 -> 8, GELU (tanh form) between layers
//   targets   (log S (6 elements), log(ks + 1e-4), log(kd + 1e-4)) - mean) / std
//             with S = R diag(sx^2, sy^2, 1) R^T the SGGX matrix: its logarithm
//             R diag(2 log sx, 2 log sy, 0) R^T depends continuously on the lobe
//             and not on the choice among the frames that give the same lobe
//   decoding  a 3x3 symmetric Jacobi eigendecomposition of the predicted log S:
//             the eigenvalue nearest 0 is the normal's, the other two give sx,
//             sy and the tangent frame
//
// Training kernels: one tiled FP32 GEMM with transposes and fused bias / GELU /
// GELU-derivative epilogues, column statistics, the MSE gradient and Adam.
// Inference: the hidden layers on the tcgen05 tensor cores (the BF16x3 GEMM of
// svf_ndf_tc.cu, FP32 accuracy), the output layer fused into the second
// layer's epilogue.  The bin features are computed by the luminance pass
// (svf_kernels.cu) from the slab it holds in shared memory.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "svf_internal.h"
#include "svf_model.cuh"

namespace svf
{

namespace
{

constexpr int kTile = 64, kTileK = 16, kGemmThreads = 256;   // 64 x 64 tile, 4 x 4 per thread

__device__ __forceinline__ float gelu(float x)
{
    const float k = 0.7978845608f;   // sqrt(2 / pi)
    return 0.5f * x * (1.0f + tanhf(k * (x + 0.044715f * x * x * x)));
}

__device__ __forceinline__ float gelu_grad(float x)
{
    const float k = 0.7978845608f;
    const float u = k * (x + 0.044715f * x * x * x);
    const float t = tanhf(u);
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * k * (1.0f + 3.0f * 0.044715f * x * x);
}

__device__ __forceinline__ float to_f(float x) { return x; }
__device__ __forceinline__ float to_f(__half x) { return __half2float(x); }

// C[M][N] = op(A) op(B) with op(A)[m][k] = kTA ? A[k][m] : A[m][k] and
// op(B)[k][n] = kTB ? B[n][k] : B[k][n] (leading dimensions lda, ldb); then
// + bias[n]; mode 1: Z = C, C = gelu(Z); mode 2: C *= gelu'(Zin).
template <bool kTA, bool kTB>
__global__ void __launch_bounds__(kGemmThreads) gemm_kernel(int M, int N, int K, const float* __restrict__ A, int lda,
                                                            const float* __restrict__ B, int ldb, float* __restrict__ C,
                                                            int ldc, const float* __restrict__ bias, int mode,
                                                            float* __restrict__ Z, const float* __restrict__ Zin)
{
    __shared__ float As[kTileK][kTile + 1];
    __shared__ float Bs[kTileK][kTile + 1];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
    float acc[4][4] = {};
    for(int k0 = 0; k0 < K; k0 += kTileK)
    {
        for(int i = threadIdx.x; i < kTile * kTileK; i += kGemmThreads)
        {
            const int mm = i / kTileK, kk = i % kTileK;
            const int m = m0 + mm, k = k0 + kk;
            As[kk][mm] = (m < M && k < K) ? (kTA ? A[(size_t)k * lda + m] : A[(size_t)m * lda + k]) : 0.0f;
            const int n = n0 + mm;
            Bs[kk][mm] = (n < N && k < K) ? (kTB ? B[(size_t)n * ldb + k] : B[(size_t)k * ldb + n]) : 0.0f;
        }
        __syncthreads();
#pragma unroll
        for(int kk = 0; kk < kTileK; ++kk)
        {
            float a[4], b[4];
#pragma unroll
            for(int i = 0; i < 4; ++i)
            {
                a[i] = As[kk][ty * 4 + i];
                b[i] = Bs[kk][tx * 4 + i];
            }
#pragma unroll
            for(int i = 0; i < 4; ++i)
#pragma unroll
                for(int j = 0; j < 4; ++j)
                    acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for(int i = 0; i < 4; ++i)
    {
        const int m = m0 + ty * 4 + i;
        if(m >= M)
            continue;
#pragma unroll
        for(int j = 0; j < 4; ++j)
        {
            const int n = n0 + tx * 4 + j;
            if(n >= N)
                continue;
            float v = acc[i][j] + (bias ? bias[n] : 0.0f);
            if(mode == 1)
            {
                if(Z)
                    Z[(size_t)m * ldc + n] = v;
                v = gelu(v);
            }
            else if(mode == 2)
                v *= gelu_grad(Zin[(size_t)m * ldc + n]);
            C[(size_t)m * ldc + n] = v;
        }
    }
}

// out[n] = sum_m X[m][n] (and, with out2, sum of squares), in FP64
__global__ void colsum_kernel(const float* __restrict__ X, int M, int N, double* __restrict__ out,
                              double* __restrict__ out2)
{
    const int n = blockIdx.x;
    double s = 0.0, s2 = 0.0;
    for(int m = threadIdx.x; m < M; m += blockDim.x)
    {
        const double v = X[(size_t)m * N + n];
        s += v;
        s2 += v * v;
    }
    __shared__ double r[2][256];
    r[0][threadIdx.x] = s;
    r[1][threadIdx.x] = s2;
    __syncthreads();
    for(int o = blockDim.x / 2; o > 0; o >>= 1)
    {
        if((int)threadIdx.x < o)
        {
            r[0][threadIdx.x] += r[0][threadIdx.x + o];
            r[1][threadIdx.x] += r[1][threadIdx.x + o];
        }
        __syncthreads();
    }
    if(threadIdx.x == 0)
    {
        out[n] = r[0][0];
        if(out2)
            out2[n] = r[1][0];
    }
}

// FP32 copy of a double vector
__global__ void to_float_kernel(const double* __restrict__ x, int n, float scale, float* __restrict__ y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if(i < n)
        y[i] = (float)(x[i] * scale);
}

// X[m][n] = (X[m][n] - mean[n]) * rstd[n]
__global__ void normalize_kernel(float* __restrict__ X, int M, int N, const float* __restrict__ mean,
                                 const float* __restrict__ rstd)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if(i < (size_t)M * N)
    {
        const int n = (int)(i % N);
        X[i] = (X[i] - mean[n]) * rstd[n];
    }
}

// dY = 2 (Y - T) / (M N); loss += sum (Y - T)^2 / (M N)
__global__ void mse_grad_kernel(const float* __restrict__ Y, const float* __restrict__ T, int M, int N,
                                float* __restrict__ dY, double* __restrict__ loss)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    double l = 0.0;
    if(i < (size_t)M * N)
    {
        const float d = Y[i] - T[i];
        dY[i] = 2.0f * d / (float)((size_t)M * N);
        l = (double)d * d / (double)((size_t)M * N);
    }
    for(int o = 16; o > 0; o >>= 1)
        l += __shfl_xor_sync(0xffffffffu, l, o);
    if((threadIdx.x & 31u) == 0 && l != 0.0)
        atomicAdd(loss, l);
}

// Adam (or plain SGD) on a flat parameter vector
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float c1, float c2,
                            int sgd)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if(i >= n)
        return;
    if(sgd)
    {
        w[i] -= lr * g[i];
        return;
    }
    const float mi = b1 * m[i] + (1.0f - b1) * g[i];
    const float vi = b2 * v[i] + (1.0f - b2) * g[i] * g[i];
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + 1e-8f);
}

// rows[i] = X[idx[i]] for both the features and the targets
__global__ void gather_rows_kernel(const float* __restrict__ X, int nx, const float* __restrict__ Y, int ny,
                                   const uint32_t* __restrict__ idx, int rows, float* __restrict__ Xb,
                                   float* __restrict__ Yb)
{
    const int r = blockIdx.x;
    if(r >= rows)
        return;
    const size_t src = idx[r];
    for(int j = threadIdx.x; j < nx; j += blockDim.x)
        Xb[(size_t)r * nx + j] = X[src * nx + j];
    for(int j = threadIdx.x; j < ny; j += blockDim.x)
        Yb[(size_t)r * ny + j] = Y[src * ny + j];
}

// Features of the 32 pairs' RGB samples (96 = 32 pairs x RGB), log-scaled and
// normalised (mean may be null)
template <typename T>
__global__ void features_rgb_kernel(const T* __restrict__ samples, uint64_t texels, uint32_t N,
                                    const uint32_t* __restrict__ pairs, const float* __restrict__ mean,
                                    const float* __restrict__ rstd, float* __restrict__ X)
{
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(i >= texels * kMlpInputs)
        return;
    const uint64_t t = i / kMlpInputs;
    const int f = (int)(i % kMlpInputs);
    const float y = to_f(samples[(t * N + pairs[f / 3]) * 3 + (f % 3)]);
    float x = logf(fmaxf(y, 1e-6f));
    if(mean)
        x = (x - mean[f]) * rstd[f];
    X[i] = x;
}

// Targets of a fitted texel (params7 {sx, sy, ks, kd, euler}): log S, log ks, log kd
__global__ void targets_kernel(const float* __restrict__ p7, uint64_t texels, float* __restrict__ Y)
{
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(t >= texels)
        return;
    const float* p = p7 + 7 * t;
    ParamSet ps;
    make_param_set(p, ps);
    const float* R = ps.R;   // columns R[0..2], R[3..5], R[6..8]
    const float l0 = 2.0f * logf(fmaxf(p[0], 1e-3f)), l1 = 2.0f * logf(fmaxf(p[1], 1e-3f));
    auto e = [&](int i, int j) { return l0 * R[i] * R[j] + l1 * R[3 + i] * R[3 + j]; };
    float* y = Y + kMlpOutputs * t;
    y[0] = e(0, 0);
    y[1] = e(1, 1);
    y[2] = e(2, 2);
    y[3] = e(0, 1);
    y[4] = e(0, 2);
    y[5] = e(1, 2);
    y[6] = logf(fmaxf(p[2], 0.0f) + 1e-4f);
    y[7] = logf(fmaxf(p[3], 0.0f) + 1e-4f);
}

// Cyclic Jacobi eigendecomposition of a symmetric 3x3 matrix (Golub & Van Loan,
// Matrix Computations, 8.5): a becomes diagonal, the columns of v the
// eigenvectors.  Each rotation zeroes a[p][q] with t = tan(angle), the root of
// t^2 + 2 theta t - 1 = 0 of smaller magnitude.
__host__ __device__ inline void jacobi3(float a[3][3], float v[3][3])
{
    for(int i = 0; i < 3; ++i)
        for(int j = 0; j < 3; ++j)
            v[i][j] = i == j ? 1.0f : 0.0f;
    for(int sweep = 0; sweep < 8; ++sweep)
    {
        const float off = a[0][1] * a[0][1] + a[0][2] * a[0][2] + a[1][2] * a[1][2];
        const float diag = a[0][0] * a[0][0] + a[1][1] * a[1][1] + a[2][2] * a[2][2];
        if(off <= 1e-14f * diag || off < 1e-30f)
            break;
        for(int r = 0; r < 3; ++r)
        {
            const int p = r == 2 ? 1 : 0, q = r == 0 ? 1 : 2;
            const float apq = a[p][q];
            if(fabsf(apq) < 1e-30f)
                continue;
            const float theta = (a[q][q] - a[p][p]) / (2.0f * apq);
            const float t = (theta >= 0.0f ? 1.0f : -1.0f) / (fabsf(theta) + sqrtf(theta * theta + 1.0f));
            const float c = 1.0f / sqrtf(t * t + 1.0f), s = t * c;
            for(int k = 0; k < 3; ++k)
            {
                const float kp = a[k][p], kq = a[k][q];
                a[k][p] = c * kp - s * kq;
                a[k][q] = s * kp + c * kq;
            }
            for(int k = 0; k < 3; ++k)
            {
                const float pk = a[p][k], qk = a[q][k];
                a[p][k] = c * pk - s * qk;
                a[q][k] = s * pk + c * qk;
            }
            for(int k = 0; k < 3; ++k)
            {
                const float kp = v[k][p], kq = v[k][q];
                v[k][p] = c * kp - s * kq;
                v[k][q] = s * kp + c * kq;
            }
        }
    }
}

// Network outputs (normalised) -> params7 {sx, sy, ks, kd, euler}
__global__ void finish_kernel(const float* __restrict__ Yn, uint64_t texels, const float* __restrict__ mean,
                              const float* __restrict__ std, float* __restrict__ p7)
{
    const uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(t >= texels)
        return;
    float y[kMlpOutputs];
    for(int k = 0; k < kMlpOutputs; ++k)
        y[k] = Yn[kMlpOutputs * t + k] * std[k] + mean[k];
    float a[3][3] = { { y[0], y[3], y[4] }, { y[3], y[1], y[5] }, { y[4], y[5], y[2] } }, v[3][3];
    jacobi3(a, v);
    const float lam[3] = { a[0][0], a[1][1], a[2][2] };
    // the normal: the eigenvalue nearest 0; the other two give sx >= sy
    int kn = 0;
    for(int k = 1; k < 3; ++k)
        if(fabsf(lam[k]) < fabsf(lam[kn]))
            kn = k;
    int k0 = kn == 0 ? 1 : 0, k1 = kn == 2 ? 1 : 2;
    if(lam[k1] > lam[k0])
    {
        const int s = k0;
        k0 = k1;
        k1 = s;
    }
    float* p = p7 + 7 * t;
    p[0] = fminf(expf(0.5f * lam[k0]), 4.0f);
    p[1] = fminf(expf(0.5f * lam[k1]), 4.0f);
    p[2] = fmaxf(expf(y[6]) - 1e-4f, 0.0f);
    p[3] = fmaxf(expf(y[7]) - 1e-4f, 0.0f);
    // a right-handed frame (first two columns from the eigenvectors, c = a x b)
    const float ca[3] = { v[0][k0], v[1][k0], v[2][k0] }, cb[3] = { v[0][k1], v[1][k1], v[2][k1] };
    const float c[3] = { ca[1] * cb[2] - ca[2] * cb[1], ca[2] * cb[0] - ca[0] * cb[2], ca[0] * cb[1] - ca[1] * cb[0] };
    // Euler angles of the frame with columns (ca, cb, c), as Matrix3::decompose
    // gives them (matrix3.hh:311-332): make_param_set reproduces the frame
    const float m20 = c[0];
    if(m20 >= 0.9999f)
    {
        p[4] = 0.0f;
        p[5] = 0.5f * kRefPi;
        p[6] = atan2f(ca[1], cb[1]);
    }
    else if(m20 <= -0.9999f)
    {
        p[4] = 0.0f;
        p[5] = -0.5f * kRefPi;
        p[6] = atan2f(ca[1], cb[1]);
    }
    else
    {
        p[4] = atan2f(-c[1], c[2]);
        p[5] = asinf(m20);
        p[6] = atan2f(-cb[0], ca[0]);
    }
}

// Inference weights of the two hidden layers for the tensor-core GEMMs, split
// x = hi + lo into BF16 pairs (the product of the split operands, three BF16
// MMAs with FP32 accumulation, carries FP32 accuracy): W1 [256][96] | W2
// [256][256], row-major (out x in).
__global__ void pack_weights_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ hi,
                                    __nv_bfloat16* __restrict__ lo)
{
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t n1 = (size_t)kMlpHidden * kMlpInputs, n2 = (size_t)kMlpHidden * kMlpHidden;
    if(i >= n1 + n2)
        return;
    const float v = i < n1 ? w[kMlpW1 + i] : w[kMlpW2 + (i - n1)];
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[i] = h;
    lo[i] = __float2bfloat16_rn(__fsub_rn(v, __bfloat162float(h)));
}

// Layer epilogue of the tensor-core path: a = gelu(C + bias), split into BF16
// hi/lo rows [rows][kMlpHidden] for the next GEMM's A operand.
__global__ void act_split_kernel(const float* __restrict__ C, uint64_t rows, const float* __restrict__ bias,
                                 __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo)
{
    const uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if(i >= rows * kMlpHidden)
        return;
    const float v = gelu(C[i] + bias[i % kMlpHidden]);
    const __nv_bfloat16 h = __float2bfloat16_rn(v);
    hi[i] = h;
    lo[i] = __float2bfloat16_rn(__fsub_rn(v, __bfloat162float(h)));
}

// Second layer's epilogue and the output layer in one pass over C: one warp per
// row, lane l holds h = gelu(C + b2) of columns 8l .. 8l+7 and the matching
// columns of W3 (in registers, loaded once per warp), Y[r][j] = sum_k h_k W3[j][k]
// + b3[j] in FP32 with a fixed butterfly reduction (every lane ends with the
// same bits).  Persistent warps stride over the rows.
__global__ void __launch_bounds__(256) act_out_kernel(const float* __restrict__ C, uint64_t rows,
                                                      const float* __restrict__ b2, const float* __restrict__ w3,
                                                      const float* __restrict__ b3, float* __restrict__ Y)
{
    static_assert(kMlpHidden == 32 * 8, "one warp covers a hidden row in 8-column slices");
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    float w[kMlpOutputs][8], b[8];
#pragma unroll
    for(int i = 0; i < 8; ++i)
    {
        b[i] = b2[8 * lane + i];
#pragma unroll
        for(int j = 0; j < kMlpOutputs; ++j)
            w[j][i] = w3[j * kMlpHidden + 8 * lane + i];
    }
    const float bo = b3[lane % kMlpOutputs];
    for(uint64_t r = warp; r < rows; r += warps)
    {
        const float4* src = reinterpret_cast<const float4*>(C + r * kMlpHidden + 8 * lane);
        const float4 u = src[0], v = src[1];
        const float a[8] = { u.x, u.y, u.z, u.w, v.x, v.y, v.z, v.w };
        float acc[kMlpOutputs];
#pragma unroll
        for(int j = 0; j < kMlpOutputs; ++j)
            acc[j] = 0.0f;
#pragma unroll
        for(int i = 0; i < 8; ++i)
        {
            const float h = gelu(a[i] + b[i]);
#pragma unroll
            for(int j = 0; j < kMlpOutputs; ++j)
                acc[j] = fmaf(h, w[j][i], acc[j]);
        }
#pragma unroll
        for(int off = 16; off > 0; off >>= 1)
#pragma unroll
            for(int j = 0; j < kMlpOutputs; ++j)
                acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], off);
        float out = acc[0];
#pragma unroll
        for(int j = 1; j < kMlpOutputs; ++j)
            out = lane == j ? acc[j] : out;
        if(lane < kMlpOutputs)
            Y[r * kMlpOutputs + lane] = out + bo;
    }
}

inline unsigned blocks_for(size_t n, unsigned threads) { return (unsigned)((n + threads - 1) / threads); }

} // namespace

cudaError_t mlp_gemm(bool ta, bool tb, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                     float* C, int ldc, const float* bias, int mode, float* Z, const float* Zin, cudaStream_t stream)
{
    dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
    if(grid.y > 65535)
        return cudaErrorInvalidValue;
#define SVF_GEMM(TA, TB) \
    gemm_kernel<TA, TB><<<grid, kGemmThreads, 0, stream>>>(M, N, K, A, lda, B, ldb, C, ldc, bias, mode, Z, Zin)
    if(!ta && tb)
        SVF_GEMM(false, true);
    else if(ta && !tb)
        SVF_GEMM(true, false);
    else if(!ta && !tb)
        SVF_GEMM(false, false);
    else
        return cudaErrorInvalidValue;
#undef SVF_GEMM
    return cudaGetLastError();
}

cudaError_t mlp_colsum(const float* X, int M, int N, double* sum, double* sumsq, cudaStream_t stream)
{
    colsum_kernel<<<N, 256, 0, stream>>>(X, M, N, sum, sumsq);
    return cudaGetLastError();
}

cudaError_t mlp_to_float(const double* x, int n, float scale, float* y, cudaStream_t stream)
{
    to_float_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(x, n, scale, y);
    return cudaGetLastError();
}

cudaError_t mlp_normalize(float* X, int M, int N, const float* mean, const float* rstd, cudaStream_t stream)
{
    normalize_kernel<<<blocks_for((size_t)M * N, 256), 256, 0, stream>>>(X, M, N, mean, rstd);
    return cudaGetLastError();
}

cudaError_t mlp_mse_grad(const float* Y, const float* T, int M, int N, float* dY, double* loss, cudaStream_t stream)
{
    mse_grad_kernel<<<blocks_for((size_t)M * N, 256), 256, 0, stream>>>(Y, T, M, N, dY, loss);
    return cudaGetLastError();
}

cudaError_t mlp_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, int step, bool sgd,
                     cudaStream_t stream)
{
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f / (1.0f - powf(b1, (float)step)), c2 = 1.0f / (1.0f - powf(b2, (float)step));
    adam_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(w, g, m, v, n, lr, b1, b2, c1, c2, sgd ? 1 : 0);
    return cudaGetLastError();
}


cudaError_t mlp_gather_rows(const float* X, int nx, const float* Y, int ny, const uint32_t* idx, int rows, float* Xb,
                            float* Yb, cudaStream_t stream)
{
    if(rows == 0)
        return cudaSuccess;
    gather_rows_kernel<<<rows, 128, 0, stream>>>(X, nx, Y, ny, idx, rows, Xb, Yb);
    return cudaGetLastError();
}

cudaError_t mlp_features_rgb(const void* samples, uint32_t sample_type, uint64_t texels, uint32_t N,
                             const uint32_t* pairs, const float* mean, const float* rstd, float* X, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    const unsigned b = (unsigned)((texels * kMlpInputs + 255) / 256);
    if(sample_type == SVF_SAMPLES_F16)
        features_rgb_kernel<__half><<<b, 256, 0, stream>>>(static_cast<const __half*>(samples), texels, N, pairs,
                                                            mean, rstd, X);
    else
        features_rgb_kernel<float><<<b, 256, 0, stream>>>(static_cast<const float*>(samples), texels, N, pairs, mean,
                                                           rstd, X);
    return cudaGetLastError();
}

cudaError_t mlp_pack_weights(const float* w, void* hi, void* lo, cudaStream_t stream)
{
    const size_t n = kMlpTcWeights;
    pack_weights_kernel<<<blocks_for(n, 256), 256, 0, stream>>>(w, static_cast<__nv_bfloat16*>(hi),
                                                                static_cast<__nv_bfloat16*>(lo));
    return cudaGetLastError();
}

cudaError_t mlp_forward_tc(const float* X, uint64_t rows, const void* w_hi, const void* w_lo, const float* params,
                           float* C, void* act, float* Y, uint32_t* error_flag, cudaStream_t stream)
{
    if(rows == 0)
        return cudaSuccess;
    __nv_bfloat16* a_hi = static_cast<__nv_bfloat16*>(act);
    const size_t o2 = (size_t)kMlpHidden * kMlpInputs;
    const __nv_bfloat16* whi = static_cast<const __nv_bfloat16*>(w_hi);
    const __nv_bfloat16* wlo = static_cast<const __nv_bfloat16*>(w_lo);
    // layer 1: A = X split, K = 96
    cudaError_t e = launch_split_bf16(X, rows * kMlpInputs, a_hi, a_hi + rows * kMlpInputs, stream);
    if(e != cudaSuccess)
        return e;
    e = launch_ndf_tc(a_hi, a_hi + rows * kMlpInputs, rows, kMlpInputs, whi, wlo, kMlpHidden, kMlpInputs, kMlpInputs,
                      C, kMlpHidden, error_flag, stream);
    if(e != cudaSuccess)
        return e;
    const unsigned bh = blocks_for(rows * kMlpHidden, 256);
    __nv_bfloat16* a_lo = a_hi + rows * kMlpHidden;
    act_split_kernel<<<bh, 256, 0, stream>>>(C, rows, params + kMlpB1, a_hi, a_lo);
    // layer 2
    e = launch_ndf_tc(a_hi, a_lo, rows, kMlpHidden, whi + o2, wlo + o2, kMlpHidden, kMlpHidden, kMlpHidden, C,
                      kMlpHidden, error_flag, stream);
    if(e != cudaSuccess)
        return e;
    // layer 2's activation and the 8-output layer
    const uint64_t blocks = std::min<uint64_t>((rows + 7) / 8, 148ull * 8);
    act_out_kernel<<<(unsigned)blocks, 256, 0, stream>>>(C, rows, params + kMlpB2, params + kMlpW3,
                                                        params + kMlpB3, Y);
    return cudaGetLastError();
}

cudaError_t mlp_targets(const float* p7, uint64_t texels, float* Y, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    targets_kernel<<<blocks_for(texels, 128), 128, 0, stream>>>(p7, texels, Y);
    return cudaGetLastError();
}

cudaError_t mlp_finish(const float* Yn, uint64_t texels, const float* mean, const float* std, float* p7,
                       cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    finish_kernel<<<blocks_for(texels, 128), 128, 0, stream>>>(Yn, texels, mean, std, p7);
    return cudaGetLastError();
}

} // namespace svf
