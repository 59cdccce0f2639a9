// svf_ndf_tc.cu - the NDF step of the default initial guess on the tcgen05 tensor
// cores: NDF rows = lum x Op^T for all texels (NDFRecord,
// tools/svbrdf-fitting/svbrdf-fitting-pipeline.cc:110-133, as a fixed linear map
// of the luminance slice; see svf_init.cu).
//
// FP32 accuracy from BF16 tensor cores: both operands are split x = hi + lo with
// hi = bf16(x), lo = bf16(x - hi) (16 significant bits together) and
// C = A_hi B_hi^T + A_hi B_lo^T + A_lo B_hi^T, accumulated in FP32 in tensor
// memory (the dropped lo*lo term is below 2^-16 relative).
//
// One CTA computes a 128 x 256 tile of C (texels x operator rows) with 128
// threads:
//   warp 0, one lane : TMA producer - K-blocks of 64 elements of A_hi, A_lo (128
//                      rows) and B_hi, B_lo (256 rows) into a 2-stage ring,
//                      128-byte swizzle, completion on mbarriers;
//   warp 1, one lane : MMA issuer - per K-block 4 K-steps x 3 products of
//                      tcgen05.mma.cta_group::1.kind::f16 (M 128, N 256, K 16),
//                      tcgen05.commit frees the stage and finally signals the
//                      accumulator;
//   all 4 warps      : epilogue - tcgen05.ld of their 32 TMEM lanes (texels),
//                      16-byte stores of the FP32 rows.
// Every mbarrier wait is bounded; on expiry the CTA flags the error, lets its
// copies and MMAs drain (again bounded), frees its tensor memory and returns.
// Columns past k and rows past the operand extents are zero-filled by the TMA
// unit, so neither operand needs padding values.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "svf_internal.h"

namespace svf
{

namespace
{

constexpr int kTileM = 128, kTileN = 256, kBlockK = 64, kStages = 2;
constexpr uint32_t kTileABytes = kTileM * kBlockK * 2;   // 16 KB per operand half
constexpr uint32_t kTileBBytes = kTileN * kBlockK * 2;   // 32 KB
constexpr uint32_t kStageBytes = 2 * kTileABytes + 2 * kTileBBytes;
constexpr uint32_t kTmemCols = kTileN;                    // FP32 accumulator columns
constexpr uint32_t kSpin = 1u << 24;                      // bound of every wait

__device__ __forceinline__ uint32_t saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t n)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(b)), "r"(n) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity)
{
    uint32_t done;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(saddr(b)), "r"(parity)
                 : "memory");
    return done != 0;
}

// Bounded wait; false when it expired or another role already gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort)
{
    for(uint32_t i = 0; i < kSpin; ++i)
    {
        if(mbar_try(b, parity))
            return true;
        if((i & 1023u) == 1023u && *abort)
            return false;
    }
    return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(saddr(b)), "r"(bytes) : "memory");
}

// 2D tiled TMA load; x (the K coordinate, innermost) is a multiple of 64 elements.
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int32_t x, int32_t y, uint64_t* bar)
{
    asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
                 ::"r"(saddr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(saddr(bar))
                 : "memory");
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B
// apart (version 1, layout type 2).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr)
{
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}

// Instruction descriptor: D FP32, A and B BF16, both K-major, N = 256, M = 128.
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kTileN >> 3) << 17) |
                            ((uint32_t)(kTileM >> 4) << 24);

__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
                 ::"r"(tmem_d), "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate)
                 : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* r)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                 "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                   "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                   "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                   "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr)
                 : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

struct TcMaps
{
    CUtensorMap a_hi, a_lo, b_hi, b_lo;
};

// Dense: every CTA runs the ktiles K-blocks, B tiles at (K-block, n0).  Tile
// list (tile_kb non-null): the CTA of row tile n runs the K-blocks
// tile_kb[tile_start[n] .. tile_start[n + 1]), and B is the packed operator
// whose tile j (256 rows x 64 columns) sits at row 256 j.
__global__ void __launch_bounds__(128, 1) ndf_tc_kernel(const __grid_constant__ TcMaps maps, uint32_t ktiles,
                                                        uint64_t M, uint32_t ldc, float* __restrict__ C,
                                                        uint32_t* error_flag, const uint32_t* __restrict__ tile_kb,
                                                        const uint32_t* __restrict__ tile_start)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment of every operand tile (the swizzle atom)
    unsigned char* smem = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) &
                                                           ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages], done, drain;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    __shared__ volatile uint32_t issued;   // K-blocks whose copies were issued

    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
    const uint64_t m0 = (uint64_t)blockIdx.y * kTileM;
    const uint32_t n0 = blockIdx.x * kTileN;
    const uint32_t j0 = tile_kb ? tile_start[blockIdx.x] : 0u;
    const uint32_t nkb = tile_kb ? tile_start[blockIdx.x + 1] - j0 : ktiles;

    if(threadIdx.x == 0)
    {
        for(int s = 0; s < kStages; ++s)
        {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&done, 1);
        mbar_init(&drain, 1);
        abort_flag = 0;
        issued = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.a_hi)) : "memory");
        asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&maps.b_hi)) : "memory");
    }
    if(warp == 0)
    {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(&tmem_base)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    auto stage_ptr = [&](int s, int which) -> unsigned char* {
        // which: 0 A_hi, 1 A_lo, 2 B_hi, 3 B_lo
        unsigned char* base = smem + (size_t)s * kStageBytes;
        return which < 2 ? base + which * kTileABytes : base + 2 * kTileABytes + (which - 2) * kTileBBytes;
    };

    if(warp == 0 && lane == 0)
    {
        // TMA producer
        for(uint32_t kb = 0; kb < nkb; ++kb)
        {
            const int s = kb % kStages;
            if(kb >= (uint32_t)kStages && !mbar_wait(&empty[s], ((kb / kStages) - 1) & 1u, &abort_flag))
            {
                abort_flag = 1;
                break;
            }
            mbar_expect_tx(&full[s], kStageBytes);
            // A: the K-block's columns; B: the dense operator at (K-block, n0) or packed tile j
            const int32_t kx = (int32_t)((tile_kb ? tile_kb[j0 + kb] : kb) * kBlockK);
            const int32_t bx = tile_kb ? 0 : kx;
            const int32_t by = tile_kb ? (int32_t)((j0 + kb) * kTileN) : (int32_t)n0;
            tma_load_2d(stage_ptr(s, 0), &maps.a_hi, kx, (int32_t)m0, &full[s]);
            tma_load_2d(stage_ptr(s, 1), &maps.a_lo, kx, (int32_t)m0, &full[s]);
            tma_load_2d(stage_ptr(s, 2), &maps.b_hi, bx, by, &full[s]);
            tma_load_2d(stage_ptr(s, 3), &maps.b_lo, bx, by, &full[s]);
            issued = kb + 1;
        }
    }
    else if(warp == 1 && lane == 0)
    {
        // MMA issuer
        uint32_t kb = 0;
        for(; kb < nkb; ++kb)
        {
            const int s = kb % kStages;
            if(!mbar_wait(&full[s], (kb / kStages) & 1u, &abort_flag))
            {
                abort_flag = 1;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t a_hi = saddr(stage_ptr(s, 0)), a_lo = saddr(stage_ptr(s, 1));
            const uint32_t b_hi = saddr(stage_ptr(s, 2)), b_lo = saddr(stage_ptr(s, 3));
#pragma unroll
            for(int k = 0; k < kBlockK / 16; ++k)
            {
                const uint32_t off = k * 32;   // 16 BF16 elements along K
                const uint32_t acc0 = (kb > 0 || k > 0) ? 1u : 0u;
                umma(tmem, smem_desc(a_hi + off), smem_desc(b_hi + off), acc0);
                umma(tmem, smem_desc(a_hi + off), smem_desc(b_lo + off), 1u);
                umma(tmem, smem_desc(a_lo + off), smem_desc(b_hi + off), 1u);
            }
            umma_commit(&empty[s]);
        }
        if(kb == nkb)
            umma_commit(&done);
    }
    __syncwarp();

    // epilogue: every warp reads its 32 TMEM lanes (texel rows)
    const bool ok = mbar_wait(&done, 0, &abort_flag) && !abort_flag;
    const bool all_ok = __syncthreads_and(ok ? 1 : 0) != 0;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if(all_ok)
    {
        const uint64_t m = m0 + warp * 32 + lane;
        for(int c = 0; c < kTileN; c += 32)
        {
            uint32_t r[32];
            if(nkb)
                tmem_ld32(tmem + ((warp * 32u) << 16) + (uint32_t)c, r);
            else
#pragma unroll
                for(int q = 0; q < 32; ++q)
                    r[q] = 0u;   // a row tile without K-blocks: its rows are 0
            if(m < M)
            {
                float4* dst = reinterpret_cast<float4*>(C + m * ldc + n0 + c);
#pragma unroll
                for(int q = 0; q < 8; ++q)
                    dst[q] = make_float4(__uint_as_float(r[4 * q]), __uint_as_float(r[4 * q + 1]),
                                         __uint_as_float(r[4 * q + 2]), __uint_as_float(r[4 * q + 3]));
            }
        }
    }
    else
    {
        if(threadIdx.x == 0)
            atomicOr(error_flag, 1u);
        // let issued copies and MMAs land before the shared memory and the tensor
        // memory are released (bounded)
        if(warp == 0 && lane == 0)
        {
            // stage s was reissued only after its previous phase completed, so the
            // parity of the last issued K-block of each stage is exact
            const uint32_t n = issued;
            for(uint32_t kb = n >= (uint32_t)kStages ? n - kStages : 0; kb < n; ++kb)
                for(uint32_t i = 0; i < kSpin && !mbar_try(&full[kb % kStages], (kb / kStages) & 1u); ++i)
                {
                }
        }
        else if(warp == 1 && lane == 0)
        {
            // a commit tracks every MMA this thread issued before it
            umma_commit(&drain);
            for(uint32_t i = 0; i < kSpin && !mbar_try(&drain, 0); ++i)
            {
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if(warp == 0)
    {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols) : "memory");
    }
}

// x -> (bf16(x), bf16(x - bf16(x))) for an [rows][cols] FP32 array into two
// [rows][cols] BF16 arrays.
__global__ void split_bf16_kernel(const float* __restrict__ x, uint64_t n, __nv_bfloat16* __restrict__ hi,
                                  __nv_bfloat16* __restrict__ lo)
{
    for(uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    {
        const float v = x[i];
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[i] = h;
        lo[i] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                              const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                              CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn()
{
    static EncodeFn fn = nullptr;
    if(!fn)
    {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
           q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    }
    return fn;
}

// [rows][cols] BF16, row pitch `pitch` elements, box = 64 columns x box_rows.
bool make_map(CUtensorMap* m, const void* base, uint64_t rows, uint64_t cols, uint64_t pitch, uint32_t box_rows)
{
    EncodeFn enc = encode_fn();
    if(!enc)
        return false;
    const cuuint64_t dims[2] = { cols, rows };
    const cuuint64_t strides[1] = { pitch * 2 };
    const cuuint32_t box[2] = { (cuuint32_t)kBlockK, box_rows };
    const cuuint32_t estr[2] = { 1, 1 };
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

} // namespace

size_t ndf_tc_smem_bytes() { return (size_t)kStages * kStageBytes + 1024; }

cudaError_t launch_split_bf16(const float* x, uint64_t n, void* hi, void* lo, cudaStream_t stream)
{
    if(n == 0)
        return cudaSuccess;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148ull * 32);
    split_bf16_kernel<<<(unsigned)blocks, 256, 0, stream>>>(x, n, static_cast<__nv_bfloat16*>(hi),
                                                             static_cast<__nv_bfloat16*>(lo));
    return cudaGetLastError();
}

cudaError_t launch_ndf_tc(const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda, const void* b_hi,
                          const void* b_lo, uint32_t rows_pad, uint64_t ldb, uint32_t k, float* C, uint32_t ldc,
                          uint32_t* error_flag, cudaStream_t stream)
{
    return launch_ndf_tc_tiles(a_hi, a_lo, texels, lda, b_hi, b_lo, rows_pad, ldb, k, C, ldc, error_flag, stream,
                               nullptr, nullptr, 0);
}

cudaError_t launch_ndf_tc_tiles(const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda, const void* b_hi,
                                const void* b_lo, uint32_t rows_pad, uint64_t ldb, uint32_t k, float* C, uint32_t ldc,
                                uint32_t* error_flag, cudaStream_t stream, const uint32_t* tile_kb,
                                const uint32_t* tile_start, uint32_t packed_tiles)
{
    if(texels == 0)
        return cudaSuccess;
    // TMA: 16-byte aligned bases and row pitches; 16-byte output rows
    const auto misaligned = [](const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) != 0; };
    if(rows_pad % kTileN != 0 || k == 0 || lda % 8 != 0 || ldb % 8 != 0 || lda < k || ldb < k || ldc % 4 != 0 ||
       ldc < rows_pad || texels > 65535ull * kTileM || misaligned(a_hi) || misaligned(a_lo) || misaligned(b_hi) ||
       misaligned(b_lo) || misaligned(C))
        return cudaErrorInvalidValue;
    if((tile_kb == nullptr) != (tile_start == nullptr) || (tile_kb && packed_tiles == 0))
        return cudaErrorInvalidValue;
    TcMaps maps;
    // B: the dense operator [rows_pad][k], or the packed tiles [packed_tiles * 256][64]
    const uint64_t b_rows = tile_kb ? (uint64_t)packed_tiles * kTileN : rows_pad;
    const uint64_t b_cols = tile_kb ? (uint64_t)kBlockK : k, b_ld = tile_kb ? (uint64_t)kBlockK : ldb;
    if(!make_map(&maps.a_hi, a_hi, texels, k, lda, kTileM) || !make_map(&maps.a_lo, a_lo, texels, k, lda, kTileM) ||
       !make_map(&maps.b_hi, b_hi, b_rows, b_cols, b_ld, kTileN) ||
       !make_map(&maps.b_lo, b_lo, b_rows, b_cols, b_ld, kTileN))
        return cudaErrorInvalidValue;
    const size_t smem = ndf_tc_smem_bytes();
    cudaError_t e = cudaFuncSetAttribute(ndf_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(e != cudaSuccess)
        return e;
    const uint32_t ktiles = (k + kBlockK - 1) / kBlockK;
    dim3 grid(rows_pad / kTileN, (unsigned)((texels + kTileM - 1) / kTileM));
    ndf_tc_kernel<<<grid, 128, smem, stream>>>(maps, ktiles, texels, ldc, C, error_flag, tile_kb, tile_start);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// the NDF operator's non-empty tiles, packed
// ---------------------------------------------------------------------------

namespace
{

// flags[n * ktiles + kb] = 1 when the operator tile of row tile n and K-block kb
// (columns in the permuted order col_of) holds a non-zero.  One thread a row.
__global__ void __launch_bounds__(kTileN) tile_flags_kernel(const float* __restrict__ op, uint32_t k_pad,
                                                             const uint32_t* __restrict__ col_of, uint32_t N,
                                                             uint32_t ktiles, uint32_t* __restrict__ flags)
{
    const uint32_t kb = blockIdx.x, n = blockIdx.y;
    const float* row = op + (uint64_t)(n * kTileN + threadIdx.x) * k_pad;
    int any = 0;
    for(uint32_t c = 0; c < (uint32_t)kBlockK; ++c)
    {
        const uint32_t p = kb * kBlockK + c;
        if(p < N && row[col_of[p]] != 0.0f)
            any = 1;
    }
    any = __syncthreads_or(any);
    if(threadIdx.x == 0)
        flags[n * ktiles + kb] = any ? 1u : 0u;
}

// Packed tile j (row tile tile_n[j], K-block tile_kb[j]) as BF16 hi/lo
// [256][64], columns in the permuted order (past N: 0).  One thread a row.
__global__ void __launch_bounds__(kTileN) tile_pack_kernel(const float* __restrict__ op, uint32_t k_pad,
                                                            const uint32_t* __restrict__ col_of, uint32_t N,
                                                            const uint32_t* __restrict__ tile_n,
                                                            const uint32_t* __restrict__ tile_kb,
                                                            __nv_bfloat16* __restrict__ hi, __nv_bfloat16* __restrict__ lo)
{
    const uint32_t j = blockIdx.x;
    const float* row = op + (uint64_t)(tile_n[j] * kTileN + threadIdx.x) * k_pad;
    const uint64_t o = ((uint64_t)j * kTileN + threadIdx.x) * kBlockK;
    for(uint32_t c = 0; c < (uint32_t)kBlockK; ++c)
    {
        const uint32_t p = tile_kb[j] * kBlockK + c;
        const float v = p < N ? row[col_of[p]] : 0.0f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[o + c] = h;
        lo[o + c] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

// hi/lo[t][p] = split of x[t][col_of[p]] for p < N, 0 for N <= p < stride.
__global__ void split_bf16_permuted_kernel(const float* __restrict__ x, uint64_t rows, uint64_t stride, uint32_t N,
                                           const uint32_t* __restrict__ col_of, __nv_bfloat16* __restrict__ hi,
                                           __nv_bfloat16* __restrict__ lo)
{
    const uint64_t t = blockIdx.x;
    for(uint32_t p = threadIdx.x; p < stride; p += blockDim.x)
    {
        const float v = p < N ? x[t * stride + col_of[p]] : 0.0f;
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[t * stride + p] = h;
        lo[t * stride + p] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
}

} // namespace

cudaError_t launch_ndf_tile_flags(const float* op, uint32_t k_pad, const uint32_t* col_of, uint32_t N,
                                  uint32_t rows_pad, uint32_t* flags, cudaStream_t stream)
{
    if(rows_pad % kTileN != 0 || N == 0)
        return cudaErrorInvalidValue;
    const uint32_t ktiles = (N + kBlockK - 1) / kBlockK;
    tile_flags_kernel<<<dim3(ktiles, rows_pad / kTileN), kTileN, 0, stream>>>(op, k_pad, col_of, N, ktiles, flags);
    return cudaGetLastError();
}

cudaError_t launch_ndf_tile_pack(const float* op, uint32_t k_pad, const uint32_t* col_of, uint32_t N,
                                 const uint32_t* tile_n, const uint32_t* tile_kb, uint32_t packed_tiles, void* hi,
                                 void* lo, cudaStream_t stream)
{
    if(packed_tiles == 0)
        return cudaSuccess;
    tile_pack_kernel<<<packed_tiles, kTileN, 0, stream>>>(op, k_pad, col_of, N, tile_n, tile_kb,
                                                         static_cast<__nv_bfloat16*>(hi), static_cast<__nv_bfloat16*>(lo));
    return cudaGetLastError();
}

cudaError_t launch_split_bf16_permuted(const float* x, uint64_t rows, uint64_t stride, uint32_t N,
                                       const uint32_t* col_of, void* hi, void* lo, cudaStream_t stream)
{
    if(rows == 0)
        return cudaSuccess;
    if(rows > 0x7fffffffull || stride < N)
        return cudaErrorInvalidValue;
    split_bf16_permuted_kernel<<<(unsigned)rows, 256, 0, stream>>>(x, rows, stride, N, col_of,
                                                                  static_cast<__nv_bfloat16*>(hi),
                                                                  static_cast<__nv_bfloat16*>(lo));
    return cudaGetLastError();
}

} // namespace svf
