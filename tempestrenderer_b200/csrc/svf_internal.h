// svf_internal.h - declarations shared by the host orchestration (svf_host*.cpp)
// and the CUDA translation units.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/svf.h"

namespace svf
{

// Per-texel LM settings (LevenbergMarquardtCurveFit, include/tempest/math/fitting.hh:457-678).
struct LmConfig
{
    uint32_t max_iter;
    double   mse_target;
    double   eps;          // BreakOnSmallStep
    float    fresnel;
    uint32_t restarts;     // continuations from a stop point with fresh damping
    uint32_t step_per_param;   // the small-step test per parameter (SVF_LSQ_STEP_PER_PARAMETER)
    uint32_t fixed_mask;       // parameters held at their initial values (bits of the parameter index)
    uint32_t zero_mask;        // parameters set to 0 before the fit (with fixed_mask: not fitted)
    uint32_t row_fit;          // slabs hold one view row (L samples): LSF_OPTION_FIT_TOP's fit
};

// A run of texels of one direction layout in an LM launch: texels
// [first, next segment's first) take their slabs from lum + (t - first) * stride.
constexpr int kLmMaxSegments = 16;
// The largest direction layout the library takes (light_count; L^2 pairs).
constexpr uint32_t kMaxLayout = 160;

struct LmSegment
{
    uint32_t     first;        // first texel of the segment (segments in increasing order, seg[0].first = 0)
    uint32_t     L;            // directions of the layout (L^2 pairs)
    uint64_t     stride;       // elements per slab; stride x element size % 16 == 0
    const void*  lum;          // [count][stride] slab elements (FP32 luminance, or FP16 RGB for the RGB fit), 16-byte aligned
    const float* geo;          // [3][L] direction table, SoA: x, y, z
    float        damping;      // initial damping relative to the reference's rule (0 counts as 1)
};

// Arguments of the persistent LM kernel.
struct LmArgs
{
    LmSegment    seg[kLmMaxSegments];
    uint32_t     n_seg;        // >= 1
    uint32_t     L;            // the largest layout of the segments
    uint64_t     lum_stride;   // the largest slab stride (floats): sizes the shared memory
    const float* init;         // [texels][7] ([texels][12] for the RGB fit)
    float*       out;          // [texels][7] ([texels][12] for the RGB fit)
    float*       rmse;         // [texels]
    svf_texel_stats* stats;    // [texels] or null
    const float* avg_chroma;   // [texels][3] or null (needed by the RGB maps)
    float* map_diffuse;        // [texels][3] or null
    float* map_specular;       // [texels][3] or null
    float* map_sigma;          // [texels][2] or null
    float* map_basis;          // [texels][4] or null
    uint32_t texels;           // texels of this launch: texel_base .. texel_base + texels - 1
    uint32_t texel_base;
    uint32_t all_up;           // every direction of every segment has z > 0
    uint32_t rgb;              // the 11-parameter RGB fit (svf_lm.cu RgbModel)
    LmConfig cfg;
    uint32_t* work_counter;    // zeroed before the launch
    uint32_t* error_flag;      // set non-zero by a bounded wait that expired
    // Fault injection for tests (the host sets it from the environment): the slab
    // copy of texel fault_skip_texel is not issued, so its wait runs out;
    // kLmNoFault for none.  wait_spins: the bound of every slab wait (0: default).
    uint32_t fault_skip_texel;
    uint32_t wait_spins;
};
constexpr uint32_t kLmNoFault = 0xffffffffu;

// LM kernel configuration (svf_lm.cu): CTA size (one control warp + pair
// workers) and the texel slots each CTA keeps in flight.
struct LmKernelChoice
{
    int threads;
    int slots;
    int pass;     // pair pass: 0 plain; 1 paired FP32 instructions; 2 J^T J on the tensor cores
                  // (1 and 2: luminance fit without a Fresnel factor)
};
constexpr int kLmCandidates = 12;
constexpr int kLmPlainCandidates = 7;   // the first candidates: plain pair passes
LmKernelChoice lm_default_choice(uint32_t L, uint64_t lum_stride, bool rgb = false);
int            lm_candidates(uint32_t L, LmKernelChoice* out, int max);
size_t         lm_smem_bytes(uint32_t L, uint64_t lum_stride, LmKernelChoice c, bool rgb = false);
int            lm_max_ctas_per_sm(uint32_t L, uint64_t lum_stride, LmKernelChoice c, bool rgb = false);
cudaError_t    launch_lm_fit(const LmArgs& args, LmKernelChoice c, int grid, cudaStream_t stream);

// svf_lsq_fit_batch_noalloc: repack, geometry and LM on `stream` with the
// library's static device scratch array; waits for the stream.  flags[0]: the
// kernel's error flag (a bounded wait expired); flags[1]: the OR of the texels'
// SVF_TEXEL_NONFINITE | SVF_TEXEL_TIMEOUT bits (0 when stats is NULL).
cudaError_t launch_lm_fit_noalloc(const float* lights_parabolic, uint32_t L, const float* lum, uint64_t lum_stride,
                                  uint32_t texels, const LmConfig& cfg, const float* init, float* out, float* rmse,
                                  svf_texel_stats* stats, cudaStream_t stream, uint32_t flags[2]);

// Luminance slice + average chromaticity (BTFParallelExtractLuminanceSlice,
// src/image/btf.cc:1078-1116) for texels [0, texels) of an RGB sample array.
// lum_hi/lum_lo (optional, both or neither): the BF16 split of the slice for the
// NDF GEMM, same row pitch (a multiple of 8), pair k at column hilo_pos[k] (the
// operator's column order), columns [N, lum_stride) zero.
// rgb16 (optional): the samples again as FP16 RGB slabs [texels][rgb_stride]
// for the RGB fit (rgb_stride >= 3 N, a multiple of 8).
// The learned guess's half-vector-bin features, computed by the luminance pass
// from the slab it holds in shared memory in bin order (X null: none): pair k
// at pos[k], so that bin b holds positions start[b] .. start[b + 1]; a bin's
// feature is the sum of its positions, in order, times bin_w[b]; then the
// luminance at the 32 single pairs' positions pair_pos; log, normalised with
// mean/rstd (mean null: raw).  X: [texels][kMlpInputs].
struct LumFeatures
{
    const uint16_t* pos = nullptr;
    const uint32_t* start = nullptr;
    const float* bin_w = nullptr;
    const uint16_t* pair_pos = nullptr;
    const float *mean = nullptr, *rstd = nullptr;
    float* X = nullptr;
};
// The luminance slabs [texels][lum_stride] of RGB samples [texels][N][3]; every
// other output is optional (null: not computed): the average chromaticity
// [texels][3], the BF16 hi/lo split of the slabs, the FP16 RGB slabs and the
// learned guess's features.
cudaError_t launch_luminance(const void* samples, uint32_t sample_type, uint64_t texels, uint32_t N,
                             float* lum, uint64_t lum_stride, float* avg_chroma, void* lum_hi, void* lum_lo,
                             const uint16_t* hilo_pos, cudaStream_t stream, void* rgb16 = nullptr,
                             uint64_t rgb_stride = 0,
                             const LumFeatures& features = LumFeatures{});

// dst[t][j] = src[t][pairs[j]] for j < n_pairs, 0 up to dst_stride.
cudaError_t launch_gather_pairs(const float* src, uint64_t src_stride, const uint32_t* pairs, uint32_t n_pairs,
                                uint64_t texels, float* dst, uint64_t dst_stride, cudaStream_t stream);

// The RGB fit's initial parameters {kd rgb, ks rgb, sx, sy, quaternion xyzw}
// from a luminance initial guess {sx, sy, ks, kd, euler} and the texel's
// average chromaticity (the colours SVBRDFFitPipeline::fit gives the maps,
// svbrdf-fitting-pipeline.cc:692-697).
cudaError_t launch_rgb_init(const float* init7, const float* avg_chroma, uint64_t texels, float* init12,
                            cudaStream_t stream);

// Repacks a caller's luminance array to the padded internal layout.
cudaError_t launch_repack(const float* src, uint64_t src_stride, uint64_t texels, uint32_t N,
                          float* dst, uint64_t dst_stride, cudaStream_t stream);

cudaError_t launch_synth(uint32_t seed, uint32_t mix, const float* lights_parabolic, uint32_t L, uint64_t first,
                         uint64_t count, uint32_t sample_type, float noise, void* samples, float* truth,
                         cudaStream_t stream);

// ---- default initial guess (svf_init.cu) ---------------------------------------

constexpr int kNdfRes = 64;               // NDFTextureResolution (svbrdf-fitting.hh:53)
constexpr int kNdfTexels = kNdfRes * kNdfRes;
constexpr int kNdfSamples = 4096;         // NDRReduceSphereSamples (svbrdf-fitting.hh:49)
constexpr int kPcaSide = 512;             // CommonSampleCount (svbrdf-fitting.hh:46)
constexpr int kPcaSamples = kPcaSide * kPcaSide;
constexpr int kDenomSamples = 256 * 256;  // svbrdf-fitting-pipeline.cc:403
constexpr int kProjSamples = 1024;        // ConvertSamples (svbrdf-fitting.hh:50)
constexpr int kTangentSteps = 512;        // EigenVectorPlaneSamples (svbrdf-fitting.hh:48)

// Device tables of one direction layout for the default initial guess.
struct InitLayout
{
    uint32_t L, N;
    uint32_t k_pad;            // N padded to a multiple of 8 (GEMM K)
    uint32_t ndf_rows;         // NDF texels inside the hemisphere (rows of the operator)
    uint32_t ndf_rows_pad;     // rows padded to a multiple of 256 (the GEMM's N tile)
    float*    ndf_op;          // [ndf_rows_pad][k_pad] NDF = op * lum (row-major, FP32)
    int32_t*  ndf_row_texel;   // [ndf_rows] NDF texel index of each operator row (rows in Morton order
                               // of their texel, so that a 256-row tile is a compact block of the NDF)
    // The GEMM runs over the operator's non-empty tiles only.  Its columns (the
    // luminance pairs) are taken in Morton order of the pair's half vector, so
    // that a 64-column K-block reaches few NDF rows; the luminance pass writes the
    // BF16 split in that order.
    uint16_t* col_pos;         // [N] position of pair k in the permuted order
    uint32_t* col_of;          // [N] pair at permuted position p
    uint32_t  packed_tiles;    // packed tiles (the non-empty 256 x 64 operator tiles; at least 1)
    uint32_t  nonempty_tiles;  // of them non-empty, and all tiles of the operator
    uint32_t  all_tiles;
    void*     tile_hi;         // [packed_tiles][256][64] BF16 hi/lo split of them
    void*     tile_lo;
    uint32_t* tile_kb;         // [packed_tiles] K-block of each, grouped by row tile
    uint32_t* tile_start;      // [ndf_rows_pad / 256 + 1] each row tile's range in them
    float*    denom_w;         // [4096] ndf_denom = denom_w . NDF
    // PCA search samples, grouped by the bilinear cell they fall in
    uint32_t  pca_cells;       // cells that hold samples
    int32_t*  pca_cell_id;     // [pca_cells] x0 + 64*y0 of the cell
    uint32_t* pca_cell_start;  // [pca_cells + 1] ranges into the sample arrays
    uint32_t* pca_index;       // [kPcaSamples] original sample order, cell-grouped
    float2*   pca_frac;        // [kPcaSamples] (fx1, fy1), cell-grouped
    float4*   pca_dir;         // [kPcaSamples] directions, in sample order
    float4*   proj_dir;        // [1024] SGGX projection sample directions
    float2*   proj_frac;       // [1024] bilinear fractions
    int32_t*  proj_cell;       // [1024] x0 + 64*y0
    float     rot_s, rot_c;    // tangent-plane rotation step
    float     pdf;             // 1/(2 pi)
    int32_t   axis_cell;       // bilinear set-up of the direction (0, 0, 1)
    float     axis_fx1, axis_fy1;
};

// Builds the NDF operator rows on the device from the mesh and sample tables.
struct MeshDevice
{
    const float*    lp;        // [L][2]
    const uint32_t* tri;       // [T][3]
    uint32_t        ntri;
    const uint32_t* edges;     // [E][3]
    const float*    eang;      // [E][2]
    uint32_t        nedge;
};
cudaError_t launch_ndf_operator(const InitLayout& lay, const MeshDevice& mesh, const float* ndf_dirs /* [4096][3] */,
                                const float* row_normals /* [rows][3] */, double ndf_scale, int32_t* light_tri,
                                float* light_bary, cudaStream_t stream);

// NDF rows C[T][ldc] = A x B^T on the tensor cores (svf_ndf_tc.cu) from BF16
// hi/lo splits of A (slabs, [T][lda]) and B (operator, [rows_pad][ldb]); k
// columns of each are used.
size_t      ndf_tc_smem_bytes();
cudaError_t launch_split_bf16(const float* x, uint64_t n, void* hi, void* lo, cudaStream_t stream);
// hi/lo[t][p] = BF16 split of x[t][col_of[p]] (p < N; 0 up to stride).
cudaError_t launch_split_bf16_permuted(const float* x, uint64_t rows, uint64_t stride, uint32_t N,
                                       const uint32_t* col_of, void* hi, void* lo, cudaStream_t stream);
// flags[n][kb]: the operator tile (row tile n, K-block kb of the permuted columns) is non-empty.
cudaError_t launch_ndf_tile_flags(const float* op, uint32_t k_pad, const uint32_t* col_of, uint32_t N,
                                  uint32_t rows_pad, uint32_t* flags, cudaStream_t stream);
// Packs the listed tiles (tile_n[j], tile_kb[j]) as BF16 hi/lo [packed_tiles][256][64].
cudaError_t launch_ndf_tile_pack(const float* op, uint32_t k_pad, const uint32_t* col_of, uint32_t N,
                                 const uint32_t* tile_n, const uint32_t* tile_kb, uint32_t packed_tiles, void* hi,
                                 void* lo, cudaStream_t stream);
cudaError_t launch_ndf_tc(const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda, const void* b_hi,
                          const void* b_lo, uint32_t rows_pad, uint64_t ldb, uint32_t k, float* C, uint32_t ldc,
                          uint32_t* error_flag, cudaStream_t stream);
// The GEMM over the packed operator tiles (tile_kb/tile_start non-null): row
// tile n multiplies only its K-blocks; b_hi/b_lo are the packed tiles.
cudaError_t launch_ndf_tc_tiles(const void* a_hi, const void* a_lo, uint64_t texels, uint64_t lda, const void* b_hi,
                                const void* b_lo, uint32_t rows_pad, uint64_t ldb, uint32_t k, float* C, uint32_t ldc,
                                uint32_t* error_flag, cudaStream_t stream, const uint32_t* tile_kb,
                                const uint32_t* tile_start, uint32_t packed_tiles);
// ndf_rows: [texels][ldr] operator-row NDF values.  init_info (optional):
// [texels][8] = ndf_denom, normal xyz, tangent xyz, pca value; ndf_out
// (optional): [texels][4096] NDF textures.
cudaError_t launch_init_finish(const InitLayout& lay, const float* ndf_rows, uint32_t ldr, uint64_t texels,
                               float* init_params, float* init_info, float* ndf_out, cudaStream_t stream);

// ---- learned initial guess (svf_mlp.cu) -----------------------------------------

constexpr int kMlpBins = 64;                   // half-vector bins (8 x 8 over the parabolic disk)
constexpr int kMlpPairs = 32;                  // single direction pairs per texel
constexpr int kMlpInputs = kMlpBins + kMlpPairs;
constexpr int kMlpHidden = 256;
constexpr int kMlpOutputs = 8;                 // log S (6 elements), log ks, log kd
// flat parameter vector: W1 [256][96], b1, W2 [256][256], b2, W3 [8][256], b3
constexpr size_t kMlpW1 = 0, kMlpB1 = kMlpW1 + (size_t)kMlpHidden * kMlpInputs;
constexpr size_t kMlpW2 = kMlpB1 + kMlpHidden, kMlpB2 = kMlpW2 + (size_t)kMlpHidden * kMlpHidden;
constexpr size_t kMlpW3 = kMlpB2 + kMlpHidden, kMlpB3 = kMlpW3 + (size_t)kMlpOutputs * kMlpHidden;
constexpr size_t kMlpParams = kMlpB3 + kMlpOutputs;

// C[M][N] = op(A) op(B) (+ bias[n]); mode 1: Z = C (if Z), C = gelu(C); mode 2:
// C *= gelu'(Zin).  FP32 (training).
cudaError_t mlp_gemm(bool ta, bool tb, int M, int N, int K, const float* A, int lda, const float* B, int ldb,
                     float* C, int ldc, const float* bias, int mode, float* Z, const float* Zin, cudaStream_t stream);
cudaError_t mlp_colsum(const float* X, int M, int N, double* sum, double* sumsq, cudaStream_t stream);
cudaError_t mlp_to_float(const double* x, int n, float scale, float* y, cudaStream_t stream);
cudaError_t mlp_normalize(float* X, int M, int N, const float* mean, const float* rstd, cudaStream_t stream);
cudaError_t mlp_mse_grad(const float* Y, const float* T, int M, int N, float* dY, double* loss, cudaStream_t stream);
cudaError_t mlp_adam(float* w, const float* g, float* m, float* v, size_t n, float lr, int step, bool sgd,
                     cudaStream_t stream);
cudaError_t mlp_gather_rows(const float* X, int nx, const float* Y, int ny, const uint32_t* idx, int rows, float* Xb,
                            float* Yb, cudaStream_t stream);
// features [texels][96] of luminance slabs [texels][stride] (normalised when mean
// != null): bins over order[start[b] .. start[b + 1]) scaled by bin_w[b], pairs
// features [texels][96] of RGB samples [texels][N][3]: 32 pairs x RGB
cudaError_t mlp_features_rgb(const void* samples, uint32_t sample_type, uint64_t texels, uint32_t N,
                             const uint32_t* pairs, const float* mean, const float* rstd, float* X, cudaStream_t stream);
// Inference weights of the hidden layers for the tensor cores: BF16 hi/lo of
// W1 | W2; kMlpTcWeights elements each.
constexpr size_t kMlpTcWeights = (size_t)kMlpHidden * kMlpInputs + (size_t)kMlpHidden * kMlpHidden;
cudaError_t mlp_pack_weights(const float* w, void* hi, void* lo, cudaStream_t stream);
// Inference with the hidden layers on the tcgen05 tensor cores (the BF16x3 GEMM
// of launch_ndf_tc) and the 8-output layer fused into the second layer's
// epilogue: X [rows][96] -> Y [rows][8]; C: FP32 scratch [rows][256]; act:
// BF16 scratch of 2 x [rows][256] (16-byte aligned); params: the FP32
// parameter vector (biases, W3).
cudaError_t mlp_forward_tc(const float* X, uint64_t rows, const void* w_hi, const void* w_lo, const float* params,
                           float* C, void* act, float* Y, uint32_t* error_flag, cudaStream_t stream);
cudaError_t mlp_targets(const float* p7, uint64_t texels, float* Y, cudaStream_t stream);
cudaError_t mlp_finish(const float* Yn, uint64_t texels, const float* mean, const float* std, float* p7,
                       cudaStream_t stream);

// ---- learned guess: fallback to the default guess (svf_kernels.cu) ------------------
cudaError_t launch_fallback_select(const float* lum, uint64_t stride, uint32_t N, const float* rmse, uint64_t n,
                                   float threshold, uint32_t* idx, uint32_t* count, cudaStream_t stream);
cudaError_t launch_gather_slabs(const float* lum, uint64_t stride, const float* avg, const uint32_t* idx, uint32_t m,
                                float* g_lum, float* g_avg, cudaStream_t stream);
cudaError_t launch_fallback_merge(const uint32_t* idx, uint32_t m, const float* g_out, const float* g_rmse,
                                  const svf_texel_stats* g_stats, const float* g_maps, const float* g_init, uint64_t n,
                                  float* out, float* rmse, svf_texel_stats* stats, float* maps, float* init,
                                  uint32_t* taken, cudaStream_t stream);

// ---- neighbourhood refit (svf_kernels.cu) --------------------------------------------
// cand [9n][7]: candidate k of texel c0 + i at row k*n + i (the 3x3 neighbour's
// parameters, the texel's own outside the image)
cudaError_t launch_refit_gather(const float* params, uint64_t c0, uint64_t n, uint32_t width, uint32_t height,
                                float* cand, cudaStream_t stream);
// sel_from (optional): 0..8 the winning neighbour, 9 the texel's own parameters
cudaError_t launch_refit_select(const float* params, const float* rmse, uint64_t c0, uint64_t n, uint32_t width,
                                uint32_t height, const float* cand_out, const float* cand_rmse, float* sel_params,
                                float* sel_rmse, uint32_t* sel_from, cudaStream_t stream);

// ---- factored BTF decode (svf_btf.cu) ----------------------------------------------

// Channel c: U_c row lv at u[c] + lv * u_row[c] elements, SxV_c row col at
// sxv[c] + col * sxv_row[c]; k[c] components; elements of data_size bytes.
struct BtfDecodeArgs
{
    const void* u[3];
    const void* sxv[3];
    uint32_t k[3];
    uint64_t u_row[3], sxv_row[3];
    uint32_t data_size, color_model, drr;
    uint32_t width, height, N;
    uint64_t first, count;     // texels [first, first + count), index y * width + x
    uint32_t out_type;         // SVF_SAMPLES_F32 / F16
    void* out;                 // device [count][N][3]
};
cudaError_t launch_btf_decode(const BtfDecodeArgs& a, cudaStream_t stream);

// ---- error of fitted maps against a BTF (svf_error.cu) -----------------------------

struct ErrorArgs
{
    const void* samples;       // device [rows * row_texels][N][3] decoded BTF rows
    uint32_t sample_type;
    uint32_t L, N;
    const float* geo;          // [3][L] directions
    uint64_t count;            // region texels in this launch: rows x region_w
    uint32_t region_w;
    uint64_t row_texels, x0;   // sample row of region texel (ry, rx): ry * row_texels + x0 + rx
    const float *diffuse, *specular, *sigma, *basis;   // device maps [count][3|3|sigma_channels|4]
    uint32_t sigma_channels;   // 2: (sx, sy); 3: (sx/sz, sy/sz)
    uint32_t method, color;    // SVF_ERROR_*; color: per-channel outputs
    float *rmse, *psnr;        // device [count] ([count][3] with color)
};
cudaError_t launch_error(const ErrorArgs& a, cudaStream_t stream);

struct RenderArgs
{
    uint32_t L;
    const float* geo;          // [3][L]
    uint64_t count;            // texels
    const float *diffuse, *specular, *sigma, *basis;   // device maps
    uint32_t sigma_channels;
    float fresnel;             // refractive index (1: no Fresnel term)
    uint32_t sample_type;
    void* out;                 // device [count][L^2][3]
};
cudaError_t launch_render(const RenderArgs& a, cudaStream_t stream);

// ---- the pseudo-volume multi-scattering BRDF (svf_ms.cu) -------------------------------

struct MsRenderArgs
{
    uint32_t L;
    const float* geo;          // [3][L]
    uint64_t count;            // texels
    const float *diffuse, *specular, *sigma, *basis;   // device maps
    uint32_t sigma_channels;
    uint32_t bounces, samples, seed;   // walk depth, walks per evaluation, LCG state
    uint32_t sample_type;
    void* out;                 // device [count][L^2][3]
};
cudaError_t launch_ms_render(const MsRenderArgs& a, cudaStream_t stream);

// The LM state of one texel of the multi-scattering fit (FP64, as the
// reference's LevenbergMarquardtCurveFit keeps it).
struct MsTexel
{
    double p[7], tmp[7], step[7], grad[7], hess[49];
    double damping, mult, last, trial, gain;
    uint32_t phase, iter, effective, jacobians, residuals;
};
enum : uint32_t
{
    kMsStep = 0,       // the next iteration computes a step
    kMsTrial = 1,      // its trial point awaits its residual
    kMsJacobian = 2,   // the accepted point awaits its Jacobian
    kMsDone = 3
};
enum : uint32_t
{
    kMsEvalCurrent = 0,    // residuals at p (the first evaluation)
    kMsEvalTrial = 1,      // residuals at the trial point
    kMsEvalJacobian = 2    // the 14 central-difference evaluations per pair at p
};
enum : uint32_t
{
    kMsStageStart = 0,     // initial damping from the first J^T J
    kMsStageStep = 1,      // damped solve, small-step and constraint tests
    kMsStageGain = 2,      // gain ratio, accept or reject
    kMsStageDamping = 3    // gradient test and damping update after a Jacobian
};
struct MsFitArgs
{
    uint32_t L;
    const float* geo;          // [3][L]
    uint32_t bounces;
    uint64_t texels;           // texels of the batch
    const float* lum;          // [texels][lum_stride] luminance slices
    uint64_t lum_stride;
    MsTexel* st;               // [texels]
    float* res;                // [texels][L^2] residuals
    float* fev;                // [texels][L^2][14] negated perturbed evaluations
    uint32_t* list;            // texels of the next evaluation
    uint32_t* counts;          // [0] trial list length, [1] Jacobian list length, [2] texels not done
    uint32_t max_iter;
    double mse_target, eps;    // LevenbergMarquardtCurveFit mean_sq_error, BreakOnSmallStep
};
cudaError_t launch_ms_setup(const MsFitArgs& a, const float* init, cudaStream_t stream);
// Evaluations of the listed texels and their reductions: `count` of them, or,
// with dcount (device) non-null, *dcount of at most `count`.
cudaError_t launch_ms_eval(const MsFitArgs& a, uint32_t mode, uint32_t count, const uint32_t* dcount,
                           cudaStream_t stream);
cudaError_t launch_ms_control(const MsFitArgs& a, uint32_t stage, cudaStream_t stream);
cudaError_t launch_ms_finish(const MsFitArgs& a, const float* init, float* out, float* rmse, svf_texel_stats* stats,
                             cudaStream_t stream);

} // namespace svf
