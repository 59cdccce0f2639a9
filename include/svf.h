/*
 * svf.h - C ABI of the B200 SVBRDF fitter (libsvf.so).
 *
 * Fits, texel by texel, a Lambert + anisotropic SGGX surface BRDF to a BTF with
 * Levenberg-Marquardt, on one NVIDIA B200 (sm_100a).  This is the drop-in for
 * the fitting path of TempestRenderer's svbrdffit tool:
 *
 *   svf_lsq_fit_sggx  replaces LeastSquaresFitSGGX
 *                     (tools/svbrdf-fitting/svbrdf-fitting.hh:126-127,
 *                      defined in svbrdf-lsq-fitting-setup.cc:234-431), and its
 *                     CUDA variant LeastSquaresFitSGGXCuda
 *                     (svbrdf-lsq-fitting-internal.hh:225-227).
 *   svf_lsq_fit_batch the same fit for many texels in one launch.
 *   svf_fit_texels    replaces the svbrdffit texel loop: PusherThread::execute
 *                     (svbrdf-fitting.cc:86-121) running SVBRDFFitPipeline::cache
 *                     and ::fit (svbrdf-fitting-pipeline.cc:240-733) on every
 *                     texel, i.e. luminance slice, default initial guess, LM and
 *                     the output maps (svbrdf-fitting.cc:713-735).
 *   svf_fit_btfs      the same loop over a batch of BTFs of uneven sizes and
 *                     layouts, sharing the persistent LM launches.
 *
 * Conventions (as in the reference):
 *   - L directions serve as both light and view directions; they are given in
 *     parabolic coordinates (BTF::LightsParabolic, btf.hh:114).
 *   - A direction pair is lv = view * L + light (light fastest).
 *   - The 7 fitted parameters are, in order, {sigma_x, sigma_y, specular,
 *     diffuse, euler_x, euler_y, euler_z} (OptimizationParameters,
 *     svbrdf-fitting.hh:55-65).
 *   - Buffers are caller-owned.  Every pointer argument may point to host
 *     memory or to device memory of the context's device; the library detects
 *     which.  Host buffers are staged through pinned memory in chunks.  A
 *     sample or output buffer in device memory of another GPU is rejected with
 *     SVF_EINVAL before anything is launched.
 *
 * Errors are returned as svf_status codes; no exception crosses the ABI.
 * svf_last_error() gives a message for the calling thread's last failure.
 * A context may be used by one host thread at a time.
 */
#ifndef SVF_H
#define SVF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SVF_ABI_VERSION 4u

typedef enum svf_status
{
    SVF_OK = 0,
    SVF_EINVAL = 1,     /* an argument is out of range or inconsistent */
    SVF_ENOMEM = 2,     /* device or pinned host allocation failed */
    SVF_ECUDA = 3,      /* a CUDA call failed; see svf_last_error() */
    SVF_ETIMEOUT = 4,   /* a bounded device wait expired (no texel result is trusted) */
    SVF_EPARTIAL = 5,   /* finished, but some texels carry a non-zero status */
    SVF_ENODEV = 6      /* no usable sm_100 device */
} svf_status;

/* per-texel status bits (svf_texel_stats::status) */
#define SVF_TEXEL_NONFINITE  1u  /* NaN/Inf in the data or the fit; params are the initial guess */
#define SVF_TEXEL_MAX_ITER   2u  /* stopped at max_iterations */
#define SVF_TEXEL_TIMEOUT    4u  /* the texel's samples did not arrive (bounded wait expired) */

/* LeastSquaresFitOptions (svbrdf-fitting.hh:100-107) for the supported path */
#define SVF_LSQ_DIFFUSE      (1u << 1)   /* LSF_OPTON_DIFFUSE: fit the Lambert term (7 parameters);
                                            without it the specular-only fit of svbrdffit's default
                                            (6 parameters {sx, sy, ks, euler}, diffuse held at 0;
                                            svbrdf-lsq-fitting-setup.cc:248-262) */
#define SVF_LSQ_DISABLE_DIRECTION_FITTING (1u << 2)   /* LSF_OPTION_DISABLE_DIRECTION_FITTING: the Euler
                                            angles are held at their initial values
                                            (svbrdf-lsq-fitting-setup.cc:265-268) */
#define SVF_LSQ_FIT_TOP      (1u << 4)   /* LSF_OPTION_FIT_TOP (svf_lsq_fit_sggx / svf_lsq_fit_batch only):
                                            fit the L samples of the top-most view (the direction nearest
                                            the pole), modelled as seen from direction 0 as the
                                            reference's evaluator sees them; RMSE over all L x L pairs at
                                            Fresnel 1 (svbrdf-lsq-fitting-setup.cc:289-313,403-421) */
/* The RGB fit (no counterpart in the reference, which fits the luminance and
 * colours the maps with the average chromaticity): 11 parameters per texel,
 * {kd rgb, ks rgb, sx, sy} plus the orientation, fitted to the three channels
 * with the same LM; the orientation is a quaternion moved by local rotations.
 * Samples are staged as FP16 for it.  svf_fit_texels / svf_fit_btfs only; its
 * parameters (params, init maps, SVF_INIT_GIVEN) are 12 floats per texel,
 * {kd rgb, ks rgb, sx, sy, quaternion xyzw}; the diffuse / specular maps are
 * the fitted albedos and rmse is over the three channels. */
#define SVF_LSQ_RGB          (1u << 8)
/* The small-step stopping test per parameter (no counterpart in the reference):
 * LM stops when every step entry is small against its own parameter,
 * |d_i| <= e (|p_i| + e) for sigma, specular and diffuse and |d_i| <= e (1 + e)
 * for the angles (e = break_on_small_step), instead of the reference's test on
 * the whole vector, |d| <= e (|p + e| + e) (fitting.hh:583-588).  The whole-vector
 * test is dominated by the largest entries (the Euler angles, up to pi), so it
 * stops while a narrow lobe's sigma (0.01 - 0.05) may still move by a tenth of
 * itself, where the residual is steep.  Set by svf_lsq_options_default; clear
 * it for the reference's test. */
#define SVF_LSQ_STEP_PER_PARAMETER (1u << 9)
/* The multi-scattering model (LeastSquaresFitOptions::MultiScatteringBounceCount
 * != ~0u, svbrdffit -m; svf_lsq_fit_sggx / svf_lsq_fit_batch, with
 * SVF_LSQ_DIFFUSE and none of the other options): the fit's BRDF is the
 * pseudo-volume SGGXMicroFlakePseudoVolumeBRDF (ggx-models-impl.hh:621-758; 256
 * random walks of at most multi_scattering_bounces events per evaluation, the
 * evaluator's LCG seed 0; Fresnel is not part of it), fitted by the reference's
 * LevenbergMarquardtCurveFit as written (fitting.hh:457-678: the central-
 * difference Jacobian of fitting.hh:883-908, the whole-vector small-step test,
 * no restarts); the RMSE is over all pairs.  Each evaluation runs its walks in
 * order, as their random numbers follow one another: a fit costs about
 * 15 L^2 x 256 x bounces walk steps per iteration. */
#define SVF_LSQ_MULTI_SCATTERING (1u << 10)

typedef struct svf_lsq_options
{
    uint32_t max_iterations;      /* CurveFitSteps (svbrdf-fitting.hh:51): 1024 */
    float    fresnel;             /* refractive index of the Fresnel term; 1 = no Fresnel */
    uint32_t flags;               /* must contain SVF_LSQ_DIFFUSE; default also SVF_LSQ_STEP_PER_PARAMETER */
    double   mse_target;          /* LevenbergMarquardtCurveFit mean_sq_error: 1e-6 */
    double   break_on_small_step; /* LevenbergMarquardtSettings::BreakOnSmallStep: 1e-3 */
    uint32_t restarts;            /* times LM continues, with fresh damping, from the point where
                                     the reference's stopping rules end it; 0 = the reference's
                                     single run.  Default 1. */
    uint32_t downsample_light_view; /* LeastSquaresFitOptions::DownSampleLightView (svbrdffit -S):
                                     when 2 <= n < L, svf_lsq_fit_sggx / svf_lsq_fit_batch fit the
                                     n x n pairs of the n directions svf_downsample_light_view
                                     picks, and report the RMSE over all L x L pairs at Fresnel 1
                                     (svbrdf-lsq-fitting-setup.cc:314-330,403-421).  0 = off
                                     (the default); the texel-loop entry points take 0 only. */
    uint32_t multi_scattering_bounces; /* MultiScatteringBounceCount with SVF_LSQ_MULTI_SCATTERING:
                                     the walk depth (0 = the pseudo volume's single-scattering
                                     term only).  Default 2. */
} svf_lsq_options;

typedef struct svf_texel_stats
{
    uint32_t iterations;   /* FitStatistics::IterationCount */
    uint32_t effective;    /* FitStatistics::EffectiveIterationCount (accepted steps) */
    uint32_t jacobians;    /* Jacobian + normal-equation builds */
    uint32_t residuals;    /* residual-only evaluations (trial steps) */
    uint32_t status;       /* SVF_TEXEL_* bits */
} svf_texel_stats;

typedef struct svf_ctx svf_ctx;

/* Library and error reporting -------------------------------------------------- */
uint32_t    svf_abi_version(void);
const char* svf_status_string(svf_status status);
const char* svf_last_error(void);

/* Fills the reference's defaults: 1024 iterations, Fresnel 1 (svbrdffit -n 1),
 * SVF_LSQ_DIFFUSE, MSE target 1e-6, small-step break 1e-3
 * (svbrdf-lsq-fitting-setup.cc:272-273,357-364). */
void svf_lsq_options_default(svf_lsq_options* options);

/* Contexts ------------------------------------------------------------------- */
/* Opens a context on CUDA device `device`; it owns streams, device workspaces
 * and the per-direction-layout tables.  Fails with SVF_ENODEV unless the device
 * is compute capability 10.x. */
svf_status svf_create(int device, svf_ctx** out_ctx);
void       svf_destroy(svf_ctx* ctx);

/* Direction layouts ------------------------------------------------------------ */
/* The interpolation mesh the default initial guess samples the luminance slice
 * with (BTF::LightIndices and BTF::Edges, built by LoadBTF, btf.cc:531-625).
 * Pass the BTF's own mesh to reproduce the reference exactly; or leave
 * `triangles` NULL and the library triangulates the directions itself
 * (Delaunay, then the boundary edges as LoadBTF builds them). */
typedef struct svf_layout_desc
{
    const float*    lights_parabolic;  /* [L][2] */
    uint32_t        light_count;       /* L, 3..160 */
    const uint32_t* triangles;         /* [triangle_count][3] or NULL */
    uint32_t        triangle_count;
    const uint32_t* edges;             /* [edge_count][3]: Index0, Index1, Triangle; or NULL */
    const float*    edge_angles;       /* [edge_count][2]: Angle0, Angle1 */
    uint32_t        edge_count;
} svf_layout_desc;

/* Writes the 81-direction ring layout (theta rings 0/15/30/45/60/75 degrees
 * holding 1/6/12/18/20/24 phi-uniform directions) in parabolic coordinates as
 * LoadBTF derives them from (theta, phi).  Returns the direction count (81). */
uint32_t svf_directions_ring81(float* lights_parabolic /* [81][2] */);

/* Writes `count` directions of a Fibonacci hemisphere lattice (z > 0) in
 * parabolic coordinates.  Returns count. */
uint32_t svf_directions_fibonacci(uint32_t count, float* lights_parabolic);

/* Computes a Delaunay mesh of the directions and the boundary edges in the
 * reference's format.  Returns the triangle count, or 0 on failure.  Sizes:
 * triangles [2L][3], edges [L][3], edge_angles [L][2] are always enough. */
uint32_t svf_layout_triangulate(const float* lights_parabolic, uint32_t light_count,
                                uint32_t* triangles, uint32_t* edges, float* edge_angles,
                                uint32_t* edge_count);

/* DownsampleLightView's choice of directions (svbrdf-lsq-fitting-setup.cc:129-163):
 * writes the n (2 <= n < L) kept direction indices, one drawn pseudo-randomly
 * per stride of (L - 1)/(n - 1) with the reference's seeded hash, to idx[n].
 * Returns n, or 0 for sizes out of range. */
uint32_t svf_downsample_light_view(uint32_t light_count, uint32_t n, uint32_t* idx);

/* LeastSquaresFitSGGX ------------------------------------------------------------ */
/* One texel, synchronous: fits `init` to the luminance slice `lum` ([L*L],
 * lv-indexed) and writes the fitted parameters and the RMSE
 * (sqrt of the final mean squared residual, as the reference reports it). */
svf_status svf_lsq_fit_sggx(svf_ctx* ctx, const float* lights_parabolic, uint32_t light_count,
                            const float* lum, const svf_lsq_options* options,
                            const float init[7], float out[7], float* rmse,
                            svf_texel_stats* stats /* may be NULL */);

/* Many texels in one persistent launch.  lum: [texel_count][lum_stride] floats
 * (lum_stride >= L*L); init/out: [texel_count][7]; rmse: [texel_count];
 * stats: [texel_count] or NULL. */
svf_status svf_lsq_fit_batch(svf_ctx* ctx, const float* lights_parabolic, uint32_t light_count,
                             const float* lum, uint64_t lum_stride, uint32_t texel_count,
                             const svf_lsq_options* options, const float* init,
                             float* out, float* rmse, svf_texel_stats* stats);

/* svf_lsq_fit_batch without any allocation.  This entry point has no
 * counterpart in the reference.
 *
 * It is for callers that must not allocate GPU memory while they fit: an
 * engine or framework that owns every device allocation through its own pool
 * and forbids cudaMalloc/cudaFree behind its back, or a frame loop that must
 * not stall or fragment memory on allocation.  It calls no cudaMalloc,
 * cudaFree or other allocating routine and needs no context.  Its working
 * memory (luminance slabs, direction table, work counter, error flag) is one
 * static device array of SVF_NOALLOC_SCRATCH_BYTES that every GPU which loads
 * the library holds until the process exits.
 *
 * - Every buffer (lights_parabolic, lum, init, out, rmse, stats) must be plain
 *   device memory of the current device (not host, managed or another GPU's
 *   memory); stats may be NULL.  Other buffers are rejected with SVF_EINVAL
 *   before anything is launched.
 * - Status: as svf_lsq_fit_batch.  SVF_ETIMEOUT when a bounded device wait
 *   expired; with stats given, SVF_EPARTIAL when some texel ends with
 *   SVF_TEXEL_NONFINITE or SVF_TEXEL_TIMEOUT.
 * - Limits: light_count <= 160 and texel_count * (L*L rounded up to 8) <=
 *   SVF_NOALLOC_MAX_SLAB_FLOATS (79 texels at 81 directions); larger sizes are
 *   rejected with SVF_EINVAL.
 * - stream is a cudaStream_t (NULL for the legacy default stream); the call
 *   enqueues its work there and waits for it before returning.
 * - The first call on each device looks up the address of the static array
 *   (cudaGetSymbolAddress) with that device current; make that first call
 *   before any stream capture.  The address is kept for the life of the
 *   process: after a cudaDeviceReset of a device this entry point must not be
 *   called on that device again in the same process.
 * - All calls share the array and it keeps the last call's contents; calls
 *   whose work overlaps on the GPU (other threads or streams) race on it and
 *   must be serialised by the caller. */
#define SVF_NOALLOC_MAX_SLAB_FLOATS (1u << 19)
#define SVF_NOALLOC_SCRATCH_BYTES   ((size_t)(SVF_NOALLOC_MAX_SLAB_FLOATS) * 4u + 4096u)
svf_status svf_lsq_fit_batch_noalloc(const float* lights_parabolic, uint32_t light_count, const float* lum,
                                     uint64_t lum_stride, uint32_t texel_count, const svf_lsq_options* options,
                                     const float* init, float* out, float* rmse, svf_texel_stats* stats,
                                     void* stream);

/* The svbrdffit texel loop ----------------------------------------------------- */
#define SVF_SAMPLES_F32 0u
#define SVF_SAMPLES_F16 1u

#define SVF_INIT_DEFAULT 0u   /* the reference's default initial guess (NDF -> PCA -> SGGX projection) */
#define SVF_INIT_GIVEN   1u   /* caller-supplied initial parameters (svbrdffit -r refit) */
#define SVF_INIT_MLP     2u   /* the learned initial guess of svf_fit_options::mlp (see svf_mlp_train) */

typedef struct svf_btf_view
{
    const void*            samples;      /* [texels][L*L][3] RGB, texel-major, row-major texels */
    uint32_t               sample_type;  /* SVF_SAMPLES_F32 or SVF_SAMPLES_F16 */
    uint32_t               width, height;
    const svf_layout_desc* layout;
} svf_btf_view;

typedef struct svf_mlp svf_mlp;

typedef struct svf_fit_options
{
    svf_lsq_options lsq;
    uint32_t        init_mode;     /* SVF_INIT_* */
    const float*    init_params;   /* [texels][7] for SVF_INIT_GIVEN */
    const svf_mlp*  mlp;           /* SVF_INIT_MLP: a model trained for the BTF's direction layout */
    float           initial_damping;  /* LM's first damping as a multiple of the reference's rule
                                         (0.75 max(1, max diag J^T J), fitting.hh:531-538).  0: that
                                         rule, except 1e-4 of it from the learned guess, which starts
                                         near a minimum where the full damping takes steps below
                                         BreakOnSmallStep and ends the fit early.  No reference
                                         counterpart. */
    float           mlp_fallback;  /* SVF_INIT_MLP, luminance fit, svf_fit_texels: texels whose RMSE
                                      exceeds this fraction of their luminance slice's RMS are fitted
                                      from the default guess as well, and keep the lower RMSE (the
                                      plain-LM fallback); 0: off */
} svf_fit_options;

/* The five output maps of svbrdffit (svbrdf-fitting.cc:713-735, values as
 * SVBRDFFitPipeline::fit assembles them, svbrdf-fitting-pipeline.cc:692-697),
 * plus optional diagnostics.  Any pointer may be NULL to skip that output. */
typedef struct svf_maps
{
    float*           diffuse;    /* [texels][3]  avg chromaticity * diffuse */
    float*           specular;   /* [texels][3]  avg chromaticity * specular */
    float*           sigma;      /* [texels][2]  SGGX standard deviations */
    float*           basis;      /* [texels][4]  quaternion xyzw = ToQuaternion(euler) */
    float*           rmse;       /* [texels] */
    float*           params;     /* [texels][7]  fitted parameters ([texels][12] with SVF_LSQ_RGB) */
    float*           init;       /* [texels][7]  initial guess used ([texels][12] with SVF_LSQ_RGB) */
    svf_texel_stats* stats;      /* [texels] */
    float*           ndf;        /* [texels][64*64]  NDF texture of the default initial
                                  * guess (getLastNDFTexture, svbrdf-fitting.hh:180),
                                  * row-major, 0 outside the hemisphere; SVF_INIT_DEFAULT
                                  * only */
} svf_maps;

typedef struct svf_run_stats
{
    uint64_t texels;
    uint64_t iterations;        /* summed over texels */
    uint64_t jacobians;
    uint64_t residuals;
    uint64_t failed_texels;     /* texels with a non-zero status */
    double   ms_total;          /* device time of the whole run */
    double   ms_luminance;      /* luminance slice + average chromaticity */
    double   ms_init;           /* default initial guess */
    double   ms_fit;            /* Levenberg-Marquardt */
    double   ms_copy;           /* host<->device staging, when host buffers were given */
    uint32_t lm_threads;        /* LM kernel configuration the autotuner chose: CTA size */
    uint32_t lm_slots;          /* and texels in flight per CTA */
    double   ms_ndf;            /* the NDF GEMM of the default initial guess (part of ms_init) */
    uint32_t graph;             /* svf_fit_texels: 0 launched directly, 1 recorded into a CUDA graph
                                   and launched, 2 replayed (a repeat of the previous call) */
    uint32_t fallback_texels;   /* SVF_INIT_MLP with mlp_fallback: texels fitted from the default guess
                                   as well (svf_fit_texels) */
    uint32_t ndf_tiles;         /* the NDF GEMM's operator tiles (256 rows x 64 pairs) that hold a
                                   non-zero, which it multiplies, */
    uint32_t ndf_tiles_total;   /* of all its tiles (0 when no default guess ran) */
} svf_run_stats;

svf_status svf_fit_texels(svf_ctx* ctx, const svf_btf_view* btf, const svf_fit_options* options,
                          const svf_maps* out, svf_run_stats* run /* may be NULL */);

/* The texel loop over a batch of BTFs of uneven sizes and any mix of direction
 * layouts (several svbrdffit runs, svbrdf-fitting.cc:86-121, in one call).
 * BTF i has its own view, options (init mode and initial parameters; the lsq
 * options must be the same for all) and maps.  Texels of up to 16 BTFs share
 * one persistent LM launch, whatever their layouts; a slot that finishes a
 * texel takes the next one of any BTF.  runs (optional): one svf_run_stats per
 * BTF (texels, iterations, Jacobians, trials, failed texels; the times are the
 * whole call's); total (optional): the whole call.  SVF_EPARTIAL when a texel
 * of any BTF produced no finite fit. */
svf_status svf_fit_btfs(svf_ctx* ctx, const svf_btf_view* btfs, uint32_t n_btf, const svf_fit_options* options,
                        const svf_maps* maps, svf_run_stats* runs /* [n_btf] or NULL */,
                        svf_run_stats* total /* may be NULL */);

/* Learned initial guess -------------------------------------------------------------
 * No counterpart in the reference, whose only initial guess is the NDF -> PCA ->
 * SGGX projection pipeline (svbrdf-fitting-pipeline.cc:350-660).  A small MLP
 * (96 -> 256 -> 256 -> 8, GELU) maps 96 log-scaled features of a texel (32
 * fixed direction pairs x RGB, or 64 half-vector bins + 32 pairs of its
 * luminance) to the luminance fit's parameters, as log S (the SGGX matrix's
 * logarithm, 6 values), log ks, log kd; it is trained on seeded synthetic texels
 * that the plain LM, started from the reference's default guess, has fitted.
 * SVF_INIT_MLP then starts LM from its prediction: the fit skips the NDF
 * pipeline, and its result is compared with the plain LM's residual.
 * Inference runs the hidden layers on the tensor cores with weights and
 * activations split into BF16 hi/lo pairs, accumulating in FP32 (the FP32
 * network to about 1e-5). */
#define SVF_MLP_FEATURES_PAIRS_RGB 0u   /* 32 fixed direction pairs x RGB, log-scaled */
#define SVF_MLP_FEATURES_BINS      1u   /* 64 half-vector bins of the luminance slab + 32 pairs' luminance */

typedef struct svf_mlp_train_options
{
    uint32_t texels;          /* synthetic training texels (default 1 << 20) */
    uint32_t seed, mix;       /* svf_synth_btf seed and parameter mix of the training texels */
    uint32_t epochs;          /* passes over the texels (default 48) */
    uint32_t batch;           /* texels per Adam step (default 4096) */
    float    lr;              /* Adam step size (default 2e-3, cosine-decayed to 5% of it) */
    uint32_t max_iterations;  /* of the LM that makes the targets (default 1024) */
    uint32_t features;        /* SVF_MLP_FEATURES_* (default SVF_MLP_FEATURES_BINS) */
} svf_mlp_train_options;

void       svf_mlp_train_options_default(svf_mlp_train_options* o);
/* Trains a model for the direction layout lights_parabolic [L][2]; *final_loss
 * (optional) is the MSE of the last epoch on the normalised targets. */
svf_status svf_mlp_train(svf_ctx* ctx, const float* lights_parabolic, uint32_t L, const svf_mlp_train_options* o,
                         svf_mlp** out, float* final_loss);
/* The model's initial guess for texels of RGB samples [texels][L*L][3] (host or
 * device): params [texels][7]; features [texels][96] (optional) receives the
 * normalised network inputs. */
svf_status svf_mlp_predict(svf_ctx* ctx, const svf_mlp* mlp, const void* samples, uint32_t sample_type,
                           uint32_t texels, float* params, float* features);
/* One optimiser step on given normalised features [rows][96] and targets
 * [rows][8] (sgd != 0: plain gradient step of size lr; else Adam); *loss is
 * the MSE before the step.  For checking the training kernels. */
svf_status svf_mlp_step(svf_ctx* ctx, svf_mlp* mlp, const float* features, const float* targets, uint32_t rows,
                        float lr, uint32_t sgd, float* loss);
/* Serialisation: *size is set to the bytes needed; with buf != NULL and
 * *size large enough the model is written. */
svf_status svf_mlp_save(const svf_mlp* mlp, void* buf, size_t* size);
svf_status svf_mlp_load(svf_ctx* ctx, const void* buf, size_t size, svf_mlp** out);
void       svf_mlp_destroy(svf_mlp* mlp);

/* Factored BTF files ---------------------------------------------------------------
 * The DFMF, FMF0 and FMF1 files LoadBTF reads (src/image/btf.cc:389-1028): the
 * SVD planes are uploaded once and decoded on the GPU (BTFEvaluateMatrix +
 * BTFFetchSpectrum, btf.hh:498-556,608-634), texel y*W + x after LoadBTF's row
 * flip.  Only RGB (3-channel) files with 2-, 4- or 8-byte elements and colour
 * model 0 or 11 are read, as BTFFetchSpectrum evaluates only those. */
typedef struct svf_btf svf_btf;

typedef struct svf_btf_info
{
    uint32_t format;          /* 0 DFMF, 1 FMF0, 2 FMF1 */
    uint32_t width, height;
    uint32_t light_count;     /* directions (views = lights) */
    uint32_t data_size;       /* bytes per plane element: 2 (half), 4, 8 */
    uint32_t color_model;     /* 0 or 11 (log-YUV) */
    uint32_t dynamic_range_reduction;
    uint32_t cosine_flag;
    uint32_t version;         /* BTFCommonHeader::Version */
    uint32_t components[3];   /* SVD components per channel */
} svf_btf_info;

/* Parses a file image on the host (no device, no context): SVF_EINVAL where
 * LoadBTF rejects the file or its content is not decodable.  lights_parabolic
 * (optional, [light_count][2], at most 160 directions) receives the directions
 * as LoadBTF derives them (BTF::LightsParabolic). */
svf_status svf_btf_probe(const void* file, size_t size, svf_btf_info* info, float* lights_parabolic);
/* Parses a file image and uploads its planes to the context's device. */
svf_status svf_btf_load(svf_ctx* ctx, const void* file, size_t size, svf_btf** out);
svf_status svf_btf_load_file(svf_ctx* ctx, const char* path, svf_btf** out);
svf_status svf_btf_get_info(const svf_btf* btf, svf_btf_info* info, float* lights_parabolic);
/* RGB samples [count][L*L][3] (F32 or F16, device or host memory) of texels
 * [first, first + count). */
svf_status svf_btf_decode(svf_ctx* ctx, const svf_btf* btf, uint64_t first, uint64_t count, uint32_t sample_type,
                          void* samples);
/* svbrdffit on a loaded BTF: decodes texels chunk by chunk into device memory
 * (FP32) and fits them as svf_fit_texels does.  mesh (optional): the
 * interpolation mesh of the default initial guess (triangles and edges of the
 * BTF's directions, e.g. LoadBTF's); NULL: the library's own triangulation. */
svf_status svf_fit_btf(svf_ctx* ctx, const svf_btf* btf, const svf_layout_desc* mesh, const svf_fit_options* options,
                       const svf_maps* maps, svf_run_stats* run);
void       svf_btf_destroy(svf_btf* btf);

/* Error of fitted maps against a BTF ------------------------------------------------
 * svbrdf-error-tool (tools/svbrdf-error-tool/svbrdf-error-tool.cc:88-250) on the
 * GPU: per texel of the maps' region, the SGGX surface BRDF of the map values
 * (Fresnel 1) against the BTF texel (x0 + x, y0 + y), residuals of the luminance
 * or per channel (color), pair-wise (MSE over all light-view pairs) or max-view
 * (the view with the largest sum over lights); RMSE and PSNR = 20 log10(peak /
 * RMSE) with the peak BTF value of the pairs taken. */
#define SVF_ERROR_PAIRWISE 0u
#define SVF_ERROR_MAX_VIEW 1u

typedef struct svf_svbrdf_maps
{
    const float* diffuse;      /* [height][width][3] */
    const float* specular;     /* [height][width][3] */
    const float* sigma;        /* [height][width][sigma_channels] */
    uint32_t     sigma_channels;   /* 2: (sx, sy); 3: (sx, sy, sz), used as (sx/sz, sy/sz) */
    const float* basis;        /* [height][width][4] quaternion xyzw */
    uint32_t     width, height;
} svf_svbrdf_maps;

/* rmse, psnr: [height][width] ([height][width][3] with color), host or device;
 * the maps likewise. */
svf_status svf_error_maps(svf_ctx* ctx, const svf_btf* btf, const svf_svbrdf_maps* maps, uint32_t x0, uint32_t y0,
                          uint32_t method, uint32_t color, float* rmse, float* psnr);

/* Refit --------------------------------------------------------------------------------
 * svbrdffit -r (refit from saved maps, svbrdf-fitting.cc:510-569 and
 * SVBRDFFitPipeline::fit's reoptimize branch, pipeline.cc:661-670): the 7 fit
 * parameters of maps -- diffuse and specular as RGBToLuminance of the albedos,
 * the SGGX scales, Euler angles of the basis quaternion (ToMatrix3 then
 * Matrix3::decompose) -- for svf_fit_texels with SVF_INIT_GIVEN; colour
 * (optional, [texels][3]) receives specular / its luminance, the chromaticity the
 * reference colours the refit maps with.  The reference decomposes an
 * uninitialised matrix there instead of the quaternion's (SGGXProjectIntegrand::
 * Basis is default-constructed); this function converts the quaternion itself. */
svf_status svf_params_from_maps(const svf_svbrdf_maps* maps, float* params /* [texels][7] */, float* colour);

/* svbrdffit -j (optimize-neighborhood, NeighborhoodPusherThread,
 * svbrdf-fitting.cc:123-178) as one batched GPU pass: every texel's luminance
 * slice is fitted from the parameters of each texel of its 3x3 neighbourhood
 * (itself included, clipped to the image) -- nine LM fits per texel in one
 * persistent launch -- and the texel keeps the first candidate, in row order,
 * whose RMSE is below its current one (params_in, rmse_in: the first fit's).
 * All candidates start from the input maps (the reference's threads update
 * the maps while others read them).  The reference's loop, as written, fits the
 * texel's own default guess nine times and stores a better result in the
 * neighbour's slot (fit is called without its reoptimize flag, and the inner
 * index shadows the texel's); this pass does what the option describes.
 * out: params, rmse and the four maps of the selected parameters (coloured by
 * the BTF's average chromaticity). */
svf_status svf_refit_neighborhood(svf_ctx* ctx, const svf_btf_view* btf, const svf_lsq_options* options,
                                  const float* params_in, const float* rmse_in, const svf_maps* out,
                                  svf_run_stats* run);

/* Rendered BTF of SVBRDF maps: samples [texels][L*L][3] (lv = view * L + light;
 * F32 or F16, device or host) of the SGGX surface BRDF (SGGXMicroFlakeSurfaceBRDF,
 * ggx-models-impl.hh:476-552) with each texel's map values as material, as
 * svbrdf-error-tool sets it up (fresnel: refractive index, 1 for none).  The
 * inverse of the fit: fitting the rendered BTF recovers the maps. */
svf_status svf_render_btf(svf_ctx* ctx, const float* lights_parabolic, uint32_t light_count,
                          const svf_svbrdf_maps* maps, float fresnel, uint32_t sample_type, void* samples);

/* Rendered BTF of SVBRDF maps with the pseudo-volume multi-scattering BRDF
 * (SGGXMicroFlakePseudoVolumeBRDF, ggx-models-impl.hh:621-758) in RGB: per
 * pair, `samples` random walks of at most `bounces` scattering events from LCG
 * state `seed` (the fitter's evaluator: 256 walks, seed 0, which is what the
 * SVF_LSQ_MULTI_SCATTERING fit models), the walk continuing while every
 * channel's throughput is above 1e-3; the basis quaternion is used as stored
 * (unnormalised, as the pseudo-volume BRDF takes it).  Layout and sample types as
 * svf_render_btf. */
svf_status svf_render_btf_ms(svf_ctx* ctx, const float* lights_parabolic, uint32_t light_count,
                             const svf_svbrdf_maps* maps, uint32_t bounces, uint32_t samples, uint32_t seed,
                             uint32_t sample_type, void* samples_out);

/* OpenEXR maps ----------------------------------------------------------------------
 * svbrdffit's output files (svbrdf-fitting.cc:713-735, SaveEXRImage in
 * src/image/exr-image.cc): uncompressed FLOAT scanlines, channels R, G, B, A
 * (the first 1..4), image row y stored as scanline height-1-y.  Host only. */
svf_status svf_exr_write(const char* path, uint32_t width, uint32_t height, uint32_t channels,
                         const float* data /* [height][width][channels] */);
/* Reads an uncompressed scanline OpenEXR file of HALF or FLOAT channels named
 * R/G/B/A into [height][width][channels] floats (LoadEXRImage's layout).  With
 * data NULL only the dimensions are returned; capacity is data's length in floats. */
svf_status svf_exr_read(const char* path, uint32_t* width, uint32_t* height, uint32_t* channels, float* data,
                        size_t capacity);
/* The svbrdffit file set <prefix>_albedo.exr (diffuse, RGB), _specular.exr (RGB),
 * _sggx_scale.exr (RG), _sggx_basis.exr (RGBA quaternion) and _rmse.exr (R) from
 * host maps of width x height texels; NULL maps are skipped. */
svf_status svf_maps_write_exr(const char* prefix, uint32_t width, uint32_t height, const svf_maps* maps);

/* Synthetic BTFs (test and benchmark inputs) ------------------------------------ */
/* Renders texels [first, first + count) of a seeded synthetic BTF straight into
 * `samples` ([count][L*L][3], device memory, F32 or F16): per texel, ground-truth
 * parameters are drawn with Philox4x32-10 (key = seed, counter = texel), the
 * BRDF is evaluated per channel and every sample is multiplied by
 * (1 + noise * N(0,1)).  mix 0: kd ~ U[0,0.8]^3, ks ~ U[0,1]^3, sigma log-U
 * [0.02,0.8], normal within 30 degrees of +z; mix 1: 20% near-diffuse
 * (ks < 0.05), 10% strongly anisotropic (sigma_x/sigma_y > 8, sigma_y < 0.05),
 * the rest as mix 0.  truth (optional, device or host): [count][16] floats =
 * kd[3], ks[3], sigma[2], quat[4], euler[3], kind. */
svf_status svf_synth_btf(svf_ctx* ctx, uint32_t seed, uint32_t mix, const float* lights_parabolic,
                         uint32_t light_count, uint64_t first, uint64_t count, uint32_t sample_type,
                         float noise, void* samples, float* truth);

#ifdef __cplusplus
}
#endif

#endif /* SVF_H */
