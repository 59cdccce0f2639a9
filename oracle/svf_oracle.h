/*
 * svf_oracle.h - CPU restatement of TempestRenderer's per-texel SVBRDF fitting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the parity oracle for the CUDA implementation
 * in tempestrenderer_b200/: tests/, bench.py's CPU-baseline leg and
 * __graft_entry__.smoke() call it as a checker.  The product library never links,
 * loads or falls back to it.
 *
 * Parity is pinned: tests/test_oracle_vs_reference.py compares every function
 * below against the reference's own code compiled from its sources
 * (oracle/_ref/libtempest_ref.so, see oracle/Makefile and ref_harness.cc), and
 * against golden vectors generated from that build (tests/golden/).
 *
 * Conventions follow the reference:
 *   - L directions shared by lights and views, given in parabolic coordinates;
 *   - a direction pair is lv = view*L + light (light fastest);
 *   - the 7 fitted parameters are {sigma_x, sigma_y, specular, diffuse,
 *     euler_x, euler_y, euler_z} (svbrdf-fitting.hh:55-65).
 */
#ifndef SVF_ORACLE_H
#define SVF_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- directions -------------------------------------------------------- */

/* The 81-direction ring layout: theta rings 0/15/30/45/60/75 deg holding
 * 1/6/12/18/20/24 phi-uniform directions.  Writes (theta, phi) in radians. */
uint32_t svfo_ring81_angles(float* theta_phi /* [81][2] */);

/* (theta, phi) -> parabolic coordinates exactly as LoadBTF derives them
 * (SphereToCartesianCoordinates vector3.hh:375-382 with the CPU FastSinCos
 * functions.hh:322-329, then CartesianToParabolicCoordinates vector3.hh:384-387). */
void svfo_angles_to_parabolic(const float* theta_phi, uint32_t count, float* parabolic);

/* ---- BRDF (svbrdf-lsq-fitting-internal.hh:91-153, ggx-models-impl.hh:476-552) -- */

/* FP32 evaluation in the reference's operation order; params are doubles as the
 * LM hands them to the evaluator. */
float svfo_brdf_f32(const double* params7, const float* lights_parabolic, uint32_t light_count,
                    uint32_t view, uint32_t light, float fresnel);
/* The same model evaluated in double precision throughout (the FP64 reference values). */
double svfo_brdf_f64(const double* params7, const float* lights_parabolic, uint32_t light_count,
                     uint32_t view, uint32_t light, double fresnel);
/* The fitter's evaluator with BounceCount = bounces (svbrdffit -m): the pseudo-volume
 * multi-scattering BRDF (SGGXMicroFlakePseudoVolumeBRDF, ggx-models-impl.hh:621-758),
 * 256 random walks from LCG seed 0, in the reference's operation order. */
float svfo_brdf_ms_f32(const double* params7, const float* lights_parabolic, uint32_t light_count,
                       uint32_t view, uint32_t light, uint32_t bounces);
/* svfo_brdf_ms_f32 over all L*L pairs (lv = view * L + light). */
void svfo_brdf_ms_eval_all(const double* params7, const float* lights_parabolic, uint32_t light_count,
                           uint32_t bounces, float* out);
/* The pseudo-volume BRDF of one material in RGB: params_rgb = sx, sy, quaternion xyzw
 * (unnormalised, as ToMatrix3 takes it), diffuse rgb, specular rgb; `samples` walks
 * of at most `bounces` events from LCG state `seed`. */
void svfo_pseudo_volume_rgb(const float* params_rgb, const float* lights_parabolic, uint32_t view, uint32_t light,
                            uint32_t bounces, uint32_t samples, uint32_t seed, float* rgb);
/* All L*L pairs. */
void svfo_brdf_eval_all(const double* params7, const float* lights_parabolic, uint32_t light_count,
                        float fresnel, float* out_f32, double* out_f64);

/* ---- LM (fitting.hh:457-678 driven as in svbrdf-lsq-fitting-setup.cc:234-431) -- */

typedef struct
{
    uint32_t iterations;        /* FitStatistics::IterationCount */
    uint32_t effective;         /* FitStatistics::EffectiveIterationCount */
    uint32_t jacobians;         /* Jacobian builds (1 + accepted steps that continued) */
    uint32_t residuals;         /* residual evaluations, trials included */
    double   mse;               /* FitStatistics::MeanSequaredError */
} svfo_lsq_stats;

/* Fits the 7 (LSF_OPTON_DIFFUSE) parameters to one luminance slice with the
 * reference LM: central finite-difference Jacobian (h = 1e-4), FP64 state,
 * MSE target 1e-6, BreakOnSmallStep 1e-3, `max_steps` iterations
 * (CurveFitSteps = 1024 in the reference).  Returns RMSE. */
float svfo_lsq_fit(const float* lum, const float* lights_parabolic, uint32_t light_count, float fresnel,
                   uint32_t max_steps, const float* init7, float* out7, svfo_lsq_stats* stats);
/* The same fit on the pseudo-volume model (LeastSquaresFitOptions::MultiScatteringBounceCount
 * = bounces, svbrdffit -m). */
float svfo_lsq_fit_ms(const float* lum, const float* lights_parabolic, uint32_t light_count, uint32_t bounces,
                      uint32_t max_steps, const float* init7, float* out7, svfo_lsq_stats* stats);

/* ---- luminance slice (btf.cc:1078-1116) --------------------------------- */

/* rgb: [N][3] samples of one texel; lum: [N]; avg_chroma: [3]. */
void svfo_lum_slice(const float* rgb, uint32_t pair_count, float* lum, float* avg_chroma);

/* ---- default initial guess (svbrdf-fitting-pipeline.cc:350-660) -------- */

typedef struct
{
    const float*    lights_parabolic;   /* [L][2] */
    uint32_t        light_count;
    const uint32_t* triangles;          /* [T][3] Delaunay mesh of the parabolic directions */
    uint32_t        triangle_count;
    const uint32_t* edges;              /* [E][3] boundary edges: Index0, Index1, Triangle */
    const float*    edge_angles;        /* [E][2] Angle0, Angle1 (sorted by Angle1) */
    uint32_t        edge_count;
} svfo_mesh;

/* Interpolated luminance lookup BTFSampleLuminanceSlice (btf.hh:229-257). */
float svfo_sample_lum(const svfo_mesh* mesh, const float* light3, const float* view3, const float* lum);

/* NDF texture, 64x64 parabolic map (NDFRecord, pipeline.cc:110-133). */
void svfo_ndf_texture(const svfo_mesh* mesh, const float* lum, float* ndf /* [64*64] */);

/* Bilinear, wrapping NDF lookup (Texture::sample, texture.hh:483-520). */
float svfo_ndf_sample(const float* ndf, float tcx, float tcy);

typedef struct
{
    float ndf_denom;            /* integral of the NDF (pipeline.cc:403-406) */
    float normal[3];            /* most prominent normal (pipeline.cc:429-489) */
    float tangent[3];           /* most prominent tangent (pipeline.cc:604-628) */
    float basis[9];             /* columns: cross(t,n), t, n */
    float sggx_stddev[3];       /* ndf_norm * integral |B^T n| NDF (pipeline.cc:639) */
} svfo_init_info;

/* Full default initial guess from a precomputed NDF texture: writes init7. */
void svfo_default_init_from_ndf(const float* ndf, float* init7, svfo_init_info* info);

/* Matrix3::decompose (matrix3.hh:311-332) of a column-major basis. */
void svfo_decompose(const float* basis9, float* scaling3, float* euler3);

/* ToMatrix3(ToQuaternion(euler)) (quaternion.hh:82-94,122-139), column-major,
 * with the CPU FastSinCos. */
void svfo_euler_to_matrix(const float* euler3, float* matrix9, float* quat4);

/* ---- synthetic BTF texels (test and benchmark inputs) -------------------- */

/* Philox4x32-10 (Salmon et al., SC'11). */
void svfo_philox4x32(const uint32_t key[2], const uint32_t ctr[4], uint32_t out[4]);

typedef struct
{
    float kd[3], ks[3];         /* RGB albedos */
    float sigma[2];             /* SGGX standard deviations */
    float quat[4];              /* orientation, xyzw, unit */
    float euler[3];             /* decompose(ToMatrix3(quat)) */
    uint32_t kind;              /* 0 regular, 1 near-diffuse, 2 strongly anisotropic */
} svfo_texel_truth;

/* Ground truth of texel `texel` for generator `seed` and mix `mix`
 * (0: every texel as config 0; 1: 20% near-diffuse, 10% anisotropic). */
void svfo_synth_truth(uint32_t seed, uint32_t mix, uint64_t texel, svfo_texel_truth* truth);

/* Renders one texel: rgb[N][3] = BRDF(truth) * (1 + N(0, noise)) per sample and channel. */
void svfo_synth_render(uint32_t seed, uint64_t texel, const svfo_texel_truth* truth,
                       const float* lights_parabolic, uint32_t light_count, float noise, float* rgb);

/* ---- factored BTF decode (BTFEvaluateMatrix btf.hh:608-634 + BTFFetchSpectrum
 * btf.hh:498-556) ---------------------------------------------------------- */

/* The planes of a factored BTF as LoadBTF leaves them (btf.cc:660-1022):
 * channel c's sample is sum_k U_c[lv][k] * SxV_c[col][k] with U_c row lv at
 * u[c] + lv * u_row[c] elements and SxV_c row col at sxv[c] + col * sxv_row[c]
 * (DFMF: one plane pair per channel; FMF: U rows interleaved by channel and one
 * shared SxV).  col is the file column of texel (x, y): LoadBTF flips rows, so
 * texel y*W + x reads column (H - 1 - y)*W + x. */
typedef struct svfo_btf_planes
{
    uint32_t data_size;              /* 2 (IEEE half), 4 (float) or 8 (double) */
    uint32_t width, height, light_count;
    uint32_t color_model;            /* 0 or 11 (log-YUV) */
    uint32_t drr;                    /* DynamicRangeReduction: exp(x) - 1e-5 */
    const void* u[3];
    const void* sxv[3];
    uint32_t k[3];
    uint64_t u_row[3], sxv_row[3];   /* row strides in elements */
} svfo_btf_planes;

/* RGB samples [count][L*L][3] of texels [first, first + count) (texel index
 * y*W + x, after the flip), each exactly as BTFFetchSpectrum computes it on the
 * CPU: a sequential sum in the data type's accumulator (float for half and
 * float, double for double), then the colour model and DRR with libm expf. */
void svfo_btf_decode(const svfo_btf_planes* p, uint64_t first, uint64_t count, float* out);

#ifdef __cplusplus
}
#endif

#endif
