// svf_ms.cu - the pseudo-volume multi-scattering BRDF (svbrdffit -m).
//
// SGGXMicroFlakePseudoVolumeBRDF (ggx-models-impl.hh:621-758): a single-
// scattering term plus `samples` random walks of at most `depth` scattering
// events inside a pseudo volume of SGGX micro-flakes, the walks of one
// evaluation drawing from one LCG sequence (FastFloatRand, functions.hh:214-
// 252) in order.  Because a walk's start state depends on how many numbers the
// walks before it drew, the walks of an evaluation run in order on one thread;
// the parallelism is over texels, direction pairs and (for the Jacobian) the
// 14 perturbed parameter vectors of a pair.
//
//   ms_render_kernel    the BTF of SVBRDF maps with this BRDF (RGB)
//   ms_eval_kernel      residuals of the luminance fit, or the 14 central-
//                       difference evaluations of a pair's Jacobian row
//   ms_reduce_kernel    a texel's residual sum, or J^T J and J^T r (FP64, fixed order)
//   ms_control_kernel   the LM step logic of LevenbergMarquardtCurveFit
//                       (fitting.hh:457-678), one thread per texel, FP64
//
// This file is compiled with -fmad=false: every float operation rounds as in
// the reference's x86-64 build (no fused multiply-adds), so an evaluation
// differs from the reference's only through the last bits of logf, expf and
// tanf (and, rarely, a walk that those bits send across one of its break tests).
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/svf.h"
#include "svf_internal.h"

namespace svf
{
namespace
{

constexpr float kPi = 3.141592f;   // functions.hh:55

struct V3
{
    float x, y, z;
};
__device__ __forceinline__ V3 v3(float x, float y, float z) { return V3{ x, y, z }; }
__device__ __forceinline__ V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
// Vector3 * float (vector3.hh:159,163)
__device__ __forceinline__ V3 scale(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float len(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
// Vector3 / float multiplies by the reciprocal (vector3.hh:185-190)
__device__ __forceinline__ V3 divs(V3 a, float s)
{
    const float r = 1.0f / s;
    return scale(a, r);
}
__device__ __forceinline__ V3 normalize(V3 a)
{
    const float l = len(a);
    return l != 0.0f ? divs(a, l) : a;
}
__device__ __forceinline__ V3 cross(V3 a, V3 b)
{
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// Reflect (vector3.hh:420): 2 (n . i) n - i
__device__ __forceinline__ V3 reflect(V3 i, V3 n) { return sub(scale(n, 2.0f * dot(n, i)), i); }

// A 3x3 matrix by columns, as Matrix3::Columns (matrix3.hh:40-56).
struct M3
{
    V3 c[3];
};

// Matrix3 * Matrix3 (matrix3.hh:355-360)
__device__ __forceinline__ M3 mmul(const M3& l, const M3& r)
{
    M3 o;
#pragma unroll
    for(int j = 0; j < 3; ++j)
        o.c[j] = add(add(scale(l.c[0], r.c[j].x), scale(l.c[1], r.c[j].y)), scale(l.c[2], r.c[j].z));
    return o;
}

__device__ __forceinline__ M3 transpose(const M3& m)
{
    M3 o;
    o.c[0] = v3(m.c[0].x, m.c[1].x, m.c[2].x);
    o.c[1] = v3(m.c[0].y, m.c[1].y, m.c[2].y);
    o.c[2] = v3(m.c[0].z, m.c[1].z, m.c[2].z);
    return o;
}

// Matrix3::transformCovariance (matrix3.hh:151-158): B diag(var) B^T
__device__ __forceinline__ M3 covariance(const M3& b, V3 var)
{
    M3 o;
    o.c[0] = add(add(scale(scale(b.c[0], var.x), b.c[0].x), scale(scale(b.c[1], var.y), b.c[1].x)),
                 scale(scale(b.c[2], var.z), b.c[2].x));
    o.c[1] = add(add(scale(scale(b.c[0], var.x), b.c[0].y), scale(scale(b.c[1], var.y), b.c[1].y)),
                 scale(scale(b.c[2], var.z), b.c[2].y));
    o.c[2] = add(add(scale(scale(b.c[0], var.x), b.c[0].z), scale(scale(b.c[1], var.y), b.c[1].z)),
                 scale(scale(b.c[2], var.z), b.c[2].z));
    return o;
}

__device__ __forceinline__ V3 transform(const M3& m, V3 v)
{
    return add(add(scale(m.c[0], v.x), scale(m.c[1], v.y)), scale(m.c[2], v.z));
}

// Matrix3::transformRotationInverse (matrix3.hh:139-142): B^T v
__device__ __forceinline__ V3 rot_inverse(const M3& m, V3 v) { return v3(dot(v, m.c[0]), dot(v, m.c[1]), dot(v, m.c[2])); }

// Matrix3::makeBasis (matrix3.hh:99-108): a frame whose third column is n
__device__ __forceinline__ M3 basis_of(V3 n)
{
    const V3 d0 = cross(v3(1.0f, 0.0f, 0.0f), n), d1 = cross(v3(0.0f, 1.0f, 0.0f), n);
    const float l0 = dot(d0, d0), l1 = dot(d1, d1);
    M3 o;
    o.c[0] = l0 > l1 ? divs(d0, sqrtf(l0)) : divs(d1, sqrtf(l1));
    o.c[1] = cross(n, o.c[0]);
    o.c[2] = n;
    return o;
}

// Matrix3::choleskyDecomposition (matrix3.hh:173-191)
__device__ __forceinline__ M3 cholesky(const M3& m)
{
    const float l00 = sqrtf(m.c[0].x);
    const float r00 = 1.0f / l00;
    const float l10 = r00 * m.c[0].y;
    const float l20 = r00 * m.c[0].z;
    const float l11 = sqrtf(m.c[1].y - l10 * l10);
    const float r11 = 1.0f / l11;
    const float l21 = r11 * (m.c[1].z - l20 * l10);
    const float l22 = sqrtf(m.c[2].z - l21 * l21 - l20 * l20);
    M3 o;
    o.c[0] = v3(l00, l10, l20);
    o.c[1] = v3(0.0f, l11, l21);
    o.c[2] = v3(0.0f, 0.0f, l22);
    return o;
}

// FloatIntelFastRand (functions.hh:214-218,249-252)
__device__ __forceinline__ float lcg(unsigned& s)
{
    s = 214013u * s + 2531011u;
    return (float)((s >> 16) & 0x7FFFu) / 32767.0f;
}

// SinCos_Tan (functions.hh:322-329), the reference's FastSinCos on the CPU
__device__ __forceinline__ void sincos_tan(float w, float* s, float* c)
{
    const float t = tanf(w * 0.5f);
    const float t2 = t * t;
    const float d = 1.0f / (1.0f + t2);
    *s = 2.0f * t * d;
    *c = (1.0f - t2) * d;
}

// SGGXProjectedArea (ggx-models-impl.hh:102-105)
__device__ __forceinline__ float projected_area(V3 sd, const M3& b, V3 w) { return len(mul(rot_inverse(b, w), sd)); }

// SGGXMicroFlakeNDF(stddev, basis, normal) (ggx-models-impl.hh:49-57), split
// into what one evaluation's parameters fix (the inverse covariance, its
// determinant test and the numerator 0.5 sqrt(det)) and the per-normal rest;
// the same operations in the same order as the reference's single function.
struct NdfConst
{
    M3 ic;
    float num;   // 0.5 sqrt(det); 0 where det < 1e-6 (the reference returns 0)
};

__device__ __forceinline__ NdfConst ndf_const(V3 sd, const M3& b)
{
    const V3 sq = mul(sd, sd);
    NdfConst k;
    k.ic = covariance(b, v3(1.0f / sq.x, 1.0f / sq.y, 1.0f / sq.z));
    const M3& ic = k.ic;
    // Matrix3::determinant (matrix3.hh:193-201), Elements[i][j] = column i, row j
    const float det = ic.c[0].x * (ic.c[1].y * ic.c[2].z - ic.c[1].z * ic.c[2].y) -
                      ic.c[1].x * (ic.c[0].y * ic.c[2].z - ic.c[0].z * ic.c[2].y) +
                      ic.c[2].x * (ic.c[0].y * ic.c[1].z - ic.c[0].z * ic.c[1].y);
    k.num = det < 1e-6f ? 0.0f : 0.5f * sqrtf(det);
    return k;
}

__device__ __forceinline__ float sggx_ndf(const NdfConst& k, V3 n)
{
    if(k.num == 0.0f)
        return 0.0f;
    const float den = dot(n, transform(k.ic, n));
    return k.num / (kPi * den * den);
}

// SGGXMicroFlakeSampleIncidentLight (ggx-models-impl.hh:554-570): a visible
// normal of the distribution seen from `wo`, and wo reflected about it.  The
// reference's GCC build evaluates the two FastFloatRand arguments of
// UniformSampleSphere right to left: the second draws first.
// cov: Matrix3::transformCovariance of the basis by stddev^2, fixed per evaluation.
__device__ __forceinline__ V3 sample_incident(V3 wo, const M3& cov, unsigned& seed)
{
    const float rb = lcg(seed);
    const float ra = lcg(seed);
    // UniformSampleSphere (sampling3.hh:106-116)
    float s, c;
    sincos_tan(2.0f * kPi * ra, &s, &c);
    const float ct = 2.0f * rb - 1.0f;
    const float st = sqrtf(1.0f - ct * ct);
    const V3 u = v3(c * st, s * st, ct);
    const M3 ob = basis_of(wo);
    const M3 S = mmul(mmul(ob, cov), transpose(ob));
    const V3 vn = transform(ob, normalize(rot_inverse(cholesky(S), u)));
    return reflect(wo, vn);
}

// SGGXMicroFlakePseudoVolumeBRDF in the fitting frame (tangent x, binormal y,
// normal z) for C spectrum channels; the walk continues while every channel's
// throughput is above 1e-3.  The reference's Fresnel branch is compiled out
// (USE_PSEUDO_VOLUME_FRESNEL is not defined).
template <int C>
__device__ void pseudo_volume(const float* spec, const float* diff, V3 sd, const M3& b, float out_density, V3 wi, V3 wo,
                              uint32_t depth, uint32_t samples, unsigned seed, float* out)
{
    const float dot_inc = wi.z, dot_out = wo.z;
#pragma unroll
    for(int c = 0; c < C; ++c)
        out[c] = 0.0f;
    if(dot_out < 0.0f || dot_inc < 0.0f)
        return;
    if(sd.x < 1e-6f || sd.y < 1e-6f)
        return;
    (void)lcg(seed);
    const float in_density = projected_area(sd, b, wi);
    const V3 h = normalize(add(wo, wi));
    const float contrib = (float)samples / (out_density + in_density * dot_out / dot_inc);
    // what the evaluation's parameters fix, computed once (the reference recomputes it per call)
    const NdfConst nk = ndf_const(sd, b);
    const M3 cov = covariance(b, mul(sd, sd));
    const float ndf = sggx_ndf(nk, h);
    float rad[C], thr[C];
#pragma unroll
    for(int c = 0; c < C; ++c)
        rad[c] = spec[c] * contrib * ndf * 2.0f * 0.25f;
    for(uint32_t s = 0; s < samples; ++s)
    {
#pragma unroll
        for(int c = 0; c < C; ++c)
            thr[c] = spec[c];
        V3 out_l = wo;
        float dd = out_density;
        float depth_in = (-logf(lcg(seed)) / dd) * dot_out;
        for(uint32_t it = 0; it < depth; ++it)
        {
            bool alive = true;
#pragma unroll
            for(int c = 0; c < C; ++c)
                alive = alive && thr[c] > 1e-3f;
            if(!alive)
                break;
            const V3 inc_l = sample_incident(out_l, cov, seed);
            dd = projected_area(sd, b, inc_l);
            out_l = v3(-inc_l.x, -inc_l.y, -inc_l.z);
            depth_in += (-logf(lcg(seed)) / dd) * out_l.z;
            if(depth_in < 0.0f)
                break;
            const float ext = expf(-in_density * (depth_in / dot_inc));
            if(ext < 1e-9f)
                break;
            const float f = sggx_ndf(nk, normalize(add(out_l, wi))) * 2.0f / (4.0f * dd);
#pragma unroll
            for(int c = 0; c < C; ++c)
            {
                thr[c] *= spec[c];
                rad[c] += ext * thr[c] * f;
            }
        }
    }
    const float rcp = 1.0f / (float)samples;
#pragma unroll
    for(int c = 0; c < C; ++c)
        out[c] = rad[c] * rcp + diff[c] * dot_inc * (1.0f / kPi);
}

// ToQuaternion(euler) (quaternion.hh:82-94) with the reference's FastSinCos,
// then ToMatrix3 (quaternion.hh:122-139) of the unnormalised quaternion, as
// the pseudo-volume BRDF takes it (ggx-models-impl.hh:660).
__device__ __forceinline__ M3 quat_matrix(const float* r)
{
    const float xx = r[0] * r[0], xy = r[0] * r[1], xz = r[0] * r[2], xw = r[0] * r[3];
    const float yy = r[1] * r[1], yz = r[1] * r[2], yw = r[1] * r[3];
    const float zz = r[2] * r[2], zw = r[2] * r[3];
    M3 m;
    m.c[0] = v3(1.0f - 2.0f * (yy + zz), 2.0f * (xy + zw), 2.0f * (xz - yw));
    m.c[1] = v3(2.0f * (xy - zw), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + xw));
    m.c[2] = v3(2.0f * (xz + yw), 2.0f * (yz - xw), 1.0f - 2.0f * (xx + yy));
    return m;
}

__device__ __forceinline__ M3 euler_matrix(const float* e)
{
    float s1, c1, s2, c2, s3, c3;
    sincos_tan(0.5f * e[0], &s1, &c1);
    sincos_tan(0.5f * e[1], &s2, &c2);
    sincos_tan(0.5f * e[2], &s3, &c3);
    const float q[4] = { s1 * c2 * c3 + c1 * s2 * s3, -s1 * c2 * s3 + c1 * s2 * c3, c1 * c2 * s3 + s1 * s2 * c3,
                         c1 * c2 * c3 - s1 * s2 * s3 };
    return quat_matrix(q);
}

// BRDFEvaluator::operator() with BounceCount = depth (svbrdf-lsq-fitting-
// internal.hh:91-153): parameters handed over as doubles and rounded to float,
// 256 walks from LCG seed 0 (the evaluator's texture coordinate is 0).
__device__ float evaluator_ms(const double* pd, V3 wi, V3 wo, uint32_t depth)
{
    float p[7];
#pragma unroll
    for(int k = 0; k < 7; ++k)
        p[k] = (float)pd[k];
    const V3 sd = v3(p[0] > 0.0f ? p[0] : 0.0f, p[1] > 0.0f ? p[1] : 0.0f, 1.0f);
    const M3 b = euler_matrix(p + 4);
    const float ks = p[2] > 0.0f ? p[2] : 0.0f;
    const float kd = p[3] > 0.0f ? p[3] : 0.0f;
    float r;
    pseudo_volume<1>(&ks, &kd, sd, b, projected_area(sd, b, wo), wi, wo, depth, 256u, 0u, &r);
    return r;
}

__device__ __forceinline__ V3 direction(const float* geo, uint32_t L, uint32_t d)
{
    return v3(geo[d], geo[L + d], geo[2 * L + d]);
}

} // namespace

// ---- rendering ----------------------------------------------------------------------

__global__ void __launch_bounds__(128) ms_render_kernel(MsRenderArgs a)
{
    const uint64_t N = (uint64_t)a.L * a.L;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= a.count * N)
        return;
    const uint64_t t = i / N;
    const uint32_t lv = (uint32_t)(i % N);
    const uint32_t view = lv / a.L, light = lv % a.L;
    float sx = a.sigma[a.sigma_channels * t], sy = a.sigma[a.sigma_channels * t + 1];
    if(a.sigma_channels == 3)
    {
        const float sz = a.sigma[3 * t + 2];
        sx = sx / sz;
        sy = sy / sz;
    }
    const V3 sd = v3(sx > 0.0f ? sx : 0.0f, sy > 0.0f ? sy : 0.0f, 1.0f);
    float q[4], kd[3], ks[3];
#pragma unroll
    for(int k = 0; k < 4; ++k)
        q[k] = a.basis[4 * t + k];
#pragma unroll
    for(int c = 0; c < 3; ++c)
    {
        kd[c] = fmaxf(a.diffuse[3 * t + c], 0.0f);
        ks[c] = fmaxf(a.specular[3 * t + c], 0.0f);
    }
    const M3 b = quat_matrix(q);
    const V3 wi = direction(a.geo, a.L, light), wo = direction(a.geo, a.L, view);
    float f[3];
    pseudo_volume<3>(ks, kd, sd, b, projected_area(sd, b, wo), wi, wo, a.bounces, a.samples, a.seed, f);
    const uint64_t o = i * 3;
#pragma unroll
    for(int c = 0; c < 3; ++c)
    {
        if(a.sample_type == SVF_SAMPLES_F16)
            static_cast<__half*>(a.out)[o + c] = __float2half_rn(f[c]);
        else
            static_cast<float*>(a.out)[o + c] = f[c];
    }
}

cudaError_t launch_ms_render(const MsRenderArgs& a, cudaStream_t stream)
{
    const uint64_t n = a.count * (uint64_t)a.L * a.L;
    if(n == 0)
        return cudaSuccess;
    const uint64_t blocks = (n + 127) / 128;
    if(blocks > 0x7fffffffull)
        return cudaErrorInvalidValue;
    ms_render_kernel<<<(unsigned)blocks, 128, 0, stream>>>(a);
    return cudaGetLastError();
}

// ---- the multi-scattering LM fit ------------------------------------------------------
//
// LevenbergMarquardtCurveFit (fitting.hh:457-678) with the central-difference
// Jacobian ParallelFDComputeResidualJacobianCenterPoint (fitting.hh:883-908,
// step (|p| + 1e-4) 1e-4) over the evaluator above, for a batch of texels.
// Each texel's LM state lives in MsTexel; the host runs the LM's iterations
// in lock step (every texel one iteration per round) as a sequence of
// launches: control (the step) -> residuals of the trial points -> control
// (gain, accept) -> Jacobians of the accepted points -> J^T J, J^T r ->
// control (damping).  The control stages append the texels that need the
// next evaluation to a list, whose length the host reads to size that launch.

namespace
{

constexpr int kMsEvals = 14;   // two evaluations per parameter

// The texel's parameters with parameter k moved by +-its finite-difference step.
__device__ __forceinline__ void fd_params(const MsTexel& s, int e, double* p)
{
#pragma unroll
    for(int i = 0; i < 7; ++i)
        p[i] = s.p[i];
    const int k = e >> 1;
    const double h = (double)1e-4f;
    const double step = (fabs(s.p[k]) + h) * h;
    p[k] = (e & 1) ? s.p[k] - step : s.p[k] + step;
}

} // namespace

// count: the list's length, or (dcount non-null) at most this many, *dcount
__global__ void __launch_bounds__(128) ms_eval_kernel(MsFitArgs a, uint32_t mode, uint32_t count,
                                                      const uint32_t* dcount)
{
    if(dcount)
        count = min(count, *dcount);
    const uint64_t N = (uint64_t)a.L * a.L;
    const uint64_t per = mode == kMsEvalJacobian ? N * kMsEvals : N;
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if(i >= (uint64_t)count * per)
        return;
    const uint32_t t = a.list[i / per];
    const uint64_t r = i % per;
    const MsTexel& s = a.st[t];
    const uint32_t idx = (uint32_t)(mode == kMsEvalJacobian ? r / kMsEvals : r);
    const V3 wi = direction(a.geo, a.L, idx % a.L), wo = direction(a.geo, a.L, idx / a.L);
    if(mode == kMsEvalJacobian)
    {
        double p[7];
        fd_params(s, (int)(r % kMsEvals), p);
        a.fev[(uint64_t)t * N * kMsEvals + r] = -evaluator_ms(p, wi, wo, a.bounces);
        return;
    }
    const float f = evaluator_ms(mode == kMsEvalTrial ? s.tmp : s.p, wi, wo, a.bounces);
    a.res[(uint64_t)t * N + idx] = a.lum[t * a.lum_stride + idx] - f;
}

// Per listed texel: the sum of squared residuals (residual modes) or J^T J and
// J^T r (Jacobian mode), in FP64 with a fixed reduction order.
__global__ void __launch_bounds__(256) ms_reduce_kernel(MsFitArgs a, uint32_t mode, const uint32_t* dcount)
{
    constexpr int kV = 35;   // J^T r (7) + the upper triangle of J^T J (28)
    __shared__ double part[8][kV];
    if(dcount && blockIdx.x >= *dcount)
        return;
    const uint32_t t = a.list[blockIdx.x];
    MsTexel& s = a.st[t];
    const uint32_t N = a.L * a.L;
    const float* res = a.res + (uint64_t)t * N;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if(mode != kMsEvalJacobian)
    {
        double sum = 0.0;
        for(uint32_t idx = threadIdx.x; idx < N; idx += blockDim.x)
        {
            const float r = res[idx];
            sum += (double)(r * r);
        }
        for(int o = 16; o > 0; o >>= 1)
            sum += __shfl_down_sync(0xffffffffu, sum, o);
        if(lane == 0)
            part[warp][0] = sum;
        __syncthreads();
        if(threadIdx.x == 0)
        {
            double tot = 0.0;
            for(int w = 0; w < (int)(blockDim.x >> 5); ++w)
                tot += part[w][0];
            if(mode == kMsEvalTrial)
                s.trial = tot;
            else
                s.last = tot;
            ++s.residuals;
        }
        return;
    }
    double step2[7];
    const double h = (double)1e-4f;
#pragma unroll
    for(int k = 0; k < 7; ++k)
        step2[k] = 2.0f * ((fabs(s.p[k]) + h) * h);
    double v[kV];
#pragma unroll
    for(int k = 0; k < kV; ++k)
        v[k] = 0.0;
    const float* fev = a.fev + (uint64_t)t * N * kMsEvals;
    for(uint32_t idx = threadIdx.x; idx < N; idx += blockDim.x)
    {
        double J[7];
#pragma unroll
        for(int k = 0; k < 7; ++k)
            J[k] = (double)(fev[(uint64_t)idx * kMsEvals + 2 * k] - fev[(uint64_t)idx * kMsEvals + 2 * k + 1]) /
                   step2[k];
        const double r = (double)res[idx];
        int o = 7;
#pragma unroll
        for(int i = 0; i < 7; ++i)
        {
            v[i] += J[i] * r;
#pragma unroll
            for(int j = i; j < 7; ++j)
                v[o++] += J[i] * J[j];
        }
    }
#pragma unroll
    for(int k = 0; k < kV; ++k)
    {
        double x = v[k];
        for(int o = 16; o > 0; o >>= 1)
            x += __shfl_down_sync(0xffffffffu, x, o);
        if(lane == 0)
            part[warp][k] = x;
    }
    __syncthreads();
    if(threadIdx.x < kV)
    {
        double tot = 0.0;
        for(int w = 0; w < (int)(blockDim.x >> 5); ++w)
            tot += part[w][threadIdx.x];
        const int k = threadIdx.x;
        if(k < 7)
            s.grad[k] = tot;
        else
        {
            int o = 7;
            for(int i = 0; i < 7; ++i)
                for(int j = i; j < 7; ++j, ++o)
                    if(o == k)
                    {
                        s.hess[7 * i + j] = tot;
                        s.hess[7 * j + i] = tot;
                    }
        }
    }
    if(threadIdx.x == 0)
        ++s.jacobians;
}

namespace
{

// Inverse by Gauss-Jordan elimination with partial pivoting (FP64), as the
// oracle restates the reference's Eigen PartialPivLU inverse.
__device__ void invert7(const double* a, double* inv)
{
    double m[7][14];
    for(int i = 0; i < 7; ++i)
        for(int j = 0; j < 14; ++j)
            m[i][j] = j < 7 ? a[7 * i + j] : (j - 7 == i ? 1.0 : 0.0);
    for(int col = 0; col < 7; ++col)
    {
        int piv = col;
        for(int r = col + 1; r < 7; ++r)
            if(fabs(m[r][col]) > fabs(m[piv][col]))
                piv = r;
        if(piv != col)
            for(int j = 0; j < 14; ++j)
            {
                const double t = m[col][j];
                m[col][j] = m[piv][j];
                m[piv][j] = t;
            }
        const double d = m[col][col];
        for(int j = 0; j < 14; ++j)
            m[col][j] /= d;
        for(int r = 0; r < 7; ++r)
        {
            if(r == col)
                continue;
            const double f = m[r][col];
            for(int j = 0; j < 14; ++j)
                m[r][j] -= f * m[col][j];
        }
    }
    for(int i = 0; i < 7; ++i)
        for(int j = 0; j < 7; ++j)
            inv[7 * i + j] = m[i][7 + j];
}

// The step stage of one texel (phase kMsStep): the damped solve, the small-step
// and constraint tests, and the trial point (listed for its residuals).
__device__ void ms_step(const MsFitArgs& a, MsTexel& s, uint32_t t)
{
    const double N = (double)a.L * a.L;
    const double eps = a.eps;
    if(!(s.iter < a.max_iter && a.mse_target < s.last / N))
    {
        s.phase = kMsDone;
        return;
    }
    double damp[49], inv[49];
    for(int i = 0; i < 49; ++i)
        damp[i] = s.hess[i];
    for(int i = 0; i < 7; ++i)
        damp[8 * i] += s.damping;
    invert7(damp, inv);
    if(!isfinite(inv[0]))
    {
        s.damping *= s.mult;
        s.mult *= s.mult;
        ++s.iter;
        return;
    }
    double step_len = 0.0, pmag = 0.0;
    for(int i = 0; i < 7; ++i)
    {
        double v = 0.0;
        for(int j = 0; j < 7; ++j)
            v += inv[7 * i + j] * s.grad[j];
        s.step[i] = v;
        step_len += v * v;
        const double q = s.p[i] + eps;
        pmag += q * q;
    }
    if(sqrt(step_len) <= eps * (sqrt(pmag) + eps))
    {
        s.phase = kMsDone;
        return;
    }
    // AcceptStepConstraints (svbrdf-lsq-fitting-internal.hh:67-77)
    bool accept = true;
    for(int i = 0; i < 4; ++i)
        if(s.p[i] - s.step[i] < 0.0f)
            accept = false;
    if(!accept)
    {
        s.damping *= s.mult;
        s.mult *= s.mult;
        ++s.iter;
        return;
    }
    for(int i = 0; i < 7; ++i)
        s.tmp[i] = s.p[i] - s.step[i];
    s.phase = kMsTrial;
    a.list[atomicAdd(&a.counts[0], 1u)] = t;
}

} // namespace

// One thread per texel of the batch.  stage: kMsStageStart (after the first
// residual and Jacobian), kMsStageStep, kMsStageGain, kMsStageDamping.
__global__ void ms_control_kernel(MsFitArgs a, uint32_t stage)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= a.texels)
        return;
    MsTexel& s = a.st[t];
    const double N = (double)a.L * a.L;
    const double eps = a.eps;
    if(stage == kMsStageStart)
    {
        double d = 1.0;
        for(int i = 0; i < 7; ++i)
            d = fmax(d, s.hess[8 * i]);
        s.damping = d * (double)0.75f;
        s.mult = 2.0;
        s.phase = kMsStep;
        return;
    }
    if(stage == kMsStageStep)
    {
        if(s.phase == kMsStep)
            ms_step(a, s, t);
        if(s.phase != kMsDone)
            atomicAdd(&a.counts[2], 1u);
        return;
    }
    if(stage == kMsStageGain)
    {
        if(s.phase != kMsTrial)
            return;
        double pred = 0.0;
        for(int i = 0; i < 7; ++i)
            pred += s.step[i] * (s.step[i] * s.damping + s.grad[i]);
        pred *= 0.5f;
        const double gain = 0.5f * (s.last - s.trial) / pred;
        if(gain > 0.0f)
        {
            ++s.effective;
            for(int i = 0; i < 7; ++i)
                s.p[i] = s.tmp[i];
            s.last = s.trial;
            if(s.last / N <= a.mse_target)
            {
                s.phase = kMsDone;
                return;
            }
            s.gain = gain;
            s.phase = kMsJacobian;
            a.list[atomicAdd(&a.counts[1], 1u)] = t;
        }
        else
        {
            s.damping *= s.mult;
            s.mult *= s.mult;
            ++s.iter;
            s.phase = kMsStep;
        }
        return;
    }
    // kMsStageDamping: after the accepted point's J^T J and J^T r
    if(s.phase != kMsJacobian)
        return;
    double glen = 0.0;
    for(int i = 0; i < 7; ++i)
        glen += s.grad[i] * s.grad[i];
    if(glen <= eps * eps)
    {
        s.phase = kMsDone;
        return;
    }
    const double min_mul = 1.0f / 3.0f;
    s.damping *= fmax(min_mul, 1.0f - pow(2.0f * s.gain - 1.0f, 3.0f));
    s.mult = 2.0f;
    ++s.iter;
    s.phase = kMsStep;
}

// The batch's state from the initial guesses; every texel listed.
__global__ void ms_setup_kernel(MsFitArgs a, const float* init)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= a.texels)
        return;
    MsTexel& s = a.st[t];
    for(int i = 0; i < 7; ++i)
        s.p[i] = init[7 * (uint64_t)t + i];
    s.iter = s.effective = s.jacobians = s.residuals = 0;
    s.phase = kMsStep;
    a.list[t] = t;
}

// The fitted parameters, RMSE and statistics; a texel whose fit is not finite
// gets its initial guess back and SVF_TEXEL_NONFINITE.
__global__ void ms_finish_kernel(MsFitArgs a, const float* init, float* out, float* rmse, svf_texel_stats* stats)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if(t >= a.texels)
        return;
    const MsTexel& s = a.st[t];
    bool finite = true;
    float v[7];
    for(int i = 0; i < 7; ++i)
    {
        v[i] = (float)s.p[i];
        finite = finite && isfinite(v[i]);
    }
    const float r = (float)sqrt(s.last / ((double)a.L * a.L));
    finite = finite && isfinite(r);
    for(int i = 0; i < 7; ++i)
        out[7 * (uint64_t)t + i] = finite ? v[i] : init[7 * (uint64_t)t + i];
    if(rmse)
        rmse[t] = r;
    if(stats)
    {
        svf_texel_stats st;
        st.iterations = s.iter;
        st.effective = s.effective;
        st.jacobians = s.jacobians;
        st.residuals = s.residuals;
        st.status = (finite ? 0u : SVF_TEXEL_NONFINITE) | (s.iter >= a.max_iter ? SVF_TEXEL_MAX_ITER : 0u);
        stats[t] = st;
    }
}

cudaError_t launch_ms_setup(const MsFitArgs& a, const float* init, cudaStream_t stream)
{
    ms_setup_kernel<<<(unsigned)((a.texels + 127) / 128), 128, 0, stream>>>(a, init);
    return cudaGetLastError();
}

cudaError_t launch_ms_eval(const MsFitArgs& a, uint32_t mode, uint32_t count, const uint32_t* dcount,
                           cudaStream_t stream)
{
    if(count == 0)
        return cudaSuccess;
    const uint64_t N = (uint64_t)a.L * a.L;
    const uint64_t n = (uint64_t)count * N * (mode == kMsEvalJacobian ? kMsEvals : 1);
    const uint64_t blocks = (n + 127) / 128;
    if(blocks > 0x7fffffffull)
        return cudaErrorInvalidValue;
    ms_eval_kernel<<<(unsigned)blocks, 128, 0, stream>>>(a, mode, count, dcount);
    cudaError_t e = cudaGetLastError();
    if(e != cudaSuccess)
        return e;
    ms_reduce_kernel<<<count, 256, 0, stream>>>(a, mode, dcount);
    return cudaGetLastError();
}

cudaError_t launch_ms_control(const MsFitArgs& a, uint32_t stage, cudaStream_t stream)
{
    ms_control_kernel<<<(unsigned)((a.texels + 127) / 128), 128, 0, stream>>>(a, stage);
    return cudaGetLastError();
}

cudaError_t launch_ms_finish(const MsFitArgs& a, const float* init, float* out, float* rmse, svf_texel_stats* stats,
                             cudaStream_t stream)
{
    ms_finish_kernel<<<(unsigned)((a.texels + 127) / 128), 128, 0, stream>>>(a, init, out, rmse, stats);
    return cudaGetLastError();
}

} // namespace svf
