/*
 * svf_oracle.c - CPU restatement of TempestRenderer's per-texel SVBRDF fitting path.
 *
 * TEST INFRASTRUCTURE ONLY (see svf_oracle.h).  Every function cites the
 * reference file:line it restates.  Floating-point expressions keep the
 * reference's operation order, and the file is compiled with
 * -ffp-contract=off so that, like the reference's x86-64 build (no -mfma), no
 * multiply-add is fused.  The parity of this file with the reference build is
 * checked by tests/test_oracle_vs_reference.py and the golden vectors in
 * tests/golden/.
 */
#include "svf_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* functions.hh:55 - the reference's value of pi */
#define REF_PI 3.141592f

typedef struct { float x, y, z; } v3;
/* Column-major 3x3 matrix: c[i] is column i, as Matrix3::Columns (matrix3.hh:40-56). */
typedef struct { v3 c[3]; } m3;

static inline v3 v3make(float x, float y, float z) { v3 r = { x, y, z }; return r; }
static inline v3 v3add(v3 a, v3 b) { return v3make(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 v3sub(v3 a, v3 b) { return v3make(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 v3mul(v3 a, v3 b) { return v3make(a.x * b.x, a.y * b.y, a.z * b.z); }
/* vector3.hh:159,163: Vector3 * float multiplies each component */
static inline v3 v3scale(v3 a, float s) { return v3make(a.x * s, a.y * s, a.z * s); }
static inline float v3dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
/* vector3.hh:72 */
static inline float v3len(v3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
/* vector3.hh:185-190: division by a scalar multiplies by its reciprocal */
static inline v3 v3div(v3 a, float s) { float r = 1.0f / s; return v3scale(a, r); }
/* vector3.hh:215-219 */
static inline v3 v3normalize(v3 a) { float l = v3len(a); return l != 0.0f ? v3div(a, l) : a; }
/* vector3.hh:102-104 */
static inline v3 v3cross(v3 a, v3 b)
{
    return v3make(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float elem(const m3* m, int i, int j)
{
    const float* c = &m->c[i].x;
    return c[j];
}

/* ---------------------------------------------------------------------------
 * RNG and trigonometry used by the reference's samplers
 * ------------------------------------------------------------------------- */

/* IntelFastRand / FloatIntelFastRand, functions.hh:214-218,249-252 */
static inline float lcg_float(unsigned* seed)
{
    *seed = 214013u * (*seed) + 2531011u;
    return (float)((*seed >> 16) & 0x7FFFu) / 0x7FFF;
}

/* SinCos_Tan, functions.hh:322-329: FastSinCos on the CPU */
static inline void sincos_tan(float omega, float* s, float* c)
{
    float t = tanf(omega * 0.5f);
    float t2 = t * t;
    float div = 1.0f / (1.0f + t2);
    *s = 2.0f * t * div;
    *c = (1.0f - t2) * div;
}

/* ---------------------------------------------------------------------------
 * Directions
 * ------------------------------------------------------------------------- */

uint32_t svfo_ring81_angles(float* theta_phi)
{
    static const int ring_deg[6] = { 0, 15, 30, 45, 60, 75 };
    static const int ring_count[6] = { 1, 6, 12, 18, 20, 24 };
    uint32_t k = 0;
    for(int r = 0; r < 6; ++r)
    {
        float theta = (float)((double)ring_deg[r] * 3.14159265358979323846 / 180.0);
        for(int i = 0; i < ring_count[r]; ++i)
        {
            float phi = (float)(2.0 * 3.14159265358979323846 * (double)i / (double)ring_count[r]);
            theta_phi[2 * k] = theta;
            theta_phi[2 * k + 1] = phi;
            ++k;
        }
    }
    return k;
}

/* SphereToCartesianCoordinates (vector3.hh:375-382), CartesianToParabolicCoordinates (vector3.hh:384-387) */
static v3 sphere_to_cartesian(float theta, float phi)
{
    float ct, st, cp, sp;
    sincos_tan(theta, &st, &ct);
    sincos_tan(phi, &sp, &cp);
    return v3make(cp * st, sp * st, ct);
}

void svfo_angles_to_parabolic(const float* theta_phi, uint32_t count, float* parabolic)
{
    for(uint32_t i = 0; i < count; ++i)
    {
        v3 d = sphere_to_cartesian(theta_phi[2 * i], theta_phi[2 * i + 1]);
        parabolic[2 * i] = d.x / (d.z + 1.0f);
        parabolic[2 * i + 1] = d.y / (d.z + 1.0f);
    }
}

/* ParabolicToCartesianCoordinates, vector3.hh:389-393 */
static inline v3 parabolic_to_cartesian(float px, float py)
{
    float len_sq = px * px + py * py;
    return v3make(2.0f * px / (len_sq + 1.0f), 2.0f * py / (len_sq + 1.0f), (1 - len_sq) / (1 + len_sq));
}

/* ---------------------------------------------------------------------------
 * SGGX surface BRDF
 * ------------------------------------------------------------------------- */

/* ToQuaternion(euler), quaternion.hh:82-94 (x, y, z, w) */
static void euler_to_quat(const float* e, float* q)
{
    float c1, c2, c3, s1, s2, s3;
    sincos_tan(0.5f * e[0], &s1, &c1);
    sincos_tan(0.5f * e[1], &s2, &c2);
    sincos_tan(0.5f * e[2], &s3, &c3);
    q[0] = s1 * c2 * c3 + c1 * s2 * s3;
    q[1] = -s1 * c2 * s3 + c1 * s2 * c3;
    q[2] = c1 * c2 * s3 + s1 * s2 * c3;
    q[3] = c1 * c2 * c3 - s1 * s2 * s3;
}

/* ToMatrix3(quaternion), quaternion.hh:122-139 */
static m3 quat_to_matrix(const float* r)
{
    float xx = r[0] * r[0], xy = r[0] * r[1], xz = r[0] * r[2], xw = r[0] * r[3];
    float yy = r[1] * r[1], yz = r[1] * r[2], yw = r[1] * r[3];
    float zz = r[2] * r[2], zw = r[2] * r[3];
    m3 m;
    m.c[0] = v3make(1.0f - 2.0f * (yy + zz), 2.0f * (xy + zw), 2.0f * (xz - yw));
    m.c[1] = v3make(2.0f * (xy - zw), 1.0f - 2.0f * (xx + zz), 2.0f * (yz + xw));
    m.c[2] = v3make(2.0f * (xz + yw), 2.0f * (yz - xw), 1.0f - 2.0f * (xx + yy));
    return m;
}

/* Normalize(Quaternion), quaternion.hh:253-270 */
static void quat_normalize(const float* q, float* out)
{
    float l = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    if(l == 0)
    {
        out[0] = out[1] = out[2] = 0.0f;
        out[3] = 1.0f;
        return;
    }
    out[0] = q[0] / l;
    out[1] = q[1] / l;
    out[2] = q[2] / l;
    out[3] = q[3] / l;
}

/* Matrix3::transformRotationInverse, matrix3.hh:139-142 */
static inline v3 m3_rot_inverse(const m3* m, v3 v)
{
    return v3make(v3dot(v, m->c[0]), v3dot(v, m->c[1]), v3dot(v, m->c[2]));
}

/* SGGXProjectedArea, ggx-models-impl.hh:102-105 */
static inline float sggx_projected_area(v3 stddev, const m3* basis, v3 w)
{
    return v3len(v3mul(m3_rot_inverse(basis, w), stddev));
}

/* SGGXMicroFlakeNDF(stddev, basis, normal), ggx-models-impl.hh:49-57, with
 * Matrix3::transformCovariance (matrix3.hh:151-158), determinant (:193-201)
 * and transform (:144-147). */
static float sggx_ndf(v3 stddev, const m3* basis, v3 normal)
{
    v3 sq = v3mul(stddev, stddev);
    v3 variance = v3make(1.0f / sq.x, 1.0f / sq.y, 1.0f / sq.z);
    const v3* C = basis->c;
    v3 tan = v3add(v3add(v3scale(v3scale(C[0], variance.x), C[0].x), v3scale(v3scale(C[1], variance.y), C[1].x)),
                   v3scale(v3scale(C[2], variance.z), C[2].x));
    v3 bin = v3add(v3add(v3scale(v3scale(C[0], variance.x), C[0].y), v3scale(v3scale(C[1], variance.y), C[1].y)),
                   v3scale(v3scale(C[2], variance.z), C[2].y));
    v3 nrm = v3add(v3add(v3scale(v3scale(C[0], variance.x), C[0].z), v3scale(v3scale(C[1], variance.y), C[1].z)),
                   v3scale(v3scale(C[2], variance.z), C[2].z));
    m3 ic;
    ic.c[0] = tan;
    ic.c[1] = bin;
    ic.c[2] = nrm;
    float det = elem(&ic, 0, 0) * (elem(&ic, 1, 1) * elem(&ic, 2, 2) - elem(&ic, 1, 2) * elem(&ic, 2, 1)) -
                elem(&ic, 1, 0) * (elem(&ic, 0, 1) * elem(&ic, 2, 2) - elem(&ic, 0, 2) * elem(&ic, 2, 1)) +
                elem(&ic, 2, 0) * (elem(&ic, 0, 1) * elem(&ic, 1, 2) - elem(&ic, 0, 2) * elem(&ic, 1, 1));
    if(det < 1e-6f)
        return 0.0f;
    v3 t = v3add(v3add(v3scale(ic.c[0], normal.x), v3scale(ic.c[1], normal.y)), v3scale(ic.c[2], normal.z));
    float den = v3dot(normal, t);
    return 0.5f * sqrtf(det) / (REF_PI * den * den);
}

/* CosTransmittance / FresnelDielectric, functions.hh:265-268,296-301 */
static float fresnel_dielectric(float refr, float cos_inc)
{
    float cos_trans = sqrtf(1.0f - (1.0f - cos_inc * cos_inc) / (refr * refr));
    float r_par = (refr * cos_inc - cos_trans) / (refr * cos_inc + cos_trans);
    float r_perp = (cos_inc - refr * cos_trans) / (cos_inc + refr * cos_trans);
    float f = 0.5f * (r_par * r_par + r_perp * r_perp);
    return f < 0.0f ? 0.0f : (f > 1.0f ? 1.0f : f);
}

/* SGGXMicroFlakeSurfaceBRDF, ggx-models-impl.hh:476-552, for one scalar channel
 * with the fitting frame (tangent x, binormal y, normal z) and no texture maps.
 * `out_basis` is the (unnormalised) ToMatrix3(quat) the evaluator uses for the
 * directional density (svbrdf-lsq-fitting-internal.hh:132); `basis` is
 * ToMatrix3(Normalize(quat)) (ggx-models-impl.hh:520). */
static float surface_brdf(float kd, float ks, v3 stddev, const m3* basis, float out_density, v3 wi, v3 wo, float refr)
{
    float dot_inc = wi.z;
    float dot_out = wo.z;
    if(dot_inc < 0.0f || dot_out < 0.0f)
        return 0.0f;
    float result = kd * dot_inc * (1.0f / REF_PI);
    if(stddev.x >= 1e-6f && stddev.y >= 1e-6f && stddev.z >= 1e-6f && out_density >= 1e-6f)
    {
        v3 micro = v3normalize(v3add(wi, wo));
        float cos_micro = v3dot(micro, wi);
        float fresnel = refr == 1.0f ? 1.0f : fresnel_dielectric(refr, cos_micro);
        float in_density = sggx_projected_area(stddev, basis, wi);
        float contrib = 1.0f / (out_density + in_density * dot_out / dot_inc);
        result += contrib * ks * sggx_ndf(stddev, basis, micro) * fresnel * 2.0f / 4.0f;
    }
    return result;
}

float svfo_brdf_f32(const double* params7, const float* lp, uint32_t light_count, uint32_t view, uint32_t light, float fresnel)
{
    /* BRDFEvaluator::operator(), svbrdf-lsq-fitting-internal.hh:91-153 */
    float p[7];
    for(int i = 0; i < 7; ++i)
        p[i] = (float)params7[i];
    v3 stddev = v3make(p[0] > 0.0f ? p[0] : 0.0f, p[1] > 0.0f ? p[1] : 0.0f, 1.0f);
    float quat[4], nq[4];
    euler_to_quat(p + 4, quat);
    float kd = p[3] > 0.0f ? p[3] : 0.0f;
    float ks = p[2] > 0.0f ? p[2] : 0.0f;
    v3 wi = parabolic_to_cartesian(lp[2 * light], lp[2 * light + 1]);
    v3 wo = parabolic_to_cartesian(lp[2 * view], lp[2 * view + 1]);
    m3 out_basis = quat_to_matrix(quat);
    float out_density = sggx_projected_area(stddev, &out_basis, wo);
    quat_normalize(quat, nq);
    m3 basis = quat_to_matrix(nq);
    (void)light_count;
    return surface_brdf(kd, ks, stddev, &basis, out_density, wi, wo, fresnel);
}

/* ---------------------------------------------------------------------------
 * Pseudo-volume multi-scattering BRDF (svbrdffit -m)
 * ------------------------------------------------------------------------- */

static inline v3 reflect(v3 inc, v3 n);

/* Matrix3 * Matrix3, matrix3.hh:355-360: column j of the product is
 * rhs.c[j].x * lhs.c[0] + rhs.c[j].y * lhs.c[1] + rhs.c[j].z * lhs.c[2]. */
static m3 m3mul(const m3* lhs, const m3* rhs)
{
    m3 r;
    for(int j = 0; j < 3; ++j)
        r.c[j] = v3add(v3add(v3scale(lhs->c[0], rhs->c[j].x), v3scale(lhs->c[1], rhs->c[j].y)),
                       v3scale(lhs->c[2], rhs->c[j].z));
    return r;
}

/* Matrix3::transpose, matrix3.hh:92-97 */
static m3 m3transpose(const m3* m)
{
    m3 r;
    r.c[0] = v3make(m->c[0].x, m->c[1].x, m->c[2].x);
    r.c[1] = v3make(m->c[0].y, m->c[1].y, m->c[2].y);
    r.c[2] = v3make(m->c[0].z, m->c[1].z, m->c[2].z);
    return r;
}

/* Matrix3::transformCovariance, matrix3.hh:151-158 */
static m3 m3covariance(const m3* b, v3 var)
{
    const v3* C = b->c;
    m3 r;
    r.c[0] = v3add(v3add(v3scale(v3scale(C[0], var.x), C[0].x), v3scale(v3scale(C[1], var.y), C[1].x)),
                   v3scale(v3scale(C[2], var.z), C[2].x));
    r.c[1] = v3add(v3add(v3scale(v3scale(C[0], var.x), C[0].y), v3scale(v3scale(C[1], var.y), C[1].y)),
                   v3scale(v3scale(C[2], var.z), C[2].y));
    r.c[2] = v3add(v3add(v3scale(v3scale(C[0], var.x), C[0].z), v3scale(v3scale(C[1], var.y), C[1].z)),
                   v3scale(v3scale(C[2], var.z), C[2].z));
    return r;
}

/* Matrix3::transform, matrix3.hh:144-147 */
static inline v3 m3transform(const m3* m, v3 v)
{
    return v3add(v3add(v3scale(m->c[0], v.x), v3scale(m->c[1], v.y)), v3scale(m->c[2], v.z));
}

/* Matrix3::makeBasis, matrix3.hh:99-108 */
static m3 m3basis(v3 n)
{
    v3 d0 = v3cross(v3make(1.0f, 0.0f, 0.0f), n), d1 = v3cross(v3make(0.0f, 1.0f, 0.0f), n);
    float l0 = v3dot(d0, d0), l1 = v3dot(d1, d1);
    m3 r;
    r.c[0] = l0 > l1 ? v3div(d0, sqrtf(l0)) : v3div(d1, sqrtf(l1));
    r.c[1] = v3cross(n, r.c[0]);
    r.c[2] = n;
    return r;
}

/* Matrix3::choleskyDecomposition, matrix3.hh:173-191 (columns of the lower factor) */
static m3 m3cholesky(const m3* m)
{
    float l00 = sqrtf(m->c[0].x);
    float rcp_l00 = 1.0f / l00;
    float l10 = rcp_l00 * m->c[0].y;
    float l20 = rcp_l00 * m->c[0].z;
    float l11 = sqrtf(m->c[1].y - l10 * l10);
    float rcp_l11 = 1.0f / l11;
    float l21 = rcp_l11 * (m->c[1].z - l20 * l10);
    float l22 = sqrtf(m->c[2].z - l21 * l21 - l20 * l20);
    m3 r;
    r.c[0] = v3make(l00, l10, l20);
    r.c[1] = v3make(0.0f, l11, l21);
    r.c[2] = v3make(0.0f, 0.0f, l22);
    return r;
}

/* UniformSampleSphere, sampling3.hh:106-116 */
static inline v3 uniform_sphere(float ra, float rb)
{
    float phi = 2.0f * REF_PI * ra;
    float s, c;
    sincos_tan(phi, &s, &c);
    float cos_theta = 2.0f * rb - 1.0f;
    float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
    return v3make(c * sin_theta, s * sin_theta, cos_theta);
}

/* SGGXMicroFlakeSampleIncidentLight(out_light, ...), ggx-models-impl.hh:554-570:
 * a visible normal of the SGGX distribution seen from out_light (the uniform
 * sphere sample mapped through the Cholesky factor of the covariance in the
 * out_light frame), and out_light reflected about it.  The reference passes two
 * FastFloatRand(seed) calls as UniformSampleSphere's arguments; its x86-64 GCC
 * build evaluates them right to left, so the second argument draws first. */
static v3 sggx_sample_incident(v3 wo, v3 stddev, const m3* basis, unsigned* seed)
{
    float rb = lcg_float(seed);
    float ra = lcg_float(seed);
    v3 u = uniform_sphere(ra, rb);
    m3 S = m3covariance(basis, v3mul(stddev, stddev));
    m3 ob = m3basis(wo), obt = m3transpose(&ob);
    m3 t = m3mul(&ob, &S);
    S = m3mul(&t, &obt);
    m3 L = m3cholesky(&S);
    v3 vn = v3normalize(m3_rot_inverse(&L, u));
    vn = m3transform(&ob, vn);
    return reflect(wo, vn);
}

/* SGGXMicroFlakePseudoVolumeBRDF, ggx-models-impl.hh:621-758, in the fitting
 * frame (tangent x, binormal y, normal z) for `channels` spectrum channels (the
 * walk is shared: it continues while every channel's throughput is above
 * 1e-3), `samples` random walks of at most `depth` scattering events from the
 * LCG state `seed` (the reference seeds it from the texture coordinate, 0 for
 * the fitter's evaluator).  The Fresnel branch is compiled out in the reference
 * (USE_PSEUDO_VOLUME_FRESNEL is not defined). */
static void pseudo_volume_brdf(const float* spec, const float* diff, int channels, v3 stddev, const m3* basis,
                               float out_density, v3 wi, v3 wo, uint32_t depth, uint32_t samples, unsigned seed,
                               float* out)
{
    float dot_inc = wi.z, dot_out = wo.z;
    for(int c = 0; c < channels; ++c)
        out[c] = 0.0f;
    if(dot_out < 0.0f || dot_inc < 0.0f)
        return;
    if(stddev.x < 1e-6f || stddev.y < 1e-6f)
        return;
    (void)lcg_float(&seed);
    float incoming_density = sggx_projected_area(stddev, basis, wi);
    v3 micro = v3normalize(v3add(wo, wi));
    float contrib = (float)samples / (out_density + incoming_density * dot_out / dot_inc);
    float ndf = sggx_ndf(stddev, basis, micro);
    float radiance[3], thr[3];
    for(int c = 0; c < channels; ++c)
        radiance[c] = spec[c] * contrib * ndf * 2.0f * (1.0f / 4.0f);
    for(uint32_t s = 0; s < samples; ++s)
    {
        for(int c = 0; c < channels; ++c)
            thr[c] = spec[c];
        v3 out_l = wo;
        float dir_density = out_density;
        float t = lcg_float(&seed);
        float log_step = -logf(t);
        float step = log_step / dir_density;
        float depth_in = step * dot_out;
        for(uint32_t it = 0; it < depth; ++it)
        {
            int alive = 1;
            for(int c = 0; c < channels; ++c)
                alive &= thr[c] > 1e-3f;
            if(!alive)
                break;
            v3 inc_l = sggx_sample_incident(out_l, stddev, basis, &seed);
            dir_density = sggx_projected_area(stddev, basis, inc_l);
            out_l = v3make(-inc_l.x, -inc_l.y, -inc_l.z);
            t = lcg_float(&seed);
            log_step = -logf(t);
            step = log_step / dir_density;
            depth_in += step * out_l.z;
            if(depth_in < 0.0f)
                break;
            float distance = depth_in / dot_inc;
            float extinction = expf(-incoming_density * distance);
            if(extinction < 1e-9f)
                break;
            v3 mn = v3normalize(v3add(out_l, wi));
            float brdf = sggx_ndf(stddev, basis, mn) * 2.0f / (4.0f * dir_density);
            for(int c = 0; c < channels; ++c)
            {
                thr[c] *= spec[c];
                radiance[c] += extinction * thr[c] * brdf;
            }
        }
    }
    float rcp = 1.0f / (float)samples;
    for(int c = 0; c < channels; ++c)
        out[c] = radiance[c] * rcp + diff[c] * dot_inc * (1.0f / REF_PI);
}

float svfo_brdf_ms_f32(const double* params7, const float* lp, uint32_t light_count, uint32_t view, uint32_t light,
                       uint32_t bounces)
{
    /* BRDFEvaluator::operator() with BounceCount = bounces, svbrdf-lsq-fitting-internal.hh:91-153:
     * SampleCount 256, Depth bounces, the unnormalised ToMatrix3(ToQuaternion(euler))
     * as the SGGX basis (ggx-models-impl.hh:660) and the directional density. */
    float p[7];
    for(int i = 0; i < 7; ++i)
        p[i] = (float)params7[i];
    v3 stddev = v3make(p[0] > 0.0f ? p[0] : 0.0f, p[1] > 0.0f ? p[1] : 0.0f, 1.0f);
    float quat[4];
    euler_to_quat(p + 4, quat);
    float kd = p[3] > 0.0f ? p[3] : 0.0f;
    float ks = p[2] > 0.0f ? p[2] : 0.0f;
    v3 wi = parabolic_to_cartesian(lp[2 * light], lp[2 * light + 1]);
    v3 wo = parabolic_to_cartesian(lp[2 * view], lp[2 * view + 1]);
    m3 basis = quat_to_matrix(quat);
    float out_density = sggx_projected_area(stddev, &basis, wo);
    float r;
    (void)light_count;
    pseudo_volume_brdf(&ks, &kd, 1, stddev, &basis, out_density, wi, wo, bounces, 256, 0u, &r);
    return r;
}

void svfo_brdf_ms_eval_all(const double* params7, const float* lp, uint32_t light_count, uint32_t bounces,
                           float* out)
{
    for(uint32_t v = 0; v < light_count; ++v)
        for(uint32_t l = 0; l < light_count; ++l)
            out[v * light_count + l] = svfo_brdf_ms_f32(params7, lp, light_count, v, l, bounces);
}

void svfo_pseudo_volume_rgb(const float* params_rgb, const float* lp, uint32_t view, uint32_t light,
                            uint32_t bounces, uint32_t samples, uint32_t seed, float* rgb)
{
    /* params_rgb: sx, sy, quaternion xyzw (as stored, unnormalised), diffuse rgb, specular rgb */
    v3 stddev = v3make(params_rgb[0] > 0.0f ? params_rgb[0] : 0.0f, params_rgb[1] > 0.0f ? params_rgb[1] : 0.0f, 1.0f);
    m3 basis = quat_to_matrix(params_rgb + 2);
    float kd[3], ks[3];
    for(int c = 0; c < 3; ++c)
    {
        kd[c] = params_rgb[6 + c];
        ks[c] = params_rgb[9 + c];
    }
    v3 wi = parabolic_to_cartesian(lp[2 * light], lp[2 * light + 1]);
    v3 wo = parabolic_to_cartesian(lp[2 * view], lp[2 * view + 1]);
    float out_density = sggx_projected_area(stddev, &basis, wo);
    pseudo_volume_brdf(ks, kd, 3, stddev, &basis, out_density, wi, wo, bounces, samples, seed, rgb);
}

/* The same model in double precision.  sin/cos replace FastSinCos (exact up to
 * rounding), pi is the true value, and the constant 1e-6 thresholds of the
 * reference are kept. */
double svfo_brdf_f64(const double* p, const float* lp, uint32_t light_count, uint32_t view, uint32_t light, double refr)
{
    const double pi = 3.14159265358979323846;
    double sx = p[0] > 0.0 ? p[0] : 0.0, sy = p[1] > 0.0 ? p[1] : 0.0;
    double ks = p[2] > 0.0 ? p[2] : 0.0, kd = p[3] > 0.0 ? p[3] : 0.0;
    double s1 = sin(0.5 * p[4]), c1 = cos(0.5 * p[4]);
    double s2 = sin(0.5 * p[5]), c2 = cos(0.5 * p[5]);
    double s3 = sin(0.5 * p[6]), c3 = cos(0.5 * p[6]);
    double q[4] = { s1 * c2 * c3 + c1 * s2 * s3, -s1 * c2 * s3 + c1 * s2 * c3,
                    c1 * c2 * s3 + s1 * s2 * c3, c1 * c2 * c3 - s1 * s2 * s3 };
    double ql = sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for(int i = 0; i < 4; ++i)
        q[i] /= ql;
    double xx = q[0] * q[0], xy = q[0] * q[1], xz = q[0] * q[2], xw = q[0] * q[3];
    double yy = q[1] * q[1], yz = q[1] * q[2], yw = q[1] * q[3], zz = q[2] * q[2], zw = q[2] * q[3];
    double R[3][3] = { { 1 - 2 * (yy + zz), 2 * (xy + zw), 2 * (xz - yw) },
                       { 2 * (xy - zw), 1 - 2 * (xx + zz), 2 * (yz + xw) },
                       { 2 * (xz + yw), 2 * (yz - xw), 1 - 2 * (xx + yy) } }; /* R[col][row] */
    double wi[3], wo[3];
    {
        double px = lp[2 * light], py = lp[2 * light + 1], l2 = px * px + py * py;
        wi[0] = 2 * px / (l2 + 1); wi[1] = 2 * py / (l2 + 1); wi[2] = (1 - l2) / (1 + l2);
        px = lp[2 * view]; py = lp[2 * view + 1]; l2 = px * px + py * py;
        wo[0] = 2 * px / (l2 + 1); wo[1] = 2 * py / (l2 + 1); wo[2] = (1 - l2) / (1 + l2);
    }
    (void)light_count;
    if(wi[2] < 0 || wo[2] < 0)
        return 0.0;
    double result = kd * wi[2] / pi;
    double sd[3] = { sx, sy, 1.0 };
    /* projected areas |diag(sd) R^T w| */
    double ai = 0, ao = 0;
    for(int c = 0; c < 3; ++c)
    {
        double di = R[c][0] * wi[0] + R[c][1] * wi[1] + R[c][2] * wi[2];
        double dd = R[c][0] * wo[0] + R[c][1] * wo[1] + R[c][2] * wo[2];
        ai += di * di * sd[c] * sd[c];
        ao += dd * dd * sd[c] * sd[c];
    }
    ai = sqrt(ai);
    ao = sqrt(ao);
    if(sx >= 1e-6 && sy >= 1e-6 && ao >= 1e-6)
    {
        double h[3] = { wi[0] + wo[0], wi[1] + wo[1], wi[2] + wo[2] };
        double hl = sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
        for(int i = 0; i < 3; ++i)
            h[i] /= hl;
        double cos_micro = h[0] * wi[0] + h[1] * wi[1] + h[2] * wi[2];
        double fr = 1.0;
        if(refr != 1.0)
        {
            double ct = sqrt(1.0 - (1.0 - cos_micro * cos_micro) / (refr * refr));
            double rp = (refr * cos_micro - ct) / (refr * cos_micro + ct);
            double rs = (cos_micro - refr * ct) / (cos_micro + refr * ct);
            fr = 0.5 * (rp * rp + rs * rs);
            fr = fr < 0 ? 0 : (fr > 1 ? 1 : fr);
        }
        /* inverse covariance R diag(1/sd^2) R^T: det = 1/(sx sy)^2, h^T S^-1 h */
        double det = 1.0 / (sx * sx * sy * sy);
        double quad = 0;
        for(int c = 0; c < 3; ++c)
        {
            double d = R[c][0] * h[0] + R[c][1] * h[1] + R[c][2] * h[2];
            quad += d * d / (sd[c] * sd[c]);
        }
        double ndf = det < 1e-6 ? 0.0 : 0.5 * sqrt(det) / (pi * quad * quad);
        double contrib = 1.0 / (ao + ai * wo[2] / wi[2]);
        result += contrib * ks * ndf * fr * 0.5;
    }
    return result;
}

void svfo_brdf_eval_all(const double* params7, const float* lp, uint32_t light_count, float fresnel, float* out_f32, double* out_f64)
{
    for(uint32_t v = 0; v < light_count; ++v)
        for(uint32_t l = 0; l < light_count; ++l)
        {
            uint32_t idx = v * light_count + l;
            if(out_f32)
                out_f32[idx] = svfo_brdf_f32(params7, lp, light_count, v, l, fresnel);
            if(out_f64)
                out_f64[idx] = svfo_brdf_f64(params7, lp, light_count, v, l, fresnel);
        }
}

/* ---------------------------------------------------------------------------
 * Levenberg-Marquardt
 * ------------------------------------------------------------------------- */

typedef struct
{
    const float* lum;
    const float* lp;
    uint32_t L, N;
    float fresnel;
    int ms;              /* the pseudo-volume model (BounceCount != ~0u) */
    uint32_t bounces;
} lsq_problem;

/* BRDFEvaluator::operator() of the problem's model */
static float model_f32(const lsq_problem* pb, const double* params, uint32_t idx)
{
    if(pb->ms)
        return svfo_brdf_ms_f32(params, pb->lp, pb->L, idx / pb->L, idx % pb->L, pb->bounces);
    return svfo_brdf_f32(params, pb->lp, pb->L, idx / pb->L, idx % pb->L, pb->fresnel);
}

/* ParallelResidualEvaluator::computeResidual, fitting.hh:106-141: residual in
 * float, squared in float, summed in double (one worker, index order). */
static double compute_residual(const lsq_problem* pb, const double* params, double* res)
{
    double sum = 0.0;
    for(uint32_t idx = 0; idx < pb->N; ++idx)
    {
        float out = pb->lum[idx];
        float f = model_f32(pb, params, idx);
        float r = out - f;
        sum += r * r;
        res[idx] = r;
    }
    return sum;
}

/* ParallelFDComputeResidualJacobianCenterPoint, fitting.hh:883-908: row-major
 * [N][P] Jacobian of the residual by central differences of the float model. */
static void compute_jacobian(const lsq_problem* pb, const double* params, uint32_t P, double* jac)
{
    const double h = (double)1e-4f;
    for(uint32_t idx = 0; idx < pb->N; ++idx)
    {
        double tmp[7];
        memcpy(tmp, params, sizeof(double) * 7);
        for(uint32_t k = 0; k < P; ++k)
        {
            double prev = tmp[k];
            double step = (fabs(prev) + h) * h;
            tmp[k] = prev + step;
            float next_res = -model_f32(pb, tmp, idx);
            tmp[k] = prev - step;
            float prev_res = -model_f32(pb, tmp, idx);
            jac[idx * P + k] = (next_res - prev_res) / (2.0f * step);
            tmp[k] = prev;
        }
    }
}

/* Inverse by Gauss-Jordan elimination with partial pivoting (the reference
 * calls Eigen's PartialPivLU inverse, matrix-variadic.cc:183-189). */
static void invert(const double* a, uint32_t n, double* inv)
{
    double m[7 * 14];
    for(uint32_t i = 0; i < n; ++i)
        for(uint32_t j = 0; j < 2 * n; ++j)
            m[i * 2 * n + j] = j < n ? a[i * n + j] : (j - n == i ? 1.0 : 0.0);
    for(uint32_t col = 0; col < n; ++col)
    {
        uint32_t piv = col;
        for(uint32_t r = col + 1; r < n; ++r)
            if(fabs(m[r * 2 * n + col]) > fabs(m[piv * 2 * n + col]))
                piv = r;
        if(piv != col)
            for(uint32_t j = 0; j < 2 * n; ++j)
            {
                double t = m[col * 2 * n + j];
                m[col * 2 * n + j] = m[piv * 2 * n + j];
                m[piv * 2 * n + j] = t;
            }
        double d = m[col * 2 * n + col];
        for(uint32_t j = 0; j < 2 * n; ++j)
            m[col * 2 * n + j] /= d;
        for(uint32_t r = 0; r < n; ++r)
        {
            if(r == col)
                continue;
            double f = m[r * 2 * n + col];
            for(uint32_t j = 0; j < 2 * n; ++j)
                m[r * 2 * n + j] -= f * m[col * 2 * n + j];
        }
    }
    for(uint32_t i = 0; i < n; ++i)
        for(uint32_t j = 0; j < n; ++j)
            inv[i * n + j] = m[i * 2 * n + n + j];
}

static float lsq_fit(const lsq_problem* problem, uint32_t max_steps, const float* init7, float* out7,
                     svfo_lsq_stats* stats);

float svfo_lsq_fit(const float* lum, const float* lp, uint32_t L, float fresnel, uint32_t max_steps,
                   const float* init7, float* out7, svfo_lsq_stats* stats)
{
    lsq_problem pb = { lum, lp, L, L * L, fresnel, 0, 0 };
    return lsq_fit(&pb, max_steps, init7, out7, stats);
}

float svfo_lsq_fit_ms(const float* lum, const float* lp, uint32_t L, uint32_t bounces, uint32_t max_steps,
                      const float* init7, float* out7, svfo_lsq_stats* stats)
{
    /* LeastSquaresFitOptions::MultiScatteringBounceCount = bounces: the same LM on the
     * pseudo-volume model (its Fresnel term is compiled out in the reference) */
    lsq_problem pb = { lum, lp, L, L * L, 1.0f, 1, bounces };
    return lsq_fit(&pb, max_steps, init7, out7, stats);
}

static float lsq_fit(const lsq_problem* problem, uint32_t max_steps, const float* init7, float* out7,
                     svfo_lsq_stats* stats)
{
    /* LeastSquaresFitSGGX with LSF_OPTON_DIFFUSE, svbrdf-lsq-fitting-setup.cc:234-431,
     * running LevenbergMarquardtCurveFit (fitting.hh:457-678). */
    const uint32_t P = 7;
    lsq_problem pb = *problem;
    const uint32_t N = pb.N;
    const double mean_sq_error = 1e-6;
    const double break_criteria = (double)1e-3f;   /* settings.BreakOnSmallStep = 1e-3f */
    const double tau = (double)0.75f, initial_min_damping = 1.0;

    double* res = (double*)malloc(sizeof(double) * N);
    double* jac = (double*)malloc(sizeof(double) * N * P);
    double p[7], tmp[7], step[7], grad[7], hess[49], damp[49], inv[49], diff[7];
    for(uint32_t i = 0; i < P; ++i)
        p[i] = init7[i];

    svfo_lsq_stats st = { 0, 0, 0, 0, 0.0 };
    double last = compute_residual(&pb, p, res);
    st.residuals++;
    compute_jacobian(&pb, p, P, jac);
    st.jacobians++;

    /* MatrixSquare (J^T J) and MatrixTransformVector (J^T r), matrix-variadic.cc:170-181,228-235 */
#define BUILD_NORMAL_EQUATIONS(do_hess)                                                  \
    do {                                                                                 \
        for(uint32_t a = 0; a < P; ++a)                                                  \
        {                                                                                \
            double g = 0.0;                                                              \
            for(uint32_t s = 0; s < N; ++s)                                              \
                g += jac[s * P + a] * res[s];                                            \
            grad[a] = g;                                                                 \
            if(do_hess)                                                                  \
                for(uint32_t b = 0; b < P; ++b)                                          \
                {                                                                        \
                    double h2 = 0.0;                                                     \
                    for(uint32_t s = 0; s < N; ++s)                                      \
                        h2 += jac[s * P + a] * jac[s * P + b];                           \
                    hess[a * P + b] = h2;                                                \
                }                                                                        \
        }                                                                                \
    } while(0)

    BUILD_NORMAL_EQUATIONS(1);

    double damping_multiplier = 2.0;
    double damping = initial_min_damping;
    for(uint32_t i = 0; i < P; ++i)
        damping = fmax(damping, hess[i * P + i]);
    damping *= tau;

    uint32_t iter, effective = 0;
    for(iter = 0; iter < max_steps && mean_sq_error < last / N; ++iter)
    {
        memcpy(damp, hess, sizeof(hess));
        for(uint32_t i = 0; i < P; ++i)
            damp[i * P + i] += damping;
        invert(damp, P, inv);
        if(!isfinite(inv[0]))
        {
            damping *= damping_multiplier;
            damping_multiplier *= damping_multiplier;
            continue;
        }
        double step_len = 0.0, pmag = 0.0;
        for(uint32_t i = 0; i < P; ++i)
        {
            double s = 0.0;
            for(uint32_t j = 0; j < P; ++j)
                s += inv[i * P + j] * grad[j];
            step[i] = s;
            step_len += s * s;
            tmp[i] = p[i] + break_criteria;
            pmag += tmp[i] * tmp[i];
        }
        step_len = sqrt(step_len);
        pmag = sqrt(pmag);
        if(step_len <= break_criteria * (pmag + break_criteria))
            break;
        /* AcceptStepConstraints, svbrdf-lsq-fitting-internal.hh:67-77 */
        int accept = 1;
        for(uint32_t i = 0; i < 4; ++i)
            if(p[i] - step[i] < 0.0f)
                accept = 0;
        if(!accept)
        {
            damping *= damping_multiplier;
            damping_multiplier *= damping_multiplier;
            continue;
        }
        for(uint32_t i = 0; i < P; ++i)
            tmp[i] = p[i] - step[i];
        double sum = compute_residual(&pb, tmp, res);
        st.residuals++;
        double pred = 0.0;
        for(uint32_t i = 0; i < P; ++i)
        {
            diff[i] = step[i] * damping + grad[i];
            pred += step[i] * diff[i];
        }
        pred *= 0.5f;
        double gain = 0.5f * (last - sum) / pred;
        if(gain > 0.0f)
        {
            ++effective;
            memcpy(p, tmp, sizeof(p));
            last = sum;
            if(last / N <= mean_sq_error)
                break;
            compute_jacobian(&pb, p, P, jac);
            st.jacobians++;
            BUILD_NORMAL_EQUATIONS(0);
            double glen = 0.0;
            for(uint32_t i = 0; i < P; ++i)
                glen += grad[i] * grad[i];
            if(glen <= break_criteria * break_criteria)
                break;
            BUILD_NORMAL_EQUATIONS(1);
            double min_mul = 1.0f / 3.0f;
            double mul = fmax(min_mul, 1.0f - pow(2.0f * gain - 1.0f, 3.0f));
            damping *= mul;
            damping_multiplier = 2.0f;
        }
        else
        {
            damping *= damping_multiplier;
            damping_multiplier *= damping_multiplier;
        }
    }
#undef BUILD_NORMAL_EQUATIONS
    st.iterations = iter;
    st.effective = effective;
    st.mse = last / N;
    for(uint32_t i = 0; i < P; ++i)
        out7[i] = (float)p[i];
    if(stats)
        *stats = st;
    free(res);
    free(jac);
    return (float)sqrt(st.mse);
}

/* ---------------------------------------------------------------------------
 * Luminance slice, btf.cc:1078-1116 with RGBToLuminance spectrum.hh:328-331
 * ------------------------------------------------------------------------- */

void svfo_lum_slice(const float* rgb, uint32_t N, float* lum, float* avg)
{
    v3 acc = v3make(0.0f, 0.0f, 0.0f);
    for(uint32_t i = 0; i < N; ++i)
    {
        v3 s = v3make(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]);
        float l = 0.2126f * s.x + 0.7152f * s.y + 0.0722f * s.z;
        v3 chroma = l > 1e-6f ? v3div(s, l) : v3make(1.0f, 1.0f, 1.0f);
        acc = v3add(acc, chroma);
        lum[i] = l;
    }
    v3 r = v3div(acc, (float)N);
    avg[0] = r.x;
    avg[1] = r.y;
    avg[2] = r.z;
}

/* ---------------------------------------------------------------------------
 * Default initial guess
 * ------------------------------------------------------------------------- */

/* TriangleBarycentricCoordinates, intersect.hh:383-401 */
static void tri_bary(float px, float py, const float* v0, const float* v1, const float* v2, float* bx, float* by)
{
    float x1_x3 = v1[0] - v0[0], x2_x3 = v2[0] - v0[0], x_x3 = px - v0[0];
    float y1_y3 = v1[1] - v0[1], y2_y3 = v2[1] - v0[1], y_y3 = py - v0[1];
    float det = x1_x3 * y2_y3 - x2_x3 * y1_y3;
    if(det < 1e-9f)
    {
        float dx = px - v0[0], dy = py - v0[1];
        *bx = *by = sqrtf(dx * dx + dy * dy);
        return;
    }
    *bx = (y2_y3 * x_x3 - x2_x3 * y_y3) / det;
    *by = (-y1_y3 * x_x3 + x1_x3 * y_y3) / det;
}

/* Point location: the first triangle (in index order) whose barycentric test
 * passes (IntersectTriangle, intersect.hh:403-419); the reference walks its
 * BVH (IntersectSSLBVHNodeSingle, sslbvh2.hh:99-130), which can pick another
 * triangle only for points on a shared edge, where both give the same
 * interpolant.  Outside the mesh: IntersectEdge (btf.hh:271-321). */
static void locate(const svfo_mesh* mesh, v3 dir, uint32_t* tri_out, float* bary)
{
    float px = dir.x / (dir.z + 1.0f), py = dir.y / (dir.z + 1.0f);
    const float* lp = mesh->lights_parabolic;
    for(uint32_t t = 0; t < mesh->triangle_count; ++t)
    {
        const uint32_t* tri = mesh->triangles + 3 * t;
        float bx, by;
        tri_bary(px, py, lp + 2 * tri[0], lp + 2 * tri[1], lp + 2 * tri[2], &bx, &by);
        float w = 1.0f - bx - by;
        if(0.0f > bx || bx > 1.0f || 0.0f > by || by > 1.0f || 0.0f > w || w > 1.0f)
            continue;
        *tri_out = t;
        bary[0] = bx;
        bary[1] = by;
        bary[2] = w;
        return;
    }
    /* IntersectEdge */
    float angle = atan2f(dir.y, dir.x);
    uint32_t first = 0, count = mesh->edge_count;
    while(count > 0)
    {
        uint32_t stp = count / 2;
        uint32_t it = first + stp;
        if(mesh->edge_angles[2 * it + 1] < angle)
        {
            first = it + 1;
            count -= stp + 1;
        }
        else
            count = stp;
    }
    if(first == mesh->edge_count)
        first = 0;
    const uint32_t* e = mesh->edges + 3 * first;
    uint32_t t = e[2];
    const uint32_t* tri = mesh->triangles + 3 * t;
    float a0 = mesh->edge_angles[2 * first], a1 = mesh->edge_angles[2 * first + 1];
    float ratio = (angle - a0) / (a1 - a0);
    /* GenericLinearInterpolate, functions.hh:459-462 */
    float qx = (1.0f - ratio) * lp[2 * e[0]] + ratio * lp[2 * e[1]];
    float qy = (1.0f - ratio) * lp[2 * e[0] + 1] + ratio * lp[2 * e[1] + 1];
    float bx, by;
    tri_bary(qx, qy, lp + 2 * tri[0], lp + 2 * tri[1], lp + 2 * tri[2], &bx, &by);
    bx = bx < 0.0f ? 0.0f : (bx > 1.0f ? 1.0f : bx);
    by = by < 0.0f ? 0.0f : (by > 1.0f ? 1.0f : by);
    *tri_out = t;
    bary[0] = bx;
    bary[1] = by;
    bary[2] = 1.0f - bx - by;
}

float svfo_sample_lum(const svfo_mesh* mesh, const float* light3, const float* view3, const float* lum)
{
    /* BTFSampleLuminanceSlice, btf.hh:229-257, via BTFFetchLightViewDirection :323-376 */
    v3 l = v3make(light3[0], light3[1], light3[2]);
    v3 v = v3make(view3[0], view3[1], view3[2]);
    if(v.z < 0.0f || l.z < 0.0f)
        return 0.0f;
    uint32_t lt, vt;
    float lb[3], vb[3];
    locate(mesh, l, &lt, lb);
    locate(mesh, v, &vt, vb);
    float result = 0.0f;
    uint32_t L = mesh->light_count;
    for(uint32_t vi = 0; vi < 3; ++vi)
    {
        uint32_t vv = mesh->triangles[vt * 3 + vi];
        float wv = vb[(vi + 2) % 3];
        for(uint32_t li = 0; li < 3; ++li)
        {
            uint32_t lv = mesh->triangles[lt * 3 + li];
            float wl = lb[(li + 2) % 3];
            result += wl * wv * lum[vv * L + lv];
        }
    }
    return result;
}

/* UniformSampleHemisphere, sampling3.hh:55-62 */
static inline v3 uniform_hemisphere(float ra, float rb)
{
    float r = sqrtf(1.0f - ra * ra);
    float phi = 2.0f * REF_PI * rb;
    float s, c;
    sincos_tan(phi, &s, &c);
    return v3make(c * r, s * r, ra);
}

/* Reflect, vector3.hh:420 */
static inline v3 reflect(v3 inc, v3 n)
{
    float d2 = 2.0f * v3dot(n, inc);
    return v3sub(v3scale(n, d2), inc);
}

void svfo_ndf_texture(const svfo_mesh* mesh, const float* lum, float* ndf)
{
    /* NDFRecord (pipeline.cc:110-133) with StratifiedMonteCarloIntegratorHemisphere
     * (numerical-methods.hh:210-237, 4096 samples, seed 1 for every texel). */
    const uint32_t R = 64, S = 4096, SQ = 64;
    v3* dirs = (v3*)malloc(sizeof(v3) * S);
    unsigned seed = 1;
    float sqrt_samples = sqrtf((float)S);
    for(uint32_t i = 0; i < S; ++i)
    {
        uint32_t xi = i % SQ, yi = i / SQ;
        float x = (xi + lcg_float(&seed)) / sqrt_samples;
        float y = (yi + lcg_float(&seed)) / sqrt_samples;
        dirs[i] = uniform_hemisphere(x, y);
    }
    float pdf = 1.0f / (2.0f * REF_PI);
    for(uint32_t y = 0; y < R; ++y)
        for(uint32_t x = 0; x < R; ++x)
        {
            uint32_t idx = y * R + x;
            float tx = (float)x / (R - 1), ty = (float)y / (R - 1);
            v3 n = parabolic_to_cartesian(2.0f * tx - 1.0f, 2.0f * ty - 1.0f);
            if(n.z <= 0.0f)
            {
                ndf[idx] = 0.0f;
                continue;
            }
            float total = 0.0f;
            for(uint32_t s = 0; s < S; ++s)
            {
                v3 out = reflect(dirs[s], n);
                total += svfo_sample_lum(mesh, &dirs[s].x, &out.x, lum);
            }
            ndf[idx] = total / ((float)S * pdf);
        }
    free(dirs);
}

/* Texture::sample bilinear (texture.hh:483-520) with FastFloorToInt64
 * (functions.hh:82-88) and Modulo (:547-550), on the 64x64 NDF. */
float svfo_ndf_sample(const float* ndf, float tcx, float tcy)
{
    const int64_t W = 64, H = 64;
    float ux = W * tcx - 0.5f, uy = H * tcy - 0.5f;
    int64_t xt = (int64_t)ux - (int64_t)(signbit(ux) ? 1 : 0);
    int64_t yt = (int64_t)uy - (int64_t)(signbit(uy) ? 1 : 0);
    int64_t x0 = ((xt % W) + W) % W, y0 = ((yt % H) + H) % H;
    int64_t x1 = (x0 + 1) % W, y1 = (y0 + 1) % H;
    float c00 = ndf[y0 * W + x0], c01 = ndf[y0 * W + x1], c10 = ndf[y1 * W + x0], c11 = ndf[y1 * W + x1];
    float fx1 = ux - (float)xt, fx0 = 1.0f - fx1, fy1 = uy - (float)yt, fy0 = 1.0f - fy1;
    return (fx0 * c00 + fx1 * c01) * fy0 + (fx0 * c10 + fx1 * c11) * fy1;
}

/* CartesianToParabolicMapCoordinates (vector3.hh:400-403) then SampleRed */
static inline float ndf_at(const float* ndf, v3 n)
{
    float tx = n.x / (n.z + 1.0f) * 0.5f + 0.5f;
    float ty = n.y / (n.z + 1.0f) * 0.5f + 0.5f;
    return svfo_ndf_sample(ndf, tx, ty);
}

/* PCAIntegrand, pipeline.cc:161-173 */
static inline float pca_integrand(const float* ndf, v3 n)
{
    if(n.z < 0.0f)
        return 0.0f;
    return ndf_at(ndf, n);
}

void svfo_decompose(const float* b, float* scaling, float* euler)
{
    /* Matrix3::decompose, matrix3.hh:302-333; b is column-major */
    m3 m;
    memcpy(&m, b, sizeof(m));
    v3 s = v3make(v3len(m.c[0]), v3len(m.c[1]), v3len(m.c[2]));
    scaling[0] = s.x;
    scaling[1] = s.y;
    scaling[2] = s.z;
    float m20 = elem(&m, 2, 0) / s.z;
    if(m20 >= 0.9999f)
    {
        euler[0] = 0.0f;
        euler[1] = REF_PI * 0.5f;
        euler[2] = atan2f(elem(&m, 0, 1), elem(&m, 1, 1));
    }
    else if(m20 <= -0.9999f)
    {
        euler[0] = 0.0f;
        euler[1] = -REF_PI * 0.5f;
        euler[2] = atan2f(elem(&m, 0, 1), elem(&m, 1, 1));
    }
    else
    {
        euler[0] = atan2f(-elem(&m, 2, 1), elem(&m, 2, 2));
        euler[1] = asinf(m20);
        euler[2] = atan2f(-elem(&m, 1, 0) / s.y, elem(&m, 0, 0) / s.x);
    }
}

void svfo_euler_to_matrix(const float* euler3, float* matrix9, float* quat4)
{
    float q[4];
    euler_to_quat(euler3, q);
    m3 m = quat_to_matrix(q);
    if(matrix9)
        memcpy(matrix9, &m, sizeof(m));
    if(quat4)
        memcpy(quat4, q, sizeof(q));
}

void svfo_default_init_from_ndf(const float* ndf, float* init7, svfo_init_info* info)
{
    /* svbrdf-fitting-pipeline.cc:403-406: ndf_denom over 256x256 stratified samples */
    float pdf = 1.0f / (2.0f * REF_PI);
    float ndf_denom;
    {
        unsigned seed = 1;
        const uint32_t S = 256 * 256, SQ = 256;
        float sq = sqrtf((float)S);
        float total = 0.0f;
        for(uint32_t i = 0; i < S; ++i)
        {
            uint32_t xi = i % SQ, yi = i / SQ;
            float x = (xi + lcg_float(&seed)) / sq;
            float y = (yi + lcg_float(&seed)) / sq;
            total += ndf_at(ndf, uniform_hemisphere(x, y));
        }
        ndf_denom = total / ((float)S * pdf);
    }
    float ndf_norm = 1 / ndf_denom;

    /* PCAHemisphere normal search, pipeline.cc:429-489 (one worker, index order) */
    v3 best_n = v3make(0.0f, 0.0f, 1.0f);
    float best_v = pca_integrand(ndf, best_n);
    {
        unsigned seed = 1;
        const uint32_t SQ = 512;
        float sq = sqrtf((float)(SQ * SQ));
        for(uint32_t idx = 0; idx < SQ * SQ; ++idx)
        {
            uint32_t x = idx % SQ, y = idx / SQ;
            float xr = (x + lcg_float(&seed)) / sq;
            float yr = (y + lcg_float(&seed)) / sq;
            v3 n = uniform_hemisphere(xr, yr);
            float v = pca_integrand(ndf, n);
            if(v > best_v)
            {
                best_n = n;
                best_v = v;
            }
        }
    }

    /* tangent search, pipeline.cc:604-628, Matrix3::makeBasis (matrix3.hh:99-108),
     * Matrix2::rotation (matrix2.hh:66-73), rotateTangentPlane (matrix3.hh:133-137) */
    v3 c0, c1;
    {
        v3 d0 = v3cross(v3make(1.0f, 0.0f, 0.0f), best_n);
        v3 d1 = v3cross(v3make(0.0f, 1.0f, 0.0f), best_n);
        float l0 = v3dot(d0, d0), l1 = v3dot(d1, d1);
        c0 = l0 > l1 ? v3div(d0, sqrtf(l0)) : v3div(d1, sqrtf(l1));
        c1 = v3cross(best_n, c0);
    }
    float rs, rc;
    sincos_tan(2.0f * REF_PI / (512 - 1), &rs, &rc);
    float tan_v = 0.0f;
    v3 best_t = v3make(1.0f, 0.0f, 0.0f);
    for(uint32_t k = 0; k < 512; ++k)
    {
        float v = pca_integrand(ndf, c0);
        if(v > tan_v)
        {
            best_t = c0;
            tan_v = v;
        }
        c0 = v3add(v3scale(c0, rc), v3scale(c1, rs));
        c1 = v3add(v3scale(c0, -rs), v3scale(c1, rc));
    }
    v3 t = v3cross(best_t, best_n);
    m3 B;
    B.c[0] = t;
    B.c[1] = best_t;
    B.c[2] = best_n;

    /* SGGX projection, pipeline.cc:639 (SGGXProjectIntegrand :175-189) via
     * ParallelStratifiedMonteCarloIntegratorHemisphere (numerical-methods.hh:261-304),
     * one worker, 1024 samples */
    v3 sig;
    {
        unsigned seed = 1;
        const uint32_t S = 1024, SQ = 32;
        float sq = sqrtf((float)S);
        v3 total = v3make(0.0f, 0.0f, 0.0f);
        for(uint32_t idx = 0; idx < S; ++idx)
        {
            uint32_t x = idx % SQ, y = idx / SQ;
            float xf = (x + lcg_float(&seed)) / sq;
            float yf = (y + lcg_float(&seed)) / sq;
            v3 n = uniform_hemisphere(xf, yf);
            v3 f;
            if(n.z <= 0.0f)
                f = v3make(0.0f, 0.0f, 0.0f);
            else
            {
                v3 r = m3_rot_inverse(&B, n);
                f = v3scale(v3make(fabsf(r.x), fabsf(r.y), fabsf(r.z)), ndf_at(ndf, n));
            }
            total = v3add(total, f);
        }
        float denom = (float)S * pdf;
        /* Vector3 / float multiplies by the reciprocal (vector3.hh:185-190) */
        sig = v3scale(v3div(total, denom), ndf_norm);
    }

    float scaling[3], euler[3];
    svfo_decompose(&B.c[0].x, scaling, euler);
    init7[0] = sig.x / sig.z;
    init7[1] = sig.y / sig.z;
    init7[2] = ndf_denom;
    init7[3] = 0.0f;
    init7[4] = euler[0];
    init7[5] = euler[1];
    init7[6] = euler[2];
    if(info)
    {
        info->ndf_denom = ndf_denom;
        memcpy(info->normal, &best_n, sizeof(v3));
        memcpy(info->tangent, &best_t, sizeof(v3));
        memcpy(info->basis, &B, sizeof(B));
        memcpy(info->sggx_stddev, &sig, sizeof(v3));
    }
}

/* ---------------------------------------------------------------------------
 * Synthetic texels
 * ------------------------------------------------------------------------- */

void svfo_philox4x32(const uint32_t key_in[2], const uint32_t ctr_in[4], uint32_t out[4])
{
    uint32_t k0 = key_in[0], k1 = key_in[1];
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    for(int r = 0; r < 10; ++r)
    {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static inline float u01(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }
static inline float loguniform(float a, float b, float u) { return a * expf(u * logf(b / a)); }

static void draw(uint32_t seed, uint64_t texel, uint32_t block, uint32_t out[4])
{
    uint32_t key[2] = { seed, 0x53564631u };
    uint32_t ctr[4] = { (uint32_t)texel, (uint32_t)(texel >> 32), block, 0u };
    svfo_philox4x32(key, ctr, out);
}

void svfo_synth_truth(uint32_t seed, uint32_t mix, uint64_t texel, svfo_texel_truth* t)
{
    uint32_t b0[4], b1[4], b2[4];
    draw(seed, texel, 0, b0);
    draw(seed, texel, 1, b1);
    draw(seed, texel, 2, b2);
    float uk = u01(b0[0]);
    uint32_t kind = 0;
    if(mix == 1)
        kind = uk < 0.2f ? 1u : (uk < 0.3f ? 2u : 0u);
    t->kind = kind;
    for(int c = 0; c < 3; ++c)
        t->kd[c] = 0.8f * u01(b0[1 + c]);
    for(int c = 0; c < 3; ++c)
        t->ks[c] = (kind == 1 ? 0.05f : 1.0f) * u01(b1[c]);
    if(kind == 2)
    {
        float smin = loguniform(0.01f, 0.05f, u01(b1[3]));
        float ratio = loguniform(8.5f, 16.0f, u01(b2[0]));
        float smax = smin * ratio;
        t->sigma[0] = smax < 0.8f ? smax : 0.8f;
        t->sigma[1] = smin;
    }
    else
    {
        t->sigma[0] = loguniform(0.02f, 0.8f, u01(b1[3]));
        t->sigma[1] = loguniform(0.02f, 0.8f, u01(b2[0]));
    }
    /* orientation: normal uniform on the spherical cap within 30 degrees of +z,
     * tangent uniform around it */
    const float cos30 = 0.866025403784f;
    const float two_pi = 6.283185307179586f;
    float nz = 1.0f - u01(b2[1]) * (1.0f - cos30);
    float nr = sqrtf(fmaxf(0.0f, 1.0f - nz * nz));
    float phi = two_pi * u01(b2[2]);
    float psi = two_pi * u01(b2[3]);
    v3 n = v3make(nr * cosf(phi), nr * sinf(phi), nz);
    /* reference tangent: x axis projected on the tangent plane */
    v3 t0 = v3normalize(v3sub(v3make(1.0f, 0.0f, 0.0f), v3scale(n, n.x)));
    v3 b0v = v3cross(n, t0);
    v3 tt = v3add(v3scale(t0, cosf(psi)), v3scale(b0v, sinf(psi)));
    v3 bb = v3cross(n, tt);
    /* rotation matrix columns (tt, bb, n) -> quaternion (x, y, z, w) for the
     * matrix convention of ToMatrix3 (quaternion.hh:122-139) */
    float m00 = tt.x, m01 = tt.y, m02 = tt.z;   /* column 0 */
    float m10 = bb.x, m11 = bb.y, m12 = bb.z;   /* column 1 */
    float m20 = n.x, m21 = n.y, m22 = n.z;      /* column 2 */
    float q[4];
    float tr = m00 + m11 + m22;
    if(tr > 0.0f)
    {
        float s = sqrtf(tr + 1.0f) * 2.0f;
        q[3] = 0.25f * s;
        q[0] = (m12 - m21) / s;
        q[1] = (m20 - m02) / s;
        q[2] = (m01 - m10) / s;
    }
    else if(m00 > m11 && m00 > m22)
    {
        float s = sqrtf(1.0f + m00 - m11 - m22) * 2.0f;
        q[3] = (m12 - m21) / s;
        q[0] = 0.25f * s;
        q[1] = (m01 + m10) / s;
        q[2] = (m02 + m20) / s;
    }
    else if(m11 > m22)
    {
        float s = sqrtf(1.0f + m11 - m00 - m22) * 2.0f;
        q[3] = (m20 - m02) / s;
        q[0] = (m01 + m10) / s;
        q[1] = 0.25f * s;
        q[2] = (m12 + m21) / s;
    }
    else
    {
        float s = sqrtf(1.0f + m22 - m00 - m11) * 2.0f;
        q[3] = (m01 - m10) / s;
        q[0] = (m02 + m20) / s;
        q[1] = (m12 + m21) / s;
        q[2] = 0.25f * s;
    }
    float ql = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for(int i = 0; i < 4; ++i)
        t->quat[i] = q[i] / ql;
    m3 R = quat_to_matrix(t->quat);
    float scaling[3];
    svfo_decompose(&R.c[0].x, scaling, t->euler);
}

void svfo_synth_render(uint32_t seed, uint64_t texel, const svfo_texel_truth* t, const float* lp, uint32_t L, float noise, float* rgb)
{
    m3 R = quat_to_matrix(t->quat);
    v3 stddev = v3make(t->sigma[0], t->sigma[1], 1.0f);
    for(uint32_t v = 0; v < L; ++v)
    {
        v3 wo = parabolic_to_cartesian(lp[2 * v], lp[2 * v + 1]);
        float out_density = sggx_projected_area(stddev, &R, wo);
        for(uint32_t l = 0; l < L; ++l)
        {
            v3 wi = parabolic_to_cartesian(lp[2 * l], lp[2 * l + 1]);
            uint32_t lv = v * L + l;
            uint32_t r[4];
            draw(seed, texel, 16u + lv, r);
            float z[4];
            for(int k = 0; k < 2; ++k)
            {
                float ua = ((r[2 * k] >> 8) + 1u) * (1.0f / 16777216.0f);
                float ub = u01(r[2 * k + 1]);
                float rad = sqrtf(-2.0f * logf(ua));
                z[2 * k] = rad * cosf(6.283185307179586f * ub);
                z[2 * k + 1] = rad * sinf(6.283185307179586f * ub);
            }
            for(int c = 0; c < 3; ++c)
            {
                float f = surface_brdf(t->kd[c], t->ks[c], stddev, &R, out_density, wi, wo, 1.0f);
                rgb[3 * lv + c] = f * (1.0f + noise * z[c]);
            }
        }
    }
}

/* ---------------------------------------------------------------------------
 * Factored BTF decode
 * ------------------------------------------------------------------------- */

/* IEEE binary16 -> float (exact) */
static float half_to_float(uint16_t h)
{
    uint32_t sign = (uint32_t)(h >> 15) << 31, e = (h >> 10) & 0x1f, m = h & 0x3ff, bits;
    if(e == 0)
    {
        if(m == 0)
            bits = sign;
        else
        {
            /* subnormal: m * 2^-24 */
            float f = (float)m * (1.0f / 16777216.0f);
            return sign ? -f : f;
        }
    }
    else if(e == 31)
        bits = sign | 0x7f800000u | (m << 13);
    else
        bits = sign | ((e + 112u) << 23) | (m << 13);
    float f;
    memcpy(&f, &bits, 4);
    return f;
}

static double plane_elem(const void* base, uint32_t data_size, uint64_t i)
{
    switch(data_size)
    {
    case 2: return half_to_float(((const uint16_t*)base)[i]);
    case 4: return ((const float*)base)[i];
    default: return ((const double*)base)[i];
    }
}

void svfo_btf_decode(const svfo_btf_planes* p, uint64_t first, uint64_t count, float* out)
{
    const uint32_t L = p->light_count, N = L * L, W = p->width, H = p->height;
    const float drr_eps = 1e-5f;
    for(uint64_t t = first; t < first + count; ++t)
    {
        const uint64_t y = t / W, x = t % W, col = (H - 1 - y) * (uint64_t)W + x;
        for(uint32_t lv = 0; lv < N; ++lv)
        {
            float c[3];
            for(int ch = 0; ch < 3; ++ch)
            {
                /* BTFEvaluateMatrix<T, TOp>: TOp sum{}; sum += u*v (btf.hh:627-632) */
                if(p->data_size == 8)
                {
                    double sum = 0.0;
                    for(uint32_t k = 0; k < p->k[ch]; ++k)
                        sum += plane_elem(p->u[ch], 8, lv * p->u_row[ch] + k) *
                               plane_elem(p->sxv[ch], 8, col * p->sxv_row[ch] + k);
                    c[ch] = (float)sum;
                }
                else
                {
                    float sum = 0.0f;
                    for(uint32_t k = 0; k < p->k[ch]; ++k)
                    {
                        float u = (float)plane_elem(p->u[ch], p->data_size, lv * p->u_row[ch] + k);
                        float v = (float)plane_elem(p->sxv[ch], p->data_size, col * p->sxv_row[ch] + k);
                        float uv = u * v;
                        sum += uv;
                    }
                    c[ch] = sum;
                }
            }
            if(p->color_model == 11)
            {
                /* btf.hh:522-531, YUVToRGB spectrum.hh:344-350 */
                float Y = expf(c[0]) - drr_eps;
                float U = c[1] * Y + drr_eps;
                float V = c[2] * Y + drr_eps;
                float r = Y * 1.0f + U * 0.0f + V * 1.13983f;
                float g = Y * 1.0f + U * -0.39465f + V * -0.5806f;
                float b = Y * 1.0f + U * 2.03211f + V * 0.0f;
                /* Vector3Clamp -> Clamp (functions.hh:156-159) */
                c[0] = r <= 0.0f ? 0.0f : (r >= 1.0f ? 1.0f : r);
                c[1] = g <= 0.0f ? 0.0f : (g >= 1.0f ? 1.0f : g);
                c[2] = b <= 0.0f ? 0.0f : (b >= 1.0f ? 1.0f : b);
            }
            if(p->drr)
                for(int ch = 0; ch < 3; ++ch)
                    c[ch] = expf(c[ch]) - drr_eps;
            float* o = out + ((t - first) * N + lv) * 3;
            o[0] = c[0];
            o[1] = c[1];
            o[2] = c[2];
        }
    }
}
