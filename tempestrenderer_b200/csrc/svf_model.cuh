// svf_model.cuh - the SGGX surface BRDF of the fit, factored for the GPU.
//
// Model (BRDFEvaluator, tools/svbrdf-fitting/svbrdf-lsq-fitting-internal.hh:91-153,
// over SGGXMicroFlakeSurfaceBRDF, include/tempest/graphics/ray-tracing/
// ggx-models-impl.hh:476-552), for parameters p = {sx, sy, ks, kd, e0, e1, e2}:
//
//   f(i, o) = kd c_i / pi + ks F D(h) / (2 (sigma(o) + sigma(i) c_o / c_i))
//   D(h)     = 1 / (2 pi sx sy (h^T S^-1 h)^2)          (ggx-models-impl.hh:49-57)
//   sigma(w) = |diag(sx, sy, 1) R^T w|                   (ggx-models-impl.hh:102-105)
//   S^-1     = R diag(1/sx^2, 1/sy^2, 1) R^T,  R = ToMatrix3(ToQuaternion(e))
//
// with c = w.z, h = (w_i + w_o)/|w_i + w_o|, pi = 3.141592f (functions.hh:55)
// and the reference's clamps: sx, sy, ks, kd are clamped at 0; the specular
// lobe is dropped when sx or sy < 1e-6, when sigma(o) < 1e-6, or when
// det S^-1 < 1e-6.
//
// Factored form used by the kernels.  With a_d = R^T w_d per direction d,
// s = a_i + a_o, W = w_i + w_o, g = |W|^2, sp_d = sigma(d)/c_d:
//
//   h^T S^-1 h = Q / g,  Q = s_x^2/sx^2 + s_y^2/sy^2 + s_z^2
//   f = kd c_i/pi + ks * K / c_o * g^2 / (Q^2 (sp_i + sp_o)),  K = F / (4 pi sx sy)
//
// so that everything that depends on one direction only (a_d, sp_d and their
// parameter derivatives) is tabulated once per parameter set, and a pair costs
// a few fused multiply-adds and one reciprocal.  The Euler-angle derivatives
// use the body-frame angular velocity w_k of R (R^T dR/de_k = [w_k]x):
// d a_d / d e_k = a_d x w_k, and dQ/de_k = 2 w_k . ((L^-1 s) x s) with
// L^-1 = diag(1/sx^2, 1/sy^2, 1).
#pragma once

#include <math.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define SVF_HD __host__ __device__ __forceinline__
#else
#define SVF_HD inline
#endif

namespace svf
{

constexpr float kRefPi = 3.141592f;   // the reference's pi (functions.hh:55)
constexpr int kParams = 7;
constexpr int kHessian = 28;          // packed upper triangle of the 7x7 J^T J

// Quantities derived from one parameter vector, shared by all pairs.
struct ParamSet
{
    float sx, sy, ks, kd;   // clamped parameters
    float ks_on, kd_on;     // 1 where the unclamped albedo is >= 0 (derivative mask)
    float R[9];             // ToMatrix3: column c is R[3c..3c+2]
    float om[3][3];         // body-frame angular velocity of R per Euler angle
    float u, v;             // 1/sx^2, 1/sy^2
    float rsx, rsy;         // 1/sx, 1/sy
    float kspec;            // F-free lobe constant 1/(4 pi sx sy), 0 when the lobe is off
};

// Reciprocal for the table set-up: the device's fast division (about 2 ulp;
// the table terms need no correctly rounded divide), IEEE on the host.
SVF_HD float rcp_model(float x)
{
#if defined(__CUDA_ARCH__)
    return __fdividef(1.0f, x);
#else
    return 1.0f / x;
#endif
}

SVF_HD void sincos_f(float x, float* s, float* c)
{
#if defined(__CUDA_ARCH__)
    sincosf(x, s, c);
#else
    *s = sinf(x);
    *c = cosf(x);
#endif
}

SVF_HD void finish_param_set(ParamSet& ps);

// ToQuaternion(euler) (include/tempest/math/quaternion.hh:82-94), then
// ToMatrix3 (quaternion.hh:122-139) and the body rates R^T dR/de_k in closed form.
SVF_HD void make_param_set(const float* p, ParamSet& ps)
{
    ps.sx = p[0] > 0.0f ? p[0] : 0.0f;
    ps.sy = p[1] > 0.0f ? p[1] : 0.0f;
    ps.ks = p[2] > 0.0f ? p[2] : 0.0f;
    ps.kd = p[3] > 0.0f ? p[3] : 0.0f;
    // Derivative masks of the clamped albedos: the step constraint keeps them
    // >= 0 (AcceptStepConstraints), so at exactly 0 the right derivative applies
    // (the default initial guess starts with diffuse = 0, pipeline.cc:659); the
    // LM's active-set rule holds a parameter at 0 when its step points below it.
    ps.ks_on = p[2] >= 0.0f ? 1.0f : 0.0f;
    ps.kd_on = p[3] >= 0.0f ? 1.0f : 0.0f;

    float s1, c1, s2, c2, s3, c3;
    sincos_f(0.5f * p[4], &s1, &c1);
    sincos_f(0.5f * p[5], &s2, &c2);
    sincos_f(0.5f * p[6], &s3, &c3);
    float q[4] = { s1 * c2 * c3 + c1 * s2 * s3, -s1 * c2 * s3 + c1 * s2 * c3,
                   c1 * c2 * s3 + s1 * s2 * c3, c1 * c2 * c3 - s1 * s2 * s3 };
    // the lobe uses ToMatrix3(Normalize(q)) (ggx-models-impl.hh:520)
    float ql = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    float rq = rcp_model(ql);
    float x = q[0] * rq, y = q[1] * rq, z = q[2] * rq, w = q[3] * rq;
    float* R = ps.R;
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + z * w);        R[2] = 2.0f * (x * z - y * w);
    R[3] = 2.0f * (x * y - z * w);        R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + x * w);
    R[6] = 2.0f * (x * z + y * w);        R[7] = 2.0f * (y * z - x * w);        R[8] = 1.0f - 2.0f * (x * x + y * y);
    // q = qx(e0) qy(e1) qz(e2), so R = Rx(e0) Ry(e1) Rz(e2) and the body-frame
    // angular velocities (R^T dR/de_k = [w_k]x) are w_2 = z, w_1 = Rz^T y and
    // w_0 = (Ry Rz)^T x, from the half-angle sines and cosines already at hand.
    const float sb = 2.0f * s2 * c2, cb = (c2 - s2) * (c2 + s2);   // sin, cos of e1
    const float sc = 2.0f * s3 * c3, cc = (c3 - s3) * (c3 + s3);   // sin, cos of e2
    ps.om[0][0] = cc * cb;
    ps.om[0][1] = -sc * cb;
    ps.om[0][2] = sb;
    ps.om[1][0] = sc;
    ps.om[1][1] = cc;
    ps.om[1][2] = 0.0f;
    ps.om[2][0] = 0.0f;
    ps.om[2][1] = 0.0f;
    ps.om[2][2] = 1.0f;

    finish_param_set(ps);
}

// The lobe constants of a parameter set whose sx, sy are set.
SVF_HD void finish_param_set(ParamSet& ps)
{
    bool lobe = ps.sx >= 1e-6f && ps.sy >= 1e-6f;
    float rsx = lobe ? rcp_model(ps.sx) : 0.0f;
    float rsy = lobe ? rcp_model(ps.sy) : 0.0f;
    float u = rsx * rsx;
    float v = rsy * rsy;
    // det S^-1 = u v (ggx-models-impl.hh:53-54 drops the lobe below 1e-6)
    lobe = lobe && (u * v >= 1e-6f);
    ps.u = u;
    ps.v = v;
    ps.rsx = lobe ? rsx : 0.0f;
    ps.rsy = lobe ? rsy : 0.0f;
    ps.kspec = lobe ? (0.25f / kRefPi) * rsx * rsy : 0.0f;
}

// RGB mode (11 parameters): p = {kd rgb, ks rgb, sx, sy, quaternion xyzw}.
// The orientation is the quaternion; its LM parameters are a rotation phi in
// the body frame, R(phi) = R Exp([phi]x), evaluated at phi = 0, so the body
// angular velocity of parameter k is the unit vector e_k.  Only the geometry
// (R, sigma and the lobe constants) goes into the table; the albedos enter per
// channel in the pair pass.
SVF_HD void make_param_set_rgb(const float* p, ParamSet& ps)
{
    ps.sx = p[6] > 0.0f ? p[6] : 0.0f;
    ps.sy = p[7] > 0.0f ? p[7] : 0.0f;
    ps.ks = ps.kd = 1.0f;
    ps.ks_on = ps.kd_on = 1.0f;
    float ql = sqrtf(p[8] * p[8] + p[9] * p[9] + p[10] * p[10] + p[11] * p[11]);
    float rq = ql > 0.0f ? rcp_model(ql) : 0.0f;
    float x = p[8] * rq, y = p[9] * rq, z = p[10] * rq, w = ql > 0.0f ? p[11] * rq : 1.0f;
    float* R = ps.R;
    R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + z * w);        R[2] = 2.0f * (x * z - y * w);
    R[3] = 2.0f * (x * y - z * w);        R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + x * w);
    R[6] = 2.0f * (x * z + y * w);        R[7] = 2.0f * (y * z - x * w);        R[8] = 1.0f - 2.0f * (x * x + y * y);
    for(int k = 0; k < 3; ++k)
        for(int j = 0; j < 3; ++j)
            ps.om[k][j] = k == j ? 1.0f : 0.0f;
    finish_param_set(ps);
}

// Per-direction table entry for one parameter set.
struct DirEntry
{
    float a[3];     // R^T w
    float sp;       // sigma(w) / c
    float dsp[5];   // d sp / d{sx, sy, e0, e1, e2}
    float kdc;      // c / pi when the direction is in the upper hemisphere, else 0 (light role)
    float kv;       // 1/c when sigma(w) >= 1e-6 and c > 0, else 0 (view role, times kspec)
    float up;       // 1 when c > 0, else 0: a pair with either direction below the horizon is 0
};

SVF_HD void make_dir_entry(const ParamSet& ps, float wx, float wy, float wz, DirEntry& e)
{
    const float* R = ps.R;
    float a0 = R[0] * wx + R[1] * wy + R[2] * wz;
    float a1 = R[3] * wx + R[4] * wy + R[5] * wz;
    float a2 = R[6] * wx + R[7] * wy + R[8] * wz;
    e.a[0] = a0;
    e.a[1] = a1;
    e.a[2] = a2;
    float sx2 = ps.sx * ps.sx, sy2 = ps.sy * ps.sy;
    float sig2 = sx2 * a0 * a0 + sy2 * a1 * a1 + a2 * a2;
#if defined(__CUDA_ARCH__)
    float rsig = sig2 > 0.0f ? rsqrtf(sig2) : 0.0f;
    float sig = sig2 * rsig;
#else
    float sig = sqrtf(sig2);
    float rsig = sig > 0.0f ? 1.0f / sig : 0.0f;
#endif
    bool up = wz > 0.0f;
    float c = up ? wz : 1.0f;
    float rc = rcp_model(c);
    e.kdc = up ? wz * (1.0f / kRefPi) : 0.0f;
    e.kv = (up && sig >= 1e-6f) ? rc : 0.0f;
    e.up = up ? 1.0f : 0.0f;
    e.sp = sig * rc;
    float k = rsig * rc;
    e.dsp[0] = ps.sx * a0 * a0 * k;
    e.dsp[1] = ps.sy * a1 * a1 * k;
    for(int j = 0; j < 3; ++j)
    {
        const float* om = ps.om[j];
        // d a / d e_j = a x om
        float d0 = a1 * om[2] - a2 * om[1];
        float d1 = a2 * om[0] - a0 * om[2];
        float d2 = a0 * om[1] - a1 * om[0];
        e.dsp[2 + j] = (sx2 * a0 * d0 + sy2 * a1 * d1 + a2 * d2) * k;
    }
}

// One pair: f and the gradient of f (not of the residual) with respect to p.
// wi/wo are the directions, li/vo the table entries in light and view roles.
template <bool kJacobian>
SVF_HD float eval_pair(const ParamSet& ps, const float* wi, const DirEntry& li, const float* wo, const DirEntry& vo,
                       float fresnel_factor, float* J)
{
    float W0 = wi[0] + wo[0], W1 = wi[1] + wo[1], W2 = wi[2] + wo[2];
    float g = W0 * W0 + W1 * W1 + W2 * W2;
    float s0 = li.a[0] + vo.a[0], s1 = li.a[1] + vo.a[1], s2 = li.a[2] + vo.a[2];
    float q0 = s0 * s0, q1 = s1 * s1;
    float Q = ps.u * q0 + ps.v * q1 + s2 * s2;
    float S = li.sp + vo.sp;
    float QQS = Q * Q * S;
    float rden = QQS > 0.0f ? 1.0f / QQS : 0.0f;
    // the pair vanishes unless both directions are above the horizon
    // (ggx-models-impl.hh:484-485); vo.kv is already 0 for a view below it
    float kk = ps.kspec * vo.kv * li.up * fresnel_factor;
    float spec = kk * g * g * rden;
    float f = vo.up * (ps.kd * li.kdc) + ps.ks * spec;
    if(kJacobian)
    {
        float A = ps.ks * spec;
        float rQ = Q * S * rden;           // 1/Q
        float rS = Q * Q * rden;           // 1/S
        // t = (L^-1 s) x s
        float t0 = s1 * s2 * (ps.v - 1.0f);
        float t1 = s0 * s2 * (1.0f - ps.u);
        float t2 = s0 * s1 * (ps.u - ps.v);
        J[0] = A * (ps.rsx * (4.0f * ps.u * q0 * rQ - 1.0f) - (li.dsp[0] + vo.dsp[0]) * rS);
        J[1] = A * (ps.rsy * (4.0f * ps.v * q1 * rQ - 1.0f) - (li.dsp[1] + vo.dsp[1]) * rS);
        J[2] = ps.ks_on * spec;
        J[3] = ps.kd_on * vo.up * li.kdc;
        float m4 = -4.0f * rQ;
        for(int k = 0; k < 3; ++k)
        {
            const float* om = ps.om[k];
            float dq = om[0] * t0 + om[1] * t1 + om[2] * t2;
            J[4 + k] = A * (m4 * dq - (li.dsp[2 + k] + vo.dsp[2 + k]) * rS);
        }
    }
    return f;
}

// Fresnel factor F(cos(h, w_i)) for refractive index `refr` != 1 (CosTransmittance
// and FresnelDielectric, include/tempest/math/functions.hh:265-268,296-301, clamped
// to [0, 1] as ggx-models-impl.hh:534-535 does).
SVF_HD float fresnel_factor(float refr, const float* wi, const float* wo)
{
    if(refr == 1.0f)
        return 1.0f;
    float W0 = wi[0] + wo[0], W1 = wi[1] + wo[1], W2 = wi[2] + wo[2];
    float rl = 1.0f / sqrtf(W0 * W0 + W1 * W1 + W2 * W2);
    float cm = (W0 * wi[0] + W1 * wi[1] + W2 * wi[2]) * rl;
    float ct = sqrtf(1.0f - (1.0f - cm * cm) / (refr * refr));
    float rp = (refr * cm - ct) / (refr * cm + ct);
    float rs = (cm - refr * ct) / (cm + refr * ct);
    float fr = 0.5f * (rp * rp + rs * rs);
    return fr < 0.0f ? 0.0f : (fr > 1.0f ? 1.0f : fr);
}

// ParabolicToCartesianCoordinates (include/tempest/math/vector3.hh:389-393).
SVF_HD void parabolic_to_cartesian(float px, float py, float* w)
{
    float len_sq = px * px + py * py;
    w[0] = 2.0f * px / (len_sq + 1.0f);
    w[1] = 2.0f * py / (len_sq + 1.0f);
    w[2] = (1 - len_sq) / (1 + len_sq);
}

// Index into the packed upper triangle of a 7x7 symmetric matrix.
SVF_HD int hidx(int i, int j)
{
    return i <= j ? i * kParams - (i * (i - 1)) / 2 + (j - i) : j * kParams - (j * (j - 1)) / 2 + (i - j);
}

} // namespace svf
