// svf_lm.cu - the persistent Levenberg-Marquardt fit (LeastSquaresFitSGGX,
// tools/svbrdf-fitting/svbrdf-lsq-fitting-setup.cc:234-431, over
// LevenbergMarquardtCurveFit, include/tempest/math/fitting.hh:457-678) for sm_100a.
//
// Work distribution: a persistent grid of (resident CTAs per SM) x (SMs) CTAs
// pulls texels from a global atomic counter (work stealing: a texel that
// converges early frees its slot at once).  Each CTA is warp-specialised and
// keeps S texels ("slots") in flight:
//
//   warp 0, the control warp: per slot, the FP64 LM control (thread 0; state in
//     shared memory), the direction table for the next evaluation (all 32
//     lanes), the texel's
//     outputs and the bulk TMA copy (cp.async.bulk, mbarrier, bounded wait) of
//     the next texel's luminance slab into the slot;
//   warps 1..NW, the pair workers: the pair passes of slot 0, 1, .., S-1, 0, ..
//     in turn; the last worker warp to finish a pass sums the warps' partials
//     in FP64, in warp order.
//
// Named barriers hand each slot back and forth: READY[s] (control -> workers:
// the command, table and constants of slot s are in place) and DONE[s]
// (workers -> control: the per-warp partial sums are written).  While the
// control warp solves the damped normal equations of one slot, the workers
// evaluate another slot's pairs, so the serial FP64 work is off the pair
// throughput's critical path.
//
// A pass evaluates nothing per pair that depends on one direction only: the
// table (svf_model.cuh) holds 12 floats per direction.  The workers walk the
// L (L + 1) / 2 unordered direction pairs, one per lane, and evaluate the
// specular core once for both ordered pairs (sym_pair).  Every pass evaluates
// the residual and the Jacobian (a trial point's Jacobian is the next one when
// the step is accepted, and most are) and accumulates the packed J^T J and J^T r in FP32 per lane and r^2 in FP64,
// reduce them within the warp (reduce-scatter), and the control warp sums the
// warps in FP64.  The LM control follows fitting.hh: the damped normal
// equations by Cholesky, the small-step and gradient tests and the gain-ratio
// accept/reject.
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

constexpr int kEntry = 12;                   // floats per direction-table entry
constexpr uint32_t kWaitSpins = 1u << 22;    // bound of every mbarrier wait

// Packed upper triangle of a symmetric P x P matrix.
template <int P>
__host__ __device__ constexpr int hix(int i, int j)
{
    return i <= j ? i * P - (i * (i - 1)) / 2 + (j - i) : j * P - (j * (j - 1)) / 2 + (i - j);
}

// The two fits.  Luminance (the reference's LeastSquaresFitSGGX): 7 parameters
// {sx, sy, ks, kd, euler xyz} on the luminance slice.  RGB: 11 parameters
// {kd rgb, ks rgb, sx, sy, rotation phi xyz} on the three channels, the
// orientation kept as a quaternion and updated by the local rotation phi.
// kAcc: FP32 sums per lane of a pass (the RGB pass keeps the channel-factored
// sums; the control warp expands them into J^T J and J^T r).
struct LumModel
{
    static constexpr int P = 7;
    static constexpr int B = 4;          // sx, sy, ks, kd are bounded below by 0
    static constexpr int kAcc = 35;      // J^T J (28) and J^T r (7)
    static constexpr int kChannels = 1;
    static constexpr int kOut = 7;       // floats per texel of initial and fitted parameters
    static constexpr bool kRgb = false;
    using Slab = float;
};

struct RgbModel
{
    static constexpr int P = 11;
    static constexpr int B = 8;          // kd rgb, ks rgb, sx, sy
    static constexpr int kAcc = 39;      // see sym_pair_rgb
    static constexpr int kChannels = 3;
    static constexpr int kOut = 12;      // {kd rgb, ks rgb, sx, sy, quaternion xyzw}
    static constexpr bool kRgb = true;
    using Slab = __half;
};

enum : int
{
    kCmdTrial = 0,
    kCmdJacobian = 1,
    kCmdDone = 2,
    kCmdContinue = 3
};

// ------------------------------------------------------------------------------
// mbarrier + bulk copy (TMA)
// ------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Arms `bar` for `bytes` and starts one bulk copy global -> shared.  dst, src
// 16-byte aligned; bytes a multiple of 16.  The fence orders earlier generic
// reads of the destination before the asynchronous write.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    const uint32_t b = smem_addr(bar);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(b)
                 : "memory");
}

// Bounded wait for phase `parity` of `bar` (at most `spins` polls, 0: the
// default bound); false when the bound expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t spins = 0)
{
    const uint32_t b = smem_addr(bar);
    const uint32_t bound = spins ? spins : kWaitSpins;
    for(uint32_t i = 0; i < bound; ++i)
    {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(b), "r"(parity)
                     : "memory");
        if(done)
            return true;
    }
    return false;
}

// ------------------------------------------------------------------------------
// FP64 LM control (thread 0; the state lives in shared memory)
// ------------------------------------------------------------------------------

template <int P>
struct LmState
{
    double p[P];            // current parameters (RGB: the rotation entries are 0)
    double pt[P];           // trial parameters
    double d[P];            // step
    double g[P];            // gradient J_r^T r of the residual r = y - f
    double H[P * (P + 1) / 2];   // J^T J, packed upper
    double q[4], qt[4];     // RGB: orientation at p and at the trial point (xyzw)
    double S;               // sum of squared residuals at p
    double lam, nu, rho;
    double damp_scale;      // of the initial damping (1: the reference's rule)
    uint32_t iter, eff, njac, nres, status, restarts_left;
    uint32_t fixed;         // parameters held (the reference's fit_params_count below 7 and its
                            // specular-only parameter set): no step, no share in the tests
};

// Fresh damping from the current normal equations (fitting.hh:531-538), times
// the texel's scale (1 unless its segment asks for a lighter start).
template <int P>
__device__ __forceinline__ void lm_reset_damping(LmState<P>& st)
{
    double damping = 1.0;   // InitialMinDamping
#pragma unroll
    for(int i = 0; i < P; ++i)
        if(!(st.fixed & (1u << i)))
            damping = fmax(damping, st.H[hix<P>(i, i)]);
    st.lam = damping * 0.75 * st.damp_scale;   // InitialDampingMultiplier
    st.nu = 2.0;               // DampingFailureMultiplier
}

// Where the reference's loop ends, optionally continue with fresh damping from
// the same point; false when the fit is finished.
template <int P>
__device__ __forceinline__ bool lm_restart(LmState<P>& st, const LmConfig& cfg, double n_pairs)
{
    if(st.restarts_left == 0 || !(st.iter < cfg.max_iter && cfg.mse_target < st.S / n_pairs))
        return false;
    --st.restarts_left;
    lm_reset_damping(st);
    return true;
}

// Damped step (H + lam I) d = g by Cholesky (register-resident, reciprocal
// square roots, no divides).  Active set at the bound: a parameter with a lower
// bound (sigma, specular, diffuse) that sits exactly at 0 and whose step points
// below it is held at 0 for this solve (its row and column are dropped) and the
// system is solved again.  The reference rejects every such step
// (AcceptStepConstraints), which with an exact derivative would hold the
// parameter at 0 for good; its central difference at exactly 0 (fitting.hh:
// 896-905, step 1e-8) is below float resolution there.  False when the
// factorisation fails.
template <int P, int B>
__device__ __noinline__ bool lm_solve(LmState<P>& st)
{
    constexpr int kH = P * (P + 1) / 2;
    uint32_t frozen = st.fixed;
    for(int round = 0; round < 5; ++round)
    {
        double A[kH], x[P];
#pragma unroll
        for(int i = 0; i < kH; ++i)
            A[i] = st.H[i];
#pragma unroll
        for(int i = 0; i < P; ++i)
        {
            A[hix<P>(i, i)] += st.lam;
            x[i] = st.g[i];
        }
#pragma unroll
        for(int i = 0; i < P; ++i)
            if(frozen & (1u << i))
            {
#pragma unroll
                for(int j = 0; j < P; ++j)
                    if(j != i)
                        A[hix<P>(i, j)] = 0.0;
                x[i] = 0.0;
            }
        // A = L L^T; the diagonal keeps 1 / L_jj
        bool ok = true;
#pragma unroll
        for(int j = 0; j < P; ++j)
        {
            double s = A[hix<P>(j, j)];
#pragma unroll
            for(int k = 0; k < j; ++k)
                s -= A[hix<P>(j, k)] * A[hix<P>(j, k)];
            ok = ok && (s > 0.0) && isfinite(s);
            const double r = rsqrt(s);
            A[hix<P>(j, j)] = r;
#pragma unroll
            for(int i = j + 1; i < P; ++i)
            {
                double t = A[hix<P>(i, j)];
#pragma unroll
                for(int k = 0; k < j; ++k)
                    t -= A[hix<P>(i, k)] * A[hix<P>(j, k)];
                A[hix<P>(i, j)] = t * r;
            }
        }
        if(!ok)
            return false;
#pragma unroll
        for(int i = 0; i < P; ++i)
        {
            double t = x[i];
#pragma unroll
            for(int k = 0; k < i; ++k)
                t -= A[hix<P>(i, k)] * x[k];
            x[i] = t * A[hix<P>(i, i)];
        }
#pragma unroll
        for(int i = P - 1; i >= 0; --i)
        {
            double t = x[i];
#pragma unroll
            for(int k = i + 1; k < P; ++k)
                t -= A[hix<P>(k, i)] * x[k];
            x[i] = t * A[hix<P>(i, i)];
        }
        uint32_t more = frozen;
#pragma unroll
        for(int i = 0; i < P; ++i)
        {
            st.d[i] = x[i];
            if(i < B && st.p[i] == 0.0 && x[i] > 0.0)
                more |= 1u << i;
        }
        if(more == frozen)
            return true;
        frozen = more;
    }
    return true;
}

// Top of one LM iteration (fitting.hh:541-590): find a step that passes the
// constraints, or finish.  kCmdTrial (st.pt holds the trial point) or kCmdDone.
// Unit quaternion of the rotation vector phi (Exp([phi]x)), xyzw.
__device__ __forceinline__ void quat_exp(const double* phi, double* q)
{
    const double a2 = phi[0] * phi[0] + phi[1] * phi[1] + phi[2] * phi[2];
    const double a = sqrt(a2);
    const double h = 0.5 * a;
    const double k = a > 1e-12 ? sin(h) / a : 0.5 - a2 / 48.0;
    q[0] = k * phi[0];
    q[1] = k * phi[1];
    q[2] = k * phi[2];
    q[3] = cos(h);
}

// r = a (x) b, Hamilton product, xyzw: the rotation of a followed, in a's body
// frame, by that of b (R(a b) = R(a) R(b)).
__device__ __forceinline__ void quat_mul(const double* a, const double* b, double* r)
{
    r[0] = a[3] * b[0] + a[0] * b[3] + a[1] * b[2] - a[2] * b[1];
    r[1] = a[3] * b[1] - a[0] * b[2] + a[1] * b[3] + a[2] * b[0];
    r[2] = a[3] * b[2] + a[0] * b[1] - a[1] * b[0] + a[2] * b[3];
    r[3] = a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2];
}

template <class M>
__device__ int lm_next(LmState<M::P>& st, const LmConfig& cfg, double n_pairs)
{
    for(;;)
    {
        if(!(st.iter < cfg.max_iter && cfg.mse_target < st.S / n_pairs))
        {
            if(st.iter >= cfg.max_iter)
                st.status |= SVF_TEXEL_MAX_ITER;
            return kCmdDone;
        }
        if(!lm_solve<M::P, M::B>(st))
        {
            // the reference's inverse came out non-finite: damp harder
            st.lam *= st.nu;
            st.nu *= st.nu;
            ++st.iter;
            continue;
        }
        double step2 = 0.0, mag2 = 0.0;
        bool each_small = true;
#pragma unroll
        for(int i = 0; i < M::P; ++i)
        {
            if(st.fixed & (1u << i))
                continue;   // (the reference's vectors hold the fitted parameters only)
            step2 += st.d[i] * st.d[i];
            const double t = st.p[i] + cfg.eps;   // (an RGB rotation entry is 0)
            mag2 += t * t;
            // per parameter: albedos and sigmas against themselves, angles against 1 rad
            const double scale = i < M::B ? fabs(st.p[i]) : 1.0;
            each_small = each_small && fabs(st.d[i]) <= cfg.eps * (scale + cfg.eps);
        }
        const double step_len = sqrt(step2);
        if(!isfinite(step_len))
        {
            st.status |= SVF_TEXEL_NONFINITE;
            return kCmdDone;
        }
        if(cfg.step_per_param ? each_small : step_len <= cfg.eps * (sqrt(mag2) + cfg.eps))
        {
            if(lm_restart(st, cfg, n_pairs))
                continue;
            return kCmdDone;
        }
        // AcceptStepConstraints (svbrdf-lsq-fitting-internal.hh:67-77)
        bool accept = true;
#pragma unroll
        for(int i = 0; i < M::B; ++i)
            if(st.p[i] - st.d[i] < 0.0f)
                accept = false;
        if(!accept)
        {
            st.lam *= st.nu;
            st.nu *= st.nu;
            ++st.iter;
            continue;
        }
#pragma unroll
        for(int i = 0; i < M::P; ++i)
            st.pt[i] = st.p[i] - st.d[i];
        if constexpr(M::kRgb)
        {
            // the orientation moves by the local rotation phi = -d
            double dq[4];
            quat_exp(st.pt + M::B, dq);
            quat_mul(st.q, dq, st.qt);
        }
        return kCmdTrial;
    }
}

// After the trial residual (fitting.hh:597-612,661-674): accept or damp.
template <class M>
__device__ int lm_after_trial(LmState<M::P>& st, const LmConfig& cfg, double S1, double n_pairs)
{
    ++st.nres;
    double pred = 0.0;
#pragma unroll
    for(int i = 0; i < M::P; ++i)
        pred += st.d[i] * (st.d[i] * st.lam + st.g[i]);
    pred *= 0.5;
    const double rho = 0.5 * (st.S - S1) / pred;
    if(rho > 0.0)
    {
        ++st.eff;
#pragma unroll
        for(int i = 0; i < M::P; ++i)
            st.p[i] = st.pt[i];
        if constexpr(M::kRgb)
        {
            const double n = sqrt(st.qt[0] * st.qt[0] + st.qt[1] * st.qt[1] + st.qt[2] * st.qt[2] +
                                  st.qt[3] * st.qt[3]);
            for(int i = 0; i < 4; ++i)
                st.q[i] = st.qt[i] / n;
            for(int i = M::B; i < M::P; ++i)
                st.p[i] = 0.0;
        }
        st.S = S1;
        st.rho = rho;
        if(S1 / n_pairs <= cfg.mse_target)
            return kCmdDone;
        return kCmdJacobian;
    }
    st.lam *= st.nu;
    st.nu *= st.nu;
    ++st.iter;
    return kCmdContinue;
}

// After the Jacobian at an accepted point (fitting.hh:612-660).
// hg: J^T J (packed upper) then J^T r, in FP64.
template <int P>
__device__ int lm_after_jacobian(LmState<P>& st, const LmConfig& cfg, const double* hg, double n_pairs)
{
    constexpr int kH = P * (P + 1) / 2;
    ++st.njac;
    double glen = 0.0;
#pragma unroll
    for(int i = 0; i < P; ++i)
    {
        st.g[i] = (st.fixed & (1u << i)) ? 0.0 : -hg[kH + i];
        glen += st.g[i] * st.g[i];
    }
#pragma unroll
    for(int i = 0; i < kH; ++i)
        st.H[i] = hg[i];
    if(glen <= cfg.eps * cfg.eps)
        return lm_restart(st, cfg, n_pairs) ? kCmdContinue : kCmdDone;
    const double min_mul = (double)(1.0f / 3.0f);
    const double t = 2.0 * st.rho - 1.0;
    st.lam *= fmax(min_mul, 1.0 - t * t * t);
    st.nu = 2.0;
    ++st.iter;
    return kCmdContinue;
}

// ------------------------------------------------------------------------------
// direction table and pair evaluation
// ------------------------------------------------------------------------------

// Per-evaluation constants shared by every pair.
struct PassConst
{
    float u, v, rsx, rsy, ks, kd, ks_on, kd_on;
    float om[9];
    float kdc[3], ksc[3];   // RGB: clamped per-channel albedos
};

__host__ __device__ inline uint32_t pad4(uint32_t x) { return (x + 3u) & ~3u; }

// Table layout: three float4 arrays of pad4(L) entries (16-byte stride, so 8
// lanes reading 8 consecutive directions hit 32 distinct banks):
//   core0[d] = (a0, a1, a2, sp), core1[d] = (kspec kv, up, kdc, dsp4),
//   deriv[d] = (dsp0, dsp1, dsp2, dsp3)
// The directions themselves are not
// kept: R is orthonormal, so |w_i + w_o| = |s| and cos(h, w_i) = s.a_i / |s|
// with s = a_i + a_o.  Built by the 32 lanes of the control warp.
template <class M>
__device__ __forceinline__ void build_table(float* tab, const float* geo, uint32_t L, const float* pf, PassConst* pc,
                                            uint32_t lane)
{
    ParamSet ps;
    if constexpr(M::kRgb)
        make_param_set_rgb(pf, ps);
    else
        make_param_set(pf, ps);
    float4* core0 = reinterpret_cast<float4*>(tab);
    float4* core1 = core0 + pad4(L);
    float4* deriv = core1 + pad4(L);
    for(uint32_t d = lane; d < L; d += 32)
    {
        const float wx = geo[d], wy = geo[L + d], wz = geo[2 * L + d];
        DirEntry e;
        make_dir_entry(ps, wx, wy, wz, e);
        core0[d] = make_float4(e.a[0], e.a[1], e.a[2], e.sp);
        core1[d] = make_float4(ps.kspec * e.kv, e.up, e.kdc, e.dsp[4]);
        deriv[d] = make_float4(e.dsp[0], e.dsp[1], e.dsp[2], e.dsp[3]);
    }
    if(lane == 0)
    {
        pc->u = ps.u;
        pc->v = ps.v;
        pc->rsx = ps.rsx;
        pc->rsy = ps.rsy;
        pc->ks = ps.ks;
        pc->kd = ps.kd;
        pc->ks_on = ps.ks_on;
        pc->kd_on = ps.kd_on;
#pragma unroll
        for(int k = 0; k < 3; ++k)
#pragma unroll
            for(int j = 0; j < 3; ++j)
                pc->om[3 * k + j] = ps.om[k][j];
        if constexpr(M::kRgb)
            for(int k = 0; k < 3; ++k)
            {
                pc->kdc[k] = pf[k] > 0.0f ? pf[k] : 0.0f;
                pc->ksc[k] = pf[3 + k] > 0.0f ? pf[3 + k] : 0.0f;
            }
    }
}

struct Entry
{
    float a0, a1, a2, sp, d0, d1, d2, d3, d4, kv, up, kdc;
};

// MUFU reciprocal (about 1 ulp); the pair terms need no correctly rounded divide.
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// Loads a direction's entry.
__device__ __forceinline__ Entry load_entry(const float* tab, uint32_t Lp, uint32_t d)
{
    const float4* core0 = reinterpret_cast<const float4*>(tab);
    const float4 x = core0[d], y = core0[Lp + d], z = core0[2 * Lp + d];
    return Entry{ x.x, x.y, x.z, x.w, z.x, z.y, z.z, z.w, y.w, y.x, y.y, y.z };
}

// Warp reduce-scatter of 32 values: on return v[0] of lane j holds the warp's
// sum of v[j] (recursive halving: 31 shuffles instead of 32 x 5).
__device__ __forceinline__ void reduce_scatter32(float* v, uint32_t lane)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
    {
        const bool upper = (lane & (uint32_t)o) != 0;
#pragma unroll
        for(int i = 0; i < o; ++i)
        {
            const float send = upper ? v[i] : v[i + o];
            const float keep = upper ? v[i + o] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
}

__device__ __forceinline__ float warp_sum(float x)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

__device__ __forceinline__ double warp_sum(double x)
{
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Symmetric pair evaluation.  For the two ordered pairs of one unordered pair
// {a, b} (light b seen from view a, and light a seen from view b) the
// specular core is the same: s = a_a + a_b, Q, S = sp_a + sp_b, g = |s|^2 and
// the Fresnel factor (cos(h, w_i) = cos(h, w_o)) do not depend on which
// direction is the light, nor do their parameter derivatives.  With
// C = F g^2 / (Q^2 S) and G the derivative factors,
//
//   spec_io = w_io C,                      w_io = kspec kv_o up_i
//   f_io    = kd h_io + ks spec_io,        h_io = up_o kdc_i
//   J_io    = spec_io V + kd_on h_io e_kd, V = (ks G_sx, ks G_sy, ks_on, 0, ks G_e0, ks G_e1, ks G_e2)
//
// so J^T J and J^T r of both ordered pairs take P = spec_1^2 + spec_2^2 times
// V V^T plus rank-one terms in e_kd, and the core is evaluated once per
// unordered pair.  On the diagonal (a = b) the second ordered pair has zero
// weights.
//
// Enumeration: unordered pair f -> view a = f / nd, offset d = f mod nd
// (nd = L/2 + 1), light b = (a + d) mod L; for even L the offset L/2 is taken
// only for a < L/2.  A warp's 32 consecutive f span at most two views a (the
// entry of a is a broadcast), consecutive lights b (distinct banks), slab
// elements a L + b (consecutive) and b L + a (stride L: distinct banks for
// odd L).
template <bool kFresnel, bool kAllUp>
__device__ __forceinline__ void sym_pair(const PassConst& c, const Entry& ea, const Entry& eb, float refr, float y1,
                                         float y2, float wt1, float wt2, float* acc, double& r2)
{
    const float s0 = ea.a0 + eb.a0, s1 = ea.a1 + eb.a1, s2 = ea.a2 + eb.a2;
    const float q0 = s0 * s0, q1 = s1 * s1, q2 = s2 * s2;
    const float g = q0 + q1 + q2;   // |w_a + w_b|^2
    const float Q = c.u * q0 + c.v * q1 + q2;
    const float S = ea.sp + eb.sp;
    const float QQ = Q * Q;
    const float QQS = QQ * S;
    // (below the normal range the lobe is treated as vanishing, as at 0)
    const float rden = QQS > 1e-37f ? rcp_approx(QQS) : 0.0f;
    float F = 1.0f;
    if(kFresnel)
    {
        const float wa[3] = { ea.a0, ea.a1, ea.a2 }, wb[3] = { eb.a0, eb.a1, eb.a2 };
        F = fresnel_factor(refr, wb, wa);
    }
    const float C = F * g * g * rden;
    // ordered pair 1: view a, light b; ordered pair 2: view b, light a
    // (with every direction above the horizon the up factors are 1)
    const float w1 = kAllUp ? wt1 * ea.kv : wt1 * ea.kv * eb.up;
    const float w2 = kAllUp ? wt2 * eb.kv : wt2 * eb.kv * ea.up;
    const float h1 = kAllUp ? wt1 * eb.kdc : wt1 * ea.up * eb.kdc;
    const float h2 = kAllUp ? wt2 * ea.kdc : wt2 * eb.up * ea.kdc;
    const float sp1 = w1 * C, sp2 = w2 * C;
    const float r1 = y1 - (c.kd * h1 + c.ks * sp1);
    const float r2b = y2 - (c.kd * h2 + c.ks * sp2);
    r2 = fma((double)r1, (double)r1, r2);
    r2 = fma((double)r2b, (double)r2b, r2);
    {
        const float rQ = Q * S * rden;   // 1/Q
        const float rS = QQ * rden;      // 1/S
        const float t0 = s1 * s2 * (c.v - 1.0f);
        const float t1 = s0 * s2 * (1.0f - c.u);
        const float t2 = s0 * s1 * (c.u - c.v);
        float V[kParams];
        V[0] = c.ks * (c.rsx * (4.0f * c.u * q0 * rQ - 1.0f) - (ea.d0 + eb.d0) * rS);
        V[1] = c.ks * (c.rsy * (4.0f * c.v * q1 * rQ - 1.0f) - (ea.d1 + eb.d1) * rS);
        V[2] = c.ks_on;
        V[3] = 0.0f;
        const float m4 = -4.0f * rQ;
        const float dd[3] = { ea.d2 + eb.d2, ea.d3 + eb.d3, ea.d4 + eb.d4 };
#pragma unroll
        for(int k = 0; k < 3; ++k)
        {
            const float dq = c.om[3 * k] * t0 + c.om[3 * k + 1] * t1 + c.om[3 * k + 2] * t2;
            V[4 + k] = c.ks * (m4 * dq - dd[k] * rS);
        }
        const float P = sp1 * sp1 + sp2 * sp2;
        const float X = c.kd_on * (sp1 * h1 + sp2 * h2);
        const float Z = c.kd_on * (h1 * h1 + h2 * h2);
        const float R = sp1 * r1 + sp2 * r2b;
        const float U = c.kd_on * (h1 * r1 + h2 * r2b);
        float PV[kParams];
#pragma unroll
        for(int i = 0; i < kParams; ++i)
            PV[i] = P * V[i];
        int n = 0;
#pragma unroll
        for(int i = 0; i < kParams; ++i)
#pragma unroll
            for(int j = i; j < kParams; ++j)
            {
                if(i == 3 && j == 3)
                    acc[n] += Z;
                else if(i == 3)
                    acc[n] = fmaf(X, V[j], acc[n]);
                else if(j == 3)
                    acc[n] = fmaf(X, V[i], acc[n]);
                else
                    acc[n] = fmaf(PV[i], V[j], acc[n]);
                ++n;
            }
#pragma unroll
        for(int i = 0; i < kParams; ++i)
        {
            if(i == 3)
                acc[kHessian + i] += U;
            else
                acc[kHessian + i] = fmaf(R, V[i], acc[kHessian + i]);
        }
    }
}

// ------------------------------------------------------------------------------
// packed pair evaluation: two unordered pairs per lane, one in each half of the
// sm_100 paired FP32 instructions (add/mul/fma .f32x2), for the luminance fit
// without a Fresnel factor.  Arithmetic per pair as in sym_pair; the two halves
// accumulate separately and are added once at the end of the pass.
// ------------------------------------------------------------------------------

__device__ __forceinline__ float2 f2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
    float2 r;
    asm("{\n\t.reg .b64 x, y, z;\n\tmov.b64 x, {%2, %3};\n\tmov.b64 y, {%4, %5};\n\t"
        "sub.rn.f32x2 z, x, y;\n\tmov.b64 {%0, %1}, z;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}

// Per-pass constants of sym_pair in paired form (both halves equal), with the
// products that do not depend on the pair folded in.
struct PassConst2
{
    float2 u, v, kd, ks, kd_on, ks_on;
    float2 k4u, nksrsx, k4v, nksrsy;   // 4 u ks rsx, -ks rsx, 4 v ks rsy, -ks rsy
    float2 c[9];                       // -4 ks om[3k+j] x {v - 1, 1 - u, u - v}[j]
};

__device__ __forceinline__ PassConst2 make_pass_const2(const PassConst& c)
{
    PassConst2 p;
    p.u = f2(c.u);
    p.v = f2(c.v);
    p.kd = f2(c.kd);
    p.ks = f2(c.ks);
    p.kd_on = f2(c.kd_on);
    p.ks_on = f2(c.ks_on);
    p.k4u = f2(4.0f * c.u * c.ks * c.rsx);
    p.nksrsx = f2(-(c.ks * c.rsx));
    p.k4v = f2(4.0f * c.v * c.ks * c.rsy);
    p.nksrsy = f2(-(c.ks * c.rsy));
    const float tf[3] = { c.v - 1.0f, 1.0f - c.u, c.u - c.v };
#pragma unroll
    for(int k = 0; k < 3; ++k)
#pragma unroll
        for(int j = 0; j < 3; ++j)
            p.c[3 * k + j] = f2(-4.0f * c.ks * c.om[3 * k + j] * tf[j]);
    return p;
}

// Two unordered pairs {a, b} (x half) and {a', b'} (y half).  ea/eb: their
// entries; y1/y2: the samples of the ordered pairs (view a, light b) and
// (view b, light a); wt1/wt2: their weights (0 for a guarded slot or the
// diagonal's second pair).  acc: 35 paired sums (the upper J^T J and J^T r).
template <bool kAllUp>
__device__ __forceinline__ void sym_pair2(const PassConst2& c, const Entry& eaA, const Entry& ebA, const Entry& eaB,
                                          const Entry& ebB, float2 y1, float2 y2, float2 wt1, float2 wt2, float2* acc,
                                          double& r2)
{
    const float2 s0 = make_float2(eaA.a0 + ebA.a0, eaB.a0 + ebB.a0);
    const float2 s1 = make_float2(eaA.a1 + ebA.a1, eaB.a1 + ebB.a1);
    const float2 s2 = make_float2(eaA.a2 + ebA.a2, eaB.a2 + ebB.a2);
    const float2 S = make_float2(eaA.sp + ebA.sp, eaB.sp + ebB.sp);
    const float2 q0 = mul2(s0, s0), q1 = mul2(s1, s1), q2 = mul2(s2, s2);
    const float2 g = add2(add2(q0, q1), q2);
    const float2 Q = fma2(c.u, q0, fma2(c.v, q1, q2));
    const float2 QQ = mul2(Q, Q);
    const float2 QQS = mul2(QQ, S);
    const float2 rden = make_float2(QQS.x > 1e-37f ? rcp_approx(QQS.x) : 0.0f, QQS.y > 1e-37f ? rcp_approx(QQS.y) : 0.0f);
    const float2 C = mul2(mul2(g, g), rden);
    const float2 kv1 = make_float2(eaA.kv, eaB.kv), kv2 = make_float2(ebA.kv, ebB.kv);
    const float2 kdc1 = make_float2(ebA.kdc, ebB.kdc), kdc2 = make_float2(eaA.kdc, eaB.kdc);
    float2 w1, w2, h1, h2;
    if(kAllUp)
    {
        w1 = mul2(wt1, kv1);
        w2 = mul2(wt2, kv2);
        h1 = mul2(wt1, kdc1);
        h2 = mul2(wt2, kdc2);
    }
    else
    {
        const float2 upa = make_float2(eaA.up, eaB.up), upb = make_float2(ebA.up, ebB.up);
        w1 = mul2(mul2(wt1, kv1), upb);
        w2 = mul2(mul2(wt2, kv2), upa);
        h1 = mul2(mul2(wt1, upa), kdc1);
        h2 = mul2(mul2(wt2, upb), kdc2);
    }
    const float2 sp1 = mul2(w1, C), sp2 = mul2(w2, C);
    const float2 r1 = sub2(y1, fma2(c.kd, h1, mul2(c.ks, sp1)));
    const float2 rb = sub2(y2, fma2(c.kd, h2, mul2(c.ks, sp2)));
    r2 = fma((double)r1.x, (double)r1.x, r2);
    r2 = fma((double)rb.x, (double)rb.x, r2);
    r2 = fma((double)r1.y, (double)r1.y, r2);
    r2 = fma((double)rb.y, (double)rb.y, r2);
    const float2 rQ = mul2(mul2(Q, S), rden);   // 1/Q
    const float2 rSk = mul2(mul2(QQ, rden), c.ks);   // ks/S
    const float2 p12 = mul2(s1, s2), p02 = mul2(s0, s2), p01 = mul2(s0, s1);
    float2 V[kParams];
    {
        const float2 nd0 = make_float2(-(eaA.d0 + ebA.d0), -(eaB.d0 + ebB.d0));
        const float2 nd1 = make_float2(-(eaA.d1 + ebA.d1), -(eaB.d1 + ebB.d1));
        V[0] = fma2(nd0, rSk, fma2(c.k4u, mul2(q0, rQ), c.nksrsx));
        V[1] = fma2(nd1, rSk, fma2(c.k4v, mul2(q1, rQ), c.nksrsy));
    }
    V[2] = c.ks_on;
    V[3] = f2(0.0f);
    {
        const float2 nd[3] = { make_float2(-(eaA.d2 + ebA.d2), -(eaB.d2 + ebB.d2)),
                               make_float2(-(eaA.d3 + ebA.d3), -(eaB.d3 + ebB.d3)),
                               make_float2(-(eaA.d4 + ebA.d4), -(eaB.d4 + ebB.d4)) };
#pragma unroll
        for(int k = 0; k < 3; ++k)
        {
            const float2 dq = fma2(c.c[3 * k], p12, fma2(c.c[3 * k + 1], p02, mul2(c.c[3 * k + 2], p01)));
            V[4 + k] = fma2(rQ, dq, mul2(nd[k], rSk));
        }
    }
    const float2 P = fma2(sp1, sp1, mul2(sp2, sp2));
    const float2 X = mul2(c.kd_on, fma2(sp1, h1, mul2(sp2, h2)));
    const float2 Z = mul2(c.kd_on, fma2(h1, h1, mul2(h2, h2)));
    const float2 R = fma2(sp1, r1, mul2(sp2, rb));
    const float2 U = mul2(c.kd_on, fma2(h1, r1, mul2(h2, rb)));
    float2 PV[kParams];
#pragma unroll
    for(int i = 0; i < kParams; ++i)
        PV[i] = mul2(P, V[i]);
    int n = 0;
#pragma unroll
    for(int i = 0; i < kParams; ++i)
#pragma unroll
        for(int j = i; j < kParams; ++j)
        {
            if(i == 3 && j == 3)
                acc[n] = add2(acc[n], Z);
            else if(i == 3)
                acc[n] = fma2(X, V[j], acc[n]);
            else if(j == 3)
                acc[n] = fma2(X, V[i], acc[n]);
            else
                acc[n] = fma2(PV[i], V[j], acc[n]);
            ++n;
        }
#pragma unroll
    for(int i = 0; i < kParams; ++i)
    {
        if(i == 3)
            acc[kHessian + i] = add2(acc[kHessian + i], U);
        else
            acc[kHessian + i] = fma2(R, V[i], acc[kHessian + i]);
    }
}

// ------------------------------------------------------------------------------
// J^T J on the tensor cores: the Jacobian rows of a warp's pairs contracted by
// mma.sync m16n8k8 TF32 with FP32 accumulation (luminance fit, no Fresnel).
// J^T r and r^2 stay on the FP32 / FP64 pipes (the gradient decides where LM
// stops, so it keeps FP32 products).
// ------------------------------------------------------------------------------

// Floats per lane of a warp's staging buffer: J1[0..7] and J2[0..7] interleaved
// as (J1[g], J2[g]); the stride of 24 makes the fragment loads of a half-warp
// hit 32 distinct banks.
constexpr uint32_t kTcLaneStride = 24;
constexpr uint32_t kTcWarpFloats = 32 * kTcLaneStride;

// D[16x8] += A[16x8] B[8x8], A and B TF32 (an FP32 bit pattern is read with its
// low 13 mantissa bits ignored), D FP32.
__device__ __forceinline__ void mma_tf32(float* d, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
                 "{%0, %1, %2, %3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// sym_pair without the J^T J sums: writes the Jacobian rows of the two ordered
// pairs, J1 = sp1 V + kd_on h1 e_kd and J2 likewise (8 entries, the last 0), to
// this lane's staging row, and accumulates J^T r (gr) and r^2.
template <bool kAllUp>
__device__ __forceinline__ void sym_pair_rows(const PassConst& c, const Entry& ea, const Entry& eb, float y1, float y2,
                                              float wt1, float wt2, float* row, float* gr, double& r2)
{
    const float s0 = ea.a0 + eb.a0, s1 = ea.a1 + eb.a1, s2 = ea.a2 + eb.a2;
    const float q0 = s0 * s0, q1 = s1 * s1, q2 = s2 * s2;
    const float g = q0 + q1 + q2;
    const float Q = c.u * q0 + c.v * q1 + q2;
    const float S = ea.sp + eb.sp;
    const float QQ = Q * Q;
    const float QQS = QQ * S;
    const float rden = QQS > 1e-37f ? rcp_approx(QQS) : 0.0f;
    const float C = g * g * rden;
    const float w1 = kAllUp ? wt1 * ea.kv : wt1 * ea.kv * eb.up;
    const float w2 = kAllUp ? wt2 * eb.kv : wt2 * eb.kv * ea.up;
    const float h1 = kAllUp ? wt1 * eb.kdc : wt1 * ea.up * eb.kdc;
    const float h2 = kAllUp ? wt2 * ea.kdc : wt2 * eb.up * ea.kdc;
    const float sp1 = w1 * C, sp2 = w2 * C;
    const float r1 = y1 - (c.kd * h1 + c.ks * sp1);
    const float r2b = y2 - (c.kd * h2 + c.ks * sp2);
    r2 = fma((double)r1, (double)r1, r2);
    r2 = fma((double)r2b, (double)r2b, r2);
    const float rQ = Q * S * rden;
    const float rS = QQ * rden;
    const float t0 = s1 * s2 * (c.v - 1.0f);
    const float t1 = s0 * s2 * (1.0f - c.u);
    const float t2 = s0 * s1 * (c.u - c.v);
    float V[kParams];
    V[0] = c.ks * (c.rsx * (4.0f * c.u * q0 * rQ - 1.0f) - (ea.d0 + eb.d0) * rS);
    V[1] = c.ks * (c.rsy * (4.0f * c.v * q1 * rQ - 1.0f) - (ea.d1 + eb.d1) * rS);
    V[2] = c.ks_on;
    V[3] = 0.0f;
    const float m4 = -4.0f * rQ;
    const float dd[3] = { ea.d2 + eb.d2, ea.d3 + eb.d3, ea.d4 + eb.d4 };
#pragma unroll
    for(int k = 0; k < 3; ++k)
    {
        const float dq = c.om[3 * k] * t0 + c.om[3 * k + 1] * t1 + c.om[3 * k + 2] * t2;
        V[4 + k] = c.ks * (m4 * dq - dd[k] * rS);
    }
    const float R = sp1 * r1 + sp2 * r2b;
#pragma unroll
    for(int i = 0; i < kParams; ++i)
        if(i != 3)
            gr[i] = fmaf(R, V[i], gr[i]);
    gr[3] += c.kd_on * (h1 * r1 + h2 * r2b);
    float J1[8], J2[8];
#pragma unroll
    for(int i = 0; i < kParams; ++i)
    {
        J1[i] = i == 3 ? c.kd_on * h1 : sp1 * V[i];
        J2[i] = i == 3 ? c.kd_on * h2 : sp2 * V[i];
    }
    J1[7] = J2[7] = 0.0f;
    float4* r4 = reinterpret_cast<float4*>(row);
#pragma unroll
    for(int i = 0; i < 8; i += 2)
        r4[i / 2] = make_float4(J1[i], J2[i], J1[i + 1], J2[i + 1]);
}

// The RGB pair: the geometry of sym_pair, three channels.  Per ordered pair k
// and channel c:  f_kc = kd_c h_k + ks_c sp_k,  r_kc = y_kc - f_kc, and
//   J_kc = kd_on_c h_k e_kd_c + ks_on_c sp_k e_ks_c + ks_c sp_k sum_j G_j e_j
// over the geometric parameters j = {sx, sy, phi xyz} (G as V / ks in
// sym_pair, with the identity body rates of the local rotation).  J^T J and
// J^T r then need only channel-free sums, which each lane accumulates:
//   acc[0..2]   sum h^2, sum sp^2, sum h sp
//   acc[3..7]   sum h sp G_j          acc[8..12]  sum sp^2 G_j
//   acc[13..27] sum sp^2 G_i G_j (i <= j)
//   acc[28..30] sum h r_c             acc[31..33] sum sp r_c
//   acc[34..38] sum sp G_j (sum_c ks_c r_c)
// and expand_rgb assembles the 11 x 11 system from them in FP64.
template <bool kFresnel, bool kAllUp>
__device__ __forceinline__ void sym_pair_rgb(const PassConst& c, const Entry& ea, const Entry& eb, float refr,
                                             const float* y1, const float* y2, float wt1, float wt2, float* acc,
                                             double& r2)
{
    const float s0 = ea.a0 + eb.a0, s1 = ea.a1 + eb.a1, s2 = ea.a2 + eb.a2;
    const float q0 = s0 * s0, q1 = s1 * s1, q2 = s2 * s2;
    const float g = q0 + q1 + q2;
    const float Q = c.u * q0 + c.v * q1 + q2;
    const float S = ea.sp + eb.sp;
    const float QQ = Q * Q;
    const float QQS = QQ * S;
    const float rden = QQS > 1e-37f ? rcp_approx(QQS) : 0.0f;
    float F = 1.0f;
    if(kFresnel)
    {
        const float wa[3] = { ea.a0, ea.a1, ea.a2 }, wb[3] = { eb.a0, eb.a1, eb.a2 };
        F = fresnel_factor(refr, wb, wa);
    }
    const float C = F * g * g * rden;
    const float w1 = kAllUp ? wt1 * ea.kv : wt1 * ea.kv * eb.up;
    const float w2 = kAllUp ? wt2 * eb.kv : wt2 * eb.kv * ea.up;
    const float h1 = kAllUp ? wt1 * eb.kdc : wt1 * ea.up * eb.kdc;
    const float h2 = kAllUp ? wt2 * ea.kdc : wt2 * eb.up * ea.kdc;
    const float sp1 = w1 * C, sp2 = w2 * C;
    float r1[3], rb[3];
    float e2 = 0.0f, k1 = 0.0f, k2 = 0.0f;
#pragma unroll
    for(int ch = 0; ch < 3; ++ch)
    {
        r1[ch] = y1[ch] - (c.kdc[ch] * h1 + c.ksc[ch] * sp1);
        rb[ch] = y2[ch] - (c.kdc[ch] * h2 + c.ksc[ch] * sp2);
        e2 = fmaf(r1[ch], r1[ch], fmaf(rb[ch], rb[ch], e2));
        k1 = fmaf(c.ksc[ch], r1[ch], k1);
        k2 = fmaf(c.ksc[ch], rb[ch], k2);
    }
    r2 += (double)e2;
    const float rQ = Q * S * rden;
    const float rS = QQ * rden;
    const float t0 = s1 * s2 * (c.v - 1.0f);
    const float t1 = s0 * s2 * (1.0f - c.u);
    const float t2 = s0 * s1 * (c.u - c.v);
    float G[5];
    G[0] = c.rsx * (4.0f * c.u * q0 * rQ - 1.0f) - (ea.d0 + eb.d0) * rS;
    G[1] = c.rsy * (4.0f * c.v * q1 * rQ - 1.0f) - (ea.d1 + eb.d1) * rS;
    const float m4 = -4.0f * rQ;
    G[2] = m4 * t0 - (ea.d2 + eb.d2) * rS;
    G[3] = m4 * t1 - (ea.d3 + eb.d3) * rS;
    G[4] = m4 * t2 - (ea.d4 + eb.d4) * rS;
    const float Phh = h1 * h1 + h2 * h2, Pss = sp1 * sp1 + sp2 * sp2, Phs = h1 * sp1 + h2 * sp2;
    const float R = sp1 * k1 + sp2 * k2;
    acc[0] += Phh;
    acc[1] += Pss;
    acc[2] += Phs;
    float PG[5];
#pragma unroll
    for(int j = 0; j < 5; ++j)
    {
        acc[3 + j] = fmaf(Phs, G[j], acc[3 + j]);
        PG[j] = Pss * G[j];
        acc[8 + j] += PG[j];
        acc[34 + j] = fmaf(R, G[j], acc[34 + j]);
    }
    int n = 13;
#pragma unroll
    for(int i = 0; i < 5; ++i)
#pragma unroll
        for(int j = i; j < 5; ++j)
        {
            acc[n] = fmaf(PG[i], G[j], acc[n]);
            ++n;
        }
#pragma unroll
    for(int ch = 0; ch < 3; ++ch)
    {
        acc[28 + ch] = fmaf(h1, r1[ch], fmaf(h2, rb[ch], acc[28 + ch]));
        acc[31 + ch] = fmaf(sp1, r1[ch], fmaf(sp2, rb[ch], acc[31 + ch]));
    }
}

// One step of a worker lane over its unordered pairs: pair f = (a, d), then
// f += 32 NW.  kGuard: f may be past the enumeration or, for even L, on the
// repeated offset L/2 (such slots get zero weights, y = 0 and in-range
// indices); without it every pair is valid (odd L, f < total).
template <class M, int NW, bool kFresnel, bool kAllUp, bool kGuard>
__device__ __forceinline__ void pair_step(const float* tab, const PassConst& c, const typename M::Slab* slab, uint32_t L,
                                          uint32_t Lp, uint32_t nd, uint32_t total, uint32_t sa, uint32_t sd, float refr,
                                          uint32_t& f, uint32_t& a, uint32_t& d, float* acc, double& r2)
{
    const bool valid = !kGuard || (f < total && !(2u * d == L && a >= (L >> 1)));
    uint32_t b = a + d;
    b = b >= L ? b - L : b;
    const uint32_t ia = valid ? a : 0u, ib = valid ? b : 0u;
    const Entry ea = load_entry(tab, Lp, ia);
    const Entry eb = load_entry(tab, Lp, ib);
    // pair 1: view a, light b (slab row a); pair 2: view b, light a
    const bool two = valid && d != 0u;
    if constexpr(M::kRgb)
    {
        float y1[3], y2[3];
        const __half* s1 = reinterpret_cast<const __half*>(slab) + 3 * (ia * L + ib);
        const __half* s2 = reinterpret_cast<const __half*>(slab) + 3 * (ib * L + ia);
#pragma unroll
        for(int ch = 0; ch < 3; ++ch)
        {
            y1[ch] = valid ? __half2float(s1[ch]) : 0.0f;
            y2[ch] = two ? __half2float(s2[ch]) : 0.0f;
        }
        sym_pair_rgb<kFresnel, kAllUp>(c, ea, eb, refr, y1, y2, kGuard ? (valid ? 1.0f : 0.0f) : 1.0f,
                                       two ? 1.0f : 0.0f, acc, r2);
    }
    else
    {
        const float* fs = reinterpret_cast<const float*>(slab);
        const float y1 = valid ? fs[ia * L + ib] : 0.0f;
        const float y2 = two ? fs[ib * L + ia] : 0.0f;
        sym_pair<kFresnel, kAllUp>(c, ea, eb, refr, y1, y2, kGuard ? (valid ? 1.0f : 0.0f) : 1.0f, two ? 1.0f : 0.0f,
                                   acc, r2);
    }
    f += 32u * NW;
    a += sa;
    d += sd;
    if(d >= nd)
    {
        d -= nd;
        ++a;
    }
}

// One worker warp's share of a pass over the pairs of a slot (unordered pairs
// wtid, wtid + 32 NW, ...).  Writes the warp's partial sums: J^T J and J^T r
// to red[wwarp][0..34] and r^2 to redd[wwarp].  Every lane runs the same
// number of steps; for odd L only the last one needs the guard.
template <class M, int NW, bool kFresnel, bool kAllUp>
__device__ void worker_pass(const float* tab, const PassConst& c, const typename M::Slab* slab, uint32_t L,
                            float refr, float* red, double* redd, uint32_t wwarp, uint32_t lane)
{
    constexpr int kAcc = M::kAcc;
    static_assert(kAcc >= 32, "reduction layout: 32 reduce-scattered sums + the rest");
    constexpr uint32_t kStride = 32u * NW;
    const uint32_t half = L >> 1, nd = half + 1, Lp = pad4(L);
    const uint32_t total = L * nd;
    const uint32_t iters = (total + kStride - 1) / kStride;
    const uint32_t full = (L & 1u) ? total / kStride : 0u;   // steps with every pair valid
    const uint32_t sa = kStride / nd, sd = kStride - sa * nd;
    uint32_t f = wwarp * 32u + lane;
    uint32_t a = f / nd, d = f - a * nd;

    double r2 = 0.0;
    float acc[kAcc];
#pragma unroll
    for(int i = 0; i < kAcc; ++i)
        acc[i] = 0.0f;

    for(uint32_t it = 0; it < full; ++it)
        pair_step<M, NW, kFresnel, kAllUp, false>(tab, c, slab, L, Lp, nd, total, sa, sd, refr, f, a, d, acc, r2);
    for(uint32_t it = full; it < iters; ++it)
        pair_step<M, NW, kFresnel, kAllUp, true>(tab, c, slab, L, Lp, nd, total, sa, sd, refr, f, a, d, acc, r2);

    r2 = warp_sum(r2);
    {
        float rest[kAcc - 32];
#pragma unroll
        for(int i = 32; i < kAcc; ++i)
            rest[i - 32] = warp_sum(acc[i]);
        reduce_scatter32(acc, lane);
        red[wwarp * kAcc + lane] = acc[0];
        if(lane == 0)
#pragma unroll
            for(int i = 32; i < kAcc; ++i)
                red[wwarp * kAcc + i] = rest[i - 32];
    }
    if(lane == 0)
        redd[wwarp] = r2;
}

// The row fit of LeastSquaresFitSGGX's LSF_OPTION_FIT_TOP
// (svbrdf-lsq-fitting-setup.cc:289-313): the slab holds one view row, the L
// samples of the top-most view, and the model sees them as the pairs (view 0,
// light b) -- the reference's evaluator maps sample b < L to view b / L = 0.
// In sym_pair's terms these are the unordered pairs {0, b} with the second
// ordered pair weighted 0.  Lanes take the lights b; same outputs as
// worker_pass.
template <int NW, bool kFresnel, bool kAllUp>
__device__ void worker_pass_row(const float* tab, const PassConst& c, const float* row, uint32_t L, float refr,
                                float* red, double* redd, uint32_t wwarp, uint32_t lane)
{
    constexpr int kAcc = LumModel::kAcc;
    constexpr uint32_t kStride = 32u * NW;
    const uint32_t Lp = pad4(L);
    double r2 = 0.0;
    float acc[kAcc];
#pragma unroll
    for(int i = 0; i < kAcc; ++i)
        acc[i] = 0.0f;
    const Entry ea = load_entry(tab, Lp, 0);
    const uint32_t iters = (L + kStride - 1) / kStride;
    for(uint32_t it = 0; it < iters; ++it)
    {
        const uint32_t b = it * kStride + wwarp * 32u + lane;
        const bool valid = b < L;
        const Entry eb = load_entry(tab, Lp, valid ? b : 0u);
        sym_pair<kFresnel, kAllUp>(c, ea, eb, refr, valid ? row[b] : 0.0f, 0.0f, valid ? 1.0f : 0.0f, 0.0f, acc, r2);
    }
    r2 = warp_sum(r2);
    float rest[kAcc - 32];
#pragma unroll
    for(int i = 32; i < kAcc; ++i)
        rest[i - 32] = warp_sum(acc[i]);
    reduce_scatter32(acc, lane);
    red[wwarp * kAcc + lane] = acc[0];
    if(lane == 0)
    {
#pragma unroll
        for(int i = 32; i < kAcc; ++i)
            red[wwarp * kAcc + i] = rest[i - 32];
        redd[wwarp] = r2;
    }
}

// Advances an unordered pair (f, a, d) by one worker stride (sa, sd): f += 32 NW.
__device__ __forceinline__ void pair_advance(uint32_t stride, uint32_t nd, uint32_t sa, uint32_t sd, uint32_t& f,
                                             uint32_t& a, uint32_t& d)
{
    f += stride;
    a += sa;
    d += sd;
    if(d >= nd)
    {
        d -= nd;
        ++a;
    }
}

// Loads one unordered pair's entries and samples (see pair_step).
template <bool kGuard>
__device__ __forceinline__ void pair_load(const float* tab, const float* fs, uint32_t L, uint32_t Lp, uint32_t total,
                                          uint32_t f, uint32_t a, uint32_t d, Entry& ea, Entry& eb, float& y1,
                                          float& y2, float& wt1, float& wt2)
{
    const bool valid = !kGuard || (f < total && !(2u * d == L && a >= (L >> 1)));
    uint32_t b = a + d;
    b = b >= L ? b - L : b;
    const uint32_t ia = valid ? a : 0u, ib = valid ? b : 0u;
    ea = load_entry(tab, Lp, ia);
    eb = load_entry(tab, Lp, ib);
    const bool two = valid && d != 0u;
    y1 = valid ? fs[ia * L + ib] : 0.0f;
    y2 = two ? fs[ib * L + ia] : 0.0f;
    wt1 = kGuard ? (valid ? 1.0f : 0.0f) : 1.0f;
    wt2 = two ? 1.0f : 0.0f;
}

// One packed step: the lane's pairs f and f + 32 NW, then f += 64 NW.
template <int NW, bool kAllUp, bool kGuard>
__device__ __forceinline__ void pair_step2(const float* tab, const PassConst2& c, const float* fs, uint32_t L, uint32_t Lp,
                                           uint32_t nd, uint32_t total, uint32_t sa, uint32_t sd, uint32_t& f,
                                           uint32_t& a, uint32_t& d, float2* acc, double& r2)
{
    constexpr uint32_t kStride = 32u * NW;
    uint32_t fB = f, aB = a, dB = d;
    pair_advance(kStride, nd, sa, sd, fB, aB, dB);
    Entry eaA, ebA, eaB, ebB;
    float yA1, yA2, yB1, yB2, wA1, wA2, wB1, wB2;
    pair_load<kGuard>(tab, fs, L, Lp, total, f, a, d, eaA, ebA, yA1, yA2, wA1, wA2);
    pair_load<kGuard>(tab, fs, L, Lp, total, fB, aB, dB, eaB, ebB, yB1, yB2, wB1, wB2);
    sym_pair2<kAllUp>(c, eaA, ebA, eaB, ebB, make_float2(yA1, yB1), make_float2(yA2, yB2), make_float2(wA1, wB1),
                      make_float2(wA2, wB2), acc, r2);
    f = fB;
    a = aB;
    d = dB;
    pair_advance(kStride, nd, sa, sd, f, a, d);
}

// worker_pass for the luminance fit without a Fresnel factor, two pairs a lane
// per step in the paired FP32 instructions.  Same enumeration and outputs.
template <int NW, bool kAllUp>
__device__ void worker_pass2(const float* tab, const PassConst& c1, const float* slab, uint32_t L, float* red,
                             double* redd, uint32_t wwarp, uint32_t lane)
{
    constexpr int kAcc = LumModel::kAcc;
    constexpr uint32_t kStride = 32u * NW;
    const uint32_t half = L >> 1, nd = half + 1, Lp = pad4(L);
    const uint32_t total = L * nd;
    const uint32_t iters = (total + kStride - 1) / kStride;
    const uint32_t full = (L & 1u) ? total / kStride : 0u;   // single steps with every pair valid
    const uint32_t sa = kStride / nd, sd = kStride - sa * nd;
    uint32_t f = wwarp * 32u + lane;
    uint32_t a = f / nd, d = f - a * nd;
    const PassConst2 c = make_pass_const2(c1);

    double r2 = 0.0;
    float2 acc2[kAcc];
#pragma unroll
    for(int i = 0; i < kAcc; ++i)
        acc2[i] = f2(0.0f);
    // double steps: the first full / 2 need no guard, the rest cover the
    // remaining single steps (a pair past the enumeration gets zero weights)
    const uint32_t full2 = full / 2u, iters2 = (iters + 1u) / 2u;
    for(uint32_t it = 0; it < full2; ++it)
        pair_step2<NW, kAllUp, false>(tab, c, slab, L, Lp, nd, total, sa, sd, f, a, d, acc2, r2);
    for(uint32_t it = full2; it < iters2; ++it)
        pair_step2<NW, kAllUp, true>(tab, c, slab, L, Lp, nd, total, sa, sd, f, a, d, acc2, r2);

    float acc[kAcc];
#pragma unroll
    for(int i = 0; i < kAcc; ++i)
        acc[i] = acc2[i].x + acc2[i].y;
    r2 = warp_sum(r2);
    {
        float rest[kAcc - 32];
#pragma unroll
        for(int i = 32; i < kAcc; ++i)
            rest[i - 32] = warp_sum(acc[i]);
        reduce_scatter32(acc, lane);
        red[wwarp * kAcc + lane] = acc[0];
        if(lane == 0)
#pragma unroll
            for(int i = 32; i < kAcc; ++i)
                red[wwarp * kAcc + i] = rest[i - 32];
    }
    if(lane == 0)
        redd[wwarp] = r2;
}

// worker_pass with J^T J on the tensor cores.  Each step every lane stages the
// Jacobian rows of its unordered pair (two ordered pairs) in the warp's buffer
// wbuf; then 8 mma.sync contract them: mma m takes the ordered pairs of lanes
// 4m .. 4m+3 (k = t: first pair of lane 4m+t, k = t+4: its second) as
// A[param][k] (rows 8-15 unused) and B[k][param], so D = sum_k J_k J_k^T.
// Lane (g, t) loads (J1[g], J2[g]) of lane 4m+t, which is both a0/a2 and b0/b1.
template <int NW, bool kAllUp>
__device__ void worker_pass_tc(const float* tab, const PassConst& c, const float* slab, uint32_t L, float* red,
                               double* redd, float* wbuf, uint32_t wwarp, uint32_t lane)
{
    constexpr int kAcc = LumModel::kAcc;
    constexpr uint32_t kStride = 32u * NW;
    const uint32_t half = L >> 1, nd = half + 1, Lp = pad4(L);
    const uint32_t total = L * nd;
    const uint32_t iters = (total + kStride - 1) / kStride;
    const uint32_t sa = kStride / nd, sd = kStride - sa * nd;
    uint32_t f = wwarp * 32u + lane;
    uint32_t a = f / nd, d = f - a * nd;
    const uint32_t g = lane >> 2, t = lane & 3u;
    float* my_row = wbuf + lane * kTcLaneStride;

    double r2 = 0.0;
    float gr[kParams];
#pragma unroll
    for(int i = 0; i < kParams; ++i)
        gr[i] = 0.0f;
    float D[4] = { 0.0f, 0.0f, 0.0f, 0.0f };
    for(uint32_t it = 0; it < iters; ++it)
    {
        Entry ea, eb;
        float y1, y2, wt1, wt2;
        pair_load<true>(tab, slab, L, Lp, total, f, a, d, ea, eb, y1, y2, wt1, wt2);
        sym_pair_rows<kAllUp>(c, ea, eb, y1, y2, wt1, wt2, my_row, gr, r2);
        __syncwarp();
#pragma unroll
        for(uint32_t m = 0; m < 8; ++m)
        {
            const float2 u = *reinterpret_cast<const float2*>(wbuf + (4u * m + t) * kTcLaneStride + 2u * g);
            const uint32_t x = __float_as_uint(u.x), y = __float_as_uint(u.y);
            mma_tf32(D, x, 0u, y, 0u, x, y);
        }
        __syncwarp();   // the rows are read before the next step writes them
        pair_advance(kStride, nd, sa, sd, f, a, d);
    }
    // J^T J: lane (g, t) holds D[g][2t] and D[g][2t + 1]; the upper triangle of
    // the 7 x 7 block goes to the partials in the packed order
#pragma unroll
    for(int q = 0; q < 2; ++q)
    {
        const uint32_t n = 2u * t + (uint32_t)q;
        if(g < (uint32_t)kParams && n < (uint32_t)kParams && g <= n)
            red[wwarp * kAcc + hix<kParams>((int)g, (int)n)] = D[q];
    }
#pragma unroll
    for(int i = 0; i < kParams; ++i)
    {
        const float s = warp_sum(gr[i]);
        if(lane == 0)
            red[wwarp * kAcc + kHessian + i] = s;
    }
    r2 = warp_sum(r2);
    if(lane == 0)
        redd[wwarp] = r2;
}

// ------------------------------------------------------------------------------
// the warp-specialised persistent kernel
// ------------------------------------------------------------------------------

enum : int
{
    kSlotIdle = 0,       // no pass (no texel, or its slab is still arriving)
    kSlotPass = 1,       // J^T J, J^T r and r^2 at the tabulated point
    kSlotExit = 3
};

constexpr uint32_t kNoTexel = 0xffffffffu;

// Per-slot control state (static shared memory).
template <class M>
struct Slot
{
    LmState<M::P> st;
    PassConst pc;
    double sums[M::kAcc + 1];                   // the pass's sums; [kAcc] = r^2
    double hg[M::P * (M::P + 1) / 2 + M::P];    // J^T J and J^T r assembled from them
    float pf[M::kOut];                          // the tabulated point
    uint64_t bar;         // the slab copy's mbarrier
    uint32_t texel;       // texel in the slot, or kNoTexel
    uint32_t parity;      // next phase of `bar`
    int cmd;              // command of the pass the workers run next
    int first;            // the pending pass is at the texel's initial point (else at a trial point)
    int loading;          // the slab copy of `texel` is in flight
    int dead;             // a copy did not arrive: the slot takes no more texels
    int issued;           // the pending slab copy was issued (it may still land)
    int drain;            // dead with a copy possibly in flight: wait for it before exit
    uint32_t arrived;     // worker warps done with the current pass (the last one sums)
    uint32_t L;           // layout of the texel in the slot
    uint32_t slab_bytes;
    double npairs;        // residuals per texel: channels x L^2
    const float* geo;
    float damping;        // the segment's initial damping scale
};

// Dynamic shared memory per slot: [stride] slab | [Lp][kEntry] table |
// [NW] double partials | [NW][kAcc] float partials (doubles first: NW * kAcc
// floats need not be a multiple of 8 bytes).  Every part starts 128-byte aligned.
template <int NW, class M>
struct SlotSmem
{
    __host__ __device__ static size_t slab_bytes(uint64_t stride)
    {
        return (sizeof(typename M::Slab) * stride + 127) & ~size_t(127);
    }
    __host__ __device__ static size_t tab_bytes(uint32_t L) { return (sizeof(float) * kEntry * pad4(L) + 127) & ~size_t(127); }
    __host__ __device__ static size_t red_bytes()
    {
        return (sizeof(float) * NW * M::kAcc + sizeof(double) * NW + 127) & ~size_t(127);
    }
    __host__ __device__ static size_t bytes(uint32_t L, uint64_t stride)
    {
        return slab_bytes(stride) + tab_bytes(L) + red_bytes();
    }
};

__device__ __forceinline__ void nbar_sync(uint32_t id, uint32_t n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

__device__ __forceinline__ void nbar_arrive(uint32_t id, uint32_t n)
{
    asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// Named barrier ids: 0 is __syncthreads; READY[s] = 1 + s, DONE[s] = 1 + S + s.
__device__ __forceinline__ uint32_t bar_ready(int s) { return 1u + (uint32_t)s; }
template <int S>
__device__ __forceinline__ uint32_t bar_done(int s) { return 1u + (uint32_t)S + (uint32_t)s; }

// Writes a finished texel's outputs (LeastSquaresFitSGGX :381-429,
// SVBRDFFitPipeline::fit :692-697).  Control thread.
template <class M>
__device__ void write_texel(const LmArgs& args, LmState<M::P>& st, uint32_t t, double n_pairs)
{
    if constexpr(M::kRgb)
    {
        // {kd rgb, ks rgb, sx, sy, quaternion xyzw}; maps: the fitted albedos,
        // sigma and the orientation
        float pout[12];
        for(int i = 0; i < 8; ++i)
            pout[i] = (float)st.p[i];
        for(int i = 0; i < 4; ++i)
            pout[8 + i] = (float)st.q[i];
        for(int i = 0; i < 12; ++i)
            args.out[(uint64_t)t * 12 + i] = pout[i];
        const double mse = st.S / n_pairs;
        if(!isfinite(mse))
            st.status |= SVF_TEXEL_NONFINITE;
        args.rmse[t] = (float)sqrt(mse);
        if(args.stats)
        {
            svf_texel_stats s;
            s.iterations = st.iter;
            s.effective = st.eff;
            s.jacobians = st.njac;
            s.residuals = st.nres;
            s.status = st.status;
            args.stats[t] = s;
        }
        for(int k = 0; k < 3; ++k)
        {
            if(args.map_diffuse)
                args.map_diffuse[3 * (uint64_t)t + k] = pout[k];
            if(args.map_specular)
                args.map_specular[3 * (uint64_t)t + k] = pout[3 + k];
        }
        if(args.map_sigma)
        {
            args.map_sigma[2 * (uint64_t)t] = pout[6];
            args.map_sigma[2 * (uint64_t)t + 1] = pout[7];
        }
        if(args.map_basis)
            for(int i = 0; i < 4; ++i)
                args.map_basis[4 * (uint64_t)t + i] = pout[8 + i];
    }
    else
    {
    float pout[7];
#pragma unroll
    for(int i = 0; i < 7; ++i)
    {
        pout[i] = (float)st.p[i];
        args.out[(uint64_t)t * 7 + i] = pout[i];
    }
    const double mse = st.S / n_pairs;
    if(!isfinite(mse))
        st.status |= SVF_TEXEL_NONFINITE;
    args.rmse[t] = (float)sqrt(mse);
    if(args.stats)
    {
        svf_texel_stats s;
        s.iterations = st.iter;
        s.effective = st.eff;
        s.jacobians = st.njac;
        s.residuals = st.nres;
        s.status = st.status;
        args.stats[t] = s;
    }
    if(args.map_sigma)
    {
        args.map_sigma[2 * (uint64_t)t] = pout[0];
        args.map_sigma[2 * (uint64_t)t + 1] = pout[1];
    }
    if(args.map_basis)
    {
        // ToQuaternion(euler), quaternion.hh:82-94
        float s1, c1, s2, c2, s3, c3;
        sincosf(0.5f * pout[4], &s1, &c1);
        sincosf(0.5f * pout[5], &s2, &c2);
        sincosf(0.5f * pout[6], &s3, &c3);
        float* q = args.map_basis + 4 * (uint64_t)t;
        q[0] = s1 * c2 * c3 + c1 * s2 * s3;
        q[1] = -s1 * c2 * s3 + c1 * s2 * c3;
        q[2] = c1 * c2 * s3 + s1 * s2 * c3;
        q[3] = c1 * c2 * c3 - s1 * s2 * s3;
    }
    if(args.avg_chroma && (args.map_diffuse || args.map_specular))
    {
        const float* a = args.avg_chroma + 3 * (uint64_t)t;
#pragma unroll
        for(int k = 0; k < 3; ++k)
        {
            if(args.map_diffuse)
                args.map_diffuse[3 * (uint64_t)t + k] = a[k] * pout[3];
            if(args.map_specular)
                args.map_specular[3 * (uint64_t)t + k] = a[k] * pout[2];
        }
    }
}
}

// Control thread: takes the next texel for slot `sl` and starts its slab copy
// (the slab is no longer read: the workers finished the slot's last pass).
template <class M>
__device__ __forceinline__ void slot_fetch(const LmArgs& args, Slot<M>& sl, void* slab)
{
    const uint32_t c = sl.dead ? kNoTexel : atomicAdd(args.work_counter, 1u);
    if(c < args.texels)
    {
        const uint32_t t = args.texel_base + c;
        uint32_t k = 0;
        for(uint32_t i = 1; i < args.n_seg; ++i)
            if(t >= args.seg[i].first)
                k = i;
        const LmSegment& g = args.seg[k];
        sl.L = g.L;
        // (a row fit has one residual per light)
        sl.npairs = args.cfg.row_fit ? (double)g.L : (double)M::kChannels * (double)g.L * (double)g.L;
        sl.geo = g.geo;
        sl.damping = g.damping > 0.0f ? g.damping : 1.0f;
        sl.slab_bytes = (uint32_t)(g.stride * sizeof(typename M::Slab));
        // (fault injection: the copy of one texel is not issued and its wait runs out)
        sl.issued = t != args.fault_skip_texel;
        if(sl.issued)
            bulk_load(slab, static_cast<const typename M::Slab*>(g.lum) + (uint64_t)(t - g.first) * g.stride,
                      sl.slab_bytes, &sl.bar);
        sl.texel = t;
        sl.loading = 1;
    }
    else
    {
        sl.texel = kNoTexel;
        sl.loading = 0;
    }
    sl.cmd = kSlotIdle;
}

// Control thread: the slot's slab has arrived; set up the fit of its texel.
// False when the copy did not arrive within the bound.
template <class M>
__device__ __forceinline__ bool slot_start(const LmArgs& args, Slot<M>& sl)
{
    if(!mbar_wait(&sl.bar, sl.parity, args.wait_spins))
    {
        atomicOr(args.error_flag, 1u);
        if(args.stats)
            args.stats[sl.texel].status = SVF_TEXEL_TIMEOUT;
        sl.dead = 1;
        sl.drain = sl.issued;   // the copy may still land in the slot's shared memory
        sl.loading = 0;
        sl.texel = kNoTexel;
        sl.cmd = kSlotIdle;
        return false;
    }
    sl.parity ^= 1u;
    sl.loading = 0;
    LmState<M::P>& st = sl.st;
    const float* in = args.init + (uint64_t)sl.texel * M::kOut;
#pragma unroll
    for(int i = 0; i < M::kOut; ++i)
        sl.pf[i] = in[i];
    if constexpr(M::kRgb)
    {
        for(int i = 0; i < M::B; ++i)
            st.p[i] = (double)in[i];
        for(int i = M::B; i < M::P; ++i)
            st.p[i] = 0.0;
        double n = 0.0;
        for(int i = 0; i < 4; ++i)
        {
            st.q[i] = (double)in[M::B + i];
            n += st.q[i] * st.q[i];
        }
        n = n > 0.0 ? 1.0 / sqrt(n) : 0.0;
        for(int i = 0; i < 4; ++i)
            st.q[i] = n > 0.0 ? st.q[i] * n : (i == 3 ? 1.0 : 0.0);
    }
    else
    {
#pragma unroll
        for(int i = 0; i < M::P; ++i)
        {
            if(args.cfg.zero_mask & (1u << i))
                sl.pf[i] = 0.0f;
            st.p[i] = (double)sl.pf[i];
        }
    }
    st.fixed = M::kRgb ? 0u : args.cfg.fixed_mask;
    st.iter = st.eff = st.njac = st.nres = st.status = 0;
    st.restarts_left = args.cfg.restarts;
    st.damp_scale = (double)sl.damping;
    sl.first = 1;
    sl.cmd = kSlotPass;
    return true;
}

// FP64 sums of the worker warps' partials, one lane per sum, warps in order.
template <int NW, int kAcc>
__device__ __forceinline__ void sum_partials(const float* red, const double* redd, double* sums, uint32_t lane)
{
    for(uint32_t i = lane; i < (uint32_t)kAcc; i += 32)
    {
        double t = 0.0;
#pragma unroll
        for(int w = 0; w < NW; ++w)
            t += (double)red[w * kAcc + i];
        sums[i] = t;
    }
    if(lane == 0)
    {
        double t = 0.0;
#pragma unroll
        for(int w = 0; w < NW; ++w)
            t += redd[w];
        sums[kAcc] = t;
    }
}

// J^T J and J^T r of the pass at the tabulated point pf (control thread).
// Luminance: the sums are already in that layout.  RGB: assembled from the
// channel-factored sums of sym_pair_rgb; the parameter order is kd rgb (0-2),
// ks rgb (3-5), sx, sy, phi xyz (6-10), and kd_on / ks_on mask the albedo
// derivatives as in the luminance fit.
template <class M>
__device__ void expand_sums(const double* sums, const float* pf, double* hg)
{
    constexpr int P = M::P, kH = P * (P + 1) / 2;
    if constexpr(!M::kRgb)
    {
        for(int i = 0; i < kH + P; ++i)
            hg[i] = sums[i];
    }
    else
    {
    for(int i = 0; i < kH + P; ++i)
        hg[i] = 0.0;
    double ks[3], kdon[3], kson[3], ks2 = 0.0;
    for(int c = 0; c < 3; ++c)
    {
        ks[c] = pf[3 + c] > 0.0f ? (double)pf[3 + c] : 0.0;
        kdon[c] = pf[c] >= 0.0f ? 1.0 : 0.0;
        kson[c] = pf[3 + c] >= 0.0f ? 1.0 : 0.0;
        ks2 += ks[c] * ks[c];
    }
    for(int c = 0; c < 3; ++c)
    {
        hg[hix<P>(c, c)] = kdon[c] * sums[0];
        hg[hix<P>(3 + c, 3 + c)] = kson[c] * sums[1];
        hg[hix<P>(c, 3 + c)] = kdon[c] * kson[c] * sums[2];
        for(int j = 0; j < 5; ++j)
        {
            hg[hix<P>(c, 6 + j)] = kdon[c] * ks[c] * sums[3 + j];
            hg[hix<P>(3 + c, 6 + j)] = kson[c] * ks[c] * sums[8 + j];
        }
        hg[kH + c] = kdon[c] * sums[28 + c];
        hg[kH + 3 + c] = kson[c] * sums[31 + c];
    }
    for(int i = 0; i < 5; ++i)
    {
        for(int j = i; j < 5; ++j)
            hg[hix<P>(6 + i, 6 + j)] = ks2 * sums[13 + hix<5>(i, j)];
        hg[kH + 6 + i] = sums[34 + i];
    }
}
}

// Resident CTAs per SM the register budget is sized for.
// Resident CTAs the register budget is sized for (128 registers a thread at
// 128 and 160 threads).
constexpr int min_blocks(int threads) { return threads <= 128 ? 4 : (threads <= 160 ? 3 : (threads <= 256 ? 2 : 1)); }

// Pair passes: 0 plain, 1 paired FP32 instructions (worker_pass2), 2 J^T J on
// the tensor cores (worker_pass_tc); 1 and 2 for the luminance fit without a
// Fresnel factor.  3: the row fit of LSF_OPTION_FIT_TOP (worker_pass_row), its
// own instance so that the other passes carry no branch for it.
enum : int
{
    kPassPlain = 0,
    kPassPacked = 1,
    kPassTc = 2,
    kPassRow = 3
};

template <class M, int NW, int S, bool kFresnel, bool kAllUp, int kPass>
__global__ void __launch_bounds__(32 * (NW + 1), kPass == kPassPacked ? 1 : min_blocks(32 * (NW + 1)))
    lm_fit_kernel(LmArgs args)
{
    static_assert(kPass == kPassPlain || (!M::kRgb && (!kFresnel || kPass == kPassRow)),
                  "the packed and tensor-core passes are the luminance fit without Fresnel, the row pass "
                  "the luminance fit");
    __shared__ __align__(16) float tc_rows[kPass == kPassTc ? NW * kTcWarpFloats : 4];
    constexpr uint32_t kThreads = 32 * (NW + 1);
    using SM = SlotSmem<NW, M>;
    using SlabT = typename M::Slab;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ Slot<M> slots[S];

    const uint32_t L = args.L;   // the largest layout: sizes each slot's shared memory
    const size_t per_slot = SM::bytes(L, args.lum_stride);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;

    auto slab_of = [&](int s) { return reinterpret_cast<SlabT*>(smem_raw + s * per_slot); };
    auto tab_of = [&](int s) { return reinterpret_cast<float*>(smem_raw + s * per_slot + SM::slab_bytes(args.lum_stride)); };
    auto redd_of = [&](int s) {
        return reinterpret_cast<double*>(smem_raw + s * per_slot + SM::slab_bytes(args.lum_stride) + SM::tab_bytes(L));
    };
    auto red_of = [&](int s) { return reinterpret_cast<float*>(redd_of(s) + NW); };

    if(warp != 0)
    {
        // ---- pair workers
        const uint32_t wwarp = warp - 1;
        for(int s = 0;; s = (s + 1 == S) ? 0 : s + 1)
        {
            nbar_sync(bar_ready(s), kThreads);
            const int cmd = slots[s].cmd;
            if(cmd == kSlotExit)
                break;
            if(cmd == kSlotPass)
            {
                if constexpr(kPass == kPassRow)
                    worker_pass_row<NW, kFresnel, kAllUp>(tab_of(s), slots[s].pc,
                                                          reinterpret_cast<const float*>(slab_of(s)), slots[s].L,
                                                          args.cfg.fresnel, red_of(s), redd_of(s), wwarp, lane);
                else if constexpr(kPass == kPassPacked)
                    worker_pass2<NW, kAllUp>(tab_of(s), slots[s].pc, reinterpret_cast<const float*>(slab_of(s)),
                                             slots[s].L, red_of(s), redd_of(s), wwarp, lane);
                else if constexpr(kPass == kPassTc)
                    worker_pass_tc<NW, kAllUp>(tab_of(s), slots[s].pc, reinterpret_cast<const float*>(slab_of(s)),
                                               slots[s].L, red_of(s), redd_of(s), tc_rows + wwarp * kTcWarpFloats,
                                               wwarp, lane);
                else
                    worker_pass<M, NW, kFresnel, kAllUp>(tab_of(s), slots[s].pc, slab_of(s), slots[s].L,
                                                         args.cfg.fresnel, red_of(s), redd_of(s), wwarp, lane);
                // the last worker warp to finish sums the partials in FP64, in warp
                // order (deterministic), while the others move on
                __syncwarp();
                uint32_t prior = 0;
                if(lane == 0)
                {
                    __threadfence_block();   // release this warp's partials
                    prior = atomicAdd(&slots[s].arrived, 1u);
                    __threadfence_block();   // acquire the other warps' partials
                }
                prior = __shfl_sync(0xffffffffu, prior, 0);
                if(prior == NW - 1)
                {
                    __syncwarp();
                    sum_partials<NW, M::kAcc>(red_of(s), redd_of(s), slots[s].sums, lane);
                    if(lane == 0)
                        slots[s].arrived = 0;
                    __syncwarp();
                }
            }
            nbar_arrive(bar_done<S>(s), kThreads);
        }
        return;
    }

    // ---- control warp
    if(lane == 0)
    {
        for(int s = 0; s < S; ++s)
        {
            Slot<M>& sl = slots[s];
            mbar_init(&sl.bar, 1);
            sl.parity = 0;
            sl.dead = 0;
            sl.drain = 0;
            sl.arrived = 0;
            slot_fetch(args, sl, slab_of(s));
        }
        for(int s = 0; s < S; ++s)
            if(slots[s].loading)
                slot_start(args, slots[s]);
    }
    __syncwarp();
    for(int s = 0; s < S; ++s)
    {
        if(slots[s].cmd == kSlotPass)
            build_table<M>(tab_of(s), slots[s].geo, slots[s].L, slots[s].pf, &slots[s].pc, lane);
        __syncwarp();
        nbar_arrive(bar_ready(s), kThreads);
    }

    for(int s = 0;; s = (s + 1 == S) ? 0 : s + 1)
    {
        Slot<M>& sl = slots[s];
        nbar_sync(bar_done<S>(s), kThreads);
        const int done_cmd = sl.cmd;   // the last worker warp has left the sums in sl.sums

        bool build = false, exit_now = false;
        if(lane == 0)
        {
            LmState<M::P>& st = sl.st;
            int next = kCmdDone;
            if(done_cmd == kSlotPass)
            {
                // Every pass evaluates J^T J and J^T r with r^2: at a trial point
                // the Jacobian of an accepted step is then already at hand, so
                // the separate Jacobian evaluation of fitting.hh:612-616 at the
                // same point is not repeated (same arithmetic, same result).
                constexpr int kH = M::P * (M::P + 1) / 2;
                expand_sums<M>(sl.sums, sl.pf, sl.hg);
                if(sl.first)
                {
                    sl.first = 0;
                    st.njac = 1;
                    st.S = sl.sums[M::kAcc];
#pragma unroll
                    for(int i = 0; i < M::P; ++i)
                        st.g[i] = (st.fixed & (1u << i)) ? 0.0 : -sl.hg[kH + i];
#pragma unroll
                    for(int i = 0; i < kH; ++i)
                        st.H[i] = sl.hg[i];
                    lm_reset_damping(st);
                    if(!isfinite(st.S))
                        st.status |= SVF_TEXEL_NONFINITE;
                    next = kCmdContinue;
                }
                else
                {
                    next = lm_after_trial<M>(st, args.cfg, sl.sums[M::kAcc], sl.npairs);
                    if(next == kCmdJacobian)
                        next = lm_after_jacobian(st, args.cfg, sl.hg, sl.npairs);
                }
                if(next == kCmdContinue)
                    next = lm_next<M>(st, args.cfg, sl.npairs);
                if(next == kCmdTrial)
                {
                    if constexpr(M::kRgb)
                    {
                        for(int i = 0; i < M::B; ++i)
                            sl.pf[i] = (float)st.pt[i];
                        for(int i = 0; i < 4; ++i)
                            sl.pf[M::B + i] = (float)st.qt[i];
                    }
                    else
#pragma unroll
                        for(int i = 0; i < M::P; ++i)
                            sl.pf[i] = (float)st.pt[i];
                    sl.cmd = kSlotPass;
                    build = true;
                }
                else
                {
                    write_texel<M>(args, st, sl.texel, sl.npairs);
                    slot_fetch(args, sl, slab_of(s));
                    // the next texel starts in this visit (its slab copy is short
                    // next to the other slots' passes, which the workers run
                    // meanwhile) rather than after a round with the slot idle
                    if(sl.loading)
                        build = slot_start(args, sl);
                }
            }
            else if(sl.loading)
            {
                // the slab was requested during an earlier visit
                build = slot_start(args, sl);
            }
            if(sl.cmd == kSlotIdle && !sl.loading)
            {
                bool all_idle = true;
                for(int j = 0; j < S; ++j)
                    all_idle = all_idle && slots[j].cmd == kSlotIdle && !slots[j].loading;
                if(all_idle)
                {
                    sl.cmd = kSlotExit;
                    exit_now = true;
                }
            }
        }
        __syncwarp();   // orders lane 0's slot updates before the other lanes read them
        build = __shfl_sync(0xffffffffu, build, 0);
        exit_now = __shfl_sync(0xffffffffu, exit_now, 0);
        if(build)
            build_table<M>(tab_of(s), sl.geo, sl.L, sl.pf, &sl.pc, lane);
        __syncwarp();
        nbar_arrive(bar_ready(s), kThreads);
        if(exit_now)
        {
            // the workers finish the passes already handed out (all idle) and
            // then meet the exit command of slot s
            for(int j = 1; j < S; ++j)
                nbar_sync(bar_done<S>((s + j) % S), kThreads);
            // a slab copy whose wait expired may still be in flight: wait for it
            // (bounded again) before the CTA's shared memory is released
            if(lane == 0)
                for(int j = 0; j < S; ++j)
                    if(slots[j].drain)
                        mbar_wait(&slots[j].bar, slots[j].parity, args.wait_spins);
            break;
        }
    }
}

using KernelFn = void (*)(LmArgs);

template <class M, int NW, int S>
KernelFn pick(bool fresnel, bool all_up)
{
    if(fresnel)
        return all_up ? lm_fit_kernel<M, NW, S, true, true, kPassPlain> : lm_fit_kernel<M, NW, S, true, false, kPassPlain>;
    return all_up ? lm_fit_kernel<M, NW, S, false, true, kPassPlain> : lm_fit_kernel<M, NW, S, false, false, kPassPlain>;
}

// The packed and tensor-core instances (luminance, no Fresnel factor).
template <int NW, int S, int kPass>
KernelFn pick_pass(bool all_up)
{
    return all_up ? lm_fit_kernel<LumModel, NW, S, false, true, kPass> : lm_fit_kernel<LumModel, NW, S, false, false, kPass>;
}

template <class M>
KernelFn kernel_for_model(LmKernelChoice c, bool fresnel, bool all_up)
{
    if constexpr(!M::kRgb)
        if(c.pass == kPassRow)
        {
            // a row slab is L floats: one configuration serves every layout
            if(c.threads != 256 || c.slots != 2)
                return nullptr;
            if(fresnel)
                return all_up ? lm_fit_kernel<LumModel, 7, 2, true, true, kPassRow>
                              : lm_fit_kernel<LumModel, 7, 2, true, false, kPassRow>;
            return all_up ? lm_fit_kernel<LumModel, 7, 2, false, true, kPassRow>
                          : lm_fit_kernel<LumModel, 7, 2, false, false, kPassRow>;
        }
        else if(c.pass == kPassPacked && !fresnel)
        {
            if(c.threads == 256 && c.slots == 3)
                return pick_pass<7, 3, kPassPacked>(all_up);
            if(c.threads == 256 && c.slots == 4)
                return pick_pass<7, 4, kPassPacked>(all_up);
            if(c.threads == 128 && c.slots == 3)
                return pick_pass<3, 3, kPassPacked>(all_up);
            return nullptr;
        }
        else if(c.pass == kPassTc && !fresnel)
        {
            if(c.threads == 256 && c.slots == 2)
                return pick_pass<7, 2, kPassTc>(all_up);
            if(c.threads == 128 && c.slots == 3)
                return pick_pass<3, 3, kPassTc>(all_up);
            return nullptr;
        }
    // (a packed or tensor-core choice runs the plain pass where those do not apply)
    if(c.threads == 256 && c.slots == 2)
        return pick<M, 7, 2>(fresnel, all_up);
    if(c.threads == 256 && c.slots == 3)
        return pick<M, 7, 3>(fresnel, all_up);
    if(c.threads == 256 && c.slots == 4)
        return pick<M, 7, 4>(fresnel, all_up);
    if(c.threads == 128 && c.slots == 2)
        return pick<M, 3, 2>(fresnel, all_up);
    if(c.threads == 128 && c.slots == 3)
        return pick<M, 3, 3>(fresnel, all_up);
    if(c.threads == 160 && c.slots == 2)
        return pick<M, 4, 2>(fresnel, all_up);
    if(c.threads == 160 && c.slots == 3)
        return pick<M, 4, 3>(fresnel, all_up);
    if(c.threads == 256 && c.slots == 1)   // the largest slabs: one texel per CTA, no overlap
        return pick<M, 7, 1>(fresnel, all_up);
    return nullptr;
}

KernelFn kernel_for(LmKernelChoice c, bool fresnel, bool all_up, bool rgb)
{
    return rgb ? kernel_for_model<RgbModel>(c, fresnel, all_up) : kernel_for_model<LumModel>(c, fresnel, all_up);
}

} // namespace

LmKernelChoice lm_default_choice(uint32_t L, uint64_t lum_stride, bool rgb)
{
    // The candidate with the most texels in flight per SM (resident CTAs x
    // slots, a single-slot CTA's counted at half: its workers wait for the
    // control warp between passes); ties go to more CTAs (more control warps
    // running the FP64 steps side by side), then to more worker warps.
    // Measured on the B200 (full launches): ring-81 slabs, 160000 texels --
    // 128 threads x 2 slots (3 CTAs, 6 texels per SM) 52.2 ms, 256 x 2 54.7,
    // 256 x 3 55.9, 128 x 3 57.7; Fibonacci-151 slabs, 589824 texels --
    // 256 x 2 (1 CTA) 564 ms, 256 x 1 (2 CTAs) 595, 128 x 2 773.
    LmKernelChoice cand[kLmPlainCandidates];
    const int n = lm_candidates(L, cand, kLmPlainCandidates);   // the plain passes
    int best = -1, best_t = 0, best_c = 0, best_w = 0;
    for(int i = 0; i < n; ++i)
    {
        const int ctas = lm_max_ctas_per_sm(L, lum_stride, cand[i], rgb);
        const int t = ctas * (cand[i].slots >= 2 ? 2 * cand[i].slots : 1);   // half-texels in flight
        const int w = ctas * (cand[i].threads / 32 - 1);
        if(ctas > 0 && (t > best_t || (t == best_t && (ctas > best_c || (ctas == best_c && w > best_w)))))
        {
            best = i;
            best_t = t;
            best_c = ctas;
            best_w = w;
        }
    }
    return best >= 0 ? cand[best] : cand[0];
}

int lm_candidates(uint32_t, LmKernelChoice* out, int max)
{
    // the plain passes first (the untuned default picks among them), then the
    // packed ones (one CTA of 256 threads per SM at their register count), then
    // the tensor-core J^T J ones (their staging rows take shared memory)
    const LmKernelChoice all[kLmCandidates] = { { 256, 3, 0 }, { 256, 2, 0 }, { 128, 3, 0 }, { 128, 2, 0 },
                                                { 256, 1, 0 }, { 160, 2, 0 }, { 160, 3, 0 }, { 256, 3, 1 },
                                                { 256, 4, 1 }, { 128, 3, 1 }, { 256, 2, 2 }, { 128, 3, 2 } };
    int n = 0;
    for(int i = 0; i < kLmCandidates && n < max; ++i)
        out[n++] = all[i];
    return n;
}

// SlotSmem<NW, M>::bytes for the configuration's worker count NW = threads / 32 - 1.
template <class M>
size_t slot_bytes(int nw, uint32_t L, uint64_t stride)
{
    const size_t red = (sizeof(float) * nw * M::kAcc + sizeof(double) * nw + 127) & ~size_t(127);
    return SlotSmem<1, M>::slab_bytes(stride) + SlotSmem<1, M>::tab_bytes(L) + red;
}

size_t lm_smem_bytes(uint32_t L, uint64_t lum_stride, LmKernelChoice c, bool rgb)
{
    const int nw = c.threads / 32 - 1;
    const size_t per = rgb ? slot_bytes<RgbModel>(nw, L, lum_stride) : slot_bytes<LumModel>(nw, L, lum_stride);
    return per * (size_t)c.slots;
}

int lm_max_ctas_per_sm(uint32_t L, uint64_t lum_stride, LmKernelChoice c, bool rgb)
{
    // the Fresnel and horizon variants share the launch configuration
    KernelFn k = kernel_for(c, false, false, rgb);
    if(!k || L == 0)
        return 0;
    const size_t smem = lm_smem_bytes(L, lum_stride, c, rgb);
    if(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess ||
       cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    int n = 0;
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, c.threads, smem) != cudaSuccess)
    {
        cudaGetLastError();
        return 0;
    }
    return n;
}

cudaError_t launch_lm_fit(const LmArgs& args, LmKernelChoice c, int grid, cudaStream_t stream)
{
    const bool rgb = args.rgb != 0;
    KernelFn k = kernel_for(c, args.cfg.fresnel != 1.0f, args.all_up != 0, rgb);
    if(!k || args.L == 0)
        return cudaErrorInvalidConfiguration;
    const size_t smem = lm_smem_bytes(args.L, args.lum_stride, c, rgb);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(e != cudaSuccess)
        return e;
    e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
    if(e != cudaSuccess)
        return e;
    k<<<grid, c.threads, smem, stream>>>(args);
    return cudaGetLastError();
}

} // namespace svf
