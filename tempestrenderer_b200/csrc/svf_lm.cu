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
constexpr int kRed = kHessian + kParams;     // FP32 partial sums per thread (J^T J, J^T r)
constexpr uint32_t kWaitSpins = 1u << 22;    // bound of every mbarrier wait

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

// Bounded wait for phase `parity` of `bar`; false when the bound expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    const uint32_t b = smem_addr(bar);
    for(uint32_t i = 0; i < kWaitSpins; ++i)
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

struct LmState
{
    double p[kParams];      // current parameters
    double pt[kParams];     // trial parameters
    double d[kParams];      // step
    double g[kParams];      // gradient J_r^T r of the residual r = y - f
    double H[kHessian];     // J^T J, packed upper
    double S;               // sum of squared residuals at p
    double lam, nu, rho;
    uint32_t iter, eff, njac, nres, status, restarts_left;
};

// Fresh damping from the current normal equations (fitting.hh:531-538).
__device__ __forceinline__ void lm_reset_damping(LmState& st)
{
    double damping = 1.0;   // InitialMinDamping
#pragma unroll
    for(int i = 0; i < kParams; ++i)
        damping = fmax(damping, st.H[hidx(i, i)]);
    st.lam = damping * 0.75;   // InitialDampingMultiplier
    st.nu = 2.0;               // DampingFailureMultiplier
}

// Where the reference's loop ends, optionally continue with fresh damping from
// the same point; false when the fit is finished.
__device__ __forceinline__ bool lm_restart(LmState& st, const LmConfig& cfg, double n_pairs)
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
__device__ __noinline__ bool lm_solve(LmState& st)
{
    uint32_t frozen = 0;
    for(int round = 0; round < 5; ++round)
    {
        double A[kHessian], x[kParams];
#pragma unroll
        for(int i = 0; i < kHessian; ++i)
            A[i] = st.H[i];
#pragma unroll
        for(int i = 0; i < kParams; ++i)
        {
            A[hidx(i, i)] += st.lam;
            x[i] = st.g[i];
        }
#pragma unroll
        for(int i = 0; i < 4; ++i)
            if(frozen & (1u << i))
            {
#pragma unroll
                for(int j = 0; j < kParams; ++j)
                    if(j != i)
                        A[hidx(i, j)] = 0.0;
                x[i] = 0.0;
            }
        // A = L L^T; the diagonal keeps 1 / L_jj
        bool ok = true;
#pragma unroll
        for(int j = 0; j < kParams; ++j)
        {
            double s = A[hidx(j, j)];
#pragma unroll
            for(int k = 0; k < j; ++k)
                s -= A[hidx(j, k)] * A[hidx(j, k)];
            ok = ok && (s > 0.0) && isfinite(s);
            const double r = rsqrt(s);
            A[hidx(j, j)] = r;
#pragma unroll
            for(int i = j + 1; i < kParams; ++i)
            {
                double t = A[hidx(i, j)];
#pragma unroll
                for(int k = 0; k < j; ++k)
                    t -= A[hidx(i, k)] * A[hidx(j, k)];
                A[hidx(i, j)] = t * r;
            }
        }
        if(!ok)
            return false;
#pragma unroll
        for(int i = 0; i < kParams; ++i)
        {
            double t = x[i];
#pragma unroll
            for(int k = 0; k < i; ++k)
                t -= A[hidx(i, k)] * x[k];
            x[i] = t * A[hidx(i, i)];
        }
#pragma unroll
        for(int i = kParams - 1; i >= 0; --i)
        {
            double t = x[i];
#pragma unroll
            for(int k = i + 1; k < kParams; ++k)
                t -= A[hidx(k, i)] * x[k];
            x[i] = t * A[hidx(i, i)];
        }
        uint32_t more = frozen;
#pragma unroll
        for(int i = 0; i < kParams; ++i)
        {
            st.d[i] = x[i];
            if(i < 4 && st.p[i] == 0.0 && x[i] > 0.0)
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
__device__ int lm_next(LmState& st, const LmConfig& cfg, double n_pairs)
{
    for(;;)
    {
        if(!(st.iter < cfg.max_iter && cfg.mse_target < st.S / n_pairs))
        {
            if(st.iter >= cfg.max_iter)
                st.status |= SVF_TEXEL_MAX_ITER;
            return kCmdDone;
        }
        if(!lm_solve(st))
        {
            // the reference's inverse came out non-finite: damp harder
            st.lam *= st.nu;
            st.nu *= st.nu;
            ++st.iter;
            continue;
        }
        double step2 = 0.0, mag2 = 0.0;
#pragma unroll
        for(int i = 0; i < kParams; ++i)
        {
            step2 += st.d[i] * st.d[i];
            const double t = st.p[i] + cfg.eps;
            mag2 += t * t;
        }
        const double step_len = sqrt(step2);
        if(!isfinite(step_len))
        {
            st.status |= SVF_TEXEL_NONFINITE;
            return kCmdDone;
        }
        if(step_len <= cfg.eps * (sqrt(mag2) + cfg.eps))
        {
            if(lm_restart(st, cfg, n_pairs))
                continue;
            return kCmdDone;
        }
        // AcceptStepConstraints (svbrdf-lsq-fitting-internal.hh:67-77)
        bool accept = true;
#pragma unroll
        for(int i = 0; i < 4; ++i)
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
        for(int i = 0; i < kParams; ++i)
            st.pt[i] = st.p[i] - st.d[i];
        return kCmdTrial;
    }
}

// After the trial residual (fitting.hh:597-612,661-674): accept or damp.
__device__ int lm_after_trial(LmState& st, const LmConfig& cfg, double S1, double n_pairs)
{
    ++st.nres;
    double pred = 0.0;
#pragma unroll
    for(int i = 0; i < kParams; ++i)
        pred += st.d[i] * (st.d[i] * st.lam + st.g[i]);
    pred *= 0.5;
    const double rho = 0.5 * (st.S - S1) / pred;
    if(rho > 0.0)
    {
        ++st.eff;
#pragma unroll
        for(int i = 0; i < kParams; ++i)
            st.p[i] = st.pt[i];
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
__device__ int lm_after_jacobian(LmState& st, const LmConfig& cfg, const double* red, double n_pairs)
{
    ++st.njac;
    double glen = 0.0;
#pragma unroll
    for(int i = 0; i < kParams; ++i)
    {
        st.g[i] = -red[kHessian + i];
        glen += st.g[i] * st.g[i];
    }
#pragma unroll
    for(int i = 0; i < kHessian; ++i)
        st.H[i] = red[i];
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
};

__host__ __device__ inline uint32_t pad4(uint32_t x) { return (x + 3u) & ~3u; }

// Table layout: three float4 arrays of pad4(L) entries (16-byte stride, so 8
// lanes reading 8 consecutive directions hit 32 distinct banks):
//   core0[d] = (a0, a1, a2, sp), core1[d] = (kspec kv, up, kdc, dsp4),
//   deriv[d] = (dsp0, dsp1, dsp2, dsp3)
// The directions themselves are not
// kept: R is orthonormal, so |w_i + w_o| = |s| and cos(h, w_i) = s.a_i / |s|
// with s = a_i + a_o.  Built by the 32 lanes of the control warp.
__device__ __forceinline__ void build_table(float* tab, const float* geo, uint32_t L, const float* pf, PassConst* pc,
                                            uint32_t lane)
{
    ParamSet ps;
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

// One step of a worker lane over its unordered pairs: pair f = (a, d), then
// f += 32 NW.  kGuard: f may be past the enumeration or, for even L, on the
// repeated offset L/2 (such slots get zero weights, y = 0 and in-range
// indices); without it every pair is valid (odd L, f < total).
template <int NW, bool kFresnel, bool kAllUp, bool kGuard>
__device__ __forceinline__ void pair_step(const float* tab, const PassConst& c, const float* slab, uint32_t L,
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
    const float y1 = valid ? slab[ia * L + ib] : 0.0f;
    const bool two = valid && d != 0u;
    const float y2 = two ? slab[ib * L + ia] : 0.0f;
    sym_pair<kFresnel, kAllUp>(c, ea, eb, refr, y1, y2, kGuard ? (valid ? 1.0f : 0.0f) : 1.0f, two ? 1.0f : 0.0f,
                               acc, r2);
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
template <int NW, bool kFresnel, bool kAllUp>
__device__ void worker_pass(const float* tab, const PassConst& c, const float* slab, uint32_t L, float refr,
                            float* red, double* redd, uint32_t wwarp, uint32_t lane)
{
    static_assert(kRed == 35, "reduction layout: 32 reduce-scattered sums + 3");
    constexpr uint32_t kStride = 32u * NW;
    const uint32_t half = L >> 1, nd = half + 1, Lp = pad4(L);
    const uint32_t total = L * nd;
    const uint32_t iters = (total + kStride - 1) / kStride;
    const uint32_t full = (L & 1u) ? total / kStride : 0u;   // steps with every pair valid
    const uint32_t sa = kStride / nd, sd = kStride - sa * nd;
    uint32_t f = wwarp * 32u + lane;
    uint32_t a = f / nd, d = f - a * nd;

    double r2 = 0.0;
    float acc[kRed];
#pragma unroll
    for(int i = 0; i < kRed; ++i)
        acc[i] = 0.0f;

    for(uint32_t it = 0; it < full; ++it)
        pair_step<NW, kFresnel, kAllUp, false>(tab, c, slab, L, Lp, nd, total, sa, sd, refr, f, a, d, acc, r2);
    for(uint32_t it = full; it < iters; ++it)
        pair_step<NW, kFresnel, kAllUp, true>(tab, c, slab, L, Lp, nd, total, sa, sd, refr, f, a, d, acc, r2);

    r2 = warp_sum(r2);
    {
        const float t32 = warp_sum(acc[32]), t33 = warp_sum(acc[33]), t34 = warp_sum(acc[34]);
        reduce_scatter32(acc, lane);
        red[wwarp * kRed + lane] = acc[0];
        if(lane == 0)
        {
            red[wwarp * kRed + 32] = t32;
            red[wwarp * kRed + 33] = t33;
            red[wwarp * kRed + 34] = t34;
        }
    }
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
struct Slot
{
    LmState st;
    PassConst pc;
    double sums[kRed + 1];
    float pf[kParams];
    uint64_t bar;         // the slab copy's mbarrier
    uint32_t texel;       // texel in the slot, or kNoTexel
    uint32_t parity;      // next phase of `bar`
    int cmd;              // command of the pass the workers run next
    int first;            // the pending pass is at the texel's initial point (else at a trial point)
    int loading;          // the slab copy of `texel` is in flight
    int dead;             // a copy did not arrive: the slot takes no more texels
    uint32_t arrived;     // worker warps done with the current pass (the last one sums)
    uint32_t L;           // layout of the texel in the slot
    uint32_t slab_bytes;
    double npairs;        // L^2
    const float* geo;
};

// Dynamic shared memory per slot: [stride] slab | [Lp][kEntry] table |
// [NW] double partials | [NW][kRed] float partials (doubles first: NW * kRed
// floats need not be a multiple of 8 bytes).  Every part starts 128-byte aligned.
template <int NW>
struct SlotSmem
{
    __host__ __device__ static size_t slab_bytes(uint64_t stride) { return (sizeof(float) * stride + 127) & ~size_t(127); }
    __host__ __device__ static size_t tab_bytes(uint32_t L) { return (sizeof(float) * kEntry * pad4(L) + 127) & ~size_t(127); }
    __host__ __device__ static size_t red_bytes() { return (sizeof(float) * NW * kRed + sizeof(double) * NW + 127) & ~size_t(127); }
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
__device__ void write_texel(const LmArgs& args, LmState& st, uint32_t t, double n_pairs)
{
    float pout[kParams];
#pragma unroll
    for(int i = 0; i < kParams; ++i)
    {
        pout[i] = (float)st.p[i];
        args.out[(uint64_t)t * kParams + i] = pout[i];
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

// Control thread: takes the next texel for slot `sl` and starts its slab copy
// (the slab is no longer read: the workers finished the slot's last pass).
__device__ __forceinline__ void slot_fetch(const LmArgs& args, Slot& sl, float* slab)
{
    const uint32_t t = sl.dead ? kNoTexel : atomicAdd(args.work_counter, 1u);
    if(t < args.texels)
    {
        uint32_t k = 0;
        for(uint32_t i = 1; i < args.n_seg; ++i)
            if(t >= args.seg[i].first)
                k = i;
        const LmSegment& g = args.seg[k];
        sl.L = g.L;
        sl.npairs = (double)g.L * (double)g.L;
        sl.geo = g.geo;
        sl.slab_bytes = (uint32_t)(g.stride * sizeof(float));
        bulk_load(slab, g.lum + (uint64_t)(t - g.first) * g.stride, sl.slab_bytes, &sl.bar);
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
__device__ __forceinline__ bool slot_start(const LmArgs& args, Slot& sl)
{
    if(!mbar_wait(&sl.bar, sl.parity))
    {
        atomicOr(args.error_flag, 1u);
        if(args.stats)
            args.stats[sl.texel].status = SVF_TEXEL_TIMEOUT;
        sl.dead = 1;
        sl.loading = 0;
        sl.texel = kNoTexel;
        sl.cmd = kSlotIdle;
        return false;
    }
    sl.parity ^= 1u;
    sl.loading = 0;
    LmState& st = sl.st;
#pragma unroll
    for(int i = 0; i < kParams; ++i)
    {
        st.p[i] = (double)args.init[(uint64_t)sl.texel * kParams + i];
        sl.pf[i] = (float)st.p[i];
    }
    st.iter = st.eff = st.njac = st.nres = st.status = 0;
    st.restarts_left = args.cfg.restarts;
    sl.first = 1;
    sl.cmd = kSlotPass;
    return true;
}

// FP64 sums of the worker warps' partials, one lane per sum, warps in order.
template <int NW>
__device__ __forceinline__ void sum_partials(const float* red, const double* redd, double* sums, uint32_t lane)
{
    for(uint32_t i = lane; i < (uint32_t)kRed; i += 32)
    {
        double t = 0.0;
#pragma unroll
        for(int w = 0; w < NW; ++w)
            t += (double)red[w * kRed + i];
        sums[i] = t;
    }
    if(lane == 0)
    {
        double t = 0.0;
#pragma unroll
        for(int w = 0; w < NW; ++w)
            t += redd[w];
        sums[kRed] = t;
    }
}

// Resident CTAs per SM the register budget is sized for.
constexpr int min_blocks(int threads) { return threads <= 128 ? 4 : 2; }

template <int NW, int S, bool kFresnel, bool kAllUp>
__global__ void __launch_bounds__(32 * (NW + 1), min_blocks(32 * (NW + 1))) lm_fit_kernel(LmArgs args)
{
    constexpr uint32_t kThreads = 32 * (NW + 1);
    using SM = SlotSmem<NW>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ Slot slots[S];

    const uint32_t L = args.L;   // the largest layout: sizes each slot's shared memory
    const size_t per_slot = SM::bytes(L, args.lum_stride);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;

    auto slab_of = [&](int s) { return reinterpret_cast<float*>(smem_raw + s * per_slot); };
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
                worker_pass<NW, kFresnel, kAllUp>(tab_of(s), slots[s].pc, slab_of(s), slots[s].L, args.cfg.fresnel,
                                                  red_of(s), redd_of(s), wwarp, lane);
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
                    sum_partials<NW>(red_of(s), redd_of(s), slots[s].sums, lane);
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
            Slot& sl = slots[s];
            mbar_init(&sl.bar, 1);
            sl.parity = 0;
            sl.dead = 0;
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
            build_table(tab_of(s), slots[s].geo, slots[s].L, slots[s].pf, &slots[s].pc, lane);
        __syncwarp();
        nbar_arrive(bar_ready(s), kThreads);
    }

    for(int s = 0;; s = (s + 1 == S) ? 0 : s + 1)
    {
        Slot& sl = slots[s];
        nbar_sync(bar_done<S>(s), kThreads);
        const int done_cmd = sl.cmd;   // the last worker warp has left the sums in sl.sums

        bool build = false, exit_now = false;
        if(lane == 0)
        {
            LmState& st = sl.st;
            int next = kCmdDone;
            if(done_cmd == kSlotPass)
            {
                // Every pass evaluates J^T J and J^T r with r^2: at a trial point
                // the Jacobian of an accepted step is then already at hand, so
                // the separate Jacobian evaluation of fitting.hh:612-616 at the
                // same point is not repeated (same arithmetic, same result).
                if(sl.first)
                {
                    sl.first = 0;
                    st.njac = 1;
                    st.S = sl.sums[kRed];
#pragma unroll
                    for(int i = 0; i < kParams; ++i)
                        st.g[i] = -sl.sums[kHessian + i];
#pragma unroll
                    for(int i = 0; i < kHessian; ++i)
                        st.H[i] = sl.sums[i];
                    lm_reset_damping(st);
                    if(!isfinite(st.S))
                        st.status |= SVF_TEXEL_NONFINITE;
                    next = kCmdContinue;
                }
                else
                {
                    next = lm_after_trial(st, args.cfg, sl.sums[kRed], sl.npairs);
                    if(next == kCmdJacobian)
                        next = lm_after_jacobian(st, args.cfg, sl.sums, sl.npairs);
                }
                if(next == kCmdContinue)
                    next = lm_next(st, args.cfg, sl.npairs);
                if(next == kCmdTrial)
                {
#pragma unroll
                    for(int i = 0; i < kParams; ++i)
                        sl.pf[i] = (float)st.pt[i];
                    sl.cmd = kSlotPass;
                    build = true;
                }
                else
                {
                    write_texel(args, st, sl.texel, sl.npairs);
                    slot_fetch(args, sl, slab_of(s));
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
            build_table(tab_of(s), sl.geo, sl.L, sl.pf, &sl.pc, lane);
        __syncwarp();
        nbar_arrive(bar_ready(s), kThreads);
        if(exit_now)
        {
            // the workers finish the passes already handed out (all idle) and
            // then meet the exit command of slot s
            for(int j = 1; j < S; ++j)
                nbar_sync(bar_done<S>((s + j) % S), kThreads);
            break;
        }
    }
}

using KernelFn = void (*)(LmArgs);

template <int NW, int S>
KernelFn pick(bool fresnel, bool all_up)
{
    if(fresnel)
        return all_up ? lm_fit_kernel<NW, S, true, true> : lm_fit_kernel<NW, S, true, false>;
    return all_up ? lm_fit_kernel<NW, S, false, true> : lm_fit_kernel<NW, S, false, false>;
}

KernelFn kernel_for(LmKernelChoice c, bool fresnel, bool all_up)
{
    if(c.threads == 256 && c.slots == 2)
        return pick<7, 2>(fresnel, all_up);
    if(c.threads == 256 && c.slots == 3)
        return pick<7, 3>(fresnel, all_up);
    if(c.threads == 128 && c.slots == 2)
        return pick<3, 2>(fresnel, all_up);
    if(c.threads == 128 && c.slots == 3)
        return pick<3, 3>(fresnel, all_up);
    return nullptr;
}

} // namespace

LmKernelChoice lm_default_choice(uint32_t L, uint64_t lum_stride)
{
    // the first candidate whose shared memory fits on an SM (fewer slots at large L)
    LmKernelChoice cand[4];
    const int n = lm_candidates(L, cand, 4);
    for(int i = 0; i < n; ++i)
        if(lm_max_ctas_per_sm(L, lum_stride, cand[i]) > 0)
            return cand[i];
    return cand[0];
}

int lm_candidates(uint32_t, LmKernelChoice* out, int max)
{
    const LmKernelChoice all[4] = { { 256, 3 }, { 256, 2 }, { 128, 3 }, { 128, 2 } };
    int n = 0;
    for(int i = 0; i < 4 && n < max; ++i)
        out[n++] = all[i];
    return n;
}

size_t lm_smem_bytes(uint32_t L, uint64_t lum_stride, LmKernelChoice c)
{
    const size_t per = c.threads == 128 ? SlotSmem<3>::bytes(L, lum_stride) : SlotSmem<7>::bytes(L, lum_stride);
    return per * (size_t)c.slots;
}

int lm_max_ctas_per_sm(uint32_t L, uint64_t lum_stride, LmKernelChoice c)
{
    // the variants share the launch configuration
    KernelFn k = kernel_for(c, false, false);
    if(!k || L == 0)
        return 0;
    const size_t smem = lm_smem_bytes(L, lum_stride, c);
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
    KernelFn k = kernel_for(c, args.cfg.fresnel != 1.0f, args.all_up != 0);
    if(!k || args.L == 0)
        return cudaErrorInvalidConfiguration;
    const size_t smem = lm_smem_bytes(args.L, args.lum_stride, c);
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
