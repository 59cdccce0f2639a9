// svf_lm.cu - the persistent Levenberg-Marquardt fit (LeastSquaresFitSGGX,
// tools/svbrdf-fitting/svbrdf-lsq-fitting-setup.cc:234-431, over
// LevenbergMarquardtCurveFit, include/tempest/math/fitting.hh:457-678) for sm_100a.
//
// Work distribution: a persistent grid of (resident CTAs per SM) x (SMs) CTAs
// pulls texels from a global atomic counter (work stealing: a texel that
// converges early frees its CTA at once).  A CTA fits one texel at a time.
// Small CTAs (64-256 threads) keep several texels in flight per SM, so that the
// serial FP64 step of one texel overlaps the pair passes of the others.
//
// Per texel: its luminance slab is staged into shared memory by one bulk TMA
// copy (cp.async.bulk, completion on an mbarrier, bounded wait); the next
// texel's copy is issued as soon as the current fit stops reading its slab.
// Per LM evaluation the CTA tabulates the direction-only terms of the model
// (svf_model.cuh) for the L directions, 16 floats per direction; then each warp
// walks its views and each lane keeps the table entries of its NC lights in
// registers, so a view's entry is four broadcast 16-byte loads used for NC
// pairs.  Jacobian passes accumulate the packed J^T J and J^T r in FP32 per
// thread and r^2 in FP64, reduced with warp shuffles and summed across warps
// in FP64.  One thread runs the LM control in FP64 (state in shared memory):
// the damped normal equations by Cholesky, the small-step and gradient tests
// and the gain-ratio accept/reject.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "svf_internal.h"
#include "svf_model.cuh"

namespace svf
{

namespace
{

constexpr int kEntry = 16;                   // floats per direction-table entry
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
__device__ bool lm_solve(LmState& st)
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
// shared memory and the direction table
// ------------------------------------------------------------------------------

// Per-texel-evaluation constants shared by every pair.
struct PassConst
{
    float u, v, rsx, rsy, ks, kd, ks_on, kd_on;
    float om[9];
};

__host__ __device__ inline uint32_t pad4(uint32_t x) { return (x + 3u) & ~3u; }

template <int THREADS>
struct Smem
{
    static constexpr int kWarps = THREADS / 32;
    // [Lp][kEntry] direction table | [stride] slab | partials | state
    __host__ __device__ static size_t tab_bytes(uint32_t L) { return sizeof(float) * kEntry * pad4(L); }
    __host__ __device__ static size_t slab_offset(uint32_t L) { return (tab_bytes(L) + 127) & ~size_t(127); }
    __host__ __device__ static size_t red_offset(uint32_t L, uint64_t stride)
    {
        return (slab_offset(L) + sizeof(float) * stride + 15) & ~size_t(15);
    }
    __host__ __device__ static size_t bytes(uint32_t L, uint64_t stride)
    {
        return red_offset(L, stride) + sizeof(float) * kWarps * kRed + sizeof(double) * kWarps;
    }
};

// Entry layout (16 floats): a0 a1 a2 sp | dsp0..3 | dsp4 kv up kdc | w0 w1 w2 0
__device__ __forceinline__ void build_table(float* tab, const float* geo, uint32_t L, const float* pf, PassConst* pc,
                                            int threads)
{
    ParamSet ps;
    make_param_set(pf, ps);
    for(uint32_t d = threadIdx.x; d < L; d += threads)
    {
        const float wx = geo[d], wy = geo[L + d], wz = geo[2 * L + d];
        DirEntry e;
        make_dir_entry(ps, wx, wy, wz, e);
        float4* t = reinterpret_cast<float4*>(tab + kEntry * d);
        t[0] = make_float4(e.a[0], e.a[1], e.a[2], e.sp);
        t[1] = make_float4(e.dsp[0], e.dsp[1], e.dsp[2], e.dsp[3]);
        t[2] = make_float4(e.dsp[4], ps.kspec * e.kv, e.up, e.kdc);
        t[3] = make_float4(wx, wy, wz, 0.0f);
    }
    if(threadIdx.x == 0)
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
    float a0, a1, a2, sp, d0, d1, d2, d3, d4, kv, up, kdc, w0, w1, w2;
};

__device__ __forceinline__ Entry load_entry(const float* tab, uint32_t d)
{
    const float4* t = reinterpret_cast<const float4*>(tab + kEntry * d);
    const float4 x = t[0], y = t[1], z = t[2], w = t[3];
    return Entry{ x.x, x.y, x.z, x.w, y.x, y.y, y.z, y.w, z.x, z.y, z.z, z.w, w.x, w.y, w.z };
}

// One pair: residual r = y - f and, for Jacobian passes, the gradient J of f
// (the factored model of svf_model.cuh with the per-view lobe constant folded
// into vo.kv).
template <bool kJac>
__device__ __forceinline__ float pair_eval(const PassConst& c, const Entry& li, const Entry& vo, float F, float y,
                                           float* J)
{
    const float W0 = li.w0 + vo.w0, W1 = li.w1 + vo.w1, W2 = li.w2 + vo.w2;
    const float g = W0 * W0 + W1 * W1 + W2 * W2;
    const float s0 = li.a0 + vo.a0, s1 = li.a1 + vo.a1, s2 = li.a2 + vo.a2;
    const float q0 = s0 * s0, q1 = s1 * s1;
    const float Q = c.u * q0 + c.v * q1 + s2 * s2;
    const float S = li.sp + vo.sp;
    const float QQS = Q * Q * S;
    const float rden = QQS > 0.0f ? __frcp_rn(QQS) : 0.0f;
    const float spec = vo.kv * li.up * F * g * g * rden;
    const float f = vo.up * (c.kd * li.kdc) + c.ks * spec;
    if(kJac)
    {
        const float A = c.ks * spec;
        const float rQ = Q * S * rden;
        const float rS = Q * Q * rden;
        const float t0 = s1 * s2 * (c.v - 1.0f);
        const float t1 = s0 * s2 * (1.0f - c.u);
        const float t2 = s0 * s1 * (c.u - c.v);
        J[0] = A * (c.rsx * (4.0f * c.u * q0 * rQ - 1.0f) - (li.d0 + vo.d0) * rS);
        J[1] = A * (c.rsy * (4.0f * c.v * q1 * rQ - 1.0f) - (li.d1 + vo.d1) * rS);
        J[2] = c.ks_on * spec;
        J[3] = c.kd_on * vo.up * li.kdc;
        const float m4 = -4.0f * rQ;
        const float dd[3] = { li.d2 + vo.d2, li.d3 + vo.d3, li.d4 + vo.d4 };
#pragma unroll
        for(int k = 0; k < 3; ++k)
        {
            const float dq = c.om[3 * k] * t0 + c.om[3 * k + 1] * t1 + c.om[3 * k + 2] * t2;
            J[4 + k] = A * (m4 * dq - dd[k] * rS);
        }
    }
    return y - f;
}

// One pass over the N pairs of the current texel; thread 0 receives the sums
// (J^T J, J^T r in out[0..34] for Jacobian passes; r^2 in out[35]).
template <int THREADS, int NC, bool kJac>
__device__ void pair_pass(const float* tab, const PassConst& c, const float* slab, uint32_t L, float refr, float* red,
                          double* redd, double* out)
{
    constexpr int kWarps = THREADS / 32;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const bool fresnel_on = refr != 1.0f;

    Entry le[NC];
    bool lv[NC];
#pragma unroll
    for(int k = 0; k < NC; ++k)
    {
        const uint32_t li = 32u * k + lane;
        lv[k] = li < L;
        le[k] = load_entry(tab, lv[k] ? li : 0u);
    }
    double r2 = 0.0;
    float acc[kJac ? kRed : 1];
#pragma unroll
    for(int i = 0; i < (kJac ? kRed : 1); ++i)
        acc[i] = 0.0f;

    for(uint32_t v = warp; v < L; v += kWarps)
    {
        const Entry vo = load_entry(tab, v);
        const float* row = slab + v * L + lane;
#pragma unroll
        for(int k = 0; k < NC; ++k)
        {
            if(!lv[k])
                continue;
            const float y = row[32 * k];
            float F = 1.0f;
            if(fresnel_on)
            {
                const float wi[3] = { le[k].w0, le[k].w1, le[k].w2 }, wo[3] = { vo.w0, vo.w1, vo.w2 };
                F = fresnel_factor(refr, wi, wo);
            }
            float J[kParams];
            const float r = pair_eval<kJac>(c, le[k], vo, F, y, J);
            r2 = fma((double)r, (double)r, r2);
            if(kJac)
            {
                int n = 0;
#pragma unroll
                for(int a = 0; a < kParams; ++a)
#pragma unroll
                    for(int b = a; b < kParams; ++b)
                    {
                        acc[n] = fmaf(J[a], J[b], acc[n]);
                        ++n;
                    }
#pragma unroll
                for(int a = 0; a < kParams; ++a)
                    acc[kHessian + a] = fmaf(J[a], r, acc[kHessian + a]);
            }
        }
    }

#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    if(kJac)
    {
#pragma unroll
        for(int i = 0; i < kRed; ++i)
        {
            float x = acc[i];
#pragma unroll
            for(int o = 16; o > 0; o >>= 1)
                x += __shfl_xor_sync(0xffffffffu, x, o);
            acc[i] = x;
        }
    }
    if(lane == 0)
    {
        redd[warp] = r2;
        if(kJac)
#pragma unroll
            for(int i = 0; i < kRed; ++i)
                red[warp * kRed + i] = acc[i];
    }
    __syncthreads();
    if(threadIdx.x == 0)
    {
        double s = 0.0;
#pragma unroll
        for(int w = 0; w < kWarps; ++w)
            s += redd[w];
        out[kRed] = s;
        if(kJac)
            for(int i = 0; i < kRed; ++i)
            {
                double t = 0.0;
#pragma unroll
                for(int w = 0; w < kWarps; ++w)
                    t += (double)red[w * kRed + i];
                out[i] = t;
            }
    }
}

// Resident CTAs per SM the register budget is sized for: with ~33 KB of shared
// memory per CTA at 81 directions, six 64-thread CTAs fit an SM.
constexpr int min_blocks(int threads) { return threads == 64 ? 6 : (threads == 128 ? 4 : 2); }

template <int THREADS, int NC>
__global__ void __launch_bounds__(THREADS, min_blocks(THREADS)) lm_fit_kernel(LmArgs args)
{
    using SM = Smem<THREADS>;
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float* tab = reinterpret_cast<float*>(smem_raw);
    float* slab = reinterpret_cast<float*>(smem_raw + SM::slab_offset(args.L));
    float* red = reinterpret_cast<float*>(smem_raw + SM::red_offset(args.L, args.lum_stride));
    double* redd = reinterpret_cast<double*>(red + SM::kWarps * kRed);

    __shared__ LmState st;
    __shared__ PassConst pc;
    __shared__ __align__(8) uint64_t bar;
    __shared__ float sh_pf[kParams];
    __shared__ int sh_cmd;
    __shared__ uint32_t sh_next;
    __shared__ double sh_out[kRed + 1];

    const uint32_t L = args.L;
    const double n_pairs = (double)args.N;
    const uint32_t slab_bytes = (uint32_t)(args.lum_stride * sizeof(float));
    const float* geo = args.geo;

    if(threadIdx.x == 0)
    {
        mbar_init(&bar, 1);
        const uint32_t t0 = atomicAdd(args.work_counter, 1u);
        if(t0 < args.texels)
            bulk_load(slab, args.lum + (uint64_t)t0 * args.lum_stride, slab_bytes, &bar);
        sh_next = t0;
    }
    __syncthreads();
    uint32_t phase = 0;
    uint32_t t = sh_next;

    while(t < args.texels)
    {
        if(!mbar_wait(&bar, phase))
        {
            // the copy did not land within the bound: flag it, give it one more
            // bounded wait, and leave
            if(threadIdx.x == 0)
            {
                atomicOr(args.error_flag, 1u);
                if(args.stats)
                    args.stats[t].status = SVF_TEXEL_TIMEOUT;
            }
            mbar_wait(&bar, phase);
            return;
        }
        phase ^= 1u;

        if(threadIdx.x == 0)
        {
#pragma unroll
            for(int i = 0; i < kParams; ++i)
            {
                st.p[i] = (double)args.init[(uint64_t)t * kParams + i];
                sh_pf[i] = (float)st.p[i];
            }
            st.iter = st.eff = st.njac = st.nres = st.status = 0;
            st.restarts_left = args.cfg.restarts;
        }
        __syncthreads();
        build_table(tab, geo, L, sh_pf, &pc, THREADS);
        __syncthreads();
        pair_pass<THREADS, NC, true>(tab, pc, slab, L, args.cfg.fresnel, red, redd, sh_out);
        if(threadIdx.x == 0)
        {
            st.njac = 1;
            st.S = sh_out[kRed];
#pragma unroll
            for(int i = 0; i < kParams; ++i)
                st.g[i] = -sh_out[kHessian + i];
#pragma unroll
            for(int i = 0; i < kHessian; ++i)
                st.H[i] = sh_out[i];
            lm_reset_damping(st);
            if(!isfinite(st.S))
                st.status |= SVF_TEXEL_NONFINITE;
        }
        for(;;)
        {
            if(threadIdx.x == 0)
            {
                const int cmd = lm_next(st, args.cfg, n_pairs);
                if(cmd == kCmdTrial)
#pragma unroll
                    for(int i = 0; i < kParams; ++i)
                        sh_pf[i] = (float)st.pt[i];
                sh_cmd = cmd;
            }
            __syncthreads();
            if(sh_cmd == kCmdDone)
                break;
            build_table(tab, geo, L, sh_pf, &pc, THREADS);
            __syncthreads();
            pair_pass<THREADS, NC, false>(tab, pc, slab, L, args.cfg.fresnel, red, redd, sh_out);
            if(threadIdx.x == 0)
                sh_cmd = lm_after_trial(st, args.cfg, sh_out[kRed], n_pairs);
            __syncthreads();
            const int cmd = sh_cmd;
            if(cmd == kCmdDone)
                break;
            if(cmd == kCmdJacobian)
            {
                // the table built for the trial point is the accepted point's
                pair_pass<THREADS, NC, true>(tab, pc, slab, L, args.cfg.fresnel, red, redd, sh_out);
                if(threadIdx.x == 0)
                    sh_cmd = lm_after_jacobian(st, args.cfg, sh_out, n_pairs);
                __syncthreads();
                if(sh_cmd == kCmdDone)
                    break;
            }
        }

        // The slab is no longer read: start the next texel's copy, then write the
        // outputs (LeastSquaresFitSGGX :381-429, SVBRDFFitPipeline::fit :692-697).
        if(threadIdx.x == 0)
        {
            const uint32_t tn = atomicAdd(args.work_counter, 1u);
            if(tn < args.texels)
                bulk_load(slab, args.lum + (uint64_t)tn * args.lum_stride, slab_bytes, &bar);
            sh_next = tn;

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
        __syncthreads();
        t = sh_next;
    }
}

using KernelFn = void (*)(LmArgs);

template <int THREADS>
KernelFn pick_nc(int nc)
{
    switch(nc)
    {
    case 1: return lm_fit_kernel<THREADS, 1>;
    case 2: return lm_fit_kernel<THREADS, 2>;
    case 3: return lm_fit_kernel<THREADS, 3>;
    case 4: return lm_fit_kernel<THREADS, 4>;
    case 5: return lm_fit_kernel<THREADS, 5>;
    default: return nullptr;
    }
}

KernelFn kernel_for(LmKernelChoice c)
{
    switch(c.threads)
    {
    case 64: return pick_nc<64>(c.nc);
    case 128: return pick_nc<128>(c.nc);
    case 256: return pick_nc<256>(c.nc);
    default: return nullptr;
    }
}

} // namespace

LmKernelChoice lm_default_choice(uint32_t L)
{
    return LmKernelChoice{ 64, (int)((L + 31) / 32) };
}

int lm_candidates(uint32_t L, LmKernelChoice* out, int max)
{
    const int nc = (int)((L + 31) / 32);
    const int threads[3] = { 64, 128, 256 };
    int n = 0;
    for(int i = 0; i < 3 && n < max; ++i)
        out[n++] = LmKernelChoice{ threads[i], nc };
    return n;
}

size_t lm_smem_bytes(uint32_t L, uint64_t lum_stride, LmKernelChoice c)
{
    switch(c.threads)
    {
    case 64: return Smem<64>::bytes(L, lum_stride);
    case 128: return Smem<128>::bytes(L, lum_stride);
    default: return Smem<256>::bytes(L, lum_stride);
    }
}

int lm_max_ctas_per_sm(uint32_t L, uint64_t lum_stride, LmKernelChoice c)
{
    KernelFn k = kernel_for(c);
    if(!k || (uint32_t)c.nc * 32u < L)
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
    KernelFn k = kernel_for(c);
    if(!k || (uint32_t)c.nc * 32u < args.L)
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
