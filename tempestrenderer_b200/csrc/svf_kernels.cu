// svf_kernels.cu - luminance slice, the persistent Levenberg-Marquardt fit and
// the synthetic BTF renderer, for sm_100a.
//
// The LM kernel is persistent: a grid of (resident CTAs per SM) x (SMs) CTAs
// pulls texels from a global atomic counter (work stealing; a texel that
// converges early frees its CTA at once).  Each CTA fits one texel at a time
// with 256 threads.  The texel's luminance slab is staged into shared memory by
// one bulk TMA copy (cp.async.bulk, completion on an mbarrier), double-buffered:
// the next texel's slab streams in while the current one is fitted.  Per LM
// evaluation the CTA tabulates the direction-only terms of the model
// (svf_model.cuh) for the L directions, then every warp walks the pairs of its
// views with lanes spread over lights, accumulating r^2 (FP64) and the packed
// J^T J and J^T r (FP32 per thread, FP64 across warps).  One thread runs the LM
// control in FP64: damped normal equations by Cholesky, the small-step and
// gradient tests and the gain-ratio accept/reject of fitting.hh:457-678.
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <stdint.h>

#include <algorithm>
#include <mutex>

#include "svf_internal.h"
#include "svf_model.cuh"

namespace svf
{

namespace
{

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kRed = 36;                     // 28 (J^T J) + 7 (J^T r) + r^2
constexpr int kTabFields = 13;               // DirEntry fields kept in shared memory
constexpr uint32_t kWaitSpins = 1u << 22;    // bound of every mbarrier wait

enum : int
{
    kCmdTrial = 0,
    kCmdJacobian = 1,
    kCmdDone = 2,
    kCmdContinue = 3
};

// ------------------------------------------------------------------------------
// mbarrier + bulk copy (TMA) helpers
// ------------------------------------------------------------------------------

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Arms `bar` for `bytes` and starts one bulk copy global -> shared.
// dst, src 16-byte aligned; bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar)
{
    uint32_t b = smem_addr(bar);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_addr(dst)), "l"(src), "r"(bytes), "r"(b)
                 : "memory");
}

// Bounded wait for phase `parity` of `bar`; false when the bound expired.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity)
{
    uint32_t b = smem_addr(bar);
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
// FP64 LM control (thread 0 only)
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
    for(int i = 0; i < kParams; ++i)
        damping = fmax(damping, st.H[hidx(i, i)]);
    st.lam = damping * 0.75;   // InitialDampingMultiplier
    st.nu = 2.0;               // DampingFailureMultiplier
}

// Where the reference's loop ends, optionally continue once more with fresh
// damping from the same point; false when the fit is finished.
__device__ __forceinline__ bool lm_restart(LmState& st, const LmConfig& cfg, double n_pairs)
{
    if(st.restarts_left == 0 || !(st.iter < cfg.max_iter && cfg.mse_target < st.S / n_pairs))
        return false;
    --st.restarts_left;
    lm_reset_damping(st);
    return true;
}

// In-place Cholesky of a packed 7x7 SPD matrix; false unless every pivot is
// positive and finite.
__device__ bool cholesky7(double* A)
{
    for(int j = 0; j < kParams; ++j)
    {
        double s = A[hidx(j, j)];
        for(int k = 0; k < j; ++k)
        {
            double l = A[hidx(j, k)];
            s -= l * l;
        }
        if(!(s > 0.0) || !isfinite(s))
            return false;
        double ljj = sqrt(s);
        A[hidx(j, j)] = ljj;
        double r = 1.0 / ljj;
        for(int i = j + 1; i < kParams; ++i)
        {
            double t = A[hidx(i, j)];
            for(int k = 0; k < j; ++k)
                t -= A[hidx(i, k)] * A[hidx(j, k)];
            A[hidx(i, j)] = t * r;
        }
    }
    return true;
}

__device__ void cholesky7_solve(const double* Lm, const double* b, double* x)
{
    double y[kParams];
    for(int i = 0; i < kParams; ++i)
    {
        double t = b[i];
        for(int k = 0; k < i; ++k)
            t -= Lm[hidx(i, k)] * y[k];
        y[i] = t / Lm[hidx(i, i)];
    }
    for(int i = kParams - 1; i >= 0; --i)
    {
        double t = y[i];
        for(int k = i + 1; k < kParams; ++k)
            t -= Lm[hidx(k, i)] * x[k];
        x[i] = t / Lm[hidx(i, i)];
    }
}

// Damped step (H + lam I) d = g by Cholesky.  Active set at the bound: a
// parameter with a lower bound (sigma, specular, diffuse) that sits exactly at 0
// and whose step points below it is held at 0 for this solve (its row and
// column are dropped) and the system is solved again.  The reference instead
// rejects every such step (AcceptStepConstraints), which with an exact
// derivative would hold the parameter at 0 for good; its finite-difference
// derivative at exactly 0 (fitting.hh:896-905, step 1e-8) is below float
// resolution there.  Returns false when the factorisation fails.
__device__ bool lm_solve(LmState& st)
{
    uint32_t frozen = 0;
    for(int round = 0; round < 5; ++round)
    {
        double A[kHessian], b[kParams];
        for(int i = 0; i < kHessian; ++i)
            A[i] = st.H[i];
        for(int i = 0; i < kParams; ++i)
        {
            A[hidx(i, i)] += st.lam;
            b[i] = st.g[i];
        }
        for(int i = 0; i < 4; ++i)
            if(frozen & (1u << i))
            {
                for(int j = 0; j < kParams; ++j)
                    if(j != i)
                        A[hidx(i, j)] = 0.0;
                b[i] = 0.0;
            }
        if(!cholesky7(A))
            return false;
        cholesky7_solve(A, b, st.d);
        uint32_t more = frozen;
        for(int i = 0; i < 4; ++i)
            if(st.p[i] == 0.0 && st.d[i] > 0.0)
                more |= 1u << i;
        if(more == frozen)
            return true;
        frozen = more;
    }
    return true;
}

// The top of one LM iteration (fitting.hh:541-590): solve for a step that passes
// the constraints, or finish.  Returns kCmdTrial (st.pt holds the trial point)
// or kCmdDone.
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
        for(int i = 0; i < kParams; ++i)
        {
            step2 += st.d[i] * st.d[i];
            double t = st.p[i] + cfg.eps;
            mag2 += t * t;
        }
        double step_len = sqrt(step2);
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
    for(int i = 0; i < kParams; ++i)
        pred += st.d[i] * (st.d[i] * st.lam + st.g[i]);
    pred *= 0.5;
    double rho = 0.5 * (st.S - S1) / pred;
    if(rho > 0.0)
    {
        ++st.eff;
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
    for(int i = 0; i < kParams; ++i)
    {
        st.g[i] = -red[kHessian + i];
        glen += st.g[i] * st.g[i];
    }
    for(int i = 0; i < kHessian; ++i)
        st.H[i] = red[i];
    if(glen <= cfg.eps * cfg.eps)
        return lm_restart(st, cfg, n_pairs) ? kCmdContinue : kCmdDone;
    const double min_mul = (double)(1.0f / 3.0f);
    double t = 2.0 * st.rho - 1.0;
    double mul = fmax(min_mul, 1.0 - t * t * t);
    st.lam *= mul;
    st.nu = 2.0;
    ++st.iter;
    return kCmdContinue;
}

// ------------------------------------------------------------------------------
// shared-memory layout of the LM kernel
// ------------------------------------------------------------------------------

struct LmShared
{
    float*  geo;     // [3][Lp]
    float*  tab;     // [kTabFields][Lp]
    float*  lum[2];  // [lum_stride] each
    float*  red;     // [kWarps][kRed]
    double* redd;    // [kWarps]
    uint64_t* bar;   // [2]
    uint32_t Lp;
};

__host__ __device__ inline uint32_t pad4(uint32_t x) { return (x + 3u) & ~3u; }

__host__ __device__ inline size_t lm_smem_layout(uint32_t L, uint64_t lum_stride, size_t* off_tab, size_t* off_lum,
                                                 size_t* off_red, size_t* off_redd, size_t* off_bar)
{
    uint32_t Lp = pad4(L);
    size_t o = 0;
    o += sizeof(float) * 3 * Lp;
    *off_tab = o;
    o += sizeof(float) * kTabFields * Lp;
    o = (o + 127) & ~size_t(127);
    *off_lum = o;
    o += sizeof(float) * 2 * lum_stride;
    o = (o + 15) & ~size_t(15);
    *off_red = o;
    o += sizeof(float) * kWarps * kRed;
    o = (o + 7) & ~size_t(7);
    *off_redd = o;
    o += sizeof(double) * kWarps;
    *off_bar = o;
    o += sizeof(uint64_t) * 2;
    return o;
}

// Tabulates DirEntry for every direction for the parameters in `pf`.
__device__ __forceinline__ void build_table(const LmShared& sh, const float* pf, uint32_t L)
{
    ParamSet ps;
    make_param_set(pf, ps);
    for(uint32_t d = threadIdx.x; d < L; d += kThreads)
    {
        DirEntry e;
        make_dir_entry(ps, sh.geo[d], sh.geo[sh.Lp + d], sh.geo[2 * sh.Lp + d], e);
        float* t = sh.tab + d;
        const uint32_t s = sh.Lp;
        t[0 * s] = e.a[0];
        t[1 * s] = e.a[1];
        t[2 * s] = e.a[2];
        t[3 * s] = e.sp;
        t[4 * s] = e.dsp[0];
        t[5 * s] = e.dsp[1];
        t[6 * s] = e.dsp[2];
        t[7 * s] = e.dsp[3];
        t[8 * s] = e.dsp[4];
        t[9 * s] = e.kdc;
        t[10 * s] = e.kv;
        t[11 * s] = e.up;
    }
}

__device__ __forceinline__ void load_entry(const LmShared& sh, uint32_t d, DirEntry& e, float* w)
{
    const float* t = sh.tab + d;
    const uint32_t s = sh.Lp;
    e.a[0] = t[0 * s];
    e.a[1] = t[1 * s];
    e.a[2] = t[2 * s];
    e.sp = t[3 * s];
    e.dsp[0] = t[4 * s];
    e.dsp[1] = t[5 * s];
    e.dsp[2] = t[6 * s];
    e.dsp[3] = t[7 * s];
    e.dsp[4] = t[8 * s];
    e.kdc = t[9 * s];
    e.kv = t[10 * s];
    e.up = t[11 * s];
    w[0] = sh.geo[d];
    w[1] = sh.geo[s + d];
    w[2] = sh.geo[2 * s + d];
}

// One pass over the N pairs of the current texel.  Warps own views
// (v = warp, warp + kWarps, ...), lanes own lights (chunks of 32), so a view's
// table entry is a broadcast read and a light's entry stays in registers for
// the whole chunk.  Jacobian passes reduce r^2, J^T J and J^T r into `out`
// (thread 0 only); residual passes reduce r^2.
template <bool kJacobian>
__device__ void pair_pass(const LmShared& sh, const float* lum, const float* pf, uint32_t L, float refr,
                          double* out)
{
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    ParamSet ps;
    make_param_set(pf, ps);
    const bool fresnel_on = refr != 1.0f;

    double r2 = 0.0;
    float acc[kJacobian ? kHessian + kParams : 1];
#pragma unroll
    for(int i = 0; i < (kJacobian ? kHessian + kParams : 1); ++i)
        acc[i] = 0.0f;

    for(uint32_t base = 0; base < L; base += 32)
    {
        const uint32_t li = base + lane;
        const bool valid = li < L;
        DirEntry le;
        float wi[3];
        load_entry(sh, valid ? li : 0, le, wi);
        for(uint32_t v = warp; v < L; v += kWarps)
        {
            DirEntry ve;
            float wo[3];
            load_entry(sh, v, ve, wo);
            if(!valid)
                continue;
            const float y = lum[v * L + li];
            const float F = fresnel_on ? fresnel_factor(refr, wi, wo) : 1.0f;
            float J[kParams];
            const float f = eval_pair<kJacobian>(ps, wi, le, wo, ve, F, J);
            const float r = y - f;
            r2 = fma((double)r, (double)r, r2);
            if(kJacobian)
            {
                int k = 0;
#pragma unroll
                for(int a = 0; a < kParams; ++a)
                {
#pragma unroll
                    for(int b = a; b < kParams; ++b)
                    {
                        acc[k] = fmaf(J[a], J[b], acc[k]);
                        ++k;
                    }
                }
#pragma unroll
                for(int a = 0; a < kParams; ++a)
                    acc[kHessian + a] = fmaf(J[a], r, acc[kHessian + a]);
            }
        }
    }

    // warp reduction, then across warps in FP64
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
        r2 += __shfl_xor_sync(0xffffffffu, r2, o);
    if(kJacobian)
    {
#pragma unroll
        for(int i = 0; i < kHessian + kParams; ++i)
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
        sh.redd[warp] = r2;
        if(kJacobian)
            for(int i = 0; i < kHessian + kParams; ++i)
                sh.red[warp * kRed + i] = acc[i];
    }
    __syncthreads();
    if(threadIdx.x == 0)
    {
        double s = 0.0;
        for(int w = 0; w < kWarps; ++w)
            s += sh.redd[w];
        out[kHessian + kParams] = s;
        if(kJacobian)
            for(int i = 0; i < kHessian + kParams; ++i)
            {
                double t = 0.0;
                for(int w = 0; w < kWarps; ++w)
                    t += (double)sh.red[w * kRed + i];
                out[i] = t;
            }
    }
}

__global__ void __launch_bounds__(kThreads) lm_fit_kernel(LmArgs args)
{
    extern __shared__ __align__(128) unsigned char smem_raw[];
    size_t off_tab, off_lum, off_red, off_redd, off_bar;
    lm_smem_layout(args.L, args.lum_stride, &off_tab, &off_lum, &off_red, &off_redd, &off_bar);
    LmShared sh;
    sh.Lp = pad4(args.L);
    sh.geo = reinterpret_cast<float*>(smem_raw);
    sh.tab = reinterpret_cast<float*>(smem_raw + off_tab);
    sh.lum[0] = reinterpret_cast<float*>(smem_raw + off_lum);
    sh.lum[1] = sh.lum[0] + args.lum_stride;
    sh.red = reinterpret_cast<float*>(smem_raw + off_red);
    sh.redd = reinterpret_cast<double*>(smem_raw + off_redd);
    sh.bar = reinterpret_cast<uint64_t*>(smem_raw + off_bar);

    __shared__ float sh_pf[kParams];
    __shared__ int sh_cmd;
    __shared__ uint32_t sh_next;
    __shared__ double sh_red_out[kHessian + kParams + 1];

    const uint32_t L = args.L, N = args.N;
    const uint32_t slab_bytes = (uint32_t)(args.lum_stride * sizeof(float));
    for(uint32_t i = threadIdx.x; i < 3 * sh.Lp; i += kThreads)
    {
        uint32_t c = i / sh.Lp, d = i % sh.Lp;
        sh.geo[i] = d < L ? args.geo[c * L + d] : 0.0f;
    }
    if(threadIdx.x == 0)
    {
        mbar_init(&sh.bar[0], 1);
        mbar_init(&sh.bar[1], 1);
        fence_barrier_init();
        uint32_t t0 = atomicAdd(args.work_counter, 1u);
        if(t0 < args.texels)
            bulk_load(sh.lum[0], args.lum + (uint64_t)t0 * args.lum_stride, slab_bytes, &sh.bar[0]);
        sh_next = t0;
    }
    __syncthreads();

    uint32_t t = sh_next;
    uint32_t buf = 0;
    uint32_t phase[2] = { 0u, 0u };
    const double n_pairs = (double)N;
    LmState st;   // meaningful in thread 0 only

    while(t < args.texels)
    {
        __syncthreads();   // everyone has read sh_next
        if(threadIdx.x == 0)
        {
            uint32_t tn = atomicAdd(args.work_counter, 1u);
            if(tn < args.texels)
            {
                fence_proxy_async();
                bulk_load(sh.lum[buf ^ 1u], args.lum + (uint64_t)tn * args.lum_stride, slab_bytes, &sh.bar[buf ^ 1u]);
            }
            sh_next = tn;
        }
        const bool arrived = mbar_wait(&sh.bar[buf], phase[buf]);
        phase[buf] ^= 1u;
        if(!arrived)
        {
            // The copy did not land within the bound: flag it, give the copies in
            // flight one more bounded wait, and leave.
            if(threadIdx.x == 0)
            {
                atomicOr(args.error_flag, 1u);
                if(args.stats)
                    args.stats[t].status = SVF_TEXEL_TIMEOUT;
            }
            mbar_wait(&sh.bar[buf], phase[buf] ^ 1u);
            mbar_wait(&sh.bar[buf ^ 1u], phase[buf ^ 1u]);
            return;
        }
        const float* lum = sh.lum[buf];

        // ---- fit texel t ----
        if(threadIdx.x == 0)
        {
            for(int i = 0; i < kParams; ++i)
            {
                st.p[i] = (double)args.init[(uint64_t)t * kParams + i];
                sh_pf[i] = (float)st.p[i];
            }
            st.iter = st.eff = st.njac = st.nres = st.status = 0;
        }
        __syncthreads();
        build_table(sh, sh_pf, L);
        __syncthreads();
        pair_pass<true>(sh, lum, sh_pf, L, args.cfg.fresnel, sh_red_out);
        if(threadIdx.x == 0)
        {
            st.njac = 1;
            st.restarts_left = args.cfg.restarts;
            st.S = sh_red_out[kHessian + kParams];
            for(int i = 0; i < kParams; ++i)
                st.g[i] = -sh_red_out[kHessian + i];
            for(int i = 0; i < kHessian; ++i)
                st.H[i] = sh_red_out[i];
            lm_reset_damping(st);
            if(!isfinite(st.S))
                st.status |= SVF_TEXEL_NONFINITE;
        }
        for(;;)
        {
            if(threadIdx.x == 0)
            {
                int cmd = lm_next(st, args.cfg, n_pairs);
                if(cmd == kCmdTrial)
                    for(int i = 0; i < kParams; ++i)
                        sh_pf[i] = (float)st.pt[i];
                sh_cmd = cmd;
            }
            __syncthreads();
            if(sh_cmd == kCmdDone)
                break;
            build_table(sh, sh_pf, L);
            __syncthreads();
            pair_pass<false>(sh, lum, sh_pf, L, args.cfg.fresnel, sh_red_out);
            if(threadIdx.x == 0)
                sh_cmd = lm_after_trial(st, args.cfg, sh_red_out[kHessian + kParams], n_pairs);
            __syncthreads();
            const int cmd = sh_cmd;
            if(cmd == kCmdDone)
                break;
            if(cmd == kCmdJacobian)
            {
                // the table built for the trial point is the accepted point's
                pair_pass<true>(sh, lum, sh_pf, L, args.cfg.fresnel, sh_red_out);
                if(threadIdx.x == 0)
                    sh_cmd = lm_after_jacobian(st, args.cfg, sh_red_out, n_pairs);
                __syncthreads();
                if(sh_cmd == kCmdDone)
                    break;
            }
        }

        // ---- outputs (LeastSquaresFitSGGX :381-429, SVBRDFFitPipeline::fit :692-697) ----
        if(threadIdx.x == 0)
        {
            float pout[kParams];
            for(int i = 0; i < kParams; ++i)
            {
                pout[i] = (float)st.p[i];
                args.out[(uint64_t)t * kParams + i] = pout[i];
            }
            double mse = st.S / n_pairs;
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
                for(int c = 0; c < 3; ++c)
                {
                    if(args.map_diffuse)
                        args.map_diffuse[3 * (uint64_t)t + c] = a[c] * pout[3];
                    if(args.map_specular)
                        args.map_specular[3 * (uint64_t)t + c] = a[c] * pout[2];
                }
            }
        }
        __syncthreads();
        t = sh_next;
        buf ^= 1u;
    }
}

// ------------------------------------------------------------------------------
// luminance slice
// ------------------------------------------------------------------------------

template <typename T>
__device__ __forceinline__ float to_f(T x);
template <>
__device__ __forceinline__ float to_f<float>(float x) { return x; }
template <>
__device__ __forceinline__ float to_f<__half>(__half x) { return __half2float(x); }

// One CTA per texel.  lum = 0.2126 R + 0.7152 G + 0.0722 B (spectrum.hh:328-331,
// evaluated without fused multiply-adds, as the reference's x86-64 build does);
// chromaticity rgb/lum, or (1,1,1) when lum <= 1e-6, averaged over the pairs.
template <typename T>
__global__ void __launch_bounds__(256) luminance_kernel(const T* __restrict__ samples, uint32_t N, float* __restrict__ lum,
                                                         uint64_t lum_stride, float* __restrict__ avg)
{
    const uint64_t t = blockIdx.x;
    const T* src = samples + t * (uint64_t)N * 3;
    float* dst = lum + t * lum_stride;
    float ax = 0.0f, ay = 0.0f, az = 0.0f;
    for(uint32_t i = threadIdx.x; i < N; i += blockDim.x)
    {
        float r = to_f(src[3 * i]), g = to_f(src[3 * i + 1]), b = to_f(src[3 * i + 2]);
        float l = __fadd_rn(__fadd_rn(__fmul_rn(0.2126f, r), __fmul_rn(0.7152f, g)), __fmul_rn(0.0722f, b));
        dst[i] = l;
        if(l > 1e-6f)
        {
            float rl = 1.0f / l;
            ax += r * rl;
            ay += g * rl;
            az += b * rl;
        }
        else
        {
            ax += 1.0f;
            ay += 1.0f;
            az += 1.0f;
        }
    }
    for(uint32_t i = N + threadIdx.x; i < lum_stride; i += blockDim.x)
        dst[i] = 0.0f;
    __shared__ float red[3][8];
#pragma unroll
    for(int o = 16; o > 0; o >>= 1)
    {
        ax += __shfl_xor_sync(0xffffffffu, ax, o);
        ay += __shfl_xor_sync(0xffffffffu, ay, o);
        az += __shfl_xor_sync(0xffffffffu, az, o);
    }
    const uint32_t warp = threadIdx.x >> 5;
    if((threadIdx.x & 31u) == 0)
    {
        red[0][warp] = ax;
        red[1][warp] = ay;
        red[2][warp] = az;
    }
    __syncthreads();
    if(threadIdx.x < 3)
    {
        float s = 0.0f;
        for(uint32_t w = 0; w < blockDim.x / 32; ++w)
            s += red[threadIdx.x][w];
        // Vector3 / float multiplies by the reciprocal (vector3.hh:185-190)
        avg[3 * t + threadIdx.x] = s * (1.0f / (float)N);
    }
}

__global__ void repack_kernel(const float* __restrict__ src, uint64_t src_stride, uint32_t N, float* __restrict__ dst,
                              uint64_t dst_stride)
{
    const uint64_t t = blockIdx.x;
    for(uint32_t i = threadIdx.x; i < dst_stride; i += blockDim.x)
        dst[t * dst_stride + i] = i < N ? src[t * src_stride + i] : 0.0f;
}

// ------------------------------------------------------------------------------
// synthetic BTF (mirrors svfo_synth_truth / svfo_synth_render of the oracle)
// ------------------------------------------------------------------------------

__device__ __forceinline__ void philox(uint32_t k0, uint32_t k1, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                       uint32_t* out)
{
#pragma unroll
    for(int r = 0; r < 10; ++r)
    {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

__device__ __forceinline__ float u01(uint32_t r) { return (float)(r >> 8) * (1.0f / 16777216.0f); }
__device__ __forceinline__ float loguni(float a, float b, float u) { return a * expf(u * logf(b / a)); }

struct Truth
{
    float kd[3], ks[3], sigma[2], quat[4], euler[3], kind;
};

__device__ void synth_truth(uint32_t seed, uint32_t mix, uint64_t texel, Truth& t)
{
    uint32_t b0[4], b1[4], b2[4];
    const uint32_t lo = (uint32_t)texel, hi = (uint32_t)(texel >> 32);
    philox(seed, 0x53564631u, lo, hi, 0, 0, b0);
    philox(seed, 0x53564631u, lo, hi, 1, 0, b1);
    philox(seed, 0x53564631u, lo, hi, 2, 0, b2);
    float uk = u01(b0[0]);
    uint32_t kind = 0;
    if(mix == 1)
        kind = uk < 0.2f ? 1u : (uk < 0.3f ? 2u : 0u);
    t.kind = (float)kind;
    for(int c = 0; c < 3; ++c)
        t.kd[c] = 0.8f * u01(b0[1 + c]);
    for(int c = 0; c < 3; ++c)
        t.ks[c] = (kind == 1 ? 0.05f : 1.0f) * u01(b1[c]);
    if(kind == 2)
    {
        float smin = loguni(0.01f, 0.05f, u01(b1[3]));
        float ratio = loguni(8.5f, 16.0f, u01(b2[0]));
        float smax = smin * ratio;
        t.sigma[0] = smax < 0.8f ? smax : 0.8f;
        t.sigma[1] = smin;
    }
    else
    {
        t.sigma[0] = loguni(0.02f, 0.8f, u01(b1[3]));
        t.sigma[1] = loguni(0.02f, 0.8f, u01(b2[0]));
    }
    const float cos30 = 0.866025403784f, two_pi = 6.283185307179586f;
    float nz = 1.0f - u01(b2[1]) * (1.0f - cos30);
    float nr = sqrtf(fmaxf(0.0f, 1.0f - nz * nz));
    float phi = two_pi * u01(b2[2]), psi = two_pi * u01(b2[3]);
    float n[3] = { nr * cosf(phi), nr * sinf(phi), nz };
    float t0[3] = { 1.0f - n[0] * n[0], -n[1] * n[0], -n[2] * n[0] };
    float l0 = sqrtf(t0[0] * t0[0] + t0[1] * t0[1] + t0[2] * t0[2]);
    float rl0 = 1.0f / l0;
    t0[0] *= rl0; t0[1] *= rl0; t0[2] *= rl0;
    float b0v[3] = { n[1] * t0[2] - n[2] * t0[1], n[2] * t0[0] - n[0] * t0[2], n[0] * t0[1] - n[1] * t0[0] };
    float cp = cosf(psi), sp = sinf(psi);
    float tt[3] = { t0[0] * cp + b0v[0] * sp, t0[1] * cp + b0v[1] * sp, t0[2] * cp + b0v[2] * sp };
    float bb[3] = { n[1] * tt[2] - n[2] * tt[1], n[2] * tt[0] - n[0] * tt[2], n[0] * tt[1] - n[1] * tt[0] };
    float m00 = tt[0], m01 = tt[1], m02 = tt[2], m10 = bb[0], m11 = bb[1], m12 = bb[2], m20 = n[0], m21 = n[1], m22 = n[2];
    float q[4];
    float tr = m00 + m11 + m22;
    if(tr > 0.0f)
    {
        float s = sqrtf(tr + 1.0f) * 2.0f;
        q[3] = 0.25f * s; q[0] = (m12 - m21) / s; q[1] = (m20 - m02) / s; q[2] = (m01 - m10) / s;
    }
    else if(m00 > m11 && m00 > m22)
    {
        float s = sqrtf(1.0f + m00 - m11 - m22) * 2.0f;
        q[3] = (m12 - m21) / s; q[0] = 0.25f * s; q[1] = (m01 + m10) / s; q[2] = (m02 + m20) / s;
    }
    else if(m11 > m22)
    {
        float s = sqrtf(1.0f + m11 - m00 - m22) * 2.0f;
        q[3] = (m20 - m02) / s; q[0] = (m01 + m10) / s; q[1] = 0.25f * s; q[2] = (m12 + m21) / s;
    }
    else
    {
        float s = sqrtf(1.0f + m22 - m00 - m11) * 2.0f;
        q[3] = (m01 - m10) / s; q[0] = (m02 + m20) / s; q[1] = (m12 + m21) / s; q[2] = 0.25f * s;
    }
    float ql = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for(int i = 0; i < 4; ++i)
        t.quat[i] = q[i] / ql;
    // Matrix3::decompose of ToMatrix3(quat) (matrix3.hh:311-332)
    const float x = t.quat[0], y = t.quat[1], z = t.quat[2], w = t.quat[3];
    float C0[3] = { 1.0f - 2.0f * (y * y + z * z), 2.0f * (x * y + z * w), 2.0f * (x * z - y * w) };
    float C1[3] = { 2.0f * (x * y - z * w), 1.0f - 2.0f * (x * x + z * z), 2.0f * (y * z + x * w) };
    float C2[3] = { 2.0f * (x * z + y * w), 2.0f * (y * z - x * w), 1.0f - 2.0f * (x * x + y * y) };
    float sc0 = sqrtf(C0[0] * C0[0] + C0[1] * C0[1] + C0[2] * C0[2]);
    float sc1 = sqrtf(C1[0] * C1[0] + C1[1] * C1[1] + C1[2] * C1[2]);
    float sc2 = sqrtf(C2[0] * C2[0] + C2[1] * C2[1] + C2[2] * C2[2]);
    float m20d = C2[0] / sc2;
    const float half_pi = kRefPi * 0.5f;
    if(m20d >= 0.9999f)
    {
        t.euler[0] = 0.0f; t.euler[1] = half_pi; t.euler[2] = atan2f(C0[1], C1[1]);
    }
    else if(m20d <= -0.9999f)
    {
        t.euler[0] = 0.0f; t.euler[1] = -half_pi; t.euler[2] = atan2f(C0[1], C1[1]);
    }
    else
    {
        t.euler[0] = atan2f(-C2[1], C2[2]);
        t.euler[1] = asinf(m20d);
        t.euler[2] = atan2f(-C1[0] / sc1, C0[0] / sc0);
    }
}

__device__ __forceinline__ float surface_brdf_rgb(float kd, float ks, float sx, float sy, const float* R, float out_density,
                                                  const float* wi, const float* wo)
{
    // SGGXMicroFlakeSurfaceBRDF in the reference's operation order (Fresnel 1)
    float dot_inc = wi[2], dot_out = wo[2];
    if(dot_inc < 0.0f || dot_out < 0.0f)
        return 0.0f;
    float result = kd * dot_inc * (1.0f / kRefPi);
    if(sx >= 1e-6f && sy >= 1e-6f && out_density >= 1e-6f)
    {
        float h[3] = { wi[0] + wo[0], wi[1] + wo[1], wi[2] + wo[2] };
        float hl = sqrtf(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
        float rh = 1.0f / hl;
        h[0] *= rh; h[1] *= rh; h[2] *= rh;
        float ai[3], ah[3];
        for(int c = 0; c < 3; ++c)
        {
            ai[c] = R[3 * c] * wi[0] + R[3 * c + 1] * wi[1] + R[3 * c + 2] * wi[2];
            ah[c] = R[3 * c] * h[0] + R[3 * c + 1] * h[1] + R[3 * c + 2] * h[2];
        }
        float in_density = sqrtf(sx * sx * ai[0] * ai[0] + sy * sy * ai[1] * ai[1] + ai[2] * ai[2]);
        float u = 1.0f / (sx * sx), v = 1.0f / (sy * sy);
        float det = u * v;
        float ndf = 0.0f;
        if(det >= 1e-6f)
        {
            float den = u * ah[0] * ah[0] + v * ah[1] * ah[1] + ah[2] * ah[2];
            ndf = 0.5f * sqrtf(det) / (kRefPi * den * den);
        }
        float contrib = 1.0f / (out_density + in_density * dot_out / dot_inc);
        result += contrib * ks * ndf * 2.0f / 4.0f;
    }
    return result;
}

// One CTA (256 threads) per texel.
template <typename T>
__global__ void __launch_bounds__(256) synth_kernel(uint32_t seed, uint32_t mix, const float* __restrict__ lp, uint32_t L,
                                                     uint64_t first, float noise, T* __restrict__ samples,
                                                     float* __restrict__ truth)
{
    __shared__ Truth tr;
    __shared__ float R[9];
    __shared__ float w[3][160];
    __shared__ float dens[160];
    const uint64_t texel = first + blockIdx.x;
    if(threadIdx.x == 0)
    {
        synth_truth(seed, mix, texel, tr);
        const float x = tr.quat[0], y = tr.quat[1], z = tr.quat[2], ww = tr.quat[3];
        R[0] = 1.0f - 2.0f * (y * y + z * z); R[1] = 2.0f * (x * y + z * ww); R[2] = 2.0f * (x * z - y * ww);
        R[3] = 2.0f * (x * y - z * ww); R[4] = 1.0f - 2.0f * (x * x + z * z); R[5] = 2.0f * (y * z + x * ww);
        R[6] = 2.0f * (x * z + y * ww); R[7] = 2.0f * (y * z - x * ww); R[8] = 1.0f - 2.0f * (x * x + y * y);
        if(truth)
        {
            float* o = truth + 16 * (uint64_t)blockIdx.x;
            for(int i = 0; i < 16; ++i)
                o[i] = (&tr.kd[0])[i];
        }
    }
    __syncthreads();
    for(uint32_t d = threadIdx.x; d < L; d += blockDim.x)
    {
        float wd[3];
        parabolic_to_cartesian(lp[2 * d], lp[2 * d + 1], wd);
        w[0][d] = wd[0]; w[1][d] = wd[1]; w[2][d] = wd[2];
        float a[3];
        for(int c = 0; c < 3; ++c)
            a[c] = R[3 * c] * wd[0] + R[3 * c + 1] * wd[1] + R[3 * c + 2] * wd[2];
        dens[d] = sqrtf(tr.sigma[0] * tr.sigma[0] * a[0] * a[0] + tr.sigma[1] * tr.sigma[1] * a[1] * a[1] + a[2] * a[2]);
    }
    __syncthreads();
    const uint32_t N = L * L;
    T* out = samples + (uint64_t)blockIdx.x * N * 3;
    const uint32_t lo = (uint32_t)texel, hi = (uint32_t)(texel >> 32);
    for(uint32_t lv = threadIdx.x; lv < N; lv += blockDim.x)
    {
        uint32_t v = lv / L, l = lv % L;
        float wi[3] = { w[0][l], w[1][l], w[2][l] };
        float wo[3] = { w[0][v], w[1][v], w[2][v] };
        uint32_t r[4];
        philox(seed, 0x53564631u, lo, hi, 16u + lv, 0u, r);
        float z[4];
        for(int k = 0; k < 2; ++k)
        {
            float ua = (float)((r[2 * k] >> 8) + 1u) * (1.0f / 16777216.0f);
            float ub = u01(r[2 * k + 1]);
            float rad = sqrtf(-2.0f * logf(ua));
            float sn, cs;
            sincosf(6.283185307179586f * ub, &sn, &cs);
            z[2 * k] = rad * cs;
            z[2 * k + 1] = rad * sn;
        }
        for(int c = 0; c < 3; ++c)
        {
            float f = surface_brdf_rgb(tr.kd[c], tr.ks[c], tr.sigma[0], tr.sigma[1], R, dens[v], wi, wo);
            float val = f * (1.0f + noise * z[c]);
            if constexpr(sizeof(T) == 2)
                out[3 * lv + c] = __float2half_rn(val);
            else
                out[3 * lv + c] = val;
        }
    }
}

// ------------------------------------------------------------------------------
// allocation-free LM batch: working memory in one static device array
// ------------------------------------------------------------------------------

// Layout of the static array: luminance slabs, then the direction table, then
// the work counter and the error flag.
constexpr size_t kNoAllocGeoOffset = size_t(SVF_NOALLOC_MAX_SLAB_FLOATS) * sizeof(float);
constexpr size_t kNoAllocFlagOffset = kNoAllocGeoOffset + 3 * 160 * sizeof(float);
static_assert(kNoAllocFlagOffset + 16 <= SVF_NOALLOC_SCRATCH_BYTES, "no-alloc scratch layout overflows");

// Direction table [3][L] from parabolic coordinates, with the operation order
// and rounding of ParabolicToCartesianCoordinates (vector3.hh:389-393) that the
// host computes for the other entry points, so both fit identical geometry.
__global__ void geo_from_parabolic_kernel(const float* __restrict__ lp, uint32_t L, float* __restrict__ geo)
{
    const uint32_t d = blockIdx.x * blockDim.x + threadIdx.x;
    if(d >= L)
        return;
    const float px = lp[2 * d], py = lp[2 * d + 1];
    const float len_sq = __fadd_rn(__fmul_rn(px, px), __fmul_rn(py, py));
    const float den = __fadd_rn(len_sq, 1.0f);
    geo[d] = __fdiv_rn(__fmul_rn(2.0f, px), den);
    geo[L + d] = __fdiv_rn(__fmul_rn(2.0f, py), den);
    geo[2 * L + d] = __fdiv_rn(__fsub_rn(1.0f, len_sq), __fadd_rn(1.0f, len_sq));
}

} // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[SVF_NOALLOC_SCRATCH_BYTES];

namespace
{
constexpr int kNoAllocMaxDevices = 64;
std::mutex g_noalloc_mutex;
void* g_noalloc_address[kNoAllocMaxDevices];

// Device address of g_noalloc_scratch on the current device, looked up once per
// device.  In host code the array's name is only a host-side stand-in.
cudaError_t noalloc_scratch_address(void** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if(e != cudaSuccess)
        return e;
    if(dev < 0 || dev >= kNoAllocMaxDevices)
        return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if(!g_noalloc_address[dev])
    {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if(e != cudaSuccess)
            return e;
        g_noalloc_address[dev] = p;
    }
    *out = g_noalloc_address[dev];
    return cudaSuccess;
}
} // namespace

cudaError_t launch_lm_fit_noalloc(const float* lights_parabolic, uint32_t L, const float* lum, uint64_t lum_stride,
                                  uint32_t texels, const LmConfig& cfg, const float* init, float* out, float* rmse,
                                  svf_texel_stats* stats, cudaStream_t stream, uint32_t* error_flag)
{
    void* base = nullptr;
    cudaError_t e = noalloc_scratch_address(&base);
    if(e != cudaSuccess)
        return e;
    unsigned char* scratch = static_cast<unsigned char*>(base);
    float* slabs = reinterpret_cast<float*>(scratch);
    float* geo = reinterpret_cast<float*>(scratch + kNoAllocGeoOffset);
    uint32_t* flags = reinterpret_cast<uint32_t*>(scratch + kNoAllocFlagOffset);
    const uint32_t N = L * L;
    const uint64_t stride = (N + 7u) & ~uint64_t(7);

    // the array keeps the previous call's contents: counter and flag start at 0
    if((e = cudaMemsetAsync(flags, 0, 16, stream)) != cudaSuccess)
        return e;
    geo_from_parabolic_kernel<<<(L + 127) / 128, 128, 0, stream>>>(lights_parabolic, L, geo);
    if((e = cudaGetLastError()) != cudaSuccess)
        return e;
    repack_kernel<<<texels, 256, 0, stream>>>(lum, lum_stride, N, slabs, stride);
    if((e = cudaGetLastError()) != cudaSuccess)
        return e;
    int dev = 0, sms = 0;
    if((e = cudaGetDevice(&dev)) != cudaSuccess ||
       (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess)
        return e;
    LmArgs a{};
    a.lum = slabs;
    a.lum_stride = stride;
    a.geo = geo;
    a.init = init;
    a.out = out;
    a.rmse = rmse;
    a.stats = stats;
    a.L = L;
    a.N = N;
    a.texels = texels;
    a.cfg = cfg;
    a.work_counter = flags;
    a.error_flag = flags + 1;
    const int per_sm = lm_max_ctas_per_sm(L, stride);
    if(per_sm <= 0)
        return cudaErrorInvalidConfiguration;
    const uint64_t grid = std::min<uint64_t>((uint64_t)per_sm * sms, texels);
    if((e = launch_lm_fit(a, (int)std::max<uint64_t>(grid, 1), stream)) != cudaSuccess)
        return e;
    if((e = cudaMemcpyAsync(error_flag, flags + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream)) != cudaSuccess)
        return e;
    return cudaStreamSynchronize(stream);
}

size_t lm_smem_bytes(uint32_t L, uint64_t lum_stride)
{
    size_t a, b, c, d, e;
    return lm_smem_layout(L, lum_stride, &a, &b, &c, &d, &e);
}

int lm_max_ctas_per_sm(uint32_t L, uint64_t lum_stride)
{
    int n = 0;
    size_t smem = lm_smem_bytes(L, lum_stride);
    cudaFuncSetAttribute(lm_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, lm_fit_kernel, kThreads, smem) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_lm_fit(const LmArgs& args, int grid, cudaStream_t stream)
{
    size_t smem = lm_smem_bytes(args.L, args.lum_stride);
    cudaError_t e = cudaFuncSetAttribute(lm_fit_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(e != cudaSuccess)
        return e;
    lm_fit_kernel<<<grid, kThreads, smem, stream>>>(args);
    return cudaGetLastError();
}

cudaError_t launch_luminance(const void* samples, uint32_t sample_type, uint64_t texels, uint32_t N, float* lum,
                             uint64_t lum_stride, float* avg, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    if(sample_type == SVF_SAMPLES_F16)
        luminance_kernel<__half><<<(unsigned)texels, 256, 0, stream>>>(static_cast<const __half*>(samples), N, lum,
                                                                     lum_stride, avg);
    else
        luminance_kernel<float><<<(unsigned)texels, 256, 0, stream>>>(static_cast<const float*>(samples), N, lum,
                                                                    lum_stride, avg);
    return cudaGetLastError();
}

cudaError_t launch_repack(const float* src, uint64_t src_stride, uint64_t texels, uint32_t N, float* dst,
                          uint64_t dst_stride, cudaStream_t stream)
{
    if(texels == 0)
        return cudaSuccess;
    repack_kernel<<<(unsigned)texels, 256, 0, stream>>>(src, src_stride, N, dst, dst_stride);
    return cudaGetLastError();
}

cudaError_t launch_synth(uint32_t seed, uint32_t mix, const float* lp, uint32_t L, uint64_t first, uint64_t count,
                         uint32_t sample_type, float noise, void* samples, float* truth, cudaStream_t stream)
{
    if(count == 0)
        return cudaSuccess;
    if(sample_type == SVF_SAMPLES_F16)
        synth_kernel<__half><<<(unsigned)count, 256, 0, stream>>>(seed, mix, lp, L, first, noise,
                                                                static_cast<__half*>(samples), truth);
    else
        synth_kernel<float><<<(unsigned)count, 256, 0, stream>>>(seed, mix, lp, L, first, noise,
                                                               static_cast<float*>(samples), truth);
    return cudaGetLastError();
}

} // namespace svf
