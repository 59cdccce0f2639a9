/*
 * The drop-in for the reference's LeastSquaresFitSGGX
 * (tools/svbrdf-fitting/svbrdf-fitting.hh:126-127; the CPU definition it
 * replaces is tools/svbrdf-fitting/svbrdf-lsq-fitting-setup.cc:234-431), as a
 * maintainer adds it to the reference tree: the same signature, the fit done by
 * libsvf.so's svf_lsq_fit_sggx on the GPU.
 *
 * oracle/Makefile compiles this file against the reference's headers and links
 * it, in place of svbrdf-lsq-fitting-setup.cc, with the reference's own
 * SVBRDFFitPipeline (svbrdf-fitting-pipeline.cc) and the other reference
 * sources into oracle/_ref/libtempest_ref_svf.so.  tests/test_gpu_shim.py runs
 * the reference pipeline through it.  Test infrastructure: the product never
 * links it.
 */
#include "svf.h"

// the headers svbrdf-fitting.hh needs before it, as the file it replaces has them
#include "tempest/graphics/ray-tracing/illumination-models.hh"
#include "tempest/image/btf.hh"
#include "tempest/utils/logging.hh"
#include "tempest/utils/threads.hh"

#include "svbrdf-fitting.hh"

static thread_local svf_ctx* g_svf = nullptr;   // one context per worker thread

void LeastSquaresFitSGGX(uint32_t id, Tempest::ThreadPool& pool, const Tempest::BTF* btf, float* lv_lum_slice,
                         const LeastSquaresFitOptions& opts, const OptimizationParameters& parameters,
                         OptimizationParameters* opt_parameters, float* rmse)
{
    (void)id;
    (void)pool;
    if(!g_svf && svf_create(0, &g_svf) != SVF_OK)
    {
        Tempest::Log(Tempest::LogLevel::Fatal, "svf_create: ", svf_last_error());
        return;
    }
    // what svf_lsq_fit_sggx does not implement stays with the CPU path
    // (LSF_OPTION_CUDA asks for the GPU fit, which this is)
    constexpr uint32_t handled = LSF_OPTON_DIFFUSE | LSF_OPTION_CUDA | LSF_OPTION_DISABLE_DIRECTION_FITTING |
                                 LSF_OPTION_FIT_TOP;
    if((opts.Flags & ~handled) != 0)
    {
        Tempest::Log(Tempest::LogLevel::Error, "svf_lsq_fit_sggx: unsupported LeastSquaresFitOptions");
        *opt_parameters = parameters;
        *rmse = -1.0f;
        return;
    }
    svf_lsq_options o;
    svf_lsq_options_default(&o);
    o.fresnel = opts.Fresnel;
    if(!(opts.Flags & LSF_OPTON_DIFFUSE))
        o.flags &= ~SVF_LSQ_DIFFUSE;
    if(opts.Flags & LSF_OPTION_DISABLE_DIRECTION_FITTING)
        o.flags |= SVF_LSQ_DISABLE_DIRECTION_FITTING;
    if(opts.Flags & LSF_OPTION_FIT_TOP)
        o.flags |= SVF_LSQ_FIT_TOP;
    // DownSampleLightView ~0u (or not below the direction count): all directions
    if(opts.DownSampleLightView < btf->LightCount)
        o.downsample_light_view = opts.DownSampleLightView;
    // svbrdffit -m: the pseudo-volume model, fitted by the reference's LM as written
    if(opts.MultiScatteringBounceCount != ~0u)
    {
        o.flags |= SVF_LSQ_MULTI_SCATTERING;
        o.flags &= ~SVF_LSQ_STEP_PER_PARAMETER;
        o.multi_scattering_bounces = opts.MultiScatteringBounceCount;
    }
    o.max_iterations = CurveFitSteps;
    svf_texel_stats st{};
    const svf_status s = svf_lsq_fit_sggx(g_svf, &btf->LightsParabolic[0].x, btf->LightCount, lv_lum_slice, &o,
                                          parameters.ParametersArray, opt_parameters->ParametersArray, rmse, &st);
    if(s != SVF_OK && s != SVF_EPARTIAL)
        Tempest::Log(Tempest::LogLevel::Error, "svf_lsq_fit_sggx: ", svf_last_error());
    Tempest::Log(Tempest::LogLevel::Info, "Iteration required for fitting: ", st.effective, "(", st.iterations,
                 "). RMSE: ", *rmse, ".");
}
