/*
 * Test infrastructure only: a C-callable harness around the reference CPU fitter.
 *
 * This translation unit is compiled together with the reference's own sources,
 * in place (see oracle/Makefile), into oracle/_ref/libtempest_ref.so.  It is the
 * checker that pins the oracle restatement (oracle/svf_oracle.c) and times the
 * reference on host cores for bench.py's CPU baseline.  The product library never
 * links or loads it.
 *
 * Reference entry points wrapped here:
 *   LoadBTF                           src/image/btf.cc:389
 *   BTFParallelExtractLuminanceSlice  src/image/btf.cc:1078-1116
 *   SVBRDFFitPipeline::cache / fit    tools/svbrdf-fitting/svbrdf-fitting-pipeline.cc:240,328
 *   LeastSquaresFitSGGX               tools/svbrdf-fitting/svbrdf-lsq-fitting-setup.cc:234
 *   BRDFEvaluator                     tools/svbrdf-fitting/svbrdf-lsq-fitting-internal.hh:91-153
 *   LevenbergMarquardtCurveFit        include/tempest/math/fitting.hh:457
 *
 * The pipeline TU is compiled with -DLeastSquaresFitSGGX=HarnessLeastSquaresFitSGGX
 * so that the initial guess the pipeline computes (fit():350-660) can be recorded
 * before the real LeastSquaresFitSGGX runs.  Tempest::Log is provided here (the
 * reference's logging.cc is not built) so that the per-texel iteration counts the
 * reference logs (svbrdf-lsq-fitting-setup.cc:429) can be captured, and so that no
 * console output is produced during timing.
 */
#define ILLUMINATION_MODEL_IMPLEMENTATION
#define EXPORT_TABLE
#include "tempest/graphics/ray-tracing/illumination-models.hh"
#include "tempest/image/btf.hh"
#include "tempest/utils/threads.hh"
#include "tempest/utils/logging.hh"
#include "tempest/utils/file-system.hh"
#include "tempest/graphics/texture.hh"
#include "tempest/image/exr-image.hh"
#include "tempest/math/fitting.hh"

#define EXPORT_EVALUATOR
#include "svbrdf-fitting.hh"
#include "svbrdf-lsq-fitting-internal.hh"

/* defined in svbrdf-lsq-fitting-setup.cc:129, declared in no header */
void DownsampleLightView(const Tempest::Vector2* orig_light_dirs, uint32_t orig_light_count, float* orig_lv_lum_slice,
                         Tempest::Vector2* downsample_light_dirs, uint32_t downsample_light_count,
                         float* downsampled_lum_slice);

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

namespace Tempest
{
/* Replacement for src/utils/logging.cc: keeps the last message per thread. */
static thread_local std::string g_last_log;
void Log(LogLevel, std::string msg) { g_last_log = std::move(msg); }
}

namespace
{
thread_local OptimizationParameters g_recorded_init, g_recorded_fit;
thread_local float g_recorded_rmse = 0.0f;
thread_local bool g_record_valid = false;
thread_local uint32_t g_iterations = 0, g_effective = 0;

/* Parses "Iteration required for fitting: E(I). RMSE: R." (svbrdf-lsq-fitting-setup.cc:429). */
void ParseIterationLog()
{
    g_iterations = g_effective = 0;
    const std::string& m = Tempest::g_last_log;
    auto pos = m.find("fitting: ");
    if(pos == std::string::npos)
        return;
    unsigned e = 0, i = 0;
    if(std::sscanf(m.c_str() + pos + 9, "%u(%u)", &e, &i) == 2)
    {
        g_effective = e;
        g_iterations = i;
    }
}

Tempest::ThreadPool* SerialPool()
{
    /* A pool without worker threads: the calling thread runs every parallel loop
     * itself, in index order, which makes the shared-seed loops of the default
     * initial guess (svbrdf-fitting-pipeline.cc:451-456) deterministic.  The pool
     * is never destroyed: ~ThreadPool reads m_WorkerThreads[0] (threads.cc), which
     * does not exist for a zero-thread pool. */
    static Tempest::ThreadPool* pool = []()
    {
        auto* p = new Tempest::ThreadPool(0);
        /* registers the caller as thread 0, so getThreadCount() is 1 and the
         * per-thread partial sums the loops allocate have one slot */
        p->allocateThreadNumber();
        return p;
    }();
    return pool;
}

LeastSquaresFitOptions MakeOptions(float fresnel, uint32_t flags, uint32_t downsample = ~0u, uint32_t bounces = ~0u)
{
    LeastSquaresFitOptions o;
    o.MultiScatteringBounceCount = bounces;
    o.Fresnel = fresnel;
    o.DownSampleLightView = downsample;
    o.Flags = flags;
    return o;
}

FitPipelineOptions MakePipelineOptions()
{
    FitPipelineOptions p;
    p.Filter = FilteringTechnique::None;
    p.BasisExtract = BasisExtractStrategy::PCAHemisphere;
    p.KernelRadius = 0;
    p.Flags = 0;
    return p;
}
}

void HarnessLeastSquaresFitSGGX(uint32_t id, Tempest::ThreadPool& pool, const Tempest::BTF* btf, float* lv_lum_slice, const LeastSquaresFitOptions& opts,
                                const OptimizationParameters& parameters, OptimizationParameters* opt_parameters, float* rmse)
{
    g_recorded_init = parameters;
    g_record_valid = true;
    LeastSquaresFitSGGX(id, pool, btf, lv_lum_slice, opts, parameters, opt_parameters, rmse);
    g_recorded_fit = *opt_parameters;
    g_recorded_rmse = *rmse;
    ParseIterationLog();
}

extern "C" {

void* ref_btf_load(const char* path)
{
    return Tempest::LoadBTF(Tempest::Path(path));
}

void ref_btf_free(void* btf)
{
    Tempest::DestroyCPUBTF(reinterpret_cast<Tempest::BTF*>(btf));
}

/* dims[0..4] = width, height, light_count, triangle_count, edge_count */
void ref_btf_info(void* handle, uint32_t* dims)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    dims[0] = btf->Width;
    dims[1] = btf->Height;
    dims[2] = btf->LightCount;
    dims[3] = btf->LightTriangleCount;
    dims[4] = btf->EdgeCount;
}

/* Copies the direction table and the interpolation mesh LoadBTF built
 * (btf.cc:519-625).  edges_u32: [EdgeCount][3] = Index0, Index1, Triangle;
 * edges_angle: [EdgeCount][2] = Angle0, Angle1. */
void ref_btf_geometry(void* handle, float* lights_parabolic, uint32_t* triangles, uint32_t* edges_u32, float* edges_angle)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    for(uint32_t i = 0; i < btf->LightCount; ++i)
    {
        lights_parabolic[2*i] = btf->LightsParabolic[i].x;
        lights_parabolic[2*i + 1] = btf->LightsParabolic[i].y;
    }
    std::memcpy(triangles, btf->LightIndices, 3*btf->LightTriangleCount*sizeof(uint32_t));
    for(uint32_t e = 0; e < btf->EdgeCount; ++e)
    {
        edges_u32[3*e] = btf->Edges[e].Index0;
        edges_u32[3*e + 1] = btf->Edges[e].Index1;
        edges_u32[3*e + 2] = btf->Edges[e].Triangle;
        edges_angle[2*e] = btf->Edges[e].Angle0;
        edges_angle[2*e + 1] = btf->Edges[e].Angle1;
    }
}

/* RGB of one sample (BTFFetchSpectrum, btf.hh:498-556). */
void ref_btf_fetch(void* handle, uint32_t lv_idx, uint32_t xy_idx, float* rgb)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    auto s = Tempest::BTFFetchSpectrum(btf, lv_idx, xy_idx);
    rgb[0] = s.x; rgb[1] = s.y; rgb[2] = s.z;
}

/* Luminance slice + average chromaticity of texel (x, y) (btf.cc:1078-1116). */
void ref_btf_lum_slice(void* handle, uint32_t x, uint32_t y, float* lum, float* avg_chroma)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    auto* pool = SerialPool();
    Tempest::Spectrum avg;
    Tempest::BTFParallelExtractLuminanceSlice(btf, 0, *pool, x, y, &lum, &avg);
    avg_chroma[0] = avg.x; avg_chroma[1] = avg.y; avg_chroma[2] = avg.z;
}

/* BRDFEvaluator over all L*L pairs (svbrdf-lsq-fitting-internal.hh:91-153). */
void ref_brdf_eval(const float* lights_parabolic, uint32_t light_count, float fresnel, const double* params, float* out)
{
    BRDFEvaluator ev{ reinterpret_cast<const Tempest::Vector2*>(lights_parabolic), light_count, ~0u, fresnel };
    for(uint32_t idx = 0; idx < light_count*light_count; ++idx)
        out[idx] = ev(0, idx, params);
}

/* BRDFEvaluator with BounceCount = bounces (svbrdffit -m): the pseudo-volume
 * multi-scattering BRDF (SGGXMicroFlakePseudoVolumeBRDF, ggx-models-impl.hh:621-758,
 * 256 random walks of at most `bounces` scattering events) over all L*L pairs. */
void ref_brdf_eval_ms(const float* lights_parabolic, uint32_t light_count, uint32_t bounces, float fresnel,
                      const double* params, float* out)
{
    BRDFEvaluator ev{ reinterpret_cast<const Tempest::Vector2*>(lights_parabolic), light_count, bounces, fresnel };
    for(uint32_t idx = 0; idx < light_count*light_count; ++idx)
        out[idx] = ev(0, idx, params);
}

/* LeastSquaresFitSGGX with LeastSquaresFitOptions::MultiScatteringBounceCount =
 * bounces (the fit's model is then the pseudo-volume BRDF).  stats as ref_lsq. */
void ref_lsq_ms(const float* lights_parabolic, uint32_t light_count, const float* lum, float fresnel, uint32_t flags,
                uint32_t bounces, const float* init7, float* out7, float* rmse, uint32_t* stats)
{
    Tempest::BTF btf;
    btf.LightCount = light_count;
    std::vector<Tempest::Vector2> lights(light_count);
    std::memcpy(lights.data(), lights_parabolic, light_count*sizeof(Tempest::Vector2));
    btf.LightsParabolic = lights.data();
    std::vector<float> lum_copy(lum, lum + (size_t)light_count*light_count);
    OptimizationParameters init, out;
    std::memcpy(init.ParametersArray, init7, sizeof(init.ParametersArray));
    auto opts = MakeOptions(fresnel, flags, ~0u, bounces);
    LeastSquaresFitSGGX(0, *SerialPool(), &btf, lum_copy.data(), opts, init, &out, rmse);
    ParseIterationLog();
    std::memcpy(out7, out.ParametersArray, sizeof(out.ParametersArray));
    stats[0] = g_iterations;
    stats[1] = g_effective;
    btf.LightsParabolic = nullptr;
}

/* LeastSquaresFitSGGX with LeastSquaresFitOptions::Flags and DownSampleLightView
 * as given (downsample ~0u: off).  stats as ref_lsq. */
void ref_lsq_opts(const float* lights_parabolic, uint32_t light_count, const float* lum, float fresnel, uint32_t flags,
                  uint32_t downsample, const float* init7, float* out7, float* rmse, uint32_t* stats)
{
    Tempest::BTF btf;
    btf.LightCount = light_count;
    std::vector<Tempest::Vector2> lights(light_count);
    std::memcpy(lights.data(), lights_parabolic, light_count*sizeof(Tempest::Vector2));
    btf.LightsParabolic = lights.data();
    std::vector<float> lum_copy(lum, lum + (size_t)light_count*light_count);
    OptimizationParameters init, out;
    std::memcpy(init.ParametersArray, init7, sizeof(init.ParametersArray));
    auto opts = MakeOptions(fresnel, flags, downsample);
    LeastSquaresFitSGGX(0, *SerialPool(), &btf, lum_copy.data(), opts, init, &out, rmse);
    ParseIterationLog();
    std::memcpy(out7, out.ParametersArray, sizeof(out.ParametersArray));
    stats[0] = g_iterations;
    stats[1] = g_effective;
    btf.LightsParabolic = nullptr;
}

#ifndef SVF_SHIM_BUILD
/* DownsampleLightView (svbrdf-lsq-fitting-setup.cc:129-163): the kept directions
 * (parabolic) and the downsampled slice.  (Not in the seam library, which has the
 * drop-in LeastSquaresFitSGGX in place of that file.) */
void ref_downsample(const float* lights_parabolic, uint32_t light_count, const float* lum, uint32_t n,
                    float* out_lights, float* out_slice)
{
    std::vector<float> lum_copy(lum, lum + (size_t)light_count*light_count);
    DownsampleLightView(reinterpret_cast<const Tempest::Vector2*>(lights_parabolic), light_count, lum_copy.data(),
                        reinterpret_cast<Tempest::Vector2*>(out_lights), n, out_slice);
}
#endif

/* LeastSquaresFitSGGX on a given luminance slice and initial guess.
 * stats[0] = iterations, stats[1] = effective (accepted) iterations. */
void ref_lsq(const float* lights_parabolic, uint32_t light_count, const float* lum, float fresnel, uint32_t flags,
             const float* init7, float* out7, float* rmse, uint32_t* stats)
{
    Tempest::BTF btf;
    btf.LightCount = light_count;
    std::vector<Tempest::Vector2> lights(light_count);
    std::memcpy(lights.data(), lights_parabolic, light_count*sizeof(Tempest::Vector2));
    btf.LightsParabolic = lights.data();
    std::vector<float> lum_copy(lum, lum + light_count*light_count);

    OptimizationParameters init, out;
    std::memcpy(init.ParametersArray, init7, sizeof(init.ParametersArray));
    auto opts = MakeOptions(fresnel, flags);
    LeastSquaresFitSGGX(0, *SerialPool(), &btf, lum_copy.data(), opts, init, &out, rmse);
    ParseIterationLog();
    std::memcpy(out7, out.ParametersArray, sizeof(out.ParametersArray));
    stats[0] = g_iterations;
    stats[1] = g_effective;
    btf.LightsParabolic = nullptr;
}

/* The full per-texel pipeline (cache + fit with the default initial guess) on
 * texel (x, y), serially.  Outputs:
 *   init7  - the 7 parameters the default initial guess produced,
 *   fit7   - LeastSquaresFitSGGX's result,
 *   maps12 - sigma(2), quaternion xyzw(4), diffuse RGB(3), specular RGB(3),
 *   rmse, stats (iterations, effective iterations),
 *   ndf    - the 64x64 NDF texture (may be null),
 *   lum    - the luminance slice (may be null). */
static int FitTexel(void* handle, uint32_t x, uint32_t y, const LeastSquaresFitOptions& opts_in, float* init7,
                    float* fit7, float* maps12, float* rmse, uint32_t* stats, float* ndf, float* lum);

int ref_fit_texel(void* handle, uint32_t x, uint32_t y, float fresnel,
                  float* init7, float* fit7, float* maps12, float* rmse, uint32_t* stats, float* ndf, float* lum)
{
    return FitTexel(handle, x, y, MakeOptions(fresnel, LSF_OPTON_DIFFUSE), init7, fit7, maps12, rmse, stats, ndf,
                    lum);
}

/* The same with LeastSquaresFitOptions::Flags, DownSampleLightView and
 * MultiScatteringBounceCount as given (~0u: off). */
int ref_fit_texel_opts(void* handle, uint32_t x, uint32_t y, float fresnel, uint32_t flags, uint32_t downsample,
                       uint32_t bounces, float* init7, float* fit7, float* maps12, float* rmse, uint32_t* stats)
{
    return FitTexel(handle, x, y, MakeOptions(fresnel, flags, downsample, bounces), init7, fit7, maps12, rmse, stats,
                    nullptr, nullptr);
}

static int FitTexel(void* handle, uint32_t x, uint32_t y, const LeastSquaresFitOptions& opts_in, float* init7,
                    float* fit7, float* maps12, float* rmse, uint32_t* stats, float* ndf, float* lum)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    auto* pool = SerialPool();
    SVBRDFFitPipeline pipeline(btf);
    auto popts = MakePipelineOptions();
    auto opts = opts_in;
    SGGXParameters out;
    g_record_valid = false;
    pipeline.cache(0, *pool, x, y, popts, nullptr);
    pipeline.fit(0, *pool, x, y, &opts, popts, nullptr, &out, false);
    if(!g_record_valid)
        return -1;
    std::memcpy(init7, g_recorded_init.ParametersArray, sizeof(g_recorded_init.ParametersArray));
    maps12[0] = out.StandardDeviation.x; maps12[1] = out.StandardDeviation.y;
    maps12[2] = out.Orientation.x; maps12[3] = out.Orientation.y; maps12[4] = out.Orientation.z; maps12[5] = out.Orientation.w;
    maps12[6] = out.Diffuse.x; maps12[7] = out.Diffuse.y; maps12[8] = out.Diffuse.z;
    maps12[9] = out.Specular.x; maps12[10] = out.Specular.y; maps12[11] = out.Specular.z;
    *rmse = out.RMSE;
    stats[0] = g_iterations;
    stats[1] = g_effective;
    if(fit7)
        std::memcpy(fit7, g_recorded_fit.ParametersArray, sizeof(g_recorded_fit.ParametersArray));
    if(ndf)
    {
        auto* tex = pipeline.getLastNDFTexture();
        std::memcpy(ndf, tex->getData(), NDFTextureResolution*NDFTextureResolution*sizeof(float));
    }
    if(lum)
        std::memcpy(lum, pipeline.getLastLuminanceSlice(), btf->LightCount*btf->LightCount*sizeof(float));
    return 0;
}

/* Times the reference's texel loop the way svbrdffit runs it
 * (svbrdf-fitting.cc:86-121,597-667): `workers` threads, each with its own
 * SVBRDFFitPipeline, pull texels from an atomic counter and run cache + fit with
 * the default initial guess; all of them share one ThreadPool of `pool_threads`
 * workers for the inner parallel loops.  Returns seconds of wall clock over the
 * texel loop only (no file I/O).  Texels are visited in row-major order starting
 * at `first_texel`. */
double ref_time_fit_texels(void* handle, uint32_t first_texel, uint32_t texel_count, uint32_t workers, uint32_t pool_threads,
                           float fresnel, float* rmse_out)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    /* pool_threads > 0: one pool shared by the workers, as svbrdffit shares one;
     * a texel's parallel loops are then partly run by other workers, which race
     * on the shared-seed loops of the default initial guess
     * (svbrdf-fitting-pipeline.cc:451-456), so results depend on scheduling.
     * pool_threads == 0: each worker runs its texels' loops itself on a private
     * zero-thread pool, so every texel's fit is the deterministic one that a
     * single-texel run gives (the same work, spread over the workers by texel). */
    const bool shared = pool_threads > 0;
    Tempest::ThreadPool* pool = shared ? new Tempest::ThreadPool(pool_threads) : nullptr;
    std::atomic<uint32_t> counter(0);
    std::vector<Tempest::ThreadPool*> pools(workers, pool);
    std::vector<uint32_t> ids(workers);
    for(uint32_t w = 0; w < workers; ++w)
    {
        if(!shared)
            pools[w] = new Tempest::ThreadPool(0);   /* never destroyed, see SerialPool() */
        ids[w] = pools[w]->allocateThreadNumber();
    }

    auto t0 = std::chrono::steady_clock::now();
    std::vector<std::thread> threads;
    for(uint32_t w = 0; w < workers; ++w)
    {
        threads.emplace_back([&, w]()
        {
            SVBRDFFitPipeline pipeline(btf);
            auto popts = MakePipelineOptions();
            auto opts = MakeOptions(fresnel, LSF_OPTON_DIFFUSE);
            for(uint32_t k; (k = counter.fetch_add(1)) < texel_count;)
            {
                uint32_t t = first_texel + k;
                uint32_t x = t % btf->Width, y = t / btf->Width;
                SGGXParameters out;
                pipeline.cache(ids[w], *pools[w], x, y, popts, nullptr);
                pipeline.fit(ids[w], *pools[w], x, y, &opts, popts, nullptr, &out, false);
                if(rmse_out)
                    rmse_out[k] = out.RMSE;
            }
        });
    }
    for(auto& t : threads)
        t.join();
    auto t1 = std::chrono::steady_clock::now();
    if(shared)
        pool->shutdown();
    /* the pool objects themselves are leaked on purpose, see SerialPool() */
    return std::chrono::duration<double>(t1 - t0).count();
}

/* ---- svbrdffit's EXR maps and svbrdf-error-tool -------------------------------- */

/* SaveEXRImage (src/image/exr-image.cc:200-330) of [h][w][channels] floats. */
int ref_exr_save(const char* path, uint32_t w, uint32_t h, uint32_t channels, const float* data)
{
    Tempest::TextureDescription desc;
    desc.Width = w;
    desc.Height = h;
    static const Tempest::DataFormat fmts[4] = { Tempest::DataFormat::R32F, Tempest::DataFormat::RG32F,
                                                 Tempest::DataFormat::RGB32F, Tempest::DataFormat::RGBA32F };
    desc.Format = fmts[channels - 1];
    return Tempest::SaveEXRImage(desc, data, Tempest::Path(path)) ? 1 : 0;
}

/* LoadEXRImage (exr-image.cc:14-198): dims = width, height, channels; data
 * (optional) receives [h][w][channels] floats. */
int ref_exr_load(const char* path, uint32_t* dims, float* data)
{
    std::unique_ptr<Tempest::Texture> tex(Tempest::LoadEXRImage(Tempest::Path(path)));
    if(!tex)
        return 0;
    auto& hdr = tex->getHeader();
    dims[0] = hdr.Width;
    dims[1] = hdr.Height;
    dims[2] = Tempest::DataFormatChannels(hdr.Format);
    if(data)
        std::memcpy(data, tex->getData(), sizeof(float) * dims[0] * dims[1] * dims[2]);
    return 1;
}

/* svbrdf-error-tool's per-texel error (tools/svbrdf-error-tool/svbrdf-error-tool.cc:
 * 88-250), restated for one texel with the reference's own functions: the
 * material from the map values (stddev: sx, sy), the SGGX surface BRDF at every
 * (light, view), residuals against the BTF's luminance (color 0) or RGB
 * (color 1) slice; method 0 pair-wise, 1 max-view.  rmse3/psnr3: [0] or [0..2]. */
void ref_error_texel(void* handle, uint32_t x, uint32_t y, const float* diffuse3, const float* specular3,
                     const float* stddev2, const float* basis4, uint32_t method, uint32_t color, float* rmse3,
                     float* psnr3)
{
    auto* btf = reinterpret_cast<Tempest::BTF*>(handle);
    auto* pool = SerialPool();
    const uint32_t L = btf->LightCount;
    Tempest::RTSGGXSurface mat;
    mat.SampleCount = 256;
    mat.Depth = 0;
    mat.Diffuse = Tempest::RGBToSpectrum(Tempest::Vector3{ diffuse3[0], diffuse3[1], diffuse3[2] });
    mat.Specular = Tempest::RGBToSpectrum(Tempest::Vector3{ specular3[0], specular3[1], specular3[2] });
    mat.SGGXBasis = Tempest::Vector4{ basis4[0], basis4[1], basis4[2], basis4[3] };
    mat.StandardDeviation = Tempest::Vector2{ stddev2[0], stddev2[1] };
    mat.SpecularMap = nullptr;
    mat.DiffuseMap = nullptr;
    mat.BasisMap = nullptr;
    mat.StandardDeviationMap = nullptr;
    mat.Fresnel = { 1.0f, 0.0f };
    std::vector<float> lum(L * L);
    std::vector<Tempest::Vector3> rgb(L * L);
    float* lum_ptr = lum.data();
    Tempest::Vector3* rgb_ptr = rgb.data();
    if(color)
        Tempest::BTFParallelExtractRGBSlice(btf, 0, *pool, x, y, &rgb_ptr);
    else
        Tempest::BTFParallelExtractLuminanceSlice(btf, 0, *pool, x, y, &lum_ptr);
    auto brdf = [&](uint32_t light_idx, uint32_t view_idx) {
        Tempest::SampleData sd{};
        sd.Material = reinterpret_cast<Tempest::RTMaterial*>(&mat);
        sd.Tangent = Tempest::Vector3{ 1.0f, 0.0f, 0.0f };
        sd.Binormal = Tempest::Vector3{ 0.0f, 1.0f, 0.0f };
        sd.Normal = Tempest::Vector3{ 0.0f, 0.0f, 1.0f };
        sd.IncidentLight = Tempest::ParabolicToCartesianCoordinates(btf->LightsParabolic[light_idx]);
        sd.OutgoingLight = Tempest::ParabolicToCartesianCoordinates(btf->LightsParabolic[view_idx]);
        Tempest::Quaternion quat;
        quat.V4 = mat.SGGXBasis;
        sd.DirectionalDensity = Tempest::SGGXProjectedArea(
            Tempest::Vector3{ mat.StandardDeviation.x, mat.StandardDeviation.y, 1.0f }, Tempest::ToMatrix3(quat),
            sd.OutgoingLight);
        return Tempest::SpectrumToRGB(Tempest::SGGXMicroFlakeSurfaceBRDF(sd));
    };
    const uint32_t nch = color ? 3 : 1;
    float sq[3] = {}, mx[3] = {};
    if(method == 0)
    {
        for(uint32_t view_idx = 0; view_idx < L; ++view_idx)
            for(uint32_t light_idx = 0; light_idx < L; ++light_idx)
            {
                const uint32_t lv = view_idx * L + light_idx;
                const auto f = brdf(light_idx, view_idx);
                for(uint32_t c = 0; c < nch; ++c)
                {
                    const float b = color ? (&rgb[lv].x)[c] : lum[lv];
                    const float m = color ? (&f.x)[c] : Tempest::RGBToLuminance(f);
                    mx[c] = std::max(b, mx[c]);
                    const float r = b - m;
                    sq[c] += r * r;
                }
            }
        for(uint32_t c = 0; c < nch; ++c)
            sq[c] = sq[c] / (float)(L * L);
    }
    else
    {
        float best[3] = {}, best_mx[3] = {};
        for(uint32_t view_idx = 0; view_idx < L; ++view_idx)
        {
            float vs[3] = {}, vm[3] = {};
            for(uint32_t light_idx = 0; light_idx < L; ++light_idx)
            {
                const uint32_t lv = view_idx * L + light_idx;
                const auto f = brdf(light_idx, view_idx);
                for(uint32_t c = 0; c < nch; ++c)
                {
                    const float b = color ? (&rgb[lv].x)[c] : lum[lv];
                    const float m = color ? (&f.x)[c] : Tempest::RGBToLuminance(f);
                    vm[c] = std::max(b, vm[c]);
                    const float r = b - m;
                    vs[c] += r * r;
                }
            }
            for(uint32_t c = 0; c < nch; ++c)
                if(vs[c] > best[c])
                {
                    best[c] = vs[c];
                    best_mx[c] = vm[c];
                }
        }
        for(uint32_t c = 0; c < nch; ++c)
        {
            sq[c] = best[c] / (float)L;
            mx[c] = best_mx[c];
        }
    }
    for(uint32_t c = 0; c < nch; ++c)
    {
        rmse3[c] = sqrtf(sq[c]);
        psnr3[c] = 20.0f * log10f(mx[c] / rmse3[c]);
    }
}

}
