// extern "C" entry points of libqtrk_b200.so (declared in include/qtrk_c_api.h).
//
// Each forwards to qtrk::Tracker like cputrack/qtrk_c_api.cpp:62-175 forwards to the
// QueuedTracker virtuals, but no C++ exception crosses the ABI: failures are reported
// through QTrkGetWarnings (per instance) or QTrkB200GetLastError (no instance).
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "kernels.h"
#include "qtrk_c_api.h"
#include "result_manager.h"
#include "serve.h"
#include "tracker.h"

using qtrk::Tracker;

namespace {

std::mutex g_err_mu;
std::string g_last_error;

void set_last_error(const std::string &m)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_error = m;
}

Tracker *T(QueuedTracker *q) { return static_cast<Tracker *>(q); }

template <class F>
void guarded(QueuedTracker *q, const char *what, F &&f)
{
    if (!q) {
        set_last_error(std::string(what) + ": null instance");
        return;
    }
    try {
        f(T(q));
    } catch (const std::exception &e) {
        T(q)->Warn(std::string(what) + ": " + e.what());
        set_last_error(std::string(what) + ": " + e.what());
    } catch (...) {
        T(q)->Warn(std::string(what) + ": unknown error");
    }
}

template <class R, class F>
R guarded_ret(QueuedTracker *q, const char *what, R fail, F &&f)
{
    if (!q) {
        set_last_error(std::string(what) + ": null instance");
        return fail;
    }
    try {
        return f(T(q));
    } catch (const std::exception &e) {
        T(q)->Warn(std::string(what) + ": " + e.what());
        set_last_error(std::string(what) + ": " + e.what());
    } catch (...) {
        T(q)->Warn(std::string(what) + ": unknown error");
    }
    return fail;
}

void copy_string(const std::string &s, char *dst, int maxlen)
{
    if (!dst || maxlen <= 0) return;
    const size_t n = std::min(s.size(), (size_t)maxlen - 1);
    std::memcpy(dst, s.data(), n);
    dst[n] = 0;
}

}  // namespace

namespace qtrk {
// For entry points defined in other translation units (the bead finder).
void set_last_error_msg(const std::string &m) { set_last_error(m); }
}  // namespace qtrk

extern "C" {

QTRK_API void QTRK_CALLCONV TestDLLCallConv(int) {}

QTRK_API void QTRK_CALLCONV QTrkGetDefaultConfig(QTrkSettings *cfg)
{
    if (!cfg) return;
    // cputrack/qtrk_c_api.h:60-80
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->width = cfg->height = 150;
    cfg->numThreads = -1;
    cfg->xc1_profileLength = 128;
    cfg->xc1_profileWidth = 32;
    cfg->xc1_iterations = 2;
    cfg->zlut_minradius = 1.0f;
    cfg->zlut_angular_coverage = 0.7f;
    cfg->zlut_radial_coverage = 3.0f;
    cfg->zlut_roi_coverage = 1.0f;
    cfg->qi_iterations = 4;
    cfg->qi_minradius = 1;
    cfg->qi_angular_coverage = 0.7f;
    cfg->qi_radial_coverage = 3.0f;
    cfg->qi_roi_coverage = 1.0f;
    cfg->qi_angstep_factor = 1.0f;
    cfg->cuda_device = QTrkCUDA_UseAll;
    cfg->com_bgcorrection = 0.0f;
    cfg->gauss2D_iterations = 6;
    cfg->gauss2D_sigma = 4;
    cfg->downsample = 0;
}

QTRK_API void QTRK_CALLCONV QTrkGetComputedConfig(QTrkSettings *base, QTrkComputedConfig *cfg)
{
    if (base && cfg) *cfg = qtrk::compute_config(*base);
}

QTRK_API QueuedTracker *QTRK_CALLCONV QTrkCreateInstance(QTrkSettings *cfg)
{
    if (!cfg) {
        set_last_error("QTrkCreateInstance: null settings");
        return nullptr;
    }
    try {
        return new Tracker(*cfg);
    } catch (const std::exception &e) {
        set_last_error(std::string("QTrkCreateInstance: ") + e.what());
    } catch (...) {
        set_last_error("QTrkCreateInstance: unknown error");
    }
    return nullptr;
}

QTRK_API void QTRK_CALLCONV QTrkFreeInstance(QueuedTracker *qtrk)
{
    try {
        delete T(qtrk);
    } catch (...) {
        set_last_error("QTrkFreeInstance: error while releasing the instance");
    }
}

QTRK_API void QTRK_CALLCONV QTrkSetLocalizationMode(QueuedTracker *q, LocMode_t locType)
{
    guarded(q, "QTrkSetLocalizationMode", [&](Tracker *t) { t->SetLocalizationMode(locType); });
}

QTRK_API void QTRK_CALLCONV QTrkSetPixelCalibrationImages(QueuedTracker *q, float *offset, float *gain)
{
    guarded(q, "QTrkSetPixelCalibrationImages", [&](Tracker *t) { t->SetPixelCalibrationImages(offset, gain); });
}

QTRK_API void QTRK_CALLCONV QTrkSetPixelCalibrationFactors(float offsetFactor, float gainFactor)
{
    qtrk::set_default_factors(offsetFactor, gainFactor);
    float f[2] = {offsetFactor, gainFactor};
    qtrk::for_each_tracker([](Tracker *t, void *a) {
        const float *v = static_cast<const float *>(a);
        t->SetPixelCalibrationFactors(v[0], v[1]);
    }, f);
}

QTRK_API void QTRK_CALLCONV QTrkScheduleLocalization(QueuedTracker *q, void *data, int pitch, QTRK_PixelDataType_t pdt,
                                                     const LocalizationJob *jobInfo)
{
    guarded(q, "QTrkScheduleLocalization", [&](Tracker *t) { t->ScheduleLocalization(data, pitch, pdt, jobInfo); });
}

QTRK_API void QTRK_CALLCONV QTrkClearResults(QueuedTracker *q)
{
    guarded(q, "QTrkClearResults", [&](Tracker *t) { t->ClearResults(); });
}

QTRK_API void QTRK_CALLCONV QTrkFlush(QueuedTracker *q)
{
    guarded(q, "QTrkFlush", [&](Tracker *t) { t->Flush(); });
}

QTRK_API int QTRK_CALLCONV QTrkScheduleFrame(QueuedTracker *q, void *imgptr, int pitch, int width, int height,
                                             ROIPosition *positions, int numROI, QTRK_PixelDataType_t pdt,
                                             const LocalizationJob *jobInfo)
{
    return guarded_ret<int>(q, "QTrkScheduleFrame", 0, [&](Tracker *t) {
        return t->ScheduleFrame(imgptr, pitch, width, height, positions, numROI, pdt, jobInfo);
    });
}

QTRK_API void QTRK_CALLCONV QTrkEnableRadialZLUTCompareProfile(bool enabled)
{
    Tracker *t = qtrk::latest_tracker();
    if (!t) {
        set_last_error("QTrkEnableRadialZLUTCompareProfile: no live instance");
        return;
    }
    guarded(t, "QTrkEnableRadialZLUTCompareProfile", [&](Tracker *tt) { tt->EnableRadialZLUTCompareProfile(enabled); });
}

QTRK_API void QTRK_CALLCONV QTrkGetRadialZLUTCompareProfile(float *dst)
{
    Tracker *t = qtrk::latest_tracker();
    if (!t) {
        set_last_error("QTrkGetRadialZLUTCompareProfile: no live instance");
        return;
    }
    guarded(t, "QTrkGetRadialZLUTCompareProfile", [&](Tracker *tt) { tt->GetRadialZLUTCompareProfile(dst); });
}

QTRK_API void QTRK_CALLCONV QTrkSetRadialZLUT(QueuedTracker *q, float *data, int count, int planes)
{
    guarded(q, "QTrkSetRadialZLUT", [&](Tracker *t) { t->SetRadialZLUT(data, count, planes); });
}

QTRK_API void QTRK_CALLCONV QTrkGetRadialZLUT(QueuedTracker *q, float *dst)
{
    guarded(q, "QTrkGetRadialZLUT", [&](Tracker *t) { t->GetRadialZLUT(dst); });
}

QTRK_API void QTRK_CALLCONV QTrkGetRadialZLUTSize(QueuedTracker *q, int *count, int *planes, int *radialsteps)
{
    guarded(q, "QTrkGetRadialZLUTSize", [&](Tracker *t) {
        int c, p, r;
        t->GetRadialZLUTSize(c, p, r);
        if (count) *count = c;
        if (planes) *planes = p;
        if (radialsteps) *radialsteps = r;
    });
}

QTRK_API void QTRK_CALLCONV QTrkSetRadialWeights(QueuedTracker *q, float *zcmp)
{
    guarded(q, "QTrkSetRadialWeights", [&](Tracker *t) { t->SetRadialWeights(zcmp); });
}

QTRK_API void QTRK_CALLCONV QTrkBeginLUT(QueuedTracker *q, unsigned int flags)
{
    guarded(q, "QTrkBeginLUT", [&](Tracker *t) { t->BeginLUT(flags); });
}

QTRK_API void QTRK_CALLCONV QTrkBuildLUT(QueuedTracker *q, void *data, int pitch, QTRK_PixelDataType_t pdt, int plane,
                                         vector2f *known_pos)
{
    guarded(q, "QTrkBuildLUT", [&](Tracker *t) { t->BuildLUT(data, pitch, pdt, plane, known_pos); });
}

// QTrkBuildLUT for a stack in pinned host memory that stays unchanged until QTrkFinalizeLUT
// returns: the call returns once the plane's copy and kernel are queued. No counterpart in the
// reference (its BuildLUT is synchronous); a pageable stack is staged before the call returns, as
// by QTrkBuildLUT.
QTRK_API void QTRK_CALLCONV QTrkB200BuildLUTAsync(QueuedTracker *q, void *data, int pitch, QTRK_PixelDataType_t pdt,
                                                  int plane, vector2f *known_pos)
{
    guarded(q, "QTrkB200BuildLUTAsync", [&](Tracker *t) { t->BuildLUT(data, pitch, pdt, plane, known_pos, true); });
}

// Declared (never defined) at cputrack/qtrk_c_api.h:184: BuildLUT from ROIs cropped out of a
// float frame; ROI i belongs to bead i.
QTRK_API void QTRK_CALLCONV QTrkBuildLUTFromFrame(QueuedTracker *q, ImageData *frame, int plane, ROIPosition *roipos,
                                                  int numroi)
{
    guarded(q, "QTrkBuildLUTFromFrame", [&](Tracker *t) {
        if (!frame || !frame->data || !roipos) throw std::invalid_argument("null argument");
        int count, planes, rs;
        t->GetRadialZLUTSize(count, planes, rs);
        if (numroi != count) throw std::invalid_argument("numroi must equal the Z-LUT bead count");
        const int W = t->cfg.base.width, H = t->cfg.base.height;
        std::vector<float> stack((size_t)W * H * numroi, 0.0f);
        for (int i = 0; i < numroi; i++) {
            const ROIPosition p = roipos[i];
            if (p.x < 0 || p.y < 0 || p.x + W > frame->w || p.y + H > frame->h)
                throw std::invalid_argument("ROI " + std::to_string(i) + " lies outside the frame");
            for (int y = 0; y < H; y++)
                std::memcpy(&stack[((size_t)i * H + y) * W], frame->data + (size_t)(p.y + y) * frame->w + p.x,
                            sizeof(float) * W);
        }
        t->BuildLUT(stack.data(), W * 4, QTrkFloat, plane, nullptr);
    });
}

QTRK_API void QTRK_CALLCONV QTrkFinalizeLUT(QueuedTracker *q)
{
    guarded(q, "QTrkFinalizeLUT", [&](Tracker *t) { t->FinalizeLUT(); });
}

QTRK_API int QTRK_CALLCONV QTrkGetResultCount(QueuedTracker *q)
{
    return guarded_ret<int>(q, "QTrkGetResultCount", 0, [&](Tracker *t) { return t->GetResultCount(); });
}

QTRK_API int QTRK_CALLCONV QTrkFetchResults(QueuedTracker *q, LocalizationResult *results, int maxResults)
{
    return guarded_ret<int>(q, "QTrkFetchResults", 0, [&](Tracker *t) { return t->FetchResults(results, maxResults); });
}

QTRK_API int QTRK_CALLCONV QTrkGetQueueLength(QueuedTracker *q, int *maxQueueLen)
{
    return guarded_ret<int>(q, "QTrkGetQueueLength", 0, [&](Tracker *t) { return t->GetQueueLength(maxQueueLen); });
}

QTRK_API bool QTRK_CALLCONV QTrkIsIdle(QueuedTracker *q)
{
    return guarded_ret<bool>(q, "QTrkIsIdle", false, [&](Tracker *t) { return t->IsIdle(); });
}

QTRK_API void QTRK_CALLCONV QTrkGetProfileReport(QueuedTracker *q, char *dst, int maxStrLen)
{
    guarded(q, "QTrkGetProfileReport", [&](Tracker *t) { copy_string(t->GetProfileReport(), dst, maxStrLen); });
}

QTRK_API void QTRK_CALLCONV QTrkGetWarnings(QueuedTracker *q, char *dst, int maxStrLen)
{
    guarded(q, "QTrkGetWarnings", [&](Tracker *t) { copy_string(t->GetWarnings(), dst, maxStrLen); });
}

// ---------------------------------------------------------------------------------------
// Profile / image utilities of the reference (cputrack/utils.h:182-188,216)
// ---------------------------------------------------------------------------------------

// NormalizeRadialProfile, cputrack/utils.cpp:230-261 (host array of a few dozen floats).
QTRK_API void QTRK_CALLCONV NormalizeRadialProfile(float *prof, int rsteps)
{
    if (!prof || rsteps <= 0) return;
    double sum = 0.0;
    for (int i = 0; i < rsteps; i++) sum += prof[i];
    const float mean = (float)(sum / rsteps);
    double rms2 = 0.0;
    for (int i = 0; i < rsteps; i++) {
        prof[i] -= mean;
        rms2 += (double)(prof[i] * prof[i]);
    }
    const double inv = 1.0f / std::sqrt(rms2 / rsteps);
    for (int i = 0; i < rsteps; i++) prof[i] = (float)(prof[i] * inv);
}

// ComputeRadialProfile, cputrack/utils.cpp:275-320, evaluated by the profile kernel on the
// current CUDA device (the same device code as the tracker's Z stage).
QTRK_API void QTRK_CALLCONV ComputeRadialProfile(float *dst, int radialSteps, int angularSteps, float minradius,
                                                 float maxradius, vector2f center, ImageData *src, float mean,
                                                 bool normalize)
{
    if (!dst || !src || !src->data || radialSteps <= 0 || angularSteps <= 0 || src->w < 2 || src->h < 2) {
        set_last_error("ComputeRadialProfile: invalid argument");
        return;
    }
    float *d_img = nullptr, *d_out = nullptr;
    void *d_dirs = nullptr;
    try {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess) throw std::runtime_error("no CUDA device");
        if (qtrk::prepare_kernels(dev) != cudaSuccess) throw std::runtime_error("kernel setup failed");
        qtrk::TrackParams P;
        std::memset(&P, 0, sizeof(P));
        P.width = src->w;
        P.height = src->h;
        P.pdt = QTrkFloat;
        P.z_nbins = radialSteps;
        P.z_angsteps = angularSteps;
        P.z_minr = minradius;
        P.z_maxr = maxradius;
        qtrk::plan_smem(P);
        if (P.smem_bytes > 227 * 1024) throw std::runtime_error("image too large for one CTA");
        std::vector<float> zd(2 * angularSteps);
        for (int j = 0; j < angularSteps; j++) {
            const float ang = 2 * 3.141593f * j / (float)angularSteps;
            zd[2 * j] = cosf(ang);
            zd[2 * j + 1] = sinf(ang);
        }
        const size_t npx = (size_t)src->w * src->h;
        auto ck = [](cudaError_t e) {
            if (e != cudaSuccess) throw std::runtime_error(cudaGetErrorString(e));
        };
        ck(cudaMalloc(&d_img, npx * 4));
        ck(cudaMalloc(&d_out, (size_t)radialSteps * 4));
        ck(cudaMalloc(&d_dirs, zd.size() * 4));
        ck(cudaMemcpy(d_img, src->data, npx * 4, cudaMemcpyHostToDevice));
        ck(cudaMemcpy(d_dirs, zd.data(), zd.size() * 4, cudaMemcpyHostToDevice));
        P.z_dirs = d_dirs;
        ck(qtrk::launch_profile(P, d_img, center.x, center.y, mean, normalize, d_out, 0));
        ck(cudaMemcpy(dst, d_out, (size_t)radialSteps * 4, cudaMemcpyDeviceToHost));
    } catch (const std::exception &e) {
        set_last_error(std::string("ComputeRadialProfile: ") + e.what());
    }
    cudaFree(d_img);
    cudaFree(d_out);
    cudaFree(d_dirs);
}

// normalize<T>, cputrack/utils.h:23-34: min-max scaling to [0, 1].
QTRK_API void QTRK_CALLCONV NormalizeImage(ImageData *img)
{
    if (!img || !img->data || img->w * img->h <= 0) return;
    const int n = img->w * img->h;
    float mx = img->data[0], mn = img->data[0];
    for (int k = 0; k < n; k++) {
        mx = std::max(mx, img->data[k]);
        mn = std::min(mn, img->data[k]);
    }
    for (int k = 0; k < n; k++) img->data[k] = (img->data[k] - mn) / (mx - mn);
}

// Noise utilities (cputrack/utils.cpp:404-433 with the samplers of cputrack/random_distr.h):
// both draw from the C library's rand(), so a caller that seeds it with srand() gets the same
// image from the reference and from this library. The samplers are the textbook ones:
// Box-Muller for a standard normal (U0 offset by 1e-9 so that log(U0) is finite), and for the
// Poisson variate Knuth's product-of-uniforms method (capped at 200 factors) up to lambda 10 and
// floor(0.5 + lambda + sqrt(lambda) N(0,1)) clamped at 0 above it. Single precision throughout.
static float uniform_f() { return rand() / (float)RAND_MAX; }

static float normal_f()
{
    const float u0 = uniform_f() + 1e-9f;
    const float u1 = uniform_f();
    // the transcendental steps run in double and the product is rounded once, as the
    // reference's unqualified log/sqrt/cos calls resolve to the double functions
    return (float)(std::sqrt(-2 * std::log((double)u0)) * std::cos((double)(2 * 3.141593f * u1)));
}

static int poisson_f(float lambda)
{
    if (lambda > 10) {
        const float v = (float)(0.5f + lambda + normal_f() * std::sqrt((double)lambda));
        return (int)std::max(0.0f, v);
    }
    const float limit = (float)std::exp((double)-lambda);
    float prod = 1;
    int k = 0;
    do {
        k++;
        prod *= uniform_f();
    } while (prod > limit && k < 200);
    return k - 1;
}

QTRK_API void QTRK_CALLCONV ApplyPoissonNoise(ImageData *img, float poissonMax, float maxValue)
{
    if (!img || !img->data) return;
    const float ratio = maxValue / poissonMax;
    const int n = img->w * img->h;
    for (int k = 0; k < n; k++) img->data[k] = (float)(int)(poisson_f(poissonMax * img->data[k]) * ratio);
}

QTRK_API void QTRK_CALLCONV ApplyGaussianNoise(ImageData *img, float sigma)
{
    if (!img || !img->data) return;
    const int n = img->w * img->h;
    for (int k = 0; k < n; k++) {
        const float v = img->data[k] + sigma * normal_f();
        img->data[k] = v < 0.0f ? 0.0f : v;
    }
}

// Abramowitz & Stegun 7.1.26, the erf the reference's utilities bind (cputrack/utils.h:395-417).
static float erf_as_host(float x)
{
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f, a4 = -1.453152027f, a5 = 1.061405429f,
                p = 0.3275911f;
    const int sign = x < 0 ? -1 : 1;
    x = std::fabs(x);
    const float t = 1.0f / (1.0f + p * x);
    const float y = 1.0f - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * std::exp(-x * x);
    return sign * y;
}

// GenerateGaussianSpotImage, cputrack/utils.cpp:393-402: integrated Gaussian spot.
QTRK_API void QTRK_CALLCONV GenerateGaussianSpotImage(ImageData *img, vector2f pos, float sigma, float I0, float Ibg)
{
    if (!img || !img->data) return;
    const float edenom = 1 / std::sqrt(2 * sigma * sigma);
    for (int y = 0; y < img->h; y++)
        for (int x = 0; x < img->w; x++) {
            const float DX = 0.5f * erf_as_host((x - pos.x + .5f) * edenom) - 0.5f * erf_as_host((x - pos.x - .5f) * edenom);
            const float DY = 0.5f * erf_as_host((y - pos.y + .5f) * edenom) - 0.5f * erf_as_host((y - pos.y - .5f) * edenom);
            img->data[y * img->w + x] = Ibg + I0 * DX * DY;
        }
}

// Uniform cubic B-spline weights for GenerateImageFromLUT's spline mode.
static void bspline_weights(float w[4], float t)
{
    const float t2 = t * t, t3 = t2 * t;
    w[0] = (1 - 3 * t + 3 * t2 - t3) / 6;
    w[1] = (4 - 6 * t2 + 3 * t3) / 6;
    w[2] = (1 + 3 * t + 3 * t2 - 3 * t3) / 6;
    w[3] = t3 / 6;
}

// GenerateImageFromLUT, cputrack/utils.cpp:325-390: render a bead image from a radial LUT
// (zlut->w bins x zlut->h planes) at pos (x, y, z in planes), ovs x ovs samples per pixel.
QTRK_API void QTRK_CALLCONV GenerateImageFromLUT(ImageData *image, ImageData *zlut, float minradius, float maxradius,
                                                 vector3f pos, bool useSplineInterp, int ovs)
{
    if (!image || !image->data || !zlut || !zlut->data || zlut->w < 2 || zlut->h < 1 || ovs <= 0) return;
    const int nb = zlut->w;
    const float radialcov = nb / (maxradius - minradius);
    std::vector<float> zi(nb);
    if (useSplineInterp && zlut->h >= 4) {
        const int iz = std::max(1, std::min(zlut->h - 3, (int)pos.z));
        float w[4];
        bspline_weights(w, pos.z - iz);
        for (int r = 0; r < nb; r++) {
            float v = 0;
            for (int i = 0; i < 4; i++) v += w[i] * zlut->data[(i - 1 + iz) * nb + r];
            zi[r] = v;
        }
    } else {
        const int iz = (int)pos.z;
        if (iz < 0) {
            for (int r = 0; r < nb; r++) zi[r] = zlut->data[r];
        } else if (iz >= zlut->h - 1) {
            for (int r = 0; r < nb; r++) zi[r] = zlut->data[(zlut->h - 1) * nb + r];
        } else {
            for (int r = 0; r < nb; r++) {
                const float a = zlut->data[iz * nb + r], b = zlut->data[(iz + 1) * nb + r];
                zi[r] = a + (b - a) * (pos.z - iz);
            }
        }
    }
    const float step = 1.0f / ovs;
    for (int y = 0; y < image->h; y++)
        for (int x = 0; x < image->w; x++) {
            float s = 0.0f;
            for (int ox = 0; ox < ovs; ox++)
                for (int oy = 0; oy < ovs; oy++) {
                    const float X = x + (ox + 0.5f) * step - pos.x - 0.5f;
                    const float Y = y + (oy + 0.5f) * step - pos.y - 0.5f;
                    float r = (std::sqrt(X * X + Y * Y) - minradius) * radialcov;
                    if (r > nb - 2) r = (float)(nb - 2);
                    if (r < 0) r = 0;
                    const int i = (int)r;
                    s += zi[i] + (zi[i + 1] - zi[i]) * (r - i);
                }
            image->data[y * image->w + x] = s / (ovs * ovs);
        }
}

// ---------------------------------------------------------------------------------------
// Extensions
// ---------------------------------------------------------------------------------------
QTRK_API int QTRK_CALLCONV QTrkB200GetLastError(char *dst, int maxStrLen)
{
    std::lock_guard<std::mutex> lk(g_err_mu);
    copy_string(g_last_error, dst, maxStrLen);
    return (int)std::min(g_last_error.size(), (size_t)std::max(maxStrLen - 1, 0));
}

QTRK_API int64_t QTRK_CALLCONV QTrkB200GetKernelLaunchCount(QueuedTracker *q)
{
    return q ? T(q)->LaunchCount() : 0;
}

QTRK_API void QTRK_CALLCONV QTrkB200SetZLUTBiasTable(QueuedTracker *q, const float *table, int bias_planes, int count)
{
    guarded(q, "QTrkB200SetZLUTBiasTable", [&](Tracker *t) { t->SetZLUTBiasTable(table, bias_planes, count); });
}

QTRK_API void QTRK_CALLCONV QTrkB200ComputeZLUTBiasTable(QueuedTracker *q, int bias_planes, float *result,
                                                         int smpPerPixel, int useSplineInterp)
{
    guarded(q, "QTrkB200ComputeZLUTBiasTable",
            [&](Tracker *t) { t->ComputeZBiasTable(bias_planes, smpPerPixel, useSplineInterp != 0, result); });
}

QTRK_API int QTRK_CALLCONV QTrkB200ZLUTCostGradient(QueuedTracker *q, const void *d_pixels, int pitch,
                                                    int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int count,
                                                    const float *d_xyz, const int *d_beads, float *d_cost,
                                                    float *d_grad_xyz, float *d_grad_lut, void *stream)
{
    return guarded_ret<int>(q, "QTrkB200ZLUTCostGradient", -100, [&](Tracker *t) {
        return t->ZLUTCostGradient(d_pixels, pitch, roi_stride_bytes, pdt, count, d_xyz, d_beads, d_cost, d_grad_xyz,
                                   d_grad_lut, static_cast<cudaStream_t>(stream));
    });
}

QTRK_API void QTRK_CALLCONV QTrkB200RefineZLUT(QueuedTracker *q, const void *d_stack, int pitch, int64_t roi_stride_bytes,
                                               QTRK_PixelDataType_t pdt, int beads, int planes, const float *d_xy,
                                               int iterations, float smoothness, float *plane_z, float *cost_history)
{
    guarded(q, "QTrkB200RefineZLUT", [&](Tracker *t) {
        t->RefineZLUT(d_stack, pitch, roi_stride_bytes, pdt, beads, planes, d_xy, iterations, smoothness, plane_z,
                      cost_history);
    });
}

QTRK_API int QTRK_CALLCONV QTrkB200GaussianNLLGradient(QueuedTracker *q, const void *d_pixels, int pitch,
                                                       int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int count,
                                                       const float *d_params, float *d_nll, float *d_grad,
                                                       void *stream)
{
    return guarded_ret<int>(q, "QTrkB200GaussianNLLGradient", -100, [&](Tracker *t) {
        return t->GaussianNLLGradient(d_pixels, pitch, roi_stride_bytes, pdt, count, d_params, d_nll, d_grad,
                                      static_cast<cudaStream_t>(stream));
    });
}

QTRK_API int QTRK_CALLCONV QTrkB200LocalizeDevice(QueuedTracker *q, const void *d_pixels, int pitch,
                                                  int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int count,
                                                  const LocalizationJob *d_jobs, LocalizationResult *d_results,
                                                  void *stream)
{
    return guarded_ret<int>(q, "QTrkB200LocalizeDevice", -100, [&](Tracker *t) {
        return t->LocalizeDevice(d_pixels, pitch, roi_stride_bytes, pdt, count, d_jobs, d_results,
                                 static_cast<cudaStream_t>(stream));
    });
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Request server
// ---------------------------------------------------------------------------------------
QTRK_API void *QTRK_CALLCONV QTrkB200ServerCreate(int device, int64_t device_memory_budget)
{
    try {
        return new qtrk::Server(device, device_memory_budget);
    } catch (const std::exception &e) {
        set_last_error(std::string("QTrkB200ServerCreate: ") + e.what());
        return nullptr;
    }
}

QTRK_API void QTRK_CALLCONV QTrkB200ServerDestroy(void *server)
{
    delete static_cast<qtrk::Server *>(server);
}

QTRK_API int QTRK_CALLCONV QTrkB200ServerAttach(void *server, QueuedTracker *q)
{
    if (!server || !q) {
        set_last_error("QTrkB200ServerAttach: null argument");
        return -1;
    }
    try {
        return static_cast<qtrk::Server *>(server)->Attach(T(q));
    } catch (const std::exception &e) {
        set_last_error(std::string("QTrkB200ServerAttach: ") + e.what());
        return -1;
    }
}

QTRK_API int64_t QTRK_CALLCONV QTrkB200ServerSubmitFrame(void *server, int instance, const void *frame, int pitch,
                                                         int width, int height, const ROIPosition *positions,
                                                         int numROI, QTRK_PixelDataType_t pdt,
                                                         const LocalizationJob *jobInfo)
{
    if (!server) {
        set_last_error("QTrkB200ServerSubmitFrame: null server");
        return -1;
    }
    try {
        return static_cast<qtrk::Server *>(server)->Submit(instance, frame, pitch, width, height, positions, numROI,
                                                           (int)pdt, jobInfo);
    } catch (const std::exception &e) {
        set_last_error(std::string("QTrkB200ServerSubmitFrame: ") + e.what());
        return -1;
    }
}

QTRK_API int QTRK_CALLCONV QTrkB200ServerPoll(void *server, int64_t request, LocalizationResult *results,
                                              int maxResults)
{
    if (!server) return -2;
    qtrk::Server *sv = static_cast<qtrk::Server *>(server);
    const int r = sv->Poll(request, results, maxResults);
    if (r == -3) set_last_error("QTrkB200ServerPoll: " + sv->LastError());
    return r;
}

QTRK_API void QTRK_CALLCONV QTrkB200ServerGetStats(void *server, QTrkB200ServeStats *stats)
{
    if (!server || !stats) return;
    *stats = static_cast<qtrk::Server *>(server)->Stats();
}

QTRK_API void QTRK_CALLCONV QTrkB200ServerHold(void *server, int hold)
{
    if (server) static_cast<qtrk::Server *>(server)->Hold(hold != 0);
}

QTRK_API void QTRK_CALLCONV QTrkB200ServerResetStats(void *server)
{
    if (server) static_cast<qtrk::Server *>(server)->ResetStats();
}

// ---------------------------------------------------------------------------------------
// ResultManager (cputrack/qtrk_c_api.cpp:181-241)
// ---------------------------------------------------------------------------------------
QTRK_API ResultManager *QTRK_CALLCONV RMCreate(const char *file, const char *frameinfo, ResultManagerConfig *cfg,
                                               const char *semicolonSeparatedNames)
{
    if (!cfg) {
        set_last_error("RMCreate: null config");
        return nullptr;
    }
    // Column names split at ';' as qtrk_c_api.cpp:185-195 does: the separator is kept as the
    // first character of the following name.
    std::vector<std::string> names;
    std::string name;
    for (const char *c = semicolonSeparatedNames ? semicolonSeparatedNames : ""; *c; c++) {
        if (*c == ';') {
            names.push_back(name);
            name.clear();
        }
        name += *c;
    }
    if (!name.empty()) names.push_back(name);
    try {
        return new ResultManager(file, frameinfo, *cfg, names);
    } catch (const std::exception &e) {
        set_last_error(std::string("RMCreate: ") + e.what());
        return nullptr;
    }
}

QTRK_API void QTRK_CALLCONV RMSetTracker(ResultManager *rm, QueuedTracker *q)
{
    if (rm) rm->SetTracker(q ? T(q) : nullptr);
}

QTRK_API void QTRK_CALLCONV RMDestroy(ResultManager *rm) { delete rm; }

QTRK_API void QTRK_CALLCONV RMStoreFrameInfo(ResultManager *rm, int frame, double timestamp, float *cols)
{
    if (rm) rm->StoreFrameInfo(frame, timestamp, cols);
}

QTRK_API int QTRK_CALLCONV RMGetBeadResults(ResultManager *rm, int start, int numFrames, int bead,
                                            LocalizationResult *results)
{
    return rm && results ? rm->GetBeadPositions(start, start + numFrames, bead, results) : 0;
}

QTRK_API void QTRK_CALLCONV RMGetFrameCounters(ResultManager *rm, RMFrameCounters *dst)
{
    if (rm && dst) *dst = rm->Counters();
}

QTRK_API void QTRK_CALLCONV RMFlush(ResultManager *rm)
{
    if (rm) rm->Flush();
}

QTRK_API int QTRK_CALLCONV RMGetResults(ResultManager *rm, int startFrame, int numFrames, LocalizationResult *results)
{
    return rm && results ? rm->GetResults(results, startFrame, numFrames) : 0;
}

QTRK_API void QTRK_CALLCONV RMRemoveBead(ResultManager *rm, int bead)
{
    if (rm) rm->RemoveBead(bead);
}

QTRK_API void QTRK_CALLCONV RMGetConfig(ResultManager *rm, ResultManagerConfig *cfg)
{
    if (rm && cfg) *cfg = rm->Config();
}

QTRK_API void QTRK_CALLCONV QTrkB200RMStoreResults(ResultManager *rm, const LocalizationResult *results, int count,
                                                   int roi_width, int roi_height)
{
    if (rm && results && count > 0) rm->StoreResults(results, count, roi_width, roi_height);
}

// ---------------------------------------------------------------------------------------
// .radialzlut files: int32 count, planes, radialsteps, then count*planes*radialsteps float32
// ([bead][plane][bin]), the layout cputrack/utils.cpp:680-710 (ReadLUTFile) reads.
// ---------------------------------------------------------------------------------------
QTRK_API int QTRK_CALLCONV QTrkB200ReadRadialZLUTFile(const char *path, float *dst, int *count, int *planes,
                                                      int *radialsteps)
{
    FILE *f = path ? std::fopen(path, "rb") : nullptr;
    if (!f) {
        set_last_error(std::string("QTrkB200ReadRadialZLUTFile: cannot open ") + (path ? path : "(null)"));
        return -1;
    }
    int32_t hdr[3];
    int rc = 0;
    if (std::fread(hdr, 4, 3, f) != 3 || hdr[0] < 0 || hdr[1] < 0 || hdr[2] < 0) {
        set_last_error("QTrkB200ReadRadialZLUTFile: bad header");
        rc = -2;
    } else {
        if (count) *count = hdr[0];
        if (planes) *planes = hdr[1];
        if (radialsteps) *radialsteps = hdr[2];
        const size_t n = (size_t)hdr[0] * hdr[1] * hdr[2];
        if (dst && std::fread(dst, 4, n, f) != n) {
            set_last_error("QTrkB200ReadRadialZLUTFile: file shorter than its header says");
            rc = -3;
        }
    }
    std::fclose(f);
    return rc;
}

QTRK_API int QTRK_CALLCONV QTrkB200WriteRadialZLUTFile(const char *path, const float *data, int count, int planes,
                                                       int radialsteps)
{
    if (!path || (!data && count * planes * radialsteps > 0) || count < 0 || planes < 0 || radialsteps < 0) {
        set_last_error("QTrkB200WriteRadialZLUTFile: invalid argument");
        return -1;
    }
    FILE *f = std::fopen(path, "wb");
    if (!f) {
        set_last_error(std::string("QTrkB200WriteRadialZLUTFile: cannot create ") + path);
        return -1;
    }
    const int32_t hdr[3] = {count, planes, radialsteps};
    const size_t n = (size_t)count * planes * radialsteps;
    const bool ok = std::fwrite(hdr, 4, 3, f) == 3 && (n == 0 || std::fwrite(data, 4, n, f) == n);
    std::fclose(f);
    if (!ok) set_last_error("QTrkB200WriteRadialZLUTFile: write failed");
    return ok ? 0 : -2;
}

// ---------------------------------------------------------------------------------------
// Instance-level forms of the reference's handle-less calls, and a ResultManager constructor
// taking its column names as an array (both for the LabVIEW layer).
// ---------------------------------------------------------------------------------------
QTRK_API void QTRK_CALLCONV QTrkB200SetPixelCalibrationFactors(QueuedTracker *q, float offsetFactor, float gainFactor)
{
    guarded(q, "QTrkB200SetPixelCalibrationFactors",
            [&](Tracker *t) { t->SetPixelCalibrationFactors(offsetFactor, gainFactor); });
}

QTRK_API void QTRK_CALLCONV QTrkB200EnableRadialZLUTCompareProfile(QueuedTracker *q, int enable)
{
    guarded(q, "QTrkB200EnableRadialZLUTCompareProfile", [&](Tracker *t) { t->EnableRadialZLUTCompareProfile(enable != 0); });
}

QTRK_API void QTRK_CALLCONV QTrkB200GetRadialZLUTCompareProfile(QueuedTracker *q, float *dst)
{
    guarded(q, "QTrkB200GetRadialZLUTCompareProfile", [&](Tracker *t) { t->GetRadialZLUTCompareProfile(dst); });
}

QTRK_API void QTRK_CALLCONV QTrkB200SetCUDADevices(const int *devices, int count)
{
    std::vector<int> d;
    for (int i = 0; devices && i < count; i++) d.push_back(devices[i]);
    qtrk::set_device_list(d);
}

QTRK_API ResultManager *QTRK_CALLCONV QTrkB200RMCreateNamed(const char *file, const char *frameinfo,
                                                           ResultManagerConfig *cfg, const char *const *names,
                                                           int count)
{
    if (!cfg) {
        set_last_error("QTrkB200RMCreateNamed: null config");
        return nullptr;
    }
    std::vector<std::string> cols;
    for (int i = 0; names && i < count; i++) cols.emplace_back(names[i] ? names[i] : "");
    try {
        return new ResultManager(file, frameinfo, *cfg, cols);
    } catch (const std::exception &e) {
        set_last_error(std::string("QTrkB200RMCreateNamed: ") + e.what());
        return nullptr;
    }
}
