// LabVIEW binding (libqtrk_b200_lv.so) over the public C ABI of libqtrk_b200.so: the qtrk_* and
// rm_* functions of cputrack/lv_queuetrk_api.cpp and cputrack/lv_resultmanager_api.cpp. See
// include/qtrk_lv_api.h for the interface and its differences from the reference.
#include "qtrk_lv_api.h"

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

// LabVIEW run-time functions, provided by the LabVIEW process that loads this library.
extern "C" MgErr NumericArrayResize(int32_t typeCode, int32_t numDims, UHandle *dataHdlP, size_t totalNewSize);
extern "C" MgErr MoveBlock(const void *src, void *dest, size_t numBytes);

namespace {

// LabVIEW numeric type codes (cputrack/labview.h:58-71)
constexpr int32_t kU8 = 5, kI32 = 3, kU32 = 7, kF32 = 9;

std::string fmt(const char *f, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, f);
    std::vsnprintf(buf, sizeof(buf), f, ap);
    va_end(ap);
    return buf;
}

// SetLVString (lv_queuetrk_api.cpp:27-36): resize the string handle and copy the text in.
void set_lv_string(LStrHandle *h, const std::string &text)
{
    if (!h) return;
    if (NumericArrayResize(kU8, 1, reinterpret_cast<UHandle *>(h), text.size()) == QTRK_LV_mgNoErr && *h) {
        MoveBlock(text.data(), (**h)->str, text.size());
        (**h)->cnt = (int32_t)text.size();
    }
}

// FillErrorCluster / ArgumentErrorMsg (lv_queuetrk_api.cpp:50-63)
void fill_error(ErrorCluster *e, MgErr code, const std::string &msg)
{
    if (!e || !code) return;
    e->status = 1;
    e->code = code;
    set_lv_string(&e->message, msg);
}
void arg_error(ErrorCluster *e, const std::string &msg) { fill_error(e, QTRK_LV_mgArgErr, msg); }

std::string lib_error()
{
    char buf[2048];
    QTrkB200GetLastError(buf, sizeof(buf));
    return buf;
}

// Resize an N-D handle to dims (element count = product) and set its dimension sizes.
template <class Hdl>
bool resize(Hdl &h, int32_t code, std::initializer_list<int> dims)
{
    size_t n = 1;
    for (int d : dims) n *= (size_t)std::max(d, 0);
    if (NumericArrayResize(code, (int32_t)dims.size(), reinterpret_cast<UHandle *>(&h), n) != QTRK_LV_mgNoErr || !h ||
        !*h)
        return false;
    int i = 0;
    for (int d : dims) reinterpret_cast<int32_t *>(*h)[i++] = d;
    return true;
}

std::mutex g_mu;
std::vector<QueuedTracker *> g_trackers;
std::unordered_map<QueuedTracker *, QTrkSettings> g_settings;
std::unordered_set<ResultManager *> g_rms;
std::unordered_map<ResultManager *, QueuedTracker *> g_rm_tracker;

// ValidateTracker (lv_queuetrk_api.cpp:65-72)
bool valid(QueuedTracker *t, ErrorCluster *e, const char *fn)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (std::find(g_trackers.begin(), g_trackers.end(), t) == g_trackers.end()) {
        arg_error(e, fmt("QTrk C++ function %s called with invalid tracker pointer: %p", fn, (void *)t));
        return false;
    }
    return true;
}

QTrkComputedConfig config_of(QueuedTracker *t)
{
    QTrkSettings s;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        s = g_settings.at(t);
    }
    QTrkComputedConfig cc;
    QTrkGetComputedConfig(&s, &cc);
    return cc;
}

// CheckImageInput (lv_queuetrk_api.cpp:262-274)
template <class Hdl>
bool check_image(QueuedTracker *t, Hdl data, ErrorCluster *e, const char *fn)
{
    if (!valid(t, e, fn)) return false;
    if (!data || !*data) {
        arg_error(e, "Image data array is empty");
        return false;
    }
    const QTrkComputedConfig cc = config_of(t);
    if ((*data)->dimSizes[1] != cc.base.width || (*data)->dimSizes[0] != cc.base.height) {
        arg_error(e, fmt("Image data array has wrong size (%d,%d). Should be: (%d,%d)", (*data)->dimSizes[1],
                         (*data)->dimSizes[0], cc.base.width, cc.base.height));
        return false;
    }
    return true;
}

// Matrix3X3::Determinant / Inverse (cputrack/utils.h:314-338), in float.
struct M3 {
    float m[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    float &operator()(int r, int c) { return m[r * 3 + c]; }
    float at(int r, int c) const { return m[r * 3 + c]; }
    float det() const
    {
        return at(0, 0) * (at(1, 1) * at(2, 2) - at(2, 1) * at(1, 2)) -
               at(0, 1) * (at(1, 0) * at(2, 2) - at(1, 2) * at(2, 0)) +
               at(0, 2) * (at(1, 0) * at(2, 1) - at(1, 1) * at(2, 0));
    }
    // The matrix of cofactors times 1/det (zero when det == 0): the inverse for the symmetric
    // matrices it is used on here.
    M3 inverse() const
    {
        const float d = det();
        M3 r;
        if (d == 0.0f) return r;
        const float inv = 1 / d;
        r(0, 0) = (at(1, 1) * at(2, 2) - at(2, 1) * at(1, 2)) * inv;
        r(1, 0) = -(at(0, 1) * at(2, 2) - at(0, 2) * at(2, 1)) * inv;
        r(2, 0) = (at(0, 1) * at(1, 2) - at(0, 2) * at(1, 1)) * inv;
        r(0, 1) = -(at(1, 0) * at(2, 2) - at(1, 2) * at(2, 0)) * inv;
        r(1, 1) = (at(0, 0) * at(2, 2) - at(0, 2) * at(2, 0)) * inv;
        r(2, 1) = -(at(0, 0) * at(1, 2) - at(1, 0) * at(0, 2)) * inv;
        r(0, 2) = (at(1, 0) * at(2, 1) - at(2, 0) * at(1, 1)) * inv;
        r(1, 2) = -(at(0, 0) * at(2, 1) - at(2, 0) * at(0, 1)) * inv;
        r(2, 2) = (at(0, 0) * at(1, 1) - at(1, 0) * at(0, 1)) * inv;
        return r;
    }
};

float rand_uniform_f() { return rand() / (float)RAND_MAX; }  // cputrack/random_distr.h:2-6

}  // namespace

// ---------------------------------------------------------------------------------------
// tracker
// ---------------------------------------------------------------------------------------
QTRK_LV_API void qtrk_free_all(void)
{
    std::vector<QueuedTracker *> all;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        all.swap(g_trackers);
        g_settings.clear();
    }
    for (QueuedTracker *t : all) QTrkFreeInstance(t);
}

QTRK_LV_API int qtrk_get_debug_image(QueuedTracker *qtrk, int, LVArray2DFloatHdl , ErrorCluster *e)
{
    valid(qtrk, e, "qtrk_get_debug_image");
    return 0;  // no debug images are kept
}

QTRK_LV_API void qtrk_set_logfile_path(const char *) {}

QTRK_LV_API void qtrk_get_computed_config(QueuedTracker *qtrk, QTrkComputedConfig *cc, ErrorCluster *err)
{
    if (valid(qtrk, err, "get computed config") && cc) *cc = config_of(qtrk);
}

// lv_queuetrk_api.cpp:102-138
QTRK_LV_API void qtrk_set_ZLUT(QueuedTracker *tracker, LVArray3DFloatHdl pZlut, LVArrayFloatHdl zcmpWindow,
                               int normalize, ErrorCluster *e)
{
    if (!valid(tracker, e, "set ZLUT")) return;
    if (!pZlut || !*pZlut) {
        arg_error(e, "set_ZLUT: no array");
        return;
    }
    LVArray3DFloat *zlut = *pZlut;
    const int n = zlut->dimSizes[0], planes = zlut->dimSizes[1], res = zlut->dimSizes[2];
    float *zcmp = nullptr;
    if (zcmpWindow && *zcmpWindow && (*zcmpWindow)->dimSize > 0) {
        if ((*zcmpWindow)->dimSize != res)
            arg_error(e, fmt("Z Compare window should have the same resolution as the ZLUT (%d elements)", res));
        else
            zcmp = (*zcmpWindow)->elem;
    }
    if (n * planes * res == 0) {
        QTrkSetRadialZLUT(tracker, nullptr, 0, 0);
        return;
    }
    const QTrkComputedConfig cc = config_of(tracker);
    if (res != cc.zlut_radialsteps) {
        arg_error(e, fmt("set_ZLUT: 3rd dimension should have size of zlut_radialsteps (%d instead of %d)",
                         cc.zlut_radialsteps, res));
        return;
    }
    if (normalize)  // NormalizeZLUT, cputrack/utils.cpp:268-273 (in place, as the reference does)
        for (int i = 0; i < n * planes; i++) NormalizeRadialProfile(zlut->elem + (size_t)i * res, res);
    QTrkSetRadialZLUT(tracker, zlut->elem, n, planes);
    QTrkSetRadialWeights(tracker, zcmp);
}

QTRK_LV_API void qtrk_get_ZLUT(QueuedTracker *tracker, LVArray3DFloatHdl pzlut, ErrorCluster *e)
{
    if (!valid(tracker, e, "get ZLUT")) return;
    int d[3];
    QTrkGetRadialZLUTSize(tracker, &d[0], &d[1], &d[2]);
    if (d[0] * d[1] * d[2] > 0) {
        if (!resize(pzlut, kF32, {d[0], d[1], d[2]})) {
            fill_error(e, QTRK_LV_kAppErrorBase, "NumericArrayResize failed");
            return;
        }
        QTrkGetRadialZLUT(tracker, (*pzlut)->elem);
    }
}

QTRK_LV_API void qtrk_get_image_lut(QueuedTracker *qtrk, LVArray4DFloatHdl imageLUT, ErrorCluster *e)
{
    if (valid(qtrk, e, "get_image_lut") && imageLUT) resize(imageLUT, kF32, {0, 0, 0, 0});
}

QTRK_LV_API void qtrk_set_image_lut(QueuedTracker *qtrk, LVArray4DFloatHdl imageLUT, LVArray3DFloatHdl ,
                                    ErrorCluster *e)
{
    if (!valid(qtrk, e, "set_image_lut")) return;
    if (imageLUT && *imageLUT) {
        const int32_t *d = (*imageLUT)->dimSizes;
        if ((size_t)d[0] * d[1] * d[2] * d[3] > 0) arg_error(e, "set_image_lut: image LUTs are not supported");
    }
}

QTRK_LV_API void qtrk_set_pixel_calib_factors(QueuedTracker *qtrk, float offsetFactor, float gainFactor, ErrorCluster *e)
{
    if (valid(qtrk, e, "set pixel calib factors")) QTrkB200SetPixelCalibrationFactors(qtrk, offsetFactor, gainFactor);
}

// lv_queuetrk_api.cpp:187-221
QTRK_LV_API void qtrk_set_pixel_calib(QueuedTracker *qtrk, LVArray3DFloatHdl offset, LVArray3DFloatHdl gain,
                                      ErrorCluster *e)
{
    if (!valid(qtrk, e, "set pixel calibration images")) return;
    int count, planes, rsteps;
    QTrkGetRadialZLUTSize(qtrk, &count, &planes, &rsteps);
    const QTrkComputedConfig cc = config_of(qtrk);
    float *data[2] = {nullptr, nullptr};
    LVArray3DFloatHdl arr[2] = {offset, gain};
    const char *what[2] = {"Offset", "Gain"}, *lower[2] = {"offset", "gain"};
    for (int k = 0; k < 2; k++) {
        if (!arr[k] || !*arr[k] || (*arr[k])->dimSizes[0] == 0) continue;
        const int32_t *d = (*arr[k])->dimSizes;
        if (cc.base.width != d[2] || cc.base.height != d[1]) {
            arg_error(e, fmt("set_pixel_calib: %s images passed with invalid dimension (%d,%d)", what[k], d[2], d[1]));
            return;
        }
        if (count != d[0]) {
            arg_error(e, fmt("set_pixel_calib: Expecting %s to have %d images (same as ZLUT). %d given", lower[k],
                             count, d[0]));
            return;
        }
        data[k] = (*arr[k])->elem;
    }
    QTrkSetPixelCalibrationImages(qtrk, data[0], data[1]);
}

// lv_queuetrk_api.cpp:224-243
QTRK_LV_API QueuedTracker *qtrk_create(QTrkSettings *settings, LStrHandle warnings, ErrorCluster *e)
{
    if (!settings) {
        fill_error(e, QTRK_LV_kAppErrorBase, "qtrk_create: null settings");
        return nullptr;
    }
    QueuedTracker *t = QTrkCreateInstance(settings);
    if (!t) {
        fill_error(e, QTRK_LV_kAppErrorBase, lib_error());
        return nullptr;
    }
    char buf[8192];
    QTrkGetWarnings(t, buf, sizeof(buf));
    if (buf[0] && warnings) set_lv_string(&warnings, buf);
    std::lock_guard<std::mutex> lk(g_mu);
    g_trackers.push_back(t);
    g_settings[t] = *settings;
    return t;
}

QTRK_LV_API void qtrk_destroy(QueuedTracker *qtrk, ErrorCluster *error)
{
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = std::find(g_trackers.begin(), g_trackers.end(), qtrk);
        if (it == g_trackers.end()) {
            arg_error(error, fmt("Trying to call qtrk_destroy with invalid qtrk pointer %p", (void *)qtrk));
            return;
        }
        g_trackers.erase(it);
        g_settings.erase(qtrk);
    }
    QTrkFreeInstance(qtrk);
}

QTRK_LV_API void qtrk_queue_u16(QueuedTracker *qtrk, ErrorCluster *error, LVArray2DU16Hdl data,
                                const LocalizationJob *jobInfo)
{
    if (check_image(qtrk, data, error, "queue_u16"))
        QTrkScheduleLocalization(qtrk, (*data)->elem, 2 * (*data)->dimSizes[1], QTrkU16, jobInfo);
}

QTRK_LV_API void qtrk_queue_u8(QueuedTracker *qtrk, ErrorCluster *error, LVArray2DU8Hdl data, const LocalizationJob *jobInfo)
{
    if (check_image(qtrk, data, error, "queue_u8"))
        QTrkScheduleLocalization(qtrk, (*data)->elem, (*data)->dimSizes[1], QTrkU8, jobInfo);
}

QTRK_LV_API void qtrk_queue_float(QueuedTracker *qtrk, ErrorCluster *error, LVArray2DFloatHdl data,
                                  const LocalizationJob *jobInfo)
{
    if (check_image(qtrk, data, error, "queue_float"))
        QTrkScheduleLocalization(qtrk, (*data)->elem, 4 * (*data)->dimSizes[1], QTrkFloat, jobInfo);
}

QTRK_LV_API void qtrk_queue_pitchedmem(QueuedTracker *qtrk, uint8_t *data, int pitch, uint32_t pdt,
                                       const LocalizationJob *jobInfo)
{
    if (valid(qtrk, nullptr, "queue_pitchedmem")) QTrkScheduleLocalization(qtrk, data, pitch, (int)pdt, jobInfo);
}

// lv_queuetrk_api.cpp:310-326: the u8 array carries u8, u16 or float pixels (dimSizes[1] of them a row).
QTRK_LV_API void qtrk_queue_array(QueuedTracker *qtrk, ErrorCluster *error, LVArray2DU8Hdl data, uint32_t pdt,
                                  const LocalizationJob *jobInfo)
{
    if (!check_image(qtrk, data, error, "queue_array")) return;
    const int bpp = pdt == QTrkFloat ? 4 : (pdt == QTrkU16 ? 2 : 1);
    QTrkScheduleLocalization(qtrk, (*data)->elem, bpp * (*data)->dimSizes[1], (int)pdt, jobInfo);
}

QTRK_LV_API uint32_t qtrk_read_timestamp(uint8_t *image, int w, int h)
{
    if (w * h < 4 || !image) return 0;
    uint32_t ts;
    std::memcpy(&ts, image, 4);  // little endian, the first 4 pixels
    return ts;
}

QTRK_LV_API uint32_t qtrk_queue_frame(QueuedTracker *qtrk, uint8_t *image, int pitch, int w, int h, uint32_t pdt,
                                      ROIPosition *pos, int numROI, const LocalizationJob *pJobInfo, QueueFrameFlags,
                                      ErrorCluster *e)
{
    if (!valid(qtrk, e, "queue_frame") || !pJobInfo) return 0;
    LocalizationJob job = *pJobInfo;
    const int n = QTrkScheduleFrame(qtrk, image, pitch, w, h, pos, numROI, (int)pdt, &job);
    if (n != numROI)
        arg_error(e, fmt("Not all ROIs (%d out of %d) where queued. Check image borders vs ROIs.", n, numROI));
    return job.timestamp;
}

QTRK_LV_API void qtrk_clear_results(QueuedTracker *qtrk, ErrorCluster *e)
{
    if (valid(qtrk, e, "clear results")) QTrkClearResults(qtrk);
}

// lv_queuetrk_api.cpp:359-378: data = [numbeads][height][width] float.
QTRK_LV_API void qtrk_build_lut_plane(QueuedTracker *qtrk, LVArray3DFloatHdl data, uint32_t, int plane, ErrorCluster *err)
{
    if (!valid(qtrk, err, "build_lut_plane")) return;
    const QTrkComputedConfig cc = config_of(qtrk);
    const int32_t *d = (*data)->dimSizes;
    if (d[2] != cc.base.width || d[1] != cc.base.height) {
        arg_error(err, fmt("Invalid size: %dx%d. Expecting %dx%d\n", d[2], d[1], cc.base.width, cc.base.height));
        return;
    }
    int cnt, planes, rsteps;
    QTrkGetRadialZLUTSize(qtrk, &cnt, &planes, &rsteps);
    if (d[0] != cnt) {
        arg_error(err, fmt("Invalid number of images given (%d). Expecting %d", d[0], cnt));
        return;
    }
    QTrkBuildLUT(qtrk, (*data)->elem, (int)sizeof(float) * cc.base.width, QTrkFloat, plane, nullptr);
}

QTRK_LV_API void qtrk_finalize_lut(QueuedTracker *qtrk, ErrorCluster *e)
{
    if (valid(qtrk, e, "finalize_lut")) QTrkFinalizeLUT(qtrk);
}

QTRK_LV_API int qtrk_get_queue_len(QueuedTracker *qtrk, int *maxQueueLen, ErrorCluster *e)
{
    return valid(qtrk, e, "fullqueue") ? QTrkGetQueueLength(qtrk, maxQueueLen) : 0;
}

QTRK_LV_API int qtrk_resultcount(QueuedTracker *qtrk, ErrorCluster *e)
{
    return valid(qtrk, e, "resultcount") ? QTrkGetResultCount(qtrk) : 0;
}

QTRK_LV_API void qtrk_flush(QueuedTracker *qtrk, ErrorCluster *e)
{
    if (valid(qtrk, e, "flush")) QTrkFlush(qtrk);
}

QTRK_LV_API int qtrk_get_results(QueuedTracker *qtrk, LocalizationResult *results, int maxResults, int sortByID,
                                 ErrorCluster *e)
{
    if (!valid(qtrk, e, "get_results")) return 0;
    const int n = QTrkFetchResults(qtrk, results, maxResults);
    if (sortByID && n > 1)
        std::sort(results, results + n,
                  [](const LocalizationResult &a, const LocalizationResult &b) { return a.job.frame < b.job.frame; });
    return n;
}

QTRK_LV_API void qtrk_get_zlut_cmpprof(QueuedTracker *qtrk, LVArray2DFloatHdl output, ErrorCluster *e)
{
    if (!valid(qtrk, e, "get zlut compare profiles")) return;
    int cnt, planes, rsteps;
    QTrkGetRadialZLUTSize(qtrk, &cnt, &planes, &rsteps);
    if (resize(output, kF32, {cnt, planes})) QTrkB200GetRadialZLUTCompareProfile(qtrk, (*output)->elem);
}

QTRK_LV_API void qtrk_enable_zlut_cmpprof(QueuedTracker *qtrk, bool enable, ErrorCluster *e)
{
    if (valid(qtrk, e, "enable zlut cmpprof")) QTrkB200EnableRadialZLUTCompareProfile(qtrk, enable ? 1 : 0);
}

QTRK_LV_API void qtrk_set_localization_mode(QueuedTracker *qtrk, uint32_t locType, ErrorCluster *e)
{
    if (valid(qtrk, e, "set_localization_mode")) QTrkSetLocalizationMode(qtrk, (int)locType);
}

QTRK_LV_API int qtrk_idle(QueuedTracker *qtrk, ErrorCluster *e)
{
    return valid(qtrk, e, "is_idle") && QTrkIsIdle(qtrk) ? 1 : 0;
}

// lv_queuetrk_api.cpp:457-466: result is [beads][bias_planes].
QTRK_LV_API void qtrk_compute_zlut_bias_table(QueuedTracker *qtrk, int bias_planes, LVArray2DFloatHdl lvresult,
                                              int smpPerPixel, int useSplineInterp, ErrorCluster *e)
{
    if (!valid(qtrk, e, "compute_zlut_bias_table")) return;
    int cnt, planes, rsteps;
    QTrkGetRadialZLUTSize(qtrk, &cnt, &planes, &rsteps);
    std::vector<float> table((size_t)cnt * std::max(bias_planes, 0));
    QTrkB200ComputeZLUTBiasTable(qtrk, bias_planes, table.data(), smpPerPixel, useSplineInterp);
    if (resize(lvresult, kF32, {cnt, bias_planes}))
        std::memcpy((*lvresult)->elem, table.data(), sizeof(float) * table.size());
}

// lv_queuetrk_api.cpp:468-481: table [numbeads][biasplanes].
QTRK_LV_API void qtrk_set_zlut_bias_table(QueuedTracker *qtrk, LVArray2DFloatHdl biastbl, ErrorCluster *e)
{
    if (!valid(qtrk, e, "set zlut bias table")) return;
    int cnt, planes, rsteps;
    QTrkGetRadialZLUTSize(qtrk, &cnt, &planes, &rsteps);
    if ((*biastbl)->dimSizes[0] != cnt) {
        arg_error(e, fmt("Bias table should be [numbeads] high and [biasplanes] wide. Expected #beads=%d", cnt));
        return;
    }
    QTrkB200SetZLUTBiasTable(qtrk, (*biastbl)->elem, (*biastbl)->dimSizes[1], (*biastbl)->dimSizes[0]);
}

QTRK_LV_API void qtrk_generate_gaussian_spot(LVArray2DFloatHdl image, vector2f *pos, float sigma, float I0, float Ibg,
                                             int applyNoise)
{
    ImageData img{(*image)->elem, (*image)->dimSizes[1], (*image)->dimSizes[0]};
    GenerateGaussianSpotImage(&img, *pos, sigma, I0, Ibg);
    if (applyNoise) ApplyPoissonNoise(&img, 1, 255);
}

QTRK_LV_API void qtrk_generate_image_from_lut(LVArray2DFloatHdl image, LVArray2DFloatHdl lut, float *LUTradii,
                                              vector2f *position, float z, float, float sigma_noise)
{
    ImageData img{(*image)->elem, (*image)->dimSizes[1], (*image)->dimSizes[0]};
    ImageData zlut{(*lut)->elem, (*lut)->dimSizes[1], (*lut)->dimSizes[0]};
    GenerateImageFromLUT(&img, &zlut, LUTradii[0], LUTradii[1], vector3f{position->x, position->y, z}, true, 4);
    if (sigma_noise > 0) ApplyGaussianNoise(&img, sigma_noise);
}

QTRK_LV_API void qtrk_dump_memleaks(void) {}

QTRK_LV_API void qtrk_get_profile_report(QueuedTracker *qtrk, LStrHandle str)
{
    if (!valid(qtrk, nullptr, "get_profile_report")) return;
    char buf[16384];
    QTrkGetProfileReport(qtrk, buf, sizeof(buf));
    set_lv_string(&str, buf);
}

// lv_queuetrk_api.cpp:520-545 with SampleFisherMatrix (cputrack/FisherMatrix.h): the Fisher matrix
// of the Poisson image model (images from the LUT, scaled so the mean image is maxPixelValue),
// from central differences (delta 0.001 in x, y, z), averaged over Nsamples positions drawn
// uniformly from [-0.5, 0.5] x [-0.5, 0.5] x [0, 1] around *pos (libc rand()).
QTRK_LV_API void qtrk_compute_fisher(LVArray2DFloatHdl lut, QTrkSettings *cfg, vector3f *pos,
                                     LVArray2DFloatHdl fisherMatrix, LVArray2DFloatHdl inverseMatrix,
                                     vector3f *xyzVariance, int Nsamples, float maxPixelValue)
{
    if (!lut || !*lut || !cfg || !pos || Nsamples <= 0) return;
    QTrkComputedConfig cc;
    QTrkGetComputedConfig(cfg, &cc);
    const int w = cfg->width, h = cfg->height;
    ImageData L{(*lut)->elem, (*lut)->dimSizes[1], (*lut)->dimSizes[0]};
    auto gen = [&](std::vector<float> &out, float x, float y, float z) {
        out.assign((size_t)w * h, 0.0f);
        ImageData img{out.data(), w, h};
        GenerateImageFromLUT(&img, &L, cc.base.zlut_minradius, cc.zlut_maxradius, vector3f{x, y, z}, true, 4);
    };
    const float delta = 0.001f;
    std::vector<float> mu, p[3], m[3];
    std::vector<M3> results(Nsamples);
    for (int s = 0; s < Nsamples; s++) {
        // vector3f(U - 0.5, U - 0.5, U) of FisherMatrix.h:111, whose arguments g++ evaluates last to first
        const float rz = rand_uniform_f();
        const float ry = rand_uniform_f() - 0.5f;
        const float rx = rand_uniform_f() - 0.5f;
        const float px = pos->x + 1.0f * rx, py = pos->y + 1.0f * ry, pz = pos->z + 1.0f * rz;
        gen(mu, px, py, pz);
        float meanv = 0.0f;
        for (float v : mu) meanv += v;
        meanv /= (float)(w * h);
        gen(p[0], px + delta, py, pz);
        gen(p[1], px, py + delta, pz);
        gen(p[2], px, py, pz + delta);
        gen(m[0], px - delta, py, pz);
        gen(m[1], px, py - delta, pz);
        gen(m[2], px, py, pz - delta);
        const float inv2d = 1.0f / (2 * delta);
        for (int k = 0; k < 3; k++)
            for (size_t i = 0; i < p[k].size(); i++) p[k][i] = (p[k][i] - m[k][i]) * inv2d;
        auto elem = [&](int a, int b) {
            double sum = 0;
            for (size_t i = 0; i < mu.size(); i++) sum += (double)p[a][i] * (double)p[b][i] / (1e-5f + (double)mu[i]);
            return sum;
        };
        M3 f;
        const double xx = elem(0, 0), yy = elem(1, 1), zz = elem(2, 2), xy = elem(0, 1), xz = elem(0, 2), yz = elem(1, 2);
        f(0, 0) = (float)xx, f(0, 1) = (float)xy, f(0, 2) = (float)xz;
        f(1, 0) = (float)xy, f(1, 1) = (float)yy, f(1, 2) = (float)yz;
        f(2, 0) = (float)xz, f(2, 1) = (float)yz, f(2, 2) = (float)zz;
        for (float &v : f.m) v *= maxPixelValue / meanv;
        results[s] = f;
    }
    M3 acc;
    for (const M3 &r : results)
        for (int i = 0; i < 9; i++) acc.m[i] += r.m[i];
    for (float &v : acc.m) v *= 1.0f / Nsamples;
    const M3 inv = acc.inverse();
    if (fisherMatrix && resize(fisherMatrix, kF32, {3, 3})) std::memcpy((*fisherMatrix)->elem, acc.m, sizeof(acc.m));
    if (inverseMatrix && resize(inverseMatrix, kF32, {3, 3})) std::memcpy((*inverseMatrix)->elem, inv.m, sizeof(inv.m));
    if (xyzVariance) *xyzVariance = vector3f{inv.at(0, 0), inv.at(1, 1), inv.at(2, 2)};
}

// lv_queuetrk_api.cpp:548-562 with BeadFinder::Find(uint8_t*, ...) (BeadFinder.cpp:225-245): the u8
// frame as float, sample at smpCornerPos (rows at the frame width; the reference steps them by the
// height). output = [beads][2] (x, y).
QTRK_LV_API void qtrk_find_beads(uint8_t *image, int pitch, int w, int h, int *smpCornerPos, int roi, float imgRelDist,
                                 float acceptance, LVArray2DUIntHdl output)
{
    if (!image || !smpCornerPos || w <= 0 || h <= 0) return;
    std::vector<float> f((size_t)w * h);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) f[(size_t)y * w + x] = image[(size_t)y * pitch + x];
    ImageData img{f.data(), w, h};
    int n = 0;
    ROIPosition *pos = QTrkFindBeads(&img, smpCornerPos[0], smpCornerPos[1], roi, imgRelDist, acceptance, &n, nullptr);
    if (output && resize(output, kU32, {n, 2}))
        for (int i = 0; i < n; i++) {
            (*output)->elem[2 * i] = (uint32_t)pos[i].x;
            (*output)->elem[2 * i + 1] = (uint32_t)pos[i].y;
        }
    QTrkFreeROIPositions(pos);
}

// lv_queuetrk_api.cpp:565-588: fills the arrays with a known pattern (binding self-test).
QTRK_LV_API void test_array_passing(int n, LVArrayFloatHdl flt1D, LVArray2DFloatHdl flt2D, LVArrayIntHdl int1D,
                                    LVArray2DIntHdl int2D)
{
    if (!resize(flt1D, kF32, {n}) || !resize(int1D, kI32, {n}) || !resize(flt2D, kF32, {n / 2, n}) ||
        !resize(int2D, kI32, {n / 2, n}))
        return;
    for (int i = 0; i < n; i++) {
        (*int1D)->elem[i] = (i + 1) * i;
        (*flt1D)->elem[i] = std::sqrt((float)i);
        for (int j = 0; j < n / 2; j++) {
            (*int2D)->elem[j * n + i] = j * 2 + i;
            (*flt2D)->elem[j * n + i] = (float)(j * 2 + i);
        }
    }
}

// lv_queuetrk_api.cpp:590-643: nsmp images of bead beadIndex's LUT at centerPos + range * U[0,1]^3
// (libc rand()), Poisson noise, localized; outBias = sum of (result - truth) (as the reference
// reports it), outScatter = RMS deviation from the mean error.
QTRK_LV_API void qtrk_simulate_tracking(QueuedTracker *qtrk, int nsmp, int beadIndex, vector3f *centerPos,
                                        vector3f *range, vector3f *outBias, vector3f *outScatter,
                                        float photonsPerWell, ErrorCluster *e)
{
    if (!valid(qtrk, e, "qtrk_simulate_tracking") || nsmp <= 0) return;
    int cnt, planes, rsteps;
    QTrkGetRadialZLUTSize(qtrk, &cnt, &planes, &rsteps);
    if (beadIndex < 0 || beadIndex >= cnt) {
        arg_error(e, fmt("qtrk_simulate_tracking: bead index %d outside the Z-LUT (%d beads)", beadIndex, cnt));
        return;
    }
    std::vector<float> lut((size_t)cnt * planes * rsteps);
    QTrkGetRadialZLUT(qtrk, lut.data());
    const QTrkComputedConfig cc = config_of(qtrk);
    const int w = cc.base.width, h = cc.base.height;
    std::vector<float> buf((size_t)w * h);
    ImageData img{buf.data(), w, h};
    ImageData zlut{lut.data() + (size_t)rsteps * planes * beadIndex, rsteps, planes};
    std::vector<vector3f> truth(nsmp);
    for (int i = 0; i < nsmp; i++) {
        // vector3f(U, U, U) of lv_queuetrk_api.cpp:607, arguments evaluated last to first (g++)
        const float uz = rand_uniform_f();
        const float uy = rand_uniform_f();
        const float ux = rand_uniform_f();
        truth[i] = vector3f{centerPos->x + range->x * ux, centerPos->y + range->y * uy, centerPos->z + range->z * uz};
        GenerateImageFromLUT(&img, &zlut, cc.base.zlut_minradius, cc.zlut_maxradius, truth[i], true, 4);
        ApplyPoissonNoise(&img, photonsPerWell, 255);
        LocalizationJob job{};
        job.frame = (uint32_t)i;
        job.timestamp = (uint32_t)i;
        job.zlutIndex = beadIndex;
        QTrkScheduleLocalization(qtrk, buf.data(), (int)sizeof(float) * w, QTrkFloat, &job);
    }
    QTrkFlush(qtrk);
    std::vector<LocalizationResult> res(nsmp);
    int got = 0;
    while (got < nsmp) {
        const int n = QTrkFetchResults(qtrk, res.data() + got, nsmp - got);
        if (n < 0) break;
        got += n;
        if (!n && QTrkIsIdle(qtrk) && QTrkGetResultCount(qtrk) == 0) break;
    }
    vector3f sb{0, 0, 0}, ss{0, 0, 0};
    for (int i = 0; i < got; i++) {
        const vector3f &t = truth[res[i].job.frame];
        sb.x += res[i].pos.x - t.x, sb.y += res[i].pos.y - t.y, sb.z += res[i].pos.z - t.z;
    }
    const vector3f mb{sb.x / nsmp, sb.y / nsmp, sb.z / nsmp};
    for (int i = 0; i < got; i++) {
        const vector3f &t = truth[res[i].job.frame];
        const float dx = res[i].pos.x - t.x - mb.x, dy = res[i].pos.y - t.y - mb.y, dz = res[i].pos.z - t.z - mb.z;
        ss.x += dx * dx, ss.y += dy * dy, ss.z += dz * dz;
    }
    if (outScatter) *outScatter = vector3f{std::sqrt(ss.x / nsmp), std::sqrt(ss.y / nsmp), std::sqrt(ss.z / nsmp)};
    if (outBias) *outBias = sb;
}

QTRK_LV_API void qtrkcuda_set_device_list(LVArrayIntHdl devices)
{
    if (devices && *devices) QTrkB200SetCUDADevices((*devices)->elem, (*devices)->dimSize);
}

QTRK_LV_API int qtrkcuda_device_count(ErrorCluster *e)
{
    int c = 0;
    const cudaError_t err = cudaGetDeviceCount(&c);
    if (err != cudaSuccess) {
        fill_error(e, QTRK_LV_kAppErrorBase, fmt("CUDA error: %s", cudaGetErrorString(err)));
        return 0;
    }
    return c;
}

QTRK_LV_API void qtrkcuda_get_device(int device, CUDADeviceInfo *info, ErrorCluster *e)
{
    cudaDeviceProp prop;
    const cudaError_t err = cudaGetDeviceProperties(&prop, device);
    if (err != cudaSuccess) {
        fill_error(e, QTRK_LV_kAppErrorBase, fmt("CUDA error: %s", cudaGetErrorString(err)));
        return;
    }
    if (!info) return;
    info->multiProcCount = prop.multiProcessorCount;
    int clock = 0;
    cudaDeviceGetAttribute(&clock, cudaDevAttrClockRate, device);
    info->clockRate = clock;
    info->major = prop.major;
    info->minor = prop.minor;
    set_lv_string(&info->name, prop.name);
}

QTRK_LV_API void qtrkcuda_enable_texture_cache(QueuedTracker *qtrk, int, ErrorCluster *e)
{
    valid(qtrk, e, "enable_texture_cache");  // no texture path: nothing to switch
}

// ---------------------------------------------------------------------------------------
// ResultManager (cputrack/lv_resultmanager_api.cpp)
// ---------------------------------------------------------------------------------------
namespace {
bool valid_rm(ResultManager *rm, ErrorCluster *err)
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_rms.count(rm)) {
        arg_error(err, "Invalid ResultManager instance passed.");
        return false;
    }
    return true;
}
}  // namespace

QTRK_LV_API void rm_destroy_all(void)
{
    std::unordered_set<ResultManager *> all;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        all.swap(g_rms);
        g_rm_tracker.clear();
    }
    for (ResultManager *rm : all) RMDestroy(rm);
}

QTRK_LV_API ResultManager *rm_create(const char *file, const char *frameinfo, ResultManagerConfig *cfg, LStrHandle *names)
{
    if (!cfg) return nullptr;
    std::vector<std::string> cols;
    std::vector<const char *> ptrs;
    if (names)
        for (int i = 0; i < cfg->numFrameInfoColumns; i++)
            cols.emplace_back(names[i] ? std::string((const char *)(*names[i])->str, (size_t)(*names[i])->cnt) : "");
    for (const std::string &c : cols) ptrs.push_back(c.c_str());
    ResultManager *rm = QTrkB200RMCreateNamed(file, frameinfo, cfg, ptrs.data(), (int)ptrs.size());
    if (rm) {
        std::lock_guard<std::mutex> lk(g_mu);
        g_rms.insert(rm);
    }
    return rm;
}

QTRK_LV_API void rm_set_tracker(ResultManager *rm, QueuedTracker *qtrk, ErrorCluster *err)
{
    if (!valid_rm(rm, err)) return;
    RMSetTracker(rm, qtrk);
    std::lock_guard<std::mutex> lk(g_mu);
    g_rm_tracker[rm] = qtrk;
}

QTRK_LV_API void rm_destroy(ResultManager *rm, ErrorCluster *err)
{
    if (!valid_rm(rm, err)) return;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        g_rms.erase(rm);
        g_rm_tracker.erase(rm);
    }
    RMDestroy(rm);
}

QTRK_LV_API void rm_store_frame_info(ResultManager *rm, int frame, double timestamp, float *cols, ErrorCluster *err)
{
    if (valid_rm(rm, err)) RMStoreFrameInfo(rm, frame, timestamp, cols);
}

QTRK_LV_API int rm_getbeadresults(ResultManager *rm, int start, int numFrames, int bead, LocalizationResult *results,
                                  ErrorCluster *err)
{
    if (!valid_rm(rm, err)) return 0;
    ResultManagerConfig cfg;
    RMGetConfig(rm, &cfg);
    if (bead < 0 || bead >= cfg.numBeads) {
        arg_error(err, fmt("Invalid bead index: %d. Accepted range: [0-%d]", bead, cfg.numBeads));
        return 0;
    }
    return RMGetBeadResults(rm, start, numFrames, bead, results);
}

QTRK_LV_API void rm_getframecounters(ResultManager *rm, int *startFrame, int *lastSaveFrame, int *endFrame,
                                     int *capturedFrames, int *localizationsDone, int *lostFrames, ErrorCluster *err)
{
    if (!valid_rm(rm, err)) return;
    RMFrameCounters c;
    RMGetFrameCounters(rm, &c);
    if (startFrame) *startFrame = c.startFrame;
    if (lastSaveFrame) *lastSaveFrame = c.lastSaveFrame;
    if (endFrame) *endFrame = c.processedFrames;
    if (capturedFrames) *capturedFrames = c.capturedFrames;
    if (localizationsDone) *localizationsDone = c.localizationsDone;
    if (lostFrames) *lostFrames = c.lostFrames;
}

QTRK_LV_API void rm_flush(ResultManager *rm, ErrorCluster *err)
{
    if (valid_rm(rm, err)) RMFlush(rm);
}

QTRK_LV_API int rm_getresults(ResultManager *rm, int startFrame, int numFrames, LocalizationResult *results,
                              ErrorCluster *err)
{
    return valid_rm(rm, err) ? RMGetResults(rm, startFrame, numFrames, results) : 0;
}

// lv_resultmanager_api.cpp:106-116: reported as an error while a tracker is attached, but the
// bead is removed all the same.
QTRK_LV_API void rm_removebead(ResultManager *rm, int bead, ErrorCluster *err)
{
    if (!valid_rm(rm, err)) return;
    bool attached;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        auto it = g_rm_tracker.find(rm);
        attached = it != g_rm_tracker.end() && it->second;
    }
    if (attached) arg_error(err, "Cannot discard bead results while tracking in progress");
    RMRemoveBead(rm, bead);
}

QTRK_LV_API void rm_getconfig(ResultManager *rm, ResultManagerConfig *cfg, ErrorCluster *err)
{
    if (valid_rm(rm, err) && cfg) RMGetConfig(rm, cfg);
}
