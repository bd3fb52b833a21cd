/*
 * Stage-level C entry points into the reference CPU tracker, compiled together with a
 * copy of the reference's cputrack/ sources into oracle/_ref/libqtrk_ref.so.
 *
 * TEST INFRASTRUCTURE ONLY: the parity tests call these to check single stages of the
 * GPU path (COM, QI, radial profile, Z-LUT compare, Gaussian MLE) against the
 * reference's own code. The whole-pipeline oracle is the reference's unmodified C ABI
 * (cputrack/qtrk_c_api.cpp), which is linked into the same library.
 */
#include "std_incl.h"
#include "utils.h"
#include "QueuedTracker.h"
#include "cpu_tracker.h"

#define REF_EXPORT extern "C" __attribute__((visibility("default")))

/* CPUTracker::ComputeMeanAndCOM (cpu_tracker.cpp:681-729). out = {com.x, com.y, mean, stdev} */
REF_EXPORT void ref_stage_com(const float *img, int w, int h, float bgcorrection, float *out)
{
    CPUTracker trk(w, h);
    trk.SetImageFloat((float *)img);
    vector2f com = trk.ComputeMeanAndCOM(bgcorrection);
    out[0] = com.x;
    out[1] = com.y;
    out[2] = trk.mean;
    out[3] = trk.stdev;
}

/*
 * CPUTracker::ComputeQI (cpu_tracker.cpp:285-360), after ComputeMeanAndCOM so that the
 * tracker's `mean` (the fallback value for sparse bins) is set exactly as in
 * QueuedCPUTracker::ProcessJob (QueuedCPUTracker.cpp:291-306).
 * out = {x, y, boundaryHit}
 */
REF_EXPORT void ref_stage_qi(const float *img, int w, int h, float init_x, float init_y, int iterations,
                             int radialsteps, int angstepspq, float angstep_factor, float minradius,
                             float maxradius, const float *radialweights, float *out)
{
    CPUTracker trk(w, h);
    trk.SetImageFloat((float *)img);
    trk.ComputeMeanAndCOM(0.0f);
    bool bhit = false;
    vector2f p = trk.ComputeQI(vector2f(init_x, init_y), iterations, radialsteps, angstepspq, angstep_factor,
                               minradius, maxradius, bhit, (float *)radialweights);
    out[0] = p.x;
    out[1] = p.y;
    out[2] = bhit ? 1.0f : 0.0f;
}

/* CPUTracker::ComputeQuadrantProfile (cpu_tracker.cpp:631-677) for one quadrant. */
REF_EXPORT void ref_stage_quadrant_profile(const float *img, int w, int h, float cx, float cy, int radialsteps,
                                           int angularsteps_pq, int angularsteps, int quadrant, float minradius,
                                           float maxradius, const float *radialweights, float *dst)
{
    CPUTracker trk(w, h);
    trk.SetImageFloat((float *)img);
    trk.ComputeMeanAndCOM(0.0f);
    /* ComputeQI fills quadrantDirs; do the same here with a zero-iteration call. */
    bool bhit;
    trk.ComputeQI(vector2f(cx, cy), 0, radialsteps, angularsteps_pq, 1.0f, minradius, maxradius, bhit, 0);
    trk.ComputeQuadrantProfile(dst, radialsteps, angularsteps, quadrant, minradius, maxradius, vector2f(cx, cy),
                               (float *)radialweights);
}

/* ::ComputeRadialProfile (utils.cpp:275-320) with the image mean as the fallback value. */
REF_EXPORT void ref_stage_radial_profile(const float *img, int w, int h, float cx, float cy, int radialsteps,
                                         int angularsteps, float minradius, float maxradius, int normalize,
                                         float *dst)
{
    CPUTracker trk(w, h);
    trk.SetImageFloat((float *)img);
    trk.ComputeMeanAndCOM(0.0f);
    trk.ComputeRadialProfile(dst, radialsteps, angularsteps, minradius, maxradius, vector2f(cx, cy), false, 0,
                             normalize != 0);
}

/*
 * CPUTracker::LUTProfileCompare (cpu_tracker.cpp:791-868), mode LUTProfMaxQuadraticFit.
 * lut = [planes][radialsteps] for one bead. scores (may be NULL) receives the per-plane
 * scores. Returns z in plane units.
 */
REF_EXPORT float ref_stage_lut_compare(const float *profile, const float *lut, int planes, int radialsteps,
                                       const float *radialweights, float *scores)
{
    CPUTracker trk(8, 8);
    trk.SetRadialZLUT((float *)lut, planes, radialsteps, 1, 0.0f, 1.0f, true, false);
    trk.SetRadialWeights((float *)radialweights);
    return trk.LUTProfileCompare((float *)profile, 0, scores, CPUTracker::LUTProfMaxQuadraticFit);
}

/*
 * CPUTracker::Compute2DGaussianMLE (cpu_tracker.cpp:514-589), after ComputeMeanAndCOM
 * as in QueuedCPUTracker::ProcessJob (QueuedCPUTracker.cpp:291,309-313).
 * out = {x, y, I0, bg}
 */
REF_EXPORT void ref_stage_gauss2d(const float *img, int w, int h, float init_x, float init_y, int iterations,
                                  float sigma, float *out)
{
    CPUTracker trk(w, h);
    trk.SetImageFloat((float *)img);
    trk.ComputeMeanAndCOM(0.0f);
    CPUTracker::Gauss2DResult r = trk.Compute2DGaussianMLE(vector2f(init_x, init_y), iterations, sigma);
    out[0] = r.pos.x;
    out[1] = r.pos.y;
    out[2] = r.I0;
    out[3] = r.bg;
}

/* ComputeRadialBinWindow (utils.cpp:665-677). */
REF_EXPORT void ref_stage_radial_bin_window(int rsteps, float *dst)
{
    std::vector<float> w = ComputeRadialBinWindow(rsteps);
    for (int i = 0; i < rsteps; i++) dst[i] = w[i];
}

/* erf<float> as bound inside cpu_tracker.cpp (utils.h:395-417). */
REF_EXPORT float ref_stage_erf(float x) { return erf(x); }

/* QueuedTracker::ScheduleFrame's zlutIndex/skip rule is reached through QTrkScheduleFrame. */

/*
 * QueuedTracker::ComputeZBiasCorrection (QueuedTracker.cpp:143-189) on a tracker created through
 * the reference's C ABI; out = the count x bias_planes table (the reference also installs it as
 * the tracker's bias table).
 */
REF_EXPORT void ref_compute_zbias(QueuedTracker *qtrk, int bias_planes, float *out, int smp_per_pixel, int spline)
{
    CImageData result;
    qtrk->ComputeZBiasCorrection(bias_planes, &result, smp_per_pixel, spline != 0);
    for (int i = 0; i < result.w * result.h; i++) out[i] = result.data[i];
}

/* ReadLUTFile (utils.cpp:680-710) of "path#bead": out (max_n floats) receives the normalised
 * planes x radialsteps LUT; *w = radialsteps, *h = planes. */
REF_EXPORT void ref_read_lut_file(const char *spec, float *out, int max_n, int *w, int *h)
{
    ImageData lut = ReadLUTFile(spec);
    *w = lut.w;
    *h = lut.h;
    for (int i = 0; i < lut.w * lut.h && i < max_n; i++) out[i] = lut.data[i];
    lut.free();
}

/* SampleFisherMatrix::ComputeAverageFisher (FisherMatrix.h:106-135) as qtrk_compute_fisher
 * (lv_queuetrk_api.cpp:520-545) calls it: images from the LUT (lw bins x lh planes), sample range
 * (1,1,1), delta 0.001. out9 = the averaged 3x3 matrix (row major). */
#include "FisherMatrix.h"
REF_EXPORT void ref_average_fisher(const float *lut, int lw, int lh, float minr, float maxr, int w, int h, float px,
                                   float py, float pz, int nsamples, float maxval, float *out9)
{
    ImageData lutImg((float *)lut, lw, lh);
    SampleFisherMatrix fm(maxval);
    Matrix3X3 mat = fm.ComputeAverageFisher(vector3f(px, py, pz), nsamples, vector3f(1, 1, 1),
                                            vector3f(1, 1, 1) * 0.001f, w, h, [&](ImageData &out, vector3f pos) {
                                                GenerateImageFromLUT(&out, &lutImg, minr, maxr, pos);
                                            });
    for (int i = 0; i < 9; i++) out9[i] = mat[i];
}

/* QueuedTracker::SetPixelCalibrationImages (QueuedTracker.h:32, defined for the CPU tracker at
 * QueuedCPUTracker.cpp:165-196). The reference's C ABI declares QTrkSetPixelCalibrationImages
 * (qtrk_c_api.h) but defines no body for it, so the tests reach the method through this export.
 * The tracker must already hold its Z-LUT (the bead count sizes the images). */
REF_EXPORT void ref_set_pixel_calibration(QueuedTracker *qtrk, float *offset, float *gain)
{
    qtrk->SetPixelCalibrationImages(offset, gain);
}
