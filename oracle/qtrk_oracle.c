/*
 * qtrk_oracle.c — FP64 CPU restatement of QTrk's bead-localization path.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the GPU library: tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg may load it; the product
 * library never does. It restates, in double precision and in my own code, the
 * algorithms of the reference CPU tracker (jcnossen/qtrk cputrack/), keeping every
 * discrete decision of the reference identical (int truncations, the bilinear
 * "outside" rule, sample-count thresholds, the argmax window of the quadratic fit).
 * It is pinned against the reference itself, compiled from its own sources into
 * oracle/_ref/libqtrk_ref.so (tests/test_oracle_pin.py) and through the committed
 * fixtures in tests/golden/.
 *
 * The QI cross-correlation is evaluated as a direct O(L^2) circular correlation in
 * double instead of KISS FFT: the result of the reference's FFT path
 * (cpu_tracker.cpp:375-406) is the same mathematical quantity, so only rounding differs.
 *
 * Beyond the reference it also holds FP64 versions of the extensions of the GPU library:
 * the 5-parameter Gaussian MLE, the radial-profile/LUT cost with its analytic gradient
 * (x, y, z and LUT entries), and the joint Gauss-Newton (x,y,z) refinement.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

/* Reference constants: QueuedTracker.h:349,359 (fit weights), QueuedTracker.h:261 (min samples). */
static const double QI_WEIGHTS[7] = {0.14, 0.5, 0.85, 1.0, 0.85, 0.5, 0.14};
static const double ZLUT_WEIGHTS[7] = {0.15, 0.5, 0.85, 1.0, 0.85, 0.5, 0.15};
#define MIN_RADPROFILE_SMP_COUNT 4
#define REF_PI_F 3.141593 /* the reference writes pi as 3.141593f in its angle tables */

/* Localization mode flags, cputrack/qtrk_c_api.h:5-20. */
#define LT_QI 2
#define LT_Gaussian2D 4
#define LT_LocalizeZ 16
#define LT_NormalizeProfile 64
#define LT_ClearFirstFourPixels 128

#pragma pack(push, 1)
typedef struct {
    int width, height, numThreads, cuda_device;
    float com_bgcorrection, zlut_minradius, zlut_radial_coverage, zlut_angular_coverage, zlut_roi_coverage;
    int qi_iterations;
    float qi_minradius, qi_radial_coverage, qi_angular_coverage, qi_roi_coverage, qi_angstep_factor;
    int xc1_profileLength, xc1_profileWidth, xc1_iterations, gauss2D_iterations;
    float gauss2D_sigma;
    int downsample;
    int zlut_radialsteps, zlut_angularsteps;
    float zlut_maxradius;
    int qi_radialsteps, qi_angstepspq;
    float qi_maxradius;
} oracle_config; /* layout of QTrkComputedConfig, cputrack/qtrk_c_api.h:59-138 */
#pragma pack(pop)

/* NearestPowerOf2, utils.cpp:644-652 (int/float arithmetic kept as in the reference). */
ORACLE_API int oracle_nearest_pow2(int v)
{
    int r = 1;
    while (r < v) r *= 2;
    if (fabsf((float)(r - v)) < fabsf((float)(r / 2 - v))) return r;
    return r / 2;
}

/* QTrkComputedConfig::Update, QueuedTracker.cpp:6-21. Float arithmetic and int truncation as
 * in the reference, because the step counts it produces are discrete. */
ORACLE_API void oracle_update_config(oracle_config *c)
{
    int roi = c->width / 2;
    c->zlut_maxradius = roi * c->zlut_roi_coverage;
    float zlut_perimeter = 2 * 3.141593f * c->zlut_maxradius;
    c->zlut_angularsteps = (int)(zlut_perimeter * c->zlut_angular_coverage);
    c->zlut_radialsteps = (int)((c->zlut_maxradius - c->zlut_minradius) * c->zlut_radial_coverage);
    c->qi_maxradius = roi * c->qi_roi_coverage;
    float qi_perimeter = 2 * 3.141593f * c->qi_maxradius;
    c->qi_angstepspq = (int)(qi_perimeter * c->qi_angular_coverage / 4);
    c->qi_radialsteps = (int)((c->qi_maxradius - c->qi_minradius) * c->qi_radial_coverage);
    c->qi_radialsteps = oracle_nearest_pow2(c->qi_radialsteps);
}

/* ComputeRadialBinWindow, utils.cpp:665-677. */
ORACLE_API void oracle_radial_bin_window(int rsteps, double *dst)
{
    for (int i = 0; i < rsteps; i++) {
        double x = i / (double)rsteps;
        double fall = 1.0 - exp(-(1 - x) * (1 - x) / 0.05);
        double rise = 1.0 - exp(-(x * x) / 0.01);
        dst[i] = sqrt(fall * rise * x * 2);
    }
}

/* Interpolate, utils.h:40-58: truncating conversion, outside when rx<0, ry<0, rx+1>=w, ry+1>=h. */
static double bilinear(const double *img, int w, int h, double x, double y, int *outside)
{
    int rx = (int)x, ry = (int)y;
    if (rx < 0 || ry < 0 || rx + 1 >= w || ry + 1 >= h) {
        *outside = 1;
        return 0.0;
    }
    *outside = 0;
    double v00 = img[w * ry + rx], v10 = img[w * ry + rx + 1];
    double v01 = img[w * (ry + 1) + rx], v11 = img[w * (ry + 1) + rx + 1];
    double fx = x - rx, fy = y - ry;
    double v0 = v00 + (v10 - v00) * fx;
    double v1 = v01 + (v11 - v01) * fx;
    return v0 + (v1 - v0) * fy;
}

/* CPUTracker::CheckBoundaries, cpu_tracker.cpp:182-188. */
static int check_boundaries(double cx, double cy, double radius, int w, int h)
{
    return cx + radius >= w || cx - radius < 0 || cy + radius >= h || cy - radius < 0;
}

/* CPUTracker::ComputeMeanAndCOM, cpu_tracker.cpp:681-729. out = {x, y, mean, stdev}. */
ORACLE_API void oracle_com(const double *img, int w, int h, double bgcorrection, double *out)
{
    double sum = 0, sum2 = 0;
    int n = w * h;
    for (int i = 0; i < n; i++) {
        sum += img[i];
        sum2 += img[i] * img[i];
    }
    double mean = sum / n;
    double stdev = sqrt(sum2 / n - mean * mean);
    double s = 0, mx = 0, my = 0;
    for (int x = 0; x < w; x++)
        for (int y = 0; y < h; y++) {
            double v = fabs(img[y * w + x] - mean) - bgcorrection * stdev;
            if (v < 0) v = 0;
            s += v;
            mx += x * v;
            my += y * v;
        }
    out[0] = mx / s;
    out[1] = my / s;
    out[2] = mean;
    out[3] = stdev;
}

/* LsqSqQuadFit + ComputeMaxInterp<T,7>::Compute, LsqQuadraticFit.h:8-129,132-176.
 * Note the reference's weight indexing: weights[0..numpoints) even when the window is
 * clipped at the start of the array. */
ORACLE_API double oracle_max_interp7(const double *data, int len, const double *weights)
{
    int iMax = 0;
    double vMax = data[0];
    for (int k = 1; k < len; k++)
        if (data[k] > vMax) {
            vMax = data[k];
            iMax = k;
        }
    int startPos = iMax - 3 > 0 ? iMax - 3 : 0;
    int endPos = iMax + 4 < len ? iMax + 4 : len;
    int np = endPos - startPos;
    if (np < 3) return iMax;
    double Sx = 0, Sy = 0, Sx2 = 0, Sx3 = 0, Sx4 = 0, Sxy = 0, Sx2y = 0, Sw = 0;
    for (int i = 0; i < np; i++) {
        double x = (startPos + i) - iMax, y = data[startPos + i], wt = weights[i];
        double sq = x * x;
        Sx += x * wt;
        Sy += y * wt;
        Sx2 += sq * wt;
        Sx3 += sq * x * wt;
        Sx4 += sq * sq * wt;
        Sxy += x * y * wt;
        Sx2y += sq * y * wt;
        Sw += wt;
    }
    double s40 = Sx4, s30 = Sx3, s20 = Sx2, s10 = Sx, s21 = Sx2y, s11 = Sxy, s01 = Sy, s00 = Sw;
    double d = s40 * (s20 * s00 - s10 * s10) - s30 * (s30 * s00 - s10 * s20) + s20 * (s30 * s10 - s20 * s20);
    double a = (s21 * (s20 * s00 - s10 * s10) - s11 * (s30 * s00 - s10 * s20) + s01 * (s30 * s10 - s20 * s20)) / d;
    double b = (s40 * (s11 * s00 - s01 * s10) - s30 * (s21 * s00 - s01 * s20) + s20 * (s21 * s10 - s11 * s20)) / d;
    if (fabs(a) < 1e-9) return iMax;
    return iMax + (-b / (2 * a));
}

/* CPUTracker::ComputeQuadrantProfile, cpu_tracker.cpp:631-677, with the quadrant
 * direction table of cpu_tracker.cpp:294-300 (angular_pq entries). */
static void quadrant_profile(const double *img, int w, int h, double mean, double *dst, int nr, int angular_pq,
                             int angsteps, int q, double minR, double maxR, double cx, double cy,
                             const double *rweights)
{
    static const int qmat[8] = {1, 1, -1, 1, -1, -1, 1, -1};
    int mx = qmat[2 * q], my = qmat[2 * q + 1];
    if (angsteps < MIN_RADPROFILE_SMP_COUNT) angsteps = MIN_RADPROFILE_SMP_COUNT;
    double rstep = (maxR - minR) / nr;
    /* (int)angstepf * a: the reference truncates the stride before multiplying (cpu_tracker.cpp:655-657). */
    int stride = (int)((double)angular_pq / angsteps);
    for (int i = 0; i < nr; i++) {
        double sum = 0, r = minR + rstep * i;
        int n = 0;
        for (int a = 0; a < angsteps; a++) {
            int j = stride * a;
            double ang = 0.5 * REF_PI_F * (j + 0.5) / angular_pq;
            double x = cx + mx * cos(ang) * r, y = cy + my * sin(ang) * r;
            int out;
            double v = bilinear(img, w, h, x, y, &out);
            if (!out) {
                sum += v;
                n++;
            }
        }
        dst[i] = n >= MIN_RADPROFILE_SMP_COUNT ? sum / n : mean;
        if (rweights) dst[i] *= rweights[i];
    }
}

/* CPUTracker::QI_ComputeOffset, cpu_tracker.cpp:375-406: autoconvolution of the profile with
 * its reverse (unnormalised inverse FFT, so values carry the factor L), fftshift by nr,
 * 7-point weighted quadratic fit, (max - nr) * pi/4. */
static double qi_offset(const double *prof, int nr)
{
    int L = 2 * nr;
    double *ac = (double *)malloc(sizeof(double) * L);
    for (int x = 0; x < L; x++) {
        int n = (x + nr) % L;
        double s = 0;
        for (int m = 0; m < L; m++) s += prof[(n + m) % L] * prof[L - 1 - m];
        ac[x] = L * s;
    }
    double maxPos = oracle_max_interp7(ac, L, QI_WEIGHTS);
    free(ac);
    return (maxPos - nr) * (3.14159265359 / 4);
}

/* CPUTracker::ComputeQI, cpu_tracker.cpp:285-360. out = {x, y, boundaryHit}. */
ORACLE_API void oracle_qi(const double *img, int w, int h, double mean, double init_x, double init_y, int iterations,
                          int nr, int angular_pq, double angstep_factor, double minR, double maxR,
                          const double *rweights, double *out)
{
    double *q = (double *)malloc(sizeof(double) * nr * 4);
    double *prof = (double *)malloc(sizeof(double) * nr * 2);
    double cx = init_x, cy = init_y;
    double pixelsPerProfLen = (maxR - minR) / nr;
    int bhit = 0;
    /* the reference keeps angsteps as a float (cpu_tracker.cpp:314) and truncates it per call */
    float angsteps = angular_pq / powf((float)angstep_factor, (float)iterations);
    for (int k = 0; k < iterations; k++) {
        bhit = check_boundaries(cx, cy, maxR, w, h);
        for (int qu = 0; qu < 4; qu++)
            quadrant_profile(img, w, h, mean, q + qu * nr, nr, angular_pq, (int)angsteps, qu, minR, maxR, cx, cy,
                             rweights);
        double *q0 = q, *q1 = q + nr, *q2 = q + 2 * nr, *q3 = q + 3 * nr;
        for (int r = 0; r < nr; r++) {
            prof[nr - r - 1] = q1[r] + q2[r];
            prof[nr + r] = q0[r] + q3[r];
        }
        double offX = qi_offset(prof, nr);
        for (int r = 0; r < nr; r++) {
            prof[nr + r] = q0[r] + q1[r];
            prof[nr - r - 1] = q2[r] + q3[r];
        }
        double offY = qi_offset(prof, nr);
        cx += offX * pixelsPerProfLen;
        cy += offY * pixelsPerProfLen;
        angsteps *= (float)angstep_factor;
    }
    out[0] = cx;
    out[1] = cy;
    out[2] = bhit;
    free(q);
    free(prof);
}

/* NormalizeRadialProfile, utils.cpp:230-261. */
ORACLE_API void oracle_normalize_profile(double *prof, int n)
{
    double sum = 0;
    for (int i = 0; i < n; i++) sum += prof[i];
    double mean = sum / n, rms2 = 0;
    for (int i = 0; i < n; i++) {
        prof[i] -= mean;
        rms2 += prof[i] * prof[i];
    }
    double inv = 1.0 / sqrt(rms2 / n);
    for (int i = 0; i < n; i++) prof[i] *= inv;
}

/* ComputeRadialProfile, utils.cpp:275-320: full-circle directions 2*pi*j/angsteps, more than
 * MIN_RADPROFILE_SMP_COUNT in-bounds samples or the fallback value `mean`. */
ORACLE_API void oracle_radial_profile(const double *img, int w, int h, double mean, double cx, double cy, int nbins,
                                      int angsteps, double minR, double maxR, int normalize, double *dst)
{
    double rstep = (maxR - minR) / nbins;
    for (int i = 0; i < nbins; i++) {
        double sum = 0, r = minR + rstep * i;
        int n = 0;
        for (int a = 0; a < angsteps; a++) {
            double ang = 2 * REF_PI_F * a / angsteps;
            int out;
            double v = bilinear(img, w, h, cx + cos(ang) * r, cy + sin(ang) * r, &out);
            if (!out) {
                sum += v;
                n++;
            }
        }
        dst[i] = n > MIN_RADPROFILE_SMP_COUNT ? sum / n : mean;
    }
    if (normalize) oracle_normalize_profile(dst, nbins);
}

/* CPUTracker::LUTProfileCompare, cpu_tracker.cpp:791-868 (LUTProfMaxQuadraticFit):
 * score_k = -sum_r (w_r (p_r - L_kr))^2, then the 7-point fit over planes. */
ORACLE_API double oracle_lut_compare(const double *prof, const float *lut, int planes, int nbins,
                                     const double *weights, double *scores)
{
    double *s = scores ? scores : (double *)malloc(sizeof(double) * planes);
    for (int k = 0; k < planes; k++) {
        double acc = 0;
        for (int r = 0; r < nbins; r++) {
            double d = prof[r] - (double)lut[k * nbins + r];
            if (weights) d *= weights[r];
            acc -= d * d;
        }
        s[k] = acc;
    }
    double z = oracle_max_interp7(s, planes, ZLUT_WEIGHTS);
    if (!scores) free(s);
    return z;
}

/* erf<T>, utils.h:395-417: Abramowitz & Stegun 7.1.26, evaluated in double. */
ORACLE_API double oracle_erf_as(double x)
{
    const double a1 = 0.254829592, a2 = -0.284496736, a3 = 1.421413741, a4 = -1.453152027, a5 = 1.061405429,
                 p = 0.3275911;
    int sign = x < 0 ? -1 : 1;
    x = fabs(x);
    double t = 1.0 / (1.0 + p * x);
    double y = 1.0 - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * exp(-x * x);
    return sign * y;
}

/* CPUTracker::Compute2DGaussianMLE, cpu_tracker.cpp:514-589: 4 parameters (x, y, I0, bg),
 * fixed sigma, per-parameter (diagonal) Newton steps. out = {x, y, I0, bg}. */
ORACLE_API void oracle_gauss2d(const double *img, int w, int h, double mean, double init_x, double init_y,
                               int iterations, double sigma, double *out)
{
    double px = init_x, py = init_y, I0 = mean * 0.5 * w * h, bg = mean * 0.5;
    const double k1 = 1.0 / (sqrt(2.0) * sigma);
    const double k2 = 1.0 / (sqrt(2 * 3.14159265359) * sigma);
    const double k3 = 1.0 / (sqrt(2 * 3.14159265359) * sigma * sigma * sigma);
    for (int it = 0; it < iterations; it++) {
        double dx = 0, dy = 0, dI = 0, dB = 0, ddx = 0, ddy = 0, ddI = 0, ddB = 0;
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++) {
                double X0 = (x - px + .5) * k1, Y0 = (y - py + .5) * k1;
                double X1 = (x - px - .5) * k1, Y1 = (y - py - .5) * k1;
                double DX = 0.5 * oracle_erf_as(X0) - 0.5 * oracle_erf_as(X1);
                double DY = 0.5 * oracle_erf_as(Y0) - 0.5 * oracle_erf_as(Y1);
                double mu = bg + I0 * DX * DY;
                double dmx = I0 * k2 * (exp(-X1 * X1) - exp(-X0 * X0)) * DY;
                double dmy = I0 * k2 * (exp(-Y1 * Y1) - exp(-Y0 * Y0)) * DX;
                double dmI = DX * DY;
                double smp = img[y * w + x];
                double f = smp / mu - 1;
                dx += dmx * f;
                dy += dmy * f;
                dI += dmI * f;
                dB += f;
                double d2x = I0 * k3 * ((x - px - .5) * exp(-X1 * X1) - (x - px + .5) * exp(-X0 * X0)) * DY;
                double d2y = I0 * k3 * ((y - py - .5) * exp(-Y1 * Y1) - (y - py + .5) * exp(-Y0 * Y0)) * DX;
                ddx += d2x * f - dmx * dmx * smp / (mu * mu);
                ddy += d2y * f - dmy * dmy * smp / (mu * mu);
                ddI += -dmI * dmI * smp / (mu * mu);
                ddB += -smp / (mu * mu);
            }
        px -= dx / ddx;
        py -= dy / ddy;
        I0 -= dI / ddI;
        bg -= dB / ddB;
    }
    out[0] = px;
    out[1] = py;
    out[2] = I0;
    out[3] = bg;
}

/*
 * One ROI through QueuedCPUTracker::ProcessJob, QueuedCPUTracker.cpp:273-361, for the modes in
 * scope (COM, QI, Gaussian2D, LocalizeZ, NormalizeProfile, ClearFirstFourPixels).
 * img: W*H pixels already converted to double (SetImage, cpu_tracker.h:123-134), after the
 * per-bead offset/gain step. lut: this ROI's bead LUT [planes][zlut_radialsteps] or NULL.
 * out = {x, y, z, com_x, com_y, error, imageMean}.
 */
ORACLE_API void oracle_localize(const oracle_config *c, int mode, double *img, const float *lut, int planes,
                                const double *zweights, double *out)
{
    int w = c->width, h = c->height;
    if (mode & LT_ClearFirstFourPixels) img[0] = img[1] = img[2] = img[3] = 0;
    double com[4];
    oracle_com(img, w, h, c->com_bgcorrection, com);
    double mean = com[2];
    if (isnan(com[0]) || isnan(com[1])) {
        com[0] = w / 2;
        com[1] = h / 2;
    }
    double x = com[0], y = com[1], z = 0;
    int bhit = 0;
    if (mode & LT_QI) {
        double *rw = (double *)malloc(sizeof(double) * c->qi_radialsteps);
        oracle_radial_bin_window(c->qi_radialsteps, rw);
        double q[3];
        oracle_qi(img, w, h, mean, com[0], com[1], c->qi_iterations, c->qi_radialsteps, c->qi_angstepspq,
                  c->qi_angstep_factor, c->qi_minradius, c->qi_maxradius, rw, q);
        x = q[0];
        y = q[1];
        bhit = (int)q[2];
        free(rw);
    } else if (mode & LT_Gaussian2D) {
        double g[4];
        oracle_gauss2d(img, w, h, mean, com[0], com[1], c->gauss2D_iterations, c->gauss2D_sigma, g);
        x = g[0];
        y = g[1];
    }
    if (mode & LT_LocalizeZ) {
        int nb = c->zlut_radialsteps;
        double *prof = (double *)malloc(sizeof(double) * nb);
        bhit = check_boundaries(x, y, c->zlut_maxradius, w, h);
        oracle_radial_profile(img, w, h, mean, x, y, nb, c->zlut_angularsteps, c->zlut_minradius, c->zlut_maxradius,
                              (mode & LT_NormalizeProfile) != 0, prof);
        z = lut ? oracle_lut_compare(prof, lut, planes, nb, zweights, 0) : 0.0;
        free(prof);
    }
    out[0] = x;
    out[1] = y;
    out[2] = z;
    out[3] = com[0];
    out[4] = com[1];
    out[5] = bhit;
    out[6] = mean;
}

/*
 * One bead of QueuedCPUTracker::BuildLUT, QueuedCPUTracker.cpp:580-646: position from
 * known_pos, or COM (no background correction) + QI without radial weights (line 603);
 * the radial profile (normalised iff BUILDLUT_NORMALIZE) uses the tracker's mean as the
 * fallback, which is 0 when known_pos skips ComputeMeanAndCOM (SetImage resets it,
 * cpu_tracker.h:135). The profile is added to lut_row.
 */
ORACLE_API void oracle_build_lut_bead(const oracle_config *c, const double *img, int has_known, double kx, double ky,
                                      int normalize, double *lut_row)
{
    int w = c->width, h = c->height;
    double x = kx, y = ky, mean = 0;
    if (!has_known) {
        double com[4], q[3];
        oracle_com(img, w, h, 0.0, com);
        mean = com[2];
        oracle_qi(img, w, h, mean, com[0], com[1], c->qi_iterations, c->qi_radialsteps, c->qi_angstepspq,
                  c->qi_angstep_factor, c->qi_minradius, c->qi_maxradius, 0, q);
        x = q[0];
        y = q[1];
    }
    int nb = c->zlut_radialsteps;
    double *prof = (double *)malloc(sizeof(double) * nb);
    oracle_radial_profile(img, w, h, mean, x, y, nb, c->zlut_angularsteps, c->zlut_minradius, c->zlut_maxradius,
                          normalize, prof);
    for (int i = 0; i < nb; i++) lut_row[i] += prof[i];
    free(prof);
}

/* QueuedTracker::ZLUTBiasCorrection, QueuedTracker.cpp:115-140, with Interpolate1D of
 * utils.h:60-67 on the bead's row of table[count][tw]. */
ORACLE_API double oracle_zlut_bias_correct(double z, int planes, const float *table, int tw, int count, int bead)
{
    if (!table || bead < 0 || bead >= count) return z;
    const float *row = table + (size_t)bead * tw;
    double pos = z;
    for (int k = 0; k < 4; k++) {
        double tblpos = pos / planes * tw;
        int fx = (int)tblpos;
        double bias;
        if (fx < 0)
            bias = row[0];
        else if (fx >= tw - 1)
            bias = row[tw - 1];
        else
            bias = (row[fx + 1] - row[fx]) * (tblpos - fx) + row[fx];
        pos = z - bias;
    }
    return pos;
}

/* ======================= extensions (no reference counterpart) ======================= */

/* Integrated-Gaussian pixel model of utils.cpp:393-402 with exact erf; used by the
 * 5-parameter MLE below. */
static void gauss_pixel(double x, double y, double px, double py, double s, double *D, double *dDx, double *dDs,
                        int axis_is_y)
{
    (void)axis_is_y;
    (void)y;
    double a0 = (x - px + 0.5) / (sqrt(2.0) * s), a1 = (x - px - 0.5) / (sqrt(2.0) * s);
    *D = 0.5 * (erf(a0) - erf(a1));
    double g0 = exp(-a0 * a0), g1 = exp(-a1 * a1);
    /* d/dpx of D */
    *dDx = (g1 - g0) / (sqrt(2 * M_PI) * s);
    /* d/ds of D */
    *dDs = -((x - px + 0.5) * g0 - (x - px - 0.5) * g1) / (sqrt(2 * M_PI) * s * s);
}

/* Solve the 5x5 system A d = b by Gaussian elimination with partial pivoting; returns 0 if singular. */
static int solve5(double A[5][5], double b[5], double d[5])
{
    double M[5][6];
    for (int i = 0; i < 5; i++) {
        for (int j = 0; j < 5; j++) M[i][j] = A[i][j];
        M[i][5] = b[i];
    }
    for (int c = 0; c < 5; c++) {
        int p = c;
        for (int r = c + 1; r < 5; r++)
            if (fabs(M[r][c]) > fabs(M[p][c])) p = r;
        if (fabs(M[p][c]) < 1e-300) return 0;
        if (p != c)
            for (int j = 0; j < 6; j++) {
                double t = M[c][j];
                M[c][j] = M[p][j];
                M[p][j] = t;
            }
        for (int r = c + 1; r < 5; r++) {
            double f = M[r][c] / M[c][c];
            for (int j = c; j < 6; j++) M[r][j] -= f * M[c][j];
        }
    }
    for (int i = 4; i >= 0; i--) {
        double s = M[i][5];
        for (int j = i + 1; j < 5; j++) s -= M[i][j] * d[j];
        d[i] = s / M[i][i];
    }
    return 1;
}

/*
 * 5-parameter Poisson MLE of an integrated Gaussian spot (x, y, I0, bg, sigma) with full
 * Newton steps (Fisher-scoring Hessian, i.e. the expected Hessian sum_i (dmu/dp)(dmu/dq)/mu),
 * a 5x5 FP64 solve per step, and parameter clamping (I0, bg > 0; 0.3 < sigma < W/2).
 * init = {x, y, I0, bg, sigma}; out = same order; fisher (may be NULL) = 5x5 Fisher matrix at
 * the solution, whose inverse diagonal is the Cramer-Rao bound.
 */
ORACLE_API void oracle_gauss5(const double *img, int w, int h, const double *init, int iterations, double *out,
                              double *fisher)
{
    double p[5];
    for (int i = 0; i < 5; i++) p[i] = init[i];
    for (int it = 0; it <= iterations; it++) {
        double H[5][5] = {{0}}, g[5] = {0};
        for (int y = 0; y < h; y++) {
            double DY, dDy, dDsy;
            gauss_pixel(y, 0, p[1], 0, p[4], &DY, &dDy, &dDsy, 1);
            for (int x = 0; x < w; x++) {
                double DX, dDx, dDsx;
                gauss_pixel(x, 0, p[0], 0, p[4], &DX, &dDx, &dDsx, 0);
                double mu = p[3] + p[2] * DX * DY;
                double j[5] = {p[2] * dDx * DY, p[2] * DX * dDy, DX * DY, 1.0, p[2] * (dDsx * DY + DX * dDsy)};
                double f = img[y * w + x] / mu - 1.0;
                for (int a = 0; a < 5; a++) {
                    g[a] += j[a] * f;
                    for (int b = 0; b < 5; b++) H[a][b] += j[a] * j[b] / mu;
                }
            }
        }
        if (it == iterations) {
            if (fisher)
                for (int a = 0; a < 5; a++)
                    for (int b = 0; b < 5; b++) fisher[a * 5 + b] = H[a][b];
            break;
        }
        double d[5];
        if (!solve5(H, g, d)) break;
        for (int a = 0; a < 5; a++) p[a] += d[a];
        if (p[2] < 1e-3) p[2] = 1e-3;
        if (p[3] < 1e-3) p[3] = 1e-3;
        if (p[4] < 0.3) p[4] = 0.3;
        if (p[4] > w * 0.5) p[4] = w * 0.5;
    }
    for (int i = 0; i < 5; i++) out[i] = p[i];
}

/*
 * Poisson negative log-likelihood of the integrated-Gaussian spot model of the 5-parameter MLE,
 *   NLL(p) = sum_pixels mu - I ln mu,   mu = bg + I0 DX(x, sigma) DY(y, sigma),
 * (the ln I! term dropped) with p = {x, y, I0, bg, sigma}, and its gradient
 *   dNLL/dp = sum (1 - I / mu) dmu/dp.  Returns NLL; grad receives the 5 derivatives.
 */
ORACLE_API double oracle_gauss_nll_grad(const double *img, int w, int h, const double *p, double *grad)
{
    double nll = 0, g[5] = {0, 0, 0, 0, 0};
    for (int y = 0; y < h; y++) {
        double DY, dDy, dDsy;
        gauss_pixel(y, 0, p[1], 0, p[4], &DY, &dDy, &dDsy, 1);
        for (int x = 0; x < w; x++) {
            double DX, dDx, dDsx;
            gauss_pixel(x, 0, p[0], 0, p[4], &DX, &dDx, &dDsx, 0);
            double mu = p[3] + p[2] * DX * DY;
            double j[5] = {p[2] * dDx * DY, p[2] * DX * dDy, DX * DY, 1.0, p[2] * (dDsx * DY + DX * dDsy)};
            double I = img[y * w + x];
            nll += mu - I * log(mu);
            for (int a = 0; a < 5; a++) g[a] += (1.0 - I / mu) * j[a];
        }
    }
    for (int a = 0; a < 5; a++) grad[a] = g[a];
    return nll;
}

/*
 * Radial-profile-to-LUT cost and its analytic gradient (the adjoint of the GPU library).
 * p(x, y) is the radial profile of utils.cpp:275-320 at (x, y): per bin the mean of the
 * in-bounds bilinear samples over `angsteps` directions, or `mean` when at most 4 samples are
 * in bounds; with `normalize` it is NormalizeRadialProfile'd (utils.cpp:230-261: minus its
 * mean, divided by its RMS), as the Z match uses it. Lz is the LUT linearly interpolated
 * between planes iz = clamp(floor(z), 0, planes-2) and iz+1. With radial weights w,
 *   cost(x, y, z, L) = sum_r (w_r (p_r(x, y) - Lz_r))^2.
 * d p_r / dx is the mean of the samples' bilinear x-derivatives ((v10-v00)(1-fy) + (v11-v01)fy),
 * and likewise for y; through the normalisation,
 *   d phat_r = (dp_r - mean(dp) - phat_r * sum_j(phat_j dp_j) / n) / rms.
 */
static void zprofile_grad(const double *img, int w, int h, double mean, double x, double y, int nbins,
                          int angsteps, double minR, double maxR, int normalize, double *p, double *dpx,
                          double *dpy)
{
    double rstep = (maxR - minR) / nbins;
    for (int i = 0; i < nbins; i++) {
        double r = minR + rstep * i, sum = 0, sx = 0, sy = 0;
        int n = 0;
        for (int a = 0; a < angsteps; a++) {
            double ang = 2 * REF_PI_F * a / angsteps;
            double px = x + cos(ang) * r, py = y + sin(ang) * r;
            int rx = (int)px, ry = (int)py;
            if (rx < 0 || ry < 0 || rx + 1 >= w || ry + 1 >= h) continue;
            double v00 = img[w * ry + rx], v10 = img[w * ry + rx + 1];
            double v01 = img[w * (ry + 1) + rx], v11 = img[w * (ry + 1) + rx + 1];
            double fx = px - rx, fy = py - ry;
            double v0 = v00 + (v10 - v00) * fx, v1 = v01 + (v11 - v01) * fx;
            sum += v0 + (v1 - v0) * fy;
            sx += (v10 - v00) * (1 - fy) + (v11 - v01) * fy;
            sy += v1 - v0;
            n++;
        }
        if (n > MIN_RADPROFILE_SMP_COUNT) {
            p[i] = sum / n;
            dpx[i] = sx / n;
            dpy[i] = sy / n;
        } else {
            p[i] = mean;
            dpx[i] = dpy[i] = 0;
        }
    }
    if (!normalize) return;
    double m = 0, mx = 0, my = 0;
    for (int i = 0; i < nbins; i++) {
        m += p[i];
        mx += dpx[i];
        my += dpy[i];
    }
    m /= nbins;
    mx /= nbins;
    my /= nbins;
    double ss = 0;
    for (int i = 0; i < nbins; i++) ss += (p[i] - m) * (p[i] - m);
    double rms = sqrt(ss / nbins), kx = 0, ky = 0;
    for (int i = 0; i < nbins; i++) {
        p[i] = (p[i] - m) / rms;
        kx += p[i] * dpx[i];
        ky += p[i] * dpy[i];
    }
    kx /= nbins;
    ky /= nbins;
    for (int i = 0; i < nbins; i++) {
        dpx[i] = (dpx[i] - mx - p[i] * kx) / rms;
        dpy[i] = (dpy[i] - my - p[i] * ky) / rms;
    }
}

/* grad = {dcost/dx, dcost/dy, dcost/dz}; glut (planes*nbins, may be NULL) = dcost/dL. */
ORACLE_API double oracle_zcost_grad(const double *img, int w, int h, double mean, double x, double y, double z,
                                    const float *lut, int planes, int nbins, int angsteps, double minR, double maxR,
                                    const double *weights, int normalize, double *grad, double *glut)
{
    double *p = (double *)malloc(sizeof(double) * 3 * nbins), *dpx = p + nbins, *dpy = p + 2 * nbins;
    zprofile_grad(img, w, h, mean, x, y, nbins, angsteps, minR, maxR, normalize, p, dpx, dpy);
    int iz = (int)floor(z);
    if (iz < 0) iz = 0;
    if (iz > planes - 2) iz = planes - 2;
    double fz = z - iz;
    double cost = 0, gx = 0, gy = 0, gz = 0;
    if (glut) memset(glut, 0, sizeof(double) * planes * nbins);
    for (int i = 0; i < nbins; i++) {
        double l0 = lut[iz * nbins + i], l1 = lut[(iz + 1) * nbins + i];
        double wr = weights ? weights[i] : 1.0;
        double e = p[i] - (l0 + (l1 - l0) * fz);
        cost += wr * wr * e * e;
        double de = 2 * wr * wr * e;
        gx += de * dpx[i];
        gy += de * dpy[i];
        gz += -de * (l1 - l0);
        if (glut) {
            glut[iz * nbins + i] += -de * (1 - fz);
            glut[(iz + 1) * nbins + i] += -de * fz;
        }
    }
    free(p);
    grad[0] = gx;
    grad[1] = gy;
    grad[2] = gz;
    return cost;
}

/* Stiffness of the joint refinement's (x, y) prior in units of the cost's curvature along z
 * (100, as the GPU path uses); settable so that tests can sweep it. */
static double g_joint_prior_scale = 100.0;

ORACLE_API void oracle_set_joint_prior_scale(double scale) { g_joint_prior_scale = scale; }

/*
 * Joint Gauss-Newton refinement of (x, y, z) on the cost above plus a quadratic prior that ties
 * (x, y) to their starting point (the QI estimate):
 *   E = cost(x, y, z) + k ((x - x0)^2 + (y - y0)^2),  k = 100 sum_r w_r^2 (L_iz+1,r - L_iz,r)^2,
 * 100 times the curvature of the cost along z at the starting plane (the factor is
 * g_joint_prior_scale, 100 unless a test sets it). The prior is needed because
 * a radial profile is, to first order, insensitive to where its centre is (the x-derivative of a
 * radially symmetric image averages to zero over a circle), so the cost alone leaves x and y
 * undetermined and its noise-driven minimum lies ~0.1 px from the truth where QI is ~0.02 px
 * off; at this stiffness x and y keep QI's precision and z follows the LUT interpolation. Per step: residuals w_r (phat_r - Lz_r), Jacobian w_r (dphat_r/dx, dphat_r/dy,
 * -(L_iz+1,r - L_iz,r)), normal equations (J^T J + diag(k, k, 0)) d = -(J^T res + k (x-x0, y-y0, 0))
 * with a Levenberg term 1e-9 * trace (+1e-30) on the diagonal, solved by Cramer's rule. The step
 * is taken if it lowers E, else halved up to 4 times; if none does, the refinement stops. z is
 * clamped to [0, planes-1]. io = {x, y, z} in, refined out.
 */
static double zcost_at(const double *img, int w, int h, double mean, double x, double y, double z, const float *lut,
                       int planes, int nbins, int angsteps, double minR, double maxR, const double *weights,
                       int normalize, double *p, double *dpx, double *dpy)
{
    zprofile_grad(img, w, h, mean, x, y, nbins, angsteps, minR, maxR, normalize, p, dpx, dpy);
    int iz = (int)floor(z);
    if (iz < 0) iz = 0;
    if (iz > planes - 2) iz = planes - 2;
    double fz = z - iz, cost = 0;
    for (int i = 0; i < nbins; i++) {
        double l0 = lut[iz * nbins + i], l1 = lut[(iz + 1) * nbins + i];
        double wr = weights ? weights[i] : 1.0;
        double e = p[i] - (l0 + (l1 - l0) * fz);
        cost += wr * wr * e * e;
    }
    return cost;
}

ORACLE_API void oracle_joint_refine(const double *img, int w, int h, double mean, double *io, const float *lut,
                                    int planes, int nbins, int angsteps, double minR, double maxR,
                                    const double *weights, int normalize, int steps)
{
    double *p = (double *)malloc(sizeof(double) * 3 * nbins), *dpx = p + nbins, *dpy = p + 2 * nbins;
    const double x0 = io[0], y0 = io[1];
    double k = 0; /* prior stiffness, set from the plane of the current z */
    double cur = 0;
    for (int s = 0; s < steps; s++) {
        double x = io[0], y = io[1], z = io[2];
        zprofile_grad(img, w, h, mean, x, y, nbins, angsteps, minR, maxR, normalize, p, dpx, dpy);
        int iz = (int)floor(z);
        if (iz < 0) iz = 0;
        if (iz > planes - 2) iz = planes - 2;
        double fz = z - iz;
        double A[3][3] = {{0}}, g[3] = {0}, cost = 0;
        for (int i = 0; i < nbins; i++) {
            double l0 = lut[iz * nbins + i], l1 = lut[(iz + 1) * nbins + i];
            double wr = weights ? weights[i] : 1.0;
            double J[3] = {dpx[i], dpy[i], -(l1 - l0)};
            double e = p[i] - (l0 + (l1 - l0) * fz);
            cost += wr * wr * e * e;
            for (int a = 0; a < 3; a++) {
                g[a] += wr * wr * J[a] * e;
                for (int b = 0; b < 3; b++) A[a][b] += wr * wr * J[a] * J[b];
            }
        }
        if (s == 0) k = g_joint_prior_scale * A[2][2];
        cur = cost + k * ((x - x0) * (x - x0) + (y - y0) * (y - y0));
        A[0][0] += k;
        A[1][1] += k;
        g[0] += k * (x - x0);
        g[1] += k * (y - y0);
        double tr = A[0][0] + A[1][1] + A[2][2];
        for (int a = 0; a < 3; a++) A[a][a] += 1e-9 * tr + 1e-30;
        double det = A[0][0] * (A[1][1] * A[2][2] - A[1][2] * A[2][1]) -
                     A[0][1] * (A[1][0] * A[2][2] - A[1][2] * A[2][0]) +
                     A[0][2] * (A[1][0] * A[2][1] - A[1][1] * A[2][0]);
        if (det == 0) break;
        double d[3];
        for (int c = 0; c < 3; c++) {
            double M[3][3];
            for (int i = 0; i < 3; i++)
                for (int j = 0; j < 3; j++) M[i][j] = (j == c) ? -g[i] : A[i][j];
            d[c] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                    M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) /
                   det;
        }
        int taken = 0;
        for (int hv = 0; hv < 5 && !taken; hv++) {
            double t = ldexp(1.0, -hv), nz = z + t * d[2], nx = x + t * d[0], ny = y + t * d[1];
            if (nz < 0) nz = 0;
            if (nz > planes - 1) nz = planes - 1;
            double c = zcost_at(img, w, h, mean, nx, ny, nz, lut, planes, nbins, angsteps, minR, maxR, weights,
                                normalize, p, dpx, dpy) +
                       k * ((nx - x0) * (nx - x0) + (ny - y0) * (ny - y0));
            if (c < cur) {
                io[0] = x + t * d[0];
                io[1] = y + t * d[1];
                io[2] = nz;
                cur = c;
                taken = 1;
            }
        }
        if (!taken) break;
    }
    free(p);
}

/*
 * Bead finder, BeadFinder.cpp:170-222 (Find) with SearchArea (:79-105) and RecenterAndFilter
 * (:108-166), as QTrkFindBeads (qtrk_c_api.cpp:33-58) calls it. The FFT convolution of the
 * reference (image minus its mean, zero-padded to powers of two, times the FFT of the
 * mean-free sample placed at offset -roi, inverse FFT) is the circular convolution
 *   conv(py,px) = sum_{a,b<roi} t(a,b) c((py+roi-a) mod H2, (px+roi-b) mod W2),
 * evaluated here directly in double (the inverse FFT's missing 1/(W2 H2) does not change any
 * decision: every test on the map is relative to its maximum). Means, the recentering sums
 * and the distance tests follow the reference's float arithmetic and int truncations.
 * Returns the number of positions (at most max_out written to out_xy as x,y pairs);
 * conv_out (W2*H2 doubles, may be NULL) receives the map before the search zeroes it.
 */
static int bf_next_pow2(int x)
{
    int y = 1;
    while (y < x) y *= 2;
    return y;
}

ORACLE_API int oracle_find_beads(const float *img, int w, int h, int sx, int sy, int roi, float rel_dist,
                                 float similarity, int *out_xy, int max_out, double *conv_out)
{
    int W2 = bf_next_pow2(w), H2 = bf_next_pow2(h);
    float mean = 0.0f, smean = 0.0f;
    for (int i = 0; i < w * h; i++) mean += img[i];
    mean /= (float)(w * h);
    float *t = (float *)malloc(sizeof(float) * roi * roi);
    for (int y = 0; y < roi; y++)
        for (int x = 0; x < roi; x++) t[y * roi + x] = img[(sy + y) * w + sx + x];
    for (int i = 0; i < roi * roi; i++) smean += t[i];
    smean /= (float)(roi * roi);
    for (int i = 0; i < roi * roi; i++) t[i] = t[i] - smean;
    double *conv = (double *)malloc(sizeof(double) * W2 * H2);
    for (int py = 0; py < H2; py++)
        for (int px = 0; px < W2; px++) {
            double acc = 0;
            for (int a = 0; a < roi; a++) {
                int yy = (py + roi - a) & (H2 - 1);
                if (yy >= h) continue;
                for (int b = 0; b < roi; b++) {
                    int xx = (px + roi - b) & (W2 - 1);
                    if (xx >= w) continue;
                    acc += (double)t[a * roi + b] * (double)(img[yy * w + xx] - mean);
                }
            }
            conv[py * W2 + px] = acc;
        }
    if (conv_out) memcpy(conv_out, conv, sizeof(double) * W2 * H2);
    double maxv = 0;
    for (int i = 0; i < W2 * H2; i++)
        if (conv[i] > maxv) maxv = conv[i];
    const float mdist = 0.5f * rel_dist * roi;
    const int dist = (int)mdist;
    int npts = 0, cap = 64;
    int *pts = (int *)malloc(sizeof(int) * 2 * cap);
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            if (!(conv[y * W2 + x] > maxv * similarity)) continue;
            /* SearchArea: the maximum inside the disc of radius dist (clipped to the padded map);
               every visited value is zeroed */
            int bx = x, by = y;
            double best = conv[y * W2 + x];
            int y0 = y - dist < 0 ? 0 : y - dist, x0 = x - dist < 0 ? 0 : x - dist;
            int x1 = x + dist > W2 - 1 ? W2 - 1 : x + dist, y1 = y + dist > H2 - 1 ? H2 - 1 : y + dist;
            for (int yy = y0; yy <= y1; yy++)
                for (int xx = x0; xx <= x1; xx++) {
                    int dx = xx - x, dy = yy - y;
                    if (dx * dx + dy * dy > dist * dist) continue;
                    if (conv[yy * W2 + xx] > best) {
                        best = conv[yy * W2 + xx];
                        bx = xx;
                        by = yy;
                    }
                    conv[yy * W2 + xx] = 0;
                }
            if (npts == cap) {
                cap *= 2;
                pts = (int *)realloc(pts, sizeof(int) * 2 * cap);
            }
            pts[2 * npts] = bx;
            pts[2 * npts + 1] = by;
            npts++;
        }
    /* RecenterAndFilter: COM of the squared deviation from the ROI mean (float sums), shift by
       it minus roi/2 (int truncation), bounds checks, and both of two positions closer than
       mdist are dropped (the earlier one from the list, the later one never added). */
    int *acc_xy = (int *)malloc(sizeof(int) * 2 * (npts + 1));
    int nacc = 0;
    for (int i = 0; i < npts; i++) {
        int px = pts[2 * i], py = pts[2 * i + 1];
        if (px < 0 || py < 0 || px > w - 1 - roi || py > h - 1 - roi) continue;
        float sum = 0.0f;
        for (int y = 0; y < roi; y++)
            for (int x = 0; x < roi; x++) sum += img[(y + py) * w + x + px];
        float m = sum / (roi * roi), sumx = 0, sumy = 0;
        sum = 0;
        for (int y = 0; y < roi; y++)
            for (int x = 0; x < roi; x++) {
                float v = img[(y + py) * w + x + px] - m;
                v = v * v;
                sum += v;
                sumx += v * x;
                sumy += v * y;
            }
        if (sum == 0.0f) continue;
        px = (int)((float)px + (sumx / sum - roi / 2));
        py = (int)((float)py + (sumy / sum - roi / 2));
        if (px < 0 || py < 0 || px > w - 1 - roi || py > h - 1 - roi) continue;
        int accepted = 1;
        for (int c = 0; c < nacc; c++) {
            int dx = acc_xy[2 * c] - px, dy = acc_xy[2 * c + 1] - py;
            if ((float)(dx * dx + dy * dy) < mdist * mdist) {
                memmove(&acc_xy[2 * c], &acc_xy[2 * c + 2], sizeof(int) * 2 * (nacc - c - 1));
                nacc--;
                accepted = 0;
                break;
            }
        }
        if (accepted) {
            acc_xy[2 * nacc] = px;
            acc_xy[2 * nacc + 1] = py;
            nacc++;
        }
    }
    for (int i = 0; i < nacc && i < max_out; i++) {
        out_xy[2 * i] = acc_xy[2 * i];
        out_xy[2 * i + 1] = acc_xy[2 * i + 1];
    }
    free(acc_xy);
    free(pts);
    free(conv);
    free(t);
    return nacc;
}
