// Parameters shared between the host tracker and the sm_100a kernels.
//
// One TrackParams value describes everything a localization launch needs: ROI geometry,
// mode bits, the derived step counts of QTrkComputedConfig::Update
// (cputrack/QueuedTracker.cpp:6-21) and device pointers to the read-only tables the
// host precomputes once per configuration (direction tables, radial weights, FFT
// twiddles, the Z-LUT). It is passed by value as a kernel parameter.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#include <cuda_runtime.h>
#else
struct float2_host { float x, y; };
#endif

namespace qtrk {

constexpr int kMaxQIIterations = 32;
// Threads per localization CTA (one ROI per CTA). Four warps: with a 100x100 float tile (45 KB of
// shared memory) five CTAs fit on an SM, and the one-warp sections of each ROI (QI transform and
// fits, Z fit) leave three warps idle rather than seven.
constexpr int kBlockThreads = 128;

// Mode bits (cputrack/qtrk_c_api.h:5-20 plus the library's extension bits).
enum : int {
    kLT_QI = 2,
    kLT_Gaussian2D = 4,
    kLT_LocalizeZ = 16,
    kLT_NormalizeProfile = 64,
    kLT_ClearFirstFourPixels = 128,
    kLT_ZMatchBF16 = 1 << 20,
    kLT_JointRefine = 1 << 21,
    kLT_Gaussian5P = 1 << 22,
    kLT_ZMatchTF32 = 1 << 23,
};

struct TrackParams {
    int width, height;  // ROI size in pixels
    int pdt;            // 0 = u8, 1 = u16, 2 = f32
    int mode;           // LocalizeModeEnum bits
    float com_bgcorrection;

    // QI (cputrack/cpu_tracker.cpp:285-406)
    int qi_iterations, qi_nr, qi_angpq;
    float qi_minr, qi_maxr;
    int qi_nang[kMaxQIIterations];    // angular samples per quadrant in iteration k (>= 4)
    int qi_stride[kMaxQIIterations];  // direction-table stride in iteration k (cpu_tracker.cpp:655-657)
    float qi_inv_nang[kMaxQIIterations];  // 1 / qi_nang[k] (bins whose samples are all in bounds)
    const void *qi_dirs;              // float2[qi_angpq]: quadrant directions (cos, sin)
    const float *qi_rweights;         // float[qi_nr] radial bin window or nullptr
    const void *qi_twiddles;          // float2[L/2], e^{-2 pi i k / L}, L = 2 qi_nr

    // Radial profile + Z-LUT (cputrack/utils.cpp:275-320, cputrack/cpu_tracker.cpp:791-868)
    int z_nbins, z_angsteps;
    float z_minr, z_maxr;
    const void *z_dirs;       // float2[z_angsteps]
    const float *lut;         // [lut_count][lut_planes][z_nbins]
    int lut_count, lut_planes;
    // The same LUT transposed, [lut_count][z_nbins][lut_t_pitch] (planes padded to a multiple of
    // 32 with zeros), for the plain match's one-thread-per-plane scoring; nullptr while stale
    const float *lut_t;
    int lut_t_pitch;
    const float *z_weights;   // float[z_nbins] or nullptr
    float *cmp_scores;        // [lut_count][lut_planes] or nullptr (compare-profile output)
    // Tensor-core match: when zprof_f32 is set the localization kernel writes each ROI's
    // normalised profile (FP32) and its weighted BF16 copy (zprof_nbp bins, zero padded)
    // instead of scoring it; the Z-match kernel then fills in z.
    float *zprof_f32;
    void *zprof_bf16;
    int zprof_nbp;

    // Z-LUT bias table (QueuedTracker::ZLUTBiasCorrection, cputrack/QueuedTracker.cpp:115-140):
    // [zbias_count][zbias_w] or nullptr
    const float *zbias;
    int zbias_w, zbias_count;

    // 2D Gaussian MLE (cputrack/cpu_tracker.cpp:514-589)
    int g_iterations;
    float g_sigma;

    // Per-bead pixel calibration (cputrack/cpu_tracker.cpp:98-112); nullptr when unset
    const float *calib_offset, *calib_gain;  // [calib_count][height][width]
    int calib_count;
    float offset_factor, gain_factor;

    // Dynamic shared-memory layout (byte offsets), filled by the host
    int sm_img, sm_tables, sm_work, sm_red, sm_misc, smem_bytes;
    unsigned *err_flag;  // mapped host word: |= 4 when a staged ROI copy did not arrive in time (QI kernel)
};

}  // namespace qtrk
