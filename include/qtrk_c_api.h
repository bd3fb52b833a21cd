/*
 * qtrk_c_api.h — C ABI of libqtrk_b200.so, a drop-in for QTrk's tracker DLL.
 *
 * Every entry point below has the name, argument list, argument meaning and packed
 * struct layout of the reference declaration it replaces (cputrack/qtrk_c_api.h and
 * cputrack/utils.h of jcnossen/qtrk), so the .NET P/Invoke mirror
 * (QTrkDotNet/QTrkDLL.cs:244-405) and ctypes/cgo-style callers bind unchanged.
 * The localization work behind them runs on one NVIDIA B200 (sm_100a) in hand-written
 * CUDA kernels; the library has no CPU fallback: when no usable GPU is present
 * QTrkCreateInstance returns NULL and QTrkGetLastError() says why.
 *
 * Differences in behaviour from the reference, all additive:
 *  - no C++ exception crosses this ABI (the reference lets them escape,
 *    cputrack/qtrk_c_api.cpp:62-175); errors are logged per instance and returned by
 *    QTrkGetWarnings, or by QTrkGetLastError for calls without an instance;
 *  - results come back in FIFO order, like the reference CUDA tracker
 *    (cudatrack/QueuedCUDATracker.cu:726-737);
 *  - the declared-but-never-defined reference entry points
 *    (QTrkSetPixelCalibrationImages, QTrkSetPixelCalibrationFactors,
 *    QTrkEnableRadialZLUTCompareProfile, QTrkGetRadialZLUTCompareProfile,
 *    QTrkBuildLUTFromFrame) are implemented;
 *  - QTrkB200* entry points at the end extend the ABI (device-resident batches,
 *    tensor-core Z match, adjoint gradients, serving statistics).
 */
#ifndef QTRK_B200_C_API_H
#define QTRK_B200_C_API_H

#include <stdint.h>
#include <stddef.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#if defined(_WIN32)
#define QTRK_CALLCONV __cdecl
#define QTRK_EXPORT __declspec(dllexport)
#else
#define QTRK_CALLCONV
#define QTRK_EXPORT __attribute__((visibility("default")))
#endif

#ifdef __cplusplus
#define QTRK_API extern "C" QTRK_EXPORT
#else
#define QTRK_API QTRK_EXPORT
#endif

/* Localization mode bit flags; values of cputrack/qtrk_c_api.h:5-20. */
enum LocalizeModeEnum {
    LT_OnlyCOM = 0,
    LT_XCor1D = 1,
    LT_QI = 2,
    LT_Gaussian2D = 4,
    LT_ZLUTAlign = 8,
    LT_LocalizeZ = 16,
    LT_NormalizeProfile = 64,
    LT_ClearFirstFourPixels = 128,
    LT_FourierLUT = 256,
    LT_LocalizeZWeighted = 512,
    /* Extension bits (no reference counterpart). */
    LT_B200_ZMatchBF16 = 1 << 20,    /* Z cross term on the tensor cores (BF16, FP32 accumulate) */
    LT_B200_JointRefine = 1 << 21,   /* joint Gauss-Newton (x,y,z) refinement after the Z fit */
    LT_B200_Gaussian5P = 1 << 22,    /* 5-parameter (x,y,I0,bg,sigma) full-Newton Gaussian MLE */
    LT_B200_ZMatchTF32 = 1 << 23,    /* Z cross term on the tensor cores with TF32 operands (FP32 accumulate) */
    LT_Force32Bit = (int)0xffffffff
};
typedef int LocMode_t;

/* cputrack/qtrk_c_api.h:24-29 */
enum QTRK_PixelDataType { QTrkU8 = 0, QTrkU16 = 1, QTrkFloat = 2 };
typedef int QTRK_PixelDataType_t;

#pragma pack(push, 4)
/* cputrack/std_incl.h:20-116 (pack(4)) */
typedef struct vector2f { float x, y; } vector2f;
typedef struct vector3f { float x, y, z; } vector3f;
/* TImageData<float>, cputrack/utils.h:77-138 (pack(4)): data, w, h */
typedef struct ImageData { float *data; int w, h; } ImageData;
#pragma pack(pop)

#pragma pack(push, 1)
/* 24 bytes; cputrack/qtrk_c_api.h:34-45 */
typedef struct LocalizationJob {
    uint32_t frame, timestamp;
    int32_t zlutIndex;
    vector3f initialPos;
} LocalizationJob;

/* 52 bytes; cputrack/qtrk_c_api.h:49-57 */
typedef struct LocalizationResult {
    LocalizationJob job;
    vector3f pos;
    vector2f firstGuess;
    uint32_t error;
    float imageMean;
} LocalizationResult;

/* 84 bytes; cputrack/qtrk_c_api.h:59-114 (field order is the ABI) */
typedef struct QTrkSettings {
    int width, height;
    int numThreads;
    int cuda_device;
    float com_bgcorrection;
    float zlut_minradius;
    float zlut_radial_coverage;
    float zlut_angular_coverage;
    float zlut_roi_coverage;
    int qi_iterations;
    float qi_minradius;
    float qi_radial_coverage;
    float qi_angular_coverage;
    float qi_roi_coverage;
    float qi_angstep_factor;
    int xc1_profileLength;
    int xc1_profileWidth;
    int xc1_iterations;
    int gauss2D_iterations;
    float gauss2D_sigma;
    int downsample;
} QTrkSettings;

/* 108 bytes; cputrack/qtrk_c_api.h:123-138 */
typedef struct QTrkComputedConfig {
    QTrkSettings base;
    int zlut_radialsteps;
    int zlut_angularsteps;
    float zlut_maxradius;
    int qi_radialsteps;
    int qi_angstepspq;
    float qi_maxradius;
} QTrkComputedConfig;

/* 8 bytes; cputrack/qtrk_c_api.h:116-119 */
typedef struct ROIPosition { int x, y; } ROIPosition;

/* 41 bytes; cputrack/qtrk_c_api.h:211-219. Output position = (pos - ROI centre + offset) * scaling. */
typedef struct ResultManagerConfig {
    int numBeads, numFrameInfoColumns;
    vector3f scaling;
    vector3f offset;
    int writeInterval;          /* frames between file writes */
    uint32_t maxFramesInMemory; /* 0: unlimited */
    uint8_t binaryOutput;
} ResultManagerConfig;

/* 28 bytes; cputrack/qtrk_c_api.h:220-229 */
typedef struct RMFrameCounters {
    int startFrame;        /* first frame still held in memory */
    int processedFrames;   /* frames whose results are complete (or given up as lost) */
    int lastSaveFrame;
    int capturedFrames;    /* frames with frame info stored */
    int localizationsDone;
    int lostFrames;
    int fileError;
} RMFrameCounters;
#pragma pack(pop)

#define QTrkCUDA_UseList -3
#define QTrkCUDA_UseAll -2
#define QTrkCUDA_UseBest -1

/* cputrack/QueuedTracker.h:305-308 */
#define BUILDLUT_IMAGELUT 1
#define BUILDLUT_FOURIER 2
#define BUILDLUT_NORMALIZE 4
#define BUILDLUT_BIASCORRECT 8

#ifdef __cplusplus
struct QueuedTracker;
#else
typedef struct QueuedTracker QueuedTracker;
#endif

/* ---- configuration (cputrack/qtrk_c_api.cpp:12-25) ---- */
QTRK_API void QTRK_CALLCONV TestDLLCallConv(int a);                                   /* qtrk_c_api.cpp:12 */
QTRK_API void QTRK_CALLCONV QTrkGetDefaultConfig(QTrkSettings *cfg);                  /* qtrk_c_api.cpp:17 */
QTRK_API void QTRK_CALLCONV QTrkGetComputedConfig(QTrkSettings *base, QTrkComputedConfig *cfg); /* qtrk_c_api.cpp:22 */

/* ---- instance lifecycle (cputrack/qtrk_c_api.h:144-148) ---- */
QTRK_API struct QueuedTracker *QTRK_CALLCONV QTrkCreateInstance(QTrkSettings *cfg);   /* qtrk_c_api.h:144 */
QTRK_API void QTRK_CALLCONV QTrkFreeInstance(struct QueuedTracker *qtrk);             /* qtrk_c_api.h:145 */
QTRK_API void QTRK_CALLCONV QTrkSetLocalizationMode(struct QueuedTracker *qtrk, LocMode_t locType); /* qtrk_c_api.h:148 */

/* ---- pixel calibration (declared, never defined, in cputrack/qtrk_c_api.h:152-153) ---- */
QTRK_API void QTRK_CALLCONV QTrkSetPixelCalibrationImages(struct QueuedTracker *qtrk, float *offset, float *gain);
/* No instance argument in the reference declaration: sets the factors of every live instance
 * and the default of instances created later. */
QTRK_API void QTRK_CALLCONV QTrkSetPixelCalibrationFactors(float offsetFactor, float gainFactor);

/* ---- scheduling (cputrack/qtrk_c_api.h:158-163) ---- */
QTRK_API void QTRK_CALLCONV QTrkScheduleLocalization(struct QueuedTracker *qtrk, void *data, int pitch,
                                                     QTRK_PixelDataType_t pdt, const LocalizationJob *jobInfo);
QTRK_API void QTRK_CALLCONV QTrkClearResults(struct QueuedTracker *qtrk);             /* qtrk_c_api.h:159 */
QTRK_API void QTRK_CALLCONV QTrkFlush(struct QueuedTracker *qtrk);                    /* qtrk_c_api.h:160 */
QTRK_API int QTRK_CALLCONV QTrkScheduleFrame(struct QueuedTracker *qtrk, void *imgptr, int pitch, int width,
                                             int height, ROIPosition *positions, int numROI,
                                             QTRK_PixelDataType_t pdt, const LocalizationJob *jobInfo); /* qtrk_c_api.h:163 */

/* ---- Z-LUT (cputrack/qtrk_c_api.h:165-185) ---- */
/* No instance argument in the reference declarations (qtrk_c_api.h:165-166): they act on the
 * most recently created live instance. */
QTRK_API void QTRK_CALLCONV QTrkEnableRadialZLUTCompareProfile(bool enabled);
QTRK_API void QTRK_CALLCONV QTrkGetRadialZLUTCompareProfile(float *dst); /* dst = [count * planes] */
QTRK_API void QTRK_CALLCONV QTrkSetRadialZLUT(struct QueuedTracker *qtrk, float *data, int count, int planes); /* qtrk_c_api.h:169 */
QTRK_API void QTRK_CALLCONV QTrkGetRadialZLUT(struct QueuedTracker *qtrk, float *dst);                        /* qtrk_c_api.h:170 */
QTRK_API void QTRK_CALLCONV QTrkGetRadialZLUTSize(struct QueuedTracker *qtrk, int *count, int *planes, int *radialsteps); /* qtrk_c_api.h:171 */
QTRK_API void QTRK_CALLCONV QTrkSetRadialWeights(struct QueuedTracker *qtrk, float *zcmp);                    /* qtrk_c_api.h:174 */
QTRK_API void QTRK_CALLCONV QTrkBeginLUT(struct QueuedTracker *qtrk, unsigned int flags);                     /* qtrk_c_api.h:178 */
QTRK_API void QTRK_CALLCONV QTrkBuildLUT(struct QueuedTracker *qtrk, void *data, int pitch, QTRK_PixelDataType_t pdt,
                                         int plane, vector2f *known_pos);                                     /* qtrk_c_api.h:179 */
QTRK_API void QTRK_CALLCONV QTrkBuildLUTFromFrame(struct QueuedTracker *qtrk, ImageData *frame, int plane,
                                                  ROIPosition *roipos, int numroi);                           /* qtrk_c_api.h:184 */
QTRK_API void QTRK_CALLCONV QTrkFinalizeLUT(struct QueuedTracker *qtrk);                                      /* qtrk_c_api.h:185 */

/* ---- results and state (cputrack/qtrk_c_api.h:187-199) ---- */
QTRK_API int QTRK_CALLCONV QTrkGetResultCount(struct QueuedTracker *qtrk);                                    /* qtrk_c_api.h:187 */
QTRK_API int QTRK_CALLCONV QTrkFetchResults(struct QueuedTracker *qtrk, LocalizationResult *results, int maxResults); /* qtrk_c_api.h:188 */
QTRK_API int QTRK_CALLCONV QTrkGetQueueLength(struct QueuedTracker *qtrk, int *maxQueueLen);                  /* qtrk_c_api.h:190 */
QTRK_API bool QTRK_CALLCONV QTrkIsIdle(struct QueuedTracker *qtrk);                                           /* qtrk_c_api.h:191 */
QTRK_API void QTRK_CALLCONV QTrkGetProfileReport(struct QueuedTracker *qtrk, char *dst, int maxStrLen);       /* qtrk_c_api.h:198 */
QTRK_API void QTRK_CALLCONV QTrkGetWarnings(struct QueuedTracker *qtrk, char *dst, int maxStrLen);            /* qtrk_c_api.h:199 */

/* ---- profile utilities exported by the reference (cputrack/utils.h:182-188,216) ---- */
QTRK_API void QTRK_CALLCONV ComputeRadialProfile(float *dst, int radialSteps, int angularSteps, float minradius,
                                                 float maxradius, vector2f center, ImageData *src, float mean,
                                                 bool normalize);                                            /* utils.h:182 */
QTRK_API void QTRK_CALLCONV NormalizeRadialProfile(float *prof, int rsteps);                                  /* utils.h:183 */
QTRK_API void QTRK_CALLCONV NormalizeImage(ImageData *image);                                                 /* utils.h:185 */
/* utils.h:187-188 (C++ references there; a pointer is the same ABI). Noise from the C library's
 * rand(): seed it with srand() for a repeatable image. */
QTRK_API void QTRK_CALLCONV ApplyPoissonNoise(ImageData *img, float poissonMax, float maxValue);
QTRK_API void QTRK_CALLCONV ApplyGaussianNoise(ImageData *img, float sigma);
QTRK_API void QTRK_CALLCONV GenerateImageFromLUT(ImageData *image, ImageData *zlut, float minradius, float maxradius,
                                                 vector3f pos, bool useSplineInterp, int ovs);                /* utils.h:186 */
QTRK_API void QTRK_CALLCONV GenerateGaussianSpotImage(ImageData *img, vector2f pos, float sigma, float I0, float Ibg); /* utils.h:216 */

/* ================= Extensions (no reference counterpart) ================= */

/* Text of the last error raised by a call that has no instance to report to (e.g. a failed
 * QTrkCreateInstance). Returns the number of characters written. */
QTRK_API int QTRK_CALLCONV QTrkB200GetLastError(char *dst, int maxStrLen);

/* Number of CUDA kernels this instance launched since creation (all streams). */
QTRK_API int64_t QTRK_CALLCONV QTrkB200GetKernelLaunchCount(struct QueuedTracker *qtrk);

/*
 * Z-LUT bias correction table, table[bead][bias_plane] (bias_planes wide, count beads high); NULL
 * removes it. Replaces QueuedTracker::SetZLUTBiasCorrection (cputrack/QueuedTracker.h:334,
 * QueuedTracker.cpp:178-182; LabVIEW: qtrk_set_zlut_bias_table, lv_queuetrk_api.cpp:467-480).
 * While set, every z is corrected by QueuedTracker::ZLUTBiasCorrection's four fixed-point steps
 * (QueuedTracker.cpp:115-140) on the device. QTrkSetRadialZLUT removes the table, as the
 * reference does (QueuedCPUTracker.cpp:368-369).
 */
QTRK_API void QTRK_CALLCONV QTrkB200SetZLUTBiasTable(struct QueuedTracker *qtrk, const float *table, int bias_planes,
                                                     int count);
/* QueuedTracker::ComputeZBiasCorrection (cputrack/QueuedTracker.cpp:143-189; the reference reaches
 * it through qtrk_compute_zlut_bias_table, lv_queuetrk_api.cpp:457-466): render every bead's LUT at
 * bias_planes evenly spaced z (smpPerPixel^2 samples per pixel, B-spline or linear over planes),
 * localize each image (COM, 2 QI iterations, Z match), and set table[bead][plane] = z - true z as the
 * instance's bias table. `result` (may be NULL) receives the count x bias_planes table. */
QTRK_API void QTRK_CALLCONV QTrkB200ComputeZLUTBiasTable(struct QueuedTracker *qtrk, int bias_planes, float *result,
                                                         int smpPerPixel, int useSplineInterp);

/*
 * Localize `count` ROIs that are already resident in device memory, on the caller's CUDA
 * stream (cudaStream_t passed as void*; NULL = legacy default stream). ROI i starts at
 * d_pixels + i * roi_stride_bytes; rows are `pitch` bytes apart. d_jobs (device,
 * LocalizationJob[count]) may be NULL (job = {frame=i, zlutIndex=0}). d_results receives
 * LocalizationResult[count] (device). Uses the instance's mode, LUT and settings. Returns 0
 * on success, a negative code on a bad argument (see QTrkGetWarnings). Asynchronous.
 */
QTRK_API int QTRK_CALLCONV QTrkB200LocalizeDevice(struct QueuedTracker *qtrk, const void *d_pixels, int pitch,
                                                  int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int count,
                                                  const LocalizationJob *d_jobs, LocalizationResult *d_results,
                                                  void *stream);

/*
 * The adjoint of the Z match. No counterpart in the reference. For `count` device-resident ROIs
 * (ROI i at d_pixels + i * roi_stride_bytes, rows `pitch` bytes apart) and device positions
 * d_xyz[3i..3i+2] (x, y in pixels, z in LUT planes) against bead d_beads[i]'s LUT (bead 0 when
 * d_beads is NULL):
 *   cost_i = sum_r (w_r (phat_r(x, y) - Lz_r))^2,
 * phat the radial profile of the Z match at (x, y) (normalised when LT_NormalizeProfile is in the
 * mode), Lz the LUT linear between planes floor(z) and floor(z)+1 (clamped), w the radial weights
 * (1 when unset). Writes d_cost[i], d_grad_xyz[3i..3i+2] = d cost_i / d(x, y, z) and, when
 * d_grad_lut is not NULL, ADDS d cost_i / d LUT into d_grad_lut [beads][planes][radialsteps]
 * (zero it first). Device pointers, asynchronous on `stream`; returns 0, or < 0 on invalid
 * arguments (-3: no Z-LUT).
 */
QTRK_API int QTRK_CALLCONV QTrkB200ZLUTCostGradient(struct QueuedTracker *qtrk, const void *d_pixels, int pitch,
                                                    int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int count,
                                                    const float *d_xyz, const int *d_beads, float *d_cost,
                                                    float *d_grad_xyz, float *d_grad_lut, void *stream);

/*
 * The adjoint of the 2D Gaussian MLE. No counterpart in the reference. For `count` device-resident
 * ROIs (layout as QTrkB200LocalizeDevice) and device parameters d_params[5i..5i+4] = (x, y, I0, bg,
 * sigma), the Poisson negative log-likelihood of the integrated-Gaussian spot model the
 * 5-parameter MLE (LT_B200_Gaussian5P) fits,
 *   NLL_i = sum_pixels mu - I ln mu,  mu = bg + I0 DX(x, sigma) DY(y, sigma)   (ln I! dropped),
 * into d_nll[i] and its gradient with respect to the 5 parameters into d_grad[5i..5i+4]. Pixel
 * calibration images and factors apply as in localization. Asynchronous on `stream`; 0 or < 0.
 */
QTRK_API int QTRK_CALLCONV QTrkB200GaussianNLLGradient(struct QueuedTracker *qtrk, const void *d_pixels, int pitch,
                                                       int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int count,
                                                       const float *d_params, float *d_nll, float *d_grad,
                                                       void *stream);

/*
 * Z-LUT refinement from a calibration stack. No counterpart in the reference. The device stack
 * holds `planes` x `beads` ROIs, ROI (plane k, bead b) at d_stack + (k * beads + b) * roi_stride_bytes
 * (the order BuildLUT is fed in); the instance's LUT must have `beads` x `planes` rows (typically the
 * BuildLUT result). d_xy (device, [planes][beads][2], may be NULL) gives each ROI's bead position; NULL
 * locates them with COM + QI. Minimises, over the LUT and one z offset per plane (the stage position
 * error, common to all beads),
 *   sum_{k,b} cost(x, y, k + d_k, L_b) + smoothness * sum |L_b,k+1 - 2 L_b,k + L_b,k-1|^2
 * (cost as in QTrkB200ZLUTCostGradient) with `iterations` diagonally preconditioned steps. The data
 * term alone is already minimal at the BuildLUT result (each row absorbs its plane's image), so the
 * smoothness weight must be > 0 for anything to change; offsets keep zero mean and zero linear trend.
 * The refined LUT replaces the instance's LUT (its bias table is kept). plane_z (host, `planes`, may
 * be NULL) receives k + d_k; cost_history (host, iterations + 1, may be NULL) the objective before each
 * iteration and at the end.
 */
QTRK_API void QTRK_CALLCONV QTrkB200RefineZLUT(struct QueuedTracker *qtrk, const void *d_stack, int pitch,
                                               int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt, int beads, int planes,
                                               const float *d_xy, int iterations, float smoothness, float *plane_z,
                                               float *cost_history);

/*
 * QTrkB200LocalizeDevice without any device-memory allocation. No counterpart in the
 * reference. For callers that cannot allocate while they run: real-time acquisition threads
 * (camera callbacks, LabVIEW timed loops) that must keep each call's latency bounded, since
 * cudaMalloc/cudaFree take the driver's allocation lock and can synchronize the device, and
 * processes whose device-memory budget is fixed at start-up. Same arguments, results and
 * kernels as QTrkB200LocalizeDevice; the intermediate profiles of the tensor-core Z match
 * (LT_B200_ZMatchBF16 / LT_B200_ZMatchTF32) go to one fixed 16 MiB array inside the library, which every GPU that
 * loads the library holds until the process exits.
 * Limit: count * (4 * zlut_radialsteps + 4 * zlut_radialsteps rounded up to 16) bytes (plus up
 * to 255 bytes of alignment) must fit in 16 MiB: 32,768 ROIs of 64 radial bins. Larger counts
 * return -3 and launch nothing. The instance's BF16 copy of the Z-LUT is made by its first
 * allocating call in this mode (QTrkB200LocalizeDevice or a queued batch) and dropped whenever
 * QTrkSetRadialZLUT installs a LUT; while there is none of the current LUT's shape this call
 * returns -4 and launches nothing. New contents of a LUT of the same shape (BuildLUT,
 * FinalizeLUT, new radial weights) are copied into the existing BF16 copy by one kernel, after
 * the work already queued on `stream`; work of earlier calls on other streams must have finished
 * before the LUT changes. With device-side jobs (d_jobs != NULL) Z uses the plain match, which
 * needs no scratch.
 * The first call on each device looks up the array's device address; make that first call
 * before any stream capture. All calls share the array and each overwrites what it reads, so
 * nothing needs clearing; calls whose GPU work overlaps (other streams, other instances on the
 * same GPU) race on it.
 */
QTRK_API int QTRK_CALLCONV QTrkB200LocalizeDeviceNoAlloc(struct QueuedTracker *qtrk, const void *d_pixels, int pitch,
                                                         int64_t roi_stride_bytes, QTRK_PixelDataType_t pdt,
                                                         int count, const LocalizationJob *d_jobs,
                                                         LocalizationResult *d_results, void *stream);

/* ---- .radialzlut files (the layout cputrack/utils.cpp:680-710 reads): int32 count, planes,
 * radialsteps, then count*planes*radialsteps float32 in [bead][plane][bin] order. Read with
 * dst = NULL to query the sizes. Return 0, or < 0 on error (QTrkB200GetLastError says why). */
QTRK_API int QTRK_CALLCONV QTrkB200ReadRadialZLUTFile(const char *path, float *dst, int *count, int *planes,
                                                      int *radialsteps);
QTRK_API int QTRK_CALLCONV QTrkB200WriteRadialZLUTFile(const char *path, const float *data, int count, int planes,
                                                       int radialsteps);

/* ---- bead finder (cputrack/qtrk_c_api.h:203-205; qtrk_c_api.cpp:28-58; BeadFinder.cpp) ----
 * Template match of the sample ROI at (smpCornerPosX, smpCornerPosY) over the image; returns
 * the ROI corners of the beads found (*beadcount of them), to be freed with
 * QTrkFreeROIPositions; `sample` (if roi x roi) receives the sample. The convolution runs on the
 * current CUDA device. Returns NULL (and *beadcount = 0) on invalid arguments; unlike the
 * reference, a sample ROI that is not inside the image is an error. */
QTRK_API void QTRK_CALLCONV QTrkFreeROIPositions(ROIPosition *data);
QTRK_API ROIPosition *QTRK_CALLCONV QTrkFindBeads(ImageData *imgData, int smpCornerPosX, int smpCornerPosY, int roi,
                                                  float imgRelDist, float acceptance, int *beadcount,
                                                  ImageData *sample);

/* ---- ResultManager (cputrack/qtrk_c_api.cpp:181-241, cputrack/ResultManager.cpp) ----
 * Bins the results of one tracker per frame and bead (bead = zlutIndex), writes completed frames
 * to a text or binary file every writeInterval frames, keeps at most maxFramesInMemory frames.
 * A background thread fetches the attached tracker's results. */
struct ResultManager;
#ifndef __cplusplus
typedef struct ResultManager ResultManager;
#endif
QTRK_API struct ResultManager *QTRK_CALLCONV RMCreate(const char *file, const char *frameinfo,
                                                      ResultManagerConfig *cfg, const char *semicolonSeparatedNames);
QTRK_API void QTRK_CALLCONV RMSetTracker(struct ResultManager *rm, struct QueuedTracker *qtrk);
QTRK_API void QTRK_CALLCONV RMDestroy(struct ResultManager *rm);
QTRK_API void QTRK_CALLCONV RMStoreFrameInfo(struct ResultManager *rm, int frame, double timestamp, float *cols);
QTRK_API int QTRK_CALLCONV RMGetBeadResults(struct ResultManager *rm, int start, int numFrames, int bead,
                                            LocalizationResult *results);
QTRK_API void QTRK_CALLCONV RMGetFrameCounters(struct ResultManager *rm, RMFrameCounters *dst);
QTRK_API void QTRK_CALLCONV RMFlush(struct ResultManager *rm);
QTRK_API int QTRK_CALLCONV RMGetResults(struct ResultManager *rm, int startFrame, int numFrames,
                                        LocalizationResult *results);
QTRK_API void QTRK_CALLCONV RMRemoveBead(struct ResultManager *rm, int bead);
QTRK_API void QTRK_CALLCONV RMGetConfig(struct ResultManager *rm, ResultManagerConfig *cfg);
/* Extension: store results that did not come from the attached tracker's queue (for example the
 * request server's per-frame results); roi_width/roi_height give the ROI centre that is
 * subtracted. No counterpart in the reference. */
QTRK_API void QTRK_CALLCONV QTrkB200RMStoreResults(struct ResultManager *rm, const LocalizationResult *results,
                                                   int count, int roi_width, int roi_height);

/* QTrkBuildLUT (qtrk_c_api.h:179) that does not wait for the plane's host-to-device copy: for a
 * stack in pinned (page-locked) host memory the call returns once the copy and the plane's kernel
 * are queued, so the copies of successive planes run back to back; the caller must keep `data`
 * unchanged until QTrkFinalizeLUT returns. A pageable stack is staged before the call returns, as by
 * QTrkBuildLUT. No counterpart in the reference (its BuildLUT is synchronous). */
QTRK_API void QTRK_CALLCONV QTrkB200BuildLUTAsync(struct QueuedTracker *qtrk, void *data, int pitch,
                                                  QTRK_PixelDataType_t pdt, int plane, vector2f *known_pos);

/* Instance-level forms of the reference's handle-less calls (qtrk_c_api.h:152-158 act on every or
 * the latest instance), as the LabVIEW layer needs them. */
QTRK_API void QTRK_CALLCONV QTrkB200SetPixelCalibrationFactors(struct QueuedTracker *qtrk, float offsetFactor,
                                                               float gainFactor);
QTRK_API void QTRK_CALLCONV QTrkB200EnableRadialZLUTCompareProfile(struct QueuedTracker *qtrk, int enable);
QTRK_API void QTRK_CALLCONV QTrkB200GetRadialZLUTCompareProfile(struct QueuedTracker *qtrk, float *dst);
/* SetCUDADevices (cudatrack/QueuedCUDATracker.cu): the device list for cuda_device = QTrkCUDA_UseList.
 * An instance drives one GPU, the first device of the list (the current device if the list is empty). */
QTRK_API void QTRK_CALLCONV QTrkB200SetCUDADevices(const int *devices, int count);
/* RMCreate with the frame-info column names as an array (rm_create of lv_resultmanager_api.cpp:26-35). */
QTRK_API struct ResultManager *QTRK_CALLCONV QTrkB200RMCreateNamed(const char *file, const char *frameinfo,
                                                                   ResultManagerConfig *cfg,
                                                                   const char *const *names, int count);

/*
 * Request server: real-time localization of frames from several instances on one GPU. No
 * counterpart in the reference (its callers run one QueuedTracker per camera and poll each).
 * A server owns device "lanes" (one stream, a 48 MiB pixel buffer and room for 8,192 ROIs each);
 * the number of lanes is device_memory_budget divided by a lane's size (at least 1, at most 16).
 * Instances are attached once; frames are then submitted from any thread. A dispatcher thread
 * admits waiting frames to free lanes in arrival order, merges waiting frames of the same
 * instance and pixel type into one launch while they fit the lane (continuous batching), copies
 * each frame's ROI band to the lane and replays a CUDA graph holding the localization kernel and
 * the result copy (one graph per lane, instance, power-of-two ROI-count bucket and band count: a
 * batch above ~6 MiB is copied in up to four row bands, each band's kernel starting as its rows
 * arrive). A frame's
 * results are the ones QTrkScheduleFrame gives for it: ROIs outside the frame are skipped and
 * result i carries zlutIndex = i + job->zlutIndex. The graphs hold the plain Z match: the tensor-core
 * match and the joint refinement (LT_B200_ZMatchBF16/TF32, LT_B200_JointRefine) are not applied here.
 */
typedef struct QTrkB200ServeStats {
    int64_t frames;            /* frames completed */
    int64_t rois;              /* ROIs localized */
    int64_t launches;          /* graph launches (one per lane batch) */
    int64_t graphs;            /* graphs captured */
    int64_t waits_for_memory;  /* frames that arrived while every lane was busy or frames waited */
    int32_t lanes;             /* lanes the memory budget allowed */
    int32_t reserved;
    double elapsed_s;          /* first submission to last completion */
    double p50_ms, p99_ms, max_ms;  /* per-frame latency, submission to results on the host */
} QTrkB200ServeStats;

QTRK_API void *QTRK_CALLCONV QTrkB200ServerCreate(int device, int64_t device_memory_budget);
QTRK_API void QTRK_CALLCONV QTrkB200ServerDestroy(void *server);
/* Attach an instance (on the server's GPU); returns its index, or -1. The instance must outlive
 * the server; its LUT and mode may change between frames (each launch reads them then). */
QTRK_API int QTRK_CALLCONV QTrkB200ServerAttach(void *server, struct QueuedTracker *qtrk);
/* Submit one frame of an attached instance. The frame (host memory, pitch in bytes) must stay
 * valid until the request completes. Returns the request id (> 0), or -1 on error (more than
 * 8,192 ROIs, a ROI band larger than a lane, a bad argument). */
QTRK_API int64_t QTRK_CALLCONV QTrkB200ServerSubmitFrame(void *server, int instance, const void *frame, int pitch,
                                                         int width, int height, const ROIPosition *positions,
                                                         int numROI, QTRK_PixelDataType_t pdt,
                                                         const LocalizationJob *jobInfo);
/* Results of a request: the number written (the request is then forgotten), -1 while it is
 * pending, -2 for an unknown id, -3 when its launch failed (QTrkB200GetLastError says why). */
QTRK_API int QTRK_CALLCONV QTrkB200ServerPoll(void *server, int64_t request, LocalizationResult *results,
                                              int maxResults);
QTRK_API void QTRK_CALLCONV QTrkB200ServerGetStats(void *server, QTrkB200ServeStats *stats);
/* Restart the statistics (frames, ROIs, launches, waits, latencies, elapsed time); captured
 * graphs and lanes are kept. Frames in flight are counted by the new statistics. */
QTRK_API void QTRK_CALLCONV QTrkB200ServerResetStats(void *server);
/* hold != 0: submitted frames wait and no new launch starts (launches in flight finish);
 * hold == 0: admission resumes and the frames that waited are batched together. For callers that
 * collect the frames of one trigger (several cameras) before they are localized together. */
QTRK_API void QTRK_CALLCONV QTrkB200ServerHold(void *server, int hold);

#endif /* QTRK_B200_C_API_H */
