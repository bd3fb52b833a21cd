/*
 * LabVIEW binding of libqtrk_b200 (libqtrk_b200_lv.so): the qtrk_* and rm_* functions of the
 * reference's LabVIEW layer (cputrack/lv_qtrk_api.h:7-46, cputrack/lv_queuetrk_api.cpp:19-695,
 * cputrack/lv_resultmanager_api.cpp:21-125) with the same names, argument order and meaning, so
 * that the QTrkLVBinding VIs call it unchanged. Arrays are LabVIEW handles (T**) to
 * {int32 dimSizes[N]; T elem[]} with natural alignment; strings are LStrHandle; errors are
 * reported in the ErrorCluster (status, code, message) and never thrown. Array arguments are
 * handles passed by value, as the reference's T** parameters. The library calls the
 * LabVIEW run-time functions NumericArrayResize and MoveBlock, which the LabVIEW process that
 * loads it provides.
 *
 * Differences from the reference, each a fix of an out-of-range access or a wrong size there:
 *   - every qtrk_* function that takes a tracker validates it (the reference skips this in the
 *     qtrk_queue_* functions);
 *   - qtrk_build_lut_plane reads rows at width * sizeof(float) (the reference passes
 *     width * sizeof(float*), twice the row length on 64-bit);
 *   - array resizes ask for the number of elements (the reference passes a byte count);
 *   - image LUTs (LT_ZLUTAlign / image-LUT modes) are not supported: qtrk_get_image_lut returns an
 *     empty array and qtrk_set_image_lut with a non-empty LUT reports an argument error.
 */
#ifndef QTRK_B200_LV_API_H
#define QTRK_B200_LV_API_H

#include "qtrk_c_api.h"

#ifdef __cplusplus
#define QTRK_LV_API extern "C" QTRK_EXPORT
#else
#define QTRK_LV_API QTRK_EXPORT
#endif

/* LabVIEW C interface types (the public LabVIEW "extcode.h" interface, restated). */
typedef int32_t MgErr;
typedef uint8_t LVBoolean;
typedef struct { int32_t cnt; uint8_t str[1]; } LStr, *LStrPtr, **LStrHandle;
typedef void **UHandle;
#define QTRK_LV_mgNoErr 0
#define QTRK_LV_mgArgErr 1
#define QTRK_LV_kAppErrorBase 5000

/* cputrack/labview.h:14-18 */
typedef struct { LVBoolean status; int32_t code; LStrHandle message; } ErrorCluster;

/* LabVIEW array handles (cputrack/labview.h:21-55) */
typedef struct { int32_t dimSize; float elem[1]; } LVArrayFloat, **LVArrayFloatHdl;
typedef struct { int32_t dimSize; int32_t elem[1]; } LVArrayInt, **LVArrayIntHdl;
typedef struct { int32_t dimSizes[2]; float elem[1]; } LVArray2DFloat, **LVArray2DFloatHdl;
typedef struct { int32_t dimSizes[2]; int32_t elem[1]; } LVArray2DInt, **LVArray2DIntHdl;
typedef struct { int32_t dimSizes[2]; uint32_t elem[1]; } LVArray2DUInt, **LVArray2DUIntHdl;
typedef struct { int32_t dimSizes[2]; uint16_t elem[1]; } LVArray2DU16, **LVArray2DU16Hdl;
typedef struct { int32_t dimSizes[2]; uint8_t elem[1]; } LVArray2DU8, **LVArray2DU8Hdl;
typedef struct { int32_t dimSizes[3]; float elem[1]; } LVArray3DFloat, **LVArray3DFloatHdl;
typedef struct { int32_t dimSizes[4]; float elem[1]; } LVArray4DFloat, **LVArray4DFloatHdl;

/* cputrack/lv_qtrk_api.h:18-20, 36-42 */
typedef int QueueFrameFlags;
typedef struct { LStrHandle name; int clockRate; int multiProcCount; int major, minor; } CUDADeviceInfo;

/* ---- tracker ---- */
QTRK_LV_API void qtrk_free_all(void);
QTRK_LV_API int qtrk_get_debug_image(struct QueuedTracker *qtrk, int id, LVArray2DFloatHdl data, ErrorCluster *e);
QTRK_LV_API void qtrk_set_logfile_path(const char *path);
QTRK_LV_API void qtrk_get_computed_config(struct QueuedTracker *qtrk, QTrkComputedConfig *cc, ErrorCluster *err);
QTRK_LV_API void qtrk_set_ZLUT(struct QueuedTracker *tracker, LVArray3DFloatHdl pZlut, LVArrayFloatHdl zcmpWindow,
                               int normalize, ErrorCluster *e);
QTRK_LV_API void qtrk_get_ZLUT(struct QueuedTracker *tracker, LVArray3DFloatHdl pzlut, ErrorCluster *e);
QTRK_LV_API void qtrk_get_image_lut(struct QueuedTracker *qtrk, LVArray4DFloatHdl imageLUT, ErrorCluster *e);
QTRK_LV_API void qtrk_set_image_lut(struct QueuedTracker *qtrk, LVArray4DFloatHdl imageLUT,
                                    LVArray3DFloatHdl radialZLUT, ErrorCluster *e);
QTRK_LV_API void qtrk_set_pixel_calib_factors(struct QueuedTracker *qtrk, float offsetFactor, float gainFactor,
                                              ErrorCluster *e);
QTRK_LV_API void qtrk_set_pixel_calib(struct QueuedTracker *qtrk, LVArray3DFloatHdl offset, LVArray3DFloatHdl gain,
                                      ErrorCluster *e);
QTRK_LV_API struct QueuedTracker *qtrk_create(QTrkSettings *settings, LStrHandle warnings, ErrorCluster *e);
QTRK_LV_API void qtrk_destroy(struct QueuedTracker *qtrk, ErrorCluster *error);
QTRK_LV_API void qtrk_queue_u16(struct QueuedTracker *qtrk, ErrorCluster *error, LVArray2DU16Hdl data,
                                const LocalizationJob *jobInfo);
QTRK_LV_API void qtrk_queue_u8(struct QueuedTracker *qtrk, ErrorCluster *error, LVArray2DU8Hdl data,
                               const LocalizationJob *jobInfo);
QTRK_LV_API void qtrk_queue_float(struct QueuedTracker *qtrk, ErrorCluster *error, LVArray2DFloatHdl data,
                                  const LocalizationJob *jobInfo);
QTRK_LV_API void qtrk_queue_pitchedmem(struct QueuedTracker *qtrk, uint8_t *data, int pitch, uint32_t pdt,
                                       const LocalizationJob *jobInfo);
QTRK_LV_API void qtrk_queue_array(struct QueuedTracker *qtrk, ErrorCluster *error, LVArray2DU8Hdl data, uint32_t pdt,
                                  const LocalizationJob *jobInfo);
QTRK_LV_API uint32_t qtrk_read_timestamp(uint8_t *image, int w, int h);
QTRK_LV_API uint32_t qtrk_queue_frame(struct QueuedTracker *qtrk, uint8_t *image, int pitch, int w, int h, uint32_t pdt,
                                      ROIPosition *pos, int numROI, const LocalizationJob *pJobInfo,
                                      QueueFrameFlags flags, ErrorCluster *e);
QTRK_LV_API void qtrk_clear_results(struct QueuedTracker *qtrk, ErrorCluster *e);
QTRK_LV_API void qtrk_build_lut_plane(struct QueuedTracker *qtrk, LVArray3DFloatHdl data, uint32_t flags, int plane,
                                      ErrorCluster *err);
QTRK_LV_API void qtrk_finalize_lut(struct QueuedTracker *qtrk, ErrorCluster *e);
QTRK_LV_API int qtrk_get_queue_len(struct QueuedTracker *qtrk, int *maxQueueLen, ErrorCluster *e);
QTRK_LV_API int qtrk_resultcount(struct QueuedTracker *qtrk, ErrorCluster *e);
QTRK_LV_API void qtrk_flush(struct QueuedTracker *qtrk, ErrorCluster *e);
QTRK_LV_API int qtrk_get_results(struct QueuedTracker *qtrk, LocalizationResult *results, int maxResults,
                                 int sortByID, ErrorCluster *e);
QTRK_LV_API void qtrk_get_zlut_cmpprof(struct QueuedTracker *qtrk, LVArray2DFloatHdl output, ErrorCluster *e);
QTRK_LV_API void qtrk_enable_zlut_cmpprof(struct QueuedTracker *qtrk, bool enable, ErrorCluster *e);
QTRK_LV_API void qtrk_set_localization_mode(struct QueuedTracker *qtrk, uint32_t locType, ErrorCluster *e);
QTRK_LV_API int qtrk_idle(struct QueuedTracker *qtrk, ErrorCluster *e);
QTRK_LV_API void qtrk_compute_zlut_bias_table(struct QueuedTracker *qtrk, int bias_planes, LVArray2DFloatHdl lvresult,
                                              int smpPerPixel, int useSplineInterp, ErrorCluster *e);
QTRK_LV_API void qtrk_set_zlut_bias_table(struct QueuedTracker *qtrk, LVArray2DFloatHdl biastbl, ErrorCluster *e);
QTRK_LV_API void qtrk_generate_gaussian_spot(LVArray2DFloatHdl image, vector2f *pos, float sigma, float I0,
                                             float Ibg, int applyNoise);
QTRK_LV_API void qtrk_generate_image_from_lut(LVArray2DFloatHdl image, LVArray2DFloatHdl lut, float *LUTradii,
                                              vector2f *position, float z, float M, float sigma_noise);
QTRK_LV_API void qtrk_dump_memleaks(void);
QTRK_LV_API void qtrk_get_profile_report(struct QueuedTracker *qtrk, LStrHandle str);
QTRK_LV_API void qtrk_compute_fisher(LVArray2DFloatHdl lut, QTrkSettings *cfg, vector3f *pos,
                                     LVArray2DFloatHdl fisherMatrix, LVArray2DFloatHdl inverseMatrix,
                                     vector3f *xyzVariance, int Nsamples, float maxPixelValue);
QTRK_LV_API void qtrk_find_beads(uint8_t *image, int pitch, int w, int h, int *smpCornerPos, int roi,
                                 float imgRelDist, float acceptance, LVArray2DUIntHdl output);
QTRK_LV_API void test_array_passing(int n, LVArrayFloatHdl flt1D, LVArray2DFloatHdl flt2D, LVArrayIntHdl int1D,
                                    LVArray2DIntHdl int2D);
QTRK_LV_API void qtrk_simulate_tracking(struct QueuedTracker *qtrk, int nsmp, int beadIndex, vector3f *centerPos,
                                        vector3f *range, vector3f *outBias, vector3f *outScatter,
                                        float photonsPerWell, ErrorCluster *e);
QTRK_LV_API void qtrkcuda_set_device_list(LVArrayIntHdl devices);
QTRK_LV_API int qtrkcuda_device_count(ErrorCluster *e);
QTRK_LV_API void qtrkcuda_get_device(int device, CUDADeviceInfo *info, ErrorCluster *e);
QTRK_LV_API void qtrkcuda_enable_texture_cache(struct QueuedTracker *qtrk, int enable, ErrorCluster *e);

/* ---- ResultManager (cputrack/lv_resultmanager_api.cpp) ---- */
QTRK_LV_API void rm_destroy_all(void);
QTRK_LV_API struct ResultManager *rm_create(const char *file, const char *frameinfo, ResultManagerConfig *cfg,
                                            LStrHandle *names);
QTRK_LV_API void rm_set_tracker(struct ResultManager *rm, struct QueuedTracker *qtrk, ErrorCluster *err);
QTRK_LV_API void rm_destroy(struct ResultManager *rm, ErrorCluster *err);
QTRK_LV_API void rm_store_frame_info(struct ResultManager *rm, int frame, double timestamp, float *cols,
                                     ErrorCluster *err);
QTRK_LV_API int rm_getbeadresults(struct ResultManager *rm, int start, int numFrames, int bead,
                                  LocalizationResult *results, ErrorCluster *err);
QTRK_LV_API void rm_getframecounters(struct ResultManager *rm, int *startFrame, int *lastSaveFrame, int *endFrame,
                                     int *capturedFrames, int *localizationsDone, int *lostFrames, ErrorCluster *err);
QTRK_LV_API void rm_flush(struct ResultManager *rm, ErrorCluster *err);
QTRK_LV_API int rm_getresults(struct ResultManager *rm, int startFrame, int numFrames, LocalizationResult *results,
                              ErrorCluster *err);
QTRK_LV_API void rm_removebead(struct ResultManager *rm, int bead, ErrorCluster *err);
QTRK_LV_API void rm_getconfig(struct ResultManager *rm, ResultManagerConfig *cfg, ErrorCluster *err);

#endif /* QTRK_B200_LV_API_H */
