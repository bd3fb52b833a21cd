// QueuedTracker implementation for one B200.
//
// Mirrors the reference's abstract QueuedTracker (cputrack/QueuedTracker.h:22-96) and the
// behaviour of its CUDA implementation (cudatrack/QueuedCUDATracker.*): jobs are copied
// into pinned staging slots on the caller's thread; a full slot (or Flush) is submitted as
// one asynchronous H2D copy + one localization kernel + one D2H copy on the slot's own
// CUDA stream; completed slots are drained in submission order (FIFO) by whichever API
// call polls next. There is no worker thread and no CPU fallback.
#pragma once
#include <atomic>
#include <cstdint>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "qtrk_c_api.h"
#include "track_params.h"
#include "zmatch_tc.h"

// The opaque handle type of the C ABI.
struct QueuedTracker {
    virtual ~QueuedTracker() {}
};

namespace qtrk {

// QTrkComputedConfig::Update, cputrack/QueuedTracker.cpp:6-21 (float arithmetic and int
// truncation as in the reference) and NearestPowerOf2, cputrack/utils.cpp:644-652.
int nearest_pow2(int v);
QTrkComputedConfig compute_config(const QTrkSettings &s);
// ComputeRadialBinWindow, cputrack/utils.cpp:665-677.
std::vector<float> radial_bin_window(int rsteps);

struct QueueStats {
    int64_t batches = 0, rois = 0;
    double gpu_ms = 0;                 // summed kernel+copy time of drained batches (CUDA events)
    std::vector<float> latency_ms;     // per batch: submission -> drained, host clock
};

class Tracker : public QueuedTracker {
  public:
    explicit Tracker(const QTrkSettings &settings);
    ~Tracker() override;

    QTrkComputedConfig cfg;

    void SetLocalizationMode(LocMode_t mode);
    void SetPixelCalibrationImages(const float *offset, const float *gain);
    void SetPixelCalibrationFactors(float offsetFactor, float gainFactor);
    void ScheduleLocalization(const void *data, int pitch, int pdt, const LocalizationJob *job);
    int ScheduleFrame(const void *img, int pitch, int width, int height, const ROIPosition *pos, int n, int pdt,
                      const LocalizationJob *job);
    void ClearResults();
    void Flush();
    void SetRadialZLUT(const float *data, int count, int planes);
    void GetRadialZLUT(float *dst);
    void GetRadialZLUTSize(int &count, int &planes, int &radialsteps) const;
    void SetRadialWeights(const float *w);
    void EnableRadialZLUTCompareProfile(bool enabled);
    void GetRadialZLUTCompareProfile(float *dst);
    void BeginLUT(uint32_t flags);
    // async: a pinned `data` may still be read after the call returns, until FinalizeLUT returns
    void BuildLUT(const void *data, int pitch, int pdt, int plane, const vector2f *known_pos, bool async = false);
    void FinalizeLUT();
    int GetResultCount();
    int FetchResults(LocalizationResult *dst, int maxResults);
    int GetQueueLength(int *maxQueueLen);
    bool IsIdle();
    std::string GetProfileReport();
    std::string GetWarnings();

    // Extensions
    void SetZLUTBiasTable(const float *table, int bias_planes, int count);
    void ComputeZBiasTable(int bias_planes, int smp_per_pixel, bool spline, float *out);
    int LocalizeDevice(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                       const LocalizationJob *d_jobs, LocalizationResult *d_results, cudaStream_t stream);
    // LocalizeDevice with caller-supplied profile scratch (scratch_bytes); allocates nothing.
    int LocalizeDeviceNoAlloc(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                              const LocalizationJob *d_jobs, LocalizationResult *d_results, cudaStream_t stream,
                              void *scratch, size_t scratch_bytes);
    void RefineZLUT(const void *d_stack, int pitch, int64_t roi_stride, int pdt, int beads, int planes, const float *d_xy,
                    int iterations, float smoothness, float *plane_z, float *cost_history);
    int GaussianNLLGradient(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                            const float *d_params, float *d_nll, float *d_grad, cudaStream_t stream);
    int ZLUTCostGradient(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count, const float *d_xyz,
                         const int *d_beads, float *d_cost, float *d_grad, float *d_glut, cudaStream_t stream);
    int64_t LaunchCount() const { return launches_.load(); }
    void Warn(const std::string &msg);
    int device() const { return device_; }
    TrackParams Params(int pdt) const;  // current parameters (the transposed LUT only if fresh)
    // Parameters for one launch that another component (the request server) puts on `stream`:
    // the stream is ordered after pending LUT work and the launch is counted.
    TrackParams AcquireLaunch(int pdt, cudaStream_t stream);

  private:
    struct Slot {
        cudaStream_t stream = nullptr;
        cudaEvent_t ev_start = nullptr, ev_done = nullptr;
        uint8_t *h_pix = nullptr, *d_pix = nullptr;
        LocalizationJob *h_jobs = nullptr, *d_jobs = nullptr;
        LocalizationResult *h_res = nullptr, *d_res = nullptr;
        int64_t *h_off = nullptr, *d_off = nullptr;
        // tensor-core Z match scratch (allocated on first use): profiles between the two
        // kernels, the bead-grouped ROI order and the tile list
        float *d_zprof = nullptr;
        __nv_bfloat16 *d_zprof_bf16 = nullptr;
        int *h_perm = nullptr, *d_perm = nullptr;
        int4 *h_tiles = nullptr, *d_tiles = nullptr;
        int count = 0, pdt = -1;
        bool frame = false;   // pixels hold frame rows addressed through d_off
        int pitch = 0;
        double t_submit = 0;  // host seconds
    };

    void AllocateSlots();
    int AcquireSlotLocked(std::unique_lock<std::mutex> &lk);  // a free slot index (may wait)
    void SubmitLocked(int idx);
    void CollectLocked();            // drain completed slots (FIFO)
    void DrainAllLocked(std::unique_lock<std::mutex> &lk);
    void WaitIdleForReconfigure();
    void CheckCuda(cudaError_t e, const char *what);
    static bool IsPinned(const void *p);
    bool UseTensorCoreMatch() const;     // mode asks for it and the LUT shape allows it
    static bool RefineAfterZ(const TrackParams &P);
    void PrepareTensorCoreLUT();         // BF16 weighted LUT + norms when stale (LUT stream)
    // Params for a localization launch: refreshes the transposed LUT first when stale (a kernel on
    // the LUT stream, no allocation); the caller's stream must wait on lut_ready_ afterwards.
    TrackParams LaunchParams(int pdt);
    ZMatchParams TensorCoreParams() const;
    int BuildTiles(const LocalizationJob *jobs, int count, int *perm, int4 *tiles) const;

    int device_ = 0;
    LocMode_t mode_ = 0;
    TrackParams base_{};
    int batch_ = 0;              // ROIs per slot
    size_t slot_bytes_ = 0;      // pixel bytes per slot
    std::vector<Slot> slots_;
    std::deque<int> free_, inflight_;
    int filling_ = -1;

    // device tables
    void *d_qdirs_ = nullptr, *d_tw_ = nullptr, *d_zdirs_ = nullptr;
    float *d_qi_rw_ = nullptr;

    // Z-LUT state
    float *d_lut_ = nullptr;
    int lut_count_ = 0, lut_planes_ = 0;
    float *d_lut_t_ = nullptr;   // transposed copy, allocated with d_lut_
    bool lut_t_stale_ = true;
    float *d_zw_ = nullptr;
    bool have_zw_ = false;
    float *d_cmp_ = nullptr;
    bool cmp_enabled_ = false;
    uint32_t lut_flags_ = 0;
    cudaStream_t lut_stream_ = nullptr;
    cudaEvent_t lut_ready_ = nullptr;
    uint8_t *h_lut_stage_[2] = {nullptr, nullptr};
    uint8_t *d_lut_stage_[2] = {nullptr, nullptr};
    cudaEvent_t lut_stage_free_[2] = {nullptr, nullptr};
    cudaStream_t lut_copy_stream_ = nullptr;          // H2D of pinned BuildLUT stacks
    cudaEvent_t lut_copy_done_[2] = {nullptr, nullptr};
    size_t lut_stage_bytes_ = 0;
    int lut_stage_next_ = 0;

    // tensor-core Z match state
    __nv_bfloat16 *d_lut_bf16_ = nullptr;
    float *d_lut_norm_ = nullptr;
    bool tc_lut_stale_ = true;
    // the (beads, padded planes, padded bins) shape d_lut_bf16_ / d_lut_norm_ were allocated for;
    // an in-place refresh is only valid while it equals the current LUT's shape
    int tc_lut_count_ = 0, tc_lut_pp_ = 0, tc_lut_nbp_ = 0;
    cudaEvent_t noalloc_order_ = nullptr;  // orders an in-place BF16 refresh after the caller's earlier work
    unsigned *h_err_ = nullptr, *d_err_ = nullptr;  // mapped pinned word set by the Z-match kernel
    float *d_dev_zprof_ = nullptr;                  // scratch of the device-resident entry point
    __nv_bfloat16 *d_dev_zprof_bf16_ = nullptr;
    int4 *d_dev_tiles_ = nullptr;
    int dev_scratch_rois_ = 0;

    // Z-LUT bias table
    float *d_zbias_ = nullptr;
    int zbias_w_ = 0, zbias_count_ = 0;

    // pixel calibration
    float *d_calib_off_ = nullptr, *d_calib_gain_ = nullptr;
    int calib_count_ = 0;
    float offset_factor_ = 1.0f, gain_factor_ = 1.0f;

    std::mutex mu_;      // slots, queues, LUT state
    std::mutex res_mu_;  // results_
    std::deque<LocalizationResult> results_;
    std::mutex warn_mu_;
    std::string warnings_;
    std::atomic<int64_t> launches_{0};
    QueueStats stats_;
};

// Process-wide registry: the reference declares some entry points without an instance
// argument (cputrack/qtrk_c_api.h:153,165-166); they act on live instances through it.
void register_tracker(Tracker *t);
void unregister_tracker(Tracker *t);
Tracker *latest_tracker();
void for_each_tracker(void (*fn)(Tracker *, void *), void *arg);
void set_device_list(const std::vector<int> &devices);  // QTrkCUDA_UseList devices
float default_offset_factor();
float default_gain_factor();
void set_default_factors(float of, float gf);

}  // namespace qtrk
