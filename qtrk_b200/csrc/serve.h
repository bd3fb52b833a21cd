// Real-time request loop over several tracker instances on one GPU (continuous batching).
//
// Frames from any number of attached QueuedTracker instances (each with its own ROI size,
// pixel type, mode and Z-LUT) are submitted as they arrive. A dispatcher thread admits them
// to device lanes as lanes free up (the number of lanes is what the device-memory budget
// allows), merges waiting frames of the same instance into one launch, copies each frame's
// ROI band to the lane, and replays a CUDA graph captured per (lane, instance, bead-count
// bucket) that holds the localization kernel and the result copy. Results are polled per
// frame; per-frame latency (submission to results on the host) is recorded.
#pragma once
#include <atomic>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "qtrk_c_api.h"
#include "tracker.h"

namespace qtrk {

class Server {
  public:
    Server(int device, int64_t memory_budget);
    ~Server();

    int Attach(Tracker *t);
    int64_t Submit(int instance, const void *frame, int pitch, int width, int height, const ROIPosition *pos, int n,
                   int pdt, const LocalizationJob *job);
    int Poll(int64_t id, LocalizationResult *out, int max);
    QTrkB200ServeStats Stats();
    std::string LastError();
    void Hold(bool hold);
    void ResetStats();     // counters and latencies restart (graphs and lanes are kept)  // while held, frames wait and no lane is given work

    static constexpr int kMaxLaneRois = 8192;
    static constexpr size_t kLaneBytes = 48u << 20;
    static constexpr double kIdleSpinSeconds = 0.005;  // dispatcher polls this long before it sleeps
    static constexpr size_t kBandBytes = 6u << 20;  // a batch is copied in bands of about this size (<= 4)

  private:
    struct Request {
        int64_t id;
        int inst, pdt;
        const uint8_t *frame;
        int pitch;
        int x0, y0, w, h;                 // band of the frame that holds the valid ROIs
        std::vector<int64_t> offs;        // ROI offsets inside the band (band pitch)
        std::vector<LocalizationJob> jobs;
        double t_submit = 0, t_done = 0;
        bool done = false, failed = false;
        std::vector<LocalizationResult> results;
    };
    static constexpr int kMaxBands = 4;
    struct Graph {
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t kernel[kMaxBands] = {};  // one localization kernel per row band
        int bands = 1;
        int bucket = 0;
    };
    struct Lane {
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        // a large batch is copied in row bands on copy_stream; band b's kernel waits on band_done[b]
        cudaStream_t copy_stream = nullptr;
        cudaEvent_t band_done[kMaxBands] = {};
        uint8_t *d_pix = nullptr;
        int64_t *d_off = nullptr, *h_off = nullptr;
        LocalizationJob *d_jobs = nullptr, *h_jobs = nullptr;
        LocalizationResult *d_res = nullptr, *h_res = nullptr;
        std::vector<int64_t> reqs;        // requests in flight on this lane, in result order
        int count = 0;
        bool busy = false;                // set and cleared under the lock
        std::map<uint64_t, Graph> graphs; // key: instance, bucket, pixel type, mode, shared memory
        // arguments patched into the graph's kernel node at each replay
        TrackParams P{};
        const uint8_t *a_pix = nullptr;
        int a_pitch = 0;
        int64_t a_stride = 0;
        const int64_t *a_off = nullptr;
        const LocalizationJob *a_jobs = nullptr;
        int a_count = 0;
        LocalizationResult *a_res = nullptr;
        void *args[8] = {};
    };

    void Run();                                   // dispatcher thread
    void LaunchBatch(Lane &lane, Tracker *t, const std::vector<Request *> &batch);
    void Fail(const std::vector<int64_t> &ids);  // mark requests done without results
    Graph &GraphFor(Lane &lane, int inst, int bucket, int bands, const TrackParams &P);
    void Complete(Lane &lane);
    void Release();  // free every lane (destructor, failed constructor)

    int device_;
    std::vector<Tracker *> inst_;
    std::vector<Lane> lanes_;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<int64_t> pending_;
    std::map<int64_t, Request> reqs_;
    int64_t next_id_ = 1;
    bool stop_ = false, hold_ = false;
    std::thread thread_;
    // statistics
    std::vector<float> latency_ms_;
    int64_t frames_ = 0, rois_ = 0, launches_ = 0, waits_ = 0;
    std::atomic<int64_t> graphs_{0};  // counted by GraphFor, which runs without the lock
    double t_first_ = -1, t_last_ = 0;
    std::string error_;
};

}  // namespace qtrk
