// ResultManager: per-frame, per-bead binning of localization results with periodic file
// output (cputrack/ResultManager.h:10-69, cputrack/ResultManager.cpp). A thread fetches the
// attached tracker's results; frames are complete when every bead has a result, or are given
// up as lost once more than 1000 captured frames lie beyond them.
#pragma once
#include <atomic>
#include <cstdint>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "qtrk_c_api.h"

namespace qtrk {
class Tracker;
}

struct ResultManager {
    ResultManager(const char *outfile, const char *frameinfo, const ResultManagerConfig &cfg,
                  std::vector<std::string> colnames);
    ~ResultManager();

    void SetTracker(qtrk::Tracker *t);
    int GetBeadPositions(int start_frame, int end_frame, int bead, LocalizationResult *dst);
    int GetResults(LocalizationResult *dst, int start_frame, int num_frames);
    void Flush();
    RMFrameCounters Counters();
    void StoreFrameInfo(int frame, double timestamp, const float *cols);
    void RemoveBead(int bead);
    void StoreResults(const LocalizationResult *r, int n, int roi_w, int roi_h);
    const ResultManagerConfig &Config() const { return cfg_; }

  private:
    struct Frame {
        Frame(int beads, int cols) : results(beads), info(cols) {}
        std::vector<LocalizationResult> results;
        std::vector<float> info;
        int count = 0;
        double timestamp = 0;
        bool has_info = false;
    };

    bool Reserve(int frame);                                          // (resultMutex held)
    void StoreLocked(const LocalizationResult &r, int roi_w, int roi_h);  // (resultMutex held)
    void WriteLocked();                                               // (resultMutex held)
    void MaintainLocked();  // periodic write and eviction (resultMutex held)
    void WriteBinary();
    void WriteText();
    void WriteBinaryHeader();
    bool Update();
    void Loop();

    ResultManagerConfig cfg_;
    std::string out_file_, info_file_;
    std::vector<std::string> names_;
    std::deque<std::unique_ptr<Frame>> frames_;
    RMFrameCounters cnt_{};
    std::mutex res_mu_, trk_mu_;
    qtrk::Tracker *trk_ = nullptr;
    std::atomic<bool> quit_{false};
    std::thread thread_;
};
