// ResultManager (see result_manager.h). Behaviour follows cputrack/ResultManager.cpp; where the
// reference indexes out of range (an unknown bead index, a read past the frames held, a removed
// bead, frames evicted before they were processed) this version bounds the access instead, and
// the binary header's data offset is a 32-bit int at byte 12 (the reference writes a C `long`
// there, which is 4 bytes on the Windows builds the format was made for).
#include "result_manager.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <stdexcept>

#include "tracker.h"

namespace {
constexpr int kBinFileVersion = 3;  // ResultManager.cpp:5
}

ResultManager::ResultManager(const char *outfile, const char *frameinfo, const ResultManagerConfig &cfg,
                             std::vector<std::string> colnames)
    : cfg_(cfg), out_file_(outfile ? outfile : ""), info_file_(frameinfo ? frameinfo : ""),
      names_(std::move(colnames))
{
    if (cfg_.numBeads < 0 || cfg_.numFrameInfoColumns < 0) throw std::invalid_argument("negative bead/column count");
    if (!out_file_.empty()) std::remove(out_file_.c_str());
    if (!info_file_.empty()) std::remove(info_file_.c_str());
    names_.resize(cfg_.numFrameInfoColumns);
    if (cfg_.binaryOutput) WriteBinaryHeader();
    thread_ = std::thread([this] { Loop(); });
}

ResultManager::~ResultManager()
{
    quit_ = true;
    if (thread_.joinable()) thread_.join();
}

// Header (ResultManager.cpp:49-75): version, numBeads, numFrameInfoColumns, offset of the
// first frame record, then the column names, each NUL-terminated.
void ResultManager::WriteBinaryHeader()
{
    if (out_file_.empty()) return;
    FILE *f = std::fopen(out_file_.c_str(), "wb");
    if (!f) throw std::runtime_error("Unable to open file " + out_file_);
    int32_t head[4] = {kBinFileVersion, cfg_.numBeads, cfg_.numFrameInfoColumns, 0};
    int32_t offset = (int32_t)sizeof(head);
    for (const std::string &n : names_) offset += (int32_t)n.size() + 1;
    head[3] = offset;
    std::fwrite(head, sizeof(head), 1, f);
    for (const std::string &n : names_) std::fwrite(n.c_str(), n.size() + 1, 1, f);
    std::fclose(f);
}

void ResultManager::SetTracker(qtrk::Tracker *t)
{
    std::lock_guard<std::mutex> lk(trk_mu_);
    trk_ = t;
}

// CheckResultSpace, ResultManager.cpp:339-354.
bool ResultManager::Reserve(int fr)
{
    if (fr < cnt_.startFrame) return false;            // already removed
    if (fr > cnt_.processedFrames + 20000) return false;  // suspiciously large frame number
    while (fr >= cnt_.startFrame + (int)frames_.size())
        frames_.emplace_back(new Frame(cfg_.numBeads, cfg_.numFrameInfoColumns));
    return true;
}

// StoreResult, ResultManager.cpp:82-111: ROI-centred, offset and scaled position; a frame is
// processed when all beads are in, or when more than 1000 captured frames lie beyond it.
void ResultManager::StoreLocked(const LocalizationResult &r, int roi_w, int roi_h)
{
    const int bead = r.job.zlutIndex;
    if (!Reserve((int)r.job.frame) || bead < 0 || bead >= cfg_.numBeads) {
        cnt_.lostFrames++;
        return;
    }
    LocalizationResult s = r;
    s.pos.x = ((s.pos.x - roi_w * 0.5f) + cfg_.offset.x) * cfg_.scaling.x;
    s.pos.y = ((s.pos.y - roi_h * 0.5f) + cfg_.offset.y) * cfg_.scaling.y;
    s.pos.z = ((s.pos.z - 0.0f) + cfg_.offset.z) * cfg_.scaling.z;
    Frame &fr = *frames_[r.job.frame - cnt_.startFrame];
    fr.results[bead] = s;
    fr.count++;
    while (cnt_.processedFrames - cnt_.startFrame < (int)frames_.size()) {
        const Frame &p = *frames_[cnt_.processedFrames - cnt_.startFrame];
        if (!(p.count == cfg_.numBeads || cnt_.capturedFrames - cnt_.processedFrames > 1000)) break;
        if (p.count < cfg_.numBeads) cnt_.lostFrames++;
        cnt_.processedFrames++;
    }
    cnt_.localizationsDone++;
}

// WriteBinaryResults, ResultManager.cpp:113-138: per frame the frame number (uint32), the
// timestamp (double), the frame-info columns (float), then all beads' positions (3 floats),
// all errors (int32) and all image means (float).
void ResultManager::WriteBinary()
{
    if (out_file_.empty()) return;
    FILE *f = std::fopen(out_file_.c_str(), "ab");
    if (!f) {
        cnt_.fileError++;
        return;
    }
    const int nb = cfg_.numBeads;
    std::vector<uint8_t> rec;
    for (int j = cnt_.lastSaveFrame; j < cnt_.processedFrames; j++) {
        const Frame &fr = *frames_[j - cnt_.startFrame];
        rec.resize(4 + 8 + 4 * cfg_.numFrameInfoColumns + (size_t)nb * 20);
        uint8_t *o = rec.data();
        const uint32_t fj = (uint32_t)j;
        std::memcpy(o, &fj, 4), o += 4;
        std::memcpy(o, &fr.timestamp, 8), o += 8;
        if (cfg_.numFrameInfoColumns) std::memcpy(o, fr.info.data(), 4 * cfg_.numFrameInfoColumns);
        o += 4 * cfg_.numFrameInfoColumns;
        for (int i = 0; i < nb; i++) std::memcpy(o, &fr.results[i].pos, 12), o += 12;
        for (int i = 0; i < nb; i++) std::memcpy(o, &fr.results[i].error, 4), o += 4;
        for (int i = 0; i < nb; i++) std::memcpy(o, &fr.results[i].imageMean, 4), o += 4;
        std::fwrite(rec.data(), rec.size(), 1, f);
    }
    std::fclose(f);
}

// WriteTextResults, ResultManager.cpp:140-166.
void ResultManager::WriteText()
{
    FILE *f = out_file_.empty() ? nullptr : std::fopen(out_file_.c_str(), "a");
    FILE *fi = info_file_.empty() ? nullptr : std::fopen(info_file_.c_str(), "a");
    for (int k = cnt_.lastSaveFrame; k < cnt_.processedFrames; k++) {
        const Frame &fr = *frames_[k - cnt_.startFrame];
        if (f) {
            std::fprintf(f, "%d\t%f\t", k, fr.timestamp);
            for (int i = 0; i < cfg_.numBeads; i++) {
                const vector3f &p = fr.results[i].pos;
                std::fprintf(f, "%.7f\t%.7f\t%.7f\t", p.x, p.y, p.z);
            }
            std::fputs("\n", f);
        }
        if (fi) {
            std::fprintf(fi, "%d\t%f\t", k, fr.timestamp);
            for (int i = 0; i < cfg_.numFrameInfoColumns; i++) std::fprintf(fi, "%.7f\t", fr.info[i]);
            std::fputs("\n", fi);
        }
    }
    if (fi) std::fclose(fi);
    if (f) std::fclose(f);
}

void ResultManager::WriteLocked()
{
    if (cfg_.binaryOutput)
        WriteBinary();
    else
        WriteText();
    cnt_.lastSaveFrame = cnt_.processedFrames;
}

// Update, ResultManager.cpp:196-247: fetch, store, write every writeInterval frames, and keep
// at most maxFramesInMemory frames (frames evicted before they completed count as lost and are
// written as they are).
bool ResultManager::Update()
{
    std::unique_lock<std::mutex> tl(trk_mu_);
    if (!trk_) return false;
    LocalizationResult buf[256];
    int n = 0;
    try {
        n = trk_->FetchResults(buf, 256);
    } catch (const std::exception &e) {
        trk_->Warn(std::string("ResultManager: ") + e.what());
        return false;
    }
    const int w = trk_->cfg.base.width, h = trk_->cfg.base.height;
    std::lock_guard<std::mutex> rl(res_mu_);
    for (int i = 0; i < n; i++) StoreLocked(buf[i], w, h);
    tl.unlock();
    MaintainLocked();
    return n > 0;
}

void ResultManager::MaintainLocked()
{
    if (cnt_.processedFrames - cnt_.lastSaveFrame >= cfg_.writeInterval) WriteLocked();
    if (cfg_.maxFramesInMemory > 0 && frames_.size() > cfg_.maxFramesInMemory) {
        const int del = (int)(frames_.size() - cfg_.maxFramesInMemory);
        if (cnt_.processedFrames < cnt_.startFrame + del) {
            const int lost = cnt_.startFrame + del - cnt_.processedFrames;
            cnt_.processedFrames += lost;
            cnt_.lostFrames += lost;
            WriteLocked();
        }
        frames_.erase(frames_.begin(), frames_.begin() + del);
        cnt_.startFrame += del;
    }
}

void ResultManager::Loop()
{
    while (!quit_) {
        if (!Update()) std::this_thread::sleep_for(std::chrono::milliseconds(2));
    }
}

// GetBeadPositions, ResultManager.cpp:264-284 (reads are bounded by the frames held).
int ResultManager::GetBeadPositions(int startfr, int end, int bead, LocalizationResult *dst)
{
    int count = end - startfr;
    std::lock_guard<std::mutex> lk(res_mu_);
    int start = startfr - cnt_.startFrame;
    if (start < 0) start = 0;
    if (count > cnt_.processedFrames - cnt_.startFrame) count = cnt_.processedFrames - cnt_.startFrame;
    if (bead < 0 || bead >= cfg_.numBeads) return 0;
    for (int i = 0; i < count && i + start < (int)frames_.size(); i++) dst[i] = frames_[i + start]->results[bead];
    return count;
}

// GetResults, ResultManager.cpp:319-337: whole frames, all beads, only when processed.
int ResultManager::GetResults(LocalizationResult *dst, int start_frame, int num_frames)
{
    std::lock_guard<std::mutex> lk(res_mu_);
    if (start_frame < cnt_.startFrame || num_frames + start_frame > cnt_.processedFrames) return 0;
    for (int f = 0; f < num_frames; f++) {
        const Frame &fr = *frames_[f + start_frame - cnt_.startFrame];
        for (int j = 0; j < cfg_.numBeads; j++) dst[(size_t)cfg_.numBeads * f + j] = fr.results[j];
    }
    return num_frames;
}

// Flush, ResultManager.cpp:287-313.
void ResultManager::Flush()
{
    {
        std::lock_guard<std::mutex> lk(trk_mu_);
        if (trk_) {
            try {
                trk_->Flush();
            } catch (const std::exception &e) {
                trk_->Warn(std::string("ResultManager: ") + e.what());
            }
        }
    }
    while (Update()) {
    }
    std::lock_guard<std::mutex> lk(res_mu_);
    WriteLocked();
}

RMFrameCounters ResultManager::Counters()
{
    std::lock_guard<std::mutex> lk(res_mu_);
    return cnt_;
}

// StoreFrameInfo, ResultManager.cpp:357-374: the first call for a frame counts it as captured.
void ResultManager::StoreFrameInfo(int frame, double timestamp, const float *cols)
{
    std::lock_guard<std::mutex> lk(res_mu_);
    if (!Reserve(frame)) return;
    Frame &fr = *frames_[frame - cnt_.startFrame];
    if (fr.has_info) return;
    fr.timestamp = timestamp;
    for (int i = 0; i < cfg_.numFrameInfoColumns; i++) fr.info[i] = cols ? cols[i] : 0.0f;
    cnt_.capturedFrames++;
    fr.has_info = true;
}

// RemoveBeadResults, ResultManager.cpp:385-398: the bead's column leaves every frame held and
// each frame's count drops by one; the last column is zero-filled so that every frame keeps
// numBeads entries.
void ResultManager::RemoveBead(int bead)
{
    std::lock_guard<std::mutex> lk(res_mu_);
    if (bead < 0 || bead >= cfg_.numBeads) return;
    for (auto &fp : frames_) {
        fp->count--;
        fp->results.erase(fp->results.begin() + bead);
        fp->results.push_back(LocalizationResult{});
    }
}

void ResultManager::StoreResults(const LocalizationResult *r, int n, int roi_w, int roi_h)
{
    std::lock_guard<std::mutex> lk(res_mu_);
    for (int i = 0; i < n; i++) StoreLocked(r[i], roi_w, roi_h);
    MaintainLocked();
}
