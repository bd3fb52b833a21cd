// Real-time request loop (see serve.h).
#include "serve.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <stdexcept>
#include <string>
#include <tuple>

#include "kernels.h"

namespace qtrk {

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

int pdt_bytes(int pdt) { return pdt == 0 ? 1 : (pdt == 1 ? 2 : 4); }

uint64_t graph_key(int inst, int bucket, int bands, int pdt, int mode, int smem)
{
    // instance (8 bits) | bucket (14) | bands - 1 (2) | pdt (2) | mode bits folded (20) | smem / 16 (18)
    return ((uint64_t)(inst & 0xff) << 56) | ((uint64_t)(bucket & 0x3fff) << 42) | ((uint64_t)((bands - 1) & 3) << 40) |
           ((uint64_t)(pdt & 3) << 38) | ((uint64_t)((mode ^ (mode >> 20)) & 0xfffff) << 18) |
           (uint64_t)((smem >> 4) & 0x3ffff);
}

}  // namespace

Server::Server(int device, int64_t memory_budget) : device_(device)
{
    ck(cudaSetDevice(device_), "cudaSetDevice");
    const size_t per_lane = kLaneBytes + (size_t)kMaxLaneRois * (8 + sizeof(LocalizationJob) + sizeof(LocalizationResult));
    int nlanes = (int)std::max<int64_t>(1, memory_budget / (int64_t)per_lane);
    nlanes = std::min(nlanes, 16);
    lanes_.resize(nlanes);  // never resized again: args[] point into the lanes
    try {
        for (Lane &l : lanes_) {
            ck(cudaStreamCreateWithFlags(&l.stream, cudaStreamNonBlocking), "cudaStreamCreate");
            ck(cudaEventCreateWithFlags(&l.done, cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaStreamCreateWithFlags(&l.copy_stream, cudaStreamNonBlocking), "cudaStreamCreate");
            for (cudaEvent_t &e : l.band_done) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
            ck(cudaMalloc(&l.d_pix, kLaneBytes), "cudaMalloc(lane pixels)");
            ck(cudaMalloc(&l.d_off, sizeof(int64_t) * kMaxLaneRois), "cudaMalloc");
            ck(cudaMalloc(&l.d_jobs, sizeof(LocalizationJob) * kMaxLaneRois), "cudaMalloc");
            ck(cudaMalloc(&l.d_res, sizeof(LocalizationResult) * kMaxLaneRois), "cudaMalloc");
            ck(cudaHostAlloc(&l.h_off, sizeof(int64_t) * kMaxLaneRois, cudaHostAllocDefault), "cudaHostAlloc");
            ck(cudaHostAlloc(&l.h_jobs, sizeof(LocalizationJob) * kMaxLaneRois, cudaHostAllocDefault), "cudaHostAlloc");
            ck(cudaHostAlloc(&l.h_res, sizeof(LocalizationResult) * kMaxLaneRois, cudaHostAllocDefault),
               "cudaHostAlloc");
            l.args[0] = &l.P;
            l.args[1] = &l.a_pix;
            l.args[2] = &l.a_pitch;
            l.args[3] = &l.a_stride;
            l.args[4] = &l.a_off;
            l.args[5] = &l.a_jobs;
            l.args[6] = &l.a_count;
            l.args[7] = &l.a_res;
        }
        ck(prepare_kernels(device_), "prepare_kernels");
    } catch (...) {
        Release();
        throw;
    }
    thread_ = std::thread([this] { Run(); });
}

Server::~Server()
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    if (thread_.joinable()) thread_.join();
    Release();
}

void Server::Release()
{
    cudaSetDevice(device_);
    for (Lane &l : lanes_) {
        if (l.stream) cudaStreamSynchronize(l.stream);
        if (l.copy_stream) cudaStreamSynchronize(l.copy_stream);
        for (auto &kv : l.graphs) {
            cudaGraphExecDestroy(kv.second.exec);
            cudaGraphDestroy(kv.second.graph);
        }
        l.graphs.clear();
        cudaFree(l.d_pix);
        cudaFree(l.d_off);
        cudaFree(l.d_jobs);
        cudaFree(l.d_res);
        cudaFreeHost(l.h_off);
        cudaFreeHost(l.h_jobs);
        cudaFreeHost(l.h_res);
        if (l.done) cudaEventDestroy(l.done);
        for (cudaEvent_t e : l.band_done)
            if (e) cudaEventDestroy(e);
        if (l.copy_stream) cudaStreamDestroy(l.copy_stream);
        if (l.stream) cudaStreamDestroy(l.stream);
        l = Lane();
    }
}

int Server::Attach(Tracker *t)
{
    if (!t) throw std::invalid_argument("null instance");
    if (t->device() != device_) throw std::invalid_argument("instance runs on another GPU than the server");
    std::lock_guard<std::mutex> lk(mu_);
    if (inst_.size() >= 255) throw std::invalid_argument("too many instances");
    inst_.push_back(t);
    return (int)inst_.size() - 1;
}

// The valid ROIs of the frame (QueuedTracker::ScheduleFrame's rule, QueuedTracker.cpp:91-111:
// ROIs outside the frame are skipped, zlutIndex = i + job.zlutIndex) and the band that holds them.
int64_t Server::Submit(int instance, const void *frame, int pitch, int width, int height, const ROIPosition *pos, int n,
                       int pdt, const LocalizationJob *job)
{
    const double t_entry = now_s();
    if (!frame || !job || (n > 0 && !pos) || pdt < 0 || pdt > 2) throw std::invalid_argument("bad argument");
    Tracker *t;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (instance < 0 || instance >= (int)inst_.size()) throw std::invalid_argument("unknown instance");
        t = inst_[instance];
    }
    const int W = t->cfg.base.width, H = t->cfg.base.height, bpp = pdt_bytes(pdt);
    Request r;
    r.inst = instance;
    r.pdt = pdt;
    r.frame = static_cast<const uint8_t *>(frame);
    r.pitch = pitch;
    int minx = width, miny = height, maxx = 0, maxy = 0;
    std::vector<int> ok;
    for (int i = 0; i < n; i++) {
        const ROIPosition &p = pos[i];
        if (p.x < 0 || p.y < 0 || p.x + W > width || p.y + H > height) continue;
        ok.push_back(i);
        minx = std::min(minx, p.x);
        miny = std::min(miny, p.y);
        maxx = std::max(maxx, p.x + W);
        maxy = std::max(maxy, p.y + H);
    }
    if ((int)ok.size() > kMaxLaneRois) throw std::invalid_argument("more ROIs in one frame than a lane holds (8192)");
    if (!ok.empty()) {
        r.x0 = minx;
        r.y0 = miny;
        r.w = maxx - minx;
        r.h = maxy - miny;
        const size_t band = (size_t)r.h * (((size_t)r.w * bpp + 15) & ~(size_t)15);
        if (band > kLaneBytes) throw std::invalid_argument("the frame band holding the ROIs exceeds a lane (48 MiB)");
    } else {
        r.x0 = r.y0 = r.w = r.h = 0;
    }
    r.offs.reserve(ok.size());
    r.jobs.reserve(ok.size());
    for (int i : ok) {
        // (x, y) inside the band, packed; turned into byte offsets at launch (band pitch known then)
        r.offs.push_back(((int64_t)(pos[i].y - r.y0) << 32) | (int64_t)(pos[i].x - r.x0));
        LocalizationJob j = *job;
        j.zlutIndex = i + job->zlutIndex;
        r.jobs.push_back(j);
    }
    std::lock_guard<std::mutex> lk(mu_);
    r.id = next_id_++;
    r.t_submit = t_entry;
    if (t_first_ < 0) t_first_ = r.t_submit;
    bool lane_free = false;
    for (const Lane &l : lanes_) lane_free |= !l.busy;
    if (!lane_free || !pending_.empty()) waits_++;
    if (r.offs.empty()) {  // nothing to localize: complete at once
        r.done = true;
        r.t_done = r.t_submit;
        const int64_t id = r.id;
        reqs_.emplace(id, std::move(r));
        return id;
    }
    const int64_t id = r.id;
    reqs_.emplace(id, std::move(r));
    pending_.push_back(id);
    cv_.notify_all();
    return id;
}

int Server::Poll(int64_t id, LocalizationResult *out, int max)
{
    std::lock_guard<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) return -2;
    Request &r = it->second;
    if (!r.done) return -1;
    const int n = std::min((int)r.results.size(), std::max(max, 0));
    if (out && n) std::memcpy(out, r.results.data(), sizeof(LocalizationResult) * n);
    const bool failed = r.failed;
    reqs_.erase(it);
    return failed ? -3 : n;
}

void Server::ResetStats()
{
    std::lock_guard<std::mutex> lk(mu_);
    latency_ms_.clear();
    frames_ = rois_ = launches_ = waits_ = 0;
    t_first_ = -1;
    t_last_ = 0;
}

void Server::Hold(bool hold)
{
    {
        std::lock_guard<std::mutex> lk(mu_);
        hold_ = hold;
    }
    cv_.notify_all();
}

std::string Server::LastError()
{
    std::lock_guard<std::mutex> lk(mu_);
    return error_;
}

QTrkB200ServeStats Server::Stats()
{
    std::lock_guard<std::mutex> lk(mu_);
    QTrkB200ServeStats s;
    std::memset(&s, 0, sizeof(s));
    s.frames = frames_;
    s.rois = rois_;
    s.launches = launches_;
    s.graphs = graphs_;
    s.waits_for_memory = waits_;
    s.lanes = (int)lanes_.size();
    s.elapsed_s = t_first_ >= 0 ? t_last_ - t_first_ : 0.0;
    if (!latency_ms_.empty()) {
        std::vector<float> l = latency_ms_;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return (double)l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
        s.p50_ms = pct(0.5);
        s.p99_ms = pct(0.99);
        s.max_ms = l.back();
    }
    return s;
}

// A graph per (lane, instance, bucket, parameters): the localization kernel over `bucket` ROIs
// followed by the copy of their results to the lane's pinned buffer. Built node by node (not
// captured) so that the kernel node's function and shared memory are the ones launch_localize
// uses; each replay patches the node's arguments and grid.
// The graph of one launch: for each row band, a wait for that band's copy (banded batches only)
// and the localization kernel over the band's ROIs, then the copy of all results to the host.
// Grids and arguments are patched into the kernel nodes at each replay.
Server::Graph &Server::GraphFor(Lane &lane, int inst, int bucket, int bands, const TrackParams &P)
{
    const uint64_t key = graph_key(inst, bucket, bands, P.pdt, P.mode, P.smem_bytes);
    auto it = lane.graphs.find(key);
    if (it != lane.graphs.end()) return it->second;
    cudaGraph_t g = nullptr;
    ck(cudaGraphCreate(&g, 0), "cudaGraphCreate");
    Graph gr;
    gr.bands = bands;
    try {
        cudaKernelNodeParams kp;
        localize_node(P, bucket, kp);
        lane.P = P;
        lane.a_pix = lane.d_pix;
        lane.a_pitch = 16;
        lane.a_stride = 0;
        lane.a_off = lane.d_off;
        lane.a_jobs = lane.d_jobs;
        lane.a_count = bucket;
        lane.a_res = lane.d_res;
        kp.kernelParams = lane.args;
        cudaGraphNode_t prev = nullptr;
        for (int b = 0; b < bands; b++) {
            if (bands > 1) {
                cudaGraphNode_t wait;
                ck(cudaGraphAddEventWaitNode(&wait, g, prev ? &prev : nullptr, prev ? 1 : 0, lane.band_done[b]),
                   "cudaGraphAddEventWaitNode");
                prev = wait;
            }
            ck(cudaGraphAddKernelNode(&gr.kernel[b], g, prev ? &prev : nullptr, prev ? 1 : 0, &kp),
               "cudaGraphAddKernelNode");
            prev = gr.kernel[b];
        }
        cudaGraphNode_t copy;
        ck(cudaGraphAddMemcpyNode1D(&copy, g, &prev, 1, lane.h_res, lane.d_res, sizeof(LocalizationResult) * bucket,
                                    cudaMemcpyDeviceToHost),
           "cudaGraphAddMemcpyNode1D");
        ck(cudaGraphInstantiate(&gr.exec, g, 0), "cudaGraphInstantiate");
    } catch (...) {
        cudaGraphDestroy(g);
        throw;
    }
    gr.graph = g;  // kept: exec-node updates name the node of the graph the exec came from
    graphs_++;
    return lane.graphs.emplace(key, gr).first->second;
}

// Runs without the server lock: touches only the lane (dispatcher-owned) and the requests'
// immutable submission fields. The requests' row bands are stacked in the lane at one pitch. A
// batch of a few MiB or less is one copy plus a graph replay (kernel + result copy). A larger one
// is split by rows into up to kMaxBands bands of about kBandBytes, copied in order on the lane's
// copy stream, and its graph runs the kernel of band b as soon as band b has arrived, over a
// prefix of the ROIs (in submission order) that lies inside the rows copied so far, so the
// kernels overlap the later copies and only the last band's kernel is left after the batch has
// crossed PCIe. Every ROI is computed the same way in either form.
void Server::LaunchBatch(Lane &lane, Tracker *t, const std::vector<Request *> &batch)
{
    const int pdt = batch[0]->pdt, bpp = pdt_bytes(pdt);
    const int H = t->cfg.base.height;
    int maxw = 0;
    for (Request *r : batch) maxw = std::max(maxw, r->w);
    const size_t pitch = ((size_t)maxw * bpp + 15) & ~(size_t)15;
    // stacked rows: request r at rows [row0[r], row0[r] + h); ROI i ends at row yend[i]
    std::vector<int> row0(batch.size()), yend;
    int rows = 0, k = 0;
    for (size_t q = 0; q < batch.size(); q++) {
        const Request *r = batch[q];
        row0[q] = rows;
        for (size_t i = 0; i < r->offs.size(); i++) {
            const int64_t ry = r->offs[i] >> 32, rx = r->offs[i] & 0xffffffff;
            lane.h_off[k] = (int64_t)rows * (int64_t)pitch + ry * (int64_t)pitch + rx * bpp;
            lane.h_jobs[k] = r->jobs[i];
            yend.push_back(rows + (int)ry + H);
            k++;
        }
        rows += r->h;
    }
    // bands: [m[b], m[b+1]) of the ROIs, rows [R[b], R[b+1]) of the stack
    int nb = (int)std::min<size_t>(kMaxBands, std::max<size_t>(1, (size_t)rows * pitch / kBandBytes));
    std::vector<int> m(1, 0), R(1, 0);
    for (int b = 1; b < nb && m.back() < k; b++) {
        const int target = std::max((int)((int64_t)k * b / nb), m.back() + 1);
        int rb = R.back();
        for (int i = m.back(); i < target; i++) rb = std::max(rb, yend[i]);
        int mb = target;
        while (mb < k && yend[mb] <= rb) mb++;
        if (mb >= k || rb >= rows) break;  // what is left is the last band
        m.push_back(mb);
        R.push_back(rb);
    }
    m.push_back(k);
    R.push_back(rows);
    nb = (int)m.size() - 1;
    cudaStream_t cs = nb > 1 ? lane.copy_stream : lane.stream;
    for (int b = 0; b < nb; b++) {
        // the rows [R[b], R[b+1]) of every request that has some
        for (size_t q = 0; q < batch.size(); q++) {
            const Request *r = batch[q];
            const int lo = std::max(R[b], row0[q]), hi = std::min(R[b + 1], row0[q] + r->h);
            if (lo >= hi) continue;
            ck(cudaMemcpy2DAsync(lane.d_pix + (size_t)lo * pitch, pitch,
                                 r->frame + (size_t)(r->y0 + lo - row0[q]) * r->pitch + (size_t)r->x0 * bpp,
                                 (size_t)r->pitch, (size_t)r->w * bpp, (size_t)(hi - lo), cudaMemcpyHostToDevice, cs),
               "H2D frame band");
        }
        if (b == 0) {
            ck(cudaMemcpyAsync(lane.d_off, lane.h_off, sizeof(int64_t) * k, cudaMemcpyHostToDevice, cs), "H2D offsets");
            ck(cudaMemcpyAsync(lane.d_jobs, lane.h_jobs, sizeof(LocalizationJob) * k, cudaMemcpyHostToDevice, cs),
               "H2D jobs");
        }
        if (nb > 1) ck(cudaEventRecord(lane.band_done[b], cs), "cudaEventRecord");
    }
    TrackParams P = t->AcquireLaunch(pdt, lane.stream);
    P.mode &= ~(kLT_ZMatchBF16 | kLT_ZMatchTF32 | kLT_JointRefine);  // the graph holds the localization kernel alone
    int bucket = 32;
    while (bucket < k) bucket <<= 1;
    Graph &g = GraphFor(lane, batch[0]->inst, bucket, nb, P);
    lane.P = P;
    lane.a_pix = lane.d_pix;
    lane.a_pitch = (int)pitch;
    lane.a_stride = 0;
    for (int b = 0; b < nb; b++) {
        lane.a_off = lane.d_off + m[b];
        lane.a_jobs = lane.d_jobs + m[b];
        lane.a_count = m[b + 1] - m[b];
        lane.a_res = lane.d_res + m[b];
        cudaKernelNodeParams kp;
        localize_node(P, lane.a_count, kp);  // same function and shared memory as the graph's node
        kp.kernelParams = lane.args;          // the argument values are copied here
        ck(cudaGraphExecKernelNodeSetParams(g.exec, g.kernel[b], &kp), "cudaGraphExecKernelNodeSetParams");
    }
    ck(cudaGraphLaunch(g.exec, lane.stream), "cudaGraphLaunch");
    ck(cudaEventRecord(lane.done, lane.stream), "cudaEventRecord");
    lane.count = k;
}

void Server::Complete(Lane &lane)
{
    const double t = now_s();
    int k = 0;
    for (int64_t id : lane.reqs) {
        auto it = reqs_.find(id);
        if (it == reqs_.end()) continue;
        Request &r = it->second;
        r.results.assign(lane.h_res + k, lane.h_res + k + r.offs.size());
        k += (int)r.offs.size();
        r.done = true;
        r.t_done = t;
        frames_++;
        rois_ += (int64_t)r.offs.size();
        if (latency_ms_.size() < (1u << 22)) latency_ms_.push_back((float)((t - r.t_submit) * 1e3));
    }
    t_last_ = t;
    lane.reqs.clear();
    lane.busy = false;
}

void Server::Run()
{
    cudaSetDevice(device_);
    std::unique_lock<std::mutex> lk(mu_);
    while (!stop_) {
        bool any_busy = false, progressed = false;
        for (Lane &lane : lanes_) {
            if (!lane.busy) continue;
            const cudaError_t q = cudaEventQuery(lane.done);
            if (q == cudaErrorNotReady) {
                any_busy = true;
                continue;
            }
            if (q != cudaSuccess) {
                error_ = cudaGetErrorString(q);
                Fail(lane.reqs);
                lane.reqs.clear();
                lane.busy = false;
            } else {
                Complete(lane);
            }
            progressed = true;
        }
        for (Lane &lane : lanes_) {
            if (lane.busy || pending_.empty() || hold_) continue;
            // continuous batching: the oldest waiting frame plus the following waiting frames of
            // the same instance and pixel type, as long as they fit the lane
            std::vector<Request *> batch;
            size_t rows = 0;
            int maxw = 0, nrois = 0;
            const Request &head = reqs_.at(pending_.front());
            const int inst = head.inst, pdt = head.pdt, bpp = pdt_bytes(pdt);
            for (auto it = pending_.begin(); it != pending_.end();) {
                Request &r = reqs_.at(*it);
                if (r.inst != inst || r.pdt != pdt) {
                    ++it;
                    continue;
                }
                const int nw = std::max(maxw, r.w);
                const size_t pitch = ((size_t)nw * bpp + 15) & ~(size_t)15;
                if (!batch.empty() &&
                    ((rows + r.h) * pitch > kLaneBytes || nrois + (int)r.offs.size() > kMaxLaneRois))
                    break;
                batch.push_back(&r);
                rows += r.h;
                maxw = nw;
                nrois += (int)r.offs.size();
                it = pending_.erase(it);
            }
            Tracker *t = inst_[inst];
            lane.busy = true;
            lane.reqs.clear();
            for (Request *r : batch) lane.reqs.push_back(r->id);
            // Requests in flight are neither erased (Poll forgets done requests only) nor
            // changed until Complete, so the copies are issued without the lock.
            lk.unlock();
            std::string err;
            try {
                LaunchBatch(lane, t, batch);
            } catch (const std::exception &e) {
                err = e.what();
            }
            lk.lock();
            if (!err.empty()) {
                error_ = err;
                cudaStreamSynchronize(lane.stream);  // copies already issued read the frames
                Fail(lane.reqs);
                lane.reqs.clear();
                lane.busy = false;
            } else {
                launches_++;
                any_busy = true;
            }
            progressed = true;
        }
        if (!any_busy && (pending_.empty() || hold_)) {
            // idle: poll for the next frame for a short while before sleeping, so that frames
            // arriving at camera rates do not each pay a thread wake-up
            const double until = now_s() + kIdleSpinSeconds;
            while (!stop_ && (pending_.empty() || hold_) && now_s() < until) {
                lk.unlock();
                std::this_thread::yield();
                lk.lock();
            }
            cv_.wait(lk, [&] { return stop_ || (!pending_.empty() && !hold_); });
        } else if (!progressed) {
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        }
    }
}

void Server::Fail(const std::vector<int64_t> &ids)
{
    const double t = now_s();
    for (int64_t id : ids) {
        auto it = reqs_.find(id);
        if (it == reqs_.end()) continue;
        it->second.done = true;
        it->second.failed = true;
        it->second.t_done = t;
    }
}

}  // namespace qtrk
