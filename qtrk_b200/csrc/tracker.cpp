// Host side of the B200 tracker: configuration, device tables, staging slots, queue.
// See tracker.h for the design; reference behaviour is cited per method.
#include "tracker.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <numeric>
#include <sstream>
#include <stdexcept>
#include <thread>

#include "kernels.h"

namespace qtrk {

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

int pdt_bytes(int pdt) { return pdt == 0 ? 1 : (pdt == 1 ? 2 : 4); }

// Sets the calling thread's current device for the lifetime of the guard.
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev)
    {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard()
    {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

constexpr double kWaitLimitSeconds = 120.0;  // bound on any host wait for the GPU

}  // namespace

// ------------------------------------------------------------------------------------
// Configuration (cputrack/QueuedTracker.cpp:6-21, cputrack/utils.cpp:644-677)
// ------------------------------------------------------------------------------------
int nearest_pow2(int v)
{
    int r = 1;
    while (r < v) r *= 2;
    if (std::fabs((float)(r - v)) < std::fabs((float)(r / 2 - v))) return r;
    return r / 2;
}

QTrkComputedConfig compute_config(const QTrkSettings &s)
{
    QTrkComputedConfig c;
    std::memset(&c, 0, sizeof(c));
    c.base = s;
    const int roi = s.width / 2;
    c.zlut_maxradius = roi * s.zlut_roi_coverage;
    const float zlut_perimeter = 2 * 3.141593f * c.zlut_maxradius;
    c.zlut_angularsteps = (int)(zlut_perimeter * s.zlut_angular_coverage);
    c.zlut_radialsteps = (int)((c.zlut_maxradius - s.zlut_minradius) * s.zlut_radial_coverage);
    c.qi_maxradius = roi * s.qi_roi_coverage;
    const float qi_perimeter = 2 * 3.141593f * c.qi_maxradius;
    c.qi_angstepspq = (int)(qi_perimeter * s.qi_angular_coverage / 4);
    c.qi_radialsteps = (int)((c.qi_maxradius - s.qi_minradius) * s.qi_radial_coverage);
    c.qi_radialsteps = nearest_pow2(c.qi_radialsteps);
    return c;
}

std::vector<float> radial_bin_window(int rsteps)
{
    std::vector<float> w(std::max(rsteps, 0));
    for (int i = 0; i < rsteps; i++) {
        const float x = i / (float)rsteps;
        const float t2 = 0.05f, t1 = 0.01f;
        const float fall = 1.0f - expf(-((1 - x) * (1 - x)) / t2);
        const float rise = 1.0f - expf(-(x * x) / t1);
        w[i] = sqrtf(fall * rise * x * 2);
    }
    return w;
}

// ------------------------------------------------------------------------------------
// Registry for the instance-less reference entry points
// ------------------------------------------------------------------------------------
static std::mutex g_reg_mu;
static std::vector<Tracker *> g_trackers;
static float g_default_of = 1.0f, g_default_gf = 1.0f;

void register_tracker(Tracker *t)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_trackers.push_back(t);
}
void unregister_tracker(Tracker *t)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_trackers.erase(std::remove(g_trackers.begin(), g_trackers.end(), t), g_trackers.end());
}
Tracker *latest_tracker()
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return g_trackers.empty() ? nullptr : g_trackers.back();
}
void for_each_tracker(void (*fn)(Tracker *, void *), void *arg)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    for (Tracker *t : g_trackers) fn(t, arg);
}
static std::vector<int> g_device_list;
void set_device_list(const std::vector<int> &devices)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_device_list = devices;
}
static std::vector<int> device_list()
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    return g_device_list;
}
float default_offset_factor() { return g_default_of; }
float default_gain_factor() { return g_default_gf; }
void set_default_factors(float of, float gf)
{
    std::lock_guard<std::mutex> lk(g_reg_mu);
    g_default_of = of;
    g_default_gf = gf;
}

// ------------------------------------------------------------------------------------
// Tracker
// ------------------------------------------------------------------------------------
void Tracker::CheckCuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) {
        throw std::runtime_error(std::string(what) + ": " + cudaGetErrorName(e) + " (" + cudaGetErrorString(e) + ")");
    }
}

void Tracker::Warn(const std::string &msg)
{
    std::lock_guard<std::mutex> lk(warn_mu_);
    if (warnings_.size() < 65536) warnings_ += msg + "\n";
}

Tracker::Tracker(const QTrkSettings &settings)
{
    cfg = compute_config(settings);
    const QTrkSettings &s = cfg.base;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0)
        throw std::runtime_error(std::string("no usable CUDA device: ") + (e ? cudaGetErrorString(e) : "count is 0"));
    if (s.cuda_device >= 0) {
        device_ = s.cuda_device;
    } else if (s.cuda_device == QTrkCUDA_UseList && !device_list().empty()) {
        device_ = device_list().front();
    } else {
        // QTrkCUDA_UseAll / UseBest / UseList: one instance drives one GPU (the current one);
        // several GPUs are served by one instance per GPU.
        CheckCuda(cudaGetDevice(&device_), "cudaGetDevice");
    }
    if (device_ >= ndev) throw std::runtime_error("cuda_device " + std::to_string(device_) + " does not exist");
    cudaDeviceProp prop;
    CheckCuda(cudaGetDeviceProperties(&prop, device_), "cudaGetDeviceProperties");
    if (prop.major != 10 || prop.minor != 0)
        throw std::runtime_error("libqtrk_b200 is built for sm_100a (B200); device " + std::to_string(device_) +
                                 " is sm_" + std::to_string(prop.major) + std::to_string(prop.minor));
    DeviceGuard dg(device_);
    CheckCuda(prepare_kernels(device_), "prepare_kernels");

    const int W = s.width, H = s.height;
    if (W < 4 || H < 4) throw std::runtime_error("ROI width and height must be at least 4");
    if (s.qi_iterations < 0 || s.qi_iterations > kMaxQIIterations)
        throw std::runtime_error("qi_iterations must be in [0, " + std::to_string(kMaxQIIterations) + "]");
    if (cfg.qi_radialsteps < 1 || cfg.qi_angstepspq < 1) throw std::runtime_error("QI step counts must be >= 1");
    if (cfg.zlut_radialsteps < 1 || cfg.zlut_angularsteps < 1)
        throw std::runtime_error("Z-LUT step counts must be >= 1");

    // ---- parameters and device tables ----
    TrackParams &P = base_;
    std::memset(&P, 0, sizeof(P));
    P.width = W;
    P.height = H;
    P.com_bgcorrection = s.com_bgcorrection;
    P.qi_iterations = s.qi_iterations;
    P.qi_nr = cfg.qi_radialsteps;
    // the QI kernel lays its threads out by shifts: compute_config rounds the step count to a
    // power of two (QueuedTracker.cpp:20), as the reference's FFT length 2 * nr assumes
    if (P.qi_nr < 1 || (P.qi_nr & (P.qi_nr - 1)))
        throw std::runtime_error("QI radial step count must be a power of two");
    P.qi_angpq = cfg.qi_angstepspq;
    P.qi_minr = s.qi_minradius;
    P.qi_maxr = cfg.qi_maxradius;
    {
        // angular samples per iteration, cpu_tracker.cpp:314,356 and 642-657
        float angsteps = cfg.qi_angstepspq / powf(s.qi_angstep_factor, (float)s.qi_iterations);
        for (int k = 0; k < s.qi_iterations; k++) {
            int n = (int)angsteps;
            if (n < 4) n = 4;
            const float angstepf = (float)cfg.qi_angstepspq / n;
            P.qi_nang[k] = n;
            P.qi_inv_nang[k] = 1.0f / (float)n;
            P.qi_stride[k] = (int)angstepf;
            angsteps *= s.qi_angstep_factor;
        }
    }
    P.z_nbins = cfg.zlut_radialsteps;
    P.z_angsteps = cfg.zlut_angularsteps;
    P.z_minr = s.zlut_minradius;
    P.z_maxr = cfg.zlut_maxradius;
    P.g_iterations = s.gauss2D_iterations;
    P.g_sigma = s.gauss2D_sigma;
    offset_factor_ = default_offset_factor();
    gain_factor_ = default_gain_factor();

    // quadrant direction table, cpu_tracker.cpp:294-300
    std::vector<float> qd(2 * P.qi_angpq);
    for (int j = 0; j < P.qi_angpq; j++) {
        const float ang = 0.5 * 3.141593f * (j + 0.5f) / (float)P.qi_angpq;
        qd[2 * j] = cosf(ang);
        qd[2 * j + 1] = sinf(ang);
    }
    // full-circle directions, utils.cpp:278-282
    std::vector<float> zd(2 * P.z_angsteps);
    for (int j = 0; j < P.z_angsteps; j++) {
        const float ang = 2 * 3.141593f * j / (float)P.z_angsteps;
        zd[2 * j] = cosf(ang);
        zd[2 * j + 1] = sinf(ang);
    }
    // FFT twiddles e^{-2 pi i k / L}, k < L/2, L = 2 nr
    const int L = 2 * P.qi_nr;
    std::vector<float> tw(2 * P.qi_nr);
    for (int k = 0; k < P.qi_nr; k++) {
        const double a = -2.0 * M_PI * k / L;
        tw[2 * k] = (float)cos(a);
        tw[2 * k + 1] = (float)sin(a);
    }
    // QI radial bin weights, QueuedCPUTracker.cpp:119
    const std::vector<float> rw = radial_bin_window(P.qi_nr);

    CheckCuda(cudaMalloc(&d_qdirs_, qd.size() * 4), "cudaMalloc(qi dirs)");
    CheckCuda(cudaMalloc(&d_zdirs_, zd.size() * 4), "cudaMalloc(z dirs)");
    CheckCuda(cudaMalloc(&d_tw_, tw.size() * 4), "cudaMalloc(twiddles)");
    CheckCuda(cudaMalloc(&d_qi_rw_, rw.size() * 4), "cudaMalloc(qi weights)");
    CheckCuda(cudaMalloc(&d_zw_, P.z_nbins * 4), "cudaMalloc(z weights)");
    CheckCuda(cudaMemcpy(d_qdirs_, qd.data(), qd.size() * 4, cudaMemcpyHostToDevice), "upload qi dirs");
    CheckCuda(cudaMemcpy(d_zdirs_, zd.data(), zd.size() * 4, cudaMemcpyHostToDevice), "upload z dirs");
    CheckCuda(cudaMemcpy(d_tw_, tw.data(), tw.size() * 4, cudaMemcpyHostToDevice), "upload twiddles");
    CheckCuda(cudaMemcpy(d_qi_rw_, rw.data(), rw.size() * 4, cudaMemcpyHostToDevice), "upload qi weights");
    P.qi_dirs = d_qdirs_;
    P.z_dirs = d_zdirs_;
    P.qi_twiddles = d_tw_;
    P.qi_rweights = d_qi_rw_;

    TrackParams probe = Params(2);
    if (probe.smem_bytes > 227 * 1024)
        throw std::runtime_error("ROI of " + std::to_string(W) + "x" + std::to_string(H) +
                                 " pixels does not fit in one CTA's shared memory");

    CheckCuda(zmatch_prepare_kernel_attrs(), "zmatch kernel attributes");
    CheckCuda(cudaHostAlloc((void **)&h_err_, sizeof(unsigned), cudaHostAllocMapped), "cudaHostAlloc(error word)");
    *h_err_ = 0;
    CheckCuda(cudaHostGetDevicePointer((void **)&d_err_, h_err_, 0), "cudaHostGetDevicePointer");
    CheckCuda(cudaStreamCreateWithFlags(&lut_stream_, cudaStreamNonBlocking), "cudaStreamCreate(lut)");
    CheckCuda(cudaEventCreateWithFlags(&lut_ready_, cudaEventDisableTiming), "cudaEventCreate");
    CheckCuda(cudaEventCreateWithFlags(&noalloc_order_, cudaEventDisableTiming), "cudaEventCreate");
    CheckCuda(cudaStreamCreateWithFlags(&lut_copy_stream_, cudaStreamNonBlocking), "cudaStreamCreate(lut copy)");
    for (int b = 0; b < 2; b++) {
        CheckCuda(cudaEventCreateWithFlags(&lut_stage_free_[b], cudaEventDisableTiming), "cudaEventCreate");
        CheckCuda(cudaEventCreateWithFlags(&lut_copy_done_[b], cudaEventDisableTiming), "cudaEventCreate");
    }
    CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
    AllocateSlots();
    register_tracker(this);
}

Tracker::~Tracker()
{
    unregister_tracker(this);
    DeviceGuard dg(device_);
    {
        std::unique_lock<std::mutex> lk(mu_);
        try {
            DrainAllLocked(lk);
        } catch (...) {
        }
    }
    if (lut_stream_) cudaStreamSynchronize(lut_stream_);
    for (Slot &s : slots_) {
        if (s.stream) cudaStreamSynchronize(s.stream);
        cudaFreeHost(s.h_pix);
        cudaFreeHost(s.h_jobs);
        cudaFreeHost(s.h_res);
        cudaFreeHost(s.h_off);
        cudaFree(s.d_pix);
        cudaFree(s.d_jobs);
        cudaFree(s.d_res);
        cudaFree(s.d_off);
        cudaFree(s.d_zprof);
        cudaFree(s.d_zprof_bf16);
        cudaFreeHost(s.h_perm);
        cudaFree(s.d_perm);
        cudaFreeHost(s.h_tiles);
        cudaFree(s.d_tiles);
        if (s.ev_start) cudaEventDestroy(s.ev_start);
        if (s.ev_done) cudaEventDestroy(s.ev_done);
        if (s.stream) cudaStreamDestroy(s.stream);
    }
    for (int b = 0; b < 2; b++) {
        cudaFreeHost(h_lut_stage_[b]);
        cudaFree(d_lut_stage_[b]);
        if (lut_stage_free_[b]) cudaEventDestroy(lut_stage_free_[b]);
        if (lut_copy_done_[b]) cudaEventDestroy(lut_copy_done_[b]);
    }
    cudaFree(d_qdirs_);
    cudaFree(d_zdirs_);
    cudaFree(d_tw_);
    cudaFree(d_qi_rw_);
    cudaFree(d_zw_);
    cudaFree(d_lut_);
    cudaFree(d_cmp_);
    cudaFree(d_calib_off_);
    cudaFree(d_calib_gain_);
    cudaFree(d_zbias_);
    cudaFree(d_lut_bf16_);
    cudaFree(d_lut_norm_);
    cudaFree(d_lut_t_);
    cudaFree(d_dev_zprof_);
    cudaFree(d_dev_zprof_bf16_);
    cudaFreeHost(h_err_);
    if (lut_ready_) cudaEventDestroy(lut_ready_);
    if (noalloc_order_) cudaEventDestroy(noalloc_order_);
    if (lut_stream_) cudaStreamDestroy(lut_stream_);
    if (lut_copy_stream_) cudaStreamDestroy(lut_copy_stream_);
}

TrackParams Tracker::Params(int pdt) const
{
    TrackParams P = base_;
    P.pdt = pdt;
    P.mode = mode_;
    P.lut = d_lut_;
    P.lut_count = lut_count_;
    P.lut_planes = lut_planes_;
    P.lut_t = lut_t_stale_ ? nullptr : d_lut_t_;
    P.lut_t_pitch = lut_t_pitch(lut_planes_);
    P.z_weights = have_zw_ ? d_zw_ : nullptr;
    P.cmp_scores = cmp_enabled_ ? d_cmp_ : nullptr;
    P.zbias = d_zbias_;
    P.zbias_w = zbias_w_;
    P.zbias_count = zbias_count_;
    P.calib_offset = d_calib_off_;
    P.calib_gain = d_calib_gain_;
    P.calib_count = (d_calib_off_ || d_calib_gain_) ? calib_count_ : 0;
    P.offset_factor = offset_factor_;
    P.gain_factor = gain_factor_;
    P.err_flag = d_err_;
    plan_smem(P);
    return P;
}

TrackParams Tracker::LaunchParams(int pdt)
{
    if (d_lut_ && d_lut_t_ && lut_t_stale_) {
        CheckCuda(launch_transpose_lut(d_lut_, lut_count_, lut_planes_, cfg.zlut_radialsteps, lut_t_pitch(lut_planes_),
                                       d_lut_t_, lut_stream_),
                  "LUT transpose");
        launches_++;
        CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
        lut_t_stale_ = false;
    }
    return Params(pdt);
}

// The adjoint of the Z match (see adjoint.cu): cost and gradients of `count` device-resident ROIs
// at device positions xyz against the instance's LUT, on the caller's stream.
int Tracker::ZLUTCostGradient(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                              const float *d_xyz, const int *d_beads, float *d_cost, float *d_grad, float *d_glut,
                              cudaStream_t stream)
{
    if (!d_pixels || !d_xyz || !d_cost || !d_grad || count < 0 || pdt < 0 || pdt > 2) {
        Warn("QTrkB200ZLUTCostGradient: invalid argument");
        return -1;
    }
    if (pitch < cfg.base.width * pdt_bytes(pdt)) {
        Warn("QTrkB200ZLUTCostGradient: pitch smaller than a row");
        return -2;
    }
    DeviceGuard dg(device_);
    TrackParams P;
    {
        std::lock_guard<std::mutex> lk(mu_);
        P = Params(pdt);
    }
    if (!P.lut || P.lut_count <= 0 || P.lut_planes < 2) {
        Warn("QTrkB200ZLUTCostGradient: no Z-LUT set");
        return -3;
    }
    CheckCuda(cudaStreamWaitEvent(stream, lut_ready_, 0), "cudaStreamWaitEvent");
    CheckCuda(launch_zcost_grad(P, static_cast<const uint8_t *>(d_pixels), pitch, roi_stride, count, d_xyz, d_beads,
                                d_cost, d_grad, d_glut, stream),
              "cost gradient launch");
    launches_++;
    return 0;
}

// Z-LUT refinement from a calibration stack (no counterpart in the reference). ROI (plane k, bead b)
// of the stack is at d_stack + (k * beads + b) * roi_stride; its bead position (x, y) comes from
// d_xy [planes][beads][2] or, when that is null, from COM + QI on the GPU (the BuildLUT rule). The
// objective over the LUT L and one z offset per plane (the stage position error, shared by all
// beads) is
//   E = sum_{k,b} cost(x_kb, y_kb, k + d_k, L_b) + smoothness * sum_{b,k} |L_b,k+1 - 2 L_b,k + L_b,k-1|^2,
// cost the radial-profile/LUT cost of the adjoint kernel. Without the smoothness term a LUT
// built from the same stack already minimises the data term exactly (each plane's row absorbs
// its image), so nothing can move; with it, noise and stage errors that make the rows rough are
// traded against the fit. Each iteration: one adjoint launch over the whole stack (cost, d/dz,
// d/dL on the GPU), then on the host a Gauss-Newton step per plane offset (gradient over the
// beads / curvature sum_r w^2 (L_k+1 - L_k)^2, clamped to +-0.5 plane; offsets keep zero mean and
// zero linear trend, the gauge a LUT cannot see), a diagonally preconditioned step on L (0.7 x
// gradient / exact diagonal curvature of data + smoothness terms), renormalisation of every LUT
// row when profiles are normalised, and the LUT upload. cost_history[i] = E before iteration i
// (iterations + 1 values); plane_z[k] = k + d_k.
void Tracker::RefineZLUT(const void *d_stack, int pitch, int64_t roi_stride, int pdt, int beads, int planes,
                         const float *d_xy, int iterations, float smoothness, float *plane_z, float *cost_history)
{
    if (!d_stack || beads <= 0 || planes < 3 || iterations < 0 || pdt < 0 || pdt > 2 || smoothness < 0)
        throw std::invalid_argument("RefineZLUT: invalid argument");
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    const int nb = cfg.zlut_radialsteps;
    TrackParams P;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (!d_lut_ || lut_count_ != beads || lut_planes_ != planes)
            throw std::invalid_argument("RefineZLUT: the instance's Z-LUT must have `beads` x `planes` rows");
        P = Params(pdt);
    }
    if (pitch < cfg.base.width * pdt_bytes(pdt)) throw std::invalid_argument("RefineZLUT: pitch smaller than a row");
    const int n = beads * planes;
    const size_t lsz = (size_t)beads * planes * nb;
    std::vector<float> L(lsz);
    GetRadialZLUT(L.data());
    std::vector<double> w2(nb, 1.0);
    if (P.z_weights) {
        std::vector<float> w(nb);
        CheckCuda(cudaMemcpy(w.data(), P.z_weights, sizeof(float) * nb, cudaMemcpyDeviceToHost), "weights");
        for (int r = 0; r < nb; r++) w2[r] = (double)w[r] * w[r];
    }
    const bool normalize = (P.mode & kLT_NormalizeProfile) != 0;
    float *d_xyz = nullptr, *d_cost = nullptr, *d_grad = nullptr, *d_glut = nullptr;
    int *d_beads = nullptr;
    LocalizationResult *d_res = nullptr;
    cudaStream_t st = nullptr;
    auto release = [&] {
        cudaFree(d_xyz);
        cudaFree(d_cost);
        cudaFree(d_grad);
        cudaFree(d_glut);
        cudaFree(d_beads);
        cudaFree(d_res);
        if (st) cudaStreamDestroy(st);
    };
    std::vector<double> d(planes, 0.0);
    try {
        CheckCuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        CheckCuda(cudaMalloc(&d_xyz, sizeof(float) * 3 * n), "cudaMalloc");
        CheckCuda(cudaMalloc(&d_cost, sizeof(float) * n), "cudaMalloc");
        CheckCuda(cudaMalloc(&d_grad, sizeof(float) * 3 * n), "cudaMalloc");
        CheckCuda(cudaMalloc(&d_glut, sizeof(float) * lsz), "cudaMalloc");
        CheckCuda(cudaMalloc(&d_beads, sizeof(int) * n), "cudaMalloc");
        std::vector<int> hb(n);
        for (int i = 0; i < n; i++) hb[i] = i % beads;
        CheckCuda(cudaMemcpyAsync(d_beads, hb.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st), "upload beads");
        // bead positions
        std::vector<float> xy(2 * (size_t)n);
        if (d_xy) {
            CheckCuda(cudaMemcpyAsync(xy.data(), d_xy, sizeof(float) * 2 * n, cudaMemcpyDeviceToHost, st), "positions");
        } else {
            TrackParams Q = P;
            Q.mode = kLT_QI | (P.mode & kLT_ClearFirstFourPixels);
            Q.qi_rweights = nullptr;  // BuildLUT's QI runs without radial weights (QueuedCPUTracker.cpp:603)
            plan_smem(Q);
            CheckCuda(cudaMalloc(&d_res, sizeof(LocalizationResult) * n), "cudaMalloc");
            CheckCuda(cudaStreamWaitEvent(st, lut_ready_, 0), "cudaStreamWaitEvent");
            CheckCuda(launch_localize(Q, static_cast<const uint8_t *>(d_stack), pitch, roi_stride, nullptr, nullptr, n,
                                      d_res, st),
                      "localize launch");
            launches_++;
            std::vector<LocalizationResult> res(n);
            CheckCuda(cudaMemcpyAsync(res.data(), d_res, sizeof(LocalizationResult) * n, cudaMemcpyDeviceToHost, st),
                      "download positions");
            CheckCuda(cudaStreamSynchronize(st), "positions");
            for (int i = 0; i < n; i++) {
                xy[2 * i] = res[i].pos.x;
                xy[2 * i + 1] = res[i].pos.y;
            }
        }
        CheckCuda(cudaStreamSynchronize(st), "positions");
        std::vector<float> xyz(3 * (size_t)n), cost(n), grad(3 * (size_t)n), glut(lsz);
        std::vector<double> H(lsz), G(lsz);
        for (int it = 0; it <= iterations; it++) {
            for (int k = 0; k < planes; k++)
                for (int b = 0; b < beads; b++) {
                    const int i = k * beads + b;
                    xyz[3 * i] = xy[2 * i];
                    xyz[3 * i + 1] = xy[2 * i + 1];
                    xyz[3 * i + 2] = (float)(k + d[k]);
                }
            CheckCuda(cudaMemcpyAsync(d_xyz, xyz.data(), sizeof(float) * 3 * n, cudaMemcpyHostToDevice, st), "xyz");
            CheckCuda(cudaMemsetAsync(d_glut, 0, sizeof(float) * lsz, st), "clear gradient");
            {
                std::lock_guard<std::mutex> lk(mu_);
                P = Params(pdt);
            }
            CheckCuda(cudaStreamWaitEvent(st, lut_ready_, 0), "cudaStreamWaitEvent");
            CheckCuda(launch_zcost_grad(P, static_cast<const uint8_t *>(d_stack), pitch, roi_stride, n, d_xyz, d_beads,
                                        d_cost, d_grad, d_glut, st),
                      "cost gradient launch");
            launches_++;
            CheckCuda(cudaMemcpyAsync(cost.data(), d_cost, sizeof(float) * n, cudaMemcpyDeviceToHost, st), "cost");
            CheckCuda(cudaMemcpyAsync(grad.data(), d_grad, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost, st), "grad");
            CheckCuda(cudaMemcpyAsync(glut.data(), d_glut, sizeof(float) * lsz, cudaMemcpyDeviceToHost, st), "glut");
            CheckCuda(cudaStreamSynchronize(st), "cost gradient");
            // data term + smoothness term and its gradient / diagonal curvature
            double E = 0;
            for (int i = 0; i < n; i++) E += cost[i];
            std::fill(G.begin(), G.end(), 0.0);
            std::fill(H.begin(), H.end(), 0.0);
            for (int b = 0; b < beads; b++)
                for (int k = 1; k + 1 < planes; k++)
                    for (int r = 0; r < nb; r++) {
                        const size_t i0 = ((size_t)b * planes + k) * nb + r;
                        const double d2 = (double)L[i0 + nb] - 2.0 * L[i0] + L[i0 - nb];
                        E += smoothness * d2 * d2;
                        G[i0 - nb] += 2 * smoothness * d2;
                        G[i0] += -4 * smoothness * d2;
                        G[i0 + nb] += 2 * smoothness * d2;
                        H[i0 - nb] += 2 * smoothness;
                        H[i0] += 8 * smoothness;
                        H[i0 + nb] += 2 * smoothness;
                    }
            if (cost_history) cost_history[it] = (float)E;
            if (it == iterations) break;
            // plane offsets: Gauss-Newton on the data term, gauge-fixed
            std::vector<double> dnew(d);
            for (int k = 0; k < planes; k++) {
                double gk = 0, hk = 0;
                const double z = k + d[k];
                const int iz = std::max(0, std::min(planes - 2, (int)std::floor(z)));
                for (int b = 0; b < beads; b++) {
                    gk += grad[3 * (k * beads + b) + 2];
                    const float *l0 = &L[((size_t)b * planes + iz) * nb];
                    for (int r = 0; r < nb; r++) {
                        const double dl = (double)l0[nb + r] - l0[r];
                        hk += 2 * w2[r] * dl * dl;
                    }
                }
                if (hk > 0) dnew[k] = d[k] - std::max(-0.5, std::min(0.5, gk / hk));
            }
            double sk = 0, skk = 0, sd = 0, skd = 0;
            for (int k = 0; k < planes; k++) {
                sk += k;
                skk += (double)k * k;
                sd += dnew[k];
                skd += k * dnew[k];
            }
            const double den = planes * skk - sk * sk;
            const double slope = den != 0 ? (planes * skd - sk * sd) / den : 0.0, icpt = (sd - slope * sk) / planes;
            for (int k = 0; k < planes; k++) dnew[k] -= icpt + slope * k;
            // LUT step: data curvature from the z each ROI was scored at
            for (int k = 0; k < planes; k++) {
                const double z = k + d[k];
                const int iz = std::max(0, std::min(planes - 2, (int)std::floor(z)));
                const double fz = z - iz;
                for (int b = 0; b < beads; b++) {
                    double *h0 = &H[((size_t)b * planes + iz) * nb];
                    for (int r = 0; r < nb; r++) {
                        h0[r] += 2 * w2[r] * (1 - fz) * (1 - fz);
                        h0[nb + r] += 2 * w2[r] * fz * fz;
                    }
                }
            }
            double hmax = 0;
            for (double h : H) hmax = std::max(hmax, h);
            for (size_t i = 0; i < lsz; i++) {
                const double g = G[i] + glut[i];
                L[i] = (float)(L[i] - 0.7 * g / (H[i] + 1e-6 * hmax + 1e-30));
            }
            if (normalize)
                for (size_t row = 0; row < (size_t)beads * planes; row++) {
                    float *p = &L[row * nb];
                    double m = 0, ss = 0;
                    for (int r = 0; r < nb; r++) m += p[r];
                    m /= nb;
                    for (int r = 0; r < nb; r++) ss += (p[r] - m) * (p[r] - m);
                    const double inv = ss > 0 ? 1.0 / std::sqrt(ss / nb) : 1.0;
                    for (int r = 0; r < nb; r++) p[r] = (float)((p[r] - m) * inv);
                }
            d = dnew;
            {
                std::lock_guard<std::mutex> lk(mu_);
                CheckCuda(cudaMemcpyAsync(d_lut_, L.data(), sizeof(float) * lsz, cudaMemcpyHostToDevice, lut_stream_),
                          "upload Z-LUT");
                tc_lut_stale_ = lut_t_stale_ = true;
                CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
            }
            CheckCuda(cudaStreamSynchronize(lut_stream_), "upload Z-LUT");
        }
    } catch (...) {
        release();
        throw;
    }
    release();
    if (plane_z)
        for (int k = 0; k < planes; k++) plane_z[k] = (float)(k + d[k]);
}

// The adjoint of the 5-parameter Gaussian MLE (see adjoint.cu), on the caller's stream.
int Tracker::GaussianNLLGradient(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                                 const float *d_params, float *d_nll, float *d_grad, cudaStream_t stream)
{
    if (!d_pixels || !d_params || !d_nll || !d_grad || count < 0 || pdt < 0 || pdt > 2) {
        Warn("QTrkB200GaussianNLLGradient: invalid argument");
        return -1;
    }
    if (pitch < cfg.base.width * pdt_bytes(pdt)) {
        Warn("QTrkB200GaussianNLLGradient: pitch smaller than a row");
        return -2;
    }
    DeviceGuard dg(device_);
    TrackParams P;
    {
        std::lock_guard<std::mutex> lk(mu_);
        P = Params(pdt);
    }
    CheckCuda(launch_gauss_nll_grad(P, static_cast<const uint8_t *>(d_pixels), pitch, roi_stride, count, d_params,
                                    d_nll, d_grad, stream),
              "Gaussian NLL gradient launch");
    launches_++;
    return 0;
}

// LT_B200_JointRefine: a joint Gauss-Newton pass follows the Z fit when the mode has one.
bool Tracker::RefineAfterZ(const TrackParams &P)
{
    return (P.mode & kLT_JointRefine) && (P.mode & kLT_LocalizeZ) && P.lut && P.lut_count > 0 && P.lut_planes >= 2;
}

TrackParams Tracker::AcquireLaunch(int pdt, cudaStream_t stream)
{
    std::lock_guard<std::mutex> lk(mu_);
    TrackParams P = LaunchParams(pdt);
    CheckCuda(cudaStreamWaitEvent(stream, lut_ready_, 0), "cudaStreamWaitEvent");
    launches_++;
    return P;
}

void Tracker::AllocateSlots()
{
    const QTrkSettings &s = cfg.base;
    const int nslots = s.numThreads < 1 ? 4 : std::min(s.numThreads, 16);
    const size_t roi_f32 = (size_t)s.width * s.height * 4;
    const size_t budget = 64u << 20;  // pixel bytes per slot
    batch_ = (int)std::max<size_t>(16, std::min<size_t>(4096, budget / roi_f32));
    slot_bytes_ = (size_t)batch_ * roi_f32;
    slots_.resize(nslots);
    for (int i = 0; i < nslots; i++) {
        Slot &sl = slots_[i];
        CheckCuda(cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking), "cudaStreamCreate");
        CheckCuda(cudaEventCreate(&sl.ev_start), "cudaEventCreate");
        CheckCuda(cudaEventCreate(&sl.ev_done), "cudaEventCreate");
        CheckCuda(cudaHostAlloc(&sl.h_pix, slot_bytes_, cudaHostAllocDefault), "cudaHostAlloc(pixels)");
        CheckCuda(cudaMalloc(&sl.d_pix, slot_bytes_), "cudaMalloc(pixels)");
        CheckCuda(cudaHostAlloc(&sl.h_jobs, sizeof(LocalizationJob) * batch_, cudaHostAllocDefault), "cudaHostAlloc");
        CheckCuda(cudaMalloc(&sl.d_jobs, sizeof(LocalizationJob) * batch_), "cudaMalloc");
        CheckCuda(cudaHostAlloc(&sl.h_res, sizeof(LocalizationResult) * batch_, cudaHostAllocDefault), "cudaHostAlloc");
        CheckCuda(cudaMalloc(&sl.d_res, sizeof(LocalizationResult) * batch_), "cudaMalloc");
        CheckCuda(cudaHostAlloc(&sl.h_off, sizeof(int64_t) * batch_, cudaHostAllocDefault), "cudaHostAlloc");
        CheckCuda(cudaMalloc(&sl.d_off, sizeof(int64_t) * batch_), "cudaMalloc");
        free_.push_back(i);
    }
}

bool Tracker::IsPinned(const void *p)
{
    cudaPointerAttributes a;
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return a.type == cudaMemoryTypeHost;
}

void Tracker::CollectLocked()
{
    if (h_err_ && *h_err_) {
        const unsigned e = *h_err_;
        *h_err_ = 0;
        if (e & 3u) Warn("tensor-core Z match: an MMA completion wait timed out; z of the affected ROIs is NaN");
        if (e & 2u)
            Warn("tensor-core Z match: the timed-out MMAs had not finished when their tensor-memory columns were "
                 "released; results of that launch are void");
        if (e & 4u)
            Warn("localization kernel: a staged ROI copy did not arrive within the wait limit; results of that "
                 "launch are void");
    }
    while (!inflight_.empty()) {
        const int idx = inflight_.front();
        Slot &s = slots_[idx];
        const cudaError_t q = cudaEventQuery(s.ev_done);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) {
            Warn(std::string("batch of ") + std::to_string(s.count) + " ROIs failed: " + cudaGetErrorString(q));
        } else {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, s.ev_start, s.ev_done) == cudaSuccess) stats_.gpu_ms += ms;
            stats_.batches++;
            stats_.rois += s.count;
            if (stats_.latency_ms.size() < (1u << 20)) stats_.latency_ms.push_back((float)((now_s() - s.t_submit) * 1e3));
            std::lock_guard<std::mutex> rl(res_mu_);
            for (int i = 0; i < s.count; i++) results_.push_back(s.h_res[i]);
        }
        inflight_.pop_front();
        s.count = 0;
        s.frame = false;
        free_.push_back(idx);
    }
}

int Tracker::AcquireSlotLocked(std::unique_lock<std::mutex> &lk)
{
    const double deadline = now_s() + kWaitLimitSeconds;
    for (;;) {
        CollectLocked();
        if (!free_.empty()) {
            const int i = free_.front();
            free_.pop_front();
            Slot &s = slots_[i];
            s.count = 0;
            s.frame = false;
            return i;
        }
        if (now_s() > deadline) return -1;
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(20));
        lk.lock();
    }
}

void Tracker::SubmitLocked(int idx)
{
    Slot &s = slots_[idx];
    TrackParams P = LaunchParams(s.pdt);
    const size_t roib = (size_t)cfg.base.width * cfg.base.height * pdt_bytes(s.pdt);
    const bool tc = UseTensorCoreMatch();
    int ntiles = 0;
    if (tc) {
        const int nb = cfg.zlut_radialsteps, nbp = zmatch_padded_bins(nb);
        if (!s.d_zprof) {
            CheckCuda(cudaMalloc(&s.d_zprof, sizeof(float) * batch_ * nb), "cudaMalloc(profiles)");
            CheckCuda(cudaMalloc(&s.d_zprof_bf16, sizeof(__nv_bfloat16) * batch_ * 2 * nbp), "cudaMalloc(profiles)");
            CheckCuda(cudaHostAlloc(&s.h_perm, sizeof(int) * batch_, cudaHostAllocDefault), "cudaHostAlloc");
            CheckCuda(cudaMalloc(&s.d_perm, sizeof(int) * batch_), "cudaMalloc");
            CheckCuda(cudaHostAlloc(&s.h_tiles, sizeof(int4) * batch_, cudaHostAllocDefault), "cudaHostAlloc");
            CheckCuda(cudaMalloc(&s.d_tiles, sizeof(int4) * batch_), "cudaMalloc");
        }
        PrepareTensorCoreLUT();
        ntiles = BuildTiles(s.h_jobs, s.count, s.h_perm, s.h_tiles);
        P.zprof_f32 = s.d_zprof;
        P.zprof_bf16 = s.d_zprof_bf16;
        P.zprof_nbp = nbp;
    }
    CheckCuda(cudaStreamWaitEvent(s.stream, lut_ready_, 0), "cudaStreamWaitEvent");
    if (tc) {
        CheckCuda(cudaMemcpyAsync(s.d_perm, s.h_perm, sizeof(int) * s.count, cudaMemcpyHostToDevice, s.stream),
                  "H2D perm");
        CheckCuda(cudaMemcpyAsync(s.d_tiles, s.h_tiles, sizeof(int4) * ntiles, cudaMemcpyHostToDevice, s.stream),
                  "H2D tiles");
    }
    if (!s.frame) {
        CheckCuda(cudaEventRecord(s.ev_start, s.stream), "cudaEventRecord");
        CheckCuda(cudaMemcpyAsync(s.d_pix, s.h_pix, roib * s.count, cudaMemcpyHostToDevice, s.stream), "H2D pixels");
    }
    CheckCuda(cudaMemcpyAsync(s.d_jobs, s.h_jobs, sizeof(LocalizationJob) * s.count, cudaMemcpyHostToDevice, s.stream),
              "H2D jobs");
    if (s.frame)
        CheckCuda(cudaMemcpyAsync(s.d_off, s.h_off, sizeof(int64_t) * s.count, cudaMemcpyHostToDevice, s.stream),
                  "H2D offsets");
    CheckCuda(launch_localize(P, s.d_pix, s.pitch, (int64_t)roib, s.frame ? s.d_off : nullptr, s.d_jobs, s.count,
                              s.d_res, s.stream),
              "localize kernel launch");
    launches_++;
    if (tc) {
        ZMatchParams Q = TensorCoreParams();
        Q.prof_f32 = s.d_zprof;
        Q.prof_bf16 = s.d_zprof_bf16;
        Q.perm = s.d_perm;
        Q.tiles = s.d_tiles;
        Q.count = s.count;
        Q.results = s.d_res;
        CheckCuda(launch_zmatch_tc(Q, ntiles, s.stream), "Z-match kernel launch");
        launches_++;
    }
    if (RefineAfterZ(P)) {
        CheckCuda(launch_joint_refine(P, s.d_pix, s.pitch, (int64_t)roib, s.frame ? s.d_off : nullptr, s.d_jobs,
                                      s.count, s.d_res, s.stream),
                  "joint refine launch");
        launches_++;
    }
    CheckCuda(cudaMemcpyAsync(s.h_res, s.d_res, sizeof(LocalizationResult) * s.count, cudaMemcpyDeviceToHost, s.stream),
              "D2H results");
    CheckCuda(cudaEventRecord(s.ev_done, s.stream), "cudaEventRecord");
    s.t_submit = now_s();
    inflight_.push_back(idx);
}

bool Tracker::UseTensorCoreMatch() const
{
    return (mode_ & (LT_B200_ZMatchBF16 | LT_B200_ZMatchTF32)) && (mode_ & LT_LocalizeZ) && d_lut_ && lut_count_ > 0 &&
           lut_planes_ > 0 && zmatch_supported(cfg.zlut_radialsteps) && !cmp_enabled_;
}

void Tracker::PrepareTensorCoreLUT()
{
    if (!tc_lut_stale_ && d_lut_bf16_) return;
    const int nb = cfg.zlut_radialsteps, nbp = zmatch_padded_bins(nb), pp = zmatch_padded_planes(lut_planes_);
    CheckCuda(cudaStreamSynchronize(lut_stream_), "cudaStreamSynchronize(lut)");
    cudaFree(d_lut_bf16_);
    cudaFree(d_lut_norm_);
    d_lut_bf16_ = nullptr;
    d_lut_norm_ = nullptr;
    tc_lut_count_ = tc_lut_pp_ = tc_lut_nbp_ = 0;
    CheckCuda(cudaMalloc(&d_lut_bf16_, sizeof(__nv_bfloat16) * (size_t)lut_count_ * 2 * pp * nbp),
              "cudaMalloc(BF16 LUT)");
    CheckCuda(cudaMalloc(&d_lut_norm_, sizeof(float) * (size_t)lut_count_ * pp), "cudaMalloc(LUT norms)");
    tc_lut_count_ = lut_count_;
    tc_lut_pp_ = pp;
    tc_lut_nbp_ = nbp;
    CheckCuda(zmatch_prepare_lut(d_lut_, have_zw_ ? d_zw_ : nullptr, lut_count_, lut_planes_, nb, d_lut_bf16_,
                                 d_lut_norm_, lut_stream_),
              "BF16 LUT preparation");
    launches_++;
    CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
    tc_lut_stale_ = false;
}

ZMatchParams Tracker::TensorCoreParams() const
{
    ZMatchParams Q;
    std::memset(&Q, 0, sizeof(Q));
    Q.nb = cfg.zlut_radialsteps;
    Q.nbp = zmatch_padded_bins(Q.nb);
    Q.planes = lut_planes_;
    Q.planes_pad = zmatch_padded_planes(lut_planes_);
    Q.lut_count = lut_count_;
    Q.lut_bf16 = d_lut_bf16_;
    Q.lut_norm = d_lut_norm_;
    Q.lut = d_lut_;
    Q.weights = have_zw_ ? d_zw_ : nullptr;
    Q.error_flag = d_err_;
    Q.tf32 = (mode_ & LT_B200_ZMatchTF32) ? 1 : 0;
    Q.zbias = d_zbias_;
    Q.zbias_w = zbias_w_;
    Q.zbias_count = zbias_count_;
    return Q;
}

// ROIs grouped by bead (stable), cut into tiles of at most 128 ROIs of one bead. ROIs whose
// bead has no LUT form tiles of bead -1 (z = 0, as in the plain path).
int Tracker::BuildTiles(const LocalizationJob *jobs, int count, int *perm, int4 *tiles) const
{
    std::vector<int> order(count);
    for (int i = 0; i < count; i++) order[i] = i;
    auto bead_of = [&](int i) {
        const int b = jobs[i].zlutIndex;
        return (b >= 0 && b < lut_count_) ? b : -1;
    };
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return bead_of(a) < bead_of(b); });
    int nt = 0;
    for (int i = 0; i < count;) {
        const int b = bead_of(order[i]);
        int j = i;
        while (j < count && bead_of(order[j]) == b && j - i < 128) j++;
        tiles[nt++] = make_int4(i, j - i, b, 0);
        i = j;
    }
    std::memcpy(perm, order.data(), sizeof(int) * count);
    return nt;
}

void Tracker::DrainAllLocked(std::unique_lock<std::mutex> &lk)
{
    if (filling_ >= 0) {
        if (slots_[filling_].count > 0) {
            SubmitLocked(filling_);
        } else {
            free_.push_back(filling_);
        }
        filling_ = -1;
    }
    const double deadline = now_s() + kWaitLimitSeconds;
    for (;;) {
        CollectLocked();
        if (inflight_.empty()) return;
        if (now_s() > deadline) throw std::runtime_error("timed out waiting for the GPU to finish queued batches");
        lk.unlock();
        std::this_thread::sleep_for(std::chrono::microseconds(50));
        lk.lock();
    }
}

void Tracker::WaitIdleForReconfigure()
{
    std::unique_lock<std::mutex> lk(mu_);
    DrainAllLocked(lk);
    CheckCuda(cudaStreamSynchronize(lut_stream_), "cudaStreamSynchronize(lut)");
}

// QueuedCPUTracker::SetLocalizationMode waits for idle (QueuedCPUTracker.cpp:513-517).
void Tracker::SetLocalizationMode(LocMode_t mode)
{
    DeviceGuard dg(device_);
    const int unsupported = LT_XCor1D | LT_ZLUTAlign | LT_FourierLUT | LT_LocalizeZWeighted;
    if (mode & unsupported)
        Warn("localization mode bits 0x" + [&] {
            std::ostringstream o;
            o << std::hex << (mode & unsupported);
            return o.str();
        }() + " (XCor1D/ZLUTAlign/FourierLUT/LocalizeZWeighted) are not supported and were ignored");
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    mode_ = mode & ~unsupported;
}

// QueuedCPUTracker::SetPixelCalibrationImages, QueuedCPUTracker.cpp:165-196: per-bead images of
// width*height*zlut_count floats; a null pointer removes that image.
void Tracker::SetPixelCalibrationImages(const float *offset, const float *gain)
{
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    if (lut_count_ <= 0) {
        Warn("SetPixelCalibrationImages needs a Z-LUT (its bead count sizes the images); ignored");
        return;
    }
    const size_t n = (size_t)cfg.base.width * cfg.base.height * lut_count_;
    auto upd = [&](float *&dptr, const float *src) {
        if (src) {
            if (!dptr) CheckCuda(cudaMalloc(&dptr, n * 4), "cudaMalloc(calibration)");
            CheckCuda(cudaMemcpy(dptr, src, n * 4, cudaMemcpyHostToDevice), "upload calibration");
        } else if (dptr) {
            cudaFree(dptr);
            dptr = nullptr;
        }
    };
    upd(d_calib_off_, offset);
    upd(d_calib_gain_, gain);
    calib_count_ = lut_count_;
}

void Tracker::SetPixelCalibrationFactors(float offsetFactor, float gainFactor)
{
    std::lock_guard<std::mutex> lk(mu_);
    offset_factor_ = offsetFactor;
    gain_factor_ = gainFactor;
}

// QueuedCPUTracker::ScheduleLocalization, QueuedCPUTracker.cpp:435-456: the ROI rows are copied
// before returning, so the caller may reuse its buffer at once.
void Tracker::ScheduleLocalization(const void *data, int pitch, int pdt, const LocalizationJob *job)
{
    if (!data || !job) throw std::invalid_argument("ScheduleLocalization: null data or job");
    if (pdt < 0 || pdt > 2) throw std::invalid_argument("ScheduleLocalization: unknown pixel data type");
    DeviceGuard dg(device_);
    const int W = cfg.base.width, H = cfg.base.height;
    const size_t rowb = (size_t)W * pdt_bytes(pdt), roib = rowb * H;
    std::unique_lock<std::mutex> lk(mu_);
    if (filling_ >= 0) {
        Slot &s = slots_[filling_];
        if (s.count > 0 && s.pdt != pdt) {
            SubmitLocked(filling_);
            filling_ = -1;
        }
    }
    if (filling_ < 0) {
        filling_ = AcquireSlotLocked(lk);
        if (filling_ < 0) {
            Warn("ScheduleLocalization: timed out waiting for a free batch slot; job dropped");
            return;
        }
        Slot &s = slots_[filling_];
        s.pdt = pdt;
        s.frame = false;
        s.pitch = (int)rowb;
    }
    Slot &s = slots_[filling_];
    uint8_t *dst = s.h_pix + (size_t)s.count * roib;
    const uint8_t *src = static_cast<const uint8_t *>(data);
    if ((size_t)pitch == rowb) {
        std::memcpy(dst, src, roib);
    } else {
        for (int y = 0; y < H; y++) std::memcpy(dst + y * rowb, src + (size_t)y * pitch, rowb);
    }
    s.h_jobs[s.count] = *job;
    s.count++;
    if (s.count == batch_) {
        SubmitLocked(filling_);
        filling_ = -1;
    }
}

// QueuedTracker::ScheduleFrame, QueuedTracker.cpp:91-111: ROIs outside the frame are skipped,
// zlutIndex = i + job.zlutIndex. Here the frame rows are copied to the device once and the
// kernel crops the ROIs from them (no host-side cropping).
int Tracker::ScheduleFrame(const void *img, int pitch, int width, int height, const ROIPosition *pos, int n, int pdt,
                           const LocalizationJob *job)
{
    if (!img || !job || (n > 0 && !pos)) throw std::invalid_argument("ScheduleFrame: null argument");
    if (pdt < 0 || pdt > 2) throw std::invalid_argument("ScheduleFrame: unknown pixel data type");
    DeviceGuard dg(device_);
    const int W = cfg.base.width, H = cfg.base.height, bpp = pdt_bytes(pdt);
    std::vector<int> idx;
    idx.reserve(n);
    int skipped = 0;
    for (int i = 0; i < n; i++) {
        const ROIPosition &p = pos[i];
        if (p.x < 0 || p.y < 0 || p.x + W > width || p.y + H > height) {
            skipped++;
            continue;
        }
        idx.push_back(i);
    }
    if (skipped) Warn("ScheduleFrame: skipped " + std::to_string(skipped) + " ROI(s) outside the frame");
    if (idx.empty()) return 0;

    // Group ROIs into row bands of at most 32 MiB (or one slot, if smaller); one band keeps the
    // caller's order. The bands' copies run one after another (each waits for the previous one),
    // so every band's kernel overlaps the next band's copy and only the last, small band's kernel
    // is left after the frame has crossed PCIe.
    const size_t band_cap = std::min(slot_bytes_, (size_t)32 << 20);
    int minx = width, maxx = 0;
    for (int i : idx) {
        minx = std::min(minx, pos[i].x);
        maxx = std::max(maxx, pos[i].x + W);
    }
    const size_t dpitch = (((size_t)(maxx - minx) * bpp) + 15) & ~(size_t)15;
    auto span_bytes = [&](int y0, int y1) { return (size_t)(y1 - y0) * dpitch; };
    std::vector<std::vector<int>> bands;
    {
        int y0 = height, y1 = 0;
        for (int i : idx) {
            y0 = std::min(y0, pos[i].y);
            y1 = std::max(y1, pos[i].y + H);
        }
        if (span_bytes(y0, y1) <= band_cap && (int)idx.size() <= batch_) {
            bands.push_back(idx);
        } else {
            std::vector<int> sorted = idx;
            auto by_row = [&](int a, int b) { return pos[a].y < pos[b].y; };
            if (!std::is_sorted(sorted.begin(), sorted.end(), by_row))  // frames are usually listed in scan order
                std::stable_sort(sorted.begin(), sorted.end(), by_row);
            std::vector<int> cur;
            int by0 = 0, by1 = 0;
            for (int i : sorted) {
                if (cur.empty()) {
                    by0 = pos[i].y;
                    by1 = pos[i].y + H;
                    cur.push_back(i);
                    continue;
                }
                const int ny1 = std::max(by1, pos[i].y + H);
                if (span_bytes(by0, ny1) <= band_cap && (int)cur.size() < batch_) {
                    by1 = ny1;
                    cur.push_back(i);
                } else {
                    bands.push_back(cur);
                    cur.assign(1, i);
                    by0 = pos[i].y;
                    by1 = pos[i].y + H;
                }
            }
            if (!cur.empty()) bands.push_back(cur);
        }
    }
    if (span_bytes(0, H) > slot_bytes_) {
        // A single ROI row span does not fit a slot (very wide frame): crop on the host.
        int count = 0;
        for (int i : idx) {
            LocalizationJob j = *job;
            j.zlutIndex = i + job->zlutIndex;
            ScheduleLocalization(static_cast<const uint8_t *>(img) + (size_t)pitch * pos[i].y + (size_t)pos[i].x * bpp,
                                 pitch, pdt, &j);
            count++;
        }
        return count;
    }

    const bool pinned = IsPinned(img);
    std::vector<cudaEvent_t> copies;  // one per band, in order: the copy chain
    std::unique_lock<std::mutex> lk(mu_);
    if (filling_ >= 0) {  // keep FIFO order with earlier single-ROI jobs
        if (slots_[filling_].count > 0)
            SubmitLocked(filling_);
        else
            free_.push_back(filling_);
        filling_ = -1;
    }
    int count = 0;
    for (const std::vector<int> &band : bands) {
        int y0 = height, y1 = 0;
        for (int i : band) {
            y0 = std::min(y0, pos[i].y);
            y1 = std::max(y1, pos[i].y + H);
        }
        const int si = AcquireSlotLocked(lk);
        if (si < 0) {
            Warn("ScheduleFrame: timed out waiting for a free batch slot; ROIs dropped");
            break;
        }
        Slot &s = slots_[si];
        s.frame = true;
        s.pdt = pdt;
        s.pitch = (int)dpitch;
        s.count = (int)band.size();
        for (int k = 0; k < s.count; k++) {
            const int i = band[k];
            s.h_off[k] = (int64_t)(pos[i].y - y0) * (int64_t)dpitch + (int64_t)(pos[i].x - minx) * bpp;
            s.h_jobs[k] = *job;
            s.h_jobs[k].zlutIndex = i + job->zlutIndex;
        }
        CheckCuda(cudaEventRecord(s.ev_start, s.stream), "cudaEventRecord");
        if (!copies.empty()) CheckCuda(cudaStreamWaitEvent(s.stream, copies.back(), 0), "cudaStreamWaitEvent");
        const uint8_t *src = static_cast<const uint8_t *>(img) + (size_t)y0 * pitch + (size_t)minx * bpp;
        CheckCuda(cudaMemcpy2DAsync(s.d_pix, dpitch, src, (size_t)pitch, (size_t)(maxx - minx) * bpp, (size_t)(y1 - y0),
                                    cudaMemcpyHostToDevice, s.stream),
                  "H2D frame rows");
        cudaEvent_t ev;
        CheckCuda(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming), "cudaEventCreate");
        CheckCuda(cudaEventRecord(ev, s.stream), "cudaEventRecord");
        copies.push_back(ev);
        SubmitLocked(si);
        count += s.count;
    }
    lk.unlock();
    // A pinned source is read by DMA after cudaMemcpy2DAsync returns: wait until it has been
    // read so the caller may reuse the frame buffer (pageable sources are staged before return).
    for (cudaEvent_t ev : copies) {
        if (pinned) cudaEventSynchronize(ev);
        cudaEventDestroy(ev);  // a pending event is released once it completes
    }
    return count;
}

void Tracker::ClearResults()
{
    std::lock_guard<std::mutex> rl(res_mu_);
    results_.clear();
}

void Tracker::Flush()
{
    DeviceGuard dg(device_);
    std::lock_guard<std::mutex> lk(mu_);
    if (filling_ >= 0 && slots_[filling_].count > 0) {
        SubmitLocked(filling_);
        filling_ = -1;
    }
}

// QueuedCPUTracker::SetRadialZLUT, QueuedCPUTracker.cpp:364-391: [count][planes][zlut_radialsteps]
// floats, zero-filled when data is null.
void Tracker::SetRadialZLUT(const float *data, int count, int planes)
{
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    cudaFree(d_lut_);
    cudaFree(d_lut_t_);
    cudaFree(d_cmp_);
    d_lut_ = nullptr;
    d_lut_t_ = nullptr;
    d_cmp_ = nullptr;
    // the tensor-core copy was sized for the old LUT: drop it (the next allocating call in a
    // tensor-core mode makes one of the new shape)
    cudaFree(d_lut_bf16_);
    cudaFree(d_lut_norm_);
    d_lut_bf16_ = nullptr;
    d_lut_norm_ = nullptr;
    tc_lut_count_ = tc_lut_pp_ = tc_lut_nbp_ = 0;
    cudaFree(d_zbias_);  // a new LUT drops the bias table, as QueuedCPUTracker.cpp:368-369
    d_zbias_ = nullptr;
    zbias_w_ = zbias_count_ = 0;
    const int res = cfg.zlut_radialsteps;
    const size_t total = (size_t)std::max(count, 0) * std::max(planes, 0) * res;
    if (total > 0) {
        CheckCuda(cudaMalloc(&d_lut_, total * 4), "cudaMalloc(Z-LUT)");
        if (data)
            CheckCuda(cudaMemcpy(d_lut_, data, total * 4, cudaMemcpyHostToDevice), "upload Z-LUT");
        else
            CheckCuda(cudaMemset(d_lut_, 0, total * 4), "clear Z-LUT");
        CheckCuda(cudaMalloc(&d_lut_t_, (size_t)count * res * lut_t_pitch(planes) * 4), "cudaMalloc(Z-LUT copy)");
        CheckCuda(cudaMalloc(&d_cmp_, (size_t)count * planes * 4), "cudaMalloc(compare profiles)");
        CheckCuda(cudaMemset(d_cmp_, 0, (size_t)count * planes * 4), "clear compare profiles");
        lut_count_ = count;
        lut_planes_ = planes;
        tc_lut_stale_ = lut_t_stale_ = true;
        if (Params(2).smem_bytes > 227 * 1024) {
            cudaFree(d_lut_);
            cudaFree(d_lut_t_);
            cudaFree(d_cmp_);
            d_lut_ = nullptr;
            d_lut_t_ = nullptr;
            d_cmp_ = nullptr;
            lut_count_ = lut_planes_ = 0;
            throw std::invalid_argument("Z-LUT with " + std::to_string(planes) +
                                        " planes does not fit the per-CTA score buffer");
        }
    } else {
        lut_count_ = lut_planes_ = 0;
    }
    CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
}

void Tracker::GetRadialZLUT(float *dst)
{
    if (!dst) throw std::invalid_argument("GetRadialZLUT: null destination");
    DeviceGuard dg(device_);
    std::lock_guard<std::mutex> lk(mu_);
    CheckCuda(cudaStreamSynchronize(lut_stream_), "cudaStreamSynchronize(lut)");
    const size_t total = (size_t)lut_count_ * lut_planes_ * cfg.zlut_radialsteps;
    if (total) CheckCuda(cudaMemcpy(dst, d_lut_, total * 4, cudaMemcpyDeviceToHost), "download Z-LUT");
}

void Tracker::GetRadialZLUTSize(int &count, int &planes, int &radialsteps) const
{
    count = lut_count_;
    planes = lut_planes_;
    radialsteps = cfg.zlut_radialsteps;
}

// QueuedCPUTracker::SetRadialWeights, QueuedCPUTracker.cpp:393-406 (null clears them).
void Tracker::SetRadialWeights(const float *w)
{
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    if (w) {
        CheckCuda(cudaMemcpy(d_zw_, w, (size_t)cfg.zlut_radialsteps * 4, cudaMemcpyHostToDevice), "upload weights");
        have_zw_ = true;
    } else {
        have_zw_ = false;
    }
    tc_lut_stale_ = true;  // the BF16 copy holds weighted rows; the transposed one does not
}

// QueuedTracker::SetZLUTBiasCorrection (cputrack/QueuedTracker.cpp:178-182): table[bead][bias_plane],
// bias_planes wide and count (beads) high; nullptr removes it.
void Tracker::SetZLUTBiasTable(const float *table, int bias_planes, int count)
{
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    cudaFree(d_zbias_);
    d_zbias_ = nullptr;
    zbias_w_ = zbias_count_ = 0;
    if (table && bias_planes > 0 && count > 0) {
        const size_t n = (size_t)bias_planes * count;
        CheckCuda(cudaMalloc(&d_zbias_, n * 4), "cudaMalloc(bias table)");
        CheckCuda(cudaMemcpy(d_zbias_, table, n * 4, cudaMemcpyHostToDevice), "upload bias table");
        zbias_w_ = bias_planes;
        zbias_count_ = count;
    }
}

// QueuedTracker::ComputeZBiasCorrection (cputrack/QueuedTracker.cpp:143-189): for every bead
// and each of bias_planes evenly spaced z (plane / bias_planes * planes), render the bead's LUT
// at the ROI centre (GenerateImageFromLUT with smp_per_pixel^2 samples per pixel), localize it
// with COM, 2 QI iterations with the QI radial window, and the Z match with the Z radial window
// on the normalised profile (a fresh CPUTracker in the reference: no calibration images, no
// background correction, no bias table), and store z - true z. Both stages run on the GPU; the
// table becomes this instance's bias table.
void Tracker::ComputeZBiasTable(int bias_planes, int smp_per_pixel, bool spline, float *out)
{
    if (bias_planes <= 0 || smp_per_pixel <= 0) throw std::invalid_argument("ComputeZBiasTable: invalid argument");
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    TrackParams P;
    int count, planes;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (!d_lut_ || lut_count_ <= 0 || lut_planes_ < 2) throw std::runtime_error("ComputeZBiasTable: no Z-LUT set");
        count = lut_count_;
        planes = lut_planes_;
        P = LaunchParams(2);
    }
    const int W = cfg.base.width, H = cfg.base.height, nb = P.z_nbins;
    P.mode = kLT_QI | kLT_LocalizeZ | kLT_NormalizeProfile;
    P.qi_iterations = 2;
    P.com_bgcorrection = 0.0f;
    P.cmp_scores = nullptr;
    P.zbias = nullptr;
    P.zbias_w = P.zbias_count = 0;
    P.calib_offset = P.calib_gain = nullptr;
    P.calib_count = 0;
    P.zprof_f32 = nullptr;
    P.zprof_bf16 = nullptr;
    plan_smem(P);
    const std::vector<float> zw = radial_bin_window(nb);
    const int total = count * bias_planes;
    const int chunk = std::max(1, std::min(total, (int)((256u << 20) / ((size_t)W * H * 4))));
    float *d_zw = nullptr, *d_img = nullptr;
    LocalizationJob *d_jobs = nullptr;
    LocalizationResult *d_res = nullptr;
    cudaStream_t st = nullptr;
    std::vector<LocalizationResult> res(total);
    auto release = [&] {
        cudaFree(d_zw);
        cudaFree(d_img);
        cudaFree(d_jobs);
        cudaFree(d_res);
        if (st) cudaStreamDestroy(st);
    };
    try {
        CheckCuda(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        CheckCuda(cudaMalloc(&d_zw, sizeof(float) * nb), "cudaMalloc");
        CheckCuda(cudaMalloc(&d_img, sizeof(float) * (size_t)chunk * W * H), "cudaMalloc(bias images)");
        CheckCuda(cudaMalloc(&d_jobs, sizeof(LocalizationJob) * chunk), "cudaMalloc");
        CheckCuda(cudaMalloc(&d_res, sizeof(LocalizationResult) * chunk), "cudaMalloc");
        CheckCuda(cudaMemcpyAsync(d_zw, zw.data(), sizeof(float) * nb, cudaMemcpyHostToDevice, st), "upload weights");
        P.z_weights = d_zw;
        CheckCuda(cudaStreamWaitEvent(st, lut_ready_, 0), "cudaStreamWaitEvent");
        for (int first = 0; first < total; first += chunk) {
            const int n = std::min(chunk, total - first);
            CheckCuda(launch_lut_images(P.lut, nb, planes, first, n, bias_planes, W, H, P.z_minr, P.z_maxr,
                                        smp_per_pixel, spline, d_img, d_jobs, st),
                      "bias image launch");
            CheckCuda(launch_localize(P, reinterpret_cast<const uint8_t *>(d_img), W * 4, (int64_t)W * H * 4, nullptr,
                                      d_jobs, n, d_res, st),
                      "localize launch");
            launches_ += 2;
            CheckCuda(cudaMemcpyAsync(res.data() + first, d_res, sizeof(LocalizationResult) * n,
                                      cudaMemcpyDeviceToHost, st),
                      "download results");
        }
        CheckCuda(cudaStreamSynchronize(st), "bias table");
    } catch (...) {
        release();
        throw;
    }
    release();
    std::vector<float> table(total);
    for (int i = 0; i < total; i++) {
        const int plane = i % bias_planes;
        table[i] = res[i].pos.z - plane / (float)bias_planes * planes;
    }
    SetZLUTBiasTable(table.data(), bias_planes, count);
    if (out) std::copy(table.begin(), table.end(), out);
}

void Tracker::EnableRadialZLUTCompareProfile(bool enabled)
{
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    cmp_enabled_ = enabled;
}

void Tracker::GetRadialZLUTCompareProfile(float *dst)
{
    if (!dst) throw std::invalid_argument("GetRadialZLUTCompareProfile: null destination");
    DeviceGuard dg(device_);
    WaitIdleForReconfigure();
    std::lock_guard<std::mutex> lk(mu_);
    if (d_cmp_ && lut_count_ * lut_planes_ > 0)
        CheckCuda(cudaMemcpy(dst, d_cmp_, (size_t)lut_count_ * lut_planes_ * 4, cudaMemcpyDeviceToHost),
                  "download compare profiles");
}

void Tracker::BeginLUT(uint32_t flags)
{
    std::lock_guard<std::mutex> lk(mu_);
    if (flags & (BUILDLUT_IMAGELUT | BUILDLUT_FOURIER))
        Warn("BeginLUT: BUILDLUT_IMAGELUT and BUILDLUT_FOURIER are not supported and were ignored");
    if (flags & BUILDLUT_BIASCORRECT) Warn("BeginLUT: BUILDLUT_BIASCORRECT is not supported and was ignored");
    lut_flags_ = flags;
}

// QueuedCPUTracker::BuildLUT, QueuedCPUTracker.cpp:580-646: `data` holds one ROI per bead,
// bead i at data + pitch*height*i. The rows are staged (double-buffered) and the profiles are
// accumulated into the device LUT by one kernel launch per plane. With `async` a pinned stack is
// still being copied when the call returns (the caller keeps it unchanged until FinalizeLUT returns),
// so the copies of successive planes run back to back instead of each waiting for the caller's
// next call; at most two planes are in flight (the device staging buffers).
void Tracker::BuildLUT(const void *data, int pitch, int pdt, int plane, const vector2f *known_pos, bool async)
{
    if (!data) throw std::invalid_argument("BuildLUT: null data");
    if (pdt < 0 || pdt > 2) throw std::invalid_argument("BuildLUT: unknown pixel data type");
    DeviceGuard dg(device_);
    std::lock_guard<std::mutex> lk(mu_);
    if (!d_lut_ || lut_count_ <= 0) {
        Warn("BuildLUT: no Z-LUT allocated (call SetRadialZLUT first); ignored");
        return;
    }
    if (plane < 0 || plane >= lut_planes_) {
        Warn("BuildLUT: plane " + std::to_string(plane) + " out of range; ignored");
        return;
    }
    const int W = cfg.base.width, H = cfg.base.height, nb = lut_count_;
    const size_t rowb = (size_t)W * pdt_bytes(pdt);
    if ((size_t)pitch < rowb) throw std::invalid_argument("BuildLUT: pitch smaller than a row");
    const size_t bytes = (size_t)pitch * ((size_t)H * nb - 1) + rowb;
    const size_t kp_off = (bytes + 15) & ~(size_t)15;
    const size_t need = kp_off + sizeof(float2) * nb;
    if (need > lut_stage_bytes_) {
        CheckCuda(cudaStreamSynchronize(lut_stream_), "cudaStreamSynchronize(lut)");
        for (int b = 0; b < 2; b++) {
            cudaFreeHost(h_lut_stage_[b]);
            cudaFree(d_lut_stage_[b]);
            h_lut_stage_[b] = d_lut_stage_[b] = nullptr;
            CheckCuda(cudaHostAlloc(&h_lut_stage_[b], need, cudaHostAllocDefault), "cudaHostAlloc(LUT stage)");
            CheckCuda(cudaMalloc(&d_lut_stage_[b], need), "cudaMalloc(LUT stage)");
        }
        lut_stage_bytes_ = need;
    }
    const int b = lut_stage_next_;
    lut_stage_next_ ^= 1;
    CheckCuda(cudaEventSynchronize(lut_stage_free_[b]), "cudaEventSynchronize");
    // A pinned stack is DMA'd straight from the caller's buffer on a copy stream, so that the copy
    // of this plane overlaps the kernel of the previous one; the call returns once the copy is done
    // (the caller may reuse the buffer, as after the reference's synchronous BuildLUT). A pageable
    // stack goes through the pinned staging buffer.
    const bool pinned = IsPinned(data);
    if (pinned) {
        CheckCuda(cudaMemcpyAsync(d_lut_stage_[b], data, bytes, cudaMemcpyHostToDevice, lut_copy_stream_),
                  "H2D LUT stack");
        if (known_pos) {
            std::memcpy(h_lut_stage_[b] + kp_off, known_pos, sizeof(float2) * nb);
            CheckCuda(cudaMemcpyAsync(d_lut_stage_[b] + kp_off, h_lut_stage_[b] + kp_off, sizeof(float2) * nb,
                                      cudaMemcpyHostToDevice, lut_copy_stream_),
                      "H2D known positions");
        }
        CheckCuda(cudaEventRecord(lut_copy_done_[b], lut_copy_stream_), "cudaEventRecord");
        CheckCuda(cudaStreamWaitEvent(lut_stream_, lut_copy_done_[b], 0), "cudaStreamWaitEvent");
    } else {
        std::memcpy(h_lut_stage_[b], data, bytes);
        if (known_pos) std::memcpy(h_lut_stage_[b] + kp_off, known_pos, sizeof(float2) * nb);
        CheckCuda(cudaMemcpyAsync(d_lut_stage_[b], h_lut_stage_[b], known_pos ? need : bytes, cudaMemcpyHostToDevice,
                                  lut_stream_),
                  "H2D LUT stack");
    }
    TrackParams P = Params(pdt);
    P.mode = 0;  // BuildLUT runs COM/QI/profile without the per-job mode bits
    CheckCuda(launch_build_lut(P, d_lut_stage_[b], pitch, nb, plane,
                               known_pos ? reinterpret_cast<const float2 *>(d_lut_stage_[b] + kp_off) : nullptr,
                               (lut_flags_ & BUILDLUT_NORMALIZE) != 0, d_lut_, lut_stream_),
              "BuildLUT kernel launch");
    launches_++;
    CheckCuda(cudaEventRecord(lut_stage_free_[b], lut_stream_), "cudaEventRecord");
    CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
    tc_lut_stale_ = lut_t_stale_ = true;
    if (pinned && !async) CheckCuda(cudaEventSynchronize(lut_copy_done_[b]), "cudaEventSynchronize(LUT copy)");
}

// QueuedCPUTracker::FinalizeLUT, QueuedCPUTracker.cpp:648-659.
void Tracker::FinalizeLUT()
{
    DeviceGuard dg(device_);
    std::lock_guard<std::mutex> lk(mu_);
    if (d_lut_) {
        CheckCuda(launch_finalize_lut(d_lut_, lut_count_ * lut_planes_, cfg.zlut_radialsteps, lut_stream_),
                  "FinalizeLUT kernel launch");
        launches_++;
    }
    CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
    CheckCuda(cudaStreamSynchronize(lut_stream_), "cudaStreamSynchronize(lut)");
    tc_lut_stale_ = lut_t_stale_ = true;
}

int Tracker::GetResultCount()
{
    DeviceGuard dg(device_);
    {
        std::lock_guard<std::mutex> lk(mu_);
        CollectLocked();
    }
    std::lock_guard<std::mutex> rl(res_mu_);
    return (int)results_.size();
}

// FIFO order, like QueuedCUDATracker::FetchResults (cudatrack/QueuedCUDATracker.cu:726-737).
int Tracker::FetchResults(LocalizationResult *dst, int maxResults)
{
    if (!dst || maxResults <= 0) return 0;
    DeviceGuard dg(device_);
    {
        std::lock_guard<std::mutex> lk(mu_);
        CollectLocked();
    }
    std::lock_guard<std::mutex> rl(res_mu_);
    int n = 0;
    while (n < maxResults && !results_.empty()) {
        dst[n++] = results_.front();
        results_.pop_front();
    }
    return n;
}

int Tracker::GetQueueLength(int *maxQueueLen)
{
    DeviceGuard dg(device_);
    std::lock_guard<std::mutex> lk(mu_);
    CollectLocked();
    int n = filling_ >= 0 ? slots_[filling_].count : 0;
    for (int i : inflight_) n += slots_[i].count;
    if (maxQueueLen) *maxQueueLen = (int)slots_.size() * batch_;
    return n;
}

bool Tracker::IsIdle() { return GetQueueLength(nullptr) == 0; }

std::string Tracker::GetProfileReport()
{
    std::lock_guard<std::mutex> lk(mu_);
    std::ostringstream o;
    o << "B200 tracker (device " << device_ << "): " << stats_.batches << " batches, " << stats_.rois << " ROIs";
    if (stats_.gpu_ms > 0) o << ", " << stats_.gpu_ms << " ms on the GPU streams";
    if (!stats_.latency_ms.empty()) {
        std::vector<float> l = stats_.latency_ms;
        std::sort(l.begin(), l.end());
        auto pct = [&](double p) { return l[std::min(l.size() - 1, (size_t)(p * (l.size() - 1) + 0.5))]; };
        o << "; batch latency p50 " << pct(0.5) << " ms, p99 " << pct(0.99) << " ms";
    }
    o << "; batch size " << batch_ << ", " << slots_.size() << " streams, " << launches_.load() << " kernel launches";
    return o.str();
}

std::string Tracker::GetWarnings()
{
    std::lock_guard<std::mutex> lk(warn_mu_);
    std::string w;
    w.swap(warnings_);
    return w;
}

int Tracker::LocalizeDevice(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                            const LocalizationJob *d_jobs, LocalizationResult *d_results, cudaStream_t stream)
{
    if (!d_pixels || !d_results || count < 0 || pdt < 0 || pdt > 2) {
        Warn("QTrkB200LocalizeDevice: invalid argument");
        return -1;
    }
    if (pitch < cfg.base.width * pdt_bytes(pdt)) {
        Warn("QTrkB200LocalizeDevice: pitch smaller than a row");
        return -2;
    }
    DeviceGuard dg(device_);
    TrackParams P;
    ZMatchParams Q;
    bool tc;
    {
        std::lock_guard<std::mutex> lk(mu_);
        P = LaunchParams(pdt);
        tc = UseTensorCoreMatch();
        if (tc && d_jobs) {
            // the bead of each ROI is only known on the device here: score with the plain path
            static bool warned = false;
            if (!warned) Warn("QTrkB200LocalizeDevice: device-side jobs use the plain Z match");
            warned = true;
            tc = false;
        }
        if (tc) {
            const int nb = cfg.zlut_radialsteps, nbp = zmatch_padded_bins(nb);
            if (dev_scratch_rois_ < count) {
                CheckCuda(cudaDeviceSynchronize(), "cudaDeviceSynchronize");
                cudaFree(d_dev_zprof_);
                cudaFree(d_dev_zprof_bf16_);
                d_dev_zprof_ = nullptr;
                d_dev_zprof_bf16_ = nullptr;
                dev_scratch_rois_ = 0;
                CheckCuda(cudaMalloc(&d_dev_zprof_, sizeof(float) * (size_t)count * nb), "cudaMalloc(profiles)");
                CheckCuda(cudaMalloc(&d_dev_zprof_bf16_, sizeof(__nv_bfloat16) * (size_t)count * 2 * nbp),
                          "cudaMalloc(profiles)");
                dev_scratch_rois_ = count;
            }
            PrepareTensorCoreLUT();
            P.zprof_f32 = d_dev_zprof_;
            P.zprof_bf16 = d_dev_zprof_bf16_;
            P.zprof_nbp = nbp;
            Q = TensorCoreParams();
            Q.prof_f32 = d_dev_zprof_;
            Q.prof_bf16 = d_dev_zprof_bf16_;
            Q.perm = nullptr;
            Q.tiles = nullptr;
            Q.count = count;
            Q.uniform_bead = 0;
            Q.results = d_results;
        }
    }
    CheckCuda(cudaStreamWaitEvent(stream, lut_ready_, 0), "cudaStreamWaitEvent");
    CheckCuda(launch_localize(P, static_cast<const uint8_t *>(d_pixels), pitch, roi_stride, nullptr, d_jobs, count,
                              d_results, stream),
              "localize kernel launch");
    launches_++;
    if (tc) {
        CheckCuda(launch_zmatch_tc(Q, (count + 127) / 128, stream), "Z-match kernel launch");
        launches_++;
    }
    if (RefineAfterZ(P)) {
        CheckCuda(launch_joint_refine(P, static_cast<const uint8_t *>(d_pixels), pitch, roi_stride, nullptr, d_jobs,
                                      count, d_results, stream),
                  "joint refine launch");
        launches_++;
    }
    return 0;
}

// The allocation-free variant of LocalizeDevice: the tensor-core match's profiles go to
// `scratch` (a fixed device array owned by the caller of this method), and the instance's
// BF16 LUT must already exist with the current LUT's shape (it is created by the first
// allocating call in this mode, and dropped when SetRadialZLUT installs a LUT); refreshing a
// stale BF16 LUT of the same shape (new contents from BuildLUT, FinalizeLUT, new radial weights)
// is a kernel launch only, ordered after the work already queued on the caller's stream, which
// may still be reading the old copy. Nothing here calls cudaMalloc/cudaFree.
int Tracker::LocalizeDeviceNoAlloc(const void *d_pixels, int pitch, int64_t roi_stride, int pdt, int count,
                                   const LocalizationJob *d_jobs, LocalizationResult *d_results, cudaStream_t stream,
                                   void *scratch, size_t scratch_bytes)
{
    if (!d_pixels || !d_results || !scratch || count < 0 || pdt < 0 || pdt > 2) {
        Warn("QTrkB200LocalizeDeviceNoAlloc: invalid argument");
        return -1;
    }
    if (pitch < cfg.base.width * pdt_bytes(pdt)) {
        Warn("QTrkB200LocalizeDeviceNoAlloc: pitch smaller than a row");
        return -2;
    }
    DeviceGuard dg(device_);
    TrackParams P;
    ZMatchParams Q;
    bool tc;
    float *zprof = nullptr;
    __nv_bfloat16 *zbf = nullptr;
    {
        std::lock_guard<std::mutex> lk(mu_);
        tc = UseTensorCoreMatch() && !d_jobs;  // device-side jobs: plain match, as LocalizeDevice
        if (tc) {
            const int nb = cfg.zlut_radialsteps, nbp = zmatch_padded_bins(nb);
            const bool shape_ok = tc_lut_count_ == lut_count_ && tc_lut_pp_ == zmatch_padded_planes(lut_planes_) &&
                                  tc_lut_nbp_ == nbp;
            if (!d_lut_bf16_ || !d_lut_norm_ || !shape_ok) {
                Warn("QTrkB200LocalizeDeviceNoAlloc: the instance has no tensor-core LUT of the current LUT's shape; "
                     "it is created by the first QTrkB200LocalizeDevice call or queued batch in this mode after "
                     "the LUT is set");
                return -4;
            }
            const size_t prof_bytes = ((sizeof(float) * (size_t)count * nb) + 255) & ~(size_t)255;
            const size_t need = prof_bytes + sizeof(__nv_bfloat16) * (size_t)count * 2 * nbp;
            if (need > scratch_bytes) {
                Warn("QTrkB200LocalizeDeviceNoAlloc: " + std::to_string(count) + " ROIs need " + std::to_string(need) +
                     " bytes of profile scratch; the fixed array holds " + std::to_string(scratch_bytes));
                return -3;
            }
            zprof = static_cast<float *>(scratch);
            zbf = reinterpret_cast<__nv_bfloat16 *>(static_cast<uint8_t *>(scratch) + prof_bytes);
            if (tc_lut_stale_) {  // refresh in place: one kernel launch into buffers of this shape
                CheckCuda(cudaEventRecord(noalloc_order_, stream), "cudaEventRecord");
                CheckCuda(cudaStreamWaitEvent(lut_stream_, noalloc_order_, 0), "cudaStreamWaitEvent");
                CheckCuda(zmatch_prepare_lut(d_lut_, have_zw_ ? d_zw_ : nullptr, lut_count_, lut_planes_, nb,
                                             d_lut_bf16_, d_lut_norm_, lut_stream_),
                          "BF16 LUT preparation");
                launches_++;
                CheckCuda(cudaEventRecord(lut_ready_, lut_stream_), "cudaEventRecord");
                tc_lut_stale_ = false;
            }
            Q = TensorCoreParams();
            Q.prof_f32 = zprof;
            Q.prof_bf16 = zbf;
            Q.perm = nullptr;
            Q.tiles = nullptr;
            Q.count = count;
            Q.uniform_bead = 0;
            Q.results = d_results;
        }
        // after the checks above, so that a refused call launches nothing
        P = LaunchParams(pdt);
        if (tc) {
            P.zprof_f32 = zprof;
            P.zprof_bf16 = zbf;
            P.zprof_nbp = Q.nbp;
        }
    }
    CheckCuda(cudaStreamWaitEvent(stream, lut_ready_, 0), "cudaStreamWaitEvent");
    CheckCuda(launch_localize(P, static_cast<const uint8_t *>(d_pixels), pitch, roi_stride, nullptr, d_jobs, count,
                              d_results, stream),
              "localize kernel launch");
    launches_++;
    if (tc) {
        CheckCuda(launch_zmatch_tc(Q, (count + 127) / 128, stream), "Z-match kernel launch");
        launches_++;
    }
    if (RefineAfterZ(P)) {
        CheckCuda(launch_joint_refine(P, static_cast<const uint8_t *>(d_pixels), pitch, roi_stride, nullptr, d_jobs,
                                      count, d_results, stream),
                  "joint refine launch");
        launches_++;
    }
    return 0;
}

}  // namespace qtrk
