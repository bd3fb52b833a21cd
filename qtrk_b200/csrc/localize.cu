// Localization kernels for sm_100a.
//
// localize_qi_kernel: one CTA per ROI runs the whole per-ROI pipeline of
//   QueuedCPUTracker::ProcessJob (cputrack/QueuedCPUTracker.cpp:273-361) on a float tile of the
//   ROI in shared memory: bulk copy (or batched loads) + convert (+ calibration) fused with the
//   first COM pass -> COM -> QI iterations -> radial profile -> Z-LUT match -> result. Pixels are
//   read from HBM exactly once; everything after the load works on-chip.
// localize_gauss_kernel: one CTA per ROI, COM -> 2D Gaussian MLE (-> Z) on a plain tile.
// gauss_warp_kernel: one warp per small ROI (<= 32x32) for the Gaussian-only mode.
// build_lut_kernel / finalize_lut_kernel: QueuedCPUTracker::BuildLUT / FinalizeLUT
//   (cputrack/QueuedCPUTracker.cpp:580-659) with the accumulation on the device.
// profile_kernel: ComputeRadialProfile (cputrack/utils.cpp:275-320) for one image.
#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cuda_runtime.h>

#include <cuda_bf16.h>

#include "bulk_copy.cuh"
#include "device_common.cuh"
#include "kernels.h"

namespace qtrk {

// QI / Z-LUT least-squares weights, cputrack/QueuedTracker.h:349,359
__device__ const float kQIWeights[7] = {0.14f, 0.5f, 0.85f, 1.0f, 0.85f, 0.5f, 0.14f};
__device__ const float kZLUTWeights[7] = {0.15f, 0.5f, 0.85f, 1.0f, 0.85f, 0.5f, 0.15f};

struct SmemView {
    float *img, *misc;
    float4 *qdirs;  // QI quadrant directions as (d.x, d.x, d.y, d.y)
    float2 *tw;
    float4 *zdirs;  // full-circle directions in pairs (j, j + n/2), see load_z_tables
    float *qrw;  // QI radial weights (qi_nr floats after the twiddles)
    uint8_t *work;
    double *red;
};

__device__ __forceinline__ SmemView smem_view(uint8_t *smem, const TrackParams &P)
{
    SmemView v;
    v.img = reinterpret_cast<float *>(smem + P.sm_img);
    v.misc = reinterpret_cast<float *>(smem + P.sm_misc);
    v.red = reinterpret_cast<double *>(smem + P.sm_red);
    v.work = smem + P.sm_work;
    float2 *tab = reinterpret_cast<float2 *>(smem + P.sm_tables);
    v.qdirs = reinterpret_cast<float4 *>(tab);
    v.tw = tab + 2 * P.qi_angpq;  // L/2 = qi_nr twiddles
    v.qrw = reinterpret_cast<float *>(v.tw + P.qi_nr);
    v.zdirs = reinterpret_cast<float4 *>(tab);  // loaded over the QI tables once QI is done
    return v;
}

// Copy the QI direction / twiddle tables into shared memory (all threads; a barrier must
// follow before use).
__device__ __forceinline__ void load_qi_tables(const SmemView &s, const TrackParams &P)
{
    const float2 *qd = static_cast<const float2 *>(P.qi_dirs);
    const float2 *tw = static_cast<const float2 *>(P.qi_twiddles);
    if (qd)
        for (int i = threadIdx.x; i < P.qi_angpq; i += blockDim.x) {
            const float2 d = qd[i];
            s.qdirs[i] = make_float4(d.x, d.x, d.y, d.y);
        }
    if (tw)
        for (int i = threadIdx.x; i < P.qi_nr; i += blockDim.x) s.tw[i] = tw[i];
    if (P.qi_rweights)
        for (int i = threadIdx.x; i < P.qi_nr; i += blockDim.x) s.qrw[i] = P.qi_rweights[i];
}

// Copy the full-circle direction table over the QI tables (all threads; the QI stage must
// be finished, and a barrier must follow before use).
__device__ __forceinline__ void load_z_tables(const SmemView &s, const TrackParams &P)
{
    const float2 *zd = static_cast<const float2 *>(P.z_dirs);
    if (zd)
        for (int j = threadIdx.x; j < (P.z_angsteps + 1) >> 1; j += blockDim.x) {
            // entry j = (d_j.x, d_{j+h}.x, d_j.y, d_{j+h}.y), h = n/2 rounded down; with n odd the
            // last entry holds d_{n-1} alone (zeros in the second place, never read)
            const int h = P.z_angsteps >> 1;
            const float2 a = zd[j < h ? j : P.z_angsteps - 1];
            const float2 b = j < h ? zd[j + h] : make_float2(0.0f, 0.0f);
            s.zdirs[j] = make_float4(a.x, b.x, a.y, b.y);
        }
}

// The QI position update from the two autoconvolutions (cpu_tracker.cpp:345-357, 400-410):
// ComputeMaxInterp over autoconv[x] = ac[(x + nr) mod L] for X (.x) and Y (.y), by one warp: a
// two-axis argmax over the warp (first index of the maximum, as warp_argmax), then the 7-point
// fits of both axes side by side (even lanes X, odd lanes Y). Lanes 0 and 1 write the new x and y
// to misc[0] and misc[1]. Runs on the warp that made ac, right after it, with no CTA barrier.
__device__ __forceinline__ void qi_fit_xy(const float2 *ac, int nr, float cx, float cy, float rstep, float *misc)
{
    const int lane = threadIdx.x & 31, L = 2 * nr;
    float bx = 0.0f, by = 0.0f;
    int ix = -1, iy = -1;
    for (int x = lane; x < L; x += 32) {
        int n = x + nr;
        if (n >= L) n -= L;
        const float2 v = ac[n];
        if (v.x == v.x && (ix < 0 || v.x > bx)) {
            bx = v.x;
            ix = x;
        }
        if (v.y == v.y && (iy < 0 || v.y > by)) {
            by = v.y;
            iy = x;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const float ox = __shfl_xor_sync(0xffffffffu, bx, o), oy = __shfl_xor_sync(0xffffffffu, by, o);
        const int oix = __shfl_xor_sync(0xffffffffu, ix, o), oiy = __shfl_xor_sync(0xffffffffu, iy, o);
        if (oix >= 0 && (ix < 0 || ox > bx || (ox == bx && oix < ix))) {
            bx = ox;
            ix = oix;
        }
        if (oiy >= 0 && (iy < 0 || oy > by || (oy == by && oiy < iy))) {
            by = oy;
            iy = oiy;
        }
    }
    ix = ix < 0 ? 0 : ix;
    iy = iy < 0 ? 0 : iy;
    const bool yaxis = (lane & 1) != 0;
    float m;
    if (ix >= 3 && ix + 4 <= L && iy >= 3 && iy + 4 <= L) {  // both windows inside: per-lane fits
        auto at = [&](int x) {
            int n = x + nr;
            if (n >= L) n -= L;
            return yaxis ? ac[n].y : ac[n].x;
        };
        m = max_interp7_sym(at, L, yaxis ? iy : ix, kQIWeights);
    } else {  // a clipped window takes the warp-wide fit, one axis after the other
        auto atx = [&](int x) {
            int n = x + nr;
            if (n >= L) n -= L;
            return ac[n].x;
        };
        auto aty = [&](int x) {
            int n = x + nr;
            if (n >= L) n -= L;
            return ac[n].y;
        };
        const float mx = max_interp7_sym(atx, L, ix, kQIWeights);
        const float my = max_interp7_sym(aty, L, iy, kQIWeights);
        m = yaxis ? my : mx;
    }
    if (lane < 2) {
        const float off = (m - (float)nr) * (3.14159265359f / 4);
        misc[lane] = (yaxis ? cy : cx) + off * rstep;
    }
}

// CPUTracker::ComputeQI, cpu_tracker.cpp:285-360. All threads call; returns the position and the
// boundary flag of the last iteration.
__device__ void qi_localize(const SmemView &s, const TrackParams &P, float mean, float &cx, float &cy, bool &bhit,
                            const float *rweights)
{
    const int W = P.width, H = P.height, nr = P.qi_nr, L = 2 * nr;
    const bool pow2 = (L & (L - 1)) == 0 && L >= 2;
    // work: [ ac (L complex) ] [ A (L complex) ] [ subset partials (2 KB) ]
    float2 *ac = reinterpret_cast<float2 *>(s.work);
    float2 *A = reinterpret_cast<float2 *>(s.work + L * 8);
    float4 *part = reinterpret_cast<float4 *>(s.work + 2 * L * 8);
    const float rstep = (P.qi_maxr - P.qi_minr) / (float)nr;  // also pixelsPerProfLen (cpu_tracker.cpp:311,649)
    for (int k = 0; k < P.qi_iterations; k++) {
        bhit = check_boundaries(cx, cy, P.qi_maxr, W, H);
        qi_profiles_sym(s.img, W, H, W, cx, cy, mean, nr, P.qi_nang[k], P.qi_inv_nang[k], P.qi_stride[k], P.qi_minr, rstep,
                        s.qdirs, rweights, part, A, pow2 ? ilog2_pow2(L) : -1);
        __syncthreads();
        if (pow2) {
            if (threadIdx.x < 32) {  // transform and fits on warp 0, the others wait at the next barrier
                qi_autoconv_fft_filled(nr, A, ac, s.tw);
                qi_fit_xy(ac, nr, cx, cy, rstep, s.misc);
            }
        } else {
            qi_autoconv_direct_filled(nr, A, ac);
            if (threadIdx.x < 32) qi_fit_xy(ac, nr, cx, cy, rstep, s.misc);
        }
        __syncthreads();
        // misc[0..1] is written again only after the next iteration's first barrier, which every
        // thread reaches after these reads
        cx = s.misc[0];
        cy = s.misc[1];
    }
}

// Radial profile + Z-LUT compare (QueuedCPUTracker.cpp:319-338). Returns z (0 without a LUT). With
// P.zprof_f32 set, the profile is written out for the tensor-core match instead.
__device__ float z_localize(const SmemView &s, const TrackParams &P, float mean, float x, float y, int bead, int roi)
{
    const int nb = P.z_nbins;
    float *prof = reinterpret_cast<float *>(s.work);
    double *scores = reinterpret_cast<double *>(s.work + (((nb * 4) + 15) & ~15));
    const float rstep = (P.z_maxr - P.z_minr) / (float)nb;
    load_z_tables(s, P);
    __syncthreads();
    radial_profile(s.img, P.width, P.height, P.width, x, y, mean, nb, P.z_angsteps, P.z_minr, rstep, s.zdirs, prof,
                   (P.mode & kLT_NormalizeProfile) != 0, s.red);
    if (P.zprof_f32) {
        // [hi | lo] BF16 split of the weighted profile: v = hi + lo + O(2^-16 v)
        __nv_bfloat16 *pb = static_cast<__nv_bfloat16 *>(P.zprof_bf16) + (size_t)roi * 2 * P.zprof_nbp;
        for (int r = threadIdx.x; r < P.zprof_nbp; r += blockDim.x) {
            float v = 0.0f;
            if (r < nb) {
                v = prof[r];
                P.zprof_f32[(size_t)roi * nb + r] = v;
                if (P.z_weights) v *= P.z_weights[r];
            }
            const __nv_bfloat16 h = __float2bfloat16_rn(v);
            pb[r] = h;
            pb[P.zprof_nbp + r] = __float2bfloat16_rn(v - __bfloat162float(h));
        }
        return 0.0f;
    }
    if (!P.lut || bead < 0 || bead >= P.lut_count) return 0.0f;
    if (!P.lut_t) return __int_as_float(0x7fc00000);  // the host launched without refreshing the transposed LUT
    const float *lut_t = P.lut_t + (size_t)bead * nb * P.lut_t_pitch;
    zlut_scores_plain(prof, lut_t, P.lut_t_pitch, P.lut_planes, nb, P.z_weights, scores);
    if (P.cmp_scores)
        for (int k = threadIdx.x; k < P.lut_planes; k += blockDim.x)
            P.cmp_scores[(size_t)bead * P.lut_planes + k] = (float)scores[k];
    if (threadIdx.x < 32) {
        auto at = [&](int i) { return scores[i]; };
        const int im = warp_argmax(at, P.lut_planes);
        const float z = max_interp7_sym(at, P.lut_planes, im, kZLUTWeights);
        if (threadIdx.x == 0) s.misc[2] = zlut_bias_correct(z, P.lut_planes, P.zbias, P.zbias_w, P.zbias_count, bead);
    }
    __syncthreads();
    return s.misc[2];
}

__device__ __forceinline__ void read_job(const LocalizationJob *jobs, int i, uint32_t (&w)[6])
{
    if (jobs) {
        const uint32_t *p = reinterpret_cast<const uint32_t *>(jobs) + (size_t)i * 6;
#pragma unroll
        for (int k = 0; k < 6; k++) w[k] = p[k];
    } else {
        w[0] = (uint32_t)i;
#pragma unroll
        for (int k = 1; k < 6; k++) w[k] = 0;
    }
}

__device__ __forceinline__ void write_result(LocalizationResult *results, int i, const uint32_t (&job)[6], float x,
                                             float y, float z, float gx, float gy, uint32_t err, float mean)
{
    uint32_t *o = reinterpret_cast<uint32_t *>(results) + (size_t)i * 13;
#pragma unroll
    for (int k = 0; k < 6; k++) o[k] = job[k];
    o[6] = __float_as_uint(x);
    o[7] = __float_as_uint(y);
    o[8] = __float_as_uint(z);
    o[9] = __float_as_uint(gx);
    o[10] = __float_as_uint(gy);
    o[11] = err;
    o[12] = __float_as_uint(mean);
}

constexpr int kMinBlocks = 5;  // CTAs per SM the QI and Gaussian kernels are compiled for (<= 96 registers)

constexpr uint32_t kStageWaitLimit = 1u << 22;  // mbarrier polls before a staged copy counts as lost

// COM / QI (+ Z): QueuedCPUTracker::ProcessJob (QueuedCPUTracker.cpp:273-361), one CTA per ROI.
// The ROI becomes a float tile in shared memory. With kStaged (ROIs back to back, 16-byte
// aligned, whole 16-byte chunks) its raw bytes arrive by one bulk copy (cp.async.bulk, completion
// on an mbarrier) started by thread 0 as the CTA begins, while the other threads fetch the QI
// tables, and are converted in place; otherwise the threads load them with batched streaming
// loads (frame bands, unaligned ROIs). The COM's first pass is fused into either conversion.
// One instantiation per form, so neither carries the other's registers.
template <bool kStaged>
__global__ void __launch_bounds__(kBlockThreads, kMinBlocks)
    localize_qi_kernel(TrackParams P, const uint8_t *__restrict__ pixels, int pitch, int64_t roi_stride,
                       const int64_t *__restrict__ roi_offsets, const LocalizationJob *__restrict__ jobs, int count,
                       LocalizationResult *__restrict__ results)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int roi = blockIdx.x;
    if (roi >= count) return;
    const SmemView s = smem_view(smem, P);
    const int W = P.width, H = P.height;
    BlockGroup g{s.red};
    uint64_t *mbar = reinterpret_cast<uint64_t *>(reinterpret_cast<uint8_t *>(s.misc) + 32);
    if constexpr (kStaged) {
        if (threadIdx.x == 0) {
            const int bpp = P.pdt == 0 ? 1 : (P.pdt == 1 ? 2 : 4);
            const int n = W * H;
            mbar_init(mbar);
            bulk_load(reinterpret_cast<uint8_t *>(s.img) + (size_t)(4 - bpp) * n, pixels + (int64_t)roi * roi_stride,
                      (uint32_t)(bpp * n), mbar);
        }
    }
    // the job's words are read again for the result (no registers held through QI and Z)
    const int bead = jobs ? (int)reinterpret_cast<const uint32_t *>(jobs)[(size_t)roi * 6 + 2] : 0;
    load_qi_tables(s, P);
    float2 part;
    if constexpr (kStaged) {
        // one thread waits for the copy (its acquire, then the barrier, order the copied bytes
        // before every thread's reads); the others wait at the barrier without polling
        if (threadIdx.x == 0 && !mbar_wait(mbar, 0, kStageWaitLimit) && P.err_flag) atomicOr(P.err_flag, 4u);
        __syncthreads();
        part = convert_staged(g, s.img, P, bead);
    } else {
        const int64_t off = roi_offsets ? roi_offsets[roi] : (int64_t)roi * roi_stride;
        part = load_roi(g, s.img, pixels + off, pitch, P, bead);
    }
    const ComResult com = com_from_sums(g, s.img, W, H, part, P.com_bgcorrection);
    float comx = com.x, comy = com.y;
    if (isnan(comx) || isnan(comy)) {  // QueuedCPUTracker.cpp:294-295
        comx = (float)(W / 2);
        comy = (float)(H / 2);
    }
    float x = comx, y = comy, z = 0.0f;
    bool bhit = false;
    if (P.mode & kLT_QI) qi_localize(s, P, com.mean, x, y, bhit, P.qi_rweights ? s.qrw : nullptr);
    if (P.mode & kLT_LocalizeZ) {
        bhit = check_boundaries(x, y, P.z_maxr, W, H);
        z = z_localize(s, P, com.mean, x, y, bead, roi);
    }
    if (threadIdx.x == 0) {
        uint32_t job[6];
        read_job(jobs, roi, job);
        write_result(results, roi, job, x, y, z, comx, comy, bhit ? 1u : 0u, com.mean);
    }
}

// 2D Gaussian MLE (+ Z) for ROIs above 32x32 or with QI/Z bits: one CTA per ROI on a plain tile.
// Kept apart from the QI kernel so that its register budget is free of the MLE's FP64 solve.
__global__ void __launch_bounds__(kBlockThreads, kMinBlocks)
    localize_gauss_kernel(TrackParams P, const uint8_t *__restrict__ pixels, int pitch, int64_t roi_stride,
                          const int64_t *__restrict__ roi_offsets, const LocalizationJob *__restrict__ jobs, int count,
                          LocalizationResult *__restrict__ results)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int roi = blockIdx.x;
    if (roi >= count) return;
    const SmemView s = smem_view(smem, P);
    uint32_t job[6];
    read_job(jobs, roi, job);
    const int bead = (int)job[2];
    const int64_t off = roi_offsets ? roi_offsets[roi] : (int64_t)roi * roi_stride;
    BlockGroup g{s.red};
    const int W = P.width, H = P.height;
    load_roi(g, s.img, pixels + off, pitch, P, bead);
    const ComResult com = compute_com(g, s.img, W, H, P.com_bgcorrection);
    float comx = com.x, comy = com.y;
    if (isnan(comx) || isnan(comy)) {  // QueuedCPUTracker.cpp:294-295
        comx = (float)(W / 2);
        comy = (float)(H / 2);
    }
    float x = comx, y = comy, z = 0.0f;
    bool bhit = false;
    float *col = reinterpret_cast<float *>(s.work);
    if (P.mode & kLT_Gaussian5P) {
        float p[5] = {x, y, com.mean * 0.5f * (float)(W * H), com.mean * 0.5f, P.g_sigma};
        gauss5_mle(g, s.img, W, H, p, P.g_iterations, col, col + 3 * W);
        x = p[0];
        y = p[1];
        z = p[4];
    } else {
        gauss4_mle(g, s.img, W, H, com.mean, x, y, P.g_iterations, P.g_sigma, col, col + 3 * W);
    }
    __syncthreads();
    if (P.mode & kLT_LocalizeZ) {
        bhit = check_boundaries(x, y, P.z_maxr, W, H);
        z = z_localize(s, P, com.mean, x, y, bead, roi);
    }
    if (threadIdx.x == 0) write_result(results, roi, job, x, y, z, comx, comy, bhit ? 1u : 0u, com.mean);
}

// Gaussian-only mode for ROIs of at most 32x32 pixels: one warp per ROI, 8 ROIs per CTA. Three
// CTAs per SM (80 registers, a few spilled) beat two without spills by 22-35 % on 16x16 ROIs.
__global__ void __launch_bounds__(256, 3) gauss_warp_kernel(TrackParams P, const uint8_t *__restrict__ pixels, int pitch,
                                                         int64_t roi_stride, const int64_t *__restrict__ roi_offsets,
                                                         const LocalizationJob *__restrict__ jobs, int count,
                                                         LocalizationResult *__restrict__ results)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int warp = threadIdx.x >> 5;
    const int roi = blockIdx.x * 8 + warp;
    if (roi >= count) return;  // whole warps exit together
    const int W = P.width, H = P.height;
    const int per_warp = ((W * H + 3 * (W + H) + 3) & ~3) * 4;
    float *img = reinterpret_cast<float *>(smem + warp * per_warp);
    float *col = img + W * H;
    float *row = col + 3 * W;
    uint32_t job[6];
    read_job(jobs, roi, job);
    const int64_t off = roi_offsets ? roi_offsets[roi] : (int64_t)roi * roi_stride;
    WarpGroup g;
    load_roi(g, img, pixels + off, pitch, P, (int)job[2]);
    const ComResult com = compute_com(g, img, W, H, P.com_bgcorrection);
    float comx = com.x, comy = com.y;
    if (isnan(comx) || isnan(comy)) {
        comx = (float)(W / 2);
        comy = (float)(H / 2);
    }
    float x = comx, y = comy, z = 0.0f;
    if (P.mode & kLT_Gaussian5P) {
        float p[5] = {x, y, com.mean * 0.5f * (float)(W * H), com.mean * 0.5f, P.g_sigma};
        gauss5_mle(g, img, W, H, p, P.g_iterations, col, row);
        x = p[0];
        y = p[1];
        z = p[4];
    } else {
        gauss4_mle(g, img, W, H, com.mean, x, y, P.g_iterations, P.g_sigma, col, row);
    }
    if ((threadIdx.x & 31) == 0) write_result(results, roi, job, x, y, z, comx, comy, 0u, com.mean);
}

// One bead of QueuedCPUTracker::BuildLUT (QueuedCPUTracker.cpp:582-645): ROI i of the stack is
// at data + pitch*H*i. Position from known_pos, else COM (no background correction) + QI
// without radial weights (line 603). The profile's fallback value is the tracker's mean,
// which SetImage resets to 0 when known_pos skips the COM (cpu_tracker.h:135).
__global__ void __launch_bounds__(kBlockThreads) build_lut_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                                  int pitch, int nbeads, int plane,
                                                                  const float2 *__restrict__ known_pos,
                                                                  int normalize, float *__restrict__ lut)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int bead = blockIdx.x;
    if (bead >= nbeads) return;
    const SmemView s = smem_view(smem, P);
    load_qi_tables(s, P);
    BlockGroup g{s.red};
    const float2 part = load_roi(g, s.img, pixels + (size_t)pitch * P.height * bead, pitch, P, bead);
    float x, y, mean = 0.0f;
    if (known_pos) {
        x = known_pos[bead].x;
        y = known_pos[bead].y;
    } else {
        const ComResult com = com_from_sums(g, s.img, P.width, P.height, part, 0.0f);
        mean = com.mean;
        x = com.x;
        y = com.y;
        bool bhit;
        qi_localize(s, P, mean, x, y, bhit, nullptr);
    }
    const int nb = P.z_nbins;
    float *prof = reinterpret_cast<float *>(s.work);
    const float rstep = (P.z_maxr - P.z_minr) / (float)nb;
    __syncthreads();
    load_z_tables(s, P);
    __syncthreads();
    radial_profile(s.img, P.width, P.height, P.width, x, y, mean, nb, P.z_angsteps, P.z_minr, rstep, s.zdirs, prof,
                   normalize != 0, s.red);
    float *dst = lut + ((size_t)bead * P.lut_planes + plane) * nb;
    for (int r = threadIdx.x; r < nb; r += blockDim.x) dst[r] += prof[r];
}

// QueuedCPUTracker::FinalizeLUT (QueuedCPUTracker.cpp:648-659): NormalizeRadialProfile
// (utils.cpp:230-261) on every (bead, plane) row. One warp per row.
__global__ void finalize_lut_kernel(float *__restrict__ lut, int rows, int nb)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= rows) return;
    const int lane = threadIdx.x & 31;
    float *p = lut + (size_t)row * nb;
    double s = 0;
    for (int i = lane; i < nb; i += 32) s += p[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    const float m = (float)(s / nb);
    double s2 = 0;
    for (int i = lane; i < nb; i += 32) {
        const float v = p[i] - m;
        p[i] = v;
        s2 += (double)(v * v);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
    const double inv = 1.0 / sqrt(s2 / nb);
    for (int i = lane; i < nb; i += 32) p[i] = (float)((double)p[i] * inv);
}

// ComputeRadialProfile (utils.cpp:275-320) of one float image with a given fallback mean.
__global__ void __launch_bounds__(kBlockThreads) profile_kernel(TrackParams P, const float *__restrict__ img_in,
                                                                float cx, float cy, float mean, int normalize,
                                                                float *__restrict__ out)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const SmemView s = smem_view(smem, P);
    load_z_tables(s, P);
    BlockGroup g{s.red};
    load_roi(g, s.img, reinterpret_cast<const uint8_t *>(img_in), P.width * 4, P, -1);
    float *prof = reinterpret_cast<float *>(s.work);
    const float rstep = (P.z_maxr - P.z_minr) / (float)P.z_nbins;
    radial_profile(s.img, P.width, P.height, P.width, cx, cy, mean, P.z_nbins, P.z_angsteps, P.z_minr, rstep, s.zdirs,
                   prof, normalize != 0, s.red);
    for (int r = threadIdx.x; r < P.z_nbins; r += blockDim.x) out[r] = prof[r];
}

// ------------------------------------------------------------------------------------------
// host-side launchers
// ------------------------------------------------------------------------------------------
static int align16(int v) { return (v + 15) & ~15; }

void plan_smem(TrackParams &P)
{
    const int W = P.width, H = P.height;
    const int nr = P.qi_nr > 0 ? P.qi_nr : 1, L = 2 * nr;
    P.sm_img = 0;
    P.sm_tables = align16(W * H * 4);
    const int qi_tables = P.qi_angpq * 16 + nr * 8 + nr * 4, z_tables = ((P.z_angsteps + 1) >> 1) * 16;
    P.sm_work = P.sm_tables + align16(qi_tables > z_tables ? qi_tables : z_tables);
    // [ ac | A ] (L complex each) + 2 KB of subset partials when the QI directions are split over warps
    const int qi_work = 2 * L * 8 + (nr < kBlockThreads / 4 ? 2048 : 0);
    const int z_work = align16(P.z_nbins * 4) + P.lut_planes * 8;
    const int g_work = (P.mode & kLT_Gaussian2D) ? (3 * W + 3 * H) * 4 : 0;
    int work = qi_work;
    if (z_work > work) work = z_work;
    if (g_work > work) work = g_work;
    P.sm_red = P.sm_work + align16(work);
    constexpr int kRed = kBlockThreads / 32 * 20;  // block_sum scratch: N * warps doubles, N <= 20
    P.sm_misc = P.sm_red + kRed * 8;
    P.smem_bytes = P.sm_misc + 64;
}

int gauss_warp_smem(const TrackParams &P)
{
    const int W = P.width, H = P.height;
    return 8 * ((W * H + 3 * (W + H) + 3) & ~3) * 4;
}

static bool g_attrs_set[64];

cudaError_t prepare_kernels(int device)
{
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    if (g_attrs_set[device]) return cudaSuccess;
    const int max_smem = 227 * 1024;
    cudaError_t e;
    if ((e = cudaFuncSetAttribute(localize_qi_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem)))
        return e;
    if ((e = cudaFuncSetAttribute(localize_qi_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem)))
        return e;
    if ((e = cudaFuncSetAttribute(localize_gauss_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem)))
        return e;
    if ((e = cudaFuncSetAttribute(build_lut_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem))) return e;
    if ((e = cudaFuncSetAttribute(profile_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem))) return e;
    if ((e = cudaFuncSetAttribute(gauss_warp_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, max_smem))) return e;
    g_attrs_set[device] = true;
    return cudaSuccess;
}

bool use_gauss_warp(const TrackParams &P)
{
    return (P.mode & kLT_Gaussian2D) && !(P.mode & (kLT_QI | kLT_LocalizeZ)) && P.width <= 32 && P.height <= 32;
}

cudaError_t launch_localize(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride,
                            const int64_t *roi_offsets, const LocalizationJob *jobs, int count,
                            LocalizationResult *results, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    if (use_com_kernel(P, pixels, pitch, roi_stride, roi_offsets))
        return launch_com(P, pixels, roi_stride, jobs, count, results, stream);
    if (use_gauss_warp(P)) {
        gauss_warp_kernel<<<(count + 7) / 8, 256, gauss_warp_smem(P), stream>>>(P, pixels, pitch, roi_stride,
                                                                              roi_offsets, jobs, count, results);
    } else if ((P.mode & kLT_Gaussian2D) && !(P.mode & kLT_QI)) {
        localize_gauss_kernel<<<count, kBlockThreads, P.smem_bytes, stream>>>(P, pixels, pitch, roi_stride,
                                                                              roi_offsets, jobs, count, results);
    } else {
        // bulk-copy staging: ROIs back to back at a 16-byte aligned stride, and a pixel count for
        // which the copy size and the in-place offset (4 - bpp) n are whole 16-byte units
        const int bpp = P.pdt == 0 ? 1 : (P.pdt == 1 ? 2 : 4);
        const int n = P.width * P.height;
        const bool staged = !roi_offsets && pitch == P.width * bpp && !(reinterpret_cast<uintptr_t>(pixels) & 15) &&
                            !(roi_stride & 15) && !(n & 15);
        if (staged)
            localize_qi_kernel<true><<<count, kBlockThreads, P.smem_bytes, stream>>>(P, pixels, pitch, roi_stride,
                                                                                    roi_offsets, jobs, count, results);
        else
            localize_qi_kernel<false><<<count, kBlockThreads, P.smem_bytes, stream>>>(P, pixels, pitch, roi_stride,
                                                                                     roi_offsets, jobs, count, results);
    }
    return cudaGetLastError();
}

// Bias-table images (QueuedTracker::ComputeZBiasCorrection, cputrack/QueuedTracker.cpp:143-189):
// image i = bead (i / bias_planes) at the ROI centre (w/2, h/2, int division) and
// z = (i % bias_planes) / bias_planes * planes, rendered as GenerateImageFromLUT
// (cputrack/utils.cpp:325-390) does: the bead's LUT interpolated over planes (uniform cubic
// B-spline over 4 planes, or linear), then ovs x ovs samples per pixel, each a linear
// interpolation of that profile at (|offset| - minradius) * bins / (maxradius - minradius),
// clamped to [0, bins - 2]. One block per image; block b renders image first + b into slot b
// of `images` and `jobs` (job: frame = image index, zlutIndex = bead).
__global__ void __launch_bounds__(256) lut_image_kernel(const float *__restrict__ lut, int nb, int planes, int first,
                                                        int bias_planes, int w, int h, float minr, float maxr,
                                                        int ovs, int spline, float *__restrict__ images,
                                                        LocalizationJob *__restrict__ jobs)
{
    extern __shared__ float zi[];  // [nb]
    const int img = first + blockIdx.x;
    const int bead = img / bias_planes, plane = img - bead * bias_planes;
    const float z = plane / (float)bias_planes * planes;
    const float *L = lut + (size_t)bead * planes * nb;
    for (int r = threadIdx.x; r < nb; r += blockDim.x) {
        float v;
        if (spline) {
            const int iz = max(1, min(planes - 3, (int)z));
            const float t = z - iz, t2 = t * t, t3 = t2 * t;
            const float wt[4] = {(1 - 3 * t + 3 * t2 - t3) / 6, (4 - 6 * t2 + 3 * t3) / 6,
                                 (1 + 3 * t + 3 * t2 - 3 * t3) / 6, t3 / 6};
            v = 0.0f;
            for (int i = 0; i < 4; i++) v += wt[i] * L[(i - 1 + iz) * nb + r];
        } else {
            const int iz = (int)z;
            if (iz >= planes - 1) {
                v = L[(planes - 1) * nb + r];
            } else {
                const float a = L[iz * nb + r], b = L[(iz + 1) * nb + r];
                v = a + (b - a) * (z - iz);
            }
        }
        zi[r] = v;
    }
    if (threadIdx.x == 0) {
        LocalizationJob j{};
        j.frame = (uint32_t)img;
        j.zlutIndex = bead;
        jobs[blockIdx.x] = j;
    }
    __syncthreads();
    const float cx = (float)(w / 2), cy = (float)(h / 2);
    const float radialcov = nb / (maxr - minr), step = 1.0f / ovs;
    for (int p = threadIdx.x; p < w * h; p += blockDim.x) {
        const int y = p / w, x = p - y * w;
        float s = 0.0f;
        for (int ox = 0; ox < ovs; ox++)
            for (int oy = 0; oy < ovs; oy++) {
                const float X = x + (ox + 0.5f) * step - cx - 0.5f;
                const float Y = y + (oy + 0.5f) * step - cy - 0.5f;
                float r = (sqrtf(X * X + Y * Y) - minr) * radialcov;
                if (r > nb - 2) r = (float)(nb - 2);
                if (r < 0) r = 0;
                const int i = (int)r;
                s += zi[i] + (zi[i + 1] - zi[i]) * (r - i);
            }
        images[(size_t)blockIdx.x * w * h + p] = s / (ovs * ovs);
    }
}

cudaError_t launch_lut_images(const float *lut, int nb, int planes, int first_image, int n_images, int bias_planes,
                              int w, int h, float minr, float maxr, int ovs, bool spline, float *images,
                              LocalizationJob *jobs, cudaStream_t stream)
{
    if (n_images <= 0) return cudaSuccess;
    lut_image_kernel<<<n_images, 256, sizeof(float) * nb, stream>>>(lut, nb, planes, first_image, bias_planes, w, h,
                                                                    minr, maxr, ovs, spline ? 1 : 0, images, jobs);
    return cudaGetLastError();
}

void localize_node(const TrackParams &P, int count, cudaKernelNodeParams &kp)
{
    kp = cudaKernelNodeParams{};
    if (use_gauss_warp(P)) {
        kp.func = reinterpret_cast<void *>(gauss_warp_kernel);
        kp.gridDim = dim3((count + 7) / 8);
        kp.blockDim = dim3(256);
        kp.sharedMemBytes = gauss_warp_smem(P);
    } else {
        kp.func = (P.mode & kLT_Gaussian2D) && !(P.mode & kLT_QI) ? reinterpret_cast<void *>(localize_gauss_kernel)
                                                                   : reinterpret_cast<void *>(localize_qi_kernel<false>);
        kp.gridDim = dim3(count);
        kp.blockDim = dim3(kBlockThreads);
        kp.sharedMemBytes = P.smem_bytes;
    }
}

cudaError_t launch_build_lut(const TrackParams &P, const uint8_t *pixels, int pitch, int nbeads, int plane,
                             const float2 *known_pos, bool normalize, float *lut, cudaStream_t stream)
{
    if (nbeads <= 0) return cudaSuccess;
    build_lut_kernel<<<nbeads, kBlockThreads, P.smem_bytes, stream>>>(P, pixels, pitch, nbeads, plane, known_pos,
                                                                      normalize ? 1 : 0, lut);
    return cudaGetLastError();
}

cudaError_t launch_finalize_lut(float *lut, int rows, int nb, cudaStream_t stream)
{
    if (rows <= 0) return cudaSuccess;
    finalize_lut_kernel<<<(rows + 7) / 8, 256, 0, stream>>>(lut, rows, nb);
    return cudaGetLastError();
}

// lut [count][planes][nb] -> lut_t [count][nb][pitch], planes pitch..planes-1 of each bin zero.
// Reads are strided, writes coalesced; it runs once per LUT change.
__global__ void transpose_lut_kernel(const float *__restrict__ lut, int count, int planes, int nb, int pitch,
                                     float *__restrict__ lut_t)
{
    const size_t total = (size_t)count * nb * pitch;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(i % pitch);
        const size_t br = i / pitch;
        const int r = (int)(br % nb);
        const size_t b = br / nb;
        lut_t[i] = k < planes ? lut[(b * planes + k) * nb + r] : 0.0f;
    }
}

cudaError_t launch_transpose_lut(const float *lut, int count, int planes, int nb, int pitch, float *lut_t,
                                 cudaStream_t stream)
{
    const size_t total = (size_t)count * nb * pitch;
    if (total == 0) return cudaSuccess;
    const int blocks = (int)std::min<size_t>((total + 255) / 256, 148 * 16);
    transpose_lut_kernel<<<blocks, 256, 0, stream>>>(lut, count, planes, nb, pitch, lut_t);
    return cudaGetLastError();
}

cudaError_t launch_profile(const TrackParams &P, const float *img, float cx, float cy, float mean, bool normalize,
                           float *out, cudaStream_t stream)
{
    profile_kernel<<<1, kBlockThreads, P.smem_bytes, stream>>>(P, img, cx, cy, mean, normalize ? 1 : 0, out);
    return cudaGetLastError();
}

}  // namespace qtrk
