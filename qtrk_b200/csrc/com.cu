// Centre-of-mass kernels for LT_OnlyCOM (sm_100a).
//
// CPUTracker::ComputeMeanAndCOM (cputrack/cpu_tracker.cpp:681-729) needs two passes over a ROI:
// mean and standard deviation first, then the background-corrected moments
//   v' = max(0, |v - mean| - bgcorrection * stdev),  COM = (sum x v', sum y v') / sum v'.
// The fused localization kernel stages every ROI as a float tile in shared memory because QI and
// the radial profile sample it many times; a COM-only localization reads each pixel twice and
// needs no tile. Three forms, by ROI size:
//  - com_warp_kernel (ROIs up to 55 KB): a group of 2-4 warps per ROI and one shared-memory buffer
//    per group, filled by a bulk copy; both passes run over the raw buffer and the sums meet
//    through warp shuffles and a named barrier per group, with no CTA-wide barrier;
//  - com_stream_kernel: one CTA per ROI in flight with a ring of bulk-copied buffers, the ROI read
//    into registers once;
//  - com_kernel (ROIs whose ring does not fit): one CTA per ROI, the ROI loaded into registers.
// The sums meet in FP64, as the reference accumulates in FP64; per-thread partial sums are FP32
// over at most 64 pixels (exact for the mean of u8/u16 data, ~1e-7 relative for the moments), or
// exact integers in the warp-group form's first pass.
//
// Moments per chunk: a chunk of ppc pixels starts at pixel i0 = (x0, y0) and may cross one row
// end (at j = W - x0). With S = sum_j v'_j, Sj = sum_j j v'_j and Sw = sum_{j >= W - x0} v'_j,
// sum x v' = x0 S + Sj - W Sw and sum y v' = y0 S + Sw, so each pixel costs two adds and one
// multiply-add on top of the background correction, and only chunks that cross a row end pay
// for Sw.
#include <cstdint>
#include <mutex>

#include <cuda_runtime.h>

#include "bulk_copy.cuh"
#include "device_common.cuh"
#include "kernels.h"

namespace qtrk {

namespace {

constexpr int kComMaxThreads = 1024;

// Pixels per 16-byte chunk, and the most chunks a thread holds (at most 40 pixels: more float
// registers than that spill under the 64-register budget of a 1024-thread CTA).
template <int PDT>
struct ChunkPixels;
template <>
struct ChunkPixels<0> {
    static constexpr int n = 16, max_chunks = 2;
};
template <>
struct ChunkPixels<1> {
    static constexpr int n = 8, max_chunks = 5;
};
template <>
struct ChunkPixels<2> {
    static constexpr int n = 4, max_chunks = 8;
};

// A 16-byte chunk as floats. Integer pixels are placed in the mantissa of 2^23 by one byte
// permute and 2^23 is subtracted (exact for values below 2^23).
template <int PDT>
__device__ __forceinline__ void unpack(const uint4 &q, float (&v)[ChunkPixels<PDT>::n])
{
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
    if (PDT == 0) {
#pragma unroll
        for (int k = 0; k < 4; k++)
#pragma unroll
            for (int b = 0; b < 4; b++)
                v[4 * k + b] = __uint_as_float(__byte_perm(w[k], 0x4B000000u, 0x7540u + b)) - 8388608.0f;
    } else if (PDT == 1) {
#pragma unroll
        for (int k = 0; k < 4; k++) {
            v[2 * k] = __uint_as_float(__byte_perm(w[k], 0x4B000000u, 0x7410u)) - 8388608.0f;
            v[2 * k + 1] = __uint_as_float(__byte_perm(w[k], 0x4B000000u, 0x7432u)) - 8388608.0f;
        }
    } else {
#pragma unroll
        for (int k = 0; k < 4; k++) v[k] = __uint_as_float(w[k]);
    }
}

// Sum N doubles over the CTA (blockDim.x a multiple of 32, at most 1024); every thread gets the
// totals. red: 32 x N doubles of shared memory. Two barriers.
template <int N>
__device__ __forceinline__ void cta_sum(double (&v)[N], double (*red)[N])
{
#pragma unroll
    for (int k = 0; k < N; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; k++) red[warp][k] = v[k];
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int k = 0; k < N; k++) {
            double s = lane < nw ? red[lane][k] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) red[0][k] = s;
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; k++) v[k] = red[0][k];
}

}  // namespace

namespace {

constexpr int kComMaxStages = 4;
constexpr uint32_t kComWaitLimit = 1u << 22;  // mbarrier polls before a staged ROI counts as lost

// Where this thread's first chunk starts (pixel t * ppc of the ROI, as float column and row) and
// how far its next chunk is (T * ppc pixels: fdx columns and fdy rows, fdx < W), so that pass 2
// walks its chunks with float counters instead of dividing by W per chunk.
struct ChunkWalk {
    float fx, fy, fdx, fdy;
};

__device__ __forceinline__ ChunkWalk chunk_walk(int t, int T, int ppc, int W)
{
    const int i0 = t * ppc, step = T * ppc;
    ChunkWalk w;
    w.fx = (float)(i0 % W);
    w.fy = (float)(i0 / W);
    w.fdx = (float)(step % W);
    w.fdy = (float)(step / W);
    return w;
}

// The moments of one chunk at walk position w (see the chunk moments above), added to the FP32
// sums q0 (v'), qx (x v') and qy (y v'). kThr: a background threshold is set (v' = max(0, |v -
// mean| - thr)); without one v' = |v - mean| exactly.
template <int PDT, bool kThr>
__device__ __forceinline__ void chunk_moments(const float (&v)[ChunkPixels<PDT>::n], const ChunkWalk &w, float fW,
                                              float mean, float thr, float &q0, float &qx, float &qy)
{
    constexpr int ppc = ChunkPixels<PDT>::n;
    float a[ppc];
    float S = 0.0f, Sj = 0.0f;
#pragma unroll
    for (int j = 0; j < ppc; j++) {
        a[j] = kThr ? fmaxf(0.0f, fabsf(v[j] - mean) - thr) : fabsf(v[j] - mean);
        S += a[j];
        if (j > 0) Sj = fmaf((float)j, a[j], Sj);
    }
    const float split = fW - w.fx;  // first j on the next row
    float Sw = 0.0f;
    if (split < (float)ppc) {
#pragma unroll
        for (int j = 0; j < ppc; j++)
            if ((float)j >= split) Sw += a[j];
    }
    q0 += S;
    qx += fmaf(w.fx, S, Sj) - fW * Sw;
    qy += fmaf(w.fy, S, Sw);
}

// chunk_moments for a chunk of 8 u16 pixels without a background threshold, on packed FP32x2
// pairs: v - mean is formed per pixel exactly as the scalar form forms it (the pixel is exact in
// FP32), and the sums S and Sj run as two interleaved halves added at the end. Chunks start at
// multiples of 8 pixels, so with W a multiple of 8 no chunk crosses a row end, and with W = 8k + 4
// a chunk that does crosses it after its fourth pixel (rows start at 0 or 4 mod 8): then the pixels
// on the next row are the second half, whose sum the packed additions already form. wmod8 = W % 8.
__device__ __forceinline__ void chunk_moments_u16(const uint4 &q, const ChunkWalk &w, float fW, int wmod8, float mean,
                                                  float &q0, float &qx, float &qy)
{
    const float2 nK = make_float2(-8388608.0f, -8388608.0f), nm = make_float2(-mean, -mean);
    const uint32_t wd[4] = {q.x, q.y, q.z, q.w};
    float2 a[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const float2 x = make_float2(__uint_as_float(__byte_perm(wd[k], 0x4B000000u, 0x7410u)),
                                     __uint_as_float(__byte_perm(wd[k], 0x4B000000u, 0x7432u)));
        const float2 d = __fadd2_rn(__fadd2_rn(x, nK), nm);
        a[k] = make_float2(fabsf(d.x), fabsf(d.y));
    }
    const float2 h23 = __fadd2_rn(a[2], a[3]);
    const float2 S2 = __fadd2_rn(__fadd2_rn(a[0], a[1]), h23);
    float2 J2 = __fmul2_rn(a[0], make_float2(0.0f, 1.0f));
    J2 = __ffma2_rn(a[1], make_float2(2.0f, 3.0f), J2);
    J2 = __ffma2_rn(a[2], make_float2(4.0f, 5.0f), J2);
    J2 = __ffma2_rn(a[3], make_float2(6.0f, 7.0f), J2);
    const float S = S2.x + S2.y, Sj = J2.x + J2.y;
    const float split = fW - w.fx;  // first j on the next row
    float Sw = 0.0f;
    if (wmod8 == 4) {
        if (split < 8.0f) Sw = h23.x + h23.y;
    } else if (wmod8 != 0 && split < 8.0f) {
#pragma unroll
        for (int j = 0; j < 8; j++)
            if ((float)j >= split) Sw += (j & 1) ? a[j >> 1].y : a[j >> 1].x;
    }
    q0 += S;
    qx += fmaf(w.fx, S, Sj) - fW * Sw;
    qy += fmaf(w.fy, S, Sw);
}

__device__ __forceinline__ void walk_step(ChunkWalk &w, float fW)
{
    w.fx += w.fdx;
    w.fy += w.fdy;
    if (w.fx >= fW) {
        w.fx -= fW;
        w.fy += 1.0f;
    }
}

// Pass 2 of ComputeMeanAndCOM on this thread's chunks t, t + T, ... (K of them, those below
// nchunks): the FP32 partial sums of v', x v' and y v'.
template <int PDT, int K, bool kThr>
__device__ __forceinline__ float3 com_moments(const float (&v)[K][ChunkPixels<PDT>::n], ChunkWalk w, int t, int T,
                                              int nchunks, int W, float mean, float thr)
{
    const float fW = (float)W;
    float q0 = 0.0f, qx = 0.0f, qy = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) {
        if (t + k * T < nchunks) chunk_moments<PDT, kThr>(v[k], w, fW, mean, thr, q0, qx, qy);
        walk_step(w, fW);
    }
    return make_float3(q0, qx, qy);
}

// Pass 1 partial sums (v, and v^2 when a background threshold needs the standard deviation) of
// this thread's converted pixels.
template <int PDT, int K>
__device__ __forceinline__ float2 com_pass1(const float (&v)[K][ChunkPixels<PDT>::n], bool squares)
{
    constexpr int ppc = ChunkPixels<PDT>::n;
    float s = 0.0f, s2 = 0.0f;
    if (squares) {
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
            for (int j = 0; j < ppc; j++) {
                s += v[k][j];
                s2 = fmaf(v[k][j], v[k][j], s2);
            }
    } else {
#pragma unroll
        for (int k = 0; k < K; k++)
#pragma unroll
            for (int j = 0; j < ppc; j++) s += v[k][j];
    }
    return make_float2(s, s2);
}

// The 13-word LocalizationResult of a COM-only localization (thread 0).
__device__ __forceinline__ void com_result(LocalizationResult *results, int roi, const LocalizationJob *jobs,
                                           const double (&m)[3], float mean, int W, int H)
{
    float cx = (float)(m[1] / m[0]), cy = (float)(m[2] / m[0]);
    if (isnan(cx) || isnan(cy)) {  // QueuedCPUTracker.cpp:294-295
        cx = (float)(W / 2);
        cy = (float)(H / 2);
    }
    uint32_t *o = reinterpret_cast<uint32_t *>(results) + (size_t)roi * 13;
    if (jobs) {
        const uint32_t *p = reinterpret_cast<const uint32_t *>(jobs) + (size_t)roi * 6;
#pragma unroll
        for (int k = 0; k < 6; k++) o[k] = p[k];
    } else {
        o[0] = (uint32_t)roi;
#pragma unroll
        for (int k = 1; k < 6; k++) o[k] = 0u;
    }
    o[6] = __float_as_uint(cx);
    o[7] = __float_as_uint(cy);
    o[8] = 0u;
    o[9] = __float_as_uint(cx);
    o[10] = __float_as_uint(cy);
    o[11] = 0u;
    o[12] = __float_as_uint(mean);
}

}  // namespace

// One CTA per ROI; ROI r is the n*bpp bytes at pixels + r * roi_stride (16-byte aligned, n*bpp a
// multiple of 16). Thread t holds chunks t, t + T, ..., t + (K-1) T.
template <int PDT, int K>
__global__ void __launch_bounds__(kComMaxThreads) com_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                              int64_t roi_stride,
                                                              const LocalizationJob *__restrict__ jobs, int count,
                                                              LocalizationResult *__restrict__ results)
{
    constexpr int ppc = ChunkPixels<PDT>::n;
    __shared__ double red2[32][2];
    __shared__ double red3[32][3];
    const int roi = blockIdx.x;
    if (roi >= count) return;
    const int W = P.width, n = W * P.height, nchunks = n / ppc, T = blockDim.x, t = threadIdx.x;
    const uint4 *src = reinterpret_cast<const uint4 *>(pixels + (int64_t)roi * roi_stride);
    uint4 q[K];
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int c = t + k * T;
        q[k] = c < nchunks ? __ldcs(src + c) : make_uint4(0, 0, 0, 0);
    }
    float v[K][ppc];
#pragma unroll
    for (int k = 0; k < K; k++) unpack<PDT>(q[k], v[k]);
    if ((P.mode & kLT_ClearFirstFourPixels) && t == 0)  // QueuedCPUTracker.cpp:280-282
#pragma unroll
        for (int j = 0; j < 4; j++) v[0][j] = 0.0f;

    // pass 1: sum and, for a background threshold, sum of squares (chunks past the ROI hold zeros)
    const bool bg = P.com_bgcorrection != 0.0f;
    const float2 p1 = com_pass1<PDT, K>(v, bg);
    double m1[2] = {(double)p1.x, (double)p1.y};
    cta_sum<2>(m1, red2);
    const float invN = 1.0f / (float)n;
    const float mean = (float)(m1[0] * (double)invN);
    const float stdev = sqrtf((float)(m1[1] * (double)invN - (double)(mean * mean)));
    const float thr = P.com_bgcorrection * stdev;

    // pass 2: background-corrected moments
    const ChunkWalk wk = chunk_walk(t, T, ppc, W);
    const float3 mo = bg ? com_moments<PDT, K, true>(v, wk, t, T, nchunks, W, mean, thr)
                         : com_moments<PDT, K, false>(v, wk, t, T, nchunks, W, mean, 0.0f);
    double m2[3] = {(double)mo.x, (double)mo.y, (double)mo.z};
    cta_sum<3>(m2, red3);
    if (t == 0) com_result(results, roi, jobs, m2, mean, W, P.height);
}


// The streaming form: CTAs stay resident (the grid is what fits on the GPU) and walk the ROIs
// r = blockIdx.x, blockIdx.x + gridDim.x, ...; each keeps `stages` ROIs in flight in a ring of
// shared-memory buffers, filled by bulk copies (cp.async.bulk, one per ROI, issued by thread 0,
// completion on one mbarrier per buffer). A ROI's buffer is read into registers once (16-byte
// shared loads, conversion to float), its buffer refilled with the ROI `stages` steps ahead as soon
// as every thread has read it, and both passes of the COM run on the registers, so HBM keeps
// streaming while the CTA reduces. ring_stride: bytes per buffer (the ROI's bytes rounded up to
// 128).
template <int PDT, int K>
__global__ void __launch_bounds__(kComMaxThreads) com_stream_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                                     int64_t roi_stride,
                                                                     const LocalizationJob *__restrict__ jobs,
                                                                     int count, LocalizationResult *__restrict__ results,
                                                                     int stages, int ring_stride)
{
    constexpr int ppc = ChunkPixels<PDT>::n;
    extern __shared__ __align__(128) uint8_t ring[];
    __shared__ uint64_t mbar[kComMaxStages];
    __shared__ double red2[32][2];
    __shared__ double red3[32][3];
    const int W = P.width, H = P.height, n = W * H, nchunks = n / ppc, T = blockDim.x, t = threadIdx.x;
    const int G = gridDim.x;
    const uint32_t bytes = (uint32_t)(n * (16 / ppc));
    if ((int)blockIdx.x >= count) return;
    if (t == 0) {
        for (int s = 0; s < stages; s++) mbar_init(&mbar[s]);
        for (int s = 0; s < stages; s++) {
            const int r = blockIdx.x + s * G;
            if (r < count) bulk_load(ring + (size_t)s * ring_stride, pixels + (int64_t)r * roi_stride, bytes, &mbar[s]);
        }
    }
    __syncthreads();
    const float invN = 1.0f / (float)n;
    const bool bg = P.com_bgcorrection != 0.0f;
    const ChunkWalk wk = chunk_walk(t, T, ppc, W);
    int it = 0;
    for (int roi = blockIdx.x; roi < count; roi += G, it++) {
        const int s = it % stages;
        if (!mbar_wait(&mbar[s], (uint32_t)(it / stages) & 1u, kComWaitLimit) && P.err_flag)
            atomicOr(P.err_flag, 4u);
        const uint4 *src = reinterpret_cast<const uint4 *>(ring + (size_t)s * ring_stride);
        float v[K][ppc];
#pragma unroll
        for (int k = 0; k < K; k++) {
            const int c = t + k * T;
            unpack<PDT>(c < nchunks ? src[c] : make_uint4(0, 0, 0, 0), v[k]);
        }
        if ((P.mode & kLT_ClearFirstFourPixels) && t == 0)  // QueuedCPUTracker.cpp:280-282
#pragma unroll
            for (int j = 0; j < 4; j++) v[0][j] = 0.0f;
        const float2 p1 = com_pass1<PDT, K>(v, bg);
        double m1[2] = {(double)p1.x, (double)p1.y};
        cta_sum<2>(m1, red2);  // every thread has read buffer s
        if (t == 0) {
            const int r = roi + stages * G;
            if (r < count) bulk_load(ring + (size_t)s * ring_stride, pixels + (int64_t)r * roi_stride, bytes, &mbar[s]);
        }
        const float mean = (float)(m1[0] * (double)invN);
        const float stdev = sqrtf((float)(m1[1] * (double)invN - (double)(mean * mean)));
        const float3 q = bg ? com_moments<PDT, K, true>(v, wk, t, T, nchunks, W, mean, P.com_bgcorrection * stdev)
                            : com_moments<PDT, K, false>(v, wk, t, T, nchunks, W, mean, 0.0f);
        double m2[3] = {(double)q.x, (double)q.y, (double)q.z};
        cta_sum<3>(m2, red3);
        if (t == 0) com_result(results, roi, jobs, m2, mean, W, H);
    }
}

namespace {

constexpr int kComWarpGroup = 32;  // pixels per FP32 partial sum before it is folded into FP64
constexpr int kComMaxGroups = 15;  // ROI buffers per CTA of the warp-group form (named barriers 1..15)

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace

// Named barrier over the `n` threads of one warp group (id 1..15; 0 is __syncthreads).
__device__ __forceinline__ void group_sync(int id, int n)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory");
}

// The same barrier, returning whether `v` holds in every thread of the group.
__device__ __forceinline__ bool group_all(bool v, int id, int n)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(n)
        : "memory");
    return r != 0;
}

// The warp-group form: a group of `wg` warps (1, 2 or 4) per ROI and one shared-memory buffer
// (buf_stride bytes) per group, with no CTA-wide barrier. A bulk copy (cp.async.bulk, completion
// on the group's mbarrier) fills the buffer with the group's ROI; the group runs both passes of
// ComputeMeanAndCOM over it (16-byte shared loads; thread t of the group on chunks t, t + 32 wg,
// ...), reduces with shuffles and then across its warps through a named barrier, writes the
// result, and only then starts the copy of its next ROI into the same buffer. The other groups of
// the SM keep the copy engine busy meanwhile, so each group's copy latency is hidden by its
// neighbours' work; splitting a ROI over several warps puts more warps on the SM than there are
// buffers. Pass 1 of integer pixels without a background threshold is an exact integer sum
// (dp2a / dp4a); otherwise FP32 partial sums over 32 pixels are folded into FP64, as in the CTA
// form. Every warp of a group adds the group's partials in the same order, so all hold the same
// totals.
template <int PDT>
__global__ void __launch_bounds__(1024, 1) com_warp_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                            int64_t roi_stride, const LocalizationJob *__restrict__ jobs,
                                                            int count, LocalizationResult *__restrict__ results,
                                                            int buf_stride, int wg)
{
    constexpr int ppc = ChunkPixels<PDT>::n, G = kComWarpGroup / ppc < 1 ? 1 : kComWarpGroup / ppc;
    extern __shared__ __align__(128) uint8_t bufs[];
    __shared__ uint64_t mbar[kComMaxGroups];
    __shared__ double red1[kComMaxGroups][4][2];
    __shared__ double red2[kComMaxGroups][4][3];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int grp = warp / wg, r = warp - grp * wg, ngrp = (blockDim.x >> 5) / wg;
    const int T = 32 * wg, t = 32 * r + lane, bar_id = 1 + grp;
    const bool leader = t == 0;
    const int W = P.width, H = P.height, n = W * H, nchunks = n / ppc;
    const uint32_t bytes = (uint32_t)(n * (16 / ppc));
    uint8_t *gbuf = bufs + (size_t)grp * buf_stride;
    const uint4 *buf = reinterpret_cast<const uint4 *>(gbuf);
    uint64_t *mb = &mbar[grp];
    const int stride = gridDim.x * ngrp;
    int roi = blockIdx.x * ngrp + grp;
    if (leader) {
        mbar_init(mb);
        if (roi < count) bulk_load(gbuf, pixels + (int64_t)roi * roi_stride, bytes, mb);
    }
    const bool clear4 = (P.mode & kLT_ClearFirstFourPixels) != 0;
    const bool bg = P.com_bgcorrection != 0.0f;
    const float invN = 1.0f / (float)n, fW = (float)W;
    const int wmod8 = W & 7;
    const ChunkWalk wk0 = chunk_walk(t, T, ppc, W);
    for (uint32_t it = 0; roi < count; roi += stride, it++) {
        // the leader waits for the copy; the barrier passes the completed copy (and, on the
        // first ROI, the mbarrier's initialisation) to the group, and makes the outcome uniform
        const bool ok = leader ? mbar_wait(mb, it & 1u, kComWaitLimit) : true;
        // LT_ClearFirstFourPixels (QueuedCPUTracker.cpp:280-282): the leader zeroes them in the buffer once
        // the copy has landed; the barrier below orders that before every thread's reads
        if (leader && ok && clear4)
            for (int k = 0; k < 16 / ppc; k++) reinterpret_cast<uint32_t *>(gbuf)[k] = 0u;
        if (!group_all(ok, bar_id, T)) {
            // the copy did not complete: flag it, give it a last bounded wait (it writes into this
            // CTA's shared memory) and stop the group
            if (leader) {
                if (P.err_flag) atomicOr(P.err_flag, 4u);
                mbar_wait(mb, it & 1u, kComWaitLimit);
            }
            return;
        }
        // pass 1: sum (and sum of squares for a background threshold)
        double m1[2] = {0.0, 0.0};
        if (PDT != 2 && !bg) {
            uint32_t si = 0u;  // exact below 2^20 pixels (u16)
            for (int c = t; c < nchunks; c += T) {
                const uint4 q = buf[c];
                if (PDT == 0) {
                    si = __dp4a(q.x, 0x01010101u, si);
                    si = __dp4a(q.y, 0x01010101u, si);
                    si = __dp4a(q.z, 0x01010101u, si);
                    si = __dp4a(q.w, 0x01010101u, si);
                } else {
                    si = __dp2a_lo(q.x, 0x0101u, si);
                    si = __dp2a_lo(q.y, 0x0101u, si);
                    si = __dp2a_lo(q.z, 0x0101u, si);
                    si = __dp2a_lo(q.w, 0x0101u, si);
                }
            }
            m1[0] = (double)si;
        } else {
            for (int c0 = t; c0 < nchunks; c0 += T * G) {
                float s = 0.0f, s2 = 0.0f;
#pragma unroll
                for (int g = 0; g < G; g++) {
                    const int c = c0 + T * g;
                    if (c < nchunks) {
                        float v[ppc];
                        unpack<PDT>(buf[c], v);
#pragma unroll
                        for (int j = 0; j < ppc; j++) {
                            s += v[j];
                            s2 = fmaf(v[j], v[j], s2);
                        }
                    }
                }
                m1[0] += (double)s;
                m1[1] += (double)s2;
            }
        }
        m1[0] = warp_sum(m1[0]);
        if (bg) m1[1] = warp_sum(m1[1]);
        if (lane == 0) {
            red1[grp][r][0] = m1[0];
            red1[grp][r][1] = m1[1];
        }
        group_sync(bar_id, T);
        m1[0] = m1[1] = 0.0;
        for (int k = 0; k < wg; k++) {
            m1[0] += red1[grp][k][0];
            m1[1] += red1[grp][k][1];
        }
        const float mean = (float)(m1[0] * (double)invN);
        const float thr = bg ? P.com_bgcorrection * sqrtf((float)(m1[1] * (double)invN - (double)(mean * mean))) : 0.0f;
        // pass 2: background-corrected moments
        double m2[3] = {0.0, 0.0, 0.0};
        ChunkWalk w = wk0;
        for (int c0 = t; c0 < nchunks; c0 += T * G) {
            float q0 = 0.0f, qx = 0.0f, qy = 0.0f;
#pragma unroll
            for (int g = 0; g < G; g++) {
                const int c = c0 + T * g;
                if (c < nchunks) {
                    const uint4 q = buf[c];
                    if (PDT == 1 && !bg) {
                        chunk_moments_u16(q, w, fW, wmod8, mean, q0, qx, qy);
                    } else {
                        float v[ppc];
                        unpack<PDT>(q, v);
                        if (bg)
                            chunk_moments<PDT, true>(v, w, fW, mean, thr, q0, qx, qy);
                        else
                            chunk_moments<PDT, false>(v, w, fW, mean, 0.0f, q0, qx, qy);
                    }
                }
                walk_step(w, fW);
            }
            m2[0] += (double)q0;
            m2[1] += (double)qx;
            m2[2] += (double)qy;
        }
#pragma unroll
        for (int k = 0; k < 3; k++) m2[k] = warp_sum(m2[k]);
        if (lane == 0)
#pragma unroll
            for (int k = 0; k < 3; k++) red2[grp][r][k] = m2[k];
        // after this barrier every thread of the group has finished reading the buffer, so the
        // leader may start the next copy into it
        group_sync(bar_id, T);
        if (leader) {
            double m[3] = {0.0, 0.0, 0.0};
            for (int k = 0; k < wg; k++)
#pragma unroll
                for (int q = 0; q < 3; q++) m[q] += red2[grp][k][q];
            com_result(results, roi, jobs, m, mean, W, H);
            const int next = roi + stride;
            if (next < count) bulk_load(gbuf, pixels + (int64_t)next * roi_stride, bytes, mb);
        }
    }
}

namespace {

using ComWarpKernel = void (*)(TrackParams, const uint8_t *, int64_t, const LocalizationJob *, int,
                               LocalizationResult *, int, int);

// Buffers (ROIs in flight) and warps per ROI of the warp-group form: as many ROI buffers as fit in
// 220 KB, at most 15, and the most warps per ROI (1, 2 or 4) that keep the CTA within 32 warps.
// Fewer than 4 buffers (ROIs above 55 KB) leaves the ROI to the CTA forms.
bool com_warp_plan(int64_t roi_bytes, int &groups, int &wg, int &stride)
{
    stride = (int)((roi_bytes + 127) & ~(int64_t)127);
    groups = (int)((220 * 1024) / stride);
    if (groups > kComMaxGroups) groups = kComMaxGroups;
    wg = 4;
    while (wg > 1 && groups * wg > 32) wg >>= 1;
    return groups >= 4;
}

using ComKernel = void (*)(TrackParams, const uint8_t *, int64_t, const LocalizationJob *, int, LocalizationResult *);
using ComStreamKernel = void (*)(TrackParams, const uint8_t *, int64_t, const LocalizationJob *, int,
                                 LocalizationResult *, int, int);

template <int PDT, int K>
ComStreamKernel com_stream_at(int k)
{
    if constexpr (K > ChunkPixels<PDT>::max_chunks)
        return nullptr;
    else
        return k == K ? com_stream_kernel<PDT, K> : com_stream_at<PDT, K + 1>(k);
}

// Ring of the streaming form: 3 buffers while they fit in 72 KB (3 CTAs of 320 threads per SM
// for 100x100 u16 ROIs), else 2 within 200 KB; larger ROIs take the one-CTA-per-ROI form.
bool com_stream_plan(int64_t roi_bytes, int &stages, int &stride)
{
    stride = (int)((roi_bytes + 127) & ~(int64_t)127);
    if (3 * (int64_t)stride <= 72 * 1024)
        stages = 3;
    else if (2 * (int64_t)stride <= 200 * 1024)
        stages = 2;
    else
        return false;
    return true;
}

// CTAs of a streaming COM kernel that fit on the current device at once (cached per kernel,
// device and shared-memory size); 0 when the query fails. The kernel's dynamic shared-memory limit
// is raised to the device's opt-in maximum (less its static shared memory) rather than to `smem`,
// so that a later query for a smaller size cannot lower it under a size already cached.
int com_stream_ctas(ComStreamKernel f, int threads, int smem)
{
    struct Entry {
        ComStreamKernel f;
        int device, threads, smem, ctas;
    };
    static std::mutex mu;
    static Entry cache[64];
    static int ncache = 0;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        std::lock_guard<std::mutex> lk(mu);
        for (int i = 0; i < ncache; i++)
            if (cache[i].f == f && cache[i].device == dev && cache[i].threads == threads && cache[i].smem == smem)
                return cache[i].ctas;
    }
    int per_sm = 0, sms = 0, optin = 0;
    cudaFuncAttributes fa{};
    if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, f) != cudaSuccess || smem > optin - (int)fa.sharedSizeBytes ||
        cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)fa.sharedSizeBytes) !=
            cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f, threads, smem) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const int ctas = per_sm * sms;
    std::lock_guard<std::mutex> lk(mu);
    if (ncache < 64) cache[ncache++] = Entry{f, dev, threads, smem, ctas};
    return ctas;
}

// com_kernel<PDT, K> for K = k (1 <= k <= ChunkPixels<PDT>::max_chunks)
template <int PDT, int K>
ComKernel com_kernel_at(int k)
{
    if constexpr (K > ChunkPixels<PDT>::max_chunks)
        return nullptr;
    else
        return k == K ? com_kernel<PDT, K> : com_kernel_at<PDT, K + 1>(k);
}

#ifndef QTRK_COM_PIXELS_PER_THREAD
#define QTRK_COM_PIXELS_PER_THREAD 32
#endif

int bytes_per_pixel(int pdt) { return pdt == 0 ? 1 : (pdt == 1 ? 2 : 4); }

}  // namespace

// Threads per CTA (a multiple of 32, 64..1024) and chunks per thread for a ROI of P's size, or
// false when the ROI does not fit the register-held form (more than 1024 threads' worth of
// chunks, a size that is not a whole number of 16-byte chunks, or rows shorter than a chunk).
bool com_shape(const TrackParams &P, int &threads, int &chunks)
{
    const int bpp = bytes_per_pixel(P.pdt), ppc = 16 / bpp;
    const int64_t bytes = (int64_t)P.width * P.height * bpp;
    if (bytes <= 0 || bytes % 16) return false;
    if (P.width < ppc) return false;  // a chunk may cross at most one row end
    const int nchunks = (int)(bytes / 16);
    const int kmax = P.pdt == 0 ? ChunkPixels<0>::max_chunks
                                : (P.pdt == 1 ? ChunkPixels<1>::max_chunks : ChunkPixels<2>::max_chunks);
    int k = QTRK_COM_PIXELS_PER_THREAD / ppc;
    if (k < 1) k = 1;
    if (k > kmax) k = kmax;
    int T = (nchunks + k - 1) / k;
    T = (T + 31) & ~31;
    if (T < 64) T = 64;
    if (T > kComMaxThreads) T = kComMaxThreads;
    k = (nchunks + T - 1) / T;
    if (k > kmax) return false;
    threads = T;
    chunks = k;
    return true;
}

bool use_com_kernel(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride,
                    const int64_t *roi_offsets)
{
    if (P.mode & (kLT_QI | kLT_Gaussian2D | kLT_LocalizeZ)) return false;
    if (P.calib_offset || P.calib_gain) return false;  // per-bead calibration: the fused kernel applies it
    if (roi_offsets) return false;                       // ROIs cropped from frame rows
    const int bpp = bytes_per_pixel(P.pdt);
    if (pitch != P.width * bpp) return false;
    if ((reinterpret_cast<uintptr_t>(pixels) & 15) || (roi_stride & 15)) return false;
    int T, K;
    return com_shape(P, T, K);
}

cudaError_t launch_com(const TrackParams &P, const uint8_t *pixels, int64_t roi_stride, const LocalizationJob *jobs,
                       int count, LocalizationResult *results, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    int T, K;
    if (!com_shape(P, T, K)) return cudaErrorInvalidValue;
    int stages = 0, stride = 0;
    const int64_t roi_bytes = (int64_t)P.width * P.height * bytes_per_pixel(P.pdt);
    int groups = 0, wg = 1;
    if (com_warp_plan(roi_bytes, groups, wg, stride)) {
        ComWarpKernel f = P.pdt == 0 ? com_warp_kernel<0> : (P.pdt == 1 ? com_warp_kernel<1> : com_warp_kernel<2>);
        const int smem = groups * stride, threads = groups * wg * 32;
        const int ctas = com_stream_ctas(reinterpret_cast<ComStreamKernel>(f), threads, smem);
        if (ctas > 0) {
            const int need = (count + groups - 1) / groups;
            f<<<need < ctas ? need : ctas, threads, smem, stream>>>(P, pixels, roi_stride, jobs, count, results, stride,
                                                                   wg);
            return cudaGetLastError();
        }
    }
    if (com_stream_plan(roi_bytes, stages, stride)) {
        ComStreamKernel f = P.pdt == 0 ? com_stream_at<0, 1>(K)
                                       : (P.pdt == 1 ? com_stream_at<1, 1>(K) : com_stream_at<2, 1>(K));
        const int smem = stages * stride;
        const int ctas = f ? com_stream_ctas(f, T, smem) : 0;
        if (ctas > 0) {
            f<<<count < ctas ? count : ctas, T, smem, stream>>>(P, pixels, roi_stride, jobs, count, results, stages,
                                                               stride);
            return cudaGetLastError();
        }
    }
    ComKernel f = P.pdt == 0 ? com_kernel_at<0, 1>(K) : (P.pdt == 1 ? com_kernel_at<1, 1>(K) : com_kernel_at<2, 1>(K));
    if (!f) return cudaErrorInvalidValue;
    f<<<count, T, 0, stream>>>(P, pixels, roi_stride, jobs, count, results);
    return cudaGetLastError();
}

}  // namespace qtrk
