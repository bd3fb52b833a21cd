// Streaming centre-of-mass kernel for LT_OnlyCOM (sm_100a).
//
// CPUTracker::ComputeMeanAndCOM (cputrack/cpu_tracker.cpp:681-729) needs two passes over a ROI:
// mean and standard deviation first, then the background-corrected moments
//   v' = max(0, |v - mean| - bgcorrection * stdev),  COM = (sum x v', sum y v') / sum v'.
// The fused localization kernel stages every ROI as a float tile in shared memory because QI and
// the radial profile sample it many times; a COM-only localization reads each pixel twice, so
// here the ROI is held in registers instead: one CTA per ROI, every thread loads its share of
// 16-byte chunks (8 u16, 16 u8 or 4 f32 pixels) with streaming loads, all of them issued before
// the first is used, converts them to float once, and both passes run on the registers. The sums
// meet across the CTA in FP64 (warp shuffles, then one value per warp in shared memory), as the
// reference accumulates in FP64; per-thread partial sums are FP32 over at most 64 pixels (exact
// for the mean of u8/u16 data, ~1e-7 relative for the moments).
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

// Pass 2 of ComputeMeanAndCOM on this thread's chunks (see the chunk moments above): returns the
// FP32 partial sums of v', x v' and y v'. kThr: a background threshold is set (v' = max(0, |v -
// mean| - thr)); without one v' = |v - mean| exactly.
template <int PDT, int K, bool kThr>
__device__ __forceinline__ float3 com_moments(const float (&v)[K][ChunkPixels<PDT>::n], ChunkWalk w, int t, int T,
                                              int nchunks, int W, float mean, float thr)
{
    constexpr int ppc = ChunkPixels<PDT>::n;
    const float fW = (float)W;
    float q0 = 0.0f, qx = 0.0f, qy = 0.0f;
#pragma unroll
    for (int k = 0; k < K; k++) {
        const int c = t + k * T;
        if (c < nchunks) {
            float a[ppc];
            float S = 0.0f, Sj = 0.0f;
#pragma unroll
            for (int j = 0; j < ppc; j++) {
                a[j] = kThr ? fmaxf(0.0f, fabsf(v[k][j] - mean) - thr) : fabsf(v[k][j] - mean);
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
        w.fx += w.fdx;
        w.fy += w.fdy;
        if (w.fx >= fW) {
            w.fx -= fW;
            w.fy += 1.0f;
        }
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
// device and shared-memory size); 0 when the query fails.
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
    int per_sm = 0, sms = 0;
    if (cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess ||
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
