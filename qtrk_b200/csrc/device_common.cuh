// Device building blocks of the localization kernels (sm_100a).
//
// Each function restates one step of the reference CPU tracker for one ROI held in
// shared memory by one CTA; the reference file:line each follows is given beside it.
// Thread mappings are chosen for the GPU (one (quadrant, radius) bin per thread or
// per aligned lane group, warp-shuffle reductions, one warp for the QI FFTs); the
// discrete decisions (int truncation, the bilinear "outside" rule, sample-count
// thresholds, the argmax window of the quadratic fit) are those of the reference.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "track_params.h"

namespace qtrk {

// -------------------------------------------------------------------------------------
// small helpers
// -------------------------------------------------------------------------------------
__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ int ilog2_pow2(int v) { return 31 - __clz(v); }

__device__ __forceinline__ unsigned bitrev(unsigned v, int bits) { return __brev(v) >> (32 - bits); }

// Sum N doubles over the whole CTA; every thread receives the totals.
// red: shared scratch of at least N * (blockDim.x / 32) doubles (256 doubles cover N <= 32
// at 256 threads).
template <int N>
__device__ __forceinline__ void block_sum(double (&v)[N], double *red)
{
#pragma unroll
    for (int k = 0; k < N; k++)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < N; k++) red[k * nw + warp] = v[k];
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; k++) {
        double s = 0;
        for (int w = 0; w < nw; w++) s += red[k * nw + w];
        v[k] = s;
    }
}

// Thread groups that process one ROI: the whole CTA, or one warp (small-ROI kernels).
struct BlockGroup {
    double *red;  // >= N*32 doubles of shared scratch for sum<N>
    __device__ __forceinline__ int rank() const { return threadIdx.x; }
    __device__ __forceinline__ int size() const { return blockDim.x; }
    __device__ __forceinline__ void sync() const { __syncthreads(); }
    template <int N>
    __device__ __forceinline__ void sum(double (&v)[N]) const { block_sum<N>(v, red); }
};

struct WarpGroup {
    __device__ __forceinline__ int rank() const { return threadIdx.x & 31; }
    __device__ __forceinline__ int size() const { return 32; }
    __device__ __forceinline__ void sync() const { __syncwarp(); }
    template <int N>
    __device__ __forceinline__ void sum(double (&v)[N]) const
    {
#pragma unroll
        for (int k = 0; k < N; k++)
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    }
};

// Interpolate, utils.h:40-58: rx = (int)x (C truncation); the sample is outside when rx < 0,
// ry < 0, rx+1 >= w or ry+1 >= h. Returns false when outside. Row y of the tile starts at
// img + y * ts (ts >= w: the tile's row pitch in floats).
// Without float->int conversions: truncation keeps a sample inside exactly when -1 < x < w-1,
// and for those x, (int)x == floor(max(x, 0)), which a round-toward-zero add of 2^23 puts in
// the low mantissa bits. The fraction x - rx is formed from the same exact float as the
// reference's x - (float)rx, so the interpolated value is unchanged.
__device__ __forceinline__ bool bilinear(const float *img, int w, int h, int ts, float x, float y, float &v)
{
    if (!(x > -1.0f && x < (float)(w - 1) && y > -1.0f && y < (float)(h - 1))) return false;
    const float kMagic = 8388608.0f;  // 2^23
    const float tx = __fadd_rz(fmaxf(x, 0.0f), kMagic), ty = __fadd_rz(fmaxf(y, 0.0f), kMagic);
    const int rx = __float_as_int(tx) - 0x4B000000, ry = __float_as_int(ty) - 0x4B000000;
    const float *p = img + ry * ts + rx;
    const float v00 = p[0], v10 = p[1], v01 = p[ts], v11 = p[ts + 1];
    const float fx = x - (tx - kMagic), fy = y - (ty - kMagic);
    const float v0 = v00 + (v10 - v00) * fx;
    const float v1 = v01 + (v11 - v01) * fx;
    v = v0 + (v1 - v0) * fy;
    return true;
}

// bilinear() for a sample known to lie strictly inside (0 < x < w-1, 0 < y < h-1): the same
// arithmetic without the range test. Callers prove the range for a whole bin at once.
__device__ __forceinline__ float bilinear_inside(const float *img, int ts, float x, float y)
{
    const float kMagic = 8388608.0f;
    const float tx = __fadd_rz(x, kMagic), ty = __fadd_rz(y, kMagic);
    const float *p = img + ((__float_as_int(ty) - 0x4B000000) * ts + (__float_as_int(tx) - 0x4B000000));
    const float v00 = p[0], v10 = p[1], v01 = p[ts], v11 = p[ts + 1];
    const float fx = x - (tx - kMagic), fy = y - (ty - kMagic);
    const float v0 = v00 + (v10 - v00) * fx;
    const float v1 = v01 + (v11 - v01) * fx;
    return v0 + (v1 - v0) * fy;
}

// Two bilinear samples at once with the packed FP32x2 operations of sm_100 (each component
// rounds as the scalar operation does): cells at p and q, fractions fx = (fx_p, fx_q) and
// fy = (fy_p, fy_q). Same arithmetic as lerp_cell, one instruction per pair of samples; the
// differences v10 - v00 are fma(v00, -1, v10), exact before their one rounding.
__device__ __forceinline__ float2 lerp_cell2(const float *p, const float *q, int ts, float2 fx, float2 fy)
{
    const float2 m1 = make_float2(-1.0f, -1.0f);
    const float2 v00 = make_float2(p[0], q[0]), v10 = make_float2(p[1], q[1]);
    const float2 v01 = make_float2(p[ts], q[ts]), v11 = make_float2(p[ts + 1], q[ts + 1]);
    const float2 v0 = __ffma2_rn(__ffma2_rn(v00, m1, v10), fx, v00);
    const float2 v1 = __ffma2_rn(__ffma2_rn(v01, m1, v11), fx, v01);
    return __ffma2_rn(__ffma2_rn(v0, m1, v1), fy, v0);
}

// bilinear_inside for two samples at (X.x, Y.x) and (X.y, Y.y) with packed FP32x2 arithmetic
// (each component rounded as bilinear_inside rounds it).
__device__ __forceinline__ float2 bilinear_inside2(const float *img, int ts, float2 X, float2 Y)
{
    const float2 K = make_float2(8388608.0f, 8388608.0f), nK = make_float2(-8388608.0f, -8388608.0f);
    const float2 m1 = make_float2(-1.0f, -1.0f);
    const float2 TX = __fadd2_rz(X, K), TY = __fadd2_rz(Y, K);
    const float2 FX = __ffma2_rn(__fadd2_rn(TX, nK), m1, X), FY = __ffma2_rn(__fadd2_rn(TY, nK), m1, Y);
    const float *p = img + ((__float_as_int(TY.x) - 0x4B000000) * ts + (__float_as_int(TX.x) - 0x4B000000));
    const float *q = img + ((__float_as_int(TY.y) - 0x4B000000) * ts + (__float_as_int(TX.y) - 0x4B000000));
    return lerp_cell2(p, q, ts, FX, FY);
}

// True when every point cx + a*r, cy + b*r with |a|, |b| <= 1 (any sample of a circle of radius
// r around (cx, cy)) lies strictly inside (0, w-1) x (0, h-1), rounding of the sample
// coordinates included (margin 1e-3 px, far above one ulp of the coordinates).
__device__ __forceinline__ bool circle_inside(float cx, float cy, float r, int w, int h)
{
    const float m = 1e-3f;
    return cx - r > m && cy - r > m && cx + r < (float)(w - 1) - m && cy + r < (float)(h - 1) - m;
}

// CPUTracker::CheckBoundaries, cpu_tracker.cpp:182-188
__device__ __forceinline__ bool check_boundaries(float cx, float cy, float radius, int w, int h)
{
    return cx + radius >= w || cx - radius < 0 || cy + radius >= h || cy - radius < 0;
}

// LsqSqQuadFit + ComputeMaxInterp<T,7>::Compute (LsqQuadraticFit.h:8-176) in FP64, with the eight
// weighted sums formed by lanes 0..6 of one warp (all 32 lanes call; every lane returns the result).
// `at(i)` returns element i of the length-`len` array; iMax is the first index of the maximum;
// the weights are indexed from 0 even when the window is clipped at the array start, as in the
// reference. maxPos = iMax - b/(2a) with a = A/d, b = B/d, so the
// determinant d cancels and one division remains; |a| < 1e-9 is tested as |A| < 1e-9 |d|.
template <typename Get>
__device__ inline double max_interp7_warp(Get at, int len, int iMax, const float (&wts)[7])
{
    const int lane = threadIdx.x & 31;
    const int startPos = max(iMax - 3, 0);
    const int endPos = min(iMax + 4, len);
    const int np = endPos - startPos;
    if (np < 3) return (double)iMax;
    double t[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (lane < np) {
        const double x = (double)(startPos + lane - iMax), y = (double)at(startPos + lane), wt = (double)wts[lane];
        const double sq = x * x;
        t[0] = x * wt;        // Sx
        t[1] = y * wt;        // Sy
        t[2] = sq * wt;       // Sx2
        t[3] = sq * x * wt;   // Sx3
        t[4] = sq * sq * wt;  // Sx4
        t[5] = x * y * wt;    // Sxy
        t[6] = sq * y * wt;   // Sx2y
        t[7] = wt;            // Sw
    }
#pragma unroll
    for (int k = 0; k < 8; k++)
#pragma unroll
        for (int o = 4; o > 0; o >>= 1) t[k] += __shfl_xor_sync(0xffffffffu, t[k], o);
#pragma unroll
    for (int k = 0; k < 8; k++) t[k] = __shfl_sync(0xffffffffu, t[k], 0);
    const double Sx = t[0], Sy = t[1], Sx2 = t[2], Sx3 = t[3], Sx4 = t[4], Sxy = t[5], Sx2y = t[6], Sw = t[7];
    const double d = Sx4 * (Sx2 * Sw - Sx * Sx) - Sx3 * (Sx3 * Sw - Sx * Sx2) + Sx2 * (Sx3 * Sx - Sx2 * Sx2);
    const double A = Sx2y * (Sx2 * Sw - Sx * Sx) - Sxy * (Sx3 * Sw - Sx * Sx2) + Sy * (Sx3 * Sx - Sx2 * Sx2);
    const double B = Sx4 * (Sxy * Sw - Sy * Sx) - Sx3 * (Sx2y * Sw - Sy * Sx2) + Sx2 * (Sx2y * Sx - Sxy * Sx2);
    if (fabs(A) < 1e-9 * fabs(d)) return (double)iMax;
    return (double)iMax - B / (2 * A);
}

// The same fit for the common case, a window iMax-3 .. iMax+3 inside the array with weights
// symmetric about its centre (the reference's QIWeights and ZLUTWeights). Then S_x = S_x3 = 0
// and the cofactor expansion of LsqSqQuadFit::Coeff::abc reduces to
//   maxPos = iMax - (p0 / (2 Sx2)) N / D,  N = sum w x y,  D = sum w (x^2 Sw - Sx2) y,
//   p0 = Sx4 Sw - Sx2^2,  S_x^k = sum w x^k,  Sw = sum w,
// and a = D / p0 (the |a| < 1e-9 test). Both stencils sum to zero, so y is taken relative to
// y[iMax]: the two 7-term sums run in FP32 on small differences, which keeps the offset to ~1e-7
// of itself, with no FP64 and no cross-lane traffic. Clipped windows take max_interp7_warp.
// All 32 lanes of a warp call (with the same arguments); every lane returns the result.
template <typename Get>
__device__ __forceinline__ float max_interp7_sym(Get at, int len, int iMax, const float (&wts)[7])
{
    if (iMax < 3 || iMax + 4 > len) return (float)max_interp7_warp(at, len, iMax, wts);
    float Sw = 0.0f, Sx2 = 0.0f, Sx4 = 0.0f;
#pragma unroll
    for (int i = 0; i < 7; i++) {
        const float x2 = (float)((i - 3) * (i - 3)), w = wts[i];
        Sw += w;
        Sx2 += w * x2;
        Sx4 += w * x2 * x2;
    }
    const auto yc = at(iMax);
    float N = 0.0f, D = 0.0f;
#pragma unroll
    for (int i = 0; i < 7; i++) {
        if (i == 3) continue;  // y - y[iMax] = 0
        const float x = (float)(i - 3), w = wts[i];
        const float d = (float)(at(iMax - 3 + i) - yc);
        N += w * x * d;
        D += w * (x * x * Sw - Sx2) * d;
    }
    const float p0 = Sx4 * Sw - Sx2 * Sx2;
    if (fabsf(D) < 1e-9f * p0) return (float)iMax;
    return (float)iMax - (p0 / (2.0f * Sx2)) * (N / D);
}

// First index of the maximum of at(0..len), reduced over one warp (all 32 lanes call).
// Matches the strict ">" scan of LsqQuadraticFit.h:140-147 (NaN values never win).
template <typename Get>
__device__ __forceinline__ int warp_argmax(Get at, int len)
{
    using T = decltype(at(0));
    const int lane = threadIdx.x & 31;
    T best = 0;
    int bi = -1;
    for (int i = lane; i < len; i += 32) {
        const T v = at(i);
        if (v == v && (bi < 0 || v > best)) {
            best = v;
            bi = i;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const T ov = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (oi >= 0 && (bi < 0 || ov > best || (ov == best && oi < bi))) {
            best = ov;
            bi = oi;
        }
    }
    return bi < 0 ? 0 : bi;
}

// -------------------------------------------------------------------------------------
// ROI load: u8/u16/f32 -> f32 tile in shared memory, with the clear-first-four-pixels
// option (QueuedCPUTracker.cpp:280-282) and the per-bead offset/gain step
// (cpu_tracker.cpp:98-112) fused into the same pass.
// -------------------------------------------------------------------------------------
// Exact conversion of an unsigned integer below 2^23 to float without the conversion pipe:
// placing it in the mantissa of 2^23 and subtracting 2^23.
__device__ __forceinline__ float u_to_float(uint32_t u) { return __uint_as_float(0x4B000000u | u) - 8388608.0f; }

__device__ __forceinline__ float finish_pixel(float v, int i, const TrackParams &P, const float *off,
                                              const float *gain)
{
    if ((P.mode & kLT_ClearFirstFourPixels) && i < 4) v = 0.0f;
    if (off && !gain) v = v + off[i] * P.offset_factor;
    if (gain && !off) v = v * gain[i] * P.gain_factor;
    if (gain && off) v = (v + off[i] * P.offset_factor) * gain[i] * P.gain_factor;
    return v;
}

// Returns this thread's FP32 partial sums of v and v^2 over the pixels it converted (the first pass
// of CPUTracker::ComputeMeanAndCOM, cpu_tracker.cpp:687-693, so that com_from_sums need not read
// the tile again for them; callers that do not use them pay nothing once the call is inlined).
template <class G>
__device__ inline float2 load_roi(const G &g, float *img, const uint8_t *src, int pitch, const TrackParams &P, int bead)
{
    const int W = P.width, H = P.height, n = W * H;
    const int bpp = P.pdt == 0 ? 1 : (P.pdt == 1 ? 2 : 4);
    const float *off = nullptr, *gain = nullptr;
    if (bead >= 0 && bead < P.calib_count) {
        if (P.calib_offset) off = P.calib_offset + (size_t)bead * n;
        if (P.calib_gain) gain = P.calib_gain + (size_t)bead * n;
    }
    const bool contiguous = pitch == W * bpp && ((reinterpret_cast<uintptr_t>(src) & 15) == 0) &&
                            ((n * bpp) & 15) == 0 && ((reinterpret_cast<uintptr_t>(img) & 15) == 0);
    float s = 0.0f, s2 = 0.0f;
    if (contiguous) {
        // Rows are back to back: the ROI is a run of n/4 chunks of four pixels (4, 8 or 16 input
        // bytes), and chunk c becomes the float4 at img + 4c, so a warp's stores fill 512
        // contiguous bytes of shared memory without bank conflicts. Each thread issues
        // kBatch streaming loads (8-16 registers' worth) before converting any of them, so the
        // HBM latency is paid about once per batch rather than once per load.
        const int nc = n >> 2;
        const bool plain = !off && !gain && !(P.mode & kLT_ClearFirstFourPixels);
        float4 *dst = reinterpret_cast<float4 *>(img);
        auto finish4 = [&](float4 f, int c) {
            if (!plain) {
                f.x = finish_pixel(f.x, 4 * c, P, off, gain);
                f.y = finish_pixel(f.y, 4 * c + 1, P, off, gain);
                f.z = finish_pixel(f.z, 4 * c + 2, P, off, gain);
                f.w = finish_pixel(f.w, 4 * c + 3, P, off, gain);
            }
            s += f.x;
            s2 = fmaf(f.x, f.x, s2);
            s += f.y;
            s2 = fmaf(f.y, f.y, s2);
            s += f.z;
            s2 = fmaf(f.z, f.z, s2);
            s += f.w;
            s2 = fmaf(f.w, f.w, s2);
            dst[c] = f;
        };
        if (P.pdt == 0) {
            constexpr int kBatch = 8;
            const uint32_t *s1 = reinterpret_cast<const uint32_t *>(src);
            for (int c0 = g.rank(); c0 < nc; c0 += kBatch * g.size()) {
                uint32_t q[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; k++) {
                    const int c = c0 + k * g.size();
                    if (c < nc) q[k] = __ldcs(s1 + c);
                }
#pragma unroll
                for (int k = 0; k < kBatch; k++) {
                    const int c = c0 + k * g.size();
                    if (c >= nc) break;
                    finish4(make_float4(u_to_float(q[k] & 0xffu), u_to_float((q[k] >> 8) & 0xffu),
                                        u_to_float((q[k] >> 16) & 0xffu), u_to_float(q[k] >> 24)),
                            c);
                }
            }
        } else if (P.pdt == 1) {
            constexpr int kBatch = 8;
            const uint2 *s2 = reinterpret_cast<const uint2 *>(src);
            for (int c0 = g.rank(); c0 < nc; c0 += kBatch * g.size()) {
                uint2 q[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; k++) {
                    const int c = c0 + k * g.size();
                    if (c < nc) q[k] = __ldcs(s2 + c);
                }
#pragma unroll
                for (int k = 0; k < kBatch; k++) {
                    const int c = c0 + k * g.size();
                    if (c >= nc) break;
                    finish4(make_float4(u_to_float(q[k].x & 0xffffu), u_to_float(q[k].x >> 16),
                                        u_to_float(q[k].y & 0xffffu), u_to_float(q[k].y >> 16)),
                            c);
                }
            }
        } else {
            constexpr int kBatch = 4;
            const float4 *s4 = reinterpret_cast<const float4 *>(src);
            for (int c0 = g.rank(); c0 < nc; c0 += kBatch * g.size()) {
                float4 q[kBatch];
#pragma unroll
                for (int k = 0; k < kBatch; k++) {
                    const int c = c0 + k * g.size();
                    if (c < nc) q[k] = __ldcs(s4 + c);
                }
#pragma unroll
                for (int k = 0; k < kBatch; k++) {
                    const int c = c0 + k * g.size();
                    if (c >= nc) break;
                    finish4(q[k], c);
                }
            }
        }
    } else {
        // Rows at a pitch (a ROI inside a frame): warps over rows, lanes along a row, so loads
        // are coalesced along the row and the stores are conflict-free.
        // With whole 4-pixel chunks the partial sums are then taken from the tile in the chunk
        // order of the contiguous loads, so that a ROI gives bit-identical results whichever way
        // it arrived (FP32 partial sums depend on which pixels each thread adds).
        const bool chunked = !(n & 3) && !(reinterpret_cast<uintptr_t>(img) & 15);
        const int lane = g.rank() & 31, wg = g.rank() >> 5, nwg = g.size() >> 5;
        for (int y = wg; y < H; y += nwg) {
            const uint8_t *row = src + (size_t)y * pitch;
#pragma unroll 4
            for (int x = lane; x < W; x += 32) {
                float v;
                if (P.pdt == 0)
                    v = u_to_float(row[x]);
                else if (P.pdt == 1)
                    v = u_to_float(reinterpret_cast<const uint16_t *>(row)[x]);
                else
                    v = reinterpret_cast<const float *>(row)[x];
                const int i = y * W + x;
                v = finish_pixel(v, i, P, off, gain);
                if (!chunked) {
                    s += v;
                    s2 = fmaf(v, v, s2);
                }
                img[i] = v;
            }
        }
        if (chunked) {
            g.sync();
            const float4 *img4 = reinterpret_cast<const float4 *>(img);
            for (int c = g.rank(); c < (n >> 2); c += g.size()) {
                const float4 f = img4[c];
                s += f.x;
                s2 = fmaf(f.x, f.x, s2);
                s += f.y;
                s2 = fmaf(f.y, f.y, s2);
                s += f.z;
                s2 = fmaf(f.z, f.z, s2);
                s += f.w;
                s2 = fmaf(f.w, f.w, s2);
            }
        }
    }
    g.sync();
    return make_float2(s, s2);
}

// load_roi for a ROI whose raw bytes (n = W*H pixels, u8/u16/f32, rows back to back) were brought
// into shared memory by a bulk copy to img + (4 - bpp) n bytes, the end of the float tile. The
// conversion runs in place in batches of kBatch chunks of four pixels per thread: a batch's raw
// chunks are read into registers, a barrier passes, and the batch's float chunks are written.
// Float chunk c (bytes 16c .. 16c+15) overlaps only raw chunks with index <= c, which the batch or
// an earlier one has already read, so a batch never overwrites raw bytes a later batch needs. The
// per-pixel steps and the returned partial sums are load_roi's. Requires n a multiple of 4. All
// threads call; the tile is complete at return.
template <class G>
__device__ inline float2 convert_staged(const G &g, float *img, const TrackParams &P, int bead)
{
    const int W = P.width, H = P.height, n = W * H, nc = n >> 2;
    const int bpp = P.pdt == 0 ? 1 : (P.pdt == 1 ? 2 : 4);
    const uint8_t *raw = reinterpret_cast<const uint8_t *>(img) + (size_t)(4 - bpp) * n;
    const float *off = nullptr, *gain = nullptr;
    if (bead >= 0 && bead < P.calib_count) {
        if (P.calib_offset) off = P.calib_offset + (size_t)bead * n;
        if (P.calib_gain) gain = P.calib_gain + (size_t)bead * n;
    }
    const bool plain = !off && !gain && !(P.mode & kLT_ClearFirstFourPixels);
    float4 *dst = reinterpret_cast<float4 *>(img);
    float s = 0.0f, s2 = 0.0f;
    constexpr int kBatch = 8;
    // every thread runs the same number of batches (the loop holds a barrier)
    for (int b0 = 0; b0 < nc; b0 += kBatch * g.size()) {
        const int c0 = b0 + g.rank();
        uint4 q[kBatch];
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
            const int c = c0 + k * g.size();
            if (c < nc) {
                if (P.pdt == 0) {
                    q[k].x = reinterpret_cast<const uint32_t *>(raw)[c];
                } else if (P.pdt == 1) {
                    const uint2 v = reinterpret_cast<const uint2 *>(raw)[c];
                    q[k].x = v.x;
                    q[k].y = v.y;
                } else {
                    q[k] = reinterpret_cast<const uint4 *>(raw)[c];
                }
            }
        }
        g.sync();
#pragma unroll
        for (int k = 0; k < kBatch; k++) {
            const int c = c0 + k * g.size();
            if (c >= nc) continue;
            float4 f;
            if (P.pdt == 0)
                f = make_float4(u_to_float(q[k].x & 0xffu), u_to_float((q[k].x >> 8) & 0xffu),
                                u_to_float((q[k].x >> 16) & 0xffu), u_to_float(q[k].x >> 24));
            else if (P.pdt == 1)
                f = make_float4(u_to_float(q[k].x & 0xffffu), u_to_float(q[k].x >> 16), u_to_float(q[k].y & 0xffffu),
                                u_to_float(q[k].y >> 16));
            else
                f = make_float4(__uint_as_float(q[k].x), __uint_as_float(q[k].y), __uint_as_float(q[k].z),
                                __uint_as_float(q[k].w));
            if (!plain) {
                f.x = finish_pixel(f.x, 4 * c, P, off, gain);
                f.y = finish_pixel(f.y, 4 * c + 1, P, off, gain);
                f.z = finish_pixel(f.z, 4 * c + 2, P, off, gain);
                f.w = finish_pixel(f.w, 4 * c + 3, P, off, gain);
            }
            s += f.x;
            s2 = fmaf(f.x, f.x, s2);
            s += f.y;
            s2 = fmaf(f.y, f.y, s2);
            s += f.z;
            s2 = fmaf(f.z, f.z, s2);
            s += f.w;
            s2 = fmaf(f.w, f.w, s2);
            dst[c] = f;
        }
    }
    g.sync();
    return make_float2(s, s2);
}

// -------------------------------------------------------------------------------------
// CPUTracker::ComputeMeanAndCOM, cpu_tracker.cpp:681-729 (FP64 accumulation as in the
// reference; mean and stdev rounded to float where the reference stores floats).
// -------------------------------------------------------------------------------------
struct ComResult {
    float x, y, mean, stdev;
};

// From this thread's partial sums of v and v^2 (first pass, part) and the tile: the FP64 sums
// across the group, mean and stdev as the reference rounds them, then the background-corrected
// moments. Each thread walks a fixed set of pixels with its column/row as float counters, keeps
// FP32 partial sums over its few dozen pixels, and the partials are added in FP64 across the
// group (the reference accumulates the whole image in FP64; the partial sums keep its result
// to ~1e-7 relative, far inside the 1e-4 px COM tolerance; for integer pixels the first pass's
// partial sums, and so the mean, are exact).
template <class G>
__device__ ComResult com_from_sums(const G &g, const float *img, int W, int H, float2 part, float bgcorr)
{
    const int n = W * H, stride = g.size();
    const int dx = stride % W, dy = stride / W;
    double s[2] = {part.x, part.y};
    g.sum(s);
    const float invN = 1.0f / (float)n;
    ComResult r;
    r.mean = (float)(s[0] * (double)invN);
    r.stdev = sqrtf((float)(s[1] * (double)invN - (double)(r.mean * r.mean)));
    const float thr = bgcorr * r.stdev;
    float q0 = 0.0f, qx = 0.0f, qy = 0.0f;
    if (!(W & 3) && !(reinterpret_cast<uintptr_t>(img) & 15)) {
        // rows are whole float4 chunks: chunk c holds pixels 4c .. 4c+3 of one row, at column fx
        // and row fy; per chunk S = sum v', Sj = sum j v', so sum x v' = fx S + Sj
        const int nc = n >> 2, cstride = stride * 4;
        const float fW = (float)W, fdx = (float)(cstride % W), fdy = (float)(cstride / W);
        float fx = (float)((4 * g.rank()) % W), fy = (float)((4 * g.rank()) / W);
        const float4 *img4 = reinterpret_cast<const float4 *>(img);
        for (int c = g.rank(); c < nc; c += stride) {
            const float4 q = img4[c];
            float a0, a1, a2, a3;
            if (thr == 0.0f) {  // max(0, |d| - 0) is |d|
                a0 = fabsf(q.x - r.mean);
                a1 = fabsf(q.y - r.mean);
                a2 = fabsf(q.z - r.mean);
                a3 = fabsf(q.w - r.mean);
            } else {
                a0 = fmaxf(0.0f, fabsf(q.x - r.mean) - thr);
                a1 = fmaxf(0.0f, fabsf(q.y - r.mean) - thr);
                a2 = fmaxf(0.0f, fabsf(q.z - r.mean) - thr);
                a3 = fmaxf(0.0f, fabsf(q.w - r.mean) - thr);
            }
            const float S = (a0 + a1) + (a2 + a3);
            const float Sj = fmaf(3.0f, a3, fmaf(2.0f, a2, a1));
            q0 += S;
            qx += fmaf(fx, S, Sj);
            qy = fmaf(fy, S, qy);
            fx += fdx;
            fy += fdy;
            if (fx >= fW) {
                fx -= fW;
                fy += 1.0f;
            }
        }
    } else {
        int x = g.rank() % W, y = g.rank() / W;
        float fx = (float)x, fy = (float)y;
        for (int i = g.rank(); i < n; i += stride) {
            const float v = fmaxf(0.0f, fabsf(img[i] - r.mean) - thr);
            q0 += v;
            qx += fx * v;
            qy += fy * v;
            x += dx;
            fx += (float)dx;
            fy += (float)dy;
            if (x >= W) {
                x -= W;
                fx -= (float)W;
                fy += 1.0f;
            }
        }
    }
    double m[3] = {q0, qx, qy};
    g.sum(m);
    r.x = (float)(m[1] / m[0]);
    r.y = (float)(m[2] / m[0]);
    return r;
}

template <class G>
__device__ ComResult compute_com(const G &g, const float *img, int W, int H, float bgcorr)
{
    float p0 = 0.0f, p1 = 0.0f;
    for (int i = g.rank(); i < W * H; i += g.size()) {
        const float v = img[i];
        p0 += v;
        p1 += v * v;
    }
    return com_from_sums(g, img, W, H, make_float2(p0, p1), bgcorr);
}

// Bilinear value at a sample whose truncated corner (ix, row) and fractions are known: row points
// at the tile row of the upper corner pixels. Arithmetic of bilinear_inside.
__device__ __forceinline__ float lerp_cell(const float *row, int ts, int ix, float fx, float fy)
{
    const float *p = row + ix;
    const float v00 = p[0], v10 = p[1], v01 = p[ts], v11 = p[ts + 1];
    const float v0 = v00 + (v10 - v00) * fx;
    const float v1 = v01 + (v11 - v01) * fx;
    return v0 + (v1 - v0) * fy;
}

// CPUTracker::ComputeQuadrantProfile (cpu_tracker.cpp:631-677) for all four quadrants at once,
// written as the FFT input of the QI autoconvolution. The four quadrants sample the same
// table direction d at radius r with mirrored signs (x = cx +- d.x r, y = cy +- d.y r), so one
// thread takes one radius and a strided subset of the directions and produces all four samples
// of each: the products d.x r, d.y r, the truncations and fractions of the two x and two y
// coordinates are shared by four samples. Coordinates are formed as the reference forms them
// (d.x r rounded, then added to the centre). The table holds each direction as (d.x, d.x, d.y, d.y)
// so that on the fast path x = (cx, cx) + (d.x, d.x) * (r, -r) gives (x+, x-) in one packed
// multiply and one packed add; the diagonal quadrants q0 (+, +) and q2 (-, -) then share
// fractions (fx+, fx-), (fy+, fy-) and are sampled as one pair, q3 (+, -) and q1 (-, +) as another. Layout: S = blockDim/nr direction subsets
// (directions sub, sub + S, ...); a warp holds R = 32/A radii x A = min(S, 4) adjacent subsets,
// so its gathers fall into a small patch. Per quadrant and radius the bin value
// is the mean of the in-bounds samples (the image mean when fewer than 4), times the radial
// weight; the subsets' partial sums meet through warp shuffles (and `part`, 2 KB of shared
// memory, when S > A). The thread of subset 0 writes the X and Y concatenations
// (cpu_tracker.cpp:327-343; X = [(q1+q2) reversed | q0+q3], Y = [(q2+q3) reversed | q0+q1]) as
// one complex value z = X + iY per position, in bit-reversed order (log2L = log2(2 nr)) or in
// natural order when log2L < 0. All threads call; a barrier must follow before A is read.
__device__ __forceinline__ void qi_profiles_sym(const float *img, int W, int H, int ts, float cx, float cy, float mean, int nr,
                                       int nang, float inv_nang, int stride, float minr, float rstep,
                                       const float4 *dirs, const float *rweights, float4 *part, float2 *A, int log2L)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    // nr and blockDim are powers of two (QTrkComputedConfig::Update rounds qi_radialsteps,
    // QueuedTracker.cpp:20), so the layout is all shifts: S = 2^lS subsets, Aw = 2^lA of them per
    // warp, R = 2^lR radii per warp, nwr = 2^lw warps along the radius, nsb subset blocks
    const int lnr = ilog2_pow2(nr), lbd = ilog2_pow2(blockDim.x);
    const int lS = lnr >= lbd ? 0 : lbd - lnr, lA = lS < 2 ? lS : 2, lR = 5 - lA;
    const int lw = lnr >= lR ? lnr - lR : 0;
    const int S = 1 << lS, Aw = 1 << lA, nwr = 1 << lw, nsb = 1 << (lS - lA);
    const float kMagic = 8388608.0f;
    for (int wi = warp; wi < nwr * nsb; wi += nw) {
        const int rb = wi & (nwr - 1), sb = wi >> lw;
        const int i = (rb << lR) + (lane >> lA), sub = (sb << lA) + (lane & (Aw - 1));
        float sm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        int cnt[4] = {0, 0, 0, 0};
        const float r = __fadd_rn(minr, __fmul_rn(rstep, (float)i));
        // One path per warp: when any lane's circle may leave the image, the whole warp takes the
        // checked body (a warp running both bodies one after the other would hold up the CTA's
        // other warps at the next barrier).
        const bool fast = __all_sync(0xffffffffu, i >= nr || circle_inside(cx, cy, fabsf(r), W, H));
        if (i < nr) {
            if (fast) {
                const float2 rr = make_float2(r, -r), cxx = make_float2(cx, cx), cyy = make_float2(cy, cy);
                const float2 K = make_float2(kMagic, kMagic), nK = make_float2(-kMagic, -kMagic);
                const float2 m1 = make_float2(-1.0f, -1.0f);
                float2 s02 = make_float2(0.0f, 0.0f), s31 = make_float2(0.0f, 0.0f);
                for (int a = sub; a < nang; a += S) {
                    const float4 d = dirs[stride * a];
                    const float2 X = __fadd2_rn(cxx, __fmul2_rn(make_float2(d.x, d.y), rr));  // (x+, x-)
                    const float2 Y = __fadd2_rn(cyy, __fmul2_rn(make_float2(d.z, d.w), rr));  // (y+, y-)
                    const float2 TX = __fadd2_rz(X, K), TY = __fadd2_rz(Y, K);
                    const float2 FX = __ffma2_rn(__fadd2_rn(TX, nK), m1, X);  // X - trunc(X)
                    const float2 FY = __ffma2_rn(__fadd2_rn(TY, nK), m1, Y);
                    const int ixp = __float_as_int(TX.x) - 0x4B000000, ixm = __float_as_int(TX.y) - 0x4B000000;
                    const float *rowp = img + (__float_as_int(TY.x) - 0x4B000000) * ts;
                    const float *rowm = img + (__float_as_int(TY.y) - 0x4B000000) * ts;
                    s02 = __fadd2_rn(s02, lerp_cell2(rowp + ixp, rowm + ixm, ts, FX, FY));
                    s31 = __fadd2_rn(s31, lerp_cell2(rowm + ixp, rowp + ixm, ts, FX, make_float2(FY.y, FY.x)));
                }
                sm[0] = s02.x;
                sm[1] = s31.y;
                sm[2] = s02.y;
                sm[3] = s31.x;
                const int c = sub < nang ? (nang - sub + S - 1) >> lS : 0;
                cnt[0] = cnt[1] = cnt[2] = cnt[3] = c;
            } else {
                // bilinear()'s rule per coordinate: a sample is inside when -1 < x < W-1 and
                // -1 < y < H-1, and its cell starts at the truncation of max(x, 0)
                const float xhi = (float)(W - 1), yhi = (float)(H - 1);
                for (int a = sub; a < nang; a += S) {
                    const float4 d = dirs[stride * a];
                    const float dx = __fmul_rn(d.x, r), dy = __fmul_rn(d.z, r);
                    const float xp = __fadd_rn(cx, dx), xm = __fadd_rn(cx, -dx);
                    const float yp = __fadd_rn(cy, dy), ym = __fadd_rn(cy, -dy);
                    const bool vxp = xp > -1.0f && xp < xhi, vxm = xm > -1.0f && xm < xhi;
                    const bool vyp = yp > -1.0f && yp < yhi, vym = ym > -1.0f && ym < yhi;
                    const float txp = __fadd_rz(fmaxf(xp, 0.0f), kMagic), txm = __fadd_rz(fmaxf(xm, 0.0f), kMagic);
                    const float typ = __fadd_rz(fmaxf(yp, 0.0f), kMagic), tym = __fadd_rz(fmaxf(ym, 0.0f), kMagic);
                    const float fxp = xp - (txp - kMagic), fxm = xm - (txm - kMagic);
                    const float fyp = yp - (typ - kMagic), fym = ym - (tym - kMagic);
                    const int ixp = __float_as_int(txp) - 0x4B000000, ixm = __float_as_int(txm) - 0x4B000000;
                    const float *rowp = img + (__float_as_int(typ) - 0x4B000000) * ts;
                    const float *rowm = img + (__float_as_int(tym) - 0x4B000000) * ts;
                    if (vxp && vyp) {
                        sm[0] += lerp_cell(rowp, ts, ixp, fxp, fyp);
                        cnt[0]++;
                    }
                    if (vxm && vyp) {
                        sm[1] += lerp_cell(rowp, ts, ixm, fxm, fyp);
                        cnt[1]++;
                    }
                    if (vxm && vym) {
                        sm[2] += lerp_cell(rowm, ts, ixm, fxm, fym);
                        cnt[2]++;
                    }
                    if (vxp && vym) {
                        sm[3] += lerp_cell(rowm, ts, ixp, fxp, fym);
                        cnt[3]++;
                    }
                }
            }
        }
        // subsets of one radius: lanes that differ in their low log2(Aw) bits (on the fast path
        // every count is nang: only the sums travel)
        for (int o = 1; o < Aw; o <<= 1)
#pragma unroll
            for (int q = 0; q < 4; q++) {
                sm[q] += __shfl_xor_sync(0xffffffffu, sm[q], o);
                if (!fast || nsb > 1) cnt[q] += __shfl_xor_sync(0xffffffffu, cnt[q], o);
            }
        if (nsb > 1) {  // subsets spread over warps (nr < blockDim/4): meet in shared memory
            if ((lane & (Aw - 1)) == 0 && i < nr) {
                part[2 * (sb * nr + i)] = make_float4(sm[0], sm[1], sm[2], sm[3]);
                part[2 * (sb * nr + i) + 1] = make_float4(__int_as_float(cnt[0]), __int_as_float(cnt[1]),
                                                          __int_as_float(cnt[2]), __int_as_float(cnt[3]));
            }
            continue;
        }
        float v[4];
        if ((lane & (Aw - 1)) == 0 && i < nr) {
            const float rw = rweights ? rweights[i] : 1.0f;
            if (fast) {  // nang >= 4 in-bounds samples per bin: the mean, as sum * (1 / nang)
#pragma unroll
                for (int k = 0; k < 4; k++) v[k] = rweights ? (sm[k] * inv_nang) * rw : sm[k] * inv_nang;
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    v[k] = cnt[k] >= 4 ? sm[k] / (float)cnt[k] : mean;
                    if (rweights) v[k] *= rw;
                }
            }
        }
        if ((lane & (Aw - 1)) == 0 && i < nr) {
            const int n0 = nr - 1 - i, n1 = nr + i;
            A[log2L >= 0 ? (int)bitrev(n0, log2L) : n0] = make_float2(v[1] + v[2], v[2] + v[3]);
            A[log2L >= 0 ? (int)bitrev(n1, log2L) : n1] = make_float2(v[0] + v[3], v[0] + v[1]);
        }
    }
    if (nsb > 1) {
        __syncthreads();
        for (int i = threadIdx.x; i < nr; i += blockDim.x) {
            float sm[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            int cnt[4] = {0, 0, 0, 0};
            for (int b = 0; b < nsb; b++) {
                const float4 p = part[2 * (b * nr + i)], c = part[2 * (b * nr + i) + 1];
                sm[0] += p.x;
                sm[1] += p.y;
                sm[2] += p.z;
                sm[3] += p.w;
                cnt[0] += __float_as_int(c.x);
                cnt[1] += __float_as_int(c.y);
                cnt[2] += __float_as_int(c.z);
                cnt[3] += __float_as_int(c.w);
            }
            float v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                v[q] = cnt[q] >= 4 ? sm[q] / (float)cnt[q] : mean;
                if (rweights) v[q] *= rweights[i];
            }
            const int n0 = nr - 1 - i, n1 = nr + i;
            A[log2L >= 0 ? (int)bitrev(n0, log2L) : n0] = make_float2(v[1] + v[2], v[2] + v[3]);
            A[log2L >= 0 ? (int)bitrev(n1, log2L) : n1] = make_float2(v[0] + v[3], v[0] + v[1]);
        }
    }
}

// Lanes per radial-profile bin: the largest power of two with nbins*lanes <= threads, at least 4
// (more than one pass over the bins when the CTA is small: with 128 threads and 64 bins, 4 lanes in
// two passes ran 0.993 ms per 10,000 100x100 ROIs against 1.007 ms for 2 lanes in one), at most 32.
__device__ __forceinline__ int lanes_per_bin(int nbins)
{
    int t = blockDim.x / nbins;
    if (t < 4) t = 4;
    if (t > 32) t = 32;
    return 1 << (31 - __clz(t));
}

// Radix-2 decimation-in-time FFT of length L (power of two, input in bit-reversed order),
// executed by one warp over shared memory. tw[k] = e^{-2 pi i k / L}, k < L/2.
// Stage s pairs (i, i + 2^(s-1)) with twiddle tw[(i mod 2^(s-1)) * (L >> s)]. Two consecutive
// stages are done together in registers on groups of four elements, which halves the
// shared-memory round trips and warp barriers without changing any butterfly.
__device__ __forceinline__ float2 fft_tw(const float2 *tw, int k, bool inverse)
{
    float2 w = tw[k];
    if (inverse) w.y = -w.y;
    return w;
}

__device__ inline void warp_fft(float2 *buf, int L, int log2L, const float2 *tw, bool inverse)
{
    const int lane = threadIdx.x & 31;
    int s = 1;
    if (log2L & 1) {  // a single radix-2 stage first (twiddle 1)
        for (int j = lane; j < (L >> 1); j += 32) {
            const float2 a = buf[2 * j], b = buf[2 * j + 1];
            buf[2 * j] = make_float2(a.x + b.x, a.y + b.y);
            buf[2 * j + 1] = make_float2(a.x - b.x, a.y - b.y);
        }
        __syncwarp();
        s = 2;
    }
    for (; s < log2L; s += 2) {
        const int h = 1 << (s - 1);
        for (int j = lane; j < (L >> 2); j += 32) {
            const int pos = j & (h - 1);
            const int i0 = ((j >> (s - 1)) << (s + 1)) + pos;
            float2 a0 = buf[i0], a1 = buf[i0 + h], a2 = buf[i0 + 2 * h], a3 = buf[i0 + 3 * h];
            const float2 w1 = fft_tw(tw, pos * (L >> s), inverse);
            float2 b = cmul(a1, w1);
            a1 = make_float2(a0.x - b.x, a0.y - b.y);
            a0 = make_float2(a0.x + b.x, a0.y + b.y);
            b = cmul(a3, w1);
            a3 = make_float2(a2.x - b.x, a2.y - b.y);
            a2 = make_float2(a2.x + b.x, a2.y + b.y);
            const float2 w2 = fft_tw(tw, pos * (L >> (s + 1)), inverse);
            const float2 w3 = fft_tw(tw, (pos + h) * (L >> (s + 1)), inverse);
            b = cmul(a2, w2);
            buf[i0] = make_float2(a0.x + b.x, a0.y + b.y);
            buf[i0 + 2 * h] = make_float2(a0.x - b.x, a0.y - b.y);
            b = cmul(a3, w3);
            buf[i0 + h] = make_float2(a1.x + b.x, a1.y + b.y);
            buf[i0 + 3 * h] = make_float2(a1.x - b.x, a1.y - b.y);
        }
        __syncwarp();
    }
}

// The unnormalised correlation of each concatenated profile p with its reverse, as
// produced by CPUTracker::QI_ComputeOffset (cpu_tracker.cpp:375-401):
//   out[n] = L * sum_m p[(n+m) mod L] * p[L-1-m].
// Both axes are packed into one complex signal z = px + i py. Because
// FFT(reverse(p))* = e^{-2 pi i k/L} FFT(p) for real p, the product the reference forms
// from two forward FFTs equals e^{-2 pi i k/L} P[k]^2, so one forward and one inverse
// FFT per iteration give both axes. Result: ac[n] = (out_x[n], out_y[n]). A holds the packed
// profile in bit-reversed order on entry (as qi_profiles_sym writes it). Warp 0 only.
__device__ inline void qi_autoconv_fft_filled(int nr, float2 *A, float2 *ac, const float2 *tw)
{
    const int lane = threadIdx.x & 31;
    const int L = 2 * nr, log2L = ilog2_pow2(L);
    warp_fft(A, L, log2L, tw, false);
    for (int k = lane; k < L; k += 32) {
        const float2 Zk = A[k];
        const float2 Zc = A[(L - k) & (L - 1)];
        // split the packed transform: Px = (Z[k] + conj Z[L-k]) / 2, Py = (Z[k] - conj Z[L-k]) / 2i
        const float2 Px = make_float2(0.5f * (Zk.x + Zc.x), 0.5f * (Zk.y - Zc.y));
        const float2 Py = make_float2(0.5f * (Zk.y + Zc.y), -0.5f * (Zk.x - Zc.x));
        float2 e = tw[k & ((L >> 1) - 1)];
        if (k >= (L >> 1)) e = make_float2(-e.x, -e.y);
        const float2 Ax = cmul(e, cmul(Px, Px));
        const float2 Ay = cmul(e, cmul(Py, Py));
        ac[bitrev(k, log2L)] = make_float2(Ax.x - Ay.y, Ax.y + Ay.x);
    }
    __syncwarp();
    warp_fft(ac, L, log2L, tw, true);
}


// Same quantity by direct summation (any L; used when 2nr is not a power of two), A already
// holding the packed profile in natural order and a barrier passed. All threads.
__device__ inline void qi_autoconv_direct_filled(int nr, const float2 *A, float2 *ac)
{
    const int L = 2 * nr;
    for (int n = threadIdx.x; n < L; n += blockDim.x) {
        float sx = 0.0f, sy = 0.0f;
        for (int m = 0; m < L; m++) {
            int idx = n + m;
            if (idx >= L) idx -= L;
            const float2 a = A[idx], b = A[L - 1 - m];
            sx += a.x * b.x;
            sy += a.y * b.y;
        }
        ac[n] = make_float2(L * sx, L * sy);
    }
    __syncthreads();
}

// -------------------------------------------------------------------------------------
// ComputeRadialProfile, utils.cpp:275-320: for each bin, the mean of the in-bounds
// bilinear samples on the full circle (FP64 sum), or `mean` when no more than 4 samples
// are in bounds; then NormalizeRadialProfile (utils.cpp:230-261) when asked.
// -------------------------------------------------------------------------------------
__device__ __forceinline__ void radial_profile(const float *img, int W, int H, int ts, float cx, float cy, float mean, int nb, int nang,
                               float minr, float rstep, const float4 *dirs, float *prof, bool normalize,
                               double *red)
{
    // dirs[j] = (d_j.x, d_{j+h}.x, d_j.y, d_{j+h}.y) for j < h = nang/2, and d_{nang-1} alone in
    // dirs[h] when nang is odd: each lane takes pairs j = sub, sub + tpb, ... (two samples per
    // step, packed FP32x2) and lane 0 of each bin the unpaired direction.
    const int tpb = lanes_per_bin(nb), ltpb = ilog2_pow2(tpb);
    const int total = nb * tpb, h = nang >> 1;
    const bool odd = (nang & 1) != 0;
    for (int base = 0; base < total; base += blockDim.x) {
        const int t = base + threadIdx.x;
        const int bin = t >> ltpb, sub = t & (tpb - 1);
        double sum = 0.0;
        int cnt = 0;
        const float r = minr + rstep * (float)bin;
        // one path per warp (see qi_profiles_sym)
        const bool inside = __all_sync(0xffffffffu, bin >= nb || circle_inside(cx, cy, fabsf(r), W, H));
        if (bin < nb && inside) {
            // Whole groups of 4 pairs (8 samples) are summed in FP32 and folded into an FP64
            // total (the reference adds every sample in FP64; 8-sample FP32 groups stay within
            // ~1e-7 of it), then the remaining pairs, then the unpaired direction.
            const float2 rr = make_float2(r, r), cxx = make_float2(cx, cx), cyy = make_float2(cy, cy);
            const int np = sub < h ? (h - sub + tpb - 1) >> ltpb : 0;
            const float4 *dl = dirs + sub;
            int k = 0;
            for (; k + 4 <= np; k += 4) {
                float2 part = make_float2(0.0f, 0.0f);
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const float4 d = dl[(k + u) << ltpb];
                    part = __fadd2_rn(part, bilinear_inside2(img, ts, __ffma2_rn(make_float2(d.x, d.y), rr, cxx),
                                                             __ffma2_rn(make_float2(d.z, d.w), rr, cyy)));
                }
                sum += (double)(part.x + part.y);
            }
            if (k < np) {
                float2 part = make_float2(0.0f, 0.0f);
                for (; k < np; k++) {
                    const float4 d = dl[k << ltpb];
                    part = __fadd2_rn(part, bilinear_inside2(img, ts, __ffma2_rn(make_float2(d.x, d.y), rr, cxx),
                                                             __ffma2_rn(make_float2(d.z, d.w), rr, cyy)));
                }
                sum += (double)(part.x + part.y);
            }
            cnt = 2 * np;
            if (odd && sub == 0) {
                const float4 d = dirs[h];
                sum += (double)bilinear_inside(img, ts, cx + d.x * r, cy + d.z * r);
                cnt++;
            }
        } else if (bin < nb) {
            // every sample checked; FP32 partials of up to 8 samples folded into FP64
            for (int j0 = sub; j0 < h; j0 += 4 * tpb) {
                float part = 0.0f;
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    const int j = j0 + u * tpb;
                    if (j >= h) break;
                    const float4 d = dirs[j];
                    float v;
                    if (bilinear(img, W, H, ts, cx + d.x * r, cy + d.z * r, v)) {
                        part += v;
                        cnt++;
                    }
                    if (bilinear(img, W, H, ts, cx + d.y * r, cy + d.w * r, v)) {
                        part += v;
                        cnt++;
                    }
                }
                sum += (double)part;
            }
            if (odd && sub == 0) {
                const float4 d = dirs[h];
                float v;
                if (bilinear(img, W, H, ts, cx + d.x * r, cy + d.z * r, v)) {
                    sum += (double)v;
                    cnt++;
                }
            }
        }
        for (int o = tpb >> 1; o > 0; o >>= 1) {
            sum += __shfl_xor_sync(0xffffffffu, sum, o);
            cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        }
        if (bin < nb && sub == 0) prof[bin] = cnt > 4 ? (float)(sum / cnt) : mean;
    }
    __syncthreads();
    if (normalize && threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double s = 0;
        for (int i = lane; i < nb; i += 32) s += prof[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        const float m = (float)(s / nb);
        double s2 = 0;
        for (int i = lane; i < nb; i += 32) {
            const float p = prof[i] - m;
            prof[i] = p;
            s2 += (double)(p * p);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        const double inv = 1.0 / sqrt(s2 / nb);
        for (int i = lane; i < nb; i += 32) prof[i] = (float)((double)prof[i] * inv);
    }
    __syncthreads();
}

// One plane's score of CPUTracker::LUTProfileCompare (cpu_tracker.cpp:820-830) in the reference's
// arithmetic and order: d = (double)(p_r - L_kr) with the difference taken in FP32, d *= w_r,
// then sum += -(d * d) over r = 0 .. nb-1 in FP64, every operation rounded on its own (no
// contraction). Given the same profile, the score equals the reference's bit for bit.
// lut_k[r * stride] is L_kr.
__device__ __forceinline__ double zlut_score(const float *prof, const float *lut_k, int stride, const float *w, int nb)
{
    double acc = 0.0;
#pragma unroll 8
    for (int r = 0; r < nb; r++) {
        double d = (double)(prof[r] - __ldg(lut_k + (size_t)r * stride));
        if (w) d = __dmul_rn(d, (double)__ldg(w + r));
        acc = __dadd_rn(acc, -__dmul_rn(d, d));
    }
    return acc;
}

// The plain Z match: one thread per plane, reading the transposed LUT ([bin][plane], `pitch`
// planes per bin) so that a warp's 32 planes are one coalesced 128-byte load per bin.
__device__ inline void zlut_scores_plain(const float *prof, const float *lut_t, int pitch, int planes, int nb,
                                         const float *weights, double *scores)
{
    for (int k = threadIdx.x; k < planes; k += blockDim.x) scores[k] = zlut_score(prof, lut_t + k, pitch, weights, nb);
    __syncthreads();
}

// QueuedTracker::ZLUTBiasCorrection, cputrack/QueuedTracker.cpp:115-140: four fixed-point steps
// pos = z - bias(pos), bias read from the bead's row of the table by Interpolate1D
// (cputrack/utils.h:60-67: truncating index, clamped to the first/last entry).
__device__ __forceinline__ float zlut_bias_correct(float z, int planes, const float *table, int tw, int tcount,
                                                   int bead)
{
    if (!table || bead < 0 || bead >= tcount || tw <= 0) return z;
    const float *row = table + (size_t)bead * tw;
    float pos = z;
    for (int k = 0; k < 4; k++) {
        const float tblpos = pos / (float)planes * tw;
        const int fx = (int)tblpos;
        float bias;
        if (fx < 0)
            bias = row[0];
        else if (fx >= tw - 1)
            bias = row[tw - 1];
        else
            bias = (row[fx + 1] - row[fx]) * (tblpos - fx) + row[fx];
        pos = z - bias;
    }
    return pos;
}

// -------------------------------------------------------------------------------------
// 2D Gaussian MLE, CPUTracker::Compute2DGaussianMLE (cpu_tracker.cpp:514-589):
// 4 parameters (x, y, I0, bg), fixed sigma, per-parameter Newton steps. The erf is the
// Abramowitz & Stegun 7.1.26 form the reference binds (utils.h:395-417). Per iteration the
// erf/exp terms depend only on the column (x) or the row (y), so they are evaluated once
// per column and per row and combined per pixel.
// -------------------------------------------------------------------------------------
__device__ __forceinline__ float erf_as(float x, float e_mx2)
{
    // e_mx2 = exp(-x*x)
    const float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f, a4 = -1.453152027f,
                a5 = 1.061405429f, p = 0.3275911f;
    const float sign = x < 0 ? -1.0f : 1.0f;
    const float ax = fabsf(x);
    const float t = 1.0f / (1.0f + p * ax);
    const float y = 1.0f - (((((a5 * t + a4) * t) + a3) * t + a2) * t + a1) * t * e_mx2;
    return sign * y;
}

// Column (or row) terms for coordinate c at position p: D = 0.5 erf(c0) - 0.5 erf(c1),
// g = e^{-c1^2} - e^{-c0^2}, h = (c-p-.5) e^{-c1^2} - (c-p+.5) e^{-c0^2}.
struct GaussAxisTerms {
    float D, g, h;
};

__device__ __forceinline__ GaussAxisTerms gauss_axis_terms(int c, float p, float k1)
{
    const float e0 = (c - p + .5f) * k1;
    const float e1 = (c - p - .5f) * k1;
    const float x0 = expf(-e0 * e0), x1 = expf(-e1 * e1);
    GaussAxisTerms t;
    t.D = 0.5f * erf_as(e0, x0) - 0.5f * erf_as(e1, x1);
    t.g = x1 - x0;
    t.h = (c - p - .5f) * x1 - (c - p + .5f) * x0;
    return t;
}


// CPUTracker::Compute2DGaussianMLE, cpu_tracker.cpp:514-589. col: 3*W floats, row: 3*H floats
// of shared scratch. px/py enter as the start position (the COM) and leave as the estimate.
template <class G>
__device__ inline void gauss4_mle(const G &g, const float *img, int W, int H, float mean, float &px, float &py, int iters,
                           float sigma, float *col, float *row)
{
    float I0 = mean * 0.5f * (float)W * (float)H;
    float bg = mean * 0.5f;
    const float k1 = 1.0f / (sqrtf(2.0f) * sigma);
    const float k2 = 1.0f / (sqrtf(2 * 3.14159265359f) * sigma);
    const float k3 = 1.0f / (sqrtf(2 * 3.14159265359f) * sigma * sigma * sigma);
    for (int it = 0; it < iters; it++) {
        g.sync();
        for (int c = g.rank(); c < W; c += g.size()) {
            const GaussAxisTerms t = gauss_axis_terms(c, px, k1);
            col[3 * c] = t.D;
            col[3 * c + 1] = t.g;
            col[3 * c + 2] = t.h;
        }
        for (int r = g.rank(); r < H; r += g.size()) {
            const GaussAxisTerms t = gauss_axis_terms(r, py, k1);
            row[3 * r] = t.D;
            row[3 * r + 1] = t.g;
            row[3 * r + 2] = t.h;
        }
        g.sync();
        double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (int i = g.rank(); i < W * H; i += g.size()) {
            const int y = i / W, x = i - y * W;
            const float DX = col[3 * x], gX = col[3 * x + 1], hX = col[3 * x + 2];
            const float DY = row[3 * y], gY = row[3 * y + 1], hY = row[3 * y + 2];
            const float mu = bg + I0 * DX * DY;
            const float dmu_dx = I0 * k2 * gX * DY;
            const float dmu_dy = I0 * k2 * gY * DX;
            const float dmu_dI0 = DX * DY;
            const float smp = img[i];
            const float f = smp / mu - 1;
            acc[0] += dmu_dx * f;
            acc[1] += dmu_dy * f;
            acc[2] += dmu_dI0 * f;
            acc[3] += f;
            const float d2mu_dx = I0 * k3 * hX * DY;
            const float d2mu_dy = I0 * k3 * hY * DX;
            const float mu2 = mu * mu;
            acc[4] += d2mu_dx * f - dmu_dx * dmu_dx * smp / mu2;
            acc[5] += d2mu_dy * f - dmu_dy * dmu_dy * smp / mu2;
            acc[6] += -dmu_dI0 * dmu_dI0 * smp / mu2;
            acc[7] += -smp / mu2;
        }
        g.sum(acc);
        px = (float)((double)px - acc[0] / acc[4]);
        py = (float)((double)py - acc[1] / acc[5]);
        I0 = (float)((double)I0 - acc[2] / acc[6]);
        bg = (float)((double)bg - acc[3] / acc[7]);
    }
}

// Solve the symmetric 5x5 system A d = b (Gaussian elimination, partial pivoting, FP64).
// Gaussian elimination with partial pivoting. The pivot row is found by swapping, row by row, any
// row whose entry is larger in magnitude into the pivot position: every index is a compile-time
// constant after unrolling, so the matrix stays in registers (a dynamically indexed row swap
// would put it in local memory). The pivot chosen and every operation on a row are those of
// the classic search-then-swap form.
__device__ __forceinline__ bool solve5(double (&A)[5][5], double (&b)[5], double (&d)[5])
{
#pragma unroll
    for (int c = 0; c < 5; c++) {
#pragma unroll
        for (int r = c + 1; r < 5; r++) {
            const bool sw = fabs(A[r][c]) > fabs(A[c][c]);
#pragma unroll
            for (int j = 0; j < 5; j++) {
                const double t = A[c][j];
                A[c][j] = sw ? A[r][j] : t;
                A[r][j] = sw ? t : A[r][j];
            }
            const double t = b[c];
            b[c] = sw ? b[r] : t;
            b[r] = sw ? t : b[r];
        }
        if (!(fabs(A[c][c]) > 1e-300)) return false;
#pragma unroll
        for (int r = c + 1; r < 5; r++) {
            const double f = A[r][c] / A[c][c];
#pragma unroll
            for (int j = c; j < 5; j++) A[r][j] -= f * A[c][j];
            b[r] -= f * b[c];
        }
    }
#pragma unroll
    for (int i = 4; i >= 0; i--) {
        double s = b[i];
#pragma unroll
        for (int j = i + 1; j < 5; j++) s -= A[i][j] * d[j];
        d[i] = s / A[i][i];
    }
    return true;
}

// Extension (no reference counterpart): 5-parameter (x, y, I0, bg, sigma) Poisson MLE of an
// integrated Gaussian spot, full Newton (Fisher-scoring) steps. Likelihood terms and
// gradients in FP32 per pixel, FP64 reduction and an FP64 5x5 solve per step. p[] = {x, y,
// I0, bg, sigma}; col/row: 5*W and 5*H floats of shared scratch.
template <class G>
__device__ inline void gauss5_mle(const G &g, const float *img, int W, int H, float (&p)[5], int iters, float *col,
                           float *row)
{
    for (int it = 0; it < iters; it++) {
        const float s = p[4];
        const float k1 = 1.0f / (sqrtf(2.0f) * s);
        const float k2 = 1.0f / (sqrtf(2 * 3.14159265359f) * s);
        g.sync();
        for (int c = g.rank(); c < W + H; c += g.size()) {
            const bool is_col = c < W;
            const int cc = is_col ? c : c - W;
            const float pc = is_col ? p[0] : p[1];
            const float a0 = (cc - pc + .5f) * k1, a1 = (cc - pc - .5f) * k1;
            const float e0 = expf(-a0 * a0), e1 = expf(-a1 * a1);
            float *t = is_col ? col + 3 * cc : row + 3 * cc;
            t[0] = 0.5f * (erff(a0) - erff(a1));
            t[1] = (e1 - e0) * k2;                                                  // dD/dp
            t[2] = ((cc - pc - .5f) * e1 - (cc - pc + .5f) * e0) * k2 / s;          // dD/dsigma
        }
        g.sync();
        float a[20];
#pragma unroll
        for (int k = 0; k < 20; k++) a[k] = 0.0f;
        for (int i = g.rank(); i < W * H; i += g.size()) {
            const int y = i / W, x = i - y * W;
            const float DX = col[3 * x], dX = col[3 * x + 1], sX = col[3 * x + 2];
            const float DY = row[3 * y], dY = row[3 * y + 1], sY = row[3 * y + 2];
            const float mu = p[3] + p[2] * DX * DY;
            const float J[5] = {p[2] * dX * DY, p[2] * DX * dY, DX * DY, 1.0f, p[2] * (sX * DY + DX * sY)};
            const float f = img[i] / mu - 1.0f;
            const float imu = 1.0f / mu;
            int k = 5;
#pragma unroll
            for (int u = 0; u < 5; u++) {
                a[u] += J[u] * f;
#pragma unroll
                for (int v = u; v < 5; v++) a[k++] += J[u] * J[v] * imu;
            }
        }
        double acc[20];
#pragma unroll
        for (int k = 0; k < 20; k++) acc[k] = a[k];
        g.sum(acc);
        double A[5][5], b[5], d[5];
        int k = 5;
#pragma unroll
        for (int u = 0; u < 5; u++) {
            b[u] = acc[u];
#pragma unroll
            for (int v = u; v < 5; v++) A[u][v] = A[v][u] = acc[k++];
        }
        if (!solve5(A, b, d)) break;
#pragma unroll
        for (int u = 0; u < 5; u++) p[u] = (float)((double)p[u] + d[u]);
        p[2] = fmaxf(p[2], 1e-3f);
        p[3] = fmaxf(p[3], 1e-3f);
        p[4] = fminf(fmaxf(p[4], 0.3f), 0.5f * (float)W);
    }
}

}  // namespace qtrk
