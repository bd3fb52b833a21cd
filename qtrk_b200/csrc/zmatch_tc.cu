// Z-LUT match on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// The plain match (cputrack/cpu_tracker.cpp:829-838) scores every plane k of a bead's LUT as
// score_k = -sum_r (w_r (p_r - L_kr))^2. Expanded,
//   score_k = -|p'|^2 + 2 p'.L'_k - |L'_k|^2,    p' = w p,  L'_k = w L_k,
// and for one ROI the first term is a constant, so the argmax only needs
// s_k = 2 p'.L'_k - |L'_k|^2. For a tile of 128 ROIs that share a bead, the cross terms are
// one GEMM [128 x K] . [K x planes] (K = radial bins): BF16 operands staged in shared memory,
// FP32 accumulators in tensor memory, one tcgen05.mma per 16-wide K slice issued by a single
// thread. The epilogue reads each ROI's row of accumulators (one TMEM lane per thread) and
// re-scores exactly (FP32 differences, FP64 sums, as the plain path) every plane whose BF16
// score can still be the best: with round-to-nearest BF16 operands the error of s_k is at most
// d_k = 2^-6 (1.01) |p'| |L'_k| (Cauchy-Schwarz on the per-product error 2^-7 |p'_r L'_kr|), so
// the exact argmax k* satisfies s~_k* >= max s~ - d_max - d_k*, and every plane passing that
// test is re-scored. Each operand is split into a high and a low BF16 part (x = x_hi + x_lo
// + O(2^-16 x)) and the cross term is p_hi.L_hi + p_hi.L_lo + p_lo.L_hi (three MMAs per K
// slice, all accumulated in the same FP32 tensor-memory tile), which brings the error bound
// down to d_k = 2^-9 |p'| |L'_k| (a generous cover of the ~3 2^-16 split error plus the FP32
// accumulation of 3 K products), so only a few planes per ROI need the exact re-score. With
// LT_B200_ZMatchTF32 the operands are w p and w L rounded to TF32 (kind::tf32, K = 8 per MMA,
// one MMA per K step) and d_k = 2^-9 (1.02) |p'| |L'_k| (kBoundScaleTF32). Threads
// record those candidate planes from their TMEM rows; warps then compute the exact scores with
// the plain path's per-plane function (zlut_score: one lane per plane, bins in order), take the
// argmax and run the 7-point fit (LsqQuadraticFit.h:132-176) with the plain path's warp code, so z
// is the plain path's bit for bit.
//
// Launch: one CTA of 128 threads per tile. Shared memory is sized so that at most two CTAs
// share an SM, so the two 256-column TMEM allocations always fit the SM's 512 columns and
// tcgen05.alloc never waits. Every wait on the MMA-completion mbarrier is bounded; on timeout
// the kernel records an error flag and skips the tensor-memory read. The MMAs it gave up on may
// still be writing the accumulator columns, so before the columns are released thread 0 waits
// again for that commit (a second, longer bound, kDrainLimit); only if that wait also gives up
// are the columns released with the MMAs possibly still in flight (flag bit 2: the results of the
// launch are void). Releasing is preferred to keeping the columns, since a CTA that exits holding
// them could leave a later CTA on the same SM waiting in tcgen05.alloc.
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "device_common.cuh"
#include "kernels.h"
#include "zmatch_tc.h"

namespace qtrk {

namespace {

constexpr int kTileM = 128;
constexpr int kMaxN = 256;   // N per tcgen05.mma (M = 128 allows N <= 256 in steps of 16)
constexpr float kBoundScale = 0.001953125f;  // 2^-9 (see above)
// TF32 operands, rounded to nearest (cvt.rna) when staged: 10 explicit mantissa bits, each factor
// within 2^-11, so a product within 2^-10 + 2^-22; with the FP32 accumulation of <= 128 products
// (2^-17) and the FP32 rounding of w p and w L, |d(p'.L'_k)| <= (2^-10 + 2^-16) |p'| |L'_k|, and
// s_k = 2 p'.L'_k - |L'_k|^2 is within 2^-9 (1.016) |p'| |L'_k|; the scale below covers it.
constexpr float kBoundScaleTF32 = 0.0020f;
constexpr int kTmemCols = 256;
constexpr uint32_t kWaitLimit = 1u << 20;   // try_wait polls before the kernel gives up
constexpr uint32_t kDrainLimit = 1u << 24;  // polls for the abandoned commit before the columns are released
constexpr int kMaxCand = 16;  // candidate planes kept per ROI; more fall back to scoring every plane
constexpr int kWarps = kTileM / 32;

// Bytes after the A/B tiles: mbarrier (8) + TMEM slot (8), then |p'| per row (kTileM floats),
// candidate counts (kTileM ints), candidate planes (kTileM x kMaxCand shorts) and one 8-double
// score window per warp.
constexpr int kTailBytes = 16 + kTileM * 4 + kTileM * 4 + kTileM * kMaxCand * 2 + kWarps * 8 * 8;

__device__ const float kZLUTWeightsTC[7] = {0.15f, 0.5f, 0.85f, 1.0f, 0.85f, 0.5f, 0.15f};

// x rounded to TF32 (round to nearest, ties away from zero), as a 32-bit pattern
__device__ __forceinline__ uint32_t to_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, K-major, no swizzle: 14-bit start address (>>4), leading
// byte offset (K direction, >>4) at bit 16, stride byte offset (M/N direction, >>4) at bit 32,
// descriptor version 1 at bit 46, layout type 0 (SWIZZLE_NONE) in bits 61-63.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// Instruction descriptor for kind::f16 / kind::tf32: FP32 accumulate (bits 4-5 = 1), A and B
// format in bits 7-9 and 10-12 (1 = BF16, 2 = TF32), both K-major, N >> 3 at bit 17, M >> 4 at
// bit 24.
__device__ __forceinline__ uint32_t make_idesc(int M, int N, bool tf32)
{
    const uint32_t fmt = tf32 ? 2u : 1u;
    return (1u << 4) | (fmt << 7) | (fmt << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
        :
        : "r"(tmem_d), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *mbar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(mbar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// Store one 16-byte chunk (8 BF16 along K) of row r, K-chunk c in the no-swizzle K-major
// core-matrix layout: core matrix (r/8, c) at (r/8)*SBO + c*LBO, row r%8 at 16 bytes each.
__device__ __forceinline__ void store_chunk(uint8_t *base, int r, int c, int sbo, uint4 v)
{
    *reinterpret_cast<uint4 *>(base + (r >> 3) * sbo + c * 128 + (r & 7) * 16) = v;
}

}  // namespace

__global__ void __launch_bounds__(kTileM, 1) zmatch_tc_kernel(ZMatchParams Q)
{
    extern __shared__ __align__(1024) uint8_t smem[];
    const int4 tile = Q.tiles ? Q.tiles[blockIdx.x]
                              : make_int4(blockIdx.x * kTileM, min(kTileM, Q.count - (int)blockIdx.x * kTileM),
                                          Q.uniform_bead, 0);
    const int start = tile.x, m = tile.y, bead = tile.z;
    const int tid = threadIdx.x, warp = tid >> 5;
    const int nbp = Q.nbp, kchunks = nbp >> 3, sbo = nbp * 16;
    // TF32: 4 elements per 16-byte chunk; A spans the A_hi and A_lo space, B the B_hi and B_lo space
    const bool tf32 = Q.tf32 != 0;
    const int kch32 = nbp >> 2, sbo32 = nbp * 32;
    const int nb = Q.nb;
    // [A_hi | A_lo | B_hi | B_lo], each in the no-swizzle K-major core-matrix layout
    uint8_t *sA = smem;
    uint8_t *sAl = sA + kTileM * nbp * 2;
    uint8_t *sB = sAl + kTileM * nbp * 2;
    uint8_t *sBl = sB + kMaxN * nbp * 2;
    uint64_t *mbar = reinterpret_cast<uint64_t *>(sBl + kMaxN * nbp * 2);
    uint32_t *tslot = reinterpret_cast<uint32_t *>(mbar + 1);
    float *s_pnorm = reinterpret_cast<float *>(mbar + 2);
    int *s_ncand = reinterpret_cast<int *>(s_pnorm + kTileM);
    short *s_cand = reinterpret_cast<short *>(s_ncand + kTileM);
    double *s_win = reinterpret_cast<double *>(s_cand + kTileM * kMaxCand);

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)),
                     "r"(kTmemCols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    }
    if (tid == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }

    // A: this tile's weighted profiles, BF16 hi/lo or FP32 (rows beyond m are zero)
    const bool valid_bead = bead >= 0 && bead < Q.lut_count;
    int my_roi = -1;
    if (tid < m) my_roi = Q.perm ? Q.perm[start + tid] : start + tid;
    for (int idx = tid; tf32 && idx < kTileM * kch32; idx += kTileM) {
        const int r = idx / kch32, c = idx - r * kch32;
        float e[4] = {0.0f, 0.0f, 0.0f, 0.0f};
        if (r < m) {
            const int roi = Q.perm ? Q.perm[start + r] : start + r;
            const float *pr = Q.prof_f32 + (size_t)roi * nb;
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const int b = 4 * c + j;
                if (b < nb) e[j] = Q.weights ? pr[b] * Q.weights[b] : pr[b];
            }
        }
        store_chunk(sA, r, c, sbo32, make_uint4(to_tf32(e[0]), to_tf32(e[1]), to_tf32(e[2]), to_tf32(e[3])));
    }
    for (int idx = tid; !tf32 && idx < kTileM * kchunks; idx += kTileM) {
        const int r = idx / kchunks, c = idx - r * kchunks;
        uint4 vh = make_uint4(0, 0, 0, 0), vl = vh;
        if (r < m) {
            const int roi = Q.perm ? Q.perm[start + r] : start + r;
            const __nv_bfloat16 *src = Q.prof_bf16 + (size_t)roi * 2 * nbp;  // [hi | lo]
            vh = *reinterpret_cast<const uint4 *>(src + c * 8);
            vl = *reinterpret_cast<const uint4 *>(src + nbp + c * 8);
        }
        store_chunk(sA, r, c, sbo, vh);
        store_chunk(sAl, r, c, sbo, vl);
    }

    // |p'| of each row's ROI (FP32 profile times the radial weights), one warp per row, lanes over
    // bins; FP64 sums rounded up by 2^-20 so that the bound below stays a bound
    const float *prof = (my_roi >= 0) ? Q.prof_f32 + (size_t)my_roi * nb : nullptr;
    for (int r = warp; r < kTileM; r += kWarps) {
        double s2 = 0.0;
        if (r < m) {
            const int roi = Q.perm ? Q.perm[start + r] : start + r;
            const float *pr = Q.prof_f32 + (size_t)roi * nb;
            for (int b = tid & 31; b < nb; b += 32) {
                const double v = Q.weights ? (double)pr[b] * Q.weights[b] : (double)pr[b];
                s2 += v * v;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        if ((tid & 31) == 0) s_pnorm[r] = (float)(sqrt(s2) * (1.0 + 0x1p-20));
    }
    float pnorm = 0.0f;  // read after the first barrier of the chunk loop
    int nc = 0;          // candidate planes of this thread's row (may exceed kMaxCand)
    const int gb = valid_bead ? bead : 0;
    const float *lut = Q.lut + (size_t)gb * Q.planes * nb;
    const float *lnorm = Q.lut_norm + (size_t)gb * Q.planes_pad;

    float smax = -INFINITY, dmax = 0.0f;  // tensor-core maximum so far and its error bound
    const float bscale = tf32 ? kBoundScaleTF32 : kBoundScale;
    bool failed = false;
    uint32_t parity = 0;
    uint32_t pending_parity = 0;  // phase of the commit a timed-out wait gave up on
    const int planes_pad = Q.planes_pad;
    for (int n0 = 0; n0 < planes_pad; n0 += kMaxN) {
        const int n = min(kMaxN, planes_pad - n0);
        // TF32: w L from the FP32 LUT (planes beyond the LUT and bins beyond nb are zero)
        for (int idx = tid; tf32 && idx < n * kch32; idx += kTileM) {
            const int r = idx / kch32, c = idx - r * kch32, k = n0 + r;
            float e[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            if (k < Q.planes) {
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    const int b = 4 * c + j;
                    if (b < nb) e[j] = Q.weights ? lut[(size_t)k * nb + b] * Q.weights[b] : lut[(size_t)k * nb + b];
                }
            }
            store_chunk(sB, r, c, sbo32, make_uint4(to_tf32(e[0]), to_tf32(e[1]), to_tf32(e[2]), to_tf32(e[3])));
        }
        // BF16 LUT layout [bead][hi, lo][planes_pad][nbp]
        const __nv_bfloat16 *lutb = Q.lut_bf16 + ((size_t)gb * 2 * planes_pad + n0) * nbp;
        const __nv_bfloat16 *lutl = lutb + (size_t)planes_pad * nbp;
        for (int idx = tid; !tf32 && idx < n * kchunks; idx += kTileM) {
            const int r = idx / kchunks, c = idx - r * kchunks;
            store_chunk(sB, r, c, sbo, *reinterpret_cast<const uint4 *>(lutb + (size_t)r * nbp + c * 8));
            store_chunk(sBl, r, c, sbo, *reinterpret_cast<const uint4 *>(lutl + (size_t)r * nbp + c * 8));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        pnorm = s_pnorm[tid];
        const uint32_t tmem = *tslot;
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t idesc = make_idesc(kTileM, n, tf32);
            const uint32_t a0 = smem_u32(sA), al = smem_u32(sAl), b0 = smem_u32(sB), bl = smem_u32(sBl);
            // TF32: K = 8 per MMA (32 bytes, two core matrices), one MMA per K step
            for (int k = 0; tf32 && k < (nbp >> 3); k++)
                mma_tf32(tmem, make_desc(a0 + k * 256, 128, sbo32), make_desc(b0 + k * 256, 128, sbo32), idesc, k > 0);
            for (int k = 0; !tf32 && k < (nbp >> 4); k++) {
                const uint64_t ah = make_desc(a0 + k * 256, 128, sbo), alo = make_desc(al + k * 256, 128, sbo);
                const uint64_t bh = make_desc(b0 + k * 256, 128, sbo), blo = make_desc(bl + k * 256, 128, sbo);
                mma_bf16(tmem, ah, bh, idesc, k > 0);
                mma_bf16(tmem, ah, blo, idesc, 1);
                mma_bf16(tmem, alo, bh, idesc, 1);
            }
            mma_commit(mbar);
        }
        uint32_t polls = 0;
        pending_parity = parity;
        while (!mbar_try_wait(mbar, parity)) {
            if (++polls > kWaitLimit) {
                failed = true;
                break;
            }
        }
        parity ^= 1;
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (__syncthreads_or(failed)) {
            failed = true;
            break;
        }
        // row tid of the accumulator is TMEM lane tid; warp w may read lanes 32w..32w+31
        const uint32_t trow = tmem + ((uint32_t)(warp * 32) << 16);
        // pass 1: BF16 maximum over this chunk (with the bound of the maximising plane)
        for (int c0 = 0; c0 < n; c0 += 16) {
            float v[16];
            tmem_ld16(trow + (uint32_t)c0, v);
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const int k = n0 + c0 + j;
                if (k < Q.planes) {
                    const float sk = 2.0f * v[j] - lnorm[k];
                    if (sk > smax) {
                        smax = sk;
                        dmax = bscale * pnorm * sqrtf(lnorm[k]);
                    }
                }
            }
        }
        // pass 2: record every plane that can still be the best (its exact score is computed by
        // the warps afterwards). The TMEM load is warp-collective (.sync.aligned), so every lane
        // executes it; lanes without a ROI record nothing.
        for (int c0 = 0; c0 < n; c0 += 16) {
            float v[16];
            tmem_ld16(trow + (uint32_t)c0, v);
            if (prof && valid_bead) {
#pragma unroll 1
                for (int j = 0; j < 16; j++) {
                    const int k = n0 + c0 + j;
                    if (k >= Q.planes) continue;
                    const float sk = 2.0f * v[j] - lnorm[k];
                    const float dk = bscale * pnorm * sqrtf(lnorm[k]);
                    const float thr = smax - dmax - dk - 1e-5f * (1.0f + fabsf(smax));
                    if (sk >= thr) {
                        if (nc < kMaxCand) s_cand[tid * kMaxCand + nc] = (short)k;
                        nc++;
                    }
                }
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();  // accumulators read before the next chunk overwrites sB / TMEM
    }

    // Exact scores of the candidates (zlut_score: the plain path's arithmetic and order, so the
    // scores, argmax and fit are the plain path's bit for bit), argmax (the first of equal maxima,
    // NaN skipped: warp_argmax of the plain path), and the 7-point fit (LsqQuadraticFit.h:148-171)
    // on exact scores around it: one warp per ROI row, one lane per candidate plane. A row with more
    // than kMaxCand candidates is scored over every plane.
    s_ncand[tid] = nc;
    __syncthreads();
    const int lane = tid & 31;
    double *win = s_win + warp * 8;
    for (int r = warp; r < m; r += kWarps) {
        const int roi = Q.perm ? Q.perm[start + r] : start + r;
        float z = 0.0f;
        if (failed) {
            z = __int_as_float(0x7fc00000);
        } else if (valid_bead) {
            const float *pr = Q.prof_f32 + (size_t)roi * nb;
            const int cnt = s_ncand[r];
            const bool all = cnt > kMaxCand;
            const int ncheck = all ? Q.planes : cnt;
            double best = 0.0;
            int bk = -1;
            for (int i = lane; i < ncheck; i += 32) {
                const int k = all ? i : s_cand[r * kMaxCand + i];
                const double e = zlut_score(pr, lut + (size_t)k * nb, 1, Q.weights, nb);
                if (e == e && (bk < 0 || e > best || (e == best && k < bk))) {
                    best = e;
                    bk = k;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(0xffffffffu, best, o);
                const int ok = __shfl_xor_sync(0xffffffffu, bk, o);
                if (ok >= 0 && (bk < 0 || ob > best || (ob == best && ok < bk))) {
                    best = ob;
                    bk = ok;
                }
            }
            if (bk < 0) bk = 0;
            const int s0 = max(bk - 3, 0), s1 = min(bk + 4, Q.planes);
            if (lane < s1 - s0) win[lane] = zlut_score(pr, lut + (size_t)(s0 + lane) * nb, 1, Q.weights, nb);
            __syncwarp();
            auto at = [&](int k) { return win[k - s0]; };
            const float zz = max_interp7_sym(at, Q.planes, bk, kZLUTWeightsTC);
            z = zlut_bias_correct((float)zz, Q.planes, Q.zbias, Q.zbias_w, Q.zbias_count, bead);
            __syncwarp();
        }
        if ((tid & 31) == 0) reinterpret_cast<float *>(Q.results)[(size_t)roi * 13 + 8] = z;
    }
    if (failed && tid == 0) {
        // Wait for the commit of the MMAs this CTA gave up on (they arrive on the mbarrier once
        // they have finished writing TMEM) before the columns are released below.
        uint32_t polls = 0;
        bool drained = true;
        while (!mbar_try_wait(mbar, pending_parity)) {
            if (++polls > kDrainLimit) {
                drained = false;
                break;
            }
        }
        if (Q.error_flag) atomicOr(Q.error_flag, drained ? 1u : 3u);
    }

    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        const uint32_t tmem = *tslot;
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
    }
}

// Weighted BF16 hi/lo split of each LUT row (padded to nbp bins and planes_pad planes with
// zeros; layout [bead][hi, lo][planes_pad][nbp]) and the FP32 norm |w L_k|^2 of each plane.
// One warp per (bead, plane) row.
__global__ void zmatch_prepare_lut_kernel(const float *__restrict__ lut, const float *__restrict__ weights,
                                          int count, int planes, int nb, int planes_pad, int nbp,
                                          __nv_bfloat16 *__restrict__ lut_bf16, float *__restrict__ lut_norm)
{
    const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (row >= count * planes_pad) return;
    const int lane = threadIdx.x & 31;
    const int bead = row / planes_pad, k = row - bead * planes_pad;
    float s = 0.0f;
    __nv_bfloat16 *hi = lut_bf16 + ((size_t)bead * 2 * planes_pad + k) * nbp;
    __nv_bfloat16 *lo = hi + (size_t)planes_pad * nbp;
    for (int r = lane; r < nbp; r += 32) {
        float v = 0.0f;
        if (k < planes && r < nb) {
            v = lut[((size_t)bead * planes + k) * nb + r];
            if (weights) v *= weights[r];
            s += v * v;
        }
        const __nv_bfloat16 h = __float2bfloat16_rn(v);
        hi[r] = h;
        lo[r] = __float2bfloat16_rn(v - __bfloat162float(h));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) lut_norm[row] = s;
}

int zmatch_smem_bytes(int nbp)
{
    const int need = 2 * (kTileM * nbp * 2 + kMaxN * nbp * 2) + kTailBytes;
    // at least 80 KB so that no more than two CTAs (2 x 256 TMEM columns) share an SM
    return need > 80 * 1024 ? need : 80 * 1024;
}

int zmatch_padded_bins(int nb) { return (nb + 15) & ~15; }
int zmatch_padded_planes(int planes) { return (planes + 15) & ~15; }
bool zmatch_supported(int nb) { return nb >= 1 && zmatch_padded_bins(nb) <= 128; }

cudaError_t zmatch_prepare_lut(const float *lut, const float *weights, int count, int planes, int nb,
                               __nv_bfloat16 *lut_bf16, float *lut_norm, cudaStream_t stream)
{
    const int rows = count * zmatch_padded_planes(planes);
    if (rows <= 0) return cudaSuccess;
    zmatch_prepare_lut_kernel<<<(rows + 7) / 8, 256, 0, stream>>>(lut, weights, count, planes, nb,
                                                                  zmatch_padded_planes(planes),
                                                                  zmatch_padded_bins(nb), lut_bf16, lut_norm);
    return cudaGetLastError();
}

cudaError_t zmatch_prepare_kernel_attrs()
{
    return cudaFuncSetAttribute(zmatch_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
}

cudaError_t launch_zmatch_tc(const ZMatchParams &Q, int ntiles, cudaStream_t stream)
{
    if (ntiles <= 0) return cudaSuccess;
    zmatch_tc_kernel<<<ntiles, kTileM, zmatch_smem_bytes(Q.nbp), stream>>>(Q);
    return cudaGetLastError();
}

}  // namespace qtrk
