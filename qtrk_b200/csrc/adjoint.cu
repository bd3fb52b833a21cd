// Differentiable Z-LUT match: the radial-profile-to-LUT cost, its adjoint (gradients with respect to
// the bead position (x, y, z) and to the LUT entries), and the joint Gauss-Newton (x, y, z)
// refinement that runs after the Z fit in the LT_B200_JointRefine mode. No counterpart in the
// reference; the cost is built from the reference's own Z-match pieces:
//   p(x, y)  radial profile (cputrack/utils.cpp:275-320): per bin the mean of the in-bounds bilinear
//            samples (utils.h:40-58 truncation and outside rule) over z_angsteps directions, or the
//            image mean with at most 4 samples in bounds;
//   phat     NormalizeRadialProfile (utils.cpp:230-261) when LT_NormalizeProfile is set;
//   Lz       the bead's LUT, linear between planes iz = clamp(floor z, 0, planes-2) and iz+1;
//   cost     sum_r (w_r (phat_r - Lz_r))^2 with the Z radial weights w (1 when unset), the score
//            LUTProfileCompare (cpu_tracker.cpp:791-868) maximises, negated, between planes.
// dp/dx is the mean of the samples' bilinear x-derivatives ((v10-v00)(1-fy) + (v11-v01)fy), likewise
// dp/dy; through the normalisation dphat = (dp - mean(dp) - phat sum_j(phat_j dp_j)/n) / rms.
// Profiles are recomputed from the ROI (kept in shared memory), never stored as polar samples.
#include <cstdint>

#include "device_common.cuh"
#include "kernels.h"

namespace qtrk {

namespace {

constexpr int kAdjThreads = 256;
constexpr int kRefineSteps = 5;
constexpr float kPriorScale = 100.0f;  // x, y prior stiffness / z curvature (see joint_refine_kernel)

// Bilinear sample with its x and y derivatives inside the cell (same index rule as bilinear()).
__device__ __forceinline__ bool bilinear_grad(const float *img, int w, int h, float x, float y, float &v, float &gx,
                                              float &gy)
{
    if (!(x > -1.0f && x < (float)(w - 1) && y > -1.0f && y < (float)(h - 1))) return false;
    const float kMagic = 8388608.0f;
    const float tx = __fadd_rz(fmaxf(x, 0.0f), kMagic), ty = __fadd_rz(fmaxf(y, 0.0f), kMagic);
    const int rx = __float_as_int(tx) - 0x4B000000, ry = __float_as_int(ty) - 0x4B000000;
    const float *p = img + ry * w + rx;
    const float v00 = p[0], v10 = p[1], v01 = p[w], v11 = p[w + 1];
    const float fx = x - (tx - kMagic), fy = y - (ty - kMagic);
    const float v0 = v00 + (v10 - v00) * fx;
    const float v1 = v01 + (v11 - v01) * fx;
    v = v0 + (v1 - v0) * fy;
    gx = (v10 - v00) * (1.0f - fy) + (v11 - v01) * fy;
    gy = v1 - v0;
    return true;
}

struct AdjSmem {
    float *img;          // [H][W]
    double *p, *dx, *dy; // [nb] profile and its x/y derivatives (normalised in place)
    double *red;         // 128 doubles of reduction scratch (BlockGroup::sum<4>)
    double *misc;        // 16 doubles: broadcast values
};

__host__ __device__ inline int adj_img_bytes(const TrackParams &P) { return ((P.width * P.height * 4) + 15) & ~15; }

__host__ __device__ inline int adj_smem_bytes(const TrackParams &P)
{
    return adj_img_bytes(P) + 3 * P.z_nbins * 8 + 128 * 8 + 16 * 8;
}

__device__ AdjSmem adj_view(uint8_t *smem, const TrackParams &P)
{
    AdjSmem s;
    s.img = reinterpret_cast<float *>(smem);
    double *d = reinterpret_cast<double *>(smem + adj_img_bytes(P));
    s.p = d;
    s.dx = d + P.z_nbins;
    s.dy = d + 2 * P.z_nbins;
    s.red = d + 3 * P.z_nbins;
    s.misc = s.red + 128;
    return s;
}

// Profile (and derivatives) at (cx, cy): warps over bins, lanes over directions; FP32 sums of the
// <= ceil(angsteps / 32) samples of a lane, FP64 across lanes. Ends with a block barrier.
__device__ void profile_grad(const float *img, const TrackParams &P, float cx, float cy, float mean, double *p,
                             double *dx, double *dy)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int nb = P.z_nbins;
    const float rstep = (P.z_maxr - P.z_minr) / (float)nb;
    const float2 *dirs = static_cast<const float2 *>(P.z_dirs);
    for (int bin = warp; bin < nb; bin += nw) {
        const float r = P.z_minr + rstep * (float)bin;
        float s = 0.0f, sx = 0.0f, sy = 0.0f;
        int c = 0;
        for (int a = lane; a < P.z_angsteps; a += 32) {
            const float2 d = dirs[a];
            float v, gx, gy;
            if (bilinear_grad(img, P.width, P.height, cx + d.x * r, cy + d.y * r, v, gx, gy)) {
                s += v;
                sx += gx;
                sy += gy;
                c++;
            }
        }
        double ds = s, dsx = sx, dsy = sy;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            ds += __shfl_xor_sync(0xffffffffu, ds, o);
            dsx += __shfl_xor_sync(0xffffffffu, dsx, o);
            dsy += __shfl_xor_sync(0xffffffffu, dsy, o);
            c += __shfl_xor_sync(0xffffffffu, c, o);
        }
        if (lane == 0) {
            if (c > 4) {
                p[bin] = ds / c;
                dx[bin] = dsx / c;
                dy[bin] = dsy / c;
            } else {
                p[bin] = mean;
                dx[bin] = dy[bin] = 0.0;
            }
        }
    }
    __syncthreads();
}

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct CostTerms {
    double cost, g[3];      // cost and its gradient
    double A[6];            // J^T J: xx, xy, xz, yy, yz, zz (residual Jacobian, weights applied)
    double Jr[3];           // J^T res
};

// Warp 0: normalise p (and its derivatives) in place when asked, then the cost against the bead's
// LUT L [planes][nb] at z and its derivatives. Every lane of warp 0 returns the totals.
__device__ CostTerms cost_terms(const TrackParams &P, double *p, double *dx, double *dy, const float *L, float z)
{
    const int lane = threadIdx.x & 31, nb = P.z_nbins, planes = P.lut_planes;
    if (P.mode & kLT_NormalizeProfile) {
        double m = 0, mx = 0, my = 0;
        for (int i = lane; i < nb; i += 32) {
            m += p[i];
            mx += dx[i];
            my += dy[i];
        }
        m = warp_sum(m) / nb;
        mx = warp_sum(mx) / nb;
        my = warp_sum(my) / nb;
        double ss = 0;
        for (int i = lane; i < nb; i += 32) ss += (p[i] - m) * (p[i] - m);
        const double rms = sqrt(warp_sum(ss) / nb);
        double kx = 0, ky = 0;
        for (int i = lane; i < nb; i += 32) {
            const double ph = (p[i] - m) / rms;
            p[i] = ph;
            kx += ph * dx[i];
            ky += ph * dy[i];
        }
        kx = warp_sum(kx) / nb;
        ky = warp_sum(ky) / nb;
        for (int i = lane; i < nb; i += 32) {
            dx[i] = (dx[i] - mx - p[i] * kx) / rms;
            dy[i] = (dy[i] - my - p[i] * ky) / rms;
        }
    }
    int iz = (int)floorf(z);
    iz = max(0, min(planes - 2, iz));
    const double fz = (double)z - iz;
    CostTerms t = {};
    for (int i = lane; i < nb; i += 32) {
        const double l0 = L[iz * nb + i], l1 = L[(iz + 1) * nb + i];
        const double w = P.z_weights ? (double)P.z_weights[i] : 1.0, w2 = w * w;
        const double e = p[i] - (l0 + (l1 - l0) * fz);
        const double J[3] = {dx[i], dy[i], -(l1 - l0)};
        t.cost += w2 * e * e;
        for (int a = 0; a < 3; a++) t.Jr[a] += w2 * J[a] * e;
        t.A[0] += w2 * J[0] * J[0];
        t.A[1] += w2 * J[0] * J[1];
        t.A[2] += w2 * J[0] * J[2];
        t.A[3] += w2 * J[1] * J[1];
        t.A[4] += w2 * J[1] * J[2];
        t.A[5] += w2 * J[2] * J[2];
    }
    t.cost = warp_sum(t.cost);
    for (int a = 0; a < 3; a++) t.Jr[a] = warp_sum(t.Jr[a]);
    for (int a = 0; a < 6; a++) t.A[a] = warp_sum(t.A[a]);
    for (int a = 0; a < 3; a++) t.g[a] = 2.0 * t.Jr[a];
    return t;
}

// Image mean of the ROI in shared memory (block-wide; every thread gets it).
__device__ double roi_mean(const float *img, int n, double *red)
{
    double v[1] = {0.0};
    for (int i = threadIdx.x; i < n; i += blockDim.x) v[0] += img[i];
    BlockGroup{red}.sum<1>(v);
    return v[0] / n;
}

// Adjoint: one block per ROI. xyz[3*roi], bead[roi] (or 0), out cost[roi], grad[3*roi], and
// glut[bead][plane][bin] += dcost/dL (atomically: ROIs of a bead share its LUT rows).
__global__ void __launch_bounds__(kAdjThreads) zcost_grad_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                                 int pitch, int64_t roi_stride, int count,
                                                                 const float *__restrict__ xyz,
                                                                 const int *__restrict__ beads, float *__restrict__ cost,
                                                                 float *__restrict__ grad, float *__restrict__ glut)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int roi = blockIdx.x;
    if (roi >= count) return;
    const AdjSmem s = adj_view(smem, P);
    const int bead = beads ? beads[roi] : 0;
    const bool ok = bead >= 0 && bead < P.lut_count && P.lut_planes >= 2;
    BlockGroup g{s.red};
    load_roi(g, s.img, pixels + (int64_t)roi * roi_stride, pitch, P, ok ? bead : 0);
    __syncthreads();
    const double mean = roi_mean(s.img, P.width * P.height, s.red);
    const float x = xyz[3 * roi], y = xyz[3 * roi + 1], z = xyz[3 * roi + 2];
    profile_grad(s.img, P, x, y, (float)mean, s.p, s.dx, s.dy);
    if (threadIdx.x >= 32) return;
    if (!ok) {
        if (threadIdx.x == 0) {
            cost[roi] = nanf("");
            grad[3 * roi] = grad[3 * roi + 1] = grad[3 * roi + 2] = nanf("");
        }
        return;
    }
    const int nb = P.z_nbins, planes = P.lut_planes;
    const float *L = P.lut + (size_t)bead * planes * nb;
    const CostTerms t = cost_terms(P, s.p, s.dx, s.dy, L, z);
    if (threadIdx.x == 0) {
        cost[roi] = (float)t.cost;
        grad[3 * roi] = (float)t.g[0];
        grad[3 * roi + 1] = (float)t.g[1];
        grad[3 * roi + 2] = (float)t.g[2];
    }
    if (glut) {
        int iz = (int)floorf(z);
        iz = max(0, min(planes - 2, iz));
        const double fz = (double)z - iz;
        float *G = glut + (size_t)bead * planes * nb;
        for (int i = threadIdx.x; i < nb; i += 32) {
            const double l0 = L[iz * nb + i], l1 = L[(iz + 1) * nb + i];
            const double w = P.z_weights ? (double)P.z_weights[i] : 1.0;
            const double de = 2.0 * w * w * (s.p[i] - (l0 + (l1 - l0) * fz));
            atomicAdd(&G[iz * nb + i], (float)(-de * (1.0 - fz)));
            atomicAdd(&G[(iz + 1) * nb + i], (float)(-de * fz));
        }
    }
}

// 3x3 solve A d = rhs by Cramer's rule (A symmetric, given as xx, xy, xz, yy, yz, zz).
__device__ bool solve3(const double A6[6], const double rhs[3], double d[3])
{
    const double a[3][3] = {{A6[0], A6[1], A6[2]}, {A6[1], A6[3], A6[4]}, {A6[2], A6[4], A6[5]}};
    const double det = a[0][0] * (a[1][1] * a[2][2] - a[1][2] * a[2][1]) - a[0][1] * (a[1][0] * a[2][2] - a[1][2] * a[2][0]) +
                       a[0][2] * (a[1][0] * a[2][1] - a[1][1] * a[2][0]);
    if (det == 0.0) return false;
    for (int c = 0; c < 3; c++) {
        double M[3][3];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++) M[i][j] = (j == c) ? rhs[i] : a[i][j];
        d[c] = (M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0])) /
               det;
    }
    return true;
}

// Joint Gauss-Newton refinement of a localized ROI (LT_B200_JointRefine), one block per ROI, in
// place on results[roi].pos. Minimises cost(x, y, z) + k ((x-x0)^2 + (y-y0)^2) from the located
// (x0, y0, z0), with k = 100 x the cost's z-curvature at the starting plane: a radial profile is
// insensitive to first order to its centre (the x-derivative of a radially symmetric image
// averages to zero over a circle), so the prior keeps QI's x, y precision while z follows the
// LUT interpolation. Per step: normal equations with the prior and a Levenberg term of
// 1e-9 x trace, Cramer's rule, and the step halved up to 4 times until the objective drops (the
// refinement stops when none does); z is clamped to [0, planes-1]. The fallback value of sparse
// bins is the ROI's image mean, as in the Z fit.
__global__ void __launch_bounds__(kAdjThreads) joint_refine_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                                   int pitch, int64_t roi_stride,
                                                                   const int64_t *__restrict__ roi_offsets,
                                                                   const LocalizationJob *__restrict__ jobs, int count,
                                                                   LocalizationResult *__restrict__ results)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int roi = blockIdx.x;
    if (roi >= count) return;
    const AdjSmem s = adj_view(smem, P);
    const int bead = jobs ? jobs[roi].zlutIndex : 0;
    if (bead < 0 || bead >= P.lut_count || P.lut_planes < 2) return;  // no LUT for this ROI: no Z fit to refine
    const int64_t off = roi_offsets ? roi_offsets[roi] : (int64_t)roi * roi_stride;
    BlockGroup g{s.red};
    load_roi(g, s.img, pixels + off, pitch, P, bead);
    __syncthreads();
    LocalizationResult *res = results + roi;
    const float mean = res->imageMean;
    const float x0 = res->pos.x, y0 = res->pos.y;
    float x = x0, y = y0, z = res->pos.z;
    const int nb = P.z_nbins, planes = P.lut_planes;
    const float *L = P.lut + (size_t)bead * planes * nb;
    double k = 0.0, cur = 0.0;
    for (int step = 0; step < kRefineSteps; step++) {
        profile_grad(s.img, P, x, y, mean, s.p, s.dx, s.dy);
        if (threadIdx.x < 32) {
            const CostTerms t = cost_terms(P, s.p, s.dx, s.dy, L, z);
            if (threadIdx.x == 0) {
                if (step == 0) k = kPriorScale * t.A[5];
                cur = t.cost + k * ((double)(x - x0) * (x - x0) + (double)(y - y0) * (y - y0));
                double A6[6] = {t.A[0] + k, t.A[1], t.A[2], t.A[3] + k, t.A[4], t.A[5]};
                const double tr = A6[0] + A6[3] + A6[5];
                A6[0] += 1e-9 * tr + 1e-30;
                A6[3] += 1e-9 * tr + 1e-30;
                A6[5] += 1e-9 * tr + 1e-30;
                const double rhs[3] = {-(t.Jr[0] + k * (x - x0)), -(t.Jr[1] + k * (y - y0)), -t.Jr[2]};
                double d[3];
                const bool solved = solve3(A6, rhs, d);
                s.misc[0] = solved ? 1.0 : 0.0;
                s.misc[1] = d[0];
                s.misc[2] = d[1];
                s.misc[3] = d[2];
                s.misc[4] = cur;
                s.misc[5] = k;
            }
        }
        __syncthreads();
        if (s.misc[0] == 0.0) break;
        const double d0 = s.misc[1], d1 = s.misc[2], d2 = s.misc[3];
        cur = s.misc[4];
        k = s.misc[5];
        bool taken = false;
        for (int hv = 0; hv < 5 && !taken; hv++) {
            const double tstep = ldexp(1.0, -hv);
            const float nx = (float)(x + tstep * d0), ny = (float)(y + tstep * d1);
            const float nz = fminf(fmaxf((float)(z + tstep * d2), 0.0f), (float)(planes - 1));
            profile_grad(s.img, P, nx, ny, mean, s.p, s.dx, s.dy);
            if (threadIdx.x < 32) {
                const CostTerms t = cost_terms(P, s.p, s.dx, s.dy, L, nz);
                if (threadIdx.x == 0)
                    s.misc[6] = t.cost + k * ((double)(nx - x0) * (nx - x0) + (double)(ny - y0) * (ny - y0));
            }
            __syncthreads();
            if (s.misc[6] < cur) {
                x = nx;
                y = ny;
                z = nz;
                cur = s.misc[6];
                taken = true;
            }
            __syncthreads();
        }
        if (!taken) break;
    }
    if (threadIdx.x == 0) {
        res->pos.x = x;
        res->pos.y = y;
        res->pos.z = z;
    }
}

// Gaussian-MLE adjoint: Poisson NLL = sum mu - I ln mu of the 5-parameter integrated-Gaussian
// model (the model gauss5_mle fits, erff per column/row, FP32 per pixel, FP64 sums) and its
// gradient sum (1 - I/mu) dmu/dp for p = (x, y, I0, bg, sigma) = params[5 roi ..]. One block per ROI.
__global__ void __launch_bounds__(kAdjThreads) gauss_nll_grad_kernel(TrackParams P, const uint8_t *__restrict__ pixels,
                                                                     int pitch, int64_t roi_stride, int count,
                                                                     const float *__restrict__ params,
                                                                     float *__restrict__ nll, float *__restrict__ grad)
{
    extern __shared__ __align__(16) uint8_t smem[];
    const int roi = blockIdx.x;
    if (roi >= count) return;
    const int W = P.width, H = P.height;
    float *img = reinterpret_cast<float *>(smem);
    float *col = img + ((W * H + 3) & ~3);
    float *row = col + 3 * W;
    double *red = reinterpret_cast<double *>(smem + (((size_t)((W * H + 3) & ~3) + 3 * (W + H)) * 4 + 15) / 16 * 16);
    BlockGroup g{red};
    load_roi(g, img, pixels + (int64_t)roi * roi_stride, pitch, P, 0);
    float p[5];
#pragma unroll
    for (int k = 0; k < 5; k++) p[k] = params[5 * roi + k];
    const float s = p[4];
    const float k1 = 1.0f / (sqrtf(2.0f) * s);
    const float k2 = 1.0f / (sqrtf(2 * 3.14159265359f) * s);
    for (int c = threadIdx.x; c < W + H; c += blockDim.x) {
        const bool is_col = c < W;
        const int cc = is_col ? c : c - W;
        const float pc = is_col ? p[0] : p[1];
        const float a0 = (cc - pc + .5f) * k1, a1 = (cc - pc - .5f) * k1;
        const float e0 = expf(-a0 * a0), e1 = expf(-a1 * a1);
        float *t = is_col ? col + 3 * cc : row + 3 * cc;
        t[0] = 0.5f * (erff(a0) - erff(a1));
        t[1] = (e1 - e0) * k2;
        t[2] = ((cc - pc - .5f) * e1 - (cc - pc + .5f) * e0) * k2 / s;
    }
    __syncthreads();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    for (int i = threadIdx.x; i < W * H; i += blockDim.x) {
        const int y = i / W, x = i - y * W;
        const float DX = col[3 * x], dX = col[3 * x + 1], sX = col[3 * x + 2];
        const float DY = row[3 * y], dY = row[3 * y + 1], sY = row[3 * y + 2];
        const float mu = p[3] + p[2] * DX * DY;
        const float I = img[i];
        const float f = 1.0f - I / mu;
        acc[0] += (double)(mu - I * logf(mu));
        acc[1] += (double)(f * p[2] * dX * DY);
        acc[2] += (double)(f * p[2] * DX * dY);
        acc[3] += (double)(f * DX * DY);
        acc[4] += (double)f;
        acc[5] += (double)(f * p[2] * (sX * DY + DX * sY));
    }
    g.sum(acc);
    if (threadIdx.x == 0) {
        nll[roi] = (float)acc[0];
#pragma unroll
        for (int k = 0; k < 5; k++) grad[5 * roi + k] = (float)acc[1 + k];
    }
}

}  // namespace

cudaError_t launch_zcost_grad(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride, int count,
                              const float *xyz, const int *beads, float *cost, float *grad, float *glut,
                              cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int smem = adj_smem_bytes(P);
    cudaError_t e = cudaFuncSetAttribute(zcost_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    zcost_grad_kernel<<<count, kAdjThreads, smem, stream>>>(P, pixels, pitch, roi_stride, count, xyz, beads, cost, grad,
                                                            glut);
    return cudaGetLastError();
}

cudaError_t launch_gauss_nll_grad(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride, int count,
                                  const float *params, float *nll, float *grad, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int W = P.width, H = P.height;
    const int smem = (int)((((size_t)((W * H + 3) & ~3) + 3 * (W + H)) * 4 + 15) / 16 * 16) + 6 * 32 * 8;
    cudaError_t e = cudaFuncSetAttribute(gauss_nll_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    gauss_nll_grad_kernel<<<count, kAdjThreads, smem, stream>>>(P, pixels, pitch, roi_stride, count, params, nll, grad);
    return cudaGetLastError();
}

cudaError_t launch_joint_refine(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride,
                                const int64_t *roi_offsets, const LocalizationJob *jobs, int count,
                                LocalizationResult *results, cudaStream_t stream)
{
    if (count <= 0) return cudaSuccess;
    const int smem = adj_smem_bytes(P);
    cudaError_t e = cudaFuncSetAttribute(joint_refine_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    joint_refine_kernel<<<count, kAdjThreads, smem, stream>>>(P, pixels, pitch, roi_stride, roi_offsets, jobs, count,
                                                              results);
    return cudaGetLastError();
}

}  // namespace qtrk
