// Host-side entry points of the CUDA kernels (implemented in localize.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "qtrk_c_api.h"
#include "track_params.h"

namespace qtrk {

// Fill the shared-memory layout fields of P from its sizes.
void plan_smem(TrackParams &P);
// Raise the dynamic shared-memory limit of the kernels once per device.
cudaError_t prepare_kernels(int device);
// True when the Gaussian-only warp-per-ROI kernel serves P.
bool use_gauss_warp(const TrackParams &P);

// Localize `count` ROIs: ROI i starts at pixels + (roi_offsets ? roi_offsets[i] : i*roi_stride).
// jobs may be null (job i = {frame=i}). One kernel launch.
cudaError_t launch_localize(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride,
                            const int64_t *roi_offsets, const LocalizationJob *jobs, int count,
                            LocalizationResult *results, cudaStream_t stream);

// LT_OnlyCOM on ROIs stored back to back (no per-bead calibration): the register-held streaming
// COM kernel (com.cu) serves them; launch_localize chooses it by itself.
bool use_com_kernel(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride,
                    const int64_t *roi_offsets);
cudaError_t launch_com(const TrackParams &P, const uint8_t *pixels, int64_t roi_stride, const LocalizationJob *jobs,
                       int count, LocalizationResult *results, cudaStream_t stream);

// The kernel node that launch_localize would launch for `count` ROIs addressed through
// roi_offsets (function, grid, block, shared memory); the caller sets kernelParams to the 8
// arguments of launch_localize's kernel (P, pixels, pitch, roi_stride, roi_offsets, jobs, count,
// results). For explicitly built graphs; never the COM kernel, which takes ROIs back to back.
void localize_node(const TrackParams &P, int count, cudaKernelNodeParams &kp);

// Bias-table images [first_image, first_image + n_images) of QueuedTracker::ComputeZBiasCorrection
// (bead = image / bias_planes, z = (image % bias_planes) / bias_planes * planes) rendered from
// the device LUT [beads][planes][nb] into images[n_images][h][w], with their jobs.
cudaError_t launch_lut_images(const float *lut, int nb, int planes, int first_image, int n_images, int bias_planes,
                              int w, int h, float minr, float maxr, int ovs, bool spline, float *images,
                              LocalizationJob *jobs, cudaStream_t stream);

// Radial-profile/LUT cost of `count` ROIs (ROI i at pixels + i*roi_stride) at xyz[3i..3i+2] against
// bead beads[i]'s LUT (bead 0 when beads is null): cost[i], grad[3i..] = d cost / d(x, y, z), and
// glut [beads][planes][bins] += d cost / d LUT (glut may be null). One kernel launch.
cudaError_t launch_zcost_grad(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride, int count,
                              const float *xyz, const int *beads, float *cost, float *grad, float *glut,
                              cudaStream_t stream);

// Poisson NLL of the 5-parameter integrated-Gaussian model at params[5i..5i+4] = (x, y, I0, bg,
// sigma) and its gradient, for `count` ROIs at pixels + i*roi_stride. One kernel launch.
cudaError_t launch_gauss_nll_grad(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride, int count,
                                  const float *params, float *nll, float *grad, cudaStream_t stream);

// Joint Gauss-Newton (x, y, z) refinement of localized ROIs, in place on results (same ROI
// addressing as launch_localize). One kernel launch.
cudaError_t launch_joint_refine(const TrackParams &P, const uint8_t *pixels, int pitch, int64_t roi_stride,
                                const int64_t *roi_offsets, const LocalizationJob *jobs, int count,
                                LocalizationResult *results, cudaStream_t stream);

// One BuildLUT plane: nbeads ROIs stacked at pitch*H; adds each profile to lut[bead][plane].
cudaError_t launch_build_lut(const TrackParams &P, const uint8_t *pixels, int pitch, int nbeads, int plane,
                             const float2 *known_pos, bool normalize, float *lut, cudaStream_t stream);

// NormalizeRadialProfile on `rows` rows of nb floats.
cudaError_t launch_finalize_lut(float *lut, int rows, int nb, cudaStream_t stream);

// The transposed copy of a Z-LUT that the plain match reads: [count][nb][pitch] from [count][planes][nb].
cudaError_t launch_transpose_lut(const float *lut, int count, int planes, int nb, int pitch, float *lut_t,
                                 cudaStream_t stream);
inline int lut_t_pitch(int planes) { return (planes + 31) & ~31; }

// Radial profile of one float image (P.width x P.height) around (cx, cy).
cudaError_t launch_profile(const TrackParams &P, const float *img, float cx, float cy, float mean, bool normalize,
                           float *out, cudaStream_t stream);

}  // namespace qtrk
