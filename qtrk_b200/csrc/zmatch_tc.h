// Tensor-core (tcgen05, BF16 or TF32 in / FP32 accumulate) Z-LUT match; see zmatch_tc.cu.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "qtrk_c_api.h"

namespace qtrk {

struct ZMatchParams {
    int nb;          // radial bins
    int nbp;         // bins padded to a multiple of 16 (the MMA K step)
    int planes;      // LUT planes
    int planes_pad;  // planes padded to a multiple of 16
    int lut_count;   // beads in the LUT
    const __nv_bfloat16 *prof_bf16;  // [rois][hi, lo][nbp]   w * normalised profile, split in two BF16
    const float *prof_f32;           // [rois][nb]    normalised profile
    const __nv_bfloat16 *lut_bf16;   // [lut_count][hi, lo][planes_pad][nbp]  w * LUT, split in two BF16
    const float *lut_norm;           // [lut_count][planes_pad]       |w L_k|^2
    const float *lut;                // [lut_count][planes][nb]       FP32 LUT
    const float *weights;            // [nb] radial weights or nullptr
    const int *perm;                 // ROI order grouped by bead, or nullptr (identity)
    const int4 *tiles;               // per CTA: {first index into perm, rows (<= 128), bead, 0}, or
                                     // nullptr: CTA i takes ROIs 128 i .. of `count`, all of bead
                                     // `uniform_bead`
    int count, uniform_bead;
    LocalizationResult *results;     // z (word 8 of each 13-word record) is written
    const float *zbias;              // Z-LUT bias table [zbias_count][zbias_w] or nullptr
    int zbias_w, zbias_count;
    unsigned *error_flag;            // |= 1 if an MMA completion wait gave up, |= 2 if the abandoned MMAs
                                     // had not committed when their columns were released
    int tf32;                        // 1: TF32 operands (w p and w L in FP32), one MMA per K step
};

int zmatch_padded_bins(int nb);
int zmatch_padded_planes(int planes);
bool zmatch_supported(int nb);
int zmatch_smem_bytes(int nbp);
cudaError_t zmatch_prepare_kernel_attrs();
cudaError_t zmatch_prepare_lut(const float *lut, const float *weights, int count, int planes, int nb,
                               __nv_bfloat16 *lut_bf16, float *lut_norm, cudaStream_t stream);
cudaError_t launch_zmatch_tc(const ZMatchParams &Q, int ntiles, cudaStream_t stream);

}  // namespace qtrk
