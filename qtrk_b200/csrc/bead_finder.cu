// QTrkFindBeads / QTrkFreeROIPositions: bead finding by template matching
// (cputrack/BeadFinder.cpp:170-222, called as in cputrack/qtrk_c_api.cpp:33-58).
//
// The reference multiplies the 2D FFT of the mean-free frame (zero-padded to powers of two) by
// the FFT of the mean-free sample ROI placed at offset -roi and transforms back: a circular
// convolution over the padded W2 x H2 map,
//   conv(py,px) = sum_{a,b<roi} t(a,b) c((py+roi-a) mod H2, (px+roi-b) mod W2).
// Here the GPU evaluates that sum directly (FP32 products, FP32 partial sums over 16-row chunks
// of the sample, FP64 across chunks): a frame of a few megapixels with a 100 px sample takes a
// few milliseconds and the result carries no FFT rounding. The map's maximum, the thresholded
// raster scan with its neighbourhood search (each search zeroes the disc it visited, so its
// order matters) and the recentering filter run on the host exactly as the reference orders
// them; they touch only the pixels above the threshold and the sample-sized boxes around the
// candidates.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <list>
#include <stdexcept>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "qtrk_c_api.h"

namespace qtrk {
void set_last_error_msg(const std::string &m);
}

namespace {

constexpr int kTileX = 32;   // outputs per block along x (one per thread column)
constexpr int kTileY = 32;   // outputs per block along y (4 per thread, 8 thread rows)
constexpr int kRowsPerThread = 4;
constexpr int kChunk = 16;   // sample rows per shared-memory pass

// One block: a 32 x 32 tile of the map. Thread (tx, ty) owns outputs (Y0 + 4ty + j, X0 + tx).
// For each chunk of 16 sample rows the block stages the chunk (zero rows past the sample) and
// the 47 x (31 + roi) frame patch those rows reach; each thread then walks the sample columns
// keeping the 19 patch values of its column in registers (19 loads feed 64 FMAs).
__global__ void __launch_bounds__(256) bead_conv_kernel(const float *__restrict__ frame, int w, int h, float mean,
                                                        const float *__restrict__ tmpl, int roi, int W2, int H2,
                                                        float *__restrict__ out)
{
    extern __shared__ float smem[];
    const int pw = kTileX - 1 + roi;  // patch width
    float *ts = smem;                 // [kChunk][roi]
    float *ps = smem + kChunk * roi;  // [kTileY + kChunk - 1][pw]
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int X0 = blockIdx.x * kTileX, Y0 = blockIdx.y * kTileY;
    double acc[kRowsPerThread] = {0, 0, 0, 0};
    for (int a0 = 0; a0 < roi; a0 += kChunk) {
        __syncthreads();
        for (int i = threadIdx.x; i < kChunk * roi; i += blockDim.x) {
            const int a = a0 + i / roi;
            ts[i] = a < roi ? tmpl[a * roi + i % roi] : 0.0f;
        }
        const int prow = kTileY + kChunk - 1;
        const int base_row = Y0 + roi - (a0 + kChunk - 1);  // global row of patch row 0 (may be < 0)
        for (int i = threadIdx.x; i < prow * pw; i += blockDim.x) {
            const int r = i / pw, c = i - r * pw;
            const int gy = ((base_row + r) % H2 + H2) % H2;
            const int gx = (X0 + 1 + c) % W2;
            ps[i] = (gy < h && gx < w) ? frame[(size_t)gy * w + gx] - mean : 0.0f;
        }
        __syncthreads();
        float part[kRowsPerThread] = {0, 0, 0, 0};
        for (int b = 0; b < roi; b++) {
            const int col = tx + roi - 1 - b;
            float v[kChunk + kRowsPerThread - 1];
#pragma unroll
            for (int i = 0; i < kChunk + kRowsPerThread - 1; i++) v[i] = ps[(kRowsPerThread * ty + i) * pw + col];
#pragma unroll
            for (int k = 0; k < kChunk; k++) {
                const float t = ts[k * roi + b];
#pragma unroll
                for (int j = 0; j < kRowsPerThread; j++) part[j] = fmaf(t, v[j + kChunk - 1 - k], part[j]);
            }
        }
#pragma unroll
        for (int j = 0; j < kRowsPerThread; j++) acc[j] += (double)part[j];
    }
    const int px = X0 + tx;
#pragma unroll
    for (int j = 0; j < kRowsPerThread; j++) {
        const int py = Y0 + kRowsPerThread * ty + j;
        if (px < W2 && py < H2) out[(size_t)py * W2 + px] = (float)acc[j];
    }
}

int next_pow2(int x)  // BeadFinder.cpp:11-17
{
    int y = 1;
    while (y < x) y *= 2;
    return y;
}

struct Pos {
    int x, y;
};

void ck(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

// The convolution map on the current GPU.
std::vector<float> convolve_on_gpu(const float *img, int w, int h, float mean, const std::vector<float> &t, int roi,
                                   int W2, int H2)
{
    float *d_img = nullptr, *d_t = nullptr, *d_out = nullptr;
    std::vector<float> map((size_t)W2 * H2);
    cudaStream_t s = nullptr;
    try {
        ck(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
        ck(cudaMalloc(&d_img, sizeof(float) * (size_t)w * h), "cudaMalloc");
        ck(cudaMalloc(&d_t, sizeof(float) * t.size()), "cudaMalloc");
        ck(cudaMalloc(&d_out, sizeof(float) * map.size()), "cudaMalloc");
        ck(cudaMemcpyAsync(d_img, img, sizeof(float) * (size_t)w * h, cudaMemcpyHostToDevice, s), "H2D frame");
        ck(cudaMemcpyAsync(d_t, t.data(), sizeof(float) * t.size(), cudaMemcpyHostToDevice, s), "H2D sample");
        const size_t smem = sizeof(float) * ((size_t)kChunk * roi + (size_t)(kTileY + kChunk - 1) * (kTileX - 1 + roi));
        ck(cudaFuncSetAttribute(bead_conv_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
           "cudaFuncSetAttribute");
        dim3 grid((W2 + kTileX - 1) / kTileX, (H2 + kTileY - 1) / kTileY);
        bead_conv_kernel<<<grid, 256, smem, s>>>(d_img, w, h, mean, d_t, roi, W2, H2, d_out);
        ck(cudaGetLastError(), "bead convolution launch");
        ck(cudaMemcpyAsync(map.data(), d_out, sizeof(float) * map.size(), cudaMemcpyDeviceToHost, s), "D2H map");
        ck(cudaStreamSynchronize(s), "bead convolution");
    } catch (...) {
        cudaFree(d_img);
        cudaFree(d_t);
        cudaFree(d_out);
        if (s) cudaStreamDestroy(s);
        throw;
    }
    cudaFree(d_img);
    cudaFree(d_t);
    cudaFree(d_out);
    cudaStreamDestroy(s);
    return map;
}

// SearchArea, BeadFinder.cpp:79-105: the first strict maximum of the disc (radius dist) around
// (px, py), clipped to the padded map; the visited values are zeroed.
Pos search_area(std::vector<float> &m, int W2, int H2, int px, int py, int dist)
{
    Pos best{px, py};
    float bv = m[(size_t)py * W2 + px];
    const int y0 = std::max(0, py - dist), x0 = std::max(0, px - dist);
    const int x1 = std::min(W2 - 1, px + dist), y1 = std::min(H2 - 1, py + dist);
    for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++) {
            const int dx = x - px, dy = y - py;
            if (dx * dx + dy * dy > dist * dist) continue;
            float &v = m[(size_t)y * W2 + x];
            if (v > bv) {
                best = {x, y};
                bv = v;
            }
            v = 0.0f;
        }
    return best;
}

// RecenterAndFilter, BeadFinder.cpp:108-166: shift each candidate corner by the centroid of the
// squared deviations from its ROI mean (float sums; the shift truncates toward zero), drop
// candidates outside the frame, and drop both members of any pair closer than min_dist.
std::vector<Pos> recenter_and_filter(const float *img, int w, int h, const std::vector<Pos> &pts, int roi,
                                     float min_dist)
{
    std::list<Pos> keep;
    for (Pos bp : pts) {
        if (bp.x < 0 || bp.y < 0 || bp.x > w - 1 - roi || bp.y > h - 1 - roi) continue;
        float sum = 0.0f;
        for (int y = 0; y < roi; y++)
            for (int x = 0; x < roi; x++) sum += img[(size_t)(y + bp.y) * w + x + bp.x];
        const float mean = sum / (roi * roi);
        float sx = 0, sy = 0;
        sum = 0;
        for (int y = 0; y < roi; y++)
            for (int x = 0; x < roi; x++) {
                float v = img[(size_t)(y + bp.y) * w + x + bp.x] - mean;
                v = v * v;
                sum += v;
                sx += v * x;
                sy += v * y;
            }
        if (sum == 0.0f) continue;
        bp.x = (int)((float)bp.x + (sx / sum - roi / 2));
        bp.y = (int)((float)bp.y + (sy / sum - roi / 2));
        if (bp.x < 0 || bp.y < 0 || bp.x > w - 1 - roi || bp.y > h - 1 - roi) continue;
        bool accepted = true;
        for (auto c = keep.begin(); c != keep.end(); ++c) {
            const int dx = c->x - bp.x, dy = c->y - bp.y;
            if ((float)(dx * dx + dy * dy) < min_dist * min_dist) {
                keep.erase(c);
                accepted = false;
                break;
            }
        }
        if (accepted) keep.push_back(bp);
    }
    return std::vector<Pos>(keep.begin(), keep.end());
}

}  // namespace

extern "C" QTRK_API ROIPosition *QTRK_CALLCONV QTrkFindBeads(ImageData *imgData, int smpCornerPosX, int smpCornerPosY,
                                                             int roi, float imgRelDist, float acceptance, int *beadcount,
                                                             ImageData *sample)
{
    if (beadcount) *beadcount = 0;
    try {
        if (!imgData || !imgData->data || imgData->w <= 0 || imgData->h <= 0 || roi <= 0 || !beadcount)
            throw std::invalid_argument("invalid argument");
        const int w = imgData->w, h = imgData->h;
        if (smpCornerPosX < 0 || smpCornerPosY < 0 || smpCornerPosX + roi > w || smpCornerPosY + roi > h)
            throw std::invalid_argument("the sample ROI must lie inside the image");
        if (roi > 800) throw std::invalid_argument("roi above 800 pixels is not supported");
        const float *img = imgData->data;
        // the sample (TImageData::subimage) and the two means (TImageData::mean: float sums)
        std::vector<float> t((size_t)roi * roi);
        for (int y = 0; y < roi; y++)
            for (int x = 0; x < roi; x++) t[(size_t)y * roi + x] = img[(size_t)(smpCornerPosY + y) * w + smpCornerPosX + x];
        if (sample && sample->data && sample->w == roi && sample->h == roi) std::memcpy(sample->data, t.data(), sizeof(float) * t.size());
        float mean = 0.0f, smean = 0.0f;
        for (size_t i = 0; i < (size_t)w * h; i++) mean += img[i];
        mean /= (float)(w * h);
        for (float v : t) smean += v;
        smean /= (float)(roi * roi);
        for (float &v : t) v -= smean;

        const int W2 = next_pow2(w), H2 = next_pow2(h);
        std::vector<float> map = convolve_on_gpu(img, w, h, mean, t, roi, W2, H2);
        float maxv = 0.0f;
        for (float v : map) maxv = std::max(maxv, v);
        const float min_dist = 0.5f * imgRelDist * roi;  // BeadFinder::Config::MinPixelDistance
        const int dist = (int)min_dist;
        std::vector<Pos> pts;
        for (int y = 0; y < h; y++)
            for (int x = 0; x < w; x++)
                if (map[(size_t)y * W2 + x] > maxv * acceptance) pts.push_back(search_area(map, W2, H2, x, y, dist));
        const std::vector<Pos> beads = recenter_and_filter(img, w, h, pts, roi, min_dist);
        ROIPosition *out = new ROIPosition[beads.size() ? beads.size() : 1];
        for (size_t i = 0; i < beads.size(); i++) out[i] = ROIPosition{beads[i].x, beads[i].y};
        *beadcount = (int)beads.size();
        return out;
    } catch (const std::exception &e) {
        qtrk::set_last_error_msg(std::string("QTrkFindBeads: ") + e.what());
        return nullptr;
    }
}

extern "C" QTRK_API void QTRK_CALLCONV QTrkFreeROIPositions(ROIPosition *data) { delete[] data; }
