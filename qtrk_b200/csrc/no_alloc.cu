// QTrkB200LocalizeDeviceNoAlloc: the device-resident localization entry point for callers that
// cannot allocate device memory while they run.
//
// Who needs it: acquisition code that runs on a real-time thread (a camera callback, a LabVIEW
// timed loop) must keep every call's latency bounded, and cudaMalloc/cudaFree take the
// driver's allocation lock and can synchronize the whole device; some host processes also fix
// their device-memory budget at start-up and are not allowed to grow it later. The regular
// QTrkB200LocalizeDevice grows a per-instance scratch buffer for the tensor-core Z match on
// first use (cudaMalloc inside the call); this variant never does.
//
// How: the intermediate radial profiles of the tensor-core Z match (an FP32 copy and a split
// BF16 copy per ROI) live in one fixed array below. A __device__ array is created in every
// GPU's memory when the library is loaded there and stays until the process exits, so its
// size is kept modest: kNoAllocScratchBytes = 16 MiB, i.e. 32,768 ROIs of 64 radial bins per
// call. In host code the array's name is a host-side stand-in, not a device address, so the
// device address is looked up once per device with cudaGetSymbolAddress (with that device
// current) and passed to the kernels like any other pointer. That lookup happens in the first
// call on each device; make that first call before any stream capture.
//
// Every call uses the same array, and each call overwrites all of the profile entries it
// reads, so nothing in it needs clearing between calls. Calls whose GPU work overlaps
// (different streams, or different instances on the same GPU) race on the array and must be
// serialized by the caller.
#include <cstdint>
#include <mutex>
#include <string>

#include <cuda_runtime.h>

#include "qtrk_c_api.h"
#include "tracker.h"

namespace {

constexpr size_t kNoAllocScratchBytes = 16u << 20;  // 16 MiB per GPU
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_scratch_mu;
void *g_scratch_ptr[kMaxDevices] = {nullptr};

// Device address of g_noalloc_scratch on `device` (current device when called); looked up once.
cudaError_t scratch_address(int device, void **out)
{
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[device]) {
        void *ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = ptr;
    }
    *out = g_scratch_ptr[device];
    return cudaSuccess;
}

}  // namespace

extern "C" QTRK_API int QTRK_CALLCONV QTrkB200LocalizeDeviceNoAlloc(QueuedTracker *q, const void *d_pixels, int pitch,
                                                                    int64_t roi_stride_bytes,
                                                                    QTRK_PixelDataType_t pdt, int count,
                                                                    const LocalizationJob *d_jobs,
                                                                    LocalizationResult *d_results, void *stream)
{
    if (!q) return -100;
    qtrk::Tracker *t = static_cast<qtrk::Tracker *>(q);
    try {
        int prev = -1;
        cudaGetDevice(&prev);
        if (prev != t->device()) cudaSetDevice(t->device());
        void *scratch = nullptr;
        const cudaError_t e = scratch_address(t->device(), &scratch);
        if (prev >= 0 && prev != t->device()) cudaSetDevice(prev);
        if (e != cudaSuccess) {
            t->Warn(std::string("QTrkB200LocalizeDeviceNoAlloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
            return -5;
        }
        return t->LocalizeDeviceNoAlloc(d_pixels, pitch, roi_stride_bytes, pdt, count, d_jobs, d_results,
                                        static_cast<cudaStream_t>(stream), scratch, kNoAllocScratchBytes);
    } catch (const std::exception &ex) {
        t->Warn(std::string("QTrkB200LocalizeDeviceNoAlloc: ") + ex.what());
    } catch (...) {
        t->Warn("QTrkB200LocalizeDeviceNoAlloc: unknown error");
    }
    return -100;
}
