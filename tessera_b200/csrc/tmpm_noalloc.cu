// tmpm_noalloc.cu -- block-order binning for callers that must not allocate.
//
// Some callers cannot let a library call cudaMalloc: a render or physics loop
// that runs under a frame-time budget (an allocation can synchronize the
// device and stall the frame), a host application that hands out all device
// memory through its own pool, or code that records work into a CUDA graph.
// tmpm_sort_by_block_noalloc gives them the binning step of the substep (the
// f32 base cell of each particle, the Morton key of its 4^3 grid block and
// the stable sort order by that key) using only the buffers they pass in plus
// a fixed scratch area that is part of the library image itself.

#include <cmath>
#include <cstdio>
#include <mutex>
#include <string>

#include <cuda.h>

#include "../../include/tmpm.h"
#include "tmpm_internal.h"

namespace {

constexpr size_t kNoAllocMaxParticles = size_t(1) << 18;  // 262,144 particles per call
constexpr size_t kNoAllocTiles = (kNoAllocMaxParticles + 4095) / 4096;
// keys[2][max] | vals[2][max] | hist[256][tiles] | totals[256], 32-bit words:
// 4 * 2^18 + 256 * 64 + 256 = 1,065,216 words = 4,260,864 bytes
constexpr size_t kNoAllocWords = 4 * kNoAllocMaxParticles + 256 * kNoAllocTiles + 256;

// Device-resident scratch shared by every call on a device.  Host code must
// never hand this symbol itself to a kernel: on the host it is only a
// stand-in, and its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_noalloc_scratch[kNoAllocWords];

// The scratch address is a property of the CUDA context that loaded this
// module, not of the device number: after cudaDeviceReset (or in another
// context on the same device) the module is loaded again and the array can
// move.  The cache therefore remembers the context it was taken in, and a
// call outside a stream capture looks the address up afresh every time; only
// a call made during a capture, where no set-up may run, takes it from the
// cache, and only when the cached context is the current one.
constexpr int kMaxDevices = 64;
struct ScratchSlot {
    CUcontext ctx = nullptr;
    uint32_t *ptr = nullptr;
};
std::mutex g_setup_mutex;
ScratchSlot g_scratch[kMaxDevices];

typedef CUresult (*CtxGetCurrentFn)(CUcontext *);

TmpmStatus noalloc_fail(TmpmStatus st, const std::string &msg) {
    tmpm::set_last_error(msg);  // readable through tmpm_last_error()
    return st;
}

// The current context, through the driver entry point the runtime exposes
// (no link against libcuda).  Null when it cannot be had.
CUcontext current_context() {
    static CtxGetCurrentFn fn = [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(f);
    }();
    CUcontext ctx = nullptr;
    if (!fn || fn(&ctx) != CUDA_SUCCESS) return nullptr;
    return ctx;
}

}  // namespace

extern "C" TmpmStatus tmpm_sort_by_block_noalloc(const float *positions, size_t count, size_t stride,
                                                 double cell_width, uint32_t *order_out, uint32_t *keys_out,
                                                 void *stream) {
    if (count > kNoAllocMaxParticles)
        return noalloc_fail(TMPM_ERR_CAPACITY, "tmpm_sort_by_block_noalloc: count " + std::to_string(count) +
                                                   " exceeds the fixed scratch limit of " +
                                                   std::to_string(kNoAllocMaxParticles) + " particles");
    if (count == 0) return TMPM_OK;
    if (!positions || !order_out || stride < count)
        return noalloc_fail(TMPM_ERR_INVALID_INPUT, "tmpm_sort_by_block_noalloc: null buffer or stride < count");
    const float h32 = static_cast<float>(cell_width);
    if (!std::isfinite(cell_width) || !std::isfinite(h32) || h32 <= 0.0f || !std::isfinite(1.0f / h32))
        return noalloc_fail(TMPM_ERR_INVALID_INPUT, "tmpm_sort_by_block_noalloc: cell width not a positive f32");

    // An error an earlier, unrelated CUDA call left unreported would
    // otherwise surface as this call's launch failure: it is cleared here.
    cudaGetLastError();
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return noalloc_fail(TMPM_ERR_DEVICE, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(TMPM_ERR_DEVICE, "device ordinal out of range");
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &capture);
    if (e != cudaSuccess)
        return noalloc_fail(TMPM_ERR_DEVICE, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    // Set-up, with the device current: the scratch symbol's device address in
    // this context.  Outside a capture it runs on every call (a host-side
    // lookup); during a capture the address comes from the last call made
    // outside one in the same context, so the first call on a device, and the
    // first after a cudaDeviceReset, must come before any stream capture.
    const CUcontext ctx = current_context();
    uint32_t *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mutex);
        ScratchSlot &slot = g_scratch[dev];
        if (capture == cudaStreamCaptureStatusNone) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess || !p)
                return noalloc_fail(TMPM_ERR_DEVICE,
                                    std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
            slot.ctx = ctx;
            slot.ptr = static_cast<uint32_t *>(p);
        } else if (!slot.ptr || !ctx || slot.ctx != ctx) {
            return noalloc_fail(TMPM_ERR_DEVICE,
                                "tmpm_sort_by_block_noalloc: called during a stream capture before any call outside "
                                "one in this context (the scratch address is looked up outside captures)");
        }
        base = slot.ptr;
    }
    tmpm::SortBuffers sb{};
    sb.keys[0] = base;
    sb.keys[1] = base + kNoAllocMaxParticles;
    sb.vals[0] = base + 2 * kNoAllocMaxParticles;
    sb.vals[1] = base + 3 * kNoAllocMaxParticles;
    sb.hist = base + 4 * kNoAllocMaxParticles;
    sb.totals = sb.hist + 256 * kNoAllocTiles;
    sb.cap = kNoAllocMaxParticles;
    // Every scratch word this call reads is written earlier in the same call
    // (keys and values by the binning kernel, histograms and totals by each
    // radix pass), so nothing has to start at zero.
    const int n = static_cast<int>(count);
    tmpm::launch_bin_keys_values(positions, stride, n, 1.0f / h32, sb.keys[0], sb.vals[0], s);
    const int r = tmpm::radix_sort_pairs(sb, n, tmpm::kSortBitsScene, s);
    e = cudaGetLastError();  // launch errors of the binning and radix kernels
    if (e != cudaSuccess) return noalloc_fail(TMPM_ERR_DEVICE, std::string("launch: ") + cudaGetErrorString(e));
    e = cudaMemcpyAsync(order_out, sb.vals[r], sizeof(uint32_t) * count, cudaMemcpyDeviceToDevice, s);
    if (e != cudaSuccess)
        return noalloc_fail(TMPM_ERR_DEVICE, std::string("copy of the order: ") + cudaGetErrorString(e));
    if (keys_out) {
        e = cudaMemcpyAsync(keys_out, sb.keys[r], sizeof(uint32_t) * count, cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess)
            return noalloc_fail(TMPM_ERR_DEVICE, std::string("copy of the keys: ") + cudaGetErrorString(e));
    }
    return TMPM_OK;
}
