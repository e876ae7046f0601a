// noalloc.cu -- psb_sort_cells_noalloc: the stable (cell key, value) radix
// sort with its scratch in a fixed device array, for callers that cannot
// allocate device memory.
//
// Who cannot allocate: a host application that hands all of the GPU's
// memory to its own pool and forbids libraries from calling cudaMalloc (a
// plugin host with a fixed memory budget), and per-frame loops -- the
// reference's GUI calls update() once per animation frame -- that must not
// stall on cudaMalloc/cudaFree, which can synchronise the whole device. The
// regular entry points allocate their buffers in psb_create; this one
// allocates nothing, ever.
//
// The scratch: a file-scope static __device__ array sized for
// PSB_NOALLOC_MAX_N elements. Every GPU that loads the library holds it
// (about 2.1 MB) until the process exits. Host code cannot pass the array's
// name to a kernel (it is a host-side stand-in, not a device address), so
// the address is fetched with cudaGetSymbolAddress once per device, on the
// first call made with that device current.
//
// All calls share the one array and it keeps the last call's contents.
// Nothing in it needs clearing: every pass writes its histogram block by
// block before the scan reads it, and the ping-pong half is fully written
// before it is read. Calls that overlap on the GPU (different streams, or
// different host threads on the same device) race on the array and corrupt
// each other's results; the caller must serialise them.
#include <cuda_runtime.h>
#include <cstdio>
#include <mutex>

#include "psb.h"
#include "psb_internal.cuh"

namespace {

constexpr int kMaxN = PSB_NOALLOC_MAX_N;
constexpr int kMaxBlocks = (kMaxN + 2047) / 2048;                 // radix tiles of 2048 keys
constexpr size_t kScratchWords = 2 * (size_t)kMaxN + 256 * (size_t)kMaxBlocks + 256;

// keys ping-pong | values ping-pong | digit histogram (256 x tiles) | digit totals (256)
static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

constexpr int kMaxDevices = 64;
uint32_t* g_scratch_addr[kMaxDevices] = {};
std::mutex g_setup_mutex;

// Device address of the scratch on the current device, fetched once.
int scratch_for_current_device(uint32_t** out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: no usable current device (%s)\n", cudaGetErrorString(e));
        return PSB_ECUDA;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_sort_scratch);
        if (e != cudaSuccess || !p) {
            std::fprintf(stderr, "psb_sort_cells_noalloc: cudaGetSymbolAddress failed on device %d: %s\n", dev,
                         cudaGetErrorString(e));
            return PSB_ECUDA;
        }
        g_scratch_addr[dev] = (uint32_t*)p;
    }
    *out = g_scratch_addr[dev];
    return PSB_OK;
}

}  // namespace

extern "C" int psb_sort_cells_noalloc(const uint32_t* keys_in, const uint32_t* vals_in, uint32_t* keys_out,
                                      uint32_t* vals_out, int32_t n, int32_t key_bits, void* stream) {
    if (n < 0 || key_bits < 1 || key_bits > 32 || (n > 0 && (!keys_in || !vals_in || !keys_out || !vals_out))) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: bad arguments (n=%d, key_bits=%d)\n", n, key_bits);
        return PSB_EINVAL;
    }
    if (n > kMaxN) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: n=%d exceeds the static scratch capacity of %d elements\n", n,
                     kMaxN);
        return PSB_EINVAL;
    }
    if (n == 0) return PSB_OK;
    uint32_t* scratch = nullptr;
    const int rc = scratch_for_current_device(&scratch);
    if (rc != PSB_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* tmp_keys = scratch;
    uint32_t* tmp_vals = scratch + kMaxN;
    uint32_t* hist = scratch + 2 * (size_t)kMaxN;
    // The sort ping-pongs between its two buffers starting from the first:
    // copy the input into the caller's output, sort between output and
    // scratch, and copy back if the last pass ended in the scratch.
    cudaMemcpyAsync(keys_out, keys_in, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    cudaMemcpyAsync(vals_out, vals_in, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    uint32_t* keys[2] = {keys_out, tmp_keys};
    uint32_t* vals[2] = {vals_out, tmp_vals};
    const int res = psb::radix_sort(st, n, key_bits, keys, vals, hist, kMaxBlocks);
    if (res == 1) {
        cudaMemcpyAsync(keys_out, tmp_keys, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(vals_out, tmp_vals, sizeof(uint32_t) * n, cudaMemcpyDeviceToDevice, st);
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: %s\n", cudaGetErrorString(e));
        return PSB_ECUDA;
    }
    return PSB_OK;
}
