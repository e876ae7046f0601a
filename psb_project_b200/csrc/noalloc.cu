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
// every call looks the address up with cudaGetSymbolAddress on the current
// device. The lookup is a host-side table read once the module is loaded;
// not caching it keeps the address right after the host application resets
// the device and the runtime loads the module again.
//
// All calls share the one array and it keeps the last call's contents.
// Nothing in it needs clearing: every pass writes its histogram block by
// block before the scan reads it, and the ping-pong half is fully written
// before it is read. Calls that overlap on the GPU (different streams, or
// different host threads on the same device) race on the array and corrupt
// each other's results; the caller must serialise them.
//
// Sorting in place (keys_out == keys_in, vals_out == vals_in, or both) is
// supported; any other overlap of the four ranges is refused.
#include <cuda_runtime.h>
#include <cstdio>

#include "psb.h"
#include "psb_internal.cuh"

namespace {

constexpr int kMaxN = PSB_NOALLOC_MAX_N;
constexpr int kMaxBlocks = (kMaxN + 2047) / 2048;                 // radix tiles of 2048 keys
constexpr size_t kScratchWords = 2 * (size_t)kMaxN + 256 * (size_t)kMaxBlocks + 256;

// keys ping-pong | values ping-pong | digit histogram (256 x tiles) | digit totals (256)
static __device__ __align__(256) uint32_t g_sort_scratch[kScratchWords];

// Device address of the scratch on the current device.
int scratch_for_current_device(uint32_t** out) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_sort_scratch);
    if (e != cudaSuccess || !p) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: cudaGetSymbolAddress failed: %s\n", cudaGetErrorString(e));
        return PSB_ECUDA;
    }
    *out = (uint32_t*)p;
    return PSB_OK;
}

// Whether the byte ranges [a, a + bytes) and [b, b + bytes) share a byte.
bool overlap(const void* a, const void* b, size_t bytes) {
    const uintptr_t x = (uintptr_t)a, y = (uintptr_t)b;
    return x < y + bytes && y < x + bytes;
}

int copy(cudaStream_t st, uint32_t* dst, const uint32_t* src, int32_t n) {
    const cudaError_t e = cudaMemcpyAsync(dst, src, sizeof(uint32_t) * (size_t)n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: copy failed: %s\n", cudaGetErrorString(e));
        return PSB_ECUDA;
    }
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
    const size_t bytes = sizeof(uint32_t) * (size_t)n;
    if (overlap(keys_out, vals_out, bytes) || overlap(keys_out, vals_in, bytes) || overlap(vals_out, keys_in, bytes) ||
        (keys_out != keys_in && overlap(keys_out, keys_in, bytes)) ||
        (vals_out != vals_in && overlap(vals_out, vals_in, bytes))) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: overlapping buffers (only keys_out == keys_in and "
                             "vals_out == vals_in may alias)\n");
        return PSB_EINVAL;
    }
    // An error left pending by an earlier call of the caller's is not this
    // sort's: refuse to run and leave it for the caller to read.
    const cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: a CUDA error is pending from before the call: %s\n",
                     cudaGetErrorString(pending));
        return PSB_ECUDA;
    }
    uint32_t* scratch = nullptr;
    int rc = scratch_for_current_device(&scratch);
    if (rc != PSB_OK) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* tmp_keys = scratch;
    uint32_t* tmp_vals = scratch + kMaxN;
    uint32_t* hist = scratch + 2 * (size_t)kMaxN;
    // The sort ping-pongs between its two buffers starting from the first:
    // copy the input into the caller's output (unless it is the input),
    // sort between output and scratch, and copy back if the last pass ended
    // in the scratch.
    if (keys_out != keys_in && (rc = copy(st, keys_out, keys_in, n)) != PSB_OK) return rc;
    if (vals_out != vals_in && (rc = copy(st, vals_out, vals_in, n)) != PSB_OK) return rc;
    uint32_t* keys[2] = {keys_out, tmp_keys};
    uint32_t* vals[2] = {vals_out, tmp_vals};
    const int res = psb::radix_sort(st, n, key_bits, keys, vals, hist, kMaxBlocks);
    const cudaError_t e = cudaGetLastError();     // the sort's launches
    if (e != cudaSuccess) {
        std::fprintf(stderr, "psb_sort_cells_noalloc: %s\n", cudaGetErrorString(e));
        return PSB_ECUDA;
    }
    if (res == 1) {
        if ((rc = copy(st, keys_out, tmp_keys, n)) != PSB_OK) return rc;
        if ((rc = copy(st, vals_out, tmp_vals, n)) != PSB_OK) return rc;
    }
    return PSB_OK;
}
