// batch.cu -- the corrector loop of batched scenes, on the device.
//
// A batch steps many independent scenes together: every sweep is one launch
// over all scenes' particles, and each scene keeps its own convergence test.
// One small kernel runs after each density pass: it records every iterating
// scene's max compression error, retires the scenes that meet eta (after at
// least min_iters corrections) and decides whether another pass is needed.
// The pressure-force pass that follows skips retired scenes, so each scene
// ends in the state it has when stepped alone: the same passes, in the same
// order, on the same data. The decision reaches the host as one word, or,
// inside a CUDA graph, the conditional handle of the while node that
// repeats {density pass, decision, pressure-force pass}.
//
// Loop words (device int array): [0] the pass index k, [1] continue,
// [2, 2 + S) corrections per scene, [2 + S, 2 + 2S) converged per scene,
// [2 + 2S, 2 + 3S) corrections summed over steps, [2 + 3S, 2 + 4S) steps
// that ended at max_iters (the sums are cleared by an upload).
#include "psb.h"
#include "psb_internal.cuh"

namespace psb {

namespace {

constexpr int kLoopThreads = 256;

__global__ void __launch_bounds__(kLoopThreads) k_batch_begin(int S, int max_it, uint8_t* __restrict__ active,
                                                             unsigned long long* __restrict__ err_scene,
                                                             unsigned long long* __restrict__ err_hist, int hist_len,
                                                             int* __restrict__ loop) {
    corrector_begin(S, max_it, active, err_scene, err_hist, hist_len, loop);
}

__global__ void __launch_bounds__(kLoopThreads) k_batch_decide(int S, int min_it, int max_it, double eta,
                                                              uint8_t* __restrict__ active,
                                                              unsigned long long* __restrict__ err_scene,
                                                              unsigned long long* __restrict__ err_hist,
                                                              int* __restrict__ loop,
                                                              cudaGraphConditionalHandle handle, int set_handle) {
    __shared__ int any;
    const int cont = corrector_decide(S, min_it, max_it, eta, active, err_scene, err_hist, loop, &any);
    if (threadIdx.x == 0 && set_handle) cudaGraphSetConditional(handle, cont ? 1u : 0u);
}

}  // namespace

void launch_batch_begin(cudaStream_t st, int S, int max_it, uint8_t* active, unsigned long long* err_scene,
                        unsigned long long* err_hist, int hist_len, int* loop) {
    k_batch_begin<<<1, kLoopThreads, 0, st>>>(S, max_it, active, err_scene, err_hist, hist_len, loop);
}

void launch_batch_decide(cudaStream_t st, int S, int min_it, int max_it, double eta, uint8_t* active,
                         unsigned long long* err_scene, unsigned long long* err_hist, int* loop,
                         cudaGraphConditionalHandle handle, int set_handle) {
    k_batch_decide<<<1, kLoopThreads, 0, st>>>(S, min_it, max_it, eta, active, err_scene, err_hist, loop, handle,
                                               set_handle);
}

}  // namespace psb
