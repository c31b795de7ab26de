// learned.cuh — shapes and launchers of the learned-proposal kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "rcmvs_internal.cuh"

namespace rcmvs {

constexpr int COSTVOL_PLANES = 32;  // fronto-parallel planes of the coarse cost volume
constexpr int COSTVOL_C = 48;       // 32 costs + grey + 15 zero channels (multiple of 16)
constexpr int NET_OUT_C = 16;       // t, nx, ny, nz, confidence logit + 11 zero channels
constexpr int NET_LAYERS = 6;
constexpr int NET_CIN[NET_LAYERS] = {48, 32, 32, 32, 32, 32};
constexpr int NET_CIN_REAL[NET_LAYERS] = {33, 32, 32, 32, 32, 32};
constexpr int NET_COUT[NET_LAYERS] = {32, 32, 32, 32, 32, 16};
constexpr int NET_COUT_REAL[NET_LAYERS] = {32, 32, 32, 32, 32, 5};

cudaError_t launch_downsample4(const DevView* full, const DevView* quarter, const int32_t* blk_start, int n_views,
                               int total_blocks, const uint8_t* gray, uint8_t* gray_q, cudaStream_t st);
// Blocks (32x8 quarter-pixel tiles) the cost-volume kernel uses for a
// w x h quarter view; a batch's jobs take consecutive tile ranges.
int costvol_tiles(int w, int h);
cudaError_t launch_costvol(const DevJob* jobs, const int32_t* blk_start, int n_jobs, int total_blocks,
                           const int64_t* out_off, const uint64_t* census_q, const float2* rays_q,
                           const uint8_t* gray_q, void* out, cudaStream_t st);
cudaError_t launch_conv3x3(int cin, int cout, bool relu, bool out_f32, const void* x, const void* mask, int N, int H,
                           int W, const void* w, const float* b, void* y, cudaStream_t st);
// Reads and clears the device word the tensor-core kernels set when one of
// their bounded waits gave up (1), 0 if none did, -1 if it could not be read.
int tc_fault_take();
// One block waits limit_ns on an mbarrier that nothing arrives on and sets
// the fault word when the wait gives up (rcmvs_diag_wait_timeout).
cudaError_t launch_wait_probe(uint64_t limit_ns, cudaStream_t st);
cudaError_t launch_conv3x3_wgrad(int cin, int cout, const void* x, const void* dy, const void* mask, int N, int H,
                                 int W, float* dW, cudaStream_t st);
cudaError_t launch_bias_grad(int c, const void* dy, const void* mask, int64_t npx, float* db, cudaStream_t st);
cudaError_t launch_flip_weights(const void* w, int cout, int cin, void* wt, cudaStream_t st);
cudaError_t launch_to_bf16(const float* a, int64_t n, void* b, cudaStream_t st);
cudaError_t launch_loss(const float* out, const float* lab, int64_t npx, float inv_n, void* dout, float* acc,
                        cudaStream_t st);
cudaError_t launch_adam(float* p, const float* g, float* m, float* v, const uint8_t* mask, int64_t n, float lr,
                        float b1, float b2, float eps, float bc1, float bc2, float gscale, void* pb, cudaStream_t st);
}  // namespace rcmvs
