// Live measurement of the integer-add rate that bounds the dedispersion sums.
// Each thread runs eight independent chains of three-input 32-bit adds whose
// operands change every iteration (so nothing can be folded), from registers
// only; the rate is additions per second with a three-input add counted as two.
#include <cuda_runtime.h>

#include <cstdint>

#include "dd_internal.h"

namespace dd {
namespace {

constexpr int kProbeIters = 1 << 14;

__global__ void k_iadd3_chains(const uint32_t* __restrict__ seed, uint32_t* __restrict__ sink) {
  uint32_t a0 = seed[threadIdx.x & 7], a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3;
  uint32_t a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
  uint32_t b = seed[8], c = seed[9];
#pragma unroll 4
  for (int i = 0; i < kProbeIters; ++i) {
    a0 = a0 + b + c; a1 = a1 + c + b; a2 = a2 + b + a0; a3 = a3 + c + a1;
    a4 = a4 + b + c; a5 = a5 + c + b; a6 = a6 + b + a4; a7 = a7 + c + a5;
    b ^= static_cast<uint32_t>(i);
    c += a7;
  }
  sink[blockIdx.x * blockDim.x + threadIdx.x] = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
}

}  // namespace

double measure_int_add_rate(int device) {
  int nsm = 0;
  DD_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device));
  const int threads = 256, blocks = nsm * 8;
  DevBuf seed, sink;
  seed.alloc(64 * sizeof(uint32_t));
  sink.alloc(static_cast<size_t>(blocks) * threads * sizeof(uint32_t));
  DD_CUDA_TRY(cudaMemset(seed.p, 1, seed.bytes));
  cudaEvent_t e0, e1;
  DD_CUDA_TRY(cudaEventCreate(&e0));
  DD_CUDA_TRY(cudaEventCreate(&e1));
  // warm up until clocks settle, then time several launches
  for (int r = 0; r < 3; ++r) {
    k_iadd3_chains<<<blocks, threads>>>(seed.as<uint32_t>(), sink.as<uint32_t>());
    DD_LAUNCHED();
  }
  const int reps = 5;
  DD_CUDA_TRY(cudaEventRecord(e0));
  for (int r = 0; r < reps; ++r) {
    k_iadd3_chains<<<blocks, threads>>>(seed.as<uint32_t>(), sink.as<uint32_t>());
    DD_LAUNCHED();
  }
  DD_CUDA_TRY(cudaEventRecord(e1));
  DD_CUDA_TRY(cudaEventSynchronize(e1));
  float ms = 0.f;
  DD_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const double adds = static_cast<double>(reps) * blocks * threads * kProbeIters * 8.0 * 2.0;
  return adds / (static_cast<double>(ms) * 1e-3);
}

}  // namespace dd
