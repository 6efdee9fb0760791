// Throughput probe of the FP64 pipe, for the FP64 roofline of the step
// kernel: no step computes here. Each thread runs NCHAIN independent chains
// x <- fma(x, a, b) (one DFMA each, 2 flops), so the pipe, not the latency of
// one chain, sets the rate. The grid is a whole number of waves on every SM.
#include <cuda_runtime.h>

#include <cstdint>

namespace {

constexpr int NCHAIN = 16;

__global__ void __launch_bounds__(256) dfma_probe_kernel(double* out, int iters, double a, double b) {
  double x[NCHAIN];
#pragma unroll
  for (int c = 0; c < NCHAIN; ++c) x[c] = 1.0 + 1.0e-3 * (threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < NCHAIN; ++c) x[c] = fma(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < NCHAIN; ++c) s += x[c];
  // one store per block keeps the chains live without a memory stream
  if (s == 12345.0 || threadIdx.x == 0) out[blockIdx.x] = s;
}

}  // namespace

// Launch `blocks_per_sm` x (SM count) blocks of 256 threads, `iters` rounds
// of NCHAIN DFMA per thread, on `stream`; *flops is the launch's flop count
// (2 per DFMA). `out` holds one double per block.
extern "C" int shield_probe_dfma(double* out, int blocks_per_sm, int iters, double* flops, void* stream) {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -3;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -3;
  if (blocks_per_sm < 1 || iters < 1 || !out) return -1;
  const int grid = nsm * blocks_per_sm;
  dfma_probe_kernel<<<grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(out, iters, 0.999999999, 1.0e-9);
  if (flops) *flops = 2.0 * NCHAIN * (double)iters * 256.0 * grid;
  return cudaGetLastError() == cudaSuccess ? 0 : -3;
}

extern "C" int shield_probe_sm_count() {
  int dev = 0, nsm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -3;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -3;
  return nsm;
}
