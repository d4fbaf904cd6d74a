// fp64_probe.cu -- the FP64 fused multiply-add rate of the device, measured
// for the bench's FP64 roofline (the HBM roofline's denominator is measured
// by the driver; the FP64 pipe's is measured here, the same way: a kernel
// that does nothing else, timed with CUDA events, best of several runs).
//
// Every thread runs 8 independent chains of dependent fused multiply-adds
// (enough independent work to cover the pipe's latency), and writes their sum
// so that none of the work can be left out.  The grid fills every SM.
#include <cuda_runtime.h>

#include <cstdio>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) dfma_kernel(int iters, double a, double b,
                                                    double* __restrict__ out) {
  double x[kChains];
#pragma unroll
  for (int c = 0; c < kChains; ++c) x[c] = 1.0 + 1e-3 * (threadIdx.x + c);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = __fma_rn(x[c], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < kChains; ++c) s += x[c];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

extern "C" {

// Best of `reps` launches of `iters` steps per chain: FP64 operations per
// second (a fused multiply-add counts two) into *flops, the launch's
// milliseconds into *ms.  4096 steps take about 0.55 ms on a B200; a launch
// is held under about half a second (iters <= 2^22), reps to 10000.  0 on
// success, -1 on a bad argument, -2 on a CUDA error.
int gfx_probe_fp64_chains(int reps, int iters, double* flops, double* ms) {
  if (reps < 1 || reps > 10000 || iters < 1 || iters > (1 << 22) || !flops || !ms) return -1;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -2;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -2;
  const int block = 256, grid = sms * 8;
  double* out = nullptr;
  if (cudaMalloc(&out, sizeof(double) * grid * block) != cudaSuccess) return -2;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  int rc = 0;
  for (int r = 0; r < reps + 1 && rc == 0; ++r) {  // the first launch warms up
    cudaEventRecord(e0);
    dfma_kernel<<<grid, block>>>(iters, 0.999999, 1e-7, out);
    cudaEventRecord(e1);
    if (cudaEventSynchronize(e1) != cudaSuccess) rc = -2;
    float t = 0.f;
    cudaEventElapsedTime(&t, e0, e1);
    if (r > 0 && t < best) best = t;
  }
  if (cudaGetLastError() != cudaSuccess) rc = -2;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  if (rc) return rc;
  *ms = best;
  *flops = 2.0 * kChains * (double)iters * grid * block / (best * 1e-3);
  return 0;
}

int gfx_probe_fp64(int reps, double* flops, double* ms) {
  return gfx_probe_fp64_chains(reps, 4096, flops, ms);
}

}  // extern "C"
