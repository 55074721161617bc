// Test-only probe: evaluates the library's fast FP64 reciprocal and
// reciprocal square root (rcp_, rsqrt_ of physics.cuh) beside CUDA's own
// 1.0 / x and rsqrt(x) on an array of inputs, so that a test can bound their
// error in ulps.  Built by tests/test_gpu_fastmath.py; not part of the
// library.
#include <cuda_runtime.h>

#include "../../include/aerof_gpu.h"

#include "../../aerof_dev_b200/csrc/physics.cuh"

__global__ void k_probe(int n, const double* __restrict__ x, double* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  out[i] = aerof::rcp_(v);
  out[(size_t)n + i] = 1.0 / v;
  out[2 * (size_t)n + i] = aerof::rsqrt_(v);
  out[3 * (size_t)n + i] = rsqrt(v);
}

// out[4][n]: rcp_, 1.0/x, rsqrt_, rsqrt.  Returns 0 or a cudaError_t.
extern "C" int fastmath_probe(const double* x, int n, double* out) {
  double *dx = nullptr, *dout = nullptr;
  cudaError_t e = cudaMalloc(&dx, sizeof(double) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dout, sizeof(double) * 4 * (size_t)n);
  if (e == cudaSuccess) e = cudaMemcpy(dx, x, sizeof(double) * n, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_probe<<<(n + 255) / 256, 256>>>(n, dx, dout);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(out, dout, sizeof(double) * 4 * (size_t)n, cudaMemcpyDeviceToHost);
  cudaFree(dx);
  cudaFree(dout);
  return (int)e;
}
