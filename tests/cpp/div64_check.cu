// Test kernel: the library's FP64 division and reciprocal (csrc/
// cep_device.cuh div64 / rcp64) over operand arrays, for tests/
// test_division_gpu.py, which compares them with IEEE division.
#include <cuda_runtime.h>

#include "cep_device.cuh"

__global__ void div_kernel(const double *a, const double *b, double *q, double *r, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  q[i] = cep::div64(a[i], b[i]);
  r[i] = cep::rcp64(b[i]);
}

extern "C" int div64_check(const double *a, const double *b, double *q, double *r, int n) {
  double *d = nullptr;
  if (cudaMalloc(&d, sizeof(double) * 4 * (size_t)n) != cudaSuccess) return 1;
  cudaMemcpy(d, a, sizeof(double) * n, cudaMemcpyHostToDevice);
  cudaMemcpy(d + n, b, sizeof(double) * n, cudaMemcpyHostToDevice);
  div_kernel<<<(n + 127) / 128, 128>>>(d, d + n, d + 2 * n, d + 3 * n, n);
  cudaMemcpy(q, d + 2 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(r, d + 3 * n, sizeof(double) * n, cudaMemcpyDeviceToHost);
  const cudaError_t e = cudaGetLastError();
  cudaFree(d);
  return e == cudaSuccess ? 0 : 2;
}
