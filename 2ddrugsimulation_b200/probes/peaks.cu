// Measurement probes for bench.py's roofline denominators: the FP32 and
// FP64 FMA throughput of the GPU the bench runs on (MEASURED_PEAKS.json
// carries only HBM and bf16 tensor figures). Independent FMA chains per
// thread, enough warps to saturate every SM; returns flops/s (2 per FMA).
#include <cuda_runtime.h>

template <class T>
__global__ void fma_loop(T *out, int iters, T a, T b) {
  T x0 = (T)threadIdx.x, x1 = x0 + (T)1, x2 = x0 + (T)2, x3 = x0 + (T)3;
  T x4 = x0 + (T)4, x5 = x0 + (T)5, x6 = x0 + (T)6, x7 = x0 + (T)7;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == (T)-12345) out[0] = s;  // keep the chains live
}

template <class T>
static double measure(int iters) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  T *out = nullptr;
  if (cudaMalloc(&out, sizeof(T)) != cudaSuccess) return -1.0;
  const int block = 256, grid = sms * 8;
  fma_loop<T><<<grid, block>>>(out, 8, (T)0.999, (T)0.001);  // warm-up
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  fma_loop<T><<<grid, block>>>(out, iters, (T)0.999, (T)0.001);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double fmas = (double)grid * block * iters * 16.0 * 8.0;
  return cudaGetLastError() == cudaSuccess && ms > 0 ? 2.0 * fmas / (ms * 1e-3) : -1.0;
}

extern "C" {
// FP32 / FP64 FMA throughput in flop/s (2 per FMA) on the current device.
double cep_probe_fp32_fma_flops(void) { return measure<float>(4096); }
double cep_probe_fp64_fma_flops(void) { return measure<double>(1024); }
}
