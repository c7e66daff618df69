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

// SFU (MUFU) throughput: independent ex2.approx chains.
__global__ void sfu_loop(float *out, int iters) {
  float x0 = threadIdx.x * 1e-3f, x1 = x0 + 0.1f, x2 = x0 + 0.2f, x3 = x0 + 0.3f;
  float x4 = x0 + 0.4f, x5 = x0 + 0.5f, x6 = x0 + 0.6f, x7 = x0 + 0.7f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      x0 = exp2f(-x0); x1 = exp2f(-x1); x2 = exp2f(-x2); x3 = exp2f(-x3);
      x4 = exp2f(-x4); x5 = exp2f(-x5); x6 = exp2f(-x6); x7 = exp2f(-x7);
    }
  }
  const float s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == -12345.f) out[0] = s;
}

// Which SM sub-partition each warp of a 4-warp block lands on: out[b*4+w] =
// %warpid & 3 for block b, warp w (launch shape of the ionic roles kernel).
__global__ void warp_slot_probe(int *out) {
  unsigned wid;
  asm volatile("mov.u32 %0, %%warpid;" : "=r"(wid));
  if ((threadIdx.x & 31) == 0) out[blockIdx.x * 4 + (threadIdx.x >> 5)] = (int)(wid & 3u);
}

// b = a over n 16-byte elements, `passes` times: with both arrays inside
// the L2 after the first pass, the copy streams at L2 bandwidth.
__global__ void l2_copy(const double2 *__restrict__ a, double2 *__restrict__ b, long n, int passes) {
  const long stride = (long)gridDim.x * blockDim.x;
  for (int p = 0; p < passes; ++p)
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) b[i] = a[i];
}

extern "C" {
// L2 copy bandwidth in bytes/s (read + write) over a 2 x 24 MiB working set.
double cep_probe_l2_copy_bytes(void) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long n = (24L << 20) / (long)sizeof(double2);
  double2 *a = nullptr, *b = nullptr;
  if (cudaMalloc(&a, n * sizeof(double2)) != cudaSuccess) return -1.0;
  if (cudaMalloc(&b, n * sizeof(double2)) != cudaSuccess) {
    cudaFree(a);
    return -1.0;
  }
  cudaMemset(a, 0, n * sizeof(double2));
  const int block = 256, grid = sms * 8, passes = 64;
  l2_copy<<<grid, block>>>(a, b, n, 2);  // warm: both arrays into the L2
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  l2_copy<<<grid, block>>>(a, b, n, passes);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(a);
  cudaFree(b);
  const double bytes = 2.0 * (double)n * sizeof(double2) * passes;
  return cudaGetLastError() == cudaSuccess && ms > 0 ? bytes / (ms * 1e-3) : -1.0;
}

// SFU operations/s (ex2.approx) on the current device.
double cep_probe_sfu_ops(void) {
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  float *out = nullptr;
  if (cudaMalloc(&out, sizeof(float)) != cudaSuccess) return -1.0;
  const int block = 256, grid = sms * 8, iters = 512;
  sfu_loop<<<grid, block>>>(out, 8);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0);
  sfu_loop<<<grid, block>>>(out, iters);
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  float ms = 0;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(out);
  const double ops = (double)grid * block * iters * 16.0 * 8.0;
  return cudaGetLastError() == cudaSuccess && ms > 0 ? ops / (ms * 1e-3) : -1.0;
}

// Fraction of 4-warp blocks (n_blocks of them, 128 threads) whose warps sit
// on four distinct SM sub-partitions.
double cep_probe_warp_slots(int n_blocks) {
  int *d = nullptr;
  if (n_blocks <= 0 || cudaMalloc(&d, sizeof(int) * 4 * n_blocks) != cudaSuccess) return -1.0;
  warp_slot_probe<<<n_blocks, 128>>>(d);
  int *h = new int[4 * n_blocks];
  cudaMemcpy(h, d, sizeof(int) * 4 * n_blocks, cudaMemcpyDeviceToHost);
  cudaFree(d);
  int ok = 0;
  for (int b = 0; b < n_blocks; ++b) {
    int m = 0;
    for (int w = 0; w < 4; ++w) m |= 1 << (h[b * 4 + w] & 3);
    ok += (m == 0xF);
  }
  delete[] h;
  return (double)ok / n_blocks;
}

// FP32 / FP64 FMA throughput in flop/s (2 per FMA) on the current device.
double cep_probe_fp32_fma_flops(void) { return measure<float>(4096); }
double cep_probe_fp64_fma_flops(void) { return measure<double>(1024); }
}
