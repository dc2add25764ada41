// marfa_probe.cu -- FP32 / FP64 FMA throughput of a GPU, measured by chains
// of independent FMAs.  The line-shape kernels run on these non-tensor pipes,
// so the benchmark uses the measured rates as their roofline denominators.
// Built into its own library (libmarfa_probe.so), which only the benchmark
// loads; it is not part of the line-by-line library's interface.
#include <cuda_runtime.h>

namespace {

template <typename T>
__global__ void __launch_bounds__(256) fma_chain_kernel(T *sink, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int j = 0; j < 8; ++j) x[j] = (T)(threadIdx.x + j);
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int j = 0; j < 8; ++j) x[j] = x[j] * a + b;
  }
  T s = 0;
#pragma unroll
  for (int j = 0; j < 8; ++j) s += x[j];
  if (s == (T)-1.2345) sink[threadIdx.x] = s; // keeps the chains alive
}

template <typename T>
cudaError_t fma_rate(T a, T b, int iters, double *flops_per_s) {
  int dev = 0, nsm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  void *sink = nullptr;
  cudaError_t e = cudaMalloc(&sink, 4096);
  if (e != cudaSuccess) return e;
  const int blocks = nsm * 8;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) { // the first launch warms up
    cudaEventRecord(e0);
    fma_chain_kernel<T><<<blocks, 256>>>((T *)sink, iters, a, b);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rep > 0) best = ms < best ? ms : best;
  }
  e = cudaGetLastError();
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(sink);
  *flops_per_s = 2.0 * 8.0 * (double)iters * blocks * 256 / (best * 1e-3);
  return e;
}

} // namespace

// FLOP/s of FP32 and FP64 FMA chains on `device` (FMA = 2 FLOP); 0 on success.
extern "C" int marfa_probe_fma_peak(int device, double *fp32_flops, double *fp64_flops) {
  if (!fp32_flops || !fp64_flops) return 1;
  if (cudaSetDevice(device) != cudaSuccess) return 2;
  if (fma_rate<float>(0.9999f, 1e-7f, 16384, fp32_flops) != cudaSuccess) return 3;
  if (fma_rate<double>(0.999999, 1e-7, 4096, fp64_flops) != cudaSuccess) return 3;
  return 0;
}
