// Throughput probes for the roofline of the issue-bound search kernel (include/qmiv_probe.h).
#include "qmiv_host.h"
#include "qmiv_probe.h"

using namespace qmiv;

namespace {

constexpr int kChains = 8;

// Eight independent add/min chains per thread; the data dependence through neighbouring chains
// keeps the compiler from closing the loop into a formula.
__global__ void __launch_bounds__(256) k_int_peak(uint32_t* out, int iters, uint32_t seed)
{
  uint32_t x[kChains];
  #pragma unroll
  for(int k = 0; k < kChains; k++) { x[k] = seed * (threadIdx.x + 1) + 2654435761u * k; }
  const uint32_t cap = seed | 0x80000000u;
  for(int i = 0; i < iters; i++)
  {
    #pragma unroll
    for(int k = 0; k < kChains; k++) { x[k] = min(x[k] + x[(k + 1) % kChains], cap + (uint32_t)k); }
  }
  uint32_t r = 0;
  #pragma unroll
  for(int k = 0; k < kChains; k++) { r ^= x[k]; }
  if(r == 0x12345678u) { out[blockIdx.x] = r; }
}

__global__ void __launch_bounds__(256) k_fp32_peak(float* out, int iters, float seed)
{
  float x[kChains];
  #pragma unroll
  for(int k = 0; k < kChains; k++) { x[k] = seed + 0.001f * (threadIdx.x + k); }
  const float a = 0.999999f, b = 1e-7f;
  for(int i = 0; i < iters; i++)
  {
    #pragma unroll
    for(int k = 0; k < kChains; k++) { x[k] = fmaf(x[k], a, b); }
  }
  float r = 0.f;
  #pragma unroll
  for(int k = 0; k < kChains; k++) { r += x[k]; }
  if(r == 1234.5f) { out[blockIdx.x] = r; }
}

// Eight independent chains of separately rounded multiply and add per thread: the instruction mix of
// the Gaussian-float SSIM window sums. Each DMUL and each DADD counts as one operation.
__global__ void __launch_bounds__(256) k_fp64_peak(double* out, int iters, double seed)
{
  double x[kChains];
  #pragma unroll
  for(int k = 0; k < kChains; k++) { x[k] = seed + 0.001 * (threadIdx.x + k); }
  const double a = 0.9999999, b = 1e-9;
  for(int i = 0; i < iters; i++)
  {
    #pragma unroll
    for(int k = 0; k < kChains; k++) { x[k] = __dadd_rn(__dmul_rn(x[k], a), b); }
  }
  double r = 0.0;
  #pragma unroll
  for(int k = 0; k < kChains; k++) { r += x[k]; }
  if(r == 1234.5) { out[blockIdx.x] = r; }
}

template <typename K>
qmiv_status time_kernel(int32_t device, K launch, double* ms_out)
{
  QMIV_CUDA(cudaSetDevice(device));
  cudaEvent_t a, b;
  QMIV_CUDA(cudaEventCreate(&a));
  QMIV_CUDA(cudaEventCreate(&b));
  launch();  // warm-up
  QMIV_CUDA(cudaGetLastError());
  QMIV_CUDA(cudaEventRecord(a));
  launch();
  QMIV_CUDA(cudaEventRecord(b));
  QMIV_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  QMIV_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  *ms_out = ms;
  return QMIV_OK;
}

}  // namespace

using namespace qmiv;

extern "C" {

qmiv_status qmiv_probe_int32_peak(int32_t device, int32_t iters, double* tops)
{
  if(!tops || iters <= 0) { return fail(QMIV_ERR_INVALID_ARG, "bad probe arguments"); }
  int sms = 0;
  QMIV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8, threads = 256;
  uint32_t* out = nullptr;
  QMIV_CUDA(cudaSetDevice(device));
  QMIV_CUDA(cudaMalloc(&out, blocks * sizeof(uint32_t)));
  double ms = 0;
  const qmiv_status st = time_kernel(device, [&] { k_int_peak<<<blocks, threads>>>(out, iters, 12345u); }, &ms);
  cudaFree(out);
  QMIV_TRY(st);
  const double ops = 2.0 * kChains * (double)iters * blocks * threads;
  *tops = ops / (ms * 1e-3) / 1e12;
  return QMIV_OK;
}

qmiv_status qmiv_probe_fp32_peak(int32_t device, int32_t iters, double* tflops)
{
  if(!tflops || iters <= 0) { return fail(QMIV_ERR_INVALID_ARG, "bad probe arguments"); }
  int sms = 0;
  QMIV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8, threads = 256;
  float* out = nullptr;
  QMIV_CUDA(cudaSetDevice(device));
  QMIV_CUDA(cudaMalloc(&out, blocks * sizeof(float)));
  double ms = 0;
  const qmiv_status st = time_kernel(device, [&] { k_fp32_peak<<<blocks, threads>>>(out, iters, 1.0f); }, &ms);
  cudaFree(out);
  QMIV_TRY(st);
  const double flops = 2.0 * kChains * (double)iters * blocks * threads;
  *tflops = flops / (ms * 1e-3) / 1e12;
  return QMIV_OK;
}

qmiv_status qmiv_probe_fp64_peak(int32_t device, int32_t iters, double* tops)
{
  if(!tops || iters <= 0) { return fail(QMIV_ERR_INVALID_ARG, "bad probe arguments"); }
  int sms = 0;
  QMIV_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  const int blocks = sms * 8, threads = 256;
  double* out = nullptr;
  QMIV_CUDA(cudaSetDevice(device));
  QMIV_CUDA(cudaMalloc(&out, blocks * sizeof(double)));
  double ms = 0;
  const qmiv_status st = time_kernel(device, [&] { k_fp64_peak<<<blocks, threads>>>(out, iters, 1.0); }, &ms);
  cudaFree(out);
  QMIV_TRY(st);
  const double ops = 2.0 * kChains * (double)iters * blocks * threads;
  *tops = ops / (ms * 1e-3) / 1e12;
  return QMIV_OK;
}

}  // extern "C"
