// QMIV metric kernels for B200 (sm_100a).
//
// Pipeline of one frame pair (the reference runs the same steps per frame on the CPU,
// apps/QMIV/src/xAppQMIV.cpp:761-827):
//   k_prepass   per raw row: SD(In1-In0), SSD, max sample        (HBM bound, reads both frames once)
//   k_reduce    totals, GCD, exactness of the fp32 search path   (one CTA)
//   k_cps       (qmiv_cps.cu) corresponding-pixel-shift search, both directions in one pass;
//               per-row SSE into 32-bit lanes, the IV-SSIM sub-block moments of (test, SCP) and,
//               when IV-MS-SSIM or the caller needs them, the shift-compensated pictures
//   k_ssim_*    (qmiv_ssim.cu) block SSIM from exact integer moments, FP64 windows, row sums
//   k_finalize  every order-dependent FP64 pooling chain of the pair (one CTA per chain)
#include "qmiv_kernels.cuh"

#include <cstdio>
#include <mutex>

namespace qmiv {

constexpr unsigned kFull = 0xffffffffu;

// =============================================================================================
// prepass
// =============================================================================================
template <typename T>
__device__ __forceinline__ void prepass_body(const PrepassArgs& a, int warp)
{
  const int lane  = threadIdx.x & 31;
  const int total = a.rows[0] + a.rows[1] + a.rows[2];
  if(warp >= total) { return; }
  int c = 0, r = warp;
  if(r >= a.rows[0]) { r -= a.rows[0]; c = 1; if(r >= a.rows[1]) { r -= a.rows[1]; c = 2; } }
  const T* p0 = static_cast<const T*>(a.in0.p[c]) + (size_t)r * a.in0.pitch[c];
  const T* p1 = static_cast<const T*>(a.in1.p[c]) + (size_t)r * a.in1.pitch[c];
  const int n = a.cols[c];

  int64_t  sd  = 0;
  uint64_t ssd = 0;
  uint32_t m0 = 0, m1 = 0;
  auto sample = [&](uint32_t v0, uint32_t v1) {
    m0 = max(m0, v0); m1 = max(m1, v1);
    v0 = min(v0, a.clip); v1 = min(v1, a.clip);
    const int32_t d = (int32_t)v1 - (int32_t)v0;
    sd  += d;
    ssd += (uint32_t)d * (uint32_t)d;                    // d^2 < 2^32 for 16-bit samples
  };
  // 16-byte loads where both rows allow them (each lane then holds 8 or 16 samples of each frame in
  // flight), the rest of the row sample by sample
  int x0 = 0;
  if((((uintptr_t)p0 | (uintptr_t)p1) & 15) == 0)
  {
    constexpr int V = 16 / (int)sizeof(T);
    const int nv = n / V;
    const uint4* q0 = reinterpret_cast<const uint4*>(p0);
    const uint4* q1 = reinterpret_cast<const uint4*>(p1);
    for(int v = lane; v < nv; v += 32)
    {
      const uint4 A = __ldg(q0 + v), B = __ldg(q1 + v);
      const uint32_t wa[4] = { A.x, A.y, A.z, A.w }, wb[4] = { B.x, B.y, B.z, B.w };
      #pragma unroll
      for(int k = 0; k < 4; k++)
      {
        if(sizeof(T) == 2)
        {
          sample(wa[k] & 0xffffu, wb[k] & 0xffffu);
          sample(wa[k] >> 16, wb[k] >> 16);
        }
        else
        {
          #pragma unroll
          for(int b = 0; b < 4; b++) { sample((wa[k] >> (8 * b)) & 0xffu, (wb[k] >> (8 * b)) & 0xffu); }
        }
      }
    }
    x0 = nv * V;
  }
  for(int x = x0 + lane; x < n; x += 32) { sample(__ldg(p0 + x), __ldg(p1 + x)); }
  #pragma unroll
  for(int o = 16; o > 0; o >>= 1)
  {
    sd  += __shfl_xor_sync(kFull, sd, o);
    ssd += __shfl_xor_sync(kFull, ssd, o);
  }
  m0 = __reduce_max_sync(kFull, m0);
  m1 = __reduce_max_sync(kFull, m1);
  if(lane == 0)
  {
    a.row_sd[warp]  = sd;
    a.row_ssd[warp] = ssd;
    atomicMax(&a.out->max_sample[0], m0);
    atomicMax(&a.out->max_sample[1], m1);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_prepass(const __grid_constant__ PrepassArgs a)
{
  prepass_body<T>(a, (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5));
}

// one job (frame pair) per blockIdx.y
template <typename T>
__global__ void __launch_bounds__(256) k_prepass_multi(const PrepassArgs* __restrict__ jobs)
{
  prepass_body<T>(jobs[blockIdx.y], (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5));
}

template <typename T>
cudaError_t launch_prepass(const PrepassArgs& a, cudaStream_t s)
{
  const int total  = a.rows[0] + a.rows[1] + a.rows[2];
  const int blocks = (total + 7) / 8;
  k_prepass<T><<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}
template cudaError_t launch_prepass<uint8_t>(const PrepassArgs&, cudaStream_t);
template cudaError_t launch_prepass<uint16_t>(const PrepassArgs&, cudaStream_t);

template <typename T>
cudaError_t launch_prepass_multi(const PrepassArgs* d_jobs, int njobs, int max_rows, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  k_prepass_multi<T><<<dim3((max_rows + 7) / 8, njobs), 256, 0, s>>>(d_jobs);
  return cudaGetLastError();
}
template cudaError_t launch_prepass_multi<uint8_t>(const PrepassArgs*, int, int, cudaStream_t);
template cudaError_t launch_prepass_multi<uint16_t>(const PrepassArgs*, int, int, cudaStream_t);

// =============================================================================================
// reduce: totals and GCD (libs/pmbb-ivqm/src/xGlobClrDiff.cpp:70-103)
// =============================================================================================
__device__ __forceinline__ void reduce_body(const ReduceArgs& a)
{
  __shared__ int64_t  s_sd[3][32];
  __shared__ uint64_t s_ssd[3][32];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int off = 0;
  for(int c = 0; c < 3; c++)
  {
    int64_t sd = 0; uint64_t ssd = 0;
    for(int r = threadIdx.x; r < a.rows[c]; r += blockDim.x) { sd += a.row_sd[off + r]; ssd += a.row_ssd[off + r]; }
    #pragma unroll
    for(int o = 16; o > 0; o >>= 1) { sd += __shfl_xor_sync(kFull, sd, o); ssd += __shfl_xor_sync(kFull, ssd, o); }
    if(lane == 0) { s_sd[c][wid] = sd; s_ssd[c][wid] = ssd; }
    off += a.rows[c];
  }
  __syncthreads();
  if(threadIdx.x == 0)
  {
    PairOut* o = a.out;
    const int nw = blockDim.x >> 5;
    for(int c = 0; c < 3; c++)
    {
      int64_t sd = 0; uint64_t ssd = 0;
      for(int w = 0; w < nw; w++) { sd += s_sd[c][w]; ssd += s_ssd[c][w]; }
      o->sd[c]  = sd * a.mult[c];
      o->ssd[c] = ssd * (uint64_t)a.mult[c];
    }
    const double area = (double)a.area;
    for(int c = 0; c < 4; c++)
    {
      int32_t g = 0;
      if(a.gcd_override_on) { g = a.gcd_override[c]; }
      else if(a.need_gcd)
      {
        const double avg = ddiv(c < 3 ? (double)o->sd[c] : 0.0, area);
        g = clampi(round_half_away(avg), -a.maxdiff[c], a.maxdiff[c]);
      }
      o->gcd[c] = g;
    }
    const int inv0 = o->max_sample[0] > (uint32_t)a.maxv;
    const int inv1 = o->max_sample[1] > (uint32_t)a.maxv;
    const int int_path = !a.fp32_ok || ((inv0 || inv1) && !a.clip_on);
    o->flags = inv0 | (inv1 << 1) | (int_path << 2);
  }
}

__global__ void __launch_bounds__(1024) k_reduce(const __grid_constant__ ReduceArgs a) { reduce_body(a); }

// one job (frame pair) per CTA
__global__ void __launch_bounds__(1024) k_reduce_multi(const ReduceArgs* __restrict__ jobs) { reduce_body(jobs[blockIdx.x]); }

cudaError_t launch_reduce(const ReduceArgs& a, cudaStream_t s)
{
  k_reduce<<<1, 1024, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_reduce_multi(const ReduceArgs* d_jobs, int njobs, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  k_reduce_multi<<<njobs, 1024, 0, s>>>(d_jobs);
  return cudaGetLastError();
}

// (CPS search: qmiv_cps.cu)

// =============================================================================================
// finalize: the order-dependent FP64 pooling chains of one pair, one thread per chain.
// Inputs are staged chunk by chunk into shared memory by all threads so that each chain only
// waits on its own floating-point dependency.
//   WS-PSNR   KBNS over rows of rowSSD * w[y]            (xWSPSNR.cpp:123-132)
//   IV-PSNR   KBNS over rows of rowSSE * w[y] (ERP)       (xIVPSNR.cpp:171-175) + exact uint64 sums
//   SSIM      KBNS over window rows (ERP: row * w[base + step j], weights KBNS) (xSSIM.cpp:348-351,
//             xIVSSIM.cpp:148-172)
// =============================================================================================
// One CTA per chain: all threads stage the chain's inputs (independent loads) into shared memory,
// then thread 0 runs the ordered compensated sum. Chains of one pair run on different SMs.
__device__ __forceinline__ double chain_value(const FinalizeArgs& a, const FinChain& ch, int y)
{
  if(ch.kind == kChainWsPsnr)
  {
    int off = 0;
    for(int q = 0; q < ch.a; q++) { off += a.rows[q]; }
    const uint64_t r = a.row_ssd[off + (y >> a.sy[ch.a])] * (uint64_t)a.mult_row[ch.a];
    return dmul((double)r, a.ws[y]);
  }
  if(ch.kind == kChainIvPsnr)
  {
    const uint64_t r = (uint64_t)(int64_t)(int32_t)a.cps_rows[((size_t)ch.a * a.H + y) * 3 + ch.b];
    return dmul((double)r, a.ws[y]);
  }
  const SsimSlot& sl = a.slot[ch.a];
  const double v = sl.row_sum[(size_t)ch.b * sl.ny + y];
  return sl.use_ws ? dmul(v, a.ws[sl.ws_base + sl.ws_step * y]) : v;
}

__device__ __forceinline__ void finalize_body(const FinalizeArgs& a, int chain, double* stage)
{
  PairOut* o = a.out;
  if(chain == a.nchains)
  {
    // exact uint64 totals of the sign-extended 32-bit CPS row sums (order independent)
    __shared__ unsigned long long acc[6];
    if(threadIdx.x < 6) { acc[threadIdx.x] = 0ull; }
    __syncthreads();
    unsigned long long loc[6] = { 0, 0, 0, 0, 0, 0 };
    for(int y = threadIdx.x; y < a.H; y += blockDim.x)
    {
      #pragma unroll
      for(int k = 0; k < 6; k++)
      {
        loc[k] += (unsigned long long)(long long)(int32_t)a.cps_rows[((size_t)(k / 3) * a.H + y) * 3 + (k % 3)];
      }
    }
    #pragma unroll
    for(int k = 0; k < 6; k++)
    {
      #pragma unroll
      for(int o2 = 16; o2 > 0; o2 >>= 1) { loc[k] += __shfl_down_sync(0xffffffffu, loc[k], o2); }
      if((threadIdx.x & 31) == 0) { atomicAdd(&acc[k], loc[k]); }
    }
    __syncthreads();
    if(threadIdx.x < 6) { o->cps_sum[threadIdx.x / 3][threadIdx.x % 3] = acc[threadIdx.x]; }
    return;
  }
  const FinChain ch = a.chain[chain];
  const bool wsum = ch.kind == kChainSsim && a.slot[ch.a].use_ws;
  const int len = ch.kind == kChainSsim ? a.slot[ch.a].ny : a.H;
  double* vals = stage;
  double* wts = stage + len;
  // eight rows per thread and pass with their loads issued together (one round trip per pass)
  constexpr int U = 8;
  for(int y0 = threadIdx.x; y0 < len; y0 += 256 * U)
  {
    double v[U], w[U];
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int y = y0 + u * 256;
      v[u] = y < len ? chain_value(a, ch, y) : 0.0;
      w[u] = (wsum && y < len) ? a.ws[a.slot[ch.a].ws_base + a.slot[ch.a].ws_step * y] : 0.0;
    }
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int y = y0 + u * 256;
      if(y < len) { vals[y] = v[u]; if(wsum) { wts[y] = w[u]; } }
    }
  }
  __syncthreads();
  if(threadIdx.x != 0) { return; }
  Kbns sum, wk;
  int y = 0;
  for(; y + 8 <= len; y += 8)
  {
    double v[8], w[8];
    #pragma unroll
    for(int u = 0; u < 8; u++) { v[u] = vals[y + u]; w[u] = wsum ? wts[y + u] : 0.0; }
    #pragma unroll
    for(int u = 0; u < 8; u++) { sum.add(v[u]); if(wsum) { wk.add(w[u]); } }
  }
  for(; y < len; y++) { sum.add(vals[y]); if(wsum) { wk.add(wts[y]); } }
  if(ch.kind == kChainWsPsnr) { o->ws_ssd[ch.a] = sum.result(); }
  else if(ch.kind == kChainIvPsnr) { o->cps_ws[ch.a][ch.b] = sum.result(); }
  else
  {
    const SsimSlot& sl = a.slot[ch.a];
    const double active = (double)((int64_t)sl.nx * sl.ny);
    double r;
    if(wsum)
    {
      const double corr = ddiv(wk.result(), (double)sl.ny);
      r = ddiv(sum.result(), dmul(active, corr));
    }
    else { r = ddiv(sum.result(), active); }
    o->ssim[ch.a][ch.b] = r;
  }
}

__global__ void __launch_bounds__(256) k_finalize(const __grid_constant__ FinalizeArgs a)
{
  extern __shared__ double stage[];  // [len] values, then [len] ERP weights for weighted SSIM chains
  finalize_body(a, blockIdx.x, stage);
}

// one (pair, chain) job per CTA
__global__ void __launch_bounds__(256) k_finalize_multi(const FinalizeArgs* __restrict__ pairs, const FinJob* __restrict__ jobs)
{
  extern __shared__ double stage[];
  const FinJob j = jobs[blockIdx.x];
  finalize_body(pairs[j.pair], j.chain, stage);
}

int finalize_plan(FinalizeArgs& a)
{
  a.nchains = 0;
  if(a.do_wspsnr && a.ws) { for(int c = 0; c < 3; c++) { a.chain[a.nchains++] = { kChainWsPsnr, c, 0 }; } }
  if(a.cps_rows && a.ws) { for(int d = 0; d < 2; d++) { for(int c = 0; c < 3; c++) { a.chain[a.nchains++] = { kChainIvPsnr, d, c }; } } }
  for(int sl = 0; sl < a.nslots; sl++)
  {
    if(a.slot[sl].row_sum == nullptr || a.slot[sl].ny <= 0) { continue; }
    for(int c = 0; c < 3; c++) { a.chain[a.nchains++] = { kChainSsim, sl, c }; }
  }
  return a.nchains + (a.cps_rows ? 1 : 0);
}

size_t finalize_smem(const FinalizeArgs& a) { return (size_t)2 * max(a.H, 1) * sizeof(double); }

static cudaError_t finalize_configure()
{
  static std::mutex mu;
  static uint64_t done = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) { return e; }
  const uint64_t bit = 1ULL << (dev & 63);
  std::lock_guard<std::mutex> lk(mu);
  if(done & bit) { return cudaSuccess; }
  e = cudaFuncSetAttribute(k_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, kFinalizeMaxSmem);
  if(e == cudaSuccess) { e = cudaFuncSetAttribute(k_finalize_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, kFinalizeMaxSmem); }
  if(e == cudaSuccess) { done |= bit; }
  return e;
}

cudaError_t launch_finalize(const FinalizeArgs& a_in, cudaStream_t s)
{
  FinalizeArgs a = a_in;
  const int blocks = finalize_plan(a);
  if(blocks == 0) { return cudaSuccess; }
  const size_t smem = finalize_smem(a);
  if(smem > kFinalizeMaxSmem) { return cudaErrorInvalidValue; }
  cudaError_t e = finalize_configure();
  if(e != cudaSuccess) { return e; }
  k_finalize<<<blocks, 256, smem, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_finalize_multi(const FinalizeArgs* d_pairs, const FinJob* d_jobs, int njobs, size_t smem, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  if(smem > kFinalizeMaxSmem) { return cudaErrorInvalidValue; }
  cudaError_t e = finalize_configure();
  if(e != cudaSuccess) { return e; }
  k_finalize_multi<<<njobs, 256, smem, s>>>(d_pairs, d_jobs);
  return cudaGetLastError();
}

}  // namespace qmiv
