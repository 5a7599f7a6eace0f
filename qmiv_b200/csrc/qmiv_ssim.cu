// Block SSIM (8x8 windows at stride 4, xSSIM.cpp:276-369, xStructSimSTD.cpp:420-461) on B200.
//
// Window moments are sums of 2x2 exact integer 4x4 sub-block moments. They come either from the
// CPS search's epilogue (IV-SSIM: test picture vs its shift-compensated picture, so the SCP never
// needs to be stored) or from k_ssim_moments (plain SSIM, MS-SSIM scales, which also writes the
// next scale's 2x2 mean, xPixelOpsSTD.cpp:50-67). k_ssim_pool evaluates every window in FP64 with the
// reference's operation order and sums each window row in x order with the compensated sum, one
// lane per row, while other warps evaluate the next windows.
#include "qmiv_kernels.cuh"

#include <mutex>

namespace qmiv {

// =============================================================================================
// moments of an image pair, one thread per 4x4 sub-block
// =============================================================================================
template <typename T>
__device__ __forceinline__ void ssim_moments_body(const SsimMomArgs& a, int c)
{
  const int bx = blockIdx.x * 32 + (threadIdx.x & 31);
  const int by = blockIdx.y * 8 + (threadIdx.x >> 5);
  const Moments& M = a.mom;
  if(bx >= M.nbx || by >= M.nby) { return; }
  uint32_t va[4][4], vb[4][4];
  #pragma unroll
  for(int yy = 0; yy < 4; yy++)
  {
    const int gy = min(4 * by + yy, a.H - 1);
    #pragma unroll
    for(int xx = 0; xx < 4; xx++)
    {
      const int gx = min(4 * bx + xx, a.W - 1);
      va[yy][xx] = min((uint32_t)fetch<T>(a.a, c, gx, gy), a.clip);
      vb[yy][xx] = min((uint32_t)fetch<T>(a.b, c, gx, gy), a.clip);
    }
  }
  uint32_t s[5] = { 0, 0, 0, 0, 0 };
  #pragma unroll
  for(int yy = 0; yy < 4; yy++)
  {
    #pragma unroll
    for(int xx = 0; xx < 4; xx++)
    {
      const uint32_t p = va[yy][xx], q = vb[yy][xx];
      s[0] += p; s[1] += q; s[2] += p * p; s[3] += q * q; s[4] += p * q;
    }
  }
  const size_t o = (size_t)by * M.pitch + bx;
  #pragma unroll
  for(int m = 0; m < 5; m++) { M.p[((size_t)c * 5 + m) * M.plane() + o] = s[m]; }

  // 2x2 means of this 4x4 block for the next scale ((W>>1) x (H>>1))
  const int dw = a.W >> 1, dh = a.H >> 1;
  #pragma unroll
  for(int dy = 0; dy < 2; dy++)
  {
    #pragma unroll
    for(int dx = 0; dx < 2; dx++)
    {
      const int ox = 2 * bx + dx, oy = 2 * by + dy;
      if(ox >= dw || oy >= dh) { continue; }
      if(a.down_a.p[c])
      {
        const uint32_t v = (va[2 * dy][2 * dx] + va[2 * dy][2 * dx + 1] + va[2 * dy + 1][2 * dx] + va[2 * dy + 1][2 * dx + 1] + 2) >> 2;
        static_cast<T*>(a.down_a.p[c])[(size_t)oy * a.down_a.pitch[c] + ox] = (T)v;
      }
      if(a.down_b.p[c])
      {
        const uint32_t v = (vb[2 * dy][2 * dx] + vb[2 * dy][2 * dx + 1] + vb[2 * dy + 1][2 * dx] + vb[2 * dy + 1][2 * dx + 1] + 2) >> 2;
        static_cast<T*>(a.down_b.p[c])[(size_t)oy * a.down_b.pitch[c] + ox] = (T)v;
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_ssim_moments(const __grid_constant__ SsimMomArgs a)
{
  ssim_moments_body<T>(a, blockIdx.z);
}

// blockIdx.z = 3 * job + component
template <typename T>
__global__ void __launch_bounds__(256) k_ssim_moments_multi(const SsimMomArgs* __restrict__ jobs)
{
  ssim_moments_body<T>(jobs[blockIdx.z / 3], blockIdx.z % 3);
}

template <typename T>
cudaError_t launch_ssim_moments_multi(const SsimMomArgs* d_jobs, int njobs, int max_nbx, int max_nby, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  const dim3 grid((max_nbx + 31) / 32, (max_nby + 7) / 8, 3 * njobs);
  k_ssim_moments_multi<T><<<grid, 256, 0, s>>>(d_jobs);
  return cudaGetLastError();
}
template cudaError_t launch_ssim_moments_multi<uint8_t>(const SsimMomArgs*, int, int, int, cudaStream_t);
template cudaError_t launch_ssim_moments_multi<uint16_t>(const SsimMomArgs*, int, int, int, cudaStream_t);

template <typename T>
cudaError_t launch_ssim_moments(const SsimMomArgs& a, cudaStream_t s)
{
  const dim3 grid((a.mom.nbx + 31) / 32, (a.mom.nby + 7) / 8, 3);
  k_ssim_moments<T><<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}
template cudaError_t launch_ssim_moments<uint8_t>(const SsimMomArgs&, cudaStream_t);
template cudaError_t launch_ssim_moments<uint16_t>(const SsimMomArgs&, cudaStream_t);

// =============================================================================================
// windows + ordered row sums (xSSIM.cpp:353-369). A CTA owns kPoolRows = 32 window rows of one job
// and walks them in chunks of kPoolCW = 32 windows. Eight producer warps copy the chunk's 33 x 33
// sub-block moments into shared memory with cp.async (double-buffered: chunk k+1 is in flight while
// chunk k is evaluated) and evaluate four independent windows per thread; a ninth warp keeps the
// 32 compensated row sums, lane j adding row j's values in x order. Window values pass through two
// shared buffers guarded by named barriers (full: producers -> summing warp, empty: summing warp ->
// producers), so evaluation and the serial sums overlap and one warp instruction advances 32 sums.
// =============================================================================================
constexpr int kPoolRows = 32, kPoolCW = 32, kPoolEval = 256, kPoolThreads = kPoolEval + 32;
constexpr int kPSubR = kPoolRows + 1, kPSubC = kPoolCW + 1;        // 33 x 33 sub-blocks per chunk
constexpr int kPStage = 5 * kPSubR * kPSubC;                       // staged moment values per chunk
constexpr size_t kPoolSmem = (size_t)2 * kPStage * 4 + (size_t)2 * kPoolRows * (kPoolCW + 1) * 8;
enum { kBarFull0 = 1, kBarEmpty0 = 3, kBarStage = 5 };            // named barrier ids (0 = __syncthreads)

__device__ __forceinline__ void bar_sync(int id, int n) { asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(n) : "memory"); }
__device__ __forceinline__ void bar_arrive(int id, int n) { asm volatile("bar.arrive %0, %1;" ::"r"(id), "r"(n) : "memory"); }
// 4-byte asynchronous global -> shared copy; src_bytes 0 writes a zero
__device__ __forceinline__ void cp_async4(void* dst, const void* src, uint32_t src_bytes)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src),
               "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__device__ __forceinline__ void ssim_pool_body(const SsimPoolJob& J)
{
  extern __shared__ __align__(16) unsigned char pool_smem[];
  uint32_t (*st)[5][kPSubR][kPSubC] = reinterpret_cast<uint32_t (*)[5][kPSubR][kPSubC]>(pool_smem);
  double (*vals)[kPoolRows][kPoolCW + 1] = reinterpret_cast<double (*)[kPoolRows][kPoolCW + 1]>(pool_smem + (size_t)2 * kPStage * 4);
  const int j0 = blockIdx.x * kPoolRows;
  if(j0 >= J.ny) { return; }
  const int nchunks = (J.nx + kPoolCW - 1) / kPoolCW;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  if(t < kPoolEval)
  {
    // ---- producers: copy, evaluate
    const int nby = J.ny + 1, nbx = J.nx + 1;  // sub-blocks any window of this job touches
    auto issue = [&](int k) {
      uint32_t* dst = &st[k & 1][0][0][0];
      const int i0 = k * kPoolCW;
      for(int rr = warp; rr < 5 * kPSubR; rr += kPoolEval / 32)
      {
        const int m = rr / kPSubR, sy = rr - m * kPSubR, gy = j0 + sy;
        const uint32_t* src = J.mom + (size_t)m * J.plane + (size_t)min(gy, nby - 1) * J.pitch;
        for(int sx = lane; sx < kPSubC; sx += 32)
        {
          const int gx = i0 + sx;
          const bool in = gy < nby && gx < nbx;
          cp_async4(dst + (m * kPSubR + sy) * kPSubC + sx, src + (in ? gx : 0), in ? 4u : 0u);
        }
      }
      cp_async_commit();
    };
    issue(0);
    cp_async_wait_all();
    bar_sync(kBarStage, kPoolEval);
    for(int k = 0; k < nchunks; k++)
    {
      const int b = k & 1;
      if(k + 1 < nchunks) { issue(k + 1); }   // st[b ^ 1] was last read by chunk k - 1, before the stage barrier
      double v[kPoolRows / 8];
      #pragma unroll
      for(int q = 0; q < kPoolRows / 8; q++)
      {
        const int jj = warp + 8 * q, i = k * kPoolCW + lane, j = j0 + jj;
        v[q] = 0.0;
        if(i < J.nx && j < J.ny)
        {
          uint64_t sm[5];
          #pragma unroll
          for(int m = 0; m < 5; m++)
          {
            sm[m] = (uint64_t)st[b][m][jj][lane] + st[b][m][jj][lane + 1] + st[b][m][jj + 1][lane] + st[b][m][jj + 1][lane + 1];
          }
          // moment 0/2 = "Tst" picture, 1/3 = "Ref" picture
          v[q] = ssim_window(sm[1], sm[0], sm[3], sm[2], sm[4], J.C1, J.C2, J.calc_l != 0);
        }
      }
      if(k >= 2) { bar_sync(kBarEmpty0 + b, kPoolThreads); }   // the summing warp is done with chunk k - 2
      #pragma unroll
      for(int q = 0; q < kPoolRows / 8; q++) { vals[b][warp + 8 * q][lane] = v[q]; }
      bar_arrive(kBarFull0 + b, kPoolThreads);
      if(k + 1 < nchunks)
      {
        cp_async_wait_all();
        bar_sync(kBarStage, kPoolEval);
      }
    }
  }
  else
  {
    // ---- summing warp: lane j owns window row j0 + j
    const bool rowv = j0 + lane < J.ny;
    Kbns row;
    for(int k = 0; k < nchunks; k++)
    {
      const int b = k & 1;
      bar_sync(kBarFull0 + b, kPoolThreads);
      const int cnt = min(kPoolCW, J.nx - k * kPoolCW);
      if(rowv)
      {
        for(int u = 0; u < cnt; u++) { row.add(vals[b][lane][u]); }
      }
      if(k + 2 < nchunks) { bar_arrive(kBarEmpty0 + b, kPoolThreads); }
    }
    if(rowv) { J.row_sum[j0 + lane] = row.result(); }
  }
}

__global__ void __launch_bounds__(kPoolThreads, 2) k_ssim_pool(const __grid_constant__ SsimPoolArgs a) { ssim_pool_body(a.job[blockIdx.y]); }

__global__ void __launch_bounds__(kPoolThreads, 2) k_ssim_pool_multi(const SsimPoolJob* __restrict__ jobs) { ssim_pool_body(jobs[blockIdx.y]); }

static cudaError_t pool_configure()
{
  static std::mutex mu;
  static uint64_t done = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) { return e; }
  const uint64_t bit = 1ULL << (dev & 63);
  std::lock_guard<std::mutex> lk(mu);
  if(done & bit) { return cudaSuccess; }
  e = cudaFuncSetAttribute(k_ssim_pool, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPoolSmem);
  if(e == cudaSuccess) { e = cudaFuncSetAttribute(k_ssim_pool_multi, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPoolSmem); }
  if(e == cudaSuccess) { done |= bit; }
  return e;
}

cudaError_t launch_ssim_pool_multi(const SsimPoolJob* d_jobs, int njobs, int max_ny, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  cudaError_t e = pool_configure();
  if(e != cudaSuccess) { return e; }
  k_ssim_pool_multi<<<dim3((max_ny + kPoolRows - 1) / kPoolRows, njobs), kPoolThreads, kPoolSmem, s>>>(d_jobs);
  return cudaGetLastError();
}

cudaError_t launch_ssim_pool(const SsimPoolArgs& a, cudaStream_t s)
{
  if(a.njobs <= 0) { return cudaSuccess; }
  cudaError_t e = pool_configure();
  if(e != cudaSuccess) { return e; }
  int maxny = 0;
  for(int k = 0; k < a.njobs; k++) { maxny = max(maxny, a.job[k].ny); }
  const dim3 grid((maxny + kPoolRows - 1) / kPoolRows, a.njobs);
  k_ssim_pool<<<grid, kPoolThreads, kPoolSmem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace qmiv
