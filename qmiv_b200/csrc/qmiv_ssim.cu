// Block SSIM (8x8 windows at stride 4, xSSIM.cpp:276-369, xStructSimSTD.cpp:420-461) on B200.
//
// Window moments are sums of 2x2 exact integer 4x4 sub-block moments. They come either from the
// CPS search's epilogue (IV-SSIM: test picture vs its shift-compensated picture, so the SCP never
// needs to be stored) or from k_ssim_moments (plain SSIM, MS-SSIM scales, which also writes the
// next scale's 2x2 mean, xPixelOpsSTD.cpp:50-67). k_ssim_pool evaluates every window in FP64 with the
// reference's operation order and sums each window row in x order with the compensated sum, one
// lane per row, from shared memory.
#include "qmiv_kernels.cuh"

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
// windows + ordered row sums. A CTA owns kBandJ window rows of one job and walks the row in chunks
// of 32 windows: the chunk's (kBandJ+1) x 33 sub-block moments are staged in shared memory (the
// next chunk's global loads are issued before the current chunk is evaluated), every thread
// evaluates one window, and lane j of warp 0 adds the chunk's 32 values of row j in x order.
// =============================================================================================
constexpr int kBandJ = 8;                       // window rows per CTA
constexpr int kChunkI = 32;                     // windows per chunk
constexpr int kSubR = kBandJ + 1, kSubC = kChunkI + 1;
constexpr int kStageN = 5 * kSubR * kSubC;      // staged moment values per chunk
constexpr int kStagePerThread = (kStageN + 255) / 256;

__device__ __forceinline__ void ssim_pool_body(const SsimPoolJob& J)
{
  __shared__ uint32_t st[2][5][kSubR][kSubC];
  __shared__ double vals[kBandJ][kChunkI + 1];
  const int j0 = blockIdx.x * kBandJ;
  if(j0 >= J.ny) { return; }
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int nchunks = (J.nx + kChunkI - 1) / kChunkI;
  const int nby = J.ny + 1, nbx = J.nx + 1;  // sub-blocks any window of this job touches

  uint32_t reg[kStagePerThread];
  auto load = [&](int k) {
    #pragma unroll
    for(int r = 0; r < kStagePerThread; r++)
    {
      const int e = threadIdx.x + 256 * r;
      uint32_t v = 0;
      if(e < kStageN)
      {
        const int m = e / (kSubR * kSubC), rem = e - m * (kSubR * kSubC);
        const int sy = rem / kSubC, sx = rem - sy * kSubC;
        const int gy = j0 + sy, gx = k * kChunkI + sx;
        if(gy < nby && gx < nbx) { v = __ldg(J.mom + (size_t)m * J.plane + (size_t)gy * J.pitch + gx); }
      }
      reg[r] = v;
    }
  };
  auto store = [&](int buf) {
    #pragma unroll
    for(int r = 0; r < kStagePerThread; r++)
    {
      const int e = threadIdx.x + 256 * r;
      if(e < kStageN) { (&st[buf][0][0][0])[e] = reg[r]; }
    }
  };

  Kbns row;
  load(0);
  store(0);
  __syncthreads();
  for(int k = 0; k < nchunks; k++)
  {
    const int buf = k & 1;
    if(k + 1 < nchunks) { load(k + 1); }
    {
      const int i = k * kChunkI + tx, j = j0 + ty;
      double v = 0.0;
      if(i < J.nx && j < J.ny)
      {
        uint64_t sm[5];
        #pragma unroll
        for(int m = 0; m < 5; m++)
        {
          sm[m] = (uint64_t)st[buf][m][ty][tx] + st[buf][m][ty][tx + 1] + st[buf][m][ty + 1][tx] + st[buf][m][ty + 1][tx + 1];
        }
        // moment 0/2 = "Tst" picture, 1/3 = "Ref" picture
        v = ssim_window(sm[1], sm[0], sm[3], sm[2], sm[4], J.C1, J.C2, J.calc_l != 0);
      }
      vals[ty][tx] = v;
    }
    __syncthreads();
    if(ty == 0 && tx < kBandJ && j0 + tx < J.ny)
    {
      const int cnt = min(kChunkI, J.nx - k * kChunkI);
      for(int u = 0; u < cnt; u++) { row.add(vals[tx][u]); }
    }
    if(k + 1 < nchunks) { store(buf ^ 1); }
    __syncthreads();
  }
  if(ty == 0 && tx < kBandJ && j0 + tx < J.ny) { J.row_sum[j0 + tx] = row.result(); }
}

__global__ void __launch_bounds__(256) k_ssim_pool(const __grid_constant__ SsimPoolArgs a) { ssim_pool_body(a.job[blockIdx.y]); }

__global__ void __launch_bounds__(256) k_ssim_pool_multi(const SsimPoolJob* __restrict__ jobs) { ssim_pool_body(jobs[blockIdx.y]); }

cudaError_t launch_ssim_pool_multi(const SsimPoolJob* d_jobs, int njobs, int max_ny, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  k_ssim_pool_multi<<<dim3((max_ny + kBandJ - 1) / kBandJ, njobs), 256, 0, s>>>(d_jobs);
  return cudaGetLastError();
}

cudaError_t launch_ssim_pool(const SsimPoolArgs& a, cudaStream_t s)
{
  if(a.njobs <= 0) { return cudaSuccess; }
  int maxny = 0;
  for(int k = 0; k < a.njobs; k++) { maxny = max(maxny, a.job[k].ny); }
  const dim3 grid((maxny + kBandJ - 1) / kBandJ, a.njobs);
  k_ssim_pool<<<grid, 256, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace qmiv
