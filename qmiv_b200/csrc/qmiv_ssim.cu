// Block SSIM (8x8 windows at stride 4, xSSIM.cpp:276-369, xStructSimSTD.cpp:420-461) on B200.
//
// Window moments are sums of 2x2 exact integer 4x4 sub-block moments. They come either from the
// CPS search's epilogue (IV-SSIM: test picture vs its shift-compensated picture, so the SCP never
// needs to be stored) or from k_ssim_moments (plain SSIM, MS-SSIM scales, which also writes the
// next scale's 2x2 mean, xPixelOpsSTD.cpp:50-67). k_ssim_win evaluates every window in FP64 with the
// reference's operation order; k_ssim_rows sums each window row in x order with the compensated sum,
// one lane per row.
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
// windows + ordered row sums (xSSIM.cpp:353-369), two kernels:
//   k_ssim_win   a CTA evaluates a 32 x 32 tile of windows of one job: the tile's 33 x 33 sub-block
//                moments are staged in shared memory, each thread evaluates four windows (FP64, the
//                reference's operation order), and the values are written transposed to the job's
//                scratch [band = y / 32][x][y % 32], so that
//   k_ssim_rows  one warp per band of 32 window rows, lane j walking row j in x order with the
//                compensated sum, reads 256 contiguous bytes per step (a deep register prefetch hides
//                the memory latency of the serial chain).
// All windows are independent work for the first kernel; only the second is order-dependent.
// =============================================================================================
constexpr int kWinT = 32;                                  // windows per tile side
constexpr int kWSub = kWinT + 1;                           // sub-blocks per tile side
constexpr int kWStage = 5 * kWSub * kWSub;
constexpr int kWPer = (kWStage + 255) / 256;

size_t pool_win_elems(int nx, int ny) { return (size_t)((ny + 31) / 32) * 32 * (size_t)nx; }

__device__ __forceinline__ void ssim_win_body(const SsimPoolJob& J, int tile_x, int tile_y)
{
  __shared__ uint32_t st[5][kWSub][kWSub];
  __shared__ double vals[kWinT][kWinT + 1];               // [x][y]
  const int i0 = tile_x * kWinT, j0 = tile_y * kWinT;
  if(i0 >= J.nx || j0 >= J.ny) { return; }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nby = J.ny + 1, nbx = J.nx + 1;
  #pragma unroll
  for(int r = 0; r < kWPer; r++)
  {
    const int e = threadIdx.x + 256 * r;
    if(e < kWStage)
    {
      const int m = e / (kWSub * kWSub), rem = e - m * (kWSub * kWSub);
      const int sy = rem / kWSub, sx = rem - sy * kWSub;
      const int gy = j0 + sy, gx = i0 + sx;
      st[m][sy][sx] = (gy < nby && gx < nbx) ? __ldg(J.mom + (size_t)m * J.plane + (size_t)gy * J.pitch + gx) : 0u;
    }
  }
  __syncthreads();
  #pragma unroll
  for(int q = 0; q < kWinT / 8; q++)
  {
    const int jj = warp + 8 * q, i = i0 + lane, j = j0 + jj;
    double v = 0.0;
    if(i < J.nx && j < J.ny)
    {
      uint64_t sm[5];
      #pragma unroll
      for(int m = 0; m < 5; m++)
      {
        sm[m] = (uint64_t)st[m][jj][lane] + st[m][jj][lane + 1] + st[m][jj + 1][lane] + st[m][jj + 1][lane + 1];
      }
      // moment 0/2 = "Tst" picture, 1/3 = "Ref" picture
      v = ssim_window(sm[1], sm[0], sm[3], sm[2], sm[4], J.C1, J.C2, J.calc_l != 0);
    }
    vals[lane][jj] = v;
  }
  __syncthreads();
  double* out = J.win + ((size_t)tile_y * J.nx + i0) * 32;
  #pragma unroll
  for(int q = 0; q < kWinT / 8; q++)
  {
    const int ii = warp + 8 * q;
    if(i0 + ii < J.nx) { out[(size_t)ii * 32 + lane] = vals[ii][lane]; }
  }
}

__device__ __forceinline__ void ssim_rows_body(const SsimPoolJob& J, int band)
{
  constexpr int U = 16;
  const int lane = threadIdx.x & 31;
  if(band * 32 >= J.ny) { return; }
  const double* p = J.win + (size_t)band * J.nx * 32 + lane;
  const int nx = J.nx;
  Kbns row;
  double cur[U], nxt[U];
  #pragma unroll
  for(int u = 0; u < U; u++) { cur[u] = u < nx ? __ldg(p + (size_t)u * 32) : 0.0; }
  for(int i0 = 0; i0 < nx; i0 += U)
  {
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int i = i0 + U + u;
      nxt[u] = i < nx ? __ldg(p + (size_t)i * 32) : 0.0;
    }
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      if(i0 + u < nx) { row.add(cur[u]); }
    }
    #pragma unroll
    for(int u = 0; u < U; u++) { cur[u] = nxt[u]; }
  }
  const int j = band * 32 + lane;
  if(j < J.ny) { J.row_sum[j] = row.result(); }
}

__global__ void __launch_bounds__(256) k_ssim_win(const __grid_constant__ SsimPoolArgs a)
{
  ssim_win_body(a.job[blockIdx.z], blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(256) k_ssim_win_multi(const SsimPoolJob* __restrict__ jobs)
{
  ssim_win_body(jobs[blockIdx.z], blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(128) k_ssim_rows(const __grid_constant__ SsimPoolArgs a)
{
  ssim_rows_body(a.job[blockIdx.y], blockIdx.x * 4 + (threadIdx.x >> 5));
}
__global__ void __launch_bounds__(128) k_ssim_rows_multi(const SsimPoolJob* __restrict__ jobs)
{
  ssim_rows_body(jobs[blockIdx.y], blockIdx.x * 4 + (threadIdx.x >> 5));
}

cudaError_t launch_ssim_pool_multi(const SsimPoolJob* d_jobs, int njobs, int max_nx, int max_ny, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  k_ssim_win_multi<<<dim3((max_nx + kWinT - 1) / kWinT, (max_ny + kWinT - 1) / kWinT, njobs), 256, 0, s>>>(d_jobs);
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) { return e; }
  const int bands = (max_ny + 31) / 32;
  k_ssim_rows_multi<<<dim3((bands + 3) / 4, njobs), 128, 0, s>>>(d_jobs);
  return cudaGetLastError();
}

cudaError_t launch_ssim_pool(const SsimPoolArgs& a, cudaStream_t s)
{
  if(a.njobs <= 0) { return cudaSuccess; }
  int maxnx = 0, maxny = 0;
  for(int k = 0; k < a.njobs; k++) { maxnx = max(maxnx, a.job[k].nx); maxny = max(maxny, a.job[k].ny); }
  k_ssim_win<<<dim3((maxnx + kWinT - 1) / kWinT, (maxny + kWinT - 1) / kWinT, a.njobs), 256, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) { return e; }
  const int bands = (maxny + 31) / 32;
  k_ssim_rows<<<dim3((bands + 3) / 4, a.njobs), 128, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace qmiv
