// Block SSIM (8x8 windows at stride 4, xSSIM.cpp:276-369, xStructSimSTD.cpp:420-461) on B200.
//
// Window moments are sums of 2x2 exact integer 4x4 sub-block moments. They come either from the
// CPS search's epilogue (IV-SSIM: test picture vs its shift-compensated picture, so the SCP never
// needs to be stored) or from k_ssim_moments (plain SSIM, MS-SSIM scales, which also writes the
// next scale's 2x2 mean, xPixelOpsSTD.cpp:50-67). k_ssim_win evaluates every window in FP64 with the
// reference's operation order; k_ssim_rows sums each window row in x order with the compensated sum,
// one lane per row.
#include "qmiv_kernels.cuh"

#include <type_traits>

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
//   k_ssim_win   a CTA (four warps) evaluates the windows [x0, x0 + 64) of one band of 32 window rows.
//                The 33 block rows x 68 columns of the five moment planes it needs (45 KB) are staged
//                in shared memory by cp.async, all in flight at once. Lane l then takes columns
//                x0 + l and x0 + 32 + l and walks its warp's 8 window rows: block row r gives the
//                horizontal pair sums h(r) = m(r, x) + m(r, x + 1), window (x, r - 1) is h(r - 1) + h(r).
//                Each window is evaluated in FP64 with the reference's operation order; the 64 x 32
//                values reuse the staging space and leave as 16 contiguous KB of the job's scratch
//                [band][x][32].
//   k_ssim_rows  one warp per band, lane j summing window row 32 band + j in x order with the
//                compensated sum. 8 KB chunks of 32 columns are staged in shared memory by cp.async,
//                three in flight per warp, so the serial chain never waits for DRAM.
// All windows are independent work for the first kernel; only the second is order-dependent.
// =============================================================================================
constexpr int kWinX = 64;                                  // windows per CTA in x
constexpr int kWinRows = 8;                                // window rows per warp
constexpr int kStRows = 33;                                // block rows of a band
constexpr int kStCols = 68;                                // block columns staged (65 used), 16-byte pieces
constexpr int kStPieces = kStCols / 4;
constexpr int kRowCols = 32;                               // columns per staged chunk of k_ssim_rows
constexpr int kRowStages = 4;
static_assert(kWinX * 33 * sizeof(double) <= 5 * kStRows * kStCols * sizeof(uint32_t), "values fit the staging space");

size_t pool_win_elems(int nx, int ny) { return (size_t)((ny + 31) / 32) * 32 * (size_t)nx; }

bool pool_job_aligned(const SsimPoolJob& J)
{
  return ((uintptr_t)J.mom & 15) == 0 && (J.pitch & 3) == 0 && (J.plane & 3) == 0 && ((uintptr_t)J.win & 15) == 0;
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((uint32_t)__cvta_generic_to_shared(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// v / 64 for an integer v < 2^52, exactly: 2^46 + v 2^-6 is the double whose mantissa field is v
// and whose exponent is 46, and removing 2^46 is exact. Equals (double)v * (1.0 / 64).
template <typename S>
__device__ __forceinline__ double div64_exact(S v)
{
  const uint32_t hi = 0x42D00000u | (uint32_t)((uint64_t)v >> 32);
  return dsub(__hiloint2double((int)hi, (int)(uint32_t)v), 70368744177664.0);
}

// The 16 windows of one thread: columns x0 + l and x0 + 32 + l, the warp's 8 rows.
// The fields of a pool job one CTA of k_ssim_win uses, read once into registers.
struct WinJob
{
  double C1, C2;
  int    nx, ny, calc_l;
};

template <bool WIDE>
__device__ __forceinline__ void ssim_win_eval(const WinJob& J, const uint32_t (*st)[kStRows][kStCols], int x0, int band,
                                              double v[2][kWinRows])
{
  using S = typename std::conditional<WIDE, uint64_t, uint32_t>::type;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int r0 = warp * kWinRows;                           // the warp's first block row in the band
  const int nrow = min(kWinRows, J.ny - band * 32 - r0);    // window rows of this warp (may be <= 0)
  #pragma unroll
  for(int h = 0; h < 2; h++)
  {
    const int xl = 32 * h + lane;
    const bool xin = x0 + xl < J.nx;
    S hp[5] = { 0, 0, 0, 0, 0 };
    #pragma unroll
    for(int k = 0; k <= kWinRows; k++)
    {
      const bool live = xin && k <= nrow;                   // block row r0 + k was staged
      S hc[5];
      #pragma unroll
      for(int m = 0; m < 5; m++) { hc[m] = live ? (S)st[m][r0 + k][xl] + (S)st[m][r0 + k][xl + 1] : (S)0; }
      if(k > 0)
      {
        double r = 0.0;
        if(live)
        {
          // moment 0/2 = "Tst" picture, 1/3 = "Ref" picture (xStructSimSTD.cpp:420-461)
          const double at = div64_exact<S>(hp[0] + hc[0]), ar = div64_exact<S>(hp[1] + hc[1]);
          const double qt = div64_exact<S>(hp[2] + hc[2]), qr = div64_exact<S>(hp[3] + hc[3]);
          const double qrt = div64_exact<S>(hp[4] + hc[4]);
          r = ssim_window_avg(ar, at, qr, qt, qrt, J.C1, J.C2, J.calc_l != 0);
        }
        v[h][k - 1] = r;
      }
      #pragma unroll
      for(int m = 0; m < 5; m++) { hp[m] = hc[m]; }
    }
  }
}

__device__ __forceinline__ void ssim_win_body(const SsimPoolJob& Jg, int tile_x, int band)
{
  __shared__ __align__(16) uint32_t st[5][kStRows][kStCols];
  const WinJob J{ Jg.C1, Jg.C2, Jg.nx, Jg.ny, Jg.calc_l };
  const int x0 = tile_x * kWinX, j0 = band * 32;
  if(x0 >= J.nx || j0 >= J.ny) { return; }                 // uniform over the CTA
  const uint32_t* mom = Jg.mom;
  const size_t plane = Jg.plane;
  const int pitch = Jg.pitch;
  // block rows j0 .. min(j0 + 32, ny) exist (ny + 1 block rows); 16-byte pieces that start inside
  // the padded row (pitch, a multiple of 4 columns) end inside it. Piece q = (m, r, c) walks in steps
  // of 128 = 7 rows + 9 pieces.
  static_assert(128 == 7 * kStPieces + 9, "piece walk");
  const int nrows = min(kStRows, J.ny + 1 - j0);
  int m = 0, r = threadIdx.x / kStPieces, c = threadIdx.x - r * kStPieces;
  for(int q = threadIdx.x; q < 5 * kStRows * kStPieces; q += 128)
  {
    if(r < nrows && x0 + 4 * c < pitch)
    {
      cp_async16(&st[m][r][4 * c], mom + (size_t)m * plane + (size_t)(j0 + r) * pitch + x0 + 4 * c);
    }
    r += 7; c += 9;
    if(c >= kStPieces) { c -= kStPieces; r++; }
    if(r >= kStRows) { r -= kStRows; m++; }
  }
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  double v[2][kWinRows];
  if(Jg.wide) { ssim_win_eval<true>(J, st, x0, band, v); }
  else { ssim_win_eval<false>(J, st, x0, band, v); }
  __syncthreads();                                          // the staging space becomes the values
  double (*vals)[33] = reinterpret_cast<double (*)[33]>(&st[0][0][0]);   // [x][row in band]
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  #pragma unroll
  for(int h = 0; h < 2; h++)
  {
    #pragma unroll
    for(int k = 0; k < kWinRows; k++) { vals[32 * h + lane][warp * kWinRows + k] = v[h][k]; }
  }
  __syncthreads();
  const int n = min(kWinX, J.nx - x0) * 32;
  double* out = Jg.win + ((size_t)band * J.nx + x0) * 32;   // this tile's columns are contiguous
  for(int e = threadIdx.x; e < n; e += 128) { out[e] = vals[e >> 5][e & 31]; }
}

__device__ __forceinline__ void ssim_rows_body(const SsimPoolJob& J, int band)
{
  __shared__ __align__(16) double st[kRowStages][kRowCols][32];   // [stage][column][row in band]
  const int lane = threadIdx.x & 31;
  if(band * 32 >= J.ny) { return; }                         // one warp per CTA: uniform
  const char* src = reinterpret_cast<const char*>(J.win + (size_t)band * J.nx * 32);
  const int nchunks = (J.nx + kRowCols - 1) / kRowCols;
  // chunk c: columns [32 c, min(32 c + 32, nx)), 256 bytes each, contiguous in the scratch
  auto issue = [&](int c) {
    if(c < nchunks)
    {
      const int pieces = min(kRowCols, J.nx - c * kRowCols) * 16;
      char* dst = reinterpret_cast<char*>(st[c % kRowStages]);
      const char* s = src + (size_t)c * kRowCols * 256;
      for(int q = lane; q < pieces; q += 32) { cp_async16(dst + 16 * q, s + 16 * q); }
    }
    cp_async_commit();                                      // empty groups keep the count uniform
  };
  #pragma unroll
  for(int c = 0; c < kRowStages - 1; c++) { issue(c); }
  Kbns row;
  for(int c = 0; c < nchunks; c++)
  {
    cp_async_wait<kRowStages - 2>();                        // chunk c has landed (this lane's part)
    __syncwarp();                                           // ... and every other lane's
    const int cols = min(kRowCols, J.nx - c * kRowCols);
    const double (*b)[32] = st[c % kRowStages];
    if(cols == kRowCols)
    {
      // straight-line code: the loads and the non-carried parts of the sums overlap the chain
      #pragma unroll
      for(int x = 0; x < kRowCols; x++) { row.add(b[x][lane]); }
    }
    else
    {
      #pragma unroll 1
      for(int x = 0; x < cols; x++) { row.add(b[x][lane]); }
    }
    __syncwarp();                                           // every lane is past its reads of chunk c - 1
    issue(c + kRowStages - 1);                              // into the stage that chunk c - 1 used
  }
  const int j = band * 32 + lane;
  if(j < J.ny) { J.row_sum[j] = row.result(); }
}

__global__ void __launch_bounds__(128) k_ssim_win(const __grid_constant__ SsimPoolArgs a)
{
  ssim_win_body(a.job[blockIdx.z], blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(128) k_ssim_win_multi(const SsimPoolJob* __restrict__ jobs)
{
  ssim_win_body(jobs[blockIdx.z], blockIdx.x, blockIdx.y);
}
__global__ void __launch_bounds__(32) k_ssim_rows(const __grid_constant__ SsimPoolArgs a)
{
  ssim_rows_body(a.job[blockIdx.y], blockIdx.x);
}
__global__ void __launch_bounds__(32) k_ssim_rows_multi(const SsimPoolJob* __restrict__ jobs)
{
  ssim_rows_body(jobs[blockIdx.y], blockIdx.x);
}

cudaError_t launch_ssim_pool_multi(const SsimPoolJob* d_jobs, int njobs, int max_nx, int max_ny, cudaStream_t s)
{
  if(njobs <= 0) { return cudaSuccess; }
  const int bands = (max_ny + 31) / 32;
  k_ssim_win_multi<<<dim3((max_nx + kWinX - 1) / kWinX, bands, njobs), 128, 0, s>>>(d_jobs);
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) { return e; }
  k_ssim_rows_multi<<<dim3(bands, njobs), 32, 0, s>>>(d_jobs);
  return cudaGetLastError();
}

cudaError_t launch_ssim_rows(const SsimPoolArgs& a, cudaStream_t s)
{
  if(a.njobs <= 0) { return cudaSuccess; }
  int maxny = 0;
  for(int k = 0; k < a.njobs; k++)
  {
    if(((uintptr_t)a.job[k].win & 15) != 0) { return cudaErrorMisalignedAddress; }
    maxny = max(maxny, a.job[k].ny);
  }
  k_ssim_rows<<<dim3((maxny + 31) / 32, a.njobs), 32, 0, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_ssim_pool(const SsimPoolArgs& a, cudaStream_t s)
{
  if(a.njobs <= 0) { return cudaSuccess; }
  int maxnx = 0, maxny = 0;
  for(int k = 0; k < a.njobs; k++)
  {
    if(!pool_job_aligned(a.job[k])) { return cudaErrorMisalignedAddress; }
    maxnx = max(maxnx, a.job[k].nx); maxny = max(maxny, a.job[k].ny);
  }
  const int bands = (maxny + 31) / 32;
  k_ssim_win<<<dim3((maxnx + kWinX - 1) / kWinX, bands, a.njobs), 128, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if(e != cudaSuccess) { return e; }
  k_ssim_rows<<<dim3(bands, a.njobs), 32, 0, s>>>(a);
  return cudaGetLastError();
}

}  // namespace qmiv
