// Structural similarity under every window option of the reference (xSSIM::setStructSimParams,
// libs/pmbb-ivqm/src/xSSIM.cpp:86-113; the app's -ssm / -ssb / -ssw / -sss, apps/QMIV/src/xAppQMIV.cpp:99-104):
//   regular 11x11 windows centred on (x, y), x, y in [5, W - 5) without a border mode or [0, W) with one
//   (xSSIM.cpp:161-196), whose reads beyond the picture see the margin extension (libs/pmbb-core/src/
//   xMarginOps.h:16-20: Nearest, Reflect, Mirror, Constant 65535 as xPicP::extend passes it, Zero):
//     Gaussian float   (xStructSimSTD.cpp:19-88)  five double sums in dy, dx order of value x coefficient,
//                      each product and sum rounded separately
//     Gaussian integer (xStructSimSTD.cpp:89-154) exact integer sums of value x integer coefficient, x 2^-18
//     averaged         (xStructSimSTD.cpp:155-193, AVX CalcBlckAvg11) exact integer sums x (1 / 121)
//   block N x N windows with their top-left sample at (x, y), x in [0, W - N] (xSSIM.cpp:182-195):
//     Gaussian integer 8 / 16 (xStructSimSTD.cpp:353-419), averaged 8 / 16 / 32 (:420-461) x (1 / N^2)
// Integer sums stay below 2^53 for 16-bit samples (65535^2 * 2^18 < 2^51), so they are formed exactly in
// double with fused multiply-adds in any order; the float Gaussian sums keep the reference's order and
// roundings (separate multiply and add). The window formula uses separately rounded operations in the
// reference's order, so every window value equals the portable reference's bit for bit.
//
// Three window kernels, all staging the samples a CTA's windows read in shared memory, both pictures
// packed (a | b << 16) after clipping and margin extension:
//   k_ssim_gen_rows (strides 1, 2, 4): each lane evaluates K neighbouring windows of a window row and
//     walks that row's input rows; a sample loaded once feeds every window that covers it.
//   k_ssim_box (averaged windows at strides 1, 2, 4): running column sums and box sums of the exact
//     integer moments.
//   k_ssim_gen (other strides): one window per thread.
// Window values go to the band-transposed scratch [ny / 32][nx][32] that k_ssim_rows (qmiv_ssim.cu)
// sums in x order, one lane per window row.
#include "qmiv_host.h"

#include <cmath>
#include <mutex>

namespace qmiv {

namespace {

enum { kGenFlt = 0, kGenInt = 1, kGenAvg = 2 };

// window coefficients, row-major dy * N + dx
constexpr int kCoefFlt11 = 0, kCoefInt11 = 121, kCoefInt8 = 242, kCoefInt16 = 306, kCoefTotal = 562;
__constant__ double c_gen_coef[kCoefTotal];

// Integer Gaussian windows (xStructSimConsts.h:111-124 for 11x11, :145-173 for 8x8 and 16x16), each the
// mirror image of its top-left quadrant in both directions. These integers define the reference's
// metric, so they are kept as they are. The 11x11 quadrant is not symmetric about its diagonal.
const int32_t kGq11[6][6] = {
  { 0, 2, 10, 29, 57, 72 },           { 2, 15, 72, 218, 424, 530 },          { 10, 72, 340, 1032, 2010, 2510 },
  { 29, 218, 1032, 3135, 6107, 7626 }, { 57, 424, 2010, 6107, 11894, 14854 }, { 72, 530, 2510, 7626, 14855, 18550 },
};
const int32_t kGq8[4][4] = {
  { 81, 308, 749, 1168 }, { 308, 1168, 2842, 4432 }, { 749, 2842, 6913, 10781 }, { 1168, 4432, 10781, 16814 },
};
const int32_t kGq16[8][8] = {
  { 0, 1, 4, 10, 19, 32, 45, 54 },                 { 1, 5, 13, 32, 64, 108, 152, 181 },
  { 4, 13, 38, 91, 181, 305, 432, 514 },           { 10, 32, 91, 216, 432, 727, 1029, 1224 },
  { 19, 64, 181, 432, 865, 1456, 2061, 2451 },     { 32, 108, 305, 727, 1456, 2451, 3469, 4126 },
  { 45, 152, 432, 1029, 2061, 3469, 4909, 5839 },  { 54, 181, 514, 1224, 2451, 4126, 5839, 6947 },
};

int32_t gauss_int(int N, int y, int x)
{
  const int qy = y < N - 1 - y ? y : N - 1 - y, qx = x < N - 1 - x ? x : N - 1 - x;
  return N == 11 ? kGq11[qy][qx] : N == 8 ? kGq8[qy][qx] : kGq16[qy][qx];
}

// The float Gaussian (c_FilterRglrGaussFlt32, xStructSimConsts.h:55-68) is the 11x11 Gaussian of sigma
// 1.5 normalised to unit sum and rounded to float.
void build_coefs(double* c)
{
  double g[11][11], sum = 0.0;
  for(int y = 0; y < 11; y++)
  {
    for(int x = 0; x < 11; x++) { g[y][x] = std::exp(-(double)((x - 5) * (x - 5) + (y - 5) * (y - 5)) / 4.5); sum += g[y][x]; }
  }
  for(int y = 0; y < 11; y++) { for(int x = 0; x < 11; x++) { c[kCoefFlt11 + 11 * y + x] = (double)(float)(g[y][x] / sum); } }
  for(int y = 0; y < 11; y++) { for(int x = 0; x < 11; x++) { c[kCoefInt11 + 11 * y + x] = gauss_int(11, y, x); } }
  for(int y = 0; y < 8; y++) { for(int x = 0; x < 8; x++) { c[kCoefInt8 + 8 * y + x] = gauss_int(8, y, x); } }
  for(int y = 0; y < 16; y++) { for(int x = 0; x < 16; x++) { c[kCoefInt16 + 16 * y + x] = gauss_int(16, y, x); } }
}

// exact double of a 16-bit integer: 2^52 + v has a unit ulp
__device__ __forceinline__ double u16_to_f64(uint32_t v) { return dsub(__hiloint2double(0x43300000, (int)v), 4503599627370496.0); }

// position of sample i of a length-n line after margin extension; in = false for the constant modes
__device__ __forceinline__ int brd_map(int i, int n, int border, bool& in)
{
  in = true;
  if(i >= 0 && i < n) { return i; }
  int j;
  switch(border)
  {
  case QMIV_BRD_REFLECT: j = i < 0 ? -1 - i : 2 * n - 1 - i; break;   // ( c b a | a b c d | d c b )
  case QMIV_BRD_MIRROR:  j = i < 0 ? -i : 2 * n - 2 - i; break;       // ( d c b | a b c d | c b a )
  case QMIV_BRD_CONSTANT:
  case QMIV_BRD_ZERO:    in = false; return 0;
  default:               j = i;                                        // Nearest; None reads only unused tile parts
  }
  return min(max(j, 0), n - 1);
}

}  // namespace

// Stages rows r0, r0 + rstep, ... < th of the tile: tile column col holds input column X0 + col of both
// pictures (a | b << 16), after conceal clipping and margin extension; idx(col) is its word in the row.
// Rows read through row pointers; columns map through the margin only where the tile crosses the
// picture's left or right edge.
template <typename IDX>
__device__ __forceinline__ void stage_tile(const SsimGenJob& J, int border, int X0, int Y0, int tw, int th, int r0, int rstep,
                                           int lane, uint32_t* tile, int pitch, IDX idx)
{
  const int c = J.comp;
  const bool x_inside = X0 >= 0 && X0 + tw <= J.W;
  const uint32_t fill = border == QMIV_BRD_CONSTANT ? 0xffffu : 0u;
  const int sxa = J.a.sx[c], sxb = J.b.sx[c];
  for(int r = r0; r < th; r += rstep)
  {
    bool yin;
    const int yi = brd_map(Y0 + r, J.H, border, yin);
    uint32_t* dst = tile + (size_t)r * pitch;
    const size_t oa = (size_t)(yi >> J.a.sy[c]) * J.a.pitch[c], ob = (size_t)(yi >> J.b.sy[c]) * J.b.pitch[c];
    for(int col = lane; col < tw; col += 32)
    {
      bool xin = true;
      const int xi = x_inside ? X0 + col : brd_map(X0 + col, J.W, border, xin);
      uint32_t va = fill, vb = fill;   // the margin constant is not clipped
      if(xin && yin)
      {
        if(J.esz == 1)
        {
          va = __ldg(static_cast<const uint8_t*>(J.a.p[c]) + oa + (xi >> sxa));
          vb = __ldg(static_cast<const uint8_t*>(J.b.p[c]) + ob + (xi >> sxb));
        }
        else
        {
          va = __ldg(static_cast<const uint16_t*>(J.a.p[c]) + oa + (xi >> sxa));
          vb = __ldg(static_cast<const uint16_t*>(J.b.p[c]) + ob + (xi >> sxb));
        }
        va = min(va, J.clip); vb = min(vb, J.clip);
      }
      dst[idx(col)] = va | (vb << 16);
    }
  }
}

// ---------------------------------------------------------------------------------------------
// window kernel
// ---------------------------------------------------------------------------------------------
template <int MODE, int N>
__device__ __forceinline__ double gen_window(const double (&m)[5], double inv, double C1, double C2, bool calc_l)
{
  // m: sums of R, T, R^2, T^2, R*T (R = "Ref" = b, T = "Tst" = a)
  double ar, at, var_r, var_t, cov;
  if(MODE == kGenFlt)                                         // xStructSimSTD.cpp:41-45
  {
    ar = m[0]; at = m[1];
    var_r = dsub(m[2], dmul(ar, ar));
    var_t = dsub(m[3], dmul(at, at));
    cov   = dsub(m[4], dmul(ar, at));
  }
  else                                                        // xStructSimSTD.cpp:110-114, :171-175
  {
    ar = dmul(m[0], inv); at = dmul(m[1], inv);
    var_r = dsub(dmul(m[2], inv), dmul(ar, ar));
    var_t = dsub(dmul(m[3], inv), dmul(at, at));
    cov   = dsub(dmul(m[4], inv), dmul(ar, at));
  }
  // 2 x is formed as x + x, which is the same double
  const double cs = ddiv(dadd(dadd(cov, cov), C2), dadd(dadd(var_r, var_t), C2));
  if(!calc_l) { return cs; }
  const double l = ddiv(dadd(dmul(dadd(ar, ar), at), C1), dadd(dadd(dmul(ar, ar), dmul(at, at)), C1));
  return dmul(l, cs);
}

// One window per thread (K = 1) for strides other than 1, 2 and 4: lane l of warp w evaluates window
// column x0 + l of window row y0 + w. With stride S > 1 the tile's columns are stored by phase (column c
// at (c % S) * cw + c / S), so the 32 lanes of a warp read 32 consecutive words.
template <int MODE, int N, int K>
__global__ void __launch_bounds__(128) k_ssim_gen(const __grid_constant__ SsimGenArgs a)
{
  extern __shared__ uint32_t tile[];                          // [th][S * cw], sample a | b << 16
  const SsimGenJob& J = a.job[blockIdx.z];
  const int S = a.S, WY = blockDim.y, lane = threadIdx.x, w = threadIdx.y;
  const int wx0 = blockIdx.x * 32, wy0 = blockIdx.y * WY * K;
  if(wx0 >= J.nx || wy0 >= J.ny) { return; }                 // uniform over the CTA
  const int pitch = S * a.cw;
  // staged part: the columns and rows the CTA's existing windows read
  const int tw = (min(32, J.nx - wx0) - 1) * S + N;
  const int th = (min(WY * K, J.ny - wy0) - 1) * S + N;
  const int X0 = J.x0 + wx0 * S, Y0 = J.y0 + wy0 * S;
  stage_tile(J, a.border, X0, Y0, tw, th, w, WY, lane, tile, pitch, [S, cw = a.cw](int col) { const int q = col / S; return (col - q * S) * cw + q; });
  __syncthreads();

  int co[N];                                                  // tile column of tap dx for this lane
  #pragma unroll
  for(int dx = 0; dx < N; dx++) { const int q = dx / S; co[dx] = (dx - q * S) * a.cw + q + lane; }
  double acc[K][5];
  #pragma unroll
  for(int k = 0; k < K; k++)
  {
    #pragma unroll
    for(int m = 0; m < 5; m++) { acc[k][m] = 0.0; }
  }
  const uint32_t* rowp = tile + (size_t)(w * K * S) * pitch;
  const int nr = (K - 1) * S + N;                             // input rows of the thread's K windows
  #pragma unroll 1
  for(int r = 0; r < nr; r++, rowp += pitch)
  {
    // window k takes this input row as its row dy = r - k S (rows in order, so each window's
    // contributions arrive in dy-major, dx-minor order)
    unsigned valid = 0;
    int crow[K];
    #pragma unroll
    for(int k = 0; k < K; k++)
    {
      const int dy = r - k * S;
      if(dy >= 0 && dy < N) { valid |= 1u << k; }
      crow[k] = a.coef + min(max(dy, 0), N - 1) * N;       // in range also where unused
    }
    #pragma unroll
    for(int dx = 0; dx < N; dx++)
    {
      const uint32_t v = rowp[co[dx]];
      const double T = u16_to_f64(v & 0xffffu), R = u16_to_f64(v >> 16);
      const double RR = dmul(R, R), TT = dmul(T, T), RT = dmul(R, T);   // exact (< 2^32)
      #pragma unroll
      for(int k = 0; k < K; k++)
      {
        if(!(valid & (1u << k))) { continue; }
        if(MODE == kGenAvg)
        {
          acc[k][0] = dadd(acc[k][0], R); acc[k][1] = dadd(acc[k][1], T);
          acc[k][2] = dadd(acc[k][2], RR); acc[k][3] = dadd(acc[k][3], TT); acc[k][4] = dadd(acc[k][4], RT);
        }
        else
        {
          const double C = c_gen_coef[crow[k] + dx];
          if(MODE == kGenFlt)                                 // SumR += R * C, ... (xStructSimSTD.cpp:34-38)
          {
            acc[k][0] = dadd(acc[k][0], dmul(R, C)); acc[k][1] = dadd(acc[k][1], dmul(T, C));
            acc[k][2] = dadd(acc[k][2], dmul(RR, C)); acc[k][3] = dadd(acc[k][3], dmul(TT, C));
            acc[k][4] = dadd(acc[k][4], dmul(RT, C));
          }
          else                                                // exact integers
          {
            acc[k][0] = __fma_rn(R, C, acc[k][0]); acc[k][1] = __fma_rn(T, C, acc[k][1]);
            acc[k][2] = __fma_rn(RR, C, acc[k][2]); acc[k][3] = __fma_rn(TT, C, acc[k][3]);
            acc[k][4] = __fma_rn(RT, C, acc[k][4]);
          }
        }
      }
    }
  }
  const int wx = wx0 + lane;
  if(wx >= J.nx) { return; }
  #pragma unroll
  for(int k = 0; k < K; k++)
  {
    const int wy = wy0 + w * K + k;
    if(wy < J.ny)
    {
      J.win[((size_t)(wy >> 5) * J.nx + wx) * 32 + (wy & 31)] = gen_window<MODE, N>(acc[k], a.inv, J.C1, J.C2, J.calc_l != 0);
    }
  }
}

// Row-walking form for strides 1, 2 and 4 (the original paper's and the app's default stride): lane l of
// warp w evaluates the K windows x0 + l K .. x0 + l K + K - 1 of window rows w, w + 4, ... of the CTA.
// For each window row it walks the N input rows in order; in input row dy, input column j of the lane's
// span (j in [0, (K - 1) S + N)) is loaded and converted once and feeds window k as its tap
// dx = j - k S wherever that lies in [0, N): every (j, k) pair is resolved at compile time, so no
// instruction is spent on a tap a window does not have, and each window still receives its taps in
// dy-major, dx-minor order. The N coefficients of row dy are loaded once per row. The tile's columns are
// stored by phase modulo K S, so the lanes of a warp read consecutive words.
template <int MODE, int N, int K, int S>
__global__ void __launch_bounds__(128) k_ssim_gen_rows(const __grid_constant__ SsimGenArgs a)
{
  constexpr int KS = K * S;
  constexpr int J = (K - 1) * S + N;                          // input columns of one lane's windows
  extern __shared__ uint32_t tile[];                          // [th][KS * cw], sample a | b << 16
  const SsimGenJob& Jb = a.job[blockIdx.z];
  const int lane = threadIdx.x, w = threadIdx.y;
  const int WR = a.wr;                                        // window rows per CTA
  const int wx0 = blockIdx.x * 32 * K, wy0 = blockIdx.y * WR;
  if(wx0 >= Jb.nx || wy0 >= Jb.ny) { return; }
  const int cw = a.cw, pitch = KS * cw;
  const int tw = (min(32 * K, Jb.nx - wx0) - 1) * S + N;
  const int rows = min(WR, Jb.ny - wy0);
  const int th = (rows - 1) * S + N;
  const int X0 = Jb.x0 + wx0 * S, Y0 = Jb.y0 + wy0 * S;
  stage_tile(Jb, a.border, X0, Y0, tw, th, w, blockDim.y, lane, tile, pitch, [cw](int col) { return (col % KS) * cw + col / KS; });
  __syncthreads();

  const int wx = wx0 + lane * K;
  for(int wr = w; wr < rows; wr += blockDim.y)
  {
    double acc[K][5];
    #pragma unroll
    for(int k = 0; k < K; k++)
    {
      #pragma unroll
      for(int m = 0; m < 5; m++) { acc[k][m] = 0.0; }
    }
    const uint32_t* rowp = tile + (size_t)(wr * S) * pitch + lane;
    #pragma unroll 1
    for(int dy = 0; dy < N; dy++, rowp += pitch)
    {
      double C[N];
      if(MODE != kGenAvg)
      {
        #pragma unroll
        for(int dx = 0; dx < N; dx++) { C[dx] = c_gen_coef[a.coef + dy * N + dx]; }
      }
      #pragma unroll
      for(int j = 0; j < J; j++)
      {
        const uint32_t v = rowp[(j % KS) * cw + j / KS];
        const double T = u16_to_f64(v & 0xffffu), R = u16_to_f64(v >> 16);
        const double RR = dmul(R, R), TT = dmul(T, T), RT = dmul(R, T);   // exact (< 2^32)
        #pragma unroll
        for(int k = 0; k < K; k++)
        {
          const int dx = j - k * S;
          if(dx < 0 || dx >= N) { continue; }                 // resolved at compile time
          if(MODE == kGenAvg)
          {
            acc[k][0] = dadd(acc[k][0], R); acc[k][1] = dadd(acc[k][1], T);
            acc[k][2] = dadd(acc[k][2], RR); acc[k][3] = dadd(acc[k][3], TT); acc[k][4] = dadd(acc[k][4], RT);
          }
          else if(MODE == kGenFlt)                            // SumR += R * C, ... (xStructSimSTD.cpp:34-38)
          {
            acc[k][0] = dadd(acc[k][0], dmul(R, C[dx])); acc[k][1] = dadd(acc[k][1], dmul(T, C[dx]));
            acc[k][2] = dadd(acc[k][2], dmul(RR, C[dx])); acc[k][3] = dadd(acc[k][3], dmul(TT, C[dx]));
            acc[k][4] = dadd(acc[k][4], dmul(RT, C[dx]));
          }
          else                                                // exact integers
          {
            acc[k][0] = __fma_rn(R, C[dx], acc[k][0]); acc[k][1] = __fma_rn(T, C[dx], acc[k][1]);
            acc[k][2] = __fma_rn(RR, C[dx], acc[k][2]); acc[k][3] = __fma_rn(TT, C[dx], acc[k][3]);
            acc[k][4] = __fma_rn(RT, C[dx], acc[k][4]);
          }
        }
      }
    }
    const int wy = wy0 + wr;
    double* out = Jb.win + ((size_t)(wy >> 5) * Jb.nx) * 32 + (wy & 31);
    #pragma unroll
    for(int k = 0; k < K; k++)
    {
      if(wx + k < Jb.nx) { out[(size_t)(wx + k) * 32] = gen_window<MODE, N>(acc[k], a.inv, Jb.C1, Jb.C2, Jb.calc_l != 0); }
    }
  }
}

// Averaged windows (regular 11x11 and block 8 / 16 / 32) at strides 1, 2 and 4 by box sums. Their five
// moments are exact integer sums (xStructSimSTD.cpp:155-193, :420-461), so any order of the additions
// gives the same integers and the same window values. A CTA takes 32 window columns x kBoxRows window
// rows: it stages the samples as the tap-by-tap kernels do (margin extension, clipping), then
//   vertical: a thread per input column walks the tile's rows with running sums of the last N rows
//     (the arriving row added, the leaving one subtracted; R, T in 32 bits, R^2, T^2, R T in 64) and
//     stores them for each window row in shared memory, columns by phase modulo S so that the
//     horizontal pass reads consecutive words;
//   horizontal: a thread per window adds the N column sums of its window and evaluates it.
// Per window this is about S^2 row steps and N column additions instead of N^2 taps.
constexpr int kBoxRows = 8;

struct BoxSums
{
  uint32_t r, t;
  uint64_t rr, tt, rt;
};

template <int N, int S>
__global__ void __launch_bounds__(32 * kBoxRows) k_ssim_box(const __grid_constant__ SsimGenArgs a)
{
  extern __shared__ __align__(16) unsigned char box_smem[];
  const SsimGenJob& Jb = a.job[blockIdx.z];
  const int wx0 = blockIdx.x * 32, wy0 = blockIdx.y * kBoxRows;
  if(wx0 >= Jb.nx || wy0 >= Jb.ny) { return; }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int tw = (min(32, Jb.nx - wx0) - 1) * S + N;
  const int rows = min(kBoxRows, Jb.ny - wy0);
  const int th = (rows - 1) * S + N;
  const int cwp = a.cw;                                       // columns per phase: ceil(31 S + N, S)
  uint32_t* tile = reinterpret_cast<uint32_t*>(box_smem);     // [th][tw]
  const size_t tile_words = (size_t)((kBoxRows - 1) * S + N) * (31 * S + N);
  // column sums [window row][S * cwp], one array per moment
  uint64_t* c_rr = reinterpret_cast<uint64_t*>(box_smem + ((tile_words * 4 + 15) & ~(size_t)15));
  uint64_t* c_tt = c_rr + kBoxRows * S * cwp;
  uint64_t* c_rt = c_tt + kBoxRows * S * cwp;
  uint32_t* c_r = reinterpret_cast<uint32_t*>(c_rt + kBoxRows * S * cwp);
  uint32_t* c_t = c_r + kBoxRows * S * cwp;
  stage_tile(Jb, a.border, Jb.x0 + wx0 * S, Jb.y0 + wy0 * S, tw, th, warp, kBoxRows, lane, tile, tw, [](int col) { return col; });
  __syncthreads();

  const int col = threadIdx.x;
  if(col < tw)
  {
    BoxSums s{ 0u, 0u, 0ull, 0ull, 0ull };
    const int slot = (col % S) * cwp + col / S;
    for(int r = 0; r < th; r++)
    {
      const uint32_t v = tile[(size_t)r * tw + col];
      const uint32_t t = v & 0xffffu, q = v >> 16;            // t = "Tst" (a), q = "Ref" (b)
      s.r += q; s.t += t;
      s.rr += (uint64_t)q * q; s.tt += (uint64_t)t * t; s.rt += (uint64_t)q * t;
      if(r >= N)
      {
        const uint32_t u = tile[(size_t)(r - N) * tw + col];
        const uint32_t tu = u & 0xffffu, qu = u >> 16;
        s.r -= qu; s.t -= tu;
        s.rr -= (uint64_t)qu * qu; s.tt -= (uint64_t)tu * tu; s.rt -= (uint64_t)qu * tu;
      }
      const int e = r - (N - 1);
      if(e >= 0 && e % S == 0)
      {
        const int o = (e / S) * S * cwp + slot;
        c_r[o] = s.r; c_t[o] = s.t; c_rr[o] = s.rr; c_tt[o] = s.tt; c_rt[o] = s.rt;
      }
    }
  }
  __syncthreads();

  const int wr = warp, wx = wx0 + lane;
  if(wr < rows && wx < Jb.nx)
  {
    const int base = wr * S * cwp;
    uint64_t m2[3] = { 0ull, 0ull, 0ull };
    uint32_t m1[2] = { 0u, 0u };
    #pragma unroll
    for(int dx = 0; dx < N; dx++)
    {
      const int o = base + (dx % S) * cwp + lane + dx / S;   // column lane S + dx
      m1[0] += c_r[o]; m1[1] += c_t[o];
      m2[0] += c_rr[o]; m2[1] += c_tt[o]; m2[2] += c_rt[o];
    }
    const double m[5] = { (double)m1[0], (double)m1[1], (double)m2[0], (double)m2[1], (double)m2[2] };   // exact: < 2^53
    const int wy = wy0 + wr;
    Jb.win[((size_t)(wy >> 5) * Jb.nx + wx) * 32 + (wy & 31)] = gen_window<kGenAvg, N>(m, a.inv, Jb.C1, Jb.C2, Jb.calc_l != 0);
  }
}

// 2x2 mean of both pictures of a pair for the next MS-SSIM scale (xPixelOpsSTD.cpp:50-67), after clipping
struct DownArgs
{
  Img      src[2];
  MutImg   dst[2];     // null planes are skipped
  int32_t  dw, dh;
  uint32_t clip;
};

template <typename T>
__global__ void __launch_bounds__(256) k_downsample2(const __grid_constant__ DownArgs a)
{
  const int x = blockIdx.x * 32 + (threadIdx.x & 31), y = blockIdx.y * 8 + (threadIdx.x >> 5), c = blockIdx.z;
  if(x >= a.dw || y >= a.dh) { return; }
  #pragma unroll
  for(int i = 0; i < 2; i++)
  {
    T* d = static_cast<T*>(a.dst[i].p[c]);
    if(!d) { continue; }
    const uint32_t v = min((uint32_t)fetch<T>(a.src[i], c, 2 * x, 2 * y), a.clip) + min((uint32_t)fetch<T>(a.src[i], c, 2 * x + 1, 2 * y), a.clip) +
                       min((uint32_t)fetch<T>(a.src[i], c, 2 * x, 2 * y + 1), a.clip) +
                       min((uint32_t)fetch<T>(a.src[i], c, 2 * x + 1, 2 * y + 1), a.clip);
    d[(size_t)y * a.dst[i].pitch[c] + x] = (T)((v + 2) >> 2);
  }
}

// ---------------------------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------------------------
namespace {

constexpr size_t kGenSmemPreferred = 48 * 1024;   // four CTAs per SM: the staging of one hides behind the others
constexpr size_t kGenSmemMax = 200 * 1024;

struct GenPlan
{
  int    WY, K;
  int    tw, th, cw, wr;
  size_t smem;
};

// Windows per lane of the row-walking form (strides 1, 2, 4): enough that a loaded sample feeds several
// windows, few enough that the tile of 32 K windows stays small.
constexpr int rows_k(int S, int N) { return S == 1 ? 8 : (S == 2 || N < 32) ? 4 : 2; }

// Launch shape of either form: the row-walking form for strides 1, 2 and 4 with as many window rows per
// CTA as fit 48 KB of tile; one window per thread otherwise (every tap of a thread's window is its own,
// so no instruction is spent on taps a window does not have).
bool gen_plan(int N, int S, GenPlan& p)
{
  if(S == 1 || S == 2 || S == 4)
  {
    const int K = rows_k(S, N), KS = K * S;
    p.K = K; p.WY = 4;
    p.tw = (32 * K - 1) * S + N;
    p.cw = (p.tw + KS - 1) / KS;
    for(int wr = 32; wr >= 4; wr >>= 1)
    {
      p.wr = wr;
      p.th = (wr - 1) * S + N;
      p.smem = (size_t)p.th * KS * p.cw * sizeof(uint32_t);
      if(p.smem <= kGenSmemPreferred) { return true; }
    }
    return p.smem <= kGenSmemMax;
  }
  p.K = 1; p.WY = 4; p.wr = 0;
  p.tw = 31 * S + N;
  p.th = (p.WY - 1) * S + N;
  p.cw = (p.tw + S - 1) / S;
  p.smem = (size_t)p.th * S * p.cw * sizeof(uint32_t);
  return p.smem <= kGenSmemMax;
}

template <int MODE, int N, int S>
cudaError_t gen_attr_rows()
{
  return cudaFuncSetAttribute(k_ssim_gen_rows<MODE, N, rows_k(S, N), S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGenSmemMax);
}

template <int MODE, int N>
cudaError_t gen_attr_all()
{
  cudaError_t e = cudaFuncSetAttribute(k_ssim_gen<MODE, N, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGenSmemMax);
  if(e == cudaSuccess) { e = gen_attr_rows<MODE, N, 1>(); }
  if(e == cudaSuccess) { e = gen_attr_rows<MODE, N, 2>(); }
  if(e == cudaSuccess) { e = gen_attr_rows<MODE, N, 4>(); }
  return e;
}

// coefficient upload and shared-memory limits, once per device
cudaError_t gen_configure()
{
  static std::mutex mu;
  static uint64_t done = 0;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) { return e; }
  const uint64_t bit = 1ULL << (dev & 63);
  std::lock_guard<std::mutex> lk(mu);
  if(done & bit) { return cudaSuccess; }
  double c[kCoefTotal];
  build_coefs(c);
  e = cudaMemcpyToSymbol(c_gen_coef, c, sizeof(c));
  if(e == cudaSuccess) { e = gen_attr_all<kGenFlt, 11>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenInt, 11>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenInt, 8>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenInt, 16>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenAvg, 11>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenAvg, 8>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenAvg, 16>(); }
  if(e == cudaSuccess) { e = gen_attr_all<kGenAvg, 32>(); }
  if(e == cudaSuccess) { done |= bit; }
  return e;
}

template <int MODE, int N>
cudaError_t gen_launch_k(const SsimGenArgs& a, const GenPlan& p, int S, int maxnx, int maxny, cudaStream_t s)
{
  const dim3 block(32, p.WY);
  if(p.wr > 0)
  {
    const dim3 grid((maxnx + 32 * p.K - 1) / (32 * p.K), (maxny + p.wr - 1) / p.wr, a.njobs);
    if(S == 1) { k_ssim_gen_rows<MODE, N, rows_k(1, N), 1><<<grid, block, p.smem, s>>>(a); }
    else if(S == 2) { k_ssim_gen_rows<MODE, N, rows_k(2, N), 2><<<grid, block, p.smem, s>>>(a); }
    else { k_ssim_gen_rows<MODE, N, rows_k(4, N), 4><<<grid, block, p.smem, s>>>(a); }
  }
  else
  {
    const dim3 grid((maxnx + 31) / 32, (maxny + p.WY - 1) / p.WY, a.njobs);
    k_ssim_gen<MODE, N, 1><<<grid, block, p.smem, s>>>(a);
  }
  return cudaGetLastError();
}

// shared memory of k_ssim_box<N, S>: the largest tile and the column sums of kBoxRows window rows
constexpr size_t box_smem(int N, int S)
{
  const size_t tile = (size_t)((kBoxRows - 1) * S + N) * (31 * S + N) * 4;
  const size_t cwp = (size_t)(31 * S + N + S - 1) / S;
  return ((tile + 15) & ~(size_t)15) + (size_t)kBoxRows * S * cwp * (3 * 8 + 2 * 4);
}

template <int N, int S>
cudaError_t box_launch_s(SsimGenArgs& a, int maxnx, int maxny, cudaStream_t s)
{
  constexpr size_t smem = box_smem(N, S);
  static_assert(smem <= kGenSmemMax, "box tile too large");
  {
    // the shared-memory limit, once per device
    static std::mutex mu;
    static uint64_t done = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if(e != cudaSuccess) { return e; }
    const uint64_t bit = 1ULL << (dev & 63);
    std::lock_guard<std::mutex> lk(mu);
    if(!(done & bit))
    {
      e = cudaFuncSetAttribute(k_ssim_box<N, S>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if(e != cudaSuccess) { return e; }
      done |= bit;
    }
  }
  a.cw = (31 * S + N + S - 1) / S;
  const dim3 grid((maxnx + 31) / 32, (maxny + kBoxRows - 1) / kBoxRows, a.njobs);
  k_ssim_box<N, S><<<grid, 32 * kBoxRows, smem, s>>>(a);
  return cudaGetLastError();
}

template <int N>
cudaError_t box_launch(SsimGenArgs& a, int S, int maxnx, int maxny, cudaStream_t s)
{
  if(S == 1) { return box_launch_s<N, 1>(a, maxnx, maxny, s); }
  if(S == 2) { return box_launch_s<N, 2>(a, maxnx, maxny, s); }
  return box_launch_s<N, 4>(a, maxnx, maxny, s);
}

}  // namespace

cudaError_t launch_ssim_gen(SsimGenArgs& a, int mode, int N, int S, int border, cudaStream_t s)
{
  if(a.njobs <= 0) { return cudaSuccess; }
  if(a.njobs > kGenMaxJobs || S < 1 || S > N) { return cudaErrorInvalidValue; }
  GenPlan p;
  if(!gen_plan(N, S, p)) { return cudaErrorInvalidValue; }
  cudaError_t e = gen_configure();
  if(e != cudaSuccess) { return e; }
  int maxnx = 0, maxny = 0;
  for(int k = 0; k < a.njobs; k++)
  {
    const SsimGenJob& J = a.job[k];
    if(J.nx < 1 || J.ny < 1 || !J.win || (J.esz != 1 && J.esz != 2)) { return cudaErrorInvalidValue; }
    maxnx = max(maxnx, J.nx); maxny = max(maxny, J.ny);
  }
  a.S = S; a.border = border; a.tw = p.tw; a.th = p.th; a.cw = p.cw; a.wr = p.wr;
  const bool box = S == 1 || S == 2 || S == 4;                      // averaged windows by box sums
  switch(mode)
  {
  case QMIV_SSM_REGULAR_GAUSSIAN_FLT:
    if(N != 11) { return cudaErrorInvalidValue; }
    a.coef = kCoefFlt11; a.inv = 1.0;
    return gen_launch_k<kGenFlt, 11>(a, p, S, maxnx, maxny, s);
  case QMIV_SSM_REGULAR_GAUSSIAN_INT:
    if(N != 11) { return cudaErrorInvalidValue; }
    a.coef = kCoefInt11; a.inv = 1.0 / (double)(1 << 18);          // c_InvFltrIntMul
    return gen_launch_k<kGenInt, 11>(a, p, S, maxnx, maxny, s);
  case QMIV_SSM_REGULAR_AVERAGED:
    if(N != 11) { return cudaErrorInvalidValue; }
    a.coef = 0; a.inv = 1.0 / (double)121;                          // c_InvFltrArea
    if(box) { return box_launch<11>(a, S, maxnx, maxny, s); }
    return gen_launch_k<kGenAvg, 11>(a, p, S, maxnx, maxny, s);
  case QMIV_SSM_BLOCK_GAUSSIAN_INT:
    a.inv = 1.0 / (double)(1 << 18);
    if(N == 8) { a.coef = kCoefInt8; return gen_launch_k<kGenInt, 8>(a, p, S, maxnx, maxny, s); }
    if(N == 16) { a.coef = kCoefInt16; return gen_launch_k<kGenInt, 16>(a, p, S, maxnx, maxny, s); }
    return cudaErrorInvalidValue;
  case QMIV_SSM_BLOCK_AVERAGED:
    a.coef = 0; a.inv = 1.0 / (double)(N * N);                      // c_InvBlockArea
    if(box && N == 8) { return box_launch<8>(a, S, maxnx, maxny, s); }
    if(box && N == 16) { return box_launch<16>(a, S, maxnx, maxny, s); }
    if(box && N == 32) { return box_launch<32>(a, S, maxnx, maxny, s); }
    if(N == 8) { return gen_launch_k<kGenAvg, 8>(a, p, S, maxnx, maxny, s); }
    if(N == 16) { return gen_launch_k<kGenAvg, 16>(a, p, S, maxnx, maxny, s); }
    if(N == 32) { return gen_launch_k<kGenAvg, 32>(a, p, S, maxnx, maxny, s); }
    return cudaErrorInvalidValue;
  default: return cudaErrorInvalidValue;
  }
}

template <typename T>
cudaError_t launch_downsample2(const Img& a, const Img& b, const MutImg& da, const MutImg& db, int dw, int dh, uint32_t clip,
                               cudaStream_t s)
{
  if(dw <= 0 || dh <= 0) { return cudaSuccess; }
  DownArgs d{};
  d.src[0] = a; d.src[1] = b; d.dst[0] = da; d.dst[1] = db; d.dw = dw; d.dh = dh; d.clip = clip;
  const dim3 grid((dw + 31) / 32, (dh + 7) / 8, 3);
  k_downsample2<T><<<grid, 256, 0, s>>>(d);
  return cudaGetLastError();
}
template cudaError_t launch_downsample2<uint8_t>(const Img&, const Img&, const MutImg&, const MutImg&, int, int, uint32_t, cudaStream_t);
template cudaError_t launch_downsample2<uint16_t>(const Img&, const Img&, const MutImg&, const MutImg&, int, int, uint32_t, cudaStream_t);

}  // namespace qmiv
