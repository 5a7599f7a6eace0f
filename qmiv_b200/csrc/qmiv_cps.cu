// Corresponding-pixel-shift search (libs/pmbb-ivqm/src/xCorrespPixelShiftSSE.cpp:18-127) for
// sm_100a: persistent CTAs, TMA tile loads, 4 x 2 pixels per thread in the search.
//
// Per tile of 128 x TH output pixels (TH = 32, or 16 when shared memory is short or the autotuner
// prefers two CTAs per SM) a CTA of 2 x TH / 4 warps
//   1. receives both pictures' raw samples of the tile plus an R-pixel halo (luma box and the
//      two chroma boxes of each picture) through TMA into shared memory; the copies of tile n+1
//      are issued as soon as tile n's raw samples are converted, so they land during its search;
//   2. converts them into two float4 tiles (Y, Cb, Cr, q + 2^23), q = sum_c w_c * ref_c^2,
//      reading every sample at its clamped picture coordinate (the reference's edge-replicated
//      margin, apps/QMIV/src/xAppQMIV.cpp:353 and :899) and the chroma of 4:2:0 / 4:2:2 at
//      (x >> sx, y >> sy) (the nearest upsampling of libs/pmbb-core/src/xPixelOpsSTD.cpp:30-87);
//      4:2:0 tiles at an even search range are converted as 2x2 units sharing one chroma sample;
//   3. searches both directions. A thread owns 4 rows x 2 columns of output pixels, so each
//      staged reference pixel is loaded once per thread for up to 8 of its pixels; the winners'
//      candidate codes go to shared memory;
//   4. re-deals the threads for the epilogue: one thread per 4x4 block and direction gathers its
//      16 winners, adds their squared differences to the 32-bit row sums, writes the shift-
//      compensated samples (SCP) or the IV-SSIM sub-block moments of (test picture, SCP).
//
// Exact fp32 keys: for a test pixel s (test + GCD, unclipped) and candidate r,
//     e - sum_c w_c s_c^2 + 2^23 = (q(r) + 2^23) + sum_c (-2 w_c s_c) r_c
// is three FFMAs. When every partial sum is an integer below 2^24 in magnitude (checked on the
// host from bit depth, weights and the GCD range) they are exact, so the order of candidates and
// all ties are those of the reference's int32 error. The value lies in [2^20, 2^24), where the IEEE
// bit pattern grows with the value, so
//     key = ((bits - bits(2^20)) << 7) + k,   k = (dy+R)(2R+1) + (dx+R)  (raster index, < 128)
// orders candidates as "first strict minimum in raster order" does (xCorrespPixelShiftSSE.cpp:
// 60-79), and the search is one unsigned min per candidate.
// When the fp32 path is not exact the same kernel runs an int32 search mirroring the SSE path's
// wrap-around arithmetic literally.
//
// Shared-memory float tiles are de-interleaved by column parity: element (y, x) sits at
// y * RP + (x & 1) * Q + (x >> 1). A warp reading column 2 * lane + rx for fixed rx touches 32
// consecutive float4 (no bank conflict), and with Q = 4 (mod 8) the conversion's stores of 32
// consecutive columns are conflict-free as well.
#include "qmiv_kernels.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <map>
#include <mutex>

namespace qmiv {

namespace {

constexpr float    kBias     = 8388608.0f;   // 2^23
constexpr uint32_t kKeyBase  = 0x49800000u;  // bit pattern of 2^20f
// 128, the key's scale, read from constant memory so that the key is one integer multiply-add
__constant__ uint32_t c_key_scale = 128u;
constexpr uint32_t kBiasBits = 0x4B000000u;  // bit pattern of 2^23f
constexpr unsigned kFull     = 0xffffffffu;
constexpr long long kWaitCycles = 1LL << 31; // bound of one tile-load wait (about a second)

template <int R, int WY>
struct Geo
{
  static constexpr int D  = 2 * R + 1;
  static constexpr int NT = 64 * WY;                  // two warps across, WY warps down
  static constexpr int TW = 128, TH = 4 * WY;
  static constexpr int SW = TW + 2 * R, SH = TH + 2 * R;
  static constexpr int Q0 = (SW + 1) / 2;
  static constexpr int Q  = Q0 + (12 - Q0 % 8) % 8;   // smallest >= Q0 with Q % 8 == 4
  static constexpr int RP = 2 * Q;                    // row pitch in float4
  static constexpr uint32_t kTileBytes = (uint32_t)SH * RP * 16u;
  static constexpr uint32_t kCodeBytes = 2u * TH * TW; // winners' candidate codes [dir][TH][TW]
};

struct CpsGeomArgs
{
  int32_t  ntx, ntiles;
  int32_t  use_tma;
  int32_t  ax;                 // 16 bytes in samples: TMA boxes start this far left of the tile
  int32_t  bwl, bhl, bwc, bhc; // raw box sizes in samples (luma, chroma)
  int32_t  sx, sy;             // chroma subsampling shifts
  uint32_t off[2][3];          // byte offsets of the raw boxes in shared memory
  uint32_t raw_bytes;          // raw region, multiple of 128
  uint32_t tx_bytes;           // bytes the six copies of one tile deliver
  int32_t* status;             // PairOut::flags: bit 3 = a tile load did not complete
};

struct alignas(64) CpsKernelArgs
{
  CUtensorMap map[2][3];       // [picture][plane]
  CpsArgs     a;
  CpsGeomArgs g;
};

// ---- TMA / mbarrier ---------------------------------------------------------------------------
__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y, uint64_t* bar)
{
  asm volatile(
    "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];"
    ::"r"(smem_u32(dst)), "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar)) : "memory");
}

// ---- tile loads ---------------------------------------------------------------------------------
// Tensor maps written to global memory by a host copy are made visible to the TMA unit
__device__ __forceinline__ void fence_tensormap_acquire(const CUtensorMap* map)
{
  asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(map) : "memory");
}

template <int R, int WY, bool GMAPS>
__device__ __forceinline__ void issue_tile(const CpsKernelArgs& k, unsigned char* raw, uint64_t* bar, int t)
{
  using G = Geo<R, WY>;
  const int x0 = (t % k.g.ntx) * G::TW, y0 = (t / k.g.ntx) * G::TH;
  const int xl = x0 - k.g.ax, yl = y0 - R;
  const int xc = (x0 >> k.g.sx) - k.g.ax, yc = (y0 - R) >> k.g.sy;
  if(GMAPS)
  {
    #pragma unroll
    for(int f = 0; f < 2; f++)
    {
      #pragma unroll
      for(int c = 0; c < 3; c++) { fence_tensormap_acquire(&k.map[f][c]); }
    }
  }
  mbar_expect_tx(bar, k.g.tx_bytes);
  #pragma unroll
  for(int f = 0; f < 2; f++)
  {
    tma_load_2d(raw + k.g.off[f][0], &k.map[f][0], xl, yl, bar);
    tma_load_2d(raw + k.g.off[f][1], &k.map[f][1], xc, yc, bar);
    tma_load_2d(raw + k.g.off[f][2], &k.map[f][2], xc, yc, bar);
  }
}

// Same boxes with plain loads, for frames whose address or pitch TMA cannot take. Samples outside
// the picture are left unwritten: the conversion only reads clamped in-picture coordinates.
template <typename T, int R, int WY>
__device__ void load_plain(const CpsArgs& a, const CpsGeomArgs& g, unsigned char* raw, int x0, int y0)
{
  constexpr int NW = Geo<R, WY>::NT / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  #pragma unroll 1
  for(int f = 0; f < 2; f++)
  {
    const Img& im = f ? a.in1 : a.in0;
    #pragma unroll 1
    for(int c = 0; c < 3; c++)
    {
      const int pw = c ? (a.W >> g.sx) : a.W, ph = c ? (a.H >> g.sy) : a.H;
      const int bw = c ? g.bwc : g.bwl, bh = c ? g.bhc : g.bhl;
      const int xs = c ? (x0 >> g.sx) - g.ax : x0 - g.ax, ys = c ? (y0 - R) >> g.sy : y0 - R;
      T* dst = reinterpret_cast<T*>(raw + g.off[f][c]);
      const T* src = static_cast<const T*>(im.p[c]);
      for(int r = warp; r < bh; r += NW)
      {
        const int gy = ys + r;
        if(gy < 0 || gy >= ph) { continue; }
        for(int col = lane; col < bw; col += 32)
        {
          const int gx = xs + col;
          if(gx >= 0 && gx < pw) { dst[r * bw + col] = __ldg(src + (size_t)gy * im.pitch[c] + gx); }
        }
      }
    }
  }
}

// raw boxes -> float4 tiles F0 (In0) and F1 (In1). The 2 * SH tile rows of both pictures are dealt
// to the warps round-robin; lane L converts columns L + 32 * kk of a row. Column offsets into the
// raw boxes (clamped to the picture) are per lane and computed once.
template <typename T, int R, int WY, bool CLIP>
__device__ void convert(const CpsArgs& a, const CpsGeomArgs& g, const unsigned char* raw, float4* F0, float4* F1,
                        int x0, int y0)
{
  using G = Geo<R, WY>;
  constexpr int NW = G::NT / 32, NK = (G::SW + 31) / 32;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int W = a.W, H = a.H, sx = g.sx, sy = g.sy;
  const int xl = x0 - g.ax, yl = y0 - R, xc = (x0 >> sx) - g.ax, yc = (y0 - R) >> sy;
  const float w0 = a.wf[0], w1 = a.wf[1], w2 = a.wf[2];
  const uint32_t clip = a.clip;
  int colL[NK], colC[NK];
  #pragma unroll
  for(int kk = 0; kk < NK; kk++)
  {
    const int gx = clampi(x0 - R + lane + 32 * kk, 0, W - 1);
    colL[kk] = gx - xl;
    colC[kk] = (gx >> sx) - xc;
  }
  #pragma unroll 1
  for(int row = warp; row < 2 * G::SH; row += NW)
  {
    const int f  = row >= G::SH ? 1 : 0;
    const int ly = row - f * G::SH;
    const int gy = clampi(y0 - R + ly, 0, H - 1);
    const T* rl = reinterpret_cast<const T*>(raw + g.off[f][0]) + (gy - yl) * g.bwl;
    const T* ru = reinterpret_cast<const T*>(raw + g.off[f][1]) + ((gy >> sy) - yc) * g.bwc;
    const T* rv = reinterpret_cast<const T*>(raw + g.off[f][2]) + ((gy >> sy) - yc) * g.bwc;
    float4* frow = (f ? F1 : F0) + ly * G::RP + (lane & 1) * G::Q + (lane >> 1);
    #pragma unroll
    for(int kk = 0; kk < NK; kk++)
    {
      if(kk < NK - 1 || lane + 32 * kk < G::SW)
      {
        uint32_t v0 = rl[colL[kk]], v1 = ru[colC[kk]], v2 = rv[colC[kk]];
        if(CLIP) { v0 = min(v0, clip); v1 = min(v1, clip); v2 = min(v2, clip); }
        const float y = u2f_exact(v0), u = u2f_exact(v1), v = u2f_exact(v2);
        frow[16 * kk] = make_float4(y, u, v, fmaf(w2, v * v, fmaf(w1, u * u, fmaf(w0, y * y, kBias))));
      }
    }
  }
}

// Two neighbouring samples of a raw row, as one 32-bit word (2-byte samples) or the low half of one
// (1-byte samples); the address is even in samples.
template <typename T>
__device__ __forceinline__ uint32_t load_pair(const T* p)
{
  if constexpr(sizeof(T) == 2) { return *reinterpret_cast<const uint32_t*>(p); }
  else { return *reinterpret_cast<const uint16_t*>(p); }
}
// Byte selectors placing the first / second sample of a pair into the low bits of 0x4B000000
// (2^23), whose float value minus 2^23 is then the sample itself.
template <typename T> struct PairSel;
template <> struct PairSel<uint16_t> { static constexpr uint32_t lo = 0x7410u, hi = 0x7432u; };
template <> struct PairSel<uint8_t>  { static constexpr uint32_t lo = 0x7440u, hi = 0x7441u; };
__device__ __forceinline__ float pair_f(uint32_t pr, uint32_t sel) { return __uint_as_float(__byte_perm(pr, kBiasBits, sel)) - kBias; }

// raw boxes -> float4 tiles for 4:2:0 pictures and an even search range. The staged samples then
// start at even picture coordinates and fall into 2x2 units that share one chroma sample; a thread
// converts whole units: each unit row's two luma samples from one load, the chroma pair and the
// chroma part of q (w1 Cb^2 + w2 Cr^2 + 2^23) once. Coordinates are clamped as in `convert`: a unit
// lies either wholly inside or wholly outside the picture in each direction (even W and H), and the
// clamped column pair and the selectors reproduce the edge replication; tiles whose halo lies inside
// the picture (INTERIOR) skip the clamps. The float4 values are those of `convert`: every term is an
// integer below 2^24, so the changed order of the sums is exact.
template <typename T, int R, int WY, bool INTERIOR>
__device__ void convert420(const CpsArgs& a, const CpsGeomArgs& g, const unsigned char* raw, float4* F0, float4* F1,
                           int x0, int y0)
{
  using G = Geo<R, WY>;
  static_assert(R % 2 == 0, "units start at even coordinates");
  constexpr int UC = G::SW / 2, UR = G::SH / 2, NU = UC * UR;
  const int W = a.W, H = a.H;
  const int cw = W >> 1, chh = H >> 1;
  const int ax = g.ax, bwl = g.bwl, bwc = g.bwc;
  const int xl = x0 - ax, yl = y0 - R, xc = (x0 >> 1) - ax, yc = (y0 - R) >> 1;
  const float w0 = a.wf[0], w1 = a.wf[1], w2 = a.wf[2];
  // the geometry is read once: the tile stores below could alias the shared argument copy
  const uint32_t offl[2] = { g.off[0][0], g.off[1][0] }, offu[2] = { g.off[0][1], g.off[1][1] },
                 offv[2] = { g.off[0][2], g.off[1][2] };
  #pragma unroll 1
  for(int u = threadIdx.x; u < 2 * NU; u += G::NT)
  {
    const int f = u >= NU ? 1 : 0;
    const int r = u - f * NU;
    const int ur = r / UC, uc = r - ur * UC;
    const T* rl = reinterpret_cast<const T*>(raw + (f ? offl[1] : offl[0]));
    const T* ru = reinterpret_cast<const T*>(raw + (f ? offu[1] : offu[0]));
    const T* rv = reinterpret_cast<const T*>(raw + (f ? offv[1] : offv[0]));
    uint32_t l0, l1, s0 = PairSel<T>::lo, s1 = PairSel<T>::hi;
    int co;
    if(INTERIOR)
    {
      // the tile and its halo lie inside the picture: unit (ur, uc) is raw luma (2 ur, ax - R + 2 uc)
      // and raw chroma (ur, ax - R / 2 + uc)
      const T* p = rl + 2 * ur * bwl + (ax - R) + 2 * uc;
      l0 = load_pair<T>(p);
      l1 = load_pair<T>(p + bwl);
      co = ur * bwc + (ax - R / 2) + uc;
    }
    else
    {
      const int gx = x0 - R + 2 * uc, gy = y0 - R + 2 * ur;
      const int px = clampi(gx, 0, W - 2);
      s0 = gx < W ? PairSel<T>::lo : PairSel<T>::hi;
      s1 = gx >= 0 ? PairSel<T>::hi : PairSel<T>::lo;
      const int gy0 = clampi(gy, 0, H - 1), gy1 = clampi(gy + 1, 0, H - 1);
      l0 = load_pair<T>(rl + (gy0 - yl) * bwl + (px - xl));
      l1 = load_pair<T>(rl + (gy1 - yl) * bwl + (px - xl));
      co = (clampi(gy >> 1, 0, chh - 1) - yc) * bwc + clampi(gx >> 1, 0, cw - 1) - xc;
    }
    const float cu = u2f_exact(ru[co]), cv = u2f_exact(rv[co]);
    const float qc = fmaf(w2, cv * cv, fmaf(w1, cu * cu, kBias));
    const float y00 = pair_f(l0, s0), y01 = pair_f(l0, s1), y10 = pair_f(l1, s0), y11 = pair_f(l1, s1);
    float4* d = (f ? F1 : F0) + 2 * ur * G::RP + uc;
    d[0]             = make_float4(y00, cu, cv, fmaf(w0, y00 * y00, qc));
    d[G::Q]          = make_float4(y01, cu, cv, fmaf(w0, y01 * y01, qc));
    d[G::RP]         = make_float4(y10, cu, cv, fmaf(w0, y10 * y10, qc));
    d[G::RP + G::Q]  = make_float4(y11, cu, cv, fmaf(w0, y11 * y11, qc));
  }
}

// ---- search ---------------------------------------------------------------------------------
// Thread (warp w, lane L) owns rows 4 * (w >> 1) + i (i < 4) of columns 64 * (w & 1) + 2L + j
// (j < 2); p = 2 * i + j indexes its eight pixels.
struct Thr
{
  int y0;     // first tile row of the thread's pixels
  int hx;     // (first column) >> 1 = 32 * (w & 1) + L
  int lane;
  __device__ __forceinline__ Thr()
  {
    const int w = threadIdx.x >> 5;
    lane = threadIdx.x & 31;
    y0 = 4 * (w >> 1);
    hx = 32 * (w & 1) + lane;
  }
};

// Code of candidate (dy + R, dx + R) in the low 7 bits of a key: increasing in raster order and,
// for 2R + 1 <= 8, two bit fields.
template <int R>
struct Code
{
  static constexpr int D  = 2 * R + 1;
  static constexpr int KS = D <= 8 ? 8 : D;
  static constexpr uint32_t kMax = (uint32_t)((D - 1) * KS + (D - 1));
  static_assert(kMax < 128, "candidate code must fit 7 bits");
  __device__ static __forceinline__ int dy(uint32_t k) { return KS == 8 ? (int)(k >> 3) : (int)(k / D); }
  __device__ static __forceinline__ int dx(uint32_t k) { return KS == 8 ? (int)(k & 7) : (int)(k - (k / D) * D); }
  __host__ __device__ static constexpr uint32_t of(int dyi, int dxi) { return (uint32_t)(dyi * KS + dxi); }
};

// float4 of tile pixel (row y, column 2 * hx + dx) for a compile-time dx >= 0
template <int R, int WY>
__device__ __forceinline__ int at_hx(int y, int hx, int dx)
{
  using G = Geo<R, WY>;
  return y * G::RP + (dx & 1) * G::Q + hx + (dx >> 1);
}

template <int R, int WY>
__device__ __forceinline__ void search_fp32(const Thr& th, const float4* tst, const float4* ref, const float wf[3],
                                            float ga, float gb, float gc, uint32_t idx[8])
{
  using G = Geo<R, WY>;
  using C = Code<R>;
  constexpr int D = G::D;
  float c0[8], c1[8], c2[8];
  uint32_t best[8], pend[8];
  // c = -2 w (t + g) = (-2 w) t + (-2 w g): integers below 2^24, exact in one FFMA
  const float m0 = -2.0f * wf[0], m1 = -2.0f * wf[1], m2 = -2.0f * wf[2];
  const float o0 = m0 * ga, o1 = m1 * gb, o2 = m2 * gc;
  #pragma unroll
  for(int p = 0; p < 8; p++)
  {
    const float4 t = tst[at_hx<R, WY>(th.y0 + (p >> 1) + R, th.hx, (p & 1) + R)];
    c0[p] = fmaf(m0, t.x, o0);
    c1[p] = fmaf(m1, t.y, o1);
    c2[p] = fmaf(m2, t.z, o2);
    best[p] = 0xffffffffu;
  }
  // The code of candidate (dyi, dxi) = (ry - i, rx - j) of pixel p = (i, j) is
  // C::of(ry, rx) - C::of(i, j). Where C::of(ry, rx) < 128 for every reference sample the thread
  // reads, the key's constant part belongs to the reference sample alone (one register for all
  // eight pixels) and C::of(i, j) is taken off after the minimum. Two candidates of a pixel go into
  // one three-input minimum.
  constexpr bool kShared = C::of(3 + 2 * R, 1 + 2 * R) < 128;
  const float4* rb = ref + at_hx<R, WY>(th.y0, th.hx, 0);
  auto key = [&](const float4& r, int p, uint32_t k) -> uint32_t {
    const float e = fmaf(c2[p], r.z, fmaf(c1[p], r.y, fmaf(c0[p], r.x, r.w)));
    return __float_as_uint(e) * c_key_scale + k;
  };
  #pragma unroll
  for(int ry = 0; ry < 4 + 2 * R; ry++)
  {
    #pragma unroll
    for(int rx = 0; rx < 2 + 2 * R; rx += 2)
    {
      const float4 ra = rb[ry * G::RP + (rx & 1) * G::Q + (rx >> 1)];
      const float4 rc = rb[ry * G::RP + ((rx + 1) & 1) * G::Q + ((rx + 1) >> 1)];
      #pragma unroll
      for(int i = 0; i < 4; i++)
      {
        const int dyi = ry - i;
        if(dyi < 0 || dyi >= D) { continue; }
        #pragma unroll
        for(int j = 0; j < 2; j++)
        {
          const int p = 2 * i + j;
          const bool va = rx - j >= 0 && rx - j < D, vc = rx + 1 - j >= 0 && rx + 1 - j < D;
          const uint32_t ka = (kShared ? C::of(ry, rx) : C::of(dyi, rx - j)) - (kKeyBase << 7);
          const uint32_t kc = (kShared ? C::of(ry, rx + 1) : C::of(dyi, rx + 1 - j)) - (kKeyBase << 7);
          if(va && vc) { best[p] = __vimin3_u32(best[p], key(ra, p, ka), key(rc, p, kc)); }
          else if(va || vc)
          {
            // a pixel's one leftover candidate per search row: rows dyi and dyi + 1 share a
            // three-input minimum, the last row's goes alone
            const uint32_t ks = va ? key(ra, p, ka) : key(rc, p, kc);
            if(dyi == D - 1) { best[p] = min(best[p], ks); }
            else if((dyi & 1) == 0) { pend[p] = ks; }
            else { best[p] = __vimin3_u32(best[p], pend[p], ks); }
          }
        }
      }
    }
  }
  #pragma unroll
  for(int p = 0; p < 8; p++)
  {
    const uint32_t base = kShared ? C::of(p >> 1, p & 1) : 0u;
    idx[p] = min((best[p] & 127u) - base, C::kMax);
  }
}

template <int R, int WY>
__device__ __forceinline__ void search_int(const Thr& th, const float4* tst, const float4* ref, const int32_t wi[3],
                                           int ga, int gb, int gc, uint32_t idx[8])
{
  using G = Geo<R, WY>;
  constexpr int D = G::D;
  const uint32_t w0 = (uint32_t)wi[0], w1 = (uint32_t)wi[1], w2 = (uint32_t)wi[2];
  #pragma unroll
  for(int p = 0; p < 8; p++)
  {
    const int i = p >> 1, j = p & 1;
    const float4 t = tst[at_hx<R, WY>(th.y0 + i + R, th.hx, j + R)];
    const int s0 = f2i_exact(t.x) + ga, s1 = f2i_exact(t.y) + gb, s2 = f2i_exact(t.z) + gc;
    int32_t  best_err = 0x7fffffff;
    uint32_t bi = 0;
    #pragma unroll 1
    for(int dyi = 0; dyi < D; dyi++)
    {
      #pragma unroll 1
      for(int dxi = 0; dxi < D; dxi++)
      {
        const int dx = j + dxi;
        const float4   r  = ref[(th.y0 + i + dyi) * G::RP + (dx & 1) * G::Q + th.hx + (dx >> 1)];
        const uint32_t d0 = (uint32_t)(s0 - f2i_exact(r.x)), d1 = (uint32_t)(s1 - f2i_exact(r.y)),
                       d2 = (uint32_t)(s2 - f2i_exact(r.z));
        const uint32_t err = d0 * d0 * w0 + d1 * d1 * w1 + d2 * d2 * w2;
        if((int32_t)err < best_err) { best_err = (int32_t)err; bi = Code<R>::of(dyi, dxi); }
      }
    }
    idx[p] = bi;
  }
}

// ---- epilogue of the int32 path ----------------------------------------------------------------
// int32 path: the SSE path's wrap-around arithmetic
template <int R, int WY, typename T>
__device__ __forceinline__ void epilogue_int(const Thr& th, const CpsArgs& a, const float4* tst, const float4* ref,
                                          const uint32_t idx[8], int dir, int x0, int y0, int ga, int gb, int gc)
{
  using G = Geo<R, WY>;
  using C = Code<R>;
  uint32_t* rows = a.rows + (size_t)dir * a.H * 3;
  T* scp = static_cast<T*>(dir ? a.scp0 : a.scp1);
  const Moments mom = a.mom[dir];
  const size_t plane = (size_t)a.W * a.H;
  const int xb = x0 + 2 * th.hx, yb = y0 + th.y0;
  const int ig[3] = { ga, gb, gc };
  uint32_t mm[3][5];
  #pragma unroll
  for(int c = 0; c < 3; c++)
  {
    #pragma unroll
    for(int m = 0; m < 5; m++) { mm[c][m] = 0u; }
  }
  #pragma unroll
  for(int i = 0; i < 4; i++)
  {
    const int  y  = yb + i;
    const bool yv = y < a.H;
    uint32_t irs[3] = { 0u, 0u, 0u };
    #pragma unroll
    for(int j = 0; j < 2; j++)
    {
      const int  x     = xb + j;
      const bool valid = yv && x < a.W;
      const uint32_t k = idx[2 * i + j];
      const int dyi = C::dy(k), dx = j + C::dx(k);
      const float4 r = ref[(th.y0 + i + dyi) * G::RP + (dx & 1) * G::Q + th.hx + (dx >> 1)];
      const float4 t = tst[at_hx<R, WY>(th.y0 + i + R, th.hx, j + R)];
      const float rv[3] = { r.x, r.y, r.z }, tv[3] = { t.x, t.y, t.z };
      #pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const int ti = f2i_exact(tv[c]), ri = f2i_exact(rv[c]);
        const uint32_t e = (uint32_t)(ti + ig[c] - ri);
        const uint32_t b = (uint32_t)clampi(ri - ig[c], 0, a.maxv);
        if(valid)
        {
          irs[c] += e * e;
          if(scp != nullptr) { scp[(size_t)c * plane + (size_t)y * a.W + x] = (T)b; }
          mm[c][0] += (uint32_t)ti;
          mm[c][1] += b;
          mm[c][2] += (uint32_t)ti * (uint32_t)ti;
          mm[c][3] += b * b;
          mm[c][4] += (uint32_t)ti * b;
        }
      }
    }
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const uint32_t s = __reduce_add_sync(kFull, irs[c]);
      if(th.lane == 0 && yv) { atomicAdd(rows + (size_t)y * 3 + c, s); }
    }
  }
  if(mom.p != nullptr)
  {
    const int bx = xb >> 2, by = yb >> 2;
    const bool store = (th.lane & 1) == 0 && bx < mom.nbx && by < mom.nby;
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      #pragma unroll
      for(int m = 0; m < 5; m++)
      {
        const uint32_t v = mm[c][m] + __shfl_xor_sync(kFull, mm[c][m], 1);
        if(store) { mom.p[((size_t)c * 5 + m) * mom.plane() + (size_t)by * mom.pitch + bx] = v; }
      }
    }
  }
}

template <int R, int WY, typename T>
__device__ __noinline__ void direction_int(const Thr& th, const CpsArgs& a, const float4* tst, const float4* ref, int dir,
                                           int x0, int y0, int ga, int gb, int gc)
{
  uint32_t idx[8];
  search_int<R, WY>(th, tst, ref, a.wi, ga, gb, gc, idx);
  epilogue_int<R, WY, T>(th, a, tst, ref, idx, dir, x0, y0, ga, gb, gc);
}

// ---- block epilogue (fp32 path) -------------------------------------------------------------------
// After both searches the winners' codes sit in shared memory ([dir][TH][TW] bytes) and the threads
// are re-dealt: warp w takes direction w / WY and the 4x4 blocks of tile rows 4 (w % WY) .. + 3,
// lane L the block of columns 4 L .. 4 L + 3. A thread then holds a whole SSIM sub-block (its moments
// need no exchange between lanes and leave as one coalesced store per moment plane), and a warp
// holds whole tile rows (one warp reduction per row and component).
//
// Staged position of candidate k of pixel (i, j) relative to the block's first candidate:
// i RP + off[j & 1][k] + (j >> 1), off[p][k] = dy RP + ((p + dx) & 1) Q + ((p + dx) >> 1) for the
// parity-split rows. Codes that no search produces map to 0 (never read, kept in bounds).
template <int R, int WY>
__device__ __forceinline__ void build_offsets(int16_t* off)
{
  using G = Geo<R, WY>;
  using C = Code<R>;
  for(int e = threadIdx.x; e < 256; e += G::NT)
  {
    const int p = e >> 7, k = e & 127;
    const int dy = C::dy((uint32_t)k), dx = C::dx((uint32_t)k);
    const bool valid = k <= (int)C::kMax && dy < G::D && dx < G::D;
    off[e] = valid ? (int16_t)(dy * G::RP + ((p + dx) & 1) * G::Q + ((p + dx) >> 1)) : (int16_t)0;
  }
}

// the eight codes a search thread owns: row 4 (w >> 1) + i, columns 64 (w & 1) + 2 L + j
template <int R, int WY>
__device__ __forceinline__ void store_codes(const Thr& th, uint8_t* codes, int dir, const uint32_t idx[8])
{
  using G = Geo<R, WY>;
  uint8_t* cw = codes + dir * (G::TH * G::TW) + th.y0 * G::TW + 2 * th.hx;
  #pragma unroll
  for(int i = 0; i < 4; i++) { *reinterpret_cast<uint16_t*>(cw + i * G::TW) = (uint16_t)(idx[2 * i] | (idx[2 * i + 1] << 8)); }
}

// fp32 path: every value is an integer below 2^24 (path condition), so the float arithmetic is exact;
// a row's four squared differences add below 2^23. Tiles that reach past the picture (EDGE) weight
// every pixel by 1 (inside) or 0 (outside).
template <int R, int WY, typename T, bool EDGE, bool MOM, bool SCP>
__device__ __forceinline__ void epilogue_blk(const CpsArgs& a, const float4* F0, const float4* F1, const uint8_t* codes,
                                             const int16_t* off, int dir, int x0, int y0, int g0, int g1, int g2)
{
  using G = Geo<R, WY>;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int by = warp - dir * WY, bx = lane;
  const float4* tst = dir ? F1 : F0;
  const float4* ref = dir ? F0 : F1;
  uint32_t* rows = a.rows + (size_t)dir * a.H * 3;
  T* scp = static_cast<T*>(dir ? a.scp0 : a.scp1);
  const size_t plane = (size_t)a.W * a.H;
  const int xb = x0 + 4 * bx, yb = y0 + 4 * by;
  const float sg = dir ? -1.f : 1.f;
  const float fg[3] = { sg * (float)g0, sg * (float)g1, sg * (float)g2 };
  const float fmax = (float)a.maxv;
  // Bank spreading: a float4 of column 4 bx + j sits 2 bx + const float4 from the row start, so lanes
  // visiting the same j would hit only four of the eight 16-byte bank groups. Lanes with bit 2 of bx
  // set visit the block's columns in the order j ^ 2, one float4 off (+1 for j < 2, -1 for j >= 2),
  // which puts the eight lanes of every shared-memory phase on eight different groups.
  const int sw = (bx >> 2) & 1;
  const float4* rb = ref + 4 * by * G::RP + 2 * bx;
  const float4* tb = tst + (4 * by + R) * G::RP + 2 * bx;
  const float4* rbs[2] = { rb + sw, rb - sw };   // j < 2, j >= 2
  const float4* tbs[2] = { tb + sw, tb - sw };
  const uint8_t* cb = codes + dir * (G::TH * G::TW) + 4 * by * G::TW + 4 * bx;
  int xj[4];                                      // picture column of visit j
  float cm[4] = { 1.f, 1.f, 1.f, 1.f };
  #pragma unroll
  for(int j = 0; j < 4; j++)
  {
    xj[j] = xb + (j ^ (2 * sw));
    if(EDGE) { cm[j] = xj[j] < a.W ? 1.f : 0.f; }
  }
  float mm[3][5];
  #pragma unroll
  for(int c = 0; c < 3; c++)
  {
    #pragma unroll
    for(int m = 0; m < 5; m++) { mm[c][m] = 0.f; }
  }
  // the four rows run as a loop (not unrolled) to keep the kernel's hot code small; lanes 0-2 add
  // the warp's row sums of components 0-2 to rows[y * 3 + c]
  const bool l1 = lane == 1, l2 = lane == 2;
  #pragma unroll 1
  for(int i = 0; i < 4; i++)
  {
    const int y = yb + i;
    const float rmask = (!EDGE || y < a.H) ? 1.f : 0.f;
    // the four codes of the row, rotated so that byte j is the code of visit j
    const uint32_t c4 = __funnelshift_l(*reinterpret_cast<const uint32_t*>(cb + i * G::TW),
                                        *reinterpret_cast<const uint32_t*>(cb + i * G::TW), 16 * sw);
    float frs[3] = { 0.f, 0.f, 0.f };
    #pragma unroll
    for(int j = 0; j < 4; j++)
    {
      const uint32_t k = (c4 >> (8 * j)) & 0xffu;
      const float4 r = rbs[j >> 1][i * G::RP + off[(j & 1) * 128 + k] + (j >> 1)];
      const float4 t = tbs[j >> 1][i * G::RP + ((j + R) & 1) * G::Q + ((j + R) >> 1)];
      const float m = EDGE ? rmask * cm[j] : 1.f;
      const float rv[3] = { r.x, r.y, r.z }, tv[3] = { t.x, t.y, t.z };
      #pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const float rg = rv[c] - fg[c];
        const float d = tv[c] - rg;
        const float b = fminf(fmaxf(rg, 0.f), fmax);
        frs[c] = fmaf(EDGE ? d * m : d, d, frs[c]);
        if(MOM)
        {
          const float tm = EDGE ? tv[c] * m : tv[c], bm = EDGE ? b * m : b;
          mm[c][0] += tm;
          mm[c][1] += bm;
          mm[c][2] = fmaf(tm, tv[c], mm[c][2]);
          mm[c][3] = fmaf(bm, b, mm[c][3]);
          mm[c][4] = fmaf(tm, b, mm[c][4]);
        }
        if(SCP && (!EDGE || m != 0.f)) { scp[(size_t)c * plane + (size_t)y * a.W + xj[j]] = (T)f2i_exact(b); }
      }
    }
    // 2^23 + (a sum below 2^23) has the sum in its low bits; 32 lanes add 32 x 0x4B000000
    const uint32_t s0 = __reduce_add_sync(kFull, __float_as_uint(frs[0] + kBias)) - 32u * kBiasBits;
    const uint32_t s1 = __reduce_add_sync(kFull, __float_as_uint(frs[1] + kBias)) - 32u * kBiasBits;
    const uint32_t s2 = __reduce_add_sync(kFull, __float_as_uint(frs[2] + kBias)) - 32u * kBiasBits;
    if(lane < 3 && (!EDGE || y < a.H)) { atomicAdd(rows + (size_t)y * 3 + lane, l2 ? s2 : (l1 ? s1 : s0)); }
  }
  if(MOM)
  {
    const Moments mom = a.mom[dir];
    const int bxg = xb >> 2, byg = yb >> 2;
    if(bxg < mom.nbx && byg < mom.nby)
    {
      uint32_t* q = mom.p + (size_t)byg * mom.pitch + bxg;
      const size_t mplane = mom.plane();
      #pragma unroll
      for(int c = 0; c < 3; c++)
      {
        #pragma unroll
        for(int m = 0; m < 5; m++) { q[0] = __float2uint_rn(mm[c][m]); q += mplane; }   // exact: integers below 2^24
      }
    }
  }
}

template <int R, int WY, typename T>
__device__ __forceinline__ void epilogue_blk_dispatch(const CpsArgs& a, const float4* F0, const float4* F1,
                                                      const uint8_t* codes, const int16_t* off, int x0, int y0,
                                                      int g0, int g1, int g2)
{
  using G = Geo<R, WY>;
  const int dir = (int)(threadIdx.x >> 5) >= WY ? 1 : 0;
  const int sel = ((x0 + G::TW > a.W || y0 + G::TH > a.H) ? 4 : 0) | (a.mom[dir].p != nullptr ? 2 : 0) |
                  ((dir ? a.scp0 : a.scp1) != nullptr ? 1 : 0);
  switch(sel)
  {
  case 0: epilogue_blk<R, WY, T, false, false, false>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  case 1: epilogue_blk<R, WY, T, false, false, true>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  case 2: epilogue_blk<R, WY, T, false, true, false>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  case 3: epilogue_blk<R, WY, T, false, true, true>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  case 4: epilogue_blk<R, WY, T, true, false, false>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  case 5: epilogue_blk<R, WY, T, true, false, true>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  case 6: epilogue_blk<R, WY, T, true, true, false>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  default: epilogue_blk<R, WY, T, true, true, true>(a, F0, F1, codes, off, dir, x0, y0, g0, g1, g2); break;
  }
}

// ---- kernel -------------------------------------------------------------------------------------
struct TileRef
{
  const CpsKernelArgs* k;     // the frame pair's arguments
  int                  tile;  // tile index within the pair
};

// Persistent tile loop. `locate` maps a work-list index to (pair, tile); GMAPS: the pairs' tensor
// maps live in global memory. raw_cap: bytes of the raw-box region (the same for every pair).
template <int R, int WY, typename T, bool GMAPS, typename Locate>
__device__ __forceinline__ void cps_loop(int ntiles, const Locate& locate, uint32_t raw_cap)
{
  using G = Geo<R, WY>;
  extern __shared__ __align__(16) unsigned char smem_dyn[];
  unsigned char* base = smem_dyn + ((128u - (smem_u32(smem_dyn) & 127u)) & 127u);   // TMA boxes: 128-byte aligned
  float4* F0 = reinterpret_cast<float4*>(base);
  float4* F1 = F0 + G::SH * G::RP;
  uint8_t* codes = reinterpret_cast<uint8_t*>(base + 2 * G::kTileBytes);
  unsigned char* raw = base + 2 * G::kTileBytes + G::kCodeBytes;
  uint64_t* bar = reinterpret_cast<uint64_t*>(raw + raw_cap);
  const Thr th;
  // the current pair's arguments, copied to shared memory whenever the work list enters a new pair
  __shared__ __align__(16) CpsArgs s_a;
  __shared__ __align__(16) CpsGeomArgs s_g;
  __shared__ int16_t s_off[256];
  static_assert(sizeof(CpsArgs) % 4 == 0 && sizeof(CpsGeomArgs) % 4 == 0, "word copies");

  if(threadIdx.x == 0) { mbar_init(bar, 1); fence_barrier_init(); }
  build_offsets<R, WY>(s_off);
  __syncthreads();
  int t = blockIdx.x;
  if(t < ntiles && threadIdx.x == 0)
  {
    const TileRef L = locate(t);
    if(L.k->g.use_tma) { issue_tile<R, WY, GMAPS>(*L.k, raw, bar, L.tile); }
  }
  uint32_t parity = 0;
  const CpsKernelArgs* cur = nullptr;
  for(; t < ntiles; t += gridDim.x)
  {
    const TileRef L = locate(t);
    if(L.k != cur)
    {
      const uint32_t* sa = reinterpret_cast<const uint32_t*>(&L.k->a);
      const uint32_t* sg = reinterpret_cast<const uint32_t*>(&L.k->g);
      for(int w = threadIdx.x; w < (int)(sizeof(CpsArgs) / 4); w += G::NT) { reinterpret_cast<uint32_t*>(&s_a)[w] = sa[w]; }
      for(int w = threadIdx.x; w < (int)(sizeof(CpsGeomArgs) / 4); w += G::NT) { reinterpret_cast<uint32_t*>(&s_g)[w] = sg[w]; }
      __syncthreads();
      cur = L.k;
    }
    const CpsArgs& a = s_a;
    const CpsGeomArgs& g = s_g;
    const int x0 = (L.tile % g.ntx) * G::TW, y0 = (L.tile / g.ntx) * G::TH;
    if(g.use_tma)
    {
      const bool ok = mbar_wait(bar, parity, kWaitCycles);
      parity ^= 1u;
      if(__syncthreads_or(!ok))
      {
        // the copies did not complete: report, give them one more bounded wait, stop
        if(threadIdx.x == 0) { atomicOr(g.status, 8); mbar_wait(bar, parity ^ 1u, kWaitCycles); }
        return;
      }
    }
    else
    {
      load_plain<T, R, WY>(a, g, raw, x0, y0);
      __syncthreads();
    }
    if(a.clip < (sizeof(T) == 1 ? 0xffu : 0xffffu)) { convert<T, R, WY, true>(a, g, raw, F0, F1, x0, y0); }
    else
    {
      if constexpr(R % 2 == 0)
      {
        if(g.sx == 1 && g.sy == 1)
        {
          if(x0 >= R && y0 >= R && x0 + G::TW + R <= a.W && y0 + G::TH + R <= a.H) { convert420<T, R, WY, true>(a, g, raw, F0, F1, x0, y0); }
          else { convert420<T, R, WY, false>(a, g, raw, F0, F1, x0, y0); }
        }
        else { convert<T, R, WY, false>(a, g, raw, F0, F1, x0, y0); }
      }
      else { convert<T, R, WY, false>(a, g, raw, F0, F1, x0, y0); }
    }
    __syncthreads();
    // the raw boxes are free again: the next tile's copies overlap this tile's search
    const int tn = t + (int)gridDim.x;
    if(tn < ntiles && threadIdx.x == 0)
    {
      const TileRef N = locate(tn);
      if(N.k->g.use_tma)
      {
        fence_proxy_async();
        issue_tile<R, WY, GMAPS>(*N.k, raw, bar, N.tile);
      }
    }
    const int g0 = a.gcd_src->gcd[0], g1 = a.gcd_src->gcd[1], g2 = a.gcd_src->gcd[2];
    const bool int_path = (a.gcd_src->flags & 4) != 0;
    // dir 0 (R2T): test = In0 + GCD searched in In1 -> rows[0], SCP1 = clip(In1[best] - GCD)
    // dir 1 (T2R): test = In1 - GCD searched in In0 -> rows[1], SCP0 = clip(In0[best] + GCD)
    if(!int_path)
    {
      #pragma unroll 1
      for(int dir = 0; dir < 2; dir++)
      {
        const float sg = dir ? -1.f : 1.f;
        uint32_t idx[8];
        search_fp32<R, WY>(th, dir ? F1 : F0, dir ? F0 : F1, a.wf, sg * (float)g0, sg * (float)g1, sg * (float)g2, idx);
        store_codes<R, WY>(th, codes, dir, idx);
      }
      __syncthreads();
      epilogue_blk_dispatch<R, WY, T>(a, F0, F1, codes, s_off, x0, y0, g0, g1, g2);
    }
    else
    {
      #pragma unroll 1
      for(int dir = 0; dir < 2; dir++)
      {
        const int sg = dir ? -1 : 1;
        direction_int<R, WY, T>(th, a, dir ? F1 : F0, dir ? F0 : F1, dir, x0, y0, sg * g0, sg * g1, sg * g2);
      }
    }
    __syncthreads();
  }
}

// one frame pair, arguments in parameter space
template <int R, int WY, typename T>
__global__ void __launch_bounds__(64 * WY, WY == 4 ? 2 : 1) k_cps(const __grid_constant__ CpsKernelArgs k)
{
  cps_loop<R, WY, T, false>(k.g.ntiles, [&](int t) { return TileRef{ &k, t }; }, k.g.raw_bytes);
}

// work list over the tiles of many frame pairs: pair p owns tiles [prefix[p], prefix[p + 1])
template <int R, int WY, typename T>
__global__ void __launch_bounds__(64 * WY, WY == 4 ? 2 : 1) k_cps_multi(const CpsKernelArgs* __restrict__ descs,
                                                          const int32_t* __restrict__ prefix, int npairs, int ntiles,
                                                          uint32_t raw_cap)
{
  cps_loop<R, WY, T, true>(ntiles, [&](int t) {
    int lo = 0, hi = npairs - 1;
    while(lo < hi)
    {
      const int mid = (lo + hi + 1) >> 1;
      if(prefix[mid] <= t) { lo = mid; } else { hi = mid - 1; }
    }
    return TileRef{ &descs[lo], t - prefix[lo] };
  }, raw_cap);
}

// ---- host -------------------------------------------------------------------------------------
PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if(cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
       q == cudaDriverEntryPointSuccess)
    {
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
  });
  return fn;
}

// One 2D tensor map per plane. Returns false when TMA cannot take the plane (alignment, pitch).
bool encode_plane(CUtensorMap* m, const void* p, int32_t w, int32_t h, int64_t pitch_elems, int esz, int bw, int bh)
{
  const uint64_t pitch = (uint64_t)pitch_elems * (uint64_t)esz;
  if(((uintptr_t)p & 15) != 0 || (pitch & 15) != 0 || pitch >= (1ULL << 40) || w <= 0 || h <= 0) { return false; }
  PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
  if(fn == nullptr) { return false; }
  const cuuint64_t dims[2] = { (cuuint64_t)w, (cuuint64_t)h };
  const cuuint64_t strides[1] = { (cuuint64_t)pitch };
  const cuuint32_t box[2] = { (cuuint32_t)bw, (cuuint32_t)bh };
  const cuuint32_t estr[2] = { 1, 1 };
  const CUresult r = fn(m, esz == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_UINT16, 2, const_cast<void*>(p),
                        dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

struct DevInfo
{
  int sms = 0, smem_optin = 0;
};
DevInfo dev_info(int dev)
{
  static std::mutex mu;
  static DevInfo cache[64];
  std::lock_guard<std::mutex> lk(mu);
  if(dev < 0 || dev >= 64) { return DevInfo{ 1, 48 * 1024 }; }
  if(cache[dev].sms == 0)
  {
    cudaDeviceGetAttribute(&cache[dev].sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&cache[dev].smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if(cache[dev].sms <= 0) { cache[dev].sms = 1; }
  }
  return cache[dev];
}

constexpr int kAlign = 128;
constexpr size_t kStaticSmem = 1024;   // the kernel's static shared memory (argument copy), rounded up
inline uint32_t align_up(uint32_t v, uint32_t a) { return (v + a - 1) / a * a; }

// Geometry for one (R, WY, sample size, subsampling); returns the dynamic shared memory size.
template <int R, int WY>
size_t plan(CpsGeomArgs& g, int esz, int sx, int sy)
{
  using G = Geo<R, WY>;
  g.ax = 16 / esz;
  g.sx = sx; g.sy = sy;
  g.bwl = (int)align_up((uint32_t)(g.ax + G::TW + R), (uint32_t)g.ax);
  g.bhl = G::SH;
  const int chi = (G::TW - 1 + R) >> sx;                          // last chroma column, relative to x0 >> sx
  g.bwc = (int)align_up((uint32_t)(g.ax + chi + 1), (uint32_t)g.ax);
  g.bhc = ((G::TH - 1 + R) >> sy) - ((-R) >> sy) + 1;
  uint32_t cur = 0;
  for(int f = 0; f < 2; f++)
  {
    g.off[f][0] = cur; cur += align_up((uint32_t)(g.bwl * g.bhl * esz), kAlign);
    g.off[f][1] = cur; cur += align_up((uint32_t)(g.bwc * g.bhc * esz), kAlign);
    g.off[f][2] = cur; cur += align_up((uint32_t)(g.bwc * g.bhc * esz), kAlign);
  }
  g.raw_bytes = cur;
  g.tx_bytes = (uint32_t)(2 * (g.bwl * g.bhl + 2 * g.bwc * g.bhc) * esz);
  return kAlign + 2 * (size_t)G::kTileBytes + G::kCodeBytes + cur + 16;
}

template <int R, int WY>
void plan_pair(CpsGeomArgs& g, size_t& smem, int esz, int sx, int sy, int W, int H)
{
  using G = Geo<R, WY>;
  smem = plan<R, WY>(g, esz, sx, sy);
  g.ntx = (W + G::TW - 1) / G::TW;
  g.ntiles = g.ntx * ((H + G::TH - 1) / G::TH);
}

// runtime (R, WY) -> plan_pair; false for combinations that are never instantiated (R = 5 with
// 128 x 32 or 128 x 24 tiles never fits shared memory; 128 x 24 tiles exist in the work-list form
// only, where the autotuner picks them)
bool plan_any(int R, int wy, CpsGeomArgs& g, size_t& smem, int esz, int sx, int sy, int W, int H)
{
  switch(R * 16 + wy)
  {
  case 1 * 16 + 8: plan_pair<1, 8>(g, smem, esz, sx, sy, W, H); return true;
  case 2 * 16 + 8: plan_pair<2, 8>(g, smem, esz, sx, sy, W, H); return true;
  case 3 * 16 + 8: plan_pair<3, 8>(g, smem, esz, sx, sy, W, H); return true;
  case 4 * 16 + 8: plan_pair<4, 8>(g, smem, esz, sx, sy, W, H); return true;
  case 1 * 16 + 6: plan_pair<1, 6>(g, smem, esz, sx, sy, W, H); return true;
  case 2 * 16 + 6: plan_pair<2, 6>(g, smem, esz, sx, sy, W, H); return true;
  case 3 * 16 + 6: plan_pair<3, 6>(g, smem, esz, sx, sy, W, H); return true;
  case 4 * 16 + 6: plan_pair<4, 6>(g, smem, esz, sx, sy, W, H); return true;
  case 1 * 16 + 4: plan_pair<1, 4>(g, smem, esz, sx, sy, W, H); return true;
  case 2 * 16 + 4: plan_pair<2, 4>(g, smem, esz, sx, sy, W, H); return true;
  case 3 * 16 + 4: plan_pair<3, 4>(g, smem, esz, sx, sy, W, H); return true;
  case 4 * 16 + 4: plan_pair<4, 4>(g, smem, esz, sx, sy, W, H); return true;
  case 5 * 16 + 4: plan_pair<5, 4>(g, smem, esz, sx, sy, W, H); return true;
  default: return false;
  }
}

// Tensor maps of the six planes; false when TMA cannot take one of them (plain loads then).
bool encode_maps(CpsKernelArgs& k, int esz)
{
  const int cw = k.a.W >> k.g.sx, ch = k.a.H >> k.g.sy;
  for(int f = 0; f < 2; f++)
  {
    const Img& im = f ? k.a.in1 : k.a.in0;
    if(!encode_plane(&k.map[f][0], im.p[0], k.a.W, k.a.H, im.pitch[0], esz, k.g.bwl, k.g.bhl)) { return false; }
    if(!encode_plane(&k.map[f][1], im.p[1], cw, ch, im.pitch[1], esz, k.g.bwc, k.g.bhc)) { return false; }
    if(!encode_plane(&k.map[f][2], im.p[2], cw, ch, im.pitch[2], esz, k.g.bwc, k.g.bhc)) { return false; }
  }
  return true;
}

// Raises the kernel's dynamic shared memory limit once per (kernel, device). The opt-in limit
// covers the kernel's static shared memory (the argument copy) and the dynamic part together.
template <typename F>
cudaError_t configure_once(F* fn, int dev)
{
  static std::mutex mu;
  static std::map<const void*, uint64_t> done;
  const uint64_t bit = 1ULL << (dev & 63);
  std::lock_guard<std::mutex> lk(mu);
  uint64_t& m = done[reinterpret_cast<const void*>(fn)];
  if(m & bit) { return cudaSuccess; }
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, fn);
  if(e != cudaSuccess) { return e; }
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, dev_info(dev).smem_optin - (int)fa.sharedSizeBytes);
  if(e == cudaSuccess) { m |= bit; }
  return e;
}

template <typename F>
int grid_for(F* fn, int threads, size_t smem, int ntiles, int dev)
{
  int occ = 1;
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, threads, smem) != cudaSuccess || occ < 1) { occ = 1; }
  return std::max(1, std::min(ntiles, dev_info(dev).sms * occ));
}

template <int R, int WY, typename T>
cudaError_t launch_inst(const CpsKernelArgs& k, size_t smem, int dev, cudaStream_t s)
{
  using G = Geo<R, WY>;
  cudaError_t e = configure_once(k_cps<R, WY, T>, dev);
  if(e != cudaSuccess) { return e; }
  k_cps<R, WY, T><<<grid_for(k_cps<R, WY, T>, G::NT, smem, k.g.ntiles, dev), G::NT, smem, s>>>(k);
  return cudaGetLastError();
}

template <int R, int WY, typename T>
cudaError_t launch_multi_inst(const CpsKernelArgs* d, const int32_t* prefix, int npairs, int ntiles, uint32_t raw_cap,
                              size_t smem, int dev, cudaStream_t s)
{
  using G = Geo<R, WY>;
  cudaError_t e = configure_once(k_cps_multi<R, WY, T>, dev);
  if(e != cudaSuccess) { return e; }
  const int grid = grid_for(k_cps_multi<R, WY, T>, G::NT, smem, ntiles, dev);
  k_cps_multi<R, WY, T><<<grid, G::NT, smem, s>>>(d, prefix, npairs, ntiles, raw_cap);
  return cudaGetLastError();
}

template <int R, typename T>
cudaError_t launch_r(CpsKernelArgs& k, cudaStream_t s)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) { return e; }
  const int esz = (int)sizeof(T);
  const int wy = cps_pick_wy(R, esz, k.a.in0.sx[1], k.a.in0.sy[1]);
  if(wy == 0) { return cudaErrorInvalidConfiguration; }
  size_t smem = 0;
  plan_any(R, wy, k.g, smem, esz, k.a.in0.sx[1], k.a.in0.sy[1], k.a.W, k.a.H);
  k.g.use_tma = encode_maps(k, esz) ? 1 : 0;
  if constexpr(R <= 4)
  {
    if(wy == 8) { return launch_inst<R, 8, T>(k, smem, dev, s); }
  }
  if(wy == 4) { return launch_inst<R, 4, T>(k, smem, dev, s); }
  return cudaErrorInvalidConfiguration;
}

template <int R, typename T>
cudaError_t launch_multi_r(const CpsKernelArgs* d, const int32_t* prefix, int npairs, int ntiles, int wy,
                           uint32_t raw_cap, size_t smem, int dev, cudaStream_t s)
{
  if constexpr(R <= 4)
  {
    if(wy == 8) { return launch_multi_inst<R, 8, T>(d, prefix, npairs, ntiles, raw_cap, smem, dev, s); }
    if(wy == 6) { return launch_multi_inst<R, 6, T>(d, prefix, npairs, ntiles, raw_cap, smem, dev, s); }
  }
  if(wy == 4) { return launch_multi_inst<R, 4, T>(d, prefix, npairs, ntiles, raw_cap, smem, dev, s); }
  return cudaErrorInvalidConfiguration;
}

}  // namespace

// 16 warps (128 x 32 tiles) where both float tiles and the raw boxes fit in shared memory (R <= 4,
// except 2-byte 4:4:4 pictures from R = 3 on, whose full-size chroma boxes are too large); 8 warps
// (128 x 16 tiles) otherwise.
int cps_pick_wy(int R, int esz, int sx, int sy)
{
  if(R <= 4 && cps_tile_fits(R, 8, esz, sx, sy)) { return 8; }
  if(cps_tile_fits(R, 4, esz, sx, sy)) { return 4; }
  return 0;
}

bool cps_tile_fits(int R, int wy, int esz, int sx, int sy)
{
  int dev = 0;
  if(cudaGetDevice(&dev) != cudaSuccess) { return false; }
  CpsGeomArgs g{};
  size_t smem = 0;
  return plan_any(R, wy, g, smem, esz, sx, sy, 1, 1) && smem + kStaticSmem <= (size_t)dev_info(dev).smem_optin;
}

size_t cps_desc_bytes() { return sizeof(CpsKernelArgs); }

cudaError_t cps_describe(void* desc, const CpsArgs& a, int R, int esz, int wy, CpsPairPlan* plan)
{
  CpsKernelArgs& k = *static_cast<CpsKernelArgs*>(desc);
  std::memset(&k, 0, sizeof(k));
  k.a = a;
  k.g.status = const_cast<int32_t*>(&a.gcd_src->flags);
  size_t smem = 0;
  if(!plan_any(R, wy, k.g, smem, esz, a.in0.sx[1], a.in0.sy[1], a.W, a.H)) { return cudaErrorInvalidConfiguration; }
  k.g.use_tma = encode_maps(k, esz) ? 1 : 0;
  plan->ntiles = k.g.ntiles;
  plan->raw_bytes = k.g.raw_bytes;
  plan->smem = smem;
  return cudaSuccess;
}

cudaError_t launch_cps_multi(const void* d_descs, const int32_t* d_prefix, int npairs, int ntiles, int R, int wy,
                             int esz, uint32_t raw_cap, size_t smem, cudaStream_t s)
{
  if(npairs <= 0 || ntiles <= 0) { return cudaSuccess; }
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) { return e; }
  const CpsKernelArgs* d = static_cast<const CpsKernelArgs*>(d_descs);
  auto go = [&](auto tag) -> cudaError_t {
    using T = decltype(tag);
    switch(R)
    {
    case 1: return launch_multi_r<1, T>(d, d_prefix, npairs, ntiles, wy, raw_cap, smem, dev, s);
    case 2: return launch_multi_r<2, T>(d, d_prefix, npairs, ntiles, wy, raw_cap, smem, dev, s);
    case 3: return launch_multi_r<3, T>(d, d_prefix, npairs, ntiles, wy, raw_cap, smem, dev, s);
    case 4: return launch_multi_r<4, T>(d, d_prefix, npairs, ntiles, wy, raw_cap, smem, dev, s);
    case 5: return launch_multi_r<5, T>(d, d_prefix, npairs, ntiles, wy, raw_cap, smem, dev, s);
    default: return cudaErrorInvalidValue;
    }
  };
  return esz == 1 ? go(uint8_t{}) : go(uint16_t{});
}

bool cps_fp32_exact(int32_t maxv, const int32_t w[3], const int32_t maxdiff[3])
{
  const int64_t bias = 1LL << 23;
  int64_t e = 0, q = 0, up = 0, lo = 0;
  for(int c = 0; c < 3; c++)
  {
    const int64_t g = maxdiff[c] < 0 ? -(int64_t)maxdiff[c] : maxdiff[c];
    if(w[c] < 0) { return false; }
    e  += (int64_t)w[c] * (maxv + g) * (maxv + g);   // max of sum_c w_c (s_c - r_c)^2 and of sum_c w_c s_c^2
    q  += (int64_t)w[c] * maxv * maxv;
    up += 2 * (int64_t)w[c] * g * maxv;              // largest positive -2 w s r (s negative)
    lo += 2 * (int64_t)w[c] * (maxv + g) * maxv;     // largest negative -2 w s r
    // epilogue: four squared differences of a row (maxv + g)^2 add below 2^23
    if(4 * (maxv + g) * (maxv + g) >= bias) { return false; }
  }
  const int64_t lim = 1LL << 24;
  if(bias - e < (1LL << 20)) { return false; }       // key base
  if(bias + e >= lim) { return false; }
  if(bias + q + up >= lim) { return false; }         // partial sums of the FFMA chain
  if(bias - lo <= -lim) { return false; }
  if(16LL * maxv * maxv >= lim) { return false; }    // float SSIM moments of a 4x4 block
  return true;
}

template <typename T>
cudaError_t launch_cps(const CpsArgs& a, int R, cudaStream_t s)
{
  CpsKernelArgs k;
  std::memset(&k, 0, sizeof(k));
  k.a = a;
  k.g.status = const_cast<int32_t*>(&a.gcd_src->flags);
  switch(R)
  {
  case 1: return launch_r<1, T>(k, s);
  case 2: return launch_r<2, T>(k, s);
  case 3: return launch_r<3, T>(k, s);
  case 4: return launch_r<4, T>(k, s);
  case 5: return launch_r<5, T>(k, s);
  default: return cudaErrorInvalidValue;
  }
}
template cudaError_t launch_cps<uint8_t>(const CpsArgs&, int, cudaStream_t);
template cudaError_t launch_cps<uint16_t>(const CpsArgs&, int, cudaStream_t);

}  // namespace qmiv
