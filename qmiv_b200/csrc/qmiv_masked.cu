// Mask mode on B200: the reference app's -im option (apps/QMIV/src/xAppQMIV.cpp:900-1030), where a
// mask picture's luma weights every sample of PSNR, WS-PSNR and IV-PSNR (the STD-only *M processor
// calls; the app refuses the SSIM family with a mask, :360-365).
//
//   k_mask_prepass   one CTA per 4:4:4 row: sum of (In1 - In0) * M (GCD-M), sum of (In1 - In0)^2 * M
//                    per row (PSNR-M, WS-PSNR-M), non-zero mask samples, exactness, samples above the
//                    maximum (the OR of all samples exceeds 2^bd - 1 exactly when one sample does);
//                    k_mask_prepass420v the same for aligned 4:2:0 frames with vector loads, one CTA
//                    per luma row pair under an 8-bit mask (the shared chroma row read once)
//   k_mask_reduce    GCD-M (xGlobClrDiff.cpp:60-91): IEEE divide by NumNonMasked * MaskMax,
//                    round half away, clip
//   k_cps_masked     the masked search (xCorrespPixelShiftSTD.cpp:151-215), both directions: masked
//                    test pixels and masked candidates are skipped, the winner's squared differences
//                    are weighted by the test pixel's mask value and summed per row in uint64;
//                    k_cps_masked_key is the same search by exact fp32 keys, both directions per
//                    CTA, four pixels per thread, where the bit depth, weights and GCD range bound
//                    every error
//   k_mask_finalize  the ordered compensated sums (xKBNS.h:36-43) of the ERP row weights and the
//                    row totals, one CTA per chain (terms staged in shared memory, one thread sums)
// dB values, exact-component fake values and the picture averages are formed on the host in
// qmiv_frame_pair_compute_masked with the reference's arithmetic, including its choice of the mask's
// bit depth for the picture's maximum in PSNR-M (xPSNR.cpp:61) and its direction labels in
// IV-PSNR-M (xIVPSNR.cpp:161-162: "R2T" searches In1 in In0).
#include "qmiv_host.h"
#include "qmiv_kernels.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace qmiv {

struct MaskOut
{
  int32_t  gcd[4];
  int32_t  flags;              // bit0 / bit1: frame 0 / 1 held samples above the maximum
  int32_t  nnm;                // non-zero mask samples (xPixelOpsSTD.cpp:273-284)
  uint32_t or_sample[2];       // OR of every sample per frame: above maxv (2^bd - 1) iff some sample is
  int64_t  sd[3];              // sum over 4:4:4 positions of (In1 - In0) * M
  uint64_t ssd[3];             // sum of (In1 - In0)^2 * M
  uint32_t differs[3];         // the component differs somewhere (whole-picture exactness)
  uint32_t pad_;
  double   ws_err[3];          // KBNS over rows of rowSSD_M * w[y]
  uint64_t cps_sum[2][3];      // [R2T, T2R] in xIVPSNRM's labels
  double   cps_ws[2][3];       // KBNS over rows of rowSSE_M * w[y]
};

struct MaskArgs
{
  Img         in0, in1;
  const void* mask;            // luma of the mask picture, W x H
  int32_t     mpitch;          // in samples
  int32_t     W, H;
  uint32_t    clip;            // samples above are clipped (conceal), 65535 = no clipping
  int32_t     maxv, mask_max;
  int32_t     maxdiff[4];
  int32_t     cws[3];
  uint64_t*   row_ssd;         // [3][H]
  uint64_t*   row_cps;         // [2][H][3]
  const double* ws;            // [H] or null
  MaskOut*    out;
  uint32_t    kscale;          // 128, read from the parameter bank so the key stays one integer multiply-add
  int32_t     pairs420;        // 4:2:0 with luma and mask rows on 2-sample boundaries (two-sample loads)
};

// Host-side description of one masked frame pair: its shape and parameters and what follows from them
// (the GCD-M clip range, which search form applies, the ERP row weights and their correction).
struct MaskPlan
{
  Shape               S;
  qmiv_params         prm{};
  int32_t             mbd = 8;       // mask bit depth
  size_t              mesz = 1;      // bytes per mask sample
  int32_t             maxdiff[4] = { 0, 0, 0, 0 };
  bool                key = false;   // the exact-key search applies (k_cps_masked_key)
  double              ws_corr = 1.0;
  std::vector<double> ws;            // [H] with ERP
};
qmiv_status plan_masked(const Shape& S, const qmiv_params& prm, const qmiv_frame* mask, int32_t mask_bitdepth, MaskPlan& P);
qmiv_status resolve_mask(const MaskPlan& P, const qmiv_frame* mask, char* staging, MaskArgs& a, cudaStream_t s);
void        fill_mask_args(const MaskPlan& P, const Img& a0, const Img& a1, uint64_t* rows, const double* ws, MaskOut* out,
                           MaskArgs& a);
qmiv_status masked_status(const MaskOut& o, const MaskPlan& P);
void        finish_masked(const MaskOut& o, const MaskPlan& P, uint32_t metrics, qmiv_result* out);

namespace {

template <typename TM>
__device__ __forceinline__ int32_t mask_at(const MaskArgs& a, int x, int y)
{
  return (int32_t)__ldg(static_cast<const TM*>(a.mask) + (size_t)y * a.mpitch + x);
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
  #pragma unroll
  for(int o = 16; o > 0; o >>= 1) { v += __shfl_down_sync(0xffffffffu, v, o); }
  return v;
}

// The row's sums: warp sums meet in shared memory, one thread writes the row's SSD and adds the
// row's totals (called by all 256 threads of the CTA).
__device__ __forceinline__ void mask_prepass_row_tail(const MaskArgs& a, int y, int64_t sd[3], uint64_t ssd[3], uint32_t nnm,
                                                      uint32_t dif, uint32_t mx0, uint32_t mx1)
{
  __shared__ uint64_t red[8][6];
  __shared__ uint32_t redu[8][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  #pragma unroll
  for(int c = 0; c < 3; c++)
  {
    sd[c] = (int64_t)warp_sum_u64((uint64_t)sd[c]);
    ssd[c] = warp_sum_u64(ssd[c]);
  }
  nnm = __reduce_add_sync(0xffffffffu, nnm);
  dif = __reduce_or_sync(0xffffffffu, dif);
  mx0 = __reduce_or_sync(0xffffffffu, mx0);
  mx1 = __reduce_or_sync(0xffffffffu, mx1);
  if(lane == 0)
  {
    #pragma unroll
    for(int c = 0; c < 3; c++) { red[warp][c] = (uint64_t)sd[c]; red[warp][3 + c] = ssd[c]; }
    redu[warp][0] = nnm; redu[warp][1] = dif; redu[warp][2] = mx0; redu[warp][3] = mx1;
  }
  __syncthreads();
  if(threadIdx.x != 0) { return; }
  uint64_t t[6] = { 0, 0, 0, 0, 0, 0 };
  nnm = 0; dif = 0; mx0 = 0; mx1 = 0;
  #pragma unroll
  for(int w = 0; w < 8; w++)
  {
    #pragma unroll
    for(int k = 0; k < 6; k++) { t[k] += red[w][k]; }
    nnm += redu[w][0]; dif |= redu[w][1]; mx0 |= redu[w][2]; mx1 |= redu[w][3];
  }
  MaskOut* o = a.out;
  #pragma unroll
  for(int c = 0; c < 3; c++)
  {
    a.row_ssd[(size_t)c * a.H + y] = t[3 + c];
    atomicAdd(reinterpret_cast<unsigned long long*>(&o->sd[c]), (unsigned long long)t[c]);
    atomicAdd(reinterpret_cast<unsigned long long*>(&o->ssd[c]), (unsigned long long)t[3 + c]);
    if(dif & (1u << c)) { atomicOr(&o->differs[c], 1u); }
  }
  atomicAdd(&o->nnm, (int32_t)nnm);
  atomicOr(&o->or_sample[0], mx0);
  atomicOr(&o->or_sample[1], mx1);
}


// One CTA per 4:4:4 row: each thread takes four columns 256 apart per step, issuing all their loads
// before any arithmetic, then the warps' sums meet in shared memory and one thread writes the row's
// SSD and adds the row's totals.
template <typename T, typename TM>
__device__ __forceinline__ void mask_prepass_body(const MaskArgs& a, int row)
{
  constexpr int U = 4;
  const int y = row;
  int64_t  sd[3] = { 0, 0, 0 };
  uint64_t ssd[3] = { 0, 0, 0 };
  uint32_t nnm = 0, dif = 0, mx0 = 0, mx1 = 0;
  for(int xb = threadIdx.x; xb < a.W; xb += 256 * U)
  {
    int32_t  m[U];
    uint32_t va[U][3], vb[U][3];
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int x = min(xb + u * 256, a.W - 1);              // columns past the row repeat the last one, masked out below
      m[u] = xb + u * 256 < a.W ? mask_at<TM>(a, x, y) : 0;
      #pragma unroll
      for(int c = 0; c < 3; c++) { va[u][c] = (uint32_t)fetch<T>(a.in0, c, x, y); vb[u][c] = (uint32_t)fetch<T>(a.in1, c, x, y); }
    }
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      if(xb + u * 256 >= a.W) { continue; }
      nnm += m[u] != 0;
      #pragma unroll
      for(int c = 0; c < 3; c++)
      {
        mx0 |= va[u][c]; mx1 |= vb[u][c];
        const uint32_t p0 = min(va[u][c], a.clip), p1 = min(vb[u][c], a.clip);
        const int32_t d = (int32_t)p1 - (int32_t)p0;
        sd[c] += (int64_t)mul_wrap(d, m[u]);                          // int32 product, xDistortionSTD.cpp:50
        ssd[c] += (uint64_t)(int64_t)mul_wrap(d, d) * (uint64_t)(uint32_t)m[u];    // xDistortionSTD.cpp:62
        dif |= (d != 0 ? 1u : 0u) << c;
      }
    }
  }
  mask_prepass_row_tail(a, y, sd, ssd, nnm, dif, mx0, mx1);
}

// 4:2:0 rows whose planes and mask are aligned for vector loads (checked on the host): a thread
// takes four adjacent pixels per group, read as one 4-sample load per luma plane, one 2-sample
// load per chroma plane and one 4-sample load of the mask; two groups 1024 pixels apart are in
// flight per step. The sums are the same integers as the generic kernel's.
__device__ __forceinline__ void ld4(const uint8_t* p, uint32_t v[4])
{
  const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(p));
  v[0] = w & 0xffu; v[1] = (w >> 8) & 0xffu; v[2] = (w >> 16) & 0xffu; v[3] = w >> 24;
}
__device__ __forceinline__ void ld4(const uint16_t* p, uint32_t v[4])
{
  const uint2 w = __ldg(reinterpret_cast<const uint2*>(p));
  v[0] = w.x & 0xffffu; v[1] = w.x >> 16; v[2] = w.y & 0xffffu; v[3] = w.y >> 16;
}
__device__ __forceinline__ void ld2(const uint8_t* p, uint32_t v[2])
{
  const uint32_t w = __ldg(reinterpret_cast<const unsigned short*>(p));
  v[0] = w & 0xffu; v[1] = w >> 8;
}
__device__ __forceinline__ void ld2(const uint16_t* p, uint32_t v[2])
{
  const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(p));
  v[0] = w & 0xffffu; v[1] = w >> 16;
}

template <typename T, typename TM>
__device__ __forceinline__ void mask_prepass420v_body(const MaskArgs& a, int row)
{
  constexpr int U = 2;
  const int y = row;
  const int ng = a.W >> 2;                                    // groups of four pixels in the row
  const T* l0 = static_cast<const T*>(a.in0.p[0]) + (size_t)y * a.in0.pitch[0];
  const T* l1 = static_cast<const T*>(a.in1.p[0]) + (size_t)y * a.in1.pitch[0];
  const T* u0 = static_cast<const T*>(a.in0.p[1]) + (size_t)(y >> 1) * a.in0.pitch[1];
  const T* v0 = static_cast<const T*>(a.in0.p[2]) + (size_t)(y >> 1) * a.in0.pitch[2];
  const T* u1 = static_cast<const T*>(a.in1.p[1]) + (size_t)(y >> 1) * a.in1.pitch[1];
  const T* v1 = static_cast<const T*>(a.in1.p[2]) + (size_t)(y >> 1) * a.in1.pitch[2];
  const TM* mr = static_cast<const TM*>(a.mask) + (size_t)y * a.mpitch;
  int64_t  sd[3] = { 0, 0, 0 };
  uint64_t ssd[3] = { 0, 0, 0 };
  uint32_t nnm = 0, dif = 0, mx0 = 0, mx1 = 0;
  for(int gb = threadIdx.x; gb < ng; gb += 256 * U)
  {
    uint32_t m[U][4], ya[U][4], yb[U][4], ca[U][2][2], cb[U][2][2];
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int g = min(gb + u * 256, ng - 1);               // groups past the row repeat the last one, skipped below
      const int x = g << 2, xc = g << 1;
      ld4(mr + x, m[u]);
      ld4(l0 + x, ya[u]); ld4(l1 + x, yb[u]);
      ld2(u0 + xc, ca[u][0]); ld2(v0 + xc, ca[u][1]);
      ld2(u1 + xc, cb[u][0]); ld2(v1 + xc, cb[u][1]);
    }
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      if(gb + u * 256 >= ng) { continue; }
      #pragma unroll
      for(int i = 0; i < 4; i++)
      {
        const int32_t mi = (int32_t)m[u][i];
        nnm += mi != 0;
        #pragma unroll
        for(int c = 0; c < 3; c++)
        {
          const uint32_t va = c ? ca[u][c - 1][i >> 1] : ya[u][i], vb = c ? cb[u][c - 1][i >> 1] : yb[u][i];
          mx0 |= va; mx1 |= vb;
          const uint32_t p0 = min(va, a.clip), p1 = min(vb, a.clip);
          const int32_t d = (int32_t)p1 - (int32_t)p0;
          sd[c] += (int64_t)mul_wrap(d, mi);                          // int32 product, xDistortionSTD.cpp:50
          ssd[c] += (uint64_t)(int64_t)mul_wrap(d, d) * (uint64_t)(uint32_t)mi;    // xDistortionSTD.cpp:62
          dif |= (d != 0 ? 1u : 0u) << c;
        }
      }
    }
  }
  mask_prepass_row_tail(a, y, sd, ssd, nnm, dif, mx0, mx1);
}

// One group of four 4:2:0 pixels as pairs of 16-bit samples: luma [0] = pixels 0-1 and [1] = pixels 2-3 of
// each frame, one pair per chroma plane and frame (the two chroma samples under the four pixels) and the
// four 8-bit mask samples.
struct Grp16
{
  uint32_t l0[2], l1[2];
  uint32_t c0[2], c1[2];       // [plane - 1]
  uint32_t m;
};

__device__ __forceinline__ void ld_grp(const uint16_t* l0, const uint16_t* l1, const uint16_t* const ch0[2],
                                       const uint16_t* const ch1[2], const uint8_t* mr, int g, Grp16& r)
{
  const uint2 a = __ldg(reinterpret_cast<const uint2*>(l0 + 4 * g)), b = __ldg(reinterpret_cast<const uint2*>(l1 + 4 * g));
  r.l0[0] = a.x; r.l0[1] = a.y; r.l1[0] = b.x; r.l1[1] = b.y;
  #pragma unroll
  for(int p = 0; p < 2; p++)
  {
    r.c0[p] = __ldg(reinterpret_cast<const uint32_t*>(ch0[p] + 2 * g));
    r.c1[p] = __ldg(reinterpret_cast<const uint32_t*>(ch1[p] + 2 * g));
  }
  r.m = __ldg(reinterpret_cast<const uint32_t*>(mr + 4 * g));
}
// 8-bit samples are spread to 16-bit pairs on loading (byte i of the word to half i of the pair)
__device__ __forceinline__ void ld_grp(const uint8_t* l0, const uint8_t* l1, const uint8_t* const ch0[2],
                                       const uint8_t* const ch1[2], const uint8_t* mr, int g, Grp16& r)
{
  const uint32_t a = __ldg(reinterpret_cast<const uint32_t*>(l0 + 4 * g)), b = __ldg(reinterpret_cast<const uint32_t*>(l1 + 4 * g));
  r.l0[0] = __byte_perm(a, 0u, 0x4140u); r.l0[1] = __byte_perm(a, 0u, 0x4342u);
  r.l1[0] = __byte_perm(b, 0u, 0x4140u); r.l1[1] = __byte_perm(b, 0u, 0x4342u);
  #pragma unroll
  for(int p = 0; p < 2; p++)
  {
    r.c0[p] = __byte_perm((uint32_t)__ldg(reinterpret_cast<const unsigned short*>(ch0[p] + 2 * g)), 0u, 0x4140u);
    r.c1[p] = __byte_perm((uint32_t)__ldg(reinterpret_cast<const unsigned short*>(ch1[p] + 2 * g)), 0u, 0x4140u);
  }
  r.m = __ldg(reinterpret_cast<const uint32_t*>(mr + 4 * g));
}

// a row's luma of both frames and its mask for group g (the chroma words are the row pair's, loaded once)
__device__ __forceinline__ void ld_luma_mask(const uint16_t* l0, const uint16_t* l1, const uint8_t* mr, int g, Grp16& r)
{
  const uint2 a = __ldg(reinterpret_cast<const uint2*>(l0 + 4 * g)), b = __ldg(reinterpret_cast<const uint2*>(l1 + 4 * g));
  r.l0[0] = a.x; r.l0[1] = a.y; r.l1[0] = b.x; r.l1[1] = b.y;
  r.m = __ldg(reinterpret_cast<const uint32_t*>(mr + 4 * g));
}
__device__ __forceinline__ void ld_luma_mask(const uint8_t* l0, const uint8_t* l1, const uint8_t* mr, int g, Grp16& r)
{
  const uint32_t a = __ldg(reinterpret_cast<const uint32_t*>(l0 + 4 * g)), b = __ldg(reinterpret_cast<const uint32_t*>(l1 + 4 * g));
  r.l0[0] = __byte_perm(a, 0u, 0x4140u); r.l0[1] = __byte_perm(a, 0u, 0x4342u);
  r.l1[0] = __byte_perm(b, 0u, 0x4140u); r.l1[1] = __byte_perm(b, 0u, 0x4342u);
  r.m = __ldg(reinterpret_cast<const uint32_t*>(mr + 4 * g));
}

// The differences of two clipped 16-bit pairs below 2^15: the 32-bit difference of the words holds the
// low difference in its low half (two's complement) and the high difference times 2^16 once the low one
// is taken off.
template <bool CLIP>
__device__ __forceinline__ void pair_diff(uint32_t w0, uint32_t w1, uint32_t clip2, uint32_t& dw, int32_t& dlo, int32_t& dhi)
{
  if(CLIP) { w0 = __vminu2(w0, clip2); w1 = __vminu2(w1, clip2); }
  dw = w1 - w0;
  dlo = (int32_t)(int16_t)(dw & 0xffffu);
  dhi = (int32_t)(dw - (uint32_t)dlo) >> 16;
}

// A group's terms when every sample is below 2^15 and the mask below 2^8: the int32 products d * m of the
// reference never overflow, so a chroma sample under two pixels of the row contributes d * (m0 + m1) and
// d^2 * (m0 + m1) once (the square term formed as d * (d * m), one wide multiply-add), and the SD terms
// of a step add up in int32 (below 2^27 for four groups). CLIP: concealment clips the samples first.
__device__ __forceinline__ void word_terms(int32_t dlo, int32_t dhi, uint32_t m0, uint32_t m1, int32_t& sd, uint64_t& ssd)
{
  const int32_t a = dlo * (int32_t)m0, b = dhi * (int32_t)m1;
  sd += a + b;
  ssd += (uint64_t)((int64_t)dlo * a) + (uint64_t)((int64_t)dhi * b);
}

template <bool CLIP>
__device__ __forceinline__ void grp_narrow(const Grp16& g, uint32_t clip2, int32_t sd[3], uint64_t ssd[3], uint32_t difw[3], uint32_t& nnm)
{
  const uint32_t mm[4] = { g.m & 0xffu, (g.m >> 8) & 0xffu, (g.m >> 16) & 0xffu, g.m >> 24 };
  const uint32_t ms[2] = { mm[0] + mm[1], mm[2] + mm[3] };
  nnm += __popc((((g.m & 0x7f7f7f7fu) + 0x7f7f7f7fu) | g.m) & 0x80808080u);    // non-zero mask bytes
  #pragma unroll
  for(int k = 0; k < 2; k++)
  {
    uint32_t dw; int32_t dlo, dhi;
    pair_diff<CLIP>(g.l0[k], g.l1[k], clip2, dw, dlo, dhi);
    difw[0] |= dw;
    word_terms(dlo, dhi, mm[2 * k], mm[2 * k + 1], sd[0], ssd[0]);
  }
  #pragma unroll
  for(int p = 0; p < 2; p++)
  {
    uint32_t dw; int32_t dlo, dhi;
    pair_diff<CLIP>(g.c0[p], g.c1[p], clip2, dw, dlo, dhi);
    difw[1 + p] |= dw;
    word_terms(dlo, dhi, ms[0], ms[1], sd[1 + p], ssd[1 + p]);
  }
}

// A step's OR of every sample of both frames (the above-maximum flags and the 2^15 test)
__device__ __forceinline__ void grp_or(const Grp16& g, uint32_t& o0, uint32_t& o1)
{
  o0 |= g.l0[0] | g.l0[1]; o0 |= g.c0[0] | g.c0[1];
  o1 |= g.l1[0] | g.l1[1]; o1 |= g.c1[0] | g.c1[1];
}

// The same group sample by sample with the reference's int32 products and 64-bit sums (a step that
// holds a sample of 2^15 or more and is not clipped below it).
__device__ __forceinline__ void grp_wide(const Grp16& g, uint32_t clip, int64_t sd[3], uint64_t ssd[3], uint32_t difw[3], uint32_t& nnm)
{
  #pragma unroll
  for(int i = 0; i < 4; i++)
  {
    const int32_t mi = (int32_t)((g.m >> (8 * i)) & 0xffu);
    nnm += mi != 0;
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const uint32_t w0 = c ? g.c0[c - 1] : g.l0[i >> 1], w1 = c ? g.c1[c - 1] : g.l1[i >> 1];
      const int sh = c ? 16 * (i >> 1) : 16 * (i & 1);
      const uint32_t p0 = min((w0 >> sh) & 0xffffu, clip), p1 = min((w1 >> sh) & 0xffffu, clip);
      const int32_t d = (int32_t)p1 - (int32_t)p0;
      sd[c] += (int64_t)mul_wrap(d, mi);                              // int32 product, xDistortionSTD.cpp:50
      ssd[c] += (uint64_t)(int64_t)mul_wrap(d, d) * (uint64_t)(uint32_t)mi;      // xDistortionSTD.cpp:62
      difw[c] |= (uint32_t)d;
    }
  }
}

// grp_narrow for the two rows of a row pair sharing their chroma words: the chroma differences once,
// each row's terms with its own mask sums, each row's SSD apart.
template <bool CLIP>
__device__ __forceinline__ void grp_pair_narrow(const Grp16 (&g)[2], uint32_t clip2, int32_t sd[3], uint64_t (*ssd)[3],
                                                uint32_t difw[3], uint32_t& nnm)
{
  uint32_t ms[2][2];
  #pragma unroll
  for(int r = 0; r < 2; r++)
  {
    const uint32_t m = g[r].m;
    const uint32_t mm[4] = { m & 0xffu, (m >> 8) & 0xffu, (m >> 16) & 0xffu, m >> 24 };
    ms[r][0] = mm[0] + mm[1]; ms[r][1] = mm[2] + mm[3];
    nnm += __popc((((m & 0x7f7f7f7fu) + 0x7f7f7f7fu) | m) & 0x80808080u);    // non-zero mask bytes
    #pragma unroll
    for(int k = 0; k < 2; k++)
    {
      uint32_t dw; int32_t dlo, dhi;
      pair_diff<CLIP>(g[r].l0[k], g[r].l1[k], clip2, dw, dlo, dhi);
      difw[0] |= dw;
      word_terms(dlo, dhi, mm[2 * k], mm[2 * k + 1], sd[0], ssd[r][0]);
    }
  }
  #pragma unroll
  for(int p = 0; p < 2; p++)
  {
    uint32_t dw; int32_t dlo, dhi;
    pair_diff<CLIP>(g[0].c0[p], g[0].c1[p], clip2, dw, dlo, dhi);
    difw[1 + p] |= dw;
    #pragma unroll
    for(int r = 0; r < 2; r++) { word_terms(dlo, dhi, ms[r][0], ms[r][1], sd[1 + p], ssd[r][1 + p]); }
  }
}

// 4:2:0 rows as in mask_prepass420v_body with an 8-bit mask: four groups of four pixels per thread and
// step, all loads issued first, the OR of the samples kept on the pairs, the terms by grp_narrow unless
// the step holds an unclipped sample of 2^15 or more (then grp_wide). The sums are the same integers.
template <typename T>
__device__ __forceinline__ void mask_prepass420n_body(const MaskArgs& a, int row)
{
  constexpr int U = 4;
  const int y = row;
  const int ng = a.W >> 2;
  const T* l0 = static_cast<const T*>(a.in0.p[0]) + (size_t)y * a.in0.pitch[0];
  const T* l1 = static_cast<const T*>(a.in1.p[0]) + (size_t)y * a.in1.pitch[0];
  const T* const ch0[2] = { static_cast<const T*>(a.in0.p[1]) + (size_t)(y >> 1) * a.in0.pitch[1],
                            static_cast<const T*>(a.in0.p[2]) + (size_t)(y >> 1) * a.in0.pitch[2] };
  const T* const ch1[2] = { static_cast<const T*>(a.in1.p[1]) + (size_t)(y >> 1) * a.in1.pitch[1],
                            static_cast<const T*>(a.in1.p[2]) + (size_t)(y >> 1) * a.in1.pitch[2] };
  const uint8_t* mr = static_cast<const uint8_t*>(a.mask) + (size_t)y * a.mpitch;
  const uint32_t clip2 = a.clip | (a.clip << 16);
  const bool chk = sizeof(T) == 2 && a.clip >= 0x8000u;       // unclipped 16-bit samples may reach 2^15
  const bool clip_on = a.clip < (sizeof(T) == 1 ? 0xffu : 0xffffu);
  int64_t  sd[3] = { 0, 0, 0 };
  uint64_t ssd[3] = { 0, 0, 0 };
  uint32_t difw[3] = { 0, 0, 0 };
  uint32_t nnm = 0, mxw0 = 0, mxw1 = 0;
  for(int gb = threadIdx.x; gb < ng; gb += 256 * U)
  {
    Grp16 g[U];
    #pragma unroll
    for(int u = 0; u < U; u++) { ld_grp(l0, l1, ch0, ch1, mr, min(gb + u * 256, ng - 1), g[u]); }   // past the row: repeats, skipped below
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      if(gb + u * 256 >= ng) { continue; }
      grp_or(g[u], mxw0, mxw1);
    }
    if(chk && ((mxw0 | mxw1) & 0x80008000u) != 0)
    {
      #pragma unroll
      for(int u = 0; u < U; u++) { if(gb + u * 256 < ng) { grp_wide(g[u], a.clip, sd, ssd, difw, nnm); } }
      continue;
    }
    int32_t s32[3] = { 0, 0, 0 };
    if(clip_on)
    {
      #pragma unroll
      for(int u = 0; u < U; u++) { if(gb + u * 256 < ng) { grp_narrow<true>(g[u], clip2, s32, ssd, difw, nnm); } }
    }
    else
    {
      #pragma unroll
      for(int u = 0; u < U; u++) { if(gb + u * 256 < ng) { grp_narrow<false>(g[u], clip2, s32, ssd, difw, nnm); } }
    }
    #pragma unroll
    for(int c = 0; c < 3; c++) { sd[c] += s32[c]; }
  }
  const uint32_t dif = (difw[0] != 0 ? 1u : 0u) | (difw[1] != 0 ? 2u : 0u) | (difw[2] != 0 ? 4u : 0u);
  const uint32_t mx0 = (mxw0 & 0xffffu) | (mxw0 >> 16), mx1 = (mxw1 & 0xffffu) | (mxw1 >> 16);
  mask_prepass_row_tail(a, y, sd, ssd, nnm, dif, mx0, mx1);
}

// The sums of a row pair leave the CTA: warp sums meet in shared memory, one thread writes both rows'
// SSD and adds the totals (called by all 256 threads).
__device__ __forceinline__ void mask_prepass_pair_tail(const MaskArgs& a, int y0, int64_t sd[3], uint64_t ssd[2][3],
                                                       uint32_t nnm, uint32_t dif, uint32_t mx0, uint32_t mx1)
{
  __shared__ uint64_t red[8][9];
  __shared__ uint32_t redu[8][4];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint64_t v[9];
  #pragma unroll
  for(int c = 0; c < 3; c++) { v[c] = (uint64_t)sd[c]; v[3 + c] = ssd[0][c]; v[6 + c] = ssd[1][c]; }
  #pragma unroll
  for(int k = 0; k < 9; k++) { v[k] = warp_sum_u64(v[k]); }
  nnm = __reduce_add_sync(0xffffffffu, nnm);
  dif = __reduce_or_sync(0xffffffffu, dif);
  mx0 = __reduce_or_sync(0xffffffffu, mx0);
  mx1 = __reduce_or_sync(0xffffffffu, mx1);
  if(lane == 0)
  {
    #pragma unroll
    for(int k = 0; k < 9; k++) { red[warp][k] = v[k]; }
    redu[warp][0] = nnm; redu[warp][1] = dif; redu[warp][2] = mx0; redu[warp][3] = mx1;
  }
  __syncthreads();
  if(threadIdx.x != 0) { return; }
  uint64_t t[9] = { 0, 0, 0, 0, 0, 0, 0, 0, 0 };
  nnm = 0; dif = 0; mx0 = 0; mx1 = 0;
  #pragma unroll
  for(int w = 0; w < 8; w++)
  {
    #pragma unroll
    for(int k = 0; k < 9; k++) { t[k] += red[w][k]; }
    nnm += redu[w][0]; dif |= redu[w][1]; mx0 |= redu[w][2]; mx1 |= redu[w][3];
  }
  MaskOut* o = a.out;
  #pragma unroll
  for(int c = 0; c < 3; c++)
  {
    a.row_ssd[(size_t)c * a.H + y0] = t[3 + c];
    a.row_ssd[(size_t)c * a.H + y0 + 1] = t[6 + c];
    atomicAdd(reinterpret_cast<unsigned long long*>(&o->sd[c]), (unsigned long long)t[c]);
    atomicAdd(reinterpret_cast<unsigned long long*>(&o->ssd[c]), (unsigned long long)(t[3 + c] + t[6 + c]));
    if(dif & (1u << c)) { atomicOr(&o->differs[c], 1u); }
  }
  atomicAdd(&o->nnm, (int32_t)nnm);
  atomicOr(&o->or_sample[0], mx0);
  atomicOr(&o->or_sample[1], mx1);
}

// Luma rows 2 pr and 2 pr + 1 of an 8-bit-mask 4:2:0 picture (its height is even) in one CTA: the chroma
// row under both is read once and its differences formed once, each row's chroma terms taking that
// row's pixel-pair mask sums; two group columns per thread and step, all loads issued first. Each row
// keeps its own SSD; the sums are the same integers as the one-row forms'.
template <typename T>
__device__ __forceinline__ void mask_prepass420p_body(const MaskArgs& a, int pr)
{
  constexpr int U = 2;
  const int y0 = 2 * pr;
  const int ng = a.W >> 2;
  const T* const chs0[2] = { static_cast<const T*>(a.in0.p[1]) + (size_t)pr * a.in0.pitch[1],
                             static_cast<const T*>(a.in0.p[2]) + (size_t)pr * a.in0.pitch[2] };
  const T* const chs1[2] = { static_cast<const T*>(a.in1.p[1]) + (size_t)pr * a.in1.pitch[1],
                             static_cast<const T*>(a.in1.p[2]) + (size_t)pr * a.in1.pitch[2] };
  const T* lr0[2];
  const T* lr1[2];
  const uint8_t* mr[2];
  #pragma unroll
  for(int r = 0; r < 2; r++)
  {
    lr0[r] = static_cast<const T*>(a.in0.p[0]) + (size_t)(y0 + r) * a.in0.pitch[0];
    lr1[r] = static_cast<const T*>(a.in1.p[0]) + (size_t)(y0 + r) * a.in1.pitch[0];
    mr[r] = static_cast<const uint8_t*>(a.mask) + (size_t)(y0 + r) * a.mpitch;
  }
  const uint32_t clip2 = a.clip | (a.clip << 16);
  const bool chk = sizeof(T) == 2 && a.clip >= 0x8000u;       // unclipped 16-bit samples may reach 2^15
  const bool clip_on = a.clip < (sizeof(T) == 1 ? 0xffu : 0xffffu);
  int64_t  sd[3] = { 0, 0, 0 };
  uint64_t ssd[2][3] = { { 0, 0, 0 }, { 0, 0, 0 } };
  uint32_t difw[3] = { 0, 0, 0 };
  uint32_t nnm = 0, mxw0 = 0, mxw1 = 0;
  for(int gb = threadIdx.x; gb < ng; gb += 256 * U)
  {
    Grp16 g[U][2];                                            // [group column][row]; the chroma words alike in both rows
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int gc = min(gb + u * 256, ng - 1);               // past the row: repeats, skipped below
      ld_grp(lr0[0], lr1[0], chs0, chs1, mr[0], gc, g[u][0]);
      g[u][1].c0[0] = g[u][0].c0[0]; g[u][1].c0[1] = g[u][0].c0[1];
      g[u][1].c1[0] = g[u][0].c1[0]; g[u][1].c1[1] = g[u][0].c1[1];
      ld_luma_mask(lr0[1], lr1[1], mr[1], gc, g[u][1]);
    }
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      if(gb + u * 256 >= ng) { continue; }
      grp_or(g[u][0], mxw0, mxw1);
      mxw0 |= g[u][1].l0[0] | g[u][1].l0[1];
      mxw1 |= g[u][1].l1[0] | g[u][1].l1[1];
    }
    if(chk && ((mxw0 | mxw1) & 0x80008000u) != 0)
    {
      #pragma unroll
      for(int u = 0; u < U; u++)
      {
        if(gb + u * 256 >= ng) { continue; }
        grp_wide(g[u][0], a.clip, sd, ssd[0], difw, nnm);
        grp_wide(g[u][1], a.clip, sd, ssd[1], difw, nnm);
      }
      continue;
    }
    int32_t s32[3] = { 0, 0, 0 };
    if(clip_on)
    {
      #pragma unroll
      for(int u = 0; u < U; u++) { if(gb + u * 256 < ng) { grp_pair_narrow<true>(g[u], clip2, s32, ssd, difw, nnm); } }
    }
    else
    {
      #pragma unroll
      for(int u = 0; u < U; u++) { if(gb + u * 256 < ng) { grp_pair_narrow<false>(g[u], clip2, s32, ssd, difw, nnm); } }
    }
    #pragma unroll
    for(int c = 0; c < 3; c++) { sd[c] += s32[c]; }
  }
  const uint32_t dif = (difw[0] != 0 ? 1u : 0u) | (difw[1] != 0 ? 2u : 0u) | (difw[2] != 0 ? 4u : 0u);
  const uint32_t mx0 = (mxw0 & 0xffffu) | (mxw0 >> 16), mx1 = (mxw1 & 0xffffu) | (mxw1 >> 16);
  mask_prepass_pair_tail(a, y0, sd, ssd, nnm, dif, mx0, mx1);
}

constexpr int kPackPairs = 32;                                 // frame pairs per batched launch

// The vector-load prepass: row pairs for 8-bit masks, sample by sample one row per CTA otherwise.
// idx: the row pair (8-bit masks) or the row.
template <typename T, typename TM>
__device__ __forceinline__ void mask_prepass420_body(const MaskArgs& a, int idx)
{
  if constexpr(sizeof(TM) == 1) { mask_prepass420p_body<T>(a, idx); }
  else { mask_prepass420v_body<T, TM>(a, idx); }
}
// CTAs of the vector-load prepass for a picture of H rows
template <typename TM>
__host__ __device__ inline int prepass420_units(int H) { return sizeof(TM) == 1 ? H / 2 : H; }

// The vector loads of k_mask_prepass420v need 4:2:0, a width divisible by 4, luma rows of both frames
// and mask rows starting on 4-sample boundaries and chroma rows on 2-sample boundaries.
bool mask_prepass_vec_ok(const MaskArgs& a, size_t esz, size_t mesz)
{
  auto al = [](const void* p, size_t n) { return (reinterpret_cast<uintptr_t>(p) % n) == 0; };
  if(a.W % 4 != 0 || a.mpitch % 4 != 0 || !al(a.mask, 4 * mesz)) { return false; }
  const Img* ims[2] = { &a.in0, &a.in1 };
  for(const Img* im : ims)
  {
    if(im->sx[0] != 0 || im->sy[0] != 0) { return false; }
    for(int c = 1; c < 3; c++) { if(im->sx[c] != 1 || im->sy[c] != 1) { return false; } }
    if(im->pitch[0] % 4 != 0 || !al(im->p[0], 4 * esz)) { return false; }
    for(int c = 1; c < 3; c++) { if(im->pitch[c] % 2 != 0 || !al(im->p[c], 2 * esz)) { return false; } }
  }
  return true;
}

// GCD-M, xGlobClrDiff.cpp:60-91 (called with swapped pictures, xGlobClrDiff.h:42: mean of In1 - In0)
__device__ __forceinline__ void mask_reduce_body(const MaskArgs& a)
{
  if(threadIdx.x != 0) { return; }
  MaskOut* o = a.out;
  const double den = (double)((int64_t)o->nnm * (int64_t)a.mask_max);
  #pragma unroll
  for(int c = 0; c < 4; c++)
  {
    int32_t g = 0;
    if(c < 3 && o->nnm > 0) { g = round_half_away(ddiv((double)o->sd[c], den)); }
    o->gcd[c] = min(max(g, -a.maxdiff[c]), a.maxdiff[c]);
  }
  o->flags |= (o->or_sample[0] > (uint32_t)a.maxv ? 1 : 0) | (o->or_sample[1] > (uint32_t)a.maxv ? 2 : 0);
}

// The masked search. A CTA takes a 32 x 8 tile of test pixels of one direction (blockIdx.z: 0 = R2T,
// test In1 searched in In0 with -GCD; 1 = T2R, test In0 searched in In1 with +GCD) and stages the
// reference samples and mask of the tile plus an R halo at clamped coordinates (the reference's
// edge-extended margin). Candidates run in raster order with a strict minimum of the int32 error.
template <typename T, typename TM, int R>
__device__ __forceinline__ void cps_masked_body(const MaskArgs& a, int bx, int by, int bz)
{
  constexpr int TW = 32, TH = 8, SW = TW + 2 * R, SH = TH + 2 * R;
  __shared__ int4 st[SH][SW];                                // (Y, Cb, Cr, mask)
  const int dir = bz;
  const Img& tst = dir ? a.in0 : a.in1;
  const Img& ref = dir ? a.in1 : a.in0;
  const int x0 = bx * TW, y0 = by * TH;
  for(int e = threadIdx.x; e < SH * SW; e += 256)
  {
    const int ly = e / SW, lx = e - ly * SW;
    const int gx = clampi(x0 - R + lx, 0, a.W - 1), gy = clampi(y0 - R + ly, 0, a.H - 1);
    st[ly][lx] = make_int4((int32_t)min((uint32_t)fetch<T>(ref, 0, gx, gy), a.clip),
                           (int32_t)min((uint32_t)fetch<T>(ref, 1, gx, gy), a.clip),
                           (int32_t)min((uint32_t)fetch<T>(ref, 2, gx, gy), a.clip), mask_at<TM>(a, gx, gy));
  }
  __syncthreads();
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int x = x0 + tx, y = y0 + ty;
  uint64_t e[3] = { 0, 0, 0 };
  if(x < a.W && y < a.H)
  {
    const int32_t m = st[ty + R][tx + R].w;
    if(m != 0)
    {
      const int32_t sg = dir ? 1 : -1;
      int32_t s[3];
      #pragma unroll
      for(int c = 0; c < 3; c++) { s[c] = (int32_t)min((uint32_t)fetch<T>(tst, c, x, y), a.clip) + sg * a.out->gcd[c]; }
      // the winner is tracked by its raster index (one select per candidate) and read back after the
      // search; the centre is never masked here, so some candidate always wins
      constexpr int D = 2 * R + 1;
      int32_t best = 0x7fffffff;
      int bidx = R * D + R;
      #pragma unroll
      for(int dy = 0; dy < D; dy++)
      {
        #pragma unroll
        for(int dx = 0; dx < D; dx++)
        {
          const int4 r = st[ty + dy][tx + dx];
          if(r.w == 0) { continue; }
          const int32_t d0 = s[0] - r.x, d1 = s[1] - r.y, d2 = s[2] - r.z;
          const uint32_t err = (uint32_t)mul_wrap(d0, d0) * (uint32_t)a.cws[0] + (uint32_t)mul_wrap(d1, d1) * (uint32_t)a.cws[1] +
                               (uint32_t)mul_wrap(d2, d2) * (uint32_t)a.cws[2];
          if((int32_t)err < best) { best = (int32_t)err; bidx = dy * D + dx; }
        }
      }
      const int4 bp = st[ty + bidx / D][tx + bidx % D];
      const int32_t d0 = s[0] - bp.x, d1 = s[1] - bp.y, d2 = s[2] - bp.z;
      e[0] = (uint64_t)(int64_t)mul_wrap(d0, d0) * (uint64_t)m;
      e[1] = (uint64_t)(int64_t)mul_wrap(d1, d1) * (uint64_t)m;
      e[2] = (uint64_t)(int64_t)mul_wrap(d2, d2) * (uint64_t)m;
    }
  }
  // a warp is 32 pixels of one row
  #pragma unroll
  for(int c = 0; c < 3; c++) { e[c] = warp_sum_u64(e[c]); }
  if(tx == 0 && y < a.H)
  {
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      if(e[c]) { atomicAdd(reinterpret_cast<unsigned long long*>(a.row_cps + ((size_t)dir * a.H + y) * 3 + c), (unsigned long long)e[c]); }
    }
  }
}

// The same search by exact fp32 keys, the form of the unmasked search (qmiv_cps.cu): for a test pixel
// s (test + GCD) and a candidate r, e - K_s + 2^23 = (q_r + 2^23) + sum_c (-2 w_c s_c) r_c with
// K_s = sum_c w_c s_c^2 and q_r = sum_c w_c r_c^2 is three FFMAs. Where the host's check holds (the
// bit depth, weights and GCD range keep every partial sum an integer below 2^24, the same condition as
// the unmasked search, and 2^23 + B <= 2^24 - 2 with B = sum_c w_c (Max + MaxDiff_c)^2 the bound of
// every error), the value lies in [2^20, 2^24 - 2], its bit pattern grows with it, and the key
// (bits - bits(2^20)) * 128 + k (k the raster index of the candidate) orders candidates as (error,
// raster index), the reference's first strict minimum. A masked reference sample is staged as
// (0, 0, 0, 2^24 - 1): its value is that constant, above every real one, so it never wins against an
// unmasked candidate (with every candidate masked the raster-first one is taken, as the integer
// kernels do).
// A CTA takes a 32 x 32 tile in both directions: it stages both pictures with an R halo (and the
// tile's mask values) once; warps 0-7 search In1's pixels in In0 (R2T, -GCD), warps 8-15 In0's in In1
// (T2R, +GCD), each thread four vertically adjacent pixels, so one staged sample read from shared
// memory feeds up to four candidates. A test pixel's own samples come from the other picture's staged
// tile (a masked one reads the sentinel, and its weight M = 0 discards the result).
constexpr float    kMaskBias    = 8388608.0f;        // 2^23
constexpr float    kMaskedValue = 16777215.0f;       // 2^24 - 1: the staged value of a masked sample
constexpr uint32_t kMaskKeyBase = 0x49800000u;       // bit pattern of 2^20f

template <int R>
struct MaskKeyGeo
{
  static constexpr int P = 4, TW = 32, TH = 8 * P, SW = TW + 2 * R, SH = TH + 2 * R, D = 2 * R + 1;
  static constexpr size_t kSmem = sizeof(float4) * 2 * SH * SW + sizeof(int32_t) * TH * TW;
};

// Two adjacent samples of one row (the host checked the alignment): low sample first
__device__ __forceinline__ void ld_pair(const uint16_t* p, uint32_t& v0, uint32_t& v1)
{
  const uint32_t w = __ldg(reinterpret_cast<const uint32_t*>(p));
  v0 = w & 0xffffu; v1 = w >> 16;
}
__device__ __forceinline__ void ld_pair(const uint8_t* p, uint32_t& v0, uint32_t& v1)
{
  const uint32_t w = __ldg(reinterpret_cast<const unsigned short*>(p));
  v0 = w & 0xffu; v1 = w >> 8;
}

// The key search's staging for a tile whose halo lies inside a 4:2:0 picture, R even: the staged area
// splits into 2 x 2 blocks at even picture coordinates, each under one chroma sample, read as two-sample
// rows of luma and mask and one sample per chroma plane; the chroma part of the key, w1 Cb^2 + w2 Cr^2,
// is formed once per block. Under the key search's bound every partial sum of the key is an integer
// below 2^24, so the key equals the per-sample form's whatever the order of the additions.
template <typename T, typename TM, int R>
__device__ __forceinline__ void stage_key420(const MaskArgs& a, float4* st0, float4* st1, int32_t* mk, int x0, int y0,
                                             float w0, float w1, float w2)
{
  using G = MaskKeyGeo<R>;
  constexpr int TW = G::TW, TH = G::TH, SW = G::SW, SH = G::SH, BW = SW / 2;
  const bool clip_on = a.clip < (sizeof(T) == 1 ? 0xffu : 0xffffu);
  for(int b = threadIdx.x; b < (SH / 2) * BW; b += 512)
  {
    const int by = b / BW, bx = b - by * BW;
    const int ly = 2 * by, lx = 2 * bx;
    const int ux = x0 - R + lx, uy = y0 - R + ly;             // even, the block inside the picture
    uint32_t m[4];
    {
      const TM* mp = static_cast<const TM*>(a.mask) + (size_t)uy * a.mpitch + ux;
      ld_pair(mp, m[0], m[1]);
      ld_pair(mp + a.mpitch, m[2], m[3]);
    }
    const Img* im[2] = { &a.in0, &a.in1 };
    float4* st[2] = { st0, st1 };
    #pragma unroll
    for(int f = 0; f < 2; f++)
    {
      const T* yp = static_cast<const T*>(im[f]->p[0]) + (size_t)uy * im[f]->pitch[0] + ux;
      uint32_t v[4];
      ld_pair(yp, v[0], v[1]);
      ld_pair(yp + im[f]->pitch[0], v[2], v[3]);
      uint32_t cb = __ldg(static_cast<const T*>(im[f]->p[1]) + (size_t)(uy >> 1) * im[f]->pitch[1] + (ux >> 1));
      uint32_t cr = __ldg(static_cast<const T*>(im[f]->p[2]) + (size_t)(uy >> 1) * im[f]->pitch[2] + (ux >> 1));
      if(clip_on)
      {
        cb = min(cb, a.clip); cr = min(cr, a.clip);
        #pragma unroll
        for(int i = 0; i < 4; i++) { v[i] = min(v[i], a.clip); }
      }
      const float fb = u2f_exact(cb), fr = u2f_exact(cr);
      const float ct = fmaf(w2, fr * fr, fmaf(w1, fb * fb, kMaskBias));
      #pragma unroll
      for(int i = 0; i < 4; i++)
      {
        const float fy = u2f_exact(v[i]);
        const int e = (ly + (i >> 1)) * SW + lx + (i & 1);
        st[f][e] = m[i] ? make_float4(fy, fb, fr, fmaf(w0, fy * fy, ct)) : make_float4(0.f, 0.f, 0.f, kMaskedValue);
      }
    }
    #pragma unroll
    for(int i = 0; i < 4; i++)
    {
      const int ty = ly + (i >> 1) - R, tx = lx + (i & 1) - R;
      if(ty >= 0 && ty < TH && tx >= 0 && tx < TW) { mk[ty * TW + tx] = (int32_t)m[i]; }
    }
  }
}

template <typename T, typename TM, int R>
// kscale: 128 from a kernel parameter at a fixed offset (the key stays one multiply-add with a constant operand)
__device__ __forceinline__ void cps_masked_key_body(const MaskArgs& a, int bx, int by, uint32_t kscale)
{
  using G = MaskKeyGeo<R>;
  constexpr int P = G::P, TW = G::TW, TH = G::TH, SW = G::SW, SH = G::SH, D = G::D;
  static_assert(D * D <= 128, "the raster index must fit the key's low 7 bits");
  extern __shared__ float4 smem[];
  float4* st0 = smem;                                         // In0: (Y, Cb, Cr, 2^23 + sum w r^2)
  float4* st1 = smem + SH * SW;                               // In1
  int32_t* mk = reinterpret_cast<int32_t*>(smem + 2 * SH * SW);   // M of the tile's pixels, 0 outside the picture
  const int x0 = bx * TW, y0 = by * TH;
  const float w0 = (float)a.cws[0], w1 = (float)a.cws[1], w2 = (float)a.cws[2];
  bool staged = false;
  if constexpr(R % 2 == 0)
  {
    if(a.pairs420 && x0 >= R && y0 >= R && x0 + TW + R <= a.W && y0 + TH + R <= a.H)
    {
      stage_key420<T, TM, R>(a, st0, st1, mk, x0, y0, w0, w1, w2);
      staged = true;
    }
  }
  for(int e = staged ? SH * SW : threadIdx.x; e < SH * SW; e += 512)
  {
    const int ly = e / SW, lx = e - ly * SW;
    const int ux = x0 - R + lx, uy = y0 - R + ly;
    const int gx = clampi(ux, 0, a.W - 1), gy = clampi(uy, 0, a.H - 1);
    // branch-free: every sample is read, a masked one is replaced by the sentinel
    const int32_t mv = mask_at<TM>(a, gx, gy);
    const float p0 = u2f_exact(min((uint32_t)fetch<T>(a.in0, 0, gx, gy), a.clip));
    const float p1 = u2f_exact(min((uint32_t)fetch<T>(a.in0, 1, gx, gy), a.clip));
    const float p2 = u2f_exact(min((uint32_t)fetch<T>(a.in0, 2, gx, gy), a.clip));
    const float q0 = u2f_exact(min((uint32_t)fetch<T>(a.in1, 0, gx, gy), a.clip));
    const float q1 = u2f_exact(min((uint32_t)fetch<T>(a.in1, 1, gx, gy), a.clip));
    const float q2 = u2f_exact(min((uint32_t)fetch<T>(a.in1, 2, gx, gy), a.clip));
    const float k0 = fmaf(w2, p2 * p2, fmaf(w1, p1 * p1, fmaf(w0, p0 * p0, kMaskBias)));
    const float k1 = fmaf(w2, q2 * q2, fmaf(w1, q1 * q1, fmaf(w0, q0 * q0, kMaskBias)));
    st0[e] = mv ? make_float4(p0, p1, p2, k0) : make_float4(0.f, 0.f, 0.f, kMaskedValue);
    st1[e] = mv ? make_float4(q0, q1, q2, k1) : make_float4(0.f, 0.f, 0.f, kMaskedValue);
    if(ly >= R && ly < R + TH && lx >= R && lx < R + TW) { mk[(ly - R) * TW + (lx - R)] = (ux < a.W && uy < a.H) ? mv : 0; }
  }
  __syncthreads();
  const int dir = threadIdx.x >> 8;                          // warp-uniform
  const float4* ref = dir ? st1 : st0;
  const float4* tst = dir ? st0 : st1;
  const int tx = threadIdx.x & 31, ty = (threadIdx.x & 255) >> 5;
  const float sg = dir ? 1.f : -1.f;
  float s[P][3], c0[P], c1[P], c2[P];
  int32_t m[P];
  uint32_t best[P];
  #pragma unroll
  for(int p = 0; p < P; p++)
  {
    const float4 t = tst[(ty * P + p + R) * SW + tx + R];
    s[p][0] = fmaf(sg, (float)a.out->gcd[0], t.x);
    s[p][1] = fmaf(sg, (float)a.out->gcd[1], t.y);
    s[p][2] = fmaf(sg, (float)a.out->gcd[2], t.z);
    c0[p] = -2.0f * w0 * s[p][0];
    c1[p] = -2.0f * w1 * s[p][1];
    c2[p] = -2.0f * w2 * s[p][2];
    m[p] = mk[(ty * P + p) * TW + tx];
    best[p] = 0xffffffffu;
  }
  // candidates in column pairs: one three-input minimum takes two keys
  auto key = [&](const float4& r, int p, int k) -> uint32_t {
    const float t = fmaf(c2[p], r.z, fmaf(c1[p], r.y, fmaf(c0[p], r.x, r.w)));
    return __float_as_uint(t) * kscale + ((uint32_t)k - (kMaskKeyBase << 7));
  };
  // a warp whose 32 x P test pixels are all masked has nothing to search: every term it adds is
  // multiplied by M = 0 (the reference skips masked test pixels, xCorrespPixelShiftSTD.cpp:151-215)
  bool any = false;
  #pragma unroll
  for(int p = 0; p < P; p++) { any = any || m[p] != 0; }
  if(__any_sync(0xffffffffu, any))
  {
    #pragma unroll
    for(int j = 0; j < D + P - 1; j++)
    {
      #pragma unroll
      for(int dx = 0; dx < D; dx += 2)
      {
        const float4 ra = ref[(ty * P + j) * SW + tx + dx];
        const float4 rb = ref[(ty * P + j) * SW + tx + min(dx + 1, D - 1)];
        #pragma unroll
        for(int p = 0; p < P; p++)
        {
          const int dy = j - p;
          if(dy < 0 || dy >= D) { continue; }                  // resolved at compile time
          if(dx + 1 < D) { best[p] = __vimin3_u32(best[p], key(ra, p, dy * D + dx), key(rb, p, dy * D + dx + 1)); }
          else { best[p] = min(best[p], key(ra, p, dy * D + dx)); }
        }
      }
    }
  }
  // Row sums. Each term d^2 M is below 2^38 here (|d| < 2^12: d^2 < 2^24 is checked with the key bound,
  // M < 2^14). Over the warp's 32 pixels of a row the parts from bit 11 up (< 2^27 each) are summed in
  // 32 bits, and the low 11 bits of two terms (sums below 2^16) share one 32-bit sum: 18 redux.sync per
  // warp for its 4 rows x 3 components, every sum exact.
  static_assert(P % 2 == 0, "low parts are reduced in pairs of rows");
  uint32_t lo[P][3], hi[P][3];
  #pragma unroll
  for(int p = 0; p < P; p++)
  {
    // the minimum is always some candidate's key (no key has low bits 127), so k < D * D; the clamp
    // keeps the read in the tile whatever the data
    const int k = min((int)(best[p] & 127u), D * D - 1);
    const float4 bp = ref[(ty * P + p + k / D) * SW + tx + k % D];
    const float d[3] = { s[p][0] - bp.x, s[p][1] - bp.y, s[p][2] - bp.z };   // exact integers
    #pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const int32_t di = f2i_exact(d[c] + 4096.0f) - 4096;   // d + 2^12 lies in (0, 2^13): exact
      const uint64_t t = (uint64_t)(uint32_t)(di * di) * (uint64_t)(uint32_t)m[p];
      hi[p][c] = __reduce_add_sync(0xffffffffu, (uint32_t)(t >> 11));
      lo[p][c] = (uint32_t)t & 0x7ffu;
    }
  }
  #pragma unroll
  for(int p = 0; p < P; p++)
  {
    const uint32_t s01 = __reduce_add_sync(0xffffffffu, lo[p][0] | (lo[p][1] << 16));
    lo[p][0] = s01 & 0xffffu; lo[p][1] = s01 >> 16;
  }
  #pragma unroll
  for(int p = 0; p < P; p += 2)
  {
    const uint32_t s2 = __reduce_add_sync(0xffffffffu, lo[p][2] | (lo[p + 1][2] << 16));
    lo[p][2] = s2 & 0xffffu; lo[p + 1][2] = s2 >> 16;
  }
  if(tx == 0)
  {
    #pragma unroll
    for(int p = 0; p < P; p++)
    {
      const int y = y0 + ty * P + p;
      if(y >= a.H) { continue; }
      #pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const uint64_t v = ((uint64_t)hi[p][c] << 11) + lo[p][c];
        if(v) { atomicAdd(reinterpret_cast<unsigned long long*>(a.row_cps + ((size_t)dir * a.H + y) * 3 + c), (unsigned long long)v); }
      }
    }
  }
}

// Chains 0..2: WS rows of component c; chains 3..8: CPS rows of (direction, component). Each is the
// reference's row-order compensated sum; the CPS chains also form the plain uint64 totals. One CTA per
// chain: all threads stage a chunk of the chain's terms (the products with the ERP weights, the same
// doubles the serial loop would form) in shared memory, then thread 0 adds them in row order, so the
// serial chain never waits on global memory.
constexpr int kMaskFinChunk = 4096;
__device__ __forceinline__ void mask_finalize_body(const MaskArgs& a, int chain)
{
  __shared__ double vals[kMaskFinChunk];
  __shared__ unsigned long long tot;
  const int k = chain;
  if(k < 3 && !a.ws) { return; }                              // uniform over the CTA
  MaskOut* o = a.out;
  const int H = a.H;
  const bool cps = k >= 3;
  const int d = cps ? (k - 3) / 3 : 0, c = cps ? (k - 3) % 3 : 0;
  const uint64_t* r = cps ? a.row_cps + (size_t)d * H * 3 + c : a.row_ssd + (size_t)k * H;
  const size_t step = cps ? 3 : 1;
  if(threadIdx.x == 0) { tot = 0ull; }
  unsigned long long loc = 0ull;
  Kbns s;                                                     // used by thread 0
  for(int base = 0; base < H; base += kMaskFinChunk)
  {
    const int n = min(kMaskFinChunk, H - base);
    __syncthreads();                                          // the previous chunk has been summed
    constexpr int U = kMaskFinChunk / 256;                    // a thread's loads all in flight at once
    uint64_t v[U];
    double w[U];
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int i = threadIdx.x + u * 256;
      v[u] = i < n ? r[(size_t)(base + i) * step] : 0ull;
      w[u] = (i < n && a.ws) ? a.ws[base + i] : 0.0;
    }
    #pragma unroll
    for(int u = 0; u < U; u++)
    {
      const int i = threadIdx.x + u * 256;
      if(i < n) { loc += v[u]; vals[i] = a.ws ? dmul((double)v[u], w[u]) : 0.0; }
    }
    __syncthreads();
    if(threadIdx.x == 0 && a.ws)
    {
      #pragma unroll 8
      for(int i = 0; i < n; i++) { s.add(vals[i]); }
    }
  }
  loc = warp_sum_u64(loc);                                    // exact: integer sum in any order
  if((threadIdx.x & 31) == 0) { atomicAdd(&tot, loc); }
  __syncthreads();
  if(threadIdx.x != 0) { return; }
  if(cps)
  {
    o->cps_sum[d][c] = tot;
    o->cps_ws[d][c] = a.ws ? s.result() : 0.0;
  }
  else { o->ws_err[k] = s.result(); }
}

// ---- kernels: one frame pair (arguments in parameter space) and many (a device table of arguments,
// one grid dimension indexing the pair; CTAs beyond their pair's extent return) -----------------
template <typename T, typename TM>
__global__ void __launch_bounds__(256) k_mask_prepass(const __grid_constant__ MaskArgs a) { mask_prepass_body<T, TM>(a, blockIdx.x); }
template <typename T, typename TM>
__global__ void __launch_bounds__(256, 2) k_mask_prepass420v(const __grid_constant__ MaskArgs a) { mask_prepass420_body<T, TM>(a, blockIdx.x); }
__global__ void k_mask_reduce(const __grid_constant__ MaskArgs a) { mask_reduce_body(a); }
template <typename T, typename TM, int R>
__global__ void __launch_bounds__(256) k_cps_masked(const __grid_constant__ MaskArgs a) { cps_masked_body<T, TM, R>(a, blockIdx.x, blockIdx.y, blockIdx.z); }
template <typename T, typename TM, int R>
__global__ void __launch_bounds__(512, 2) k_cps_masked_key(const __grid_constant__ MaskArgs a) { cps_masked_key_body<T, TM, R>(a, blockIdx.x, blockIdx.y, a.kscale); }
__global__ void __launch_bounds__(256) k_mask_finalize(const __grid_constant__ MaskArgs a) { mask_finalize_body(a, blockIdx.x); }

// The arguments of up to kPackPairs pairs of one launch group, passed by value: every CTA reads its
// pair's arguments from the constant bank as the one-pair kernels do, without a dependent global load.
struct MaskPack
{
  MaskArgs a[kPackPairs];
  uint32_t kscale;             // 128, the key scale at a fixed parameter offset
};
static_assert(sizeof(MaskPack) <= 32000, "kernel parameters are limited to 32 KB");

// vec: the group's pairs take the vector-load prepass
template <typename T, typename TM, bool VEC>
__global__ void __launch_bounds__(256, 2) k_mask_prepass_multi(const __grid_constant__ MaskPack pk)
{
  const MaskArgs& a = pk.a[blockIdx.y];
  if((int)blockIdx.x >= (VEC ? prepass420_units<TM>(a.H) : a.H)) { return; }
  if(VEC) { mask_prepass420_body<T, TM>(a, blockIdx.x); } else { mask_prepass_body<T, TM>(a, blockIdx.x); }
}
__global__ void k_mask_reduce_multi(const __grid_constant__ MaskPack pk) { mask_reduce_body(pk.a[blockIdx.x]); }
template <typename T, typename TM, int R>
__global__ void __launch_bounds__(256) k_cps_masked_multi(const __grid_constant__ MaskPack pk)
{
  const MaskArgs& a = pk.a[blockIdx.z >> 1];
  if((int)blockIdx.x * 32 >= a.W || (int)blockIdx.y * 8 >= a.H) { return; }
  cps_masked_body<T, TM, R>(a, blockIdx.x, blockIdx.y, blockIdx.z & 1);
}
template <typename T, typename TM, int R>
__global__ void __launch_bounds__(512, 2) k_cps_masked_key_multi(const __grid_constant__ MaskPack pk)
{
  const MaskArgs& a = pk.a[blockIdx.z];
  if((int)blockIdx.x * MaskKeyGeo<R>::TW >= a.W || (int)blockIdx.y * MaskKeyGeo<R>::TH >= a.H) { return; }
  cps_masked_key_body<T, TM, R>(a, blockIdx.x, blockIdx.y, pk.kscale);
}
__global__ void __launch_bounds__(256) k_mask_finalize_multi(const __grid_constant__ MaskPack pk)
{
  mask_finalize_body(pk.a[blockIdx.x / 9], blockIdx.x % 9);
}

// A kernel's dynamic shared-memory limit, set once per kernel and device (not on every launch)
template <typename F>
cudaError_t smem_attr_once(F* fn, int bytes)
{
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, bool> done;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) { return e; }
  std::lock_guard<std::mutex> lk(mu);
  bool& d = done[std::make_pair(reinterpret_cast<const void*>(fn), dev)];
  if(d) { return cudaSuccess; }
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if(e == cudaSuccess) { d = true; }
  return e;
}

template <typename T, typename TM, int R>
cudaError_t launch_masked_key(const MaskArgs& a, cudaStream_t s)
{
  constexpr size_t smem = MaskKeyGeo<R>::kSmem;
  const cudaError_t e = smem_attr_once(k_cps_masked_key<T, TM, R>, (int)smem);
  if(e != cudaSuccess) { return e; }
  const dim3 grid((a.W + MaskKeyGeo<R>::TW - 1) / MaskKeyGeo<R>::TW, (a.H + MaskKeyGeo<R>::TH - 1) / MaskKeyGeo<R>::TH);
  k_cps_masked_key<T, TM, R><<<grid, 512, smem, s>>>(a);
  return cudaSuccess;
}

// pipe: the stage timers of the calling calc (events around each stage when its context profiles)
template <typename T, typename TM>
cudaError_t launch_masked_t(const MaskArgs& a, int R, bool key, PairPipeline& pipe, cudaStream_t s)
{
  int tok = pipe.prof_begin(s);
  if(mask_prepass_vec_ok(a, sizeof(T), sizeof(TM))) { k_mask_prepass420v<T, TM><<<prepass420_units<TM>(a.H), 256, 0, s>>>(a); }
  else { k_mask_prepass<T, TM><<<a.H, 256, 0, s>>>(a); }
  pipe.prof_end(s, QMIV_STAGE_PREPASS, tok);
  tok = pipe.prof_begin(s);
  k_mask_reduce<<<1, 32, 0, s>>>(a);
  pipe.prof_end(s, QMIV_STAGE_REDUCE, tok);
  tok = pipe.prof_begin(s);
  const dim3 grid((a.W + 31) / 32, (a.H + 7) / 8, 2);
  if(key)
  {
    cudaError_t e;
    switch(R)
    {
    case 1: e = launch_masked_key<T, TM, 1>(a, s); break;
    case 2: e = launch_masked_key<T, TM, 2>(a, s); break;
    case 3: e = launch_masked_key<T, TM, 3>(a, s); break;
    case 4: e = launch_masked_key<T, TM, 4>(a, s); break;
    case 5: e = launch_masked_key<T, TM, 5>(a, s); break;
    default: return cudaErrorInvalidValue;
    }
    if(e != cudaSuccess) { return e; }
  }
  else switch(R)
  {
  case 1: k_cps_masked<T, TM, 1><<<grid, 256, 0, s>>>(a); break;
  case 2: k_cps_masked<T, TM, 2><<<grid, 256, 0, s>>>(a); break;
  case 3: k_cps_masked<T, TM, 3><<<grid, 256, 0, s>>>(a); break;
  case 4: k_cps_masked<T, TM, 4><<<grid, 256, 0, s>>>(a); break;
  case 5: k_cps_masked<T, TM, 5><<<grid, 256, 0, s>>>(a); break;
  default: return cudaErrorInvalidValue;
  }
  pipe.prof_end(s, QMIV_STAGE_CPS, tok);
  tok = pipe.prof_begin(s);
  k_mask_finalize<<<9, 256, 0, s>>>(a);
  pipe.prof_end(s, QMIV_STAGE_FINALIZE, tok);
  return cudaGetLastError();
}

// xPSNR::CalcPSNRfromMaskedSSD, xPSNR.cpp:198-205: MAX = NumNonMasked * MaxPic^2 * MaxMsk in int64
double psnr_masked(double ssd, int32_t nnm, int32_t bitdepth_pic, int32_t bitdepth_msk)
{
  const uint64_t mp = (uint64_t)((1 << bitdepth_pic) - 1), mm = (uint64_t)((1 << bitdepth_msk) - 1);
  const int64_t  MAX = (int64_t)((uint64_t)(int64_t)nnm * (mp * mp) * mm);
  return ssd > 0 ? 10.0 * log10((double)MAX / ssd) : DBL_MAX;
}

}  // namespace

// ---- host side, shared by the one-pair call and the batched form ---------------------------------
// ERP row weights and their correction for one height and latitude range (xWeightedSpherically.cpp:13-29),
// computed once per process: mask-mode calls plan every call, and the weights depend on these two only.
void ws_weights_cached(int32_t H, int32_t lat_range, std::vector<double>& w, double& correction)
{
  static std::mutex mu;
  static std::map<std::pair<int32_t, int32_t>, std::pair<std::vector<double>, double>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto it = cache.find(std::make_pair(H, lat_range));
  if(it == cache.end())
  {
    if(cache.size() >= 64) { cache.clear(); }
    std::pair<std::vector<double>, double> v;
    ws_weights(H, lat_range, v.first, v.second);
    it = cache.emplace(std::make_pair(H, lat_range), std::move(v)).first;
  }
  w = it->second.first;
  correction = it->second.second;
}

qmiv_status plan_masked(const Shape& S, const qmiv_params& prm, const qmiv_frame* mask, int32_t mask_bitdepth, MaskPlan& P)
{
  if(mask_bitdepth < 8 || mask_bitdepth > 14) { return fail(QMIV_ERR_INVALID_ARG, "mask bit depth must be in 8..14"); }
  if(!mask || !mask->plane[0]) { return fail(QMIV_ERR_INVALID_ARG, "mask plane is null"); }
  if(mask->mem != QMIV_MEM_HOST && mask->mem != QMIV_MEM_DEVICE) { return fail(QMIV_ERR_INVALID_ARG, "mask mem must be QMIV_MEM_HOST or QMIV_MEM_DEVICE"); }
  P.mesz = mask_bitdepth <= 8 ? 1 : 2;
  const size_t mrow = (size_t)S.W * P.mesz;
  if(mask->pitch[0] < (int64_t)mrow || (mask->pitch[0] % (int64_t)P.mesz) != 0) { return fail(QMIV_ERR_INVALID_ARG, "bad mask pitch"); }
  if(S.bitdepth > 14) { return fail(QMIV_ERR_UNSUPPORTED, "mask mode needs bit depth <= 14"); }
  P.S = S;
  P.prm = prm;
  P.mbd = mask_bitdepth;
  for(int c = 0; c < 4; c++) { P.maxdiff[c] = round_f32_half_away(prm.unc[c] * (float)S.maxv); }   // xGlobClrDiff.cpp:76
  // the key search needs samples in range (STOP fails on any other, CNCL clips), the fp32 exactness of
  // the unmasked search, 2^23 + B <= 2^24 - 2 with B = sum_c w_c (Max + MaxDiff_c)^2, the bound of every
  // error (so that the masked sentinel 2^24 - 1 is above every real value), and every squared
  // difference below 2^24 (its row sums split the terms into two 32-bit parts)
  int64_t bound = 0, dmax2 = 0;
  for(int c = 0; c < 3; c++)
  {
    const int64_t m = (int64_t)S.maxv + std::abs((int64_t)P.maxdiff[c]);
    bound += (int64_t)prm.cws[c] * m * m;
    dmax2 = std::max(dmax2, m * m);
  }
  P.key = (prm.invalid_pel_action == QMIV_PEL_STOP || prm.invalid_pel_action == QMIV_PEL_CNCL) &&
          cps_fp32_exact(S.maxv, prm.cws, P.maxdiff) && ((int64_t)1 << 23) + bound <= ((int64_t)1 << 24) - 2 &&
          dmax2 < ((int64_t)1 << 24);
  P.ws.clear();
  P.ws_corr = 1.0;
  if(prm.erp) { ws_weights_cached(S.H, prm.lat_range_deg, P.ws, P.ws_corr); }
  return QMIV_OK;
}

qmiv_status resolve_mask(const MaskPlan& P, const qmiv_frame* mask, char* staging, MaskArgs& a, cudaStream_t s)
{
  const size_t mrow = (size_t)P.S.W * P.mesz;
  if(mask->mem == QMIV_MEM_DEVICE)
  {
    a.mask = mask->plane[0];
    a.mpitch = (int32_t)(mask->pitch[0] / (int64_t)P.mesz);
    return QMIV_OK;
  }
  if(!staging) { return fail(QMIV_ERR_INVALID_ARG, "mask staging not prepared"); }
  QMIV_CUDA(cudaMemcpy2DAsync(staging, mrow, mask->plane[0], (size_t)mask->pitch[0], mrow, P.S.H, cudaMemcpyHostToDevice, s));
  a.mask = staging;
  a.mpitch = P.S.W;
  return QMIV_OK;
}

void fill_mask_args(const MaskPlan& P, const Img& a0, const Img& a1, uint64_t* rows, const double* ws, MaskOut* out, MaskArgs& a)
{
  const Shape& S = P.S;
  a.in0 = a0; a.in1 = a1;
  a.W = S.W; a.H = S.H;
  a.clip = P.prm.invalid_pel_action == QMIV_PEL_CNCL ? (uint32_t)S.maxv : 0xffffu;
  a.maxv = S.maxv; a.mask_max = (1 << P.mbd) - 1;
  for(int c = 0; c < 4; c++) { a.maxdiff[c] = P.maxdiff[c]; }
  for(int c = 0; c < 3; c++) { a.cws[c] = P.prm.cws[c]; }
  a.row_ssd = rows;
  a.row_cps = rows + (size_t)3 * S.H;
  a.ws = P.prm.erp ? ws : nullptr;
  a.out = out;
  a.kscale = 128u;
  auto al = [](const void* q, size_t n) { return (reinterpret_cast<uintptr_t>(q) % n) == 0; };
  bool ok = a.mask != nullptr && a.mpitch % 2 == 0 && al(a.mask, 2 * P.mesz);
  for(const Img* im : { &a.in0, &a.in1 })
  {
    ok = ok && im->sx[0] == 0 && im->sy[0] == 0 && im->pitch[0] % 2 == 0 && al(im->p[0], 2 * S.esz);
    for(int c = 1; c < 3; c++) { ok = ok && im->sx[c] == 1 && im->sy[c] == 1; }
  }
  a.pairs420 = ok ? 1 : 0;
}

qmiv_status masked_status(const MaskOut& o, const MaskPlan& P)
{
  if(P.prm.invalid_pel_action == QMIV_PEL_STOP && (o.flags & 3))
  {
    return fail(QMIV_ERR_INVALID_PIXEL, "input frame contains samples above the bit depth's maximum");
  }
  if(o.nnm == 0) { return fail(QMIV_ERR_INVALID_ARG, "the mask has no non-zero sample"); }
  return QMIV_OK;
}

// dB values with the reference's arithmetic and conventions
void finish_masked(const MaskOut& o, const MaskPlan& P, uint32_t metrics, qmiv_result* out)
{
  const Shape& S = P.S;
  const qmiv_params& prm = P.prm;
  std::memset(out, 0, sizeof(*out));
  const int64_t area = (int64_t)S.W * S.H;
  const int32_t bd = S.bitdepth, mbd = P.mbd;
  for(int c = 0; c < 4; c++) { out->gcd_r2t[c] = o.gcd[c]; }
  for(int c = 0; c < 3; c++)
  {
    out->exact[c] = o.differs[c] == 0;
    out->ssd[c] = o.ssd[c];
    out->cps_sse_r2t[c] = o.cps_sum[0][c];
    out->cps_sse_t2r[c] = o.cps_sum[1][c];
  }
  out->invalid_pel[0] = (o.flags & 1) != 0;
  out->invalid_pel[1] = (o.flags & 2) != 0;
  const double fake = psnr_from_ssd(1, area, bd);          // getFakePSNR(area, picture bit depth), xAppQMIV.cpp:976
  const int32_t* cwa = prm.cwa;
  const double inv = 1.0 / (double)(cwa[0] + cwa[1] + cwa[2] + cwa[3]);
  auto per_pic3 = [&](const double v[4]) { return (v[0] * cwa[0] + v[1] * cwa[1] + v[2] * cwa[2]) * inv; };   // xMetricQMIV.cpp:91-97
  if(metrics & QMIV_PSNR)                                     // xPSNR.cpp:54-66: the mask's bit depth for both
  {
    for(int c = 0; c < 3; c++) { out->psnr[c] = out->exact[c] ? fake : psnr_masked((double)o.ssd[c], o.nnm, mbd, mbd); }
    out->psnr_pic = per_pic3(out->psnr);
  }
  if(metrics & QMIV_WSPSNR)                                   // xWSPSNR.cpp:51-77, :108-133
  {
    for(int c = 0; c < 3; c++)
    {
      const double v = prm.erp ? psnr_masked(o.ws_err[c] * P.ws_corr, o.nnm, bd, mbd) : psnr_masked((double)o.ssd[c], o.nnm, mbd, mbd);
      out->wspsnr[c] = out->exact[c] ? fake : v;
    }
    out->wspsnr_pic = per_pic3(out->wspsnr);
  }
  if(metrics & QMIV_IVPSNR)                                   // xIVPSNR.cpp:153-200
  {
    double q[2];
    for(int d = 0; d < 2; d++)
    {
      double qc[4] = { 0, 0, 0, 0 };
      for(int c = 0; c < 3; c++)
      {
        const double err = prm.erp ? o.cps_ws[d][c] : (double)o.cps_sum[d][c];
        qc[c] = psnr_masked(err > 0 ? err : 1.0, o.nnm, bd, mbd);
      }
      q[d] = (qc[0] * (double)cwa[0] + qc[1] * (double)cwa[1] + qc[2] * (double)cwa[2] + qc[3] * (double)cwa[3]) * inv;
    }
    out->ivpsnr_r2t = q[0]; out->ivpsnr_t2r = q[1];
    out->ivpsnr = (q[1] < q[0]) ? q[1] : q[0];
  }
}

MaskedPipeline::~MaskedPipeline()
{
  if(h_out_) { cudaFreeHost(h_out_); }
}

qmiv_status MaskedPipeline::run(qmiv_calc_s* calc, const qmiv_frame* in0, const qmiv_frame* in1, const qmiv_frame* mask,
                                int32_t mask_bitdepth, uint32_t metrics, qmiv_result* out, int32_t* num_non_masked)
{
  PairPipeline& pipe = calc->pipe;
  const Shape& S = pipe.shape();
  cudaStream_t s = calc->stream;
  MaskPlan P;
  QMIV_TRY(plan_masked(S, calc->prm, mask, mask_bitdepth, P));
  const bool host = in0->mem == QMIV_MEM_HOST || in1->mem == QMIV_MEM_HOST;
  QMIV_TRY(pipe.prepare(QMIV_PSNR, false, host));           // staging for host frames, ERP weights on the device
  Img a0{}, a1{};
  QMIV_TRY(pipe.resolve(in0, 0, a0, s));
  QMIV_TRY(pipe.resolve(in1, 1, a1, s));
  QMIV_TRY(out_.ensure(calc->ctx, sizeof(MaskOut)));
  QMIV_TRY(rows_.ensure(calc->ctx, (size_t)9 * S.H * sizeof(uint64_t)));
  if(!h_out_) { QMIV_CUDA(cudaMallocHost(&h_out_, sizeof(MaskOut))); }
  MaskArgs a{};
  if(mask->mem == QMIV_MEM_HOST) { QMIV_TRY(stage_.ensure(calc->ctx, (size_t)S.W * P.mesz * S.H)); }
  QMIV_TRY(resolve_mask(P, mask, stage_.as<char>(), a, s));
  fill_mask_args(P, a0, a1, rows_.as<uint64_t>(), pipe.ws_device(), out_.as<MaskOut>(), a);
  QMIV_CUDA(cudaMemsetAsync(out_.p, 0, sizeof(MaskOut), s));
  QMIV_CUDA(cudaMemsetAsync(a.row_cps, 0, (size_t)6 * S.H * sizeof(uint64_t), s));
  const int R = P.prm.search_range;
  cudaError_t e;
  if(S.esz == 1) { e = P.mesz == 1 ? launch_masked_t<uint8_t, uint8_t>(a, R, P.key, pipe, s) : launch_masked_t<uint8_t, uint16_t>(a, R, P.key, pipe, s); }
  else { e = P.mesz == 1 ? launch_masked_t<uint16_t, uint8_t>(a, R, P.key, pipe, s) : launch_masked_t<uint16_t, uint16_t>(a, R, P.key, pipe, s); }
  if(e != cudaSuccess) { return cuda_fail(e, "masked launches"); }
  const int tok = pipe.prof_begin(s);
  QMIV_CUDA(cudaMemcpyAsync(h_out_, out_.p, sizeof(MaskOut), cudaMemcpyDeviceToHost, s));
  pipe.prof_end(s, QMIV_STAGE_D2H, tok);
  QMIV_CUDA(cudaStreamSynchronize(s));
  pipe.harvest_profile();
  const MaskOut& o = *static_cast<const MaskOut*>(h_out_);
  QMIV_TRY(masked_status(o, P));
  if(num_non_masked) { *num_non_masked = o.nnm; }
  if(out) { finish_masked(o, P, metrics, out); }
  return QMIV_OK;
}

// ---- batched form ---------------------------------------------------------------------------------
namespace {

constexpr size_t kMaskAlign = 256;
inline size_t malign(size_t v) { return (v + kMaskAlign - 1) & ~(kMaskAlign - 1); }

// form: 1 = vector loads, 0 = generic
template <typename T, typename TM>
cudaError_t launch_prepass_group(const MaskPack& pk, int count, int max_h, int form, cudaStream_t s)
{
  const dim3 grid(form == 1 ? prepass420_units<TM>(max_h) : max_h, count);
  if(form == 1) { k_mask_prepass_multi<T, TM, true><<<grid, 256, 0, s>>>(pk); }
  else { k_mask_prepass_multi<T, TM, false><<<grid, 256, 0, s>>>(pk); }
  return cudaSuccess;
}

template <typename T, typename TM, int R>
cudaError_t launch_search_group_r(const MaskPack& pk, int count, int max_w, int max_h, bool key, cudaStream_t s)
{
  if(key)
  {
    using G = MaskKeyGeo<R>;
    const cudaError_t e = smem_attr_once(k_cps_masked_key_multi<T, TM, R>, (int)G::kSmem);
    if(e != cudaSuccess) { return e; }
    const dim3 grid((max_w + G::TW - 1) / G::TW, (max_h + G::TH - 1) / G::TH, count);
    k_cps_masked_key_multi<T, TM, R><<<grid, 512, G::kSmem, s>>>(pk);
  }
  else
  {
    const dim3 grid((max_w + 31) / 32, (max_h + 7) / 8, 2 * count);
    k_cps_masked_multi<T, TM, R><<<grid, 256, 0, s>>>(pk);
  }
  return cudaSuccess;
}

template <typename T, typename TM>
cudaError_t launch_search_group(const MaskPack& pk, int count, int max_w, int max_h, int R, bool key, cudaStream_t s)
{
  switch(R)
  {
  case 1: return launch_search_group_r<T, TM, 1>(pk, count, max_w, max_h, key, s);
  case 2: return launch_search_group_r<T, TM, 2>(pk, count, max_w, max_h, key, s);
  case 3: return launch_search_group_r<T, TM, 3>(pk, count, max_w, max_h, key, s);
  case 4: return launch_search_group_r<T, TM, 4>(pk, count, max_w, max_h, key, s);
  case 5: return launch_search_group_r<T, TM, 5>(pk, count, max_w, max_h, key, s);
  default: return cudaErrorInvalidValue;
  }
}

struct GroupInfo
{
  std::vector<int32_t> pairs;
};

}  // namespace

MaskedBatch::~MaskedBatch()
{
  if(h_) { cudaFreeHost(h_); }
}

// One call: plans every pair (as the one-pair call does), lays out one device arena (results, row
// sums, ERP weights, host-frame and host-mask staging, the argument table and the groups' pair
// indices), copies the tables with one H2D, launches prepass / reduce / search / finalize each once per
// group, and reads every pair's result block back with one D2H.
qmiv_status MaskedBatch::run(qmiv_ctx_s* ctx, const qmiv_params& prm0, cudaStream_t s, const qmiv_pair_desc* pairs,
                             const qmiv_frame* masks, const int32_t* mask_bitdepths, int32_t n, qmiv_result* out,
                             int32_t* num_non_masked)
{
  std::vector<MaskPlan> P(n);
  size_t off_out = 0, off_rows = malign(sizeof(MaskOut) * n), cur = 0;
  std::vector<size_t> o_rows(n), o_stage(n), o_mstage(n);
  cur = off_rows;
  for(int i = 0; i < n; i++)
  {
    const qmiv_pair_desc& d = pairs[i];
    if((d.metric_mask & ~(uint32_t)(QMIV_PSNR | QMIV_WSPSNR | QMIV_IVPSNR)) != 0 || d.metric_mask == 0)
    {
      return fail(QMIV_ERR_UNSUPPORTED, "mask mode computes PSNR, WS-PSNR and IV-PSNR only (as the reference)");
    }
    Shape S;
    QMIV_TRY(S.init(d.width, d.height, d.bitdepth, d.chroma_format));
    qmiv_params prm = prm0;
    prm.search_range = d.search_range;
    QMIV_TRY(validate_params(prm));
    QMIV_TRY(plan_masked(S, prm, &masks[i], mask_bitdepths[i], P[i]));
    o_rows[i] = cur; cur += malign(sizeof(uint64_t) * 9 * S.H);
    const bool host = d.in0.mem == QMIV_MEM_HOST || d.in1.mem == QMIV_MEM_HOST;
    o_stage[i] = cur; cur += host ? malign(2 * S.staged_frame_bytes()) : 0;
    o_mstage[i] = cur; cur += masks[i].mem == QMIV_MEM_HOST ? malign((size_t)S.W * P[i].mesz * S.H) : 0;
  }
  // groups: prepass by (sample sizes, prepass form), search by (sample sizes, R, search form)
  std::map<std::tuple<int, int, int>, GroupInfo> pre;
  std::map<std::tuple<int, int, int, int>, GroupInfo> srch;
  const size_t total = cur;
  QMIV_TRY(arena_.ensure(ctx, total));
  const size_t hbytes = sizeof(MaskOut) * n;
  if(h_bytes_ < hbytes)
  {
    if(h_) { cudaFreeHost(h_); h_ = nullptr; h_bytes_ = 0; }
    QMIV_CUDA(cudaMallocHost(&h_, hbytes));
    h_bytes_ = hbytes;
  }
  char* dbase = arena_.as<char>();
  std::vector<MaskArgs> hargs(n);
  MaskOut* hout = static_cast<MaskOut*>(h_);
  QMIV_CUDA(cudaMemsetAsync(dbase, 0, total, s));          // results and row sums start at zero
  for(int i = 0; i < n; i++)
  {
    const MaskPlan& p = P[i];
    const Shape& S = p.S;
    char* stage = dbase + o_stage[i];
    Img a0{}, a1{};
    QMIV_TRY(resolve_frame(S, &pairs[i].in0, stage, a0, s));
    QMIV_TRY(resolve_frame(S, &pairs[i].in1, stage + S.staged_frame_bytes(), a1, s));
    MaskArgs& a = hargs[i];
    a = MaskArgs{};
    QMIV_TRY(resolve_mask(p, &masks[i], dbase + o_mstage[i], a, s));
    // ERP row weights: one device copy per (height, latitude range), uploaded on first use
    double* ws = nullptr;
    if(p.prm.erp)
    {
      DevMem& wd = ws_dev_[std::make_pair(S.H, p.prm.lat_range_deg)];
      if(!wd.p)
      {
        QMIV_TRY(wd.alloc(ctx, sizeof(double) * S.H));
        QMIV_CUDA(cudaMemcpy(wd.p, p.ws.data(), sizeof(double) * S.H, cudaMemcpyHostToDevice));
      }
      ws = wd.as<double>();
    }
    fill_mask_args(p, a0, a1, reinterpret_cast<uint64_t*>(dbase + o_rows[i]), ws,
                   reinterpret_cast<MaskOut*>(dbase + off_out) + i, a);
    const int t = (int)S.esz, tm = (int)p.mesz;
    const int form = mask_prepass_vec_ok(a, S.esz, p.mesz) ? 1 : 0;
    pre[std::make_tuple(t, tm, form)].pairs.push_back(i);
    srch[std::make_tuple(t, tm, p.prm.search_range, (int)p.key)].pairs.push_back(i);
  }
  // launches over chunks of up to kPackPairs pairs, each chunk's arguments in the launch's parameters
  std::vector<int32_t> all(n);
  for(int i = 0; i < n; i++) { all[i] = i; }
  MaskPack pk{};
  pk.kscale = 128u;
  int max_w = 0, max_h = 0;
  auto pack = [&](const std::vector<int32_t>& ids, size_t first) -> int {
    const int cnt = (int)std::min(ids.size() - first, (size_t)kPackPairs);
    max_w = 0; max_h = 0;
    for(int j = 0; j < cnt; j++)
    {
      pk.a[j] = hargs[ids[first + j]];
      max_w = std::max(max_w, pk.a[j].W); max_h = std::max(max_h, pk.a[j].H);
    }
    return cnt;
  };
  int tok = clock_.begin(ctx, s);
  for(auto& g : pre)
  {
    const int t = std::get<0>(g.first), tm = std::get<1>(g.first), form = std::get<2>(g.first);
    for(size_t f = 0; f < g.second.pairs.size(); f += kPackPairs)
    {
      const int cnt = pack(g.second.pairs, f);
      cudaError_t e;
      if(t == 1) { e = tm == 1 ? launch_prepass_group<uint8_t, uint8_t>(pk, cnt, max_h, form, s) : launch_prepass_group<uint8_t, uint16_t>(pk, cnt, max_h, form, s); }
      else { e = tm == 1 ? launch_prepass_group<uint16_t, uint8_t>(pk, cnt, max_h, form, s) : launch_prepass_group<uint16_t, uint16_t>(pk, cnt, max_h, form, s); }
      if(e != cudaSuccess) { return cuda_fail(e, "masked prepass launch"); }
    }
  }
  clock_.end(s, QMIV_STAGE_PREPASS, tok);
  tok = clock_.begin(ctx, s);
  for(size_t f = 0; f < all.size(); f += kPackPairs) { const int cnt = pack(all, f); k_mask_reduce_multi<<<cnt, 32, 0, s>>>(pk); }
  clock_.end(s, QMIV_STAGE_REDUCE, tok);
  tok = clock_.begin(ctx, s);
  for(auto& g : srch)
  {
    const int t = std::get<0>(g.first), tm = std::get<1>(g.first), R = std::get<2>(g.first);
    const bool key = std::get<3>(g.first) != 0;
    for(size_t f = 0; f < g.second.pairs.size(); f += kPackPairs)
    {
      const int cnt = pack(g.second.pairs, f);
      cudaError_t e;
      if(t == 1) { e = tm == 1 ? launch_search_group<uint8_t, uint8_t>(pk, cnt, max_w, max_h, R, key, s) : launch_search_group<uint8_t, uint16_t>(pk, cnt, max_w, max_h, R, key, s); }
      else { e = tm == 1 ? launch_search_group<uint16_t, uint8_t>(pk, cnt, max_w, max_h, R, key, s) : launch_search_group<uint16_t, uint16_t>(pk, cnt, max_w, max_h, R, key, s); }
      if(e != cudaSuccess) { return cuda_fail(e, "masked search launch"); }
    }
  }
  clock_.end(s, QMIV_STAGE_CPS, tok);
  tok = clock_.begin(ctx, s);
  for(size_t f = 0; f < all.size(); f += kPackPairs) { const int cnt = pack(all, f); k_mask_finalize_multi<<<9 * cnt, 256, 0, s>>>(pk); }
  clock_.end(s, QMIV_STAGE_FINALIZE, tok);
  QMIV_CUDA(cudaGetLastError());
  tok = clock_.begin(ctx, s);
  QMIV_CUDA(cudaMemcpyAsync(hout, dbase + off_out, sizeof(MaskOut) * n, cudaMemcpyDeviceToHost, s));
  clock_.end(s, QMIV_STAGE_D2H, tok);
  QMIV_CUDA(cudaStreamSynchronize(s));
  clock_.harvest(ctx);
  qmiv_status first = QMIV_OK;
  for(int i = 0; i < n; i++)
  {
    const qmiv_status st = masked_status(hout[i], P[i]);
    if(st != QMIV_OK && first == QMIV_OK) { first = st; }
    if(num_non_masked) { num_non_masked[i] = hout[i].nnm; }
    if(out) { finish_masked(hout[i], P[i], pairs[i].metric_mask, &out[i]); }
  }
  return first;
}

}  // namespace qmiv

extern "C" qmiv_status qmiv_frame_pair_compute_masked(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1,
                                                      const qmiv_frame* mask, int32_t mask_bitdepth, uint32_t metric_mask,
                                                      qmiv_result* out, int32_t* num_non_masked)
{
  using namespace qmiv;
  if(!calc || !in0 || !in1 || !mask) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  if(calc->pending) { return fail(QMIV_ERR_BUSY, "a submission is already in flight on this calc"); }
  if((metric_mask & ~(uint32_t)QMIV_ALL) != 0) { return fail(QMIV_ERR_INVALID_ARG, "unknown metric bits"); }
  if(metric_mask & ~(uint32_t)(QMIV_PSNR | QMIV_WSPSNR | QMIV_IVPSNR))
  {
    return fail(QMIV_ERR_UNSUPPORTED, "mask mode computes PSNR, WS-PSNR and IV-PSNR only (as the reference)");
  }
  QMIV_CUDA(cudaSetDevice(calc->ctx->device));
  if(!calc->masked) { calc->masked.reset(new MaskedPipeline()); }
  return calc->masked->run(calc, in0, in1, mask, mask_bitdepth, metric_mask, out, num_non_masked);
}
