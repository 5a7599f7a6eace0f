// Device-side building blocks shared by the QMIV kernels (sm_100a).
//
// Data layout in HBM: frames stay in their native planar layout (Y, Cb, Cr; 1 byte per sample up
// to 8 bits, else 2 bytes). Chroma of 4:2:0/4:2:2 is never upsampled into a buffer: every consumer
// reads sample (x >> sx, y >> sy) of the chroma plane, which is exactly the 2x2 (or 2x1) nearest
// replication of the reference loader (libs/pmbb-core/src/xPixelOpsSTD.cpp:30-49, :68-87).
// Out-of-picture reads clamp the coordinate, which equals the reference's edge-replicated margin
// (margin = roundUp(R,2) >= R, apps/QMIV/src/xAppQMIV.cpp:353, extend(Nearest) at :899).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace qmiv {

// A planar picture as the kernels see it. Pitches are in elements of the sample type.
struct Img
{
  const void* p[3];
  int32_t     pitch[3];
  int8_t      sx[3], sy[3];   // chroma subsampling shifts per component (0 for luma / 4:4:4)
};

struct MutImg
{
  void*   p[3];
  int32_t pitch[3];
};

template <typename T>
__device__ __forceinline__ int32_t fetch(const Img& im, int c, int32_t x, int32_t y)
{
  const T* base = static_cast<const T*>(im.p[c]);
  return (int32_t)__ldg(base + (size_t)(y >> im.sy[c]) * im.pitch[c] + (x >> im.sx[c]));
}

__device__ __forceinline__ int32_t clampi(int32_t v, int32_t lo, int32_t hi) { return min(max(v, lo), hi); }
// The int32 product of the reference's integer code where it may wrap (two's complement), formed in
// unsigned arithmetic: a signed overflow is undefined in C++ and lets the compiler widen the product.
__device__ __forceinline__ int32_t mul_wrap(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }

// Exact conversions between integers in [0, 2^23) and floats without the (quarter-rate) conversion
// pipe: a float in [2^23, 2^24) has a unit ulp, so its low mantissa bits are the integer.
__device__ __forceinline__ float u2f_exact(uint32_t v) { return __uint_as_float(v | 0x4B000000u) - 8388608.0f; }
__device__ __forceinline__ int32_t f2i_exact(float f) { return (int32_t)(__float_as_uint(f + 8388608.0f) - 0x4B000000u); }

// Exact IEEE double operations, never contracted into FMA, so device results equal the host
// reference's separately rounded operations bit for bit.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Kahan-Babuska-Neumaier compensated sum (libs/pmbb-core/src/xKBNS.h:36-43).
// The reference adds to c the rounding error of s + v, computed by Fast2Sum with the larger of the
// two operands first: (big - t) + small. Here the operands are chosen by a compare and two selects
// instead of a branch, four FP64 additions and one FP64 compare per term (Knuth's branch-free TwoSum,
// which yields the same exactly representable error, takes six additions).
struct Kbns
{
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v)
  {
    const double t = dadd(s, v);
    const bool   sb = fabs(s) >= fabs(v);
    const double big = sb ? s : v, small = sb ? v : s;
    c = dadd(c, dadd(dsub(big, t), small));
    s = t;
  }
  __device__ __forceinline__ double result() const { return dadd(s, c); }
};

// SSIM of one window (xStructSimSTD.cpp:420-461, same operation order; AVX-512 CalcBlckAvg8 /
// CalcMultiBlckAvg8S4 give the same per-window value) from its moments divided by the window area:
// ar = SumR / 64, at = SumT / 64, qr = SumR2 / 64, qt = SumT2 / 64, qrt = SumRT / 64 (all exact).
// 2 x is formed as x + x, which is the same double.
__device__ __forceinline__ double ssim_window_avg(double ar, double at, double qr, double qt, double qrt, double C1,
                                                  double C2, bool calc_l)
{
  const double ar2 = dmul(ar, ar), at2 = dmul(at, at);
  const double var_r = dsub(qr, ar2);
  const double var_t = dsub(qt, at2);
  const double cov   = dsub(qrt, dmul(ar, at));
  const double cs    = ddiv(dadd(dadd(cov, cov), C2), dadd(dadd(var_r, var_t), C2));
  if(!calc_l) { return cs; }
  const double l = ddiv(dadd(dmul(dadd(ar, ar), at), C1), dadd(dadd(ar2, at2), C1));
  return dmul(l, cs);
}

// 4x4 sub-block moments of an SSIM picture pair, five uint32 planes per component:
// [c][m][nby][pitch], m = 0: sum a, 1: sum b, 2: sum a^2, 3: sum b^2, 4: sum a*b
// (a = the "Tst" picture, b = the "Ref" picture of xSSIM::xCalcPicSSIM). Every 8x8/stride-4 window is
// the sum of 2x2 sub-blocks, so window moments are exact integers.
struct Moments
{
  uint32_t* p;      // base of component 0, moment 0
  int32_t   nbx, nby, pitch;
  __host__ __device__ size_t plane() const { return (size_t)nby * pitch; }
};

// Round half away from zero by adding +-0.5 in double and truncating (xHelpersFLT.h:33).
__device__ __forceinline__ int32_t round_half_away(double v)
{
  const double t = dadd(v, copysign(0.5, v));
  return (int32_t)t;  // truncation toward zero, as cvttsd2si
}

// Per-pair device outputs consumed by the host finishing step.
constexpr int kMaxSsimSlots = 18;   // SSIM 1 + IV-SSIM 2 + MS-SSIM 5 + IV-MS-SSIM 2x5

struct PairOut
{
  int32_t  gcd[4];
  int32_t  flags;            // bit0: frame0 invalid, bit1: frame1 invalid, bit2: integer CPS path,
                             // bit3: a CPS tile load did not complete (bounded wait ran out)
  uint32_t max_sample[2];
  int64_t  sd[3];            // 4:4:4 totals of In1 - In0
  uint64_t ssd[3];           // 4:4:4 totals
  double   ws_ssd[3];        // KBNS over rows of rowSSD*w[y] (WS-PSNR, before correction)
  uint64_t cps_sum[2][3];    // sum over rows of sign-extended 32-bit row sums, [R2T, T2R]
  double   cps_ws[2][3];     // KBNS over rows of rowSSE*w[y]
  double   ssim[kMaxSsimSlots][3];
};

// ---- mbarriers and bulk copies ----------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_barrier_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile(
    "{\n\t.reg .pred p;\n\t"
    "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
    "selp.u32 %0, 1, 0, p;\n\t}"
    : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
  return ok != 0;
}
// Waits for the phase with the given parity; gives up (false) after about `limit` cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, long long limit)
{
  if(mbar_try_wait(bar, parity)) { return true; }
  const long long t0 = clock64();
  do
  {
    if(mbar_try_wait(bar, parity)) { return true; }
  } while(clock64() - t0 <= limit);
  return false;
}
}  // namespace qmiv
