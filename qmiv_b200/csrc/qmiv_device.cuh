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

// Exact IEEE double operations, never contracted into FMA, so device results equal the host
// reference's separately rounded operations bit for bit.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Kahan-Babuska-Neumaier compensated sum (libs/pmbb-core/src/xKBNS.h:36-43).
struct Kbns
{
  double s = 0.0, c = 0.0;
  __device__ __forceinline__ void add(double v)
  {
    const double t = dadd(s, v);
    if(fabs(s) >= fabs(v)) { c = dadd(c, dadd(dsub(s, t), v)); }
    else                   { c = dadd(c, dadd(dsub(v, t), s)); }
    s = t;
  }
  __device__ __forceinline__ double result() const { return dadd(s, c); }
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
  int32_t  flags;            // bit0: frame0 invalid, bit1: frame1 invalid, bit2: integer CPS path
  uint32_t max_sample[2];
  int64_t  sd[3];            // 4:4:4 totals of In1 - In0
  uint64_t ssd[3];           // 4:4:4 totals
  double   ws_ssd[3];        // KBNS over rows of rowSSD*w[y] (WS-PSNR, before correction)
  uint64_t cps_sum[2][3];    // sum over rows of sign-extended 32-bit row sums, [R2T, T2R]
  double   cps_ws[2][3];     // KBNS over rows of rowSSE*w[y]
  double   ssim[kMaxSsimSlots][3];
};

}  // namespace qmiv
