// QMIV metric kernels for B200 (sm_100a).
//
// Pipeline of one frame pair (the reference runs the same steps per frame on the CPU,
// apps/QMIV/src/xAppQMIV.cpp:761-827):
//   k_prepass   per raw row: SD(In1-In0), SSD, max sample        (HBM bound, reads both frames once)
//   k_reduce    totals, GCD, exactness of the fp32 search path   (one CTA)
//   k_cps       corresponding-pixel-shift search, both directions in one pass; per-row SSE into
//               32-bit lanes, the IV-SSIM sub-block moments of (test, SCP) and, when IV-MS-SSIM or
//               the caller needs them, the shift-compensated pictures
//   k_ssim_*    (qmiv_ssim.cu) block SSIM from exact integer moments, FP64 windows, row sums
//   k_finalize  every order-dependent FP64 pooling chain of the pair (one CTA per chain)
#include "qmiv_kernels.cuh"

#include <cstdio>

namespace qmiv {

constexpr unsigned kFull = 0xffffffffu;

// =============================================================================================
// prepass
// =============================================================================================
template <typename T>
__global__ void __launch_bounds__(256) k_prepass(const __grid_constant__ PrepassArgs a)
{
  const int warp  = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
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
  for(int x = lane; x < n; x += 32)
  {
    uint32_t v0 = __ldg(p0 + x), v1 = __ldg(p1 + x);
    m0 = max(m0, v0); m1 = max(m1, v1);
    v0 = min(v0, a.clip); v1 = min(v1, a.clip);
    const int32_t d = (int32_t)v1 - (int32_t)v0;
    sd  += d;
    ssd += (uint64_t)((int64_t)d * d);
  }
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
cudaError_t launch_prepass(const PrepassArgs& a, cudaStream_t s)
{
  const int total  = a.rows[0] + a.rows[1] + a.rows[2];
  const int blocks = (total + 7) / 8;
  k_prepass<T><<<blocks, 256, 0, s>>>(a);
  return cudaGetLastError();
}
template cudaError_t launch_prepass<uint8_t>(const PrepassArgs&, cudaStream_t);
template cudaError_t launch_prepass<uint16_t>(const PrepassArgs&, cudaStream_t);

// =============================================================================================
// reduce: totals and GCD (libs/pmbb-ivqm/src/xGlobClrDiff.cpp:70-103)
// =============================================================================================
__global__ void __launch_bounds__(1024) k_reduce(const __grid_constant__ ReduceArgs a)
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

cudaError_t launch_reduce(const ReduceArgs& a, cudaStream_t s)
{
  k_reduce<<<1, 1024, 0, s>>>(a);
  return cudaGetLastError();
}

// =============================================================================================
// CPS search (libs/pmbb-ivqm/src/xCorrespPixelShiftSSE.cpp:18-127)
//
// Both pictures of a tile (plus an R-pixel halo, clamped) are staged in shared memory as
// float4 (Y, Cb, Cr, q + 2^23) with q = sum_c w_c * ref_c^2. For a test pixel s (test + GCD,
// unclipped) the weighted error of candidate r is e = sum_c w_c (s_c - r_c)^2, and
//     e - sum_c w_c s_c^2 + 2^23 = (q(r) + 2^23) + sum_c (-2 w_c s_c) r_c
// is three FFMAs. When every partial sum is an integer below 2^24 in magnitude (checked on the host
// from bit depth, weights and the GCD clip range) the FFMAs are exact, so the ordering of candidates
// and all ties are those of the reference's int32 error. The result lies in [2^20, 2^24), where the
// IEEE bit pattern grows with the value, so
//     key = ((bits - bits(2^20)) << 7) + k,   k = (dy+R)(2R+1) + (dx+R)  (raster index, < 128)
// orders candidates exactly as the reference's "first strict minimum in raster order" does, and the
// search is one unsigned min per candidate. Each thread owns P vertically adjacent pixels, so every
// staged reference pixel is reused by up to 2R+1 of them from registers.
//
// When the fp32 path is not exact (bit depth > 10, large weights, out-of-range samples) the same
// kernel runs an int32 search that mirrors the SSE path's wrap-around arithmetic literally.
// =============================================================================================
constexpr float    kBias    = 8388608.0f;   // 2^23
constexpr uint32_t kKeyBase = 0x49800000u;  // bit pattern of 2^20f

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
  }
  const int64_t lim = 1LL << 24;
  if(bias - e < (1LL << 20)) { return false; }       // key base
  if(bias + e >= lim) { return false; }
  if(bias + q + up >= lim) { return false; }         // partial sums of the FFMA chain
  if(bias - lo <= -lim) { return false; }
  return true;
}

template <int R, int P, typename T>
__global__ void __launch_bounds__(128) k_cps(const __grid_constant__ CpsArgs a)
{
  constexpr int D  = 2 * R + 1;
  constexpr int TX = 32, TY = 4;
  constexpr int TW = TX, TH = TY * P;
  constexpr int SW = TW + 2 * R, SH = TH + 2 * R;
  extern __shared__ float4 sm[];
  float4* const tile0 = sm;
  float4* const tile1 = sm + SH * SW;

  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int x0 = blockIdx.x * TW, y0 = blockIdx.y * TH;
  const int W = a.W, H = a.H;
  const int g0 = a.gcd_src->gcd[0], g1 = a.gcd_src->gcd[1], g2 = a.gcd_src->gcd[2];
  const bool int_path = (a.gcd_src->flags & 4) != 0;

  {
    const T* p0[2] = { static_cast<const T*>(a.in0.p[0]), static_cast<const T*>(a.in1.p[0]) };
    const T* p1[2] = { static_cast<const T*>(a.in0.p[1]), static_cast<const T*>(a.in1.p[1]) };
    const T* p2[2] = { static_cast<const T*>(a.in0.p[2]), static_cast<const T*>(a.in1.p[2]) };
    const int sx = a.in0.sx[1], sy = a.in0.sy[1];
    for(int i = threadIdx.x; i < SH * SW; i += TX * TY)
    {
      const int ly = i / SW, lx = i - ly * SW;
      const int gx = clampi(x0 + lx - R, 0, W - 1), gy = clampi(y0 + ly - R, 0, H - 1);
      const int cx = gx >> sx, cy = gy >> sy;
      #pragma unroll
      for(int f = 0; f < 2; f++)
      {
        const Img& im = f ? a.in1 : a.in0;
        const float v0 = u2f_exact(min((uint32_t)__ldg(p0[f] + gy * im.pitch[0] + gx), a.clip));
        const float v1 = u2f_exact(min((uint32_t)__ldg(p1[f] + cy * im.pitch[1] + cx), a.clip));
        const float v2 = u2f_exact(min((uint32_t)__ldg(p2[f] + cy * im.pitch[2] + cx), a.clip));
        const float q  = fmaf(a.wf[2], v2 * v2, fmaf(a.wf[1], v1 * v1, fmaf(a.wf[0], v0 * v0, kBias)));
        (f ? tile1 : tile0)[i] = make_float4(v0, v1, v2, q);
      }
    }
  }
  __syncthreads();

  #pragma unroll 1
  for(int dir = 0; dir < 2; dir++)
  {
    // dir 0 (R2T): test = In0 + GCD searched in In1 -> rows[0], SCP1 = clip(In1[best] - GCD)
    // dir 1 (T2R): test = In1 - GCD searched in In0 -> rows[1], SCP0 = clip(In0[best] + GCD)
    const float4* tst = dir ? tile1 : tile0;
    const float4* ref = dir ? tile0 : tile1;
    const int sg = dir ? -1 : 1;
    const int ga = sg * g0, gb = sg * g1, gc = sg * g2;

    uint32_t idx[P];
    if(!int_path)
    {
      float    c0[P], c1[P], c2[P];
      uint32_t best[P];
      #pragma unroll
      for(int i = 0; i < P; i++)
      {
        const float4 t = tst[(ty * P + i + R) * SW + tx + R];
        c0[i] = -2.0f * a.wf[0] * (t.x + (float)ga);
        c1[i] = -2.0f * a.wf[1] * (t.y + (float)gb);
        c2[i] = -2.0f * a.wf[2] * (t.z + (float)gc);
        best[i] = 0xffffffffu;
      }
      #pragma unroll
      for(int dxi = 0; dxi < D; dxi++)
      {
        #pragma unroll
        for(int ry = 0; ry < P + 2 * R; ry++)
        {
          const float4 r = ref[(ty * P + ry) * SW + tx + dxi];
          #pragma unroll
          for(int i = 0; i < P; i++)
          {
            const int dyi = ry - i;
            if(dyi >= 0 && dyi < D)
            {
              const float    e   = fmaf(c2[i], r.z, fmaf(c1[i], r.y, fmaf(c0[i], r.x, r.w)));
              const uint32_t key = (__float_as_uint(e) << 7) + (uint32_t)(dyi * D + dxi) - (kKeyBase << 7);
              best[i] = min(best[i], key);
            }
          }
        }
      }
      #pragma unroll
      for(int i = 0; i < P; i++) { idx[i] = min(best[i] & 127u, (uint32_t)(D * D - 1)); }
    }
    else
    {
      #pragma unroll 1
      for(int i = 0; i < P; i++)
      {
        const float4 t = tst[(ty * P + i + R) * SW + tx + R];
        const int s0 = (int)t.x + ga, s1 = (int)t.y + gb, s2 = (int)t.z + gc;
        int32_t  best_err = 0x7fffffff;
        uint32_t bi = 0;
        for(int dyi = 0; dyi < D; dyi++)
        {
          for(int dxi = 0; dxi < D; dxi++)
          {
            const float4   r  = ref[(ty * P + i + dyi) * SW + tx + dxi];
            const uint32_t d0 = (uint32_t)(s0 - (int)r.x), d1 = (uint32_t)(s1 - (int)r.y), d2 = (uint32_t)(s2 - (int)r.z);
            const uint32_t err = d0 * d0 * (uint32_t)a.wi[0] + d1 * d1 * (uint32_t)a.wi[1] + d2 * d2 * (uint32_t)a.wi[2];
            if((int32_t)err < best_err) { best_err = (int32_t)err; bi = (uint32_t)(dyi * D + dxi); }
          }
        }
        idx[i] = bi;
      }
    }

    // epilogue: winner's per-component squared difference into the row sums, SCP store, and the
    // SSIM moments of (test picture, SCP) per 4x4 sub-block (4 rows of a thread x 4 lanes)
    uint32_t* rows = a.rows + (size_t)dir * H * 3;
    T* scp = static_cast<T*>(dir ? a.scp0 : a.scp1);
    const Moments mom = a.mom[dir];
    const size_t plane = (size_t)W * H;
    const int x = x0 + tx;
    static_assert(P % 4 == 0, "rows per thread must cover whole 4x4 sub-blocks");
    uint32_t mm[P / 4][3][5];
    #pragma unroll
    for(int q = 0; q < P / 4; q++)
      #pragma unroll
      for(int c = 0; c < 3; c++)
        #pragma unroll
        for(int m = 0; m < 5; m++) { mm[q][c][m] = 0u; }
    #pragma unroll
    for(int i = 0; i < P; i++)
    {
      const int y = y0 + ty * P + i;
      const bool valid = (x < W) && (y < H);
      const int dyi = (int)(idx[i] / D), dxi = (int)(idx[i] - dyi * D);
      const float4 r = ref[(ty * P + i + dyi) * SW + tx + dxi];
      const float4 t = tst[(ty * P + i + R) * SW + tx + R];
      const int r0 = f2i_exact(r.x), r1 = f2i_exact(r.y), r2 = f2i_exact(r.z);
      const int t0 = f2i_exact(t.x), t1 = f2i_exact(t.y), t2 = f2i_exact(t.z);
      const uint32_t e0 = (uint32_t)(t0 + ga - r0), e1 = (uint32_t)(t1 + gb - r1), e2 = (uint32_t)(t2 + gc - r2);
      const uint32_t s0 = __reduce_add_sync(kFull, valid ? e0 * e0 : 0u);
      const uint32_t s1 = __reduce_add_sync(kFull, valid ? e1 * e1 : 0u);
      const uint32_t s2 = __reduce_add_sync(kFull, valid ? e2 * e2 : 0u);
      if(tx == 0 && y < H)
      {
        atomicAdd(rows + (size_t)y * 3 + 0, s0);
        atomicAdd(rows + (size_t)y * 3 + 1, s1);
        atomicAdd(rows + (size_t)y * 3 + 2, s2);
      }
      const int c0 = clampi(r0 - ga, 0, a.maxv), c1 = clampi(r1 - gb, 0, a.maxv), c2 = clampi(r2 - gc, 0, a.maxv);
      if(scp != nullptr && valid)
      {
        const size_t o = (size_t)y * W + x;
        scp[o]             = (T)c0;
        scp[plane + o]     = (T)c1;
        scp[2 * plane + o] = (T)c2;
      }
      if(mom.p != nullptr && valid)
      {
        const int q = i >> 2;
        const uint32_t av[3] = { (uint32_t)t0, (uint32_t)t1, (uint32_t)t2 };
        const uint32_t bv[3] = { (uint32_t)c0, (uint32_t)c1, (uint32_t)c2 };
        #pragma unroll
        for(int c = 0; c < 3; c++)
        {
          mm[q][c][0] += av[c];
          mm[q][c][1] += bv[c];
          mm[q][c][2] += av[c] * av[c];
          mm[q][c][3] += bv[c] * bv[c];
          mm[q][c][4] += av[c] * bv[c];
        }
      }
    }
    if(mom.p != nullptr)
    {
      const int bx = x >> 2;
      #pragma unroll
      for(int q = 0; q < P / 4; q++)
      {
        const int by = ((y0 + ty * P) >> 2) + q;
        #pragma unroll
        for(int c = 0; c < 3; c++)
        {
          #pragma unroll
          for(int m = 0; m < 5; m++)
          {
            uint32_t v = mm[q][c][m];
            v += __shfl_xor_sync(kFull, v, 1);
            v += __shfl_xor_sync(kFull, v, 2);
            if((tx & 3) == 0 && bx < mom.nbx && by < mom.nby)
            {
              mom.p[((size_t)c * 5 + m) * mom.plane() + (size_t)by * mom.pitch + bx] = v;
            }
          }
        }
      }
    }
  }
}

template <int R, typename T>
static cudaError_t launch_cps_r(const CpsArgs& a, cudaStream_t s)
{
  constexpr int P = 8, TW = 32, TH = 4 * P;
  constexpr size_t smem = 2 * sizeof(float4) * (TW + 2 * R) * (TH + 2 * R);
  static bool configured = false;
  if(!configured)
  {
    const cudaError_t e = cudaFuncSetAttribute(k_cps<R, P, T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if(e != cudaSuccess) { return e; }
    configured = true;
  }
  const dim3 grid((a.W + TW - 1) / TW, (a.H + TH - 1) / TH);
  k_cps<R, P, T><<<grid, 128, smem, s>>>(a);
  return cudaGetLastError();
}

template <typename T>
cudaError_t launch_cps(const CpsArgs& a, int R, cudaStream_t s)
{
  switch(R)
  {
  case 1: return launch_cps_r<1, T>(a, s);
  case 2: return launch_cps_r<2, T>(a, s);
  case 3: return launch_cps_r<3, T>(a, s);
  case 4: return launch_cps_r<4, T>(a, s);
  case 5: return launch_cps_r<5, T>(a, s);
  default: return cudaErrorInvalidValue;
  }
}
template cudaError_t launch_cps<uint8_t>(const CpsArgs&, int, cudaStream_t);
template cudaError_t launch_cps<uint16_t>(const CpsArgs&, int, cudaStream_t);

// =============================================================================================
// finalize: the order-dependent FP64 pooling chains of one pair, one thread per chain.
// Inputs are staged chunk by chunk into shared memory by all threads so that each chain only
// waits on its own floating-point dependency.
//   WS-PSNR   KBNS over rows of rowSSD * w[y]            (xWSPSNR.cpp:123-132)
//   IV-PSNR   KBNS over rows of rowSSE * w[y] (ERP)       (xIVPSNR.cpp:171-175) + exact uint64 sums
//   SSIM      KBNS over window rows (ERP: row * w[y + 4], weights KBNS) (xSSIM.cpp:348-351,
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
  return sl.use_ws ? dmul(v, a.ws[4 * y + 4]) : v;
}

__global__ void __launch_bounds__(256) k_finalize(const __grid_constant__ FinalizeArgs a)
{
  extern __shared__ double stage[];  // [len] values, then [len] ERP weights for weighted SSIM chains
  PairOut* o = a.out;
  if(blockIdx.x == (unsigned)a.nchains)
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
    for(int k = 0; k < 6; k++) { atomicAdd(&acc[k], loc[k]); }
    __syncthreads();
    if(threadIdx.x < 6) { o->cps_sum[threadIdx.x / 3][threadIdx.x % 3] = acc[threadIdx.x]; }
    return;
  }
  const FinChain ch = a.chain[blockIdx.x];
  const bool wsum = ch.kind == kChainSsim && a.slot[ch.a].use_ws;
  const int len = ch.kind == kChainSsim ? a.slot[ch.a].ny : a.H;
  double* vals = stage;
  double* wts = stage + len;
  for(int y = threadIdx.x; y < len; y += blockDim.x)
  {
    vals[y] = chain_value(a, ch, y);
    if(wsum) { wts[y] = a.ws[4 * y + 4]; }
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

cudaError_t launch_finalize(const FinalizeArgs& a_in, cudaStream_t s)
{
  FinalizeArgs a = a_in;
  a.nchains = 0;
  if(a.do_wspsnr && a.ws) { for(int c = 0; c < 3; c++) { a.chain[a.nchains++] = { kChainWsPsnr, c, 0 }; } }
  if(a.cps_rows && a.ws) { for(int d = 0; d < 2; d++) { for(int c = 0; c < 3; c++) { a.chain[a.nchains++] = { kChainIvPsnr, d, c }; } } }
  for(int sl = 0; sl < a.nslots; sl++)
  {
    if(a.slot[sl].row_sum == nullptr || a.slot[sl].ny <= 0) { continue; }
    for(int c = 0; c < 3; c++) { a.chain[a.nchains++] = { kChainSsim, sl, c }; }
  }
  const int blocks = a.nchains + (a.cps_rows ? 1 : 0);
  if(blocks == 0) { return cudaSuccess; }
  const size_t smem = (size_t)2 * max(a.H, 1) * sizeof(double);
  static bool configured = false;
  if(!configured)
  {
    const cudaError_t e = cudaFuncSetAttribute(k_finalize, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    if(e != cudaSuccess) { return e; }
    configured = true;
  }
  if(smem > 200 * 1024) { return cudaErrorInvalidValue; }
  k_finalize<<<blocks, 256, smem, s>>>(a);
  return cudaGetLastError();
}

}  // namespace qmiv
