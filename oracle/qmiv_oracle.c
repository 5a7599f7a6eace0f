/*
  qmiv_oracle.c — CPU restatement of the QMIV metric hot path (see qmiv_oracle.h).

  TEST INFRASTRUCTURE ONLY: the checker for the CUDA library, never part of it.
  Compiled with -ffp-contract=off so that every floating-point operation is the single IEEE
  operation written here, in the order the reference writes it.
  Citations are file:line inside the QMIV repository.
*/
#include "qmiv_oracle.h"
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ----------------------------------------------------------------------------------------------- */
/* helpers                                                                                         */
/* ----------------------------------------------------------------------------------------------- */

static inline int32_t qo_clampi(int32_t v, int32_t lo, int32_t hi) { return v < lo ? lo : (v > hi ? hi : v); }
/* The reference's int32 products and sums where they may wrap (two's complement), formed in unsigned
   arithmetic: a signed overflow is undefined in C and lets the compiler widen the result. */
static inline int32_t qo_mul_wrap(int32_t a, int32_t b) { return (int32_t)((uint32_t)a * (uint32_t)b); }
static inline int32_t qo_add_wrap(int32_t a, int32_t b) { return (int32_t)((uint32_t)a + (uint32_t)b); }
static inline int32_t qo_max_value(int32_t bitdepth) { return (1 << bitdepth) - 1; } /* xCommonDefCORE.h:156 */

/* Round half away from zero by adding +-0.5 and truncating, as xRoundF32ToI32 / xRoundF64ToI32
   (libs/pmbb-core/src/xHelpersFLT.h:32-33). The addition happens in the source precision. */
static inline int32_t qo_round_f32(float f) { volatile float t = f + copysignf(0.5f, f); return (int32_t)t; }
static inline int32_t qo_round_f64(double f) { volatile double t = f + copysign(0.5, f); return (int32_t)t; }

/* Kahan-Babuska-Neumaier summation, libs/pmbb-core/src/xKBNS.h:36-43 (scalar) and
   libs/pmbb-core/src/xKBNS.cpp (SSE/AVX lane-wise variants compute the same per lane). */
typedef struct { double s, c; } qo_kbns;
static inline void qo_kbns_add(qo_kbns* k, double v)
{
  double t = k->s + v;
  if(fabs(k->s) >= fabs(v)) { k->c += ((k->s - t) + v); }
  else                      { k->c += ((v - t) + k->s); }
  k->s = t;
}
static inline double qo_kbns_result(const qo_kbns* k) { return k->s + k->c; }

/* xPSNR::CalcPSNRfromSSD, libs/pmbb-ivqm/src/xPSNR.cpp:186-192 */
static double qo_psnr_from_ssd(double ssd, int64_t area, int32_t bitdepth)
{
  const uint64_t maxv = (uint64_t)qo_max_value(bitdepth);
  const uint64_t MAX  = (uint64_t)area * (maxv * maxv);
  return ssd > 0 ? 10.0 * log10((double)MAX / ssd) : DBL_MAX;
}

/* ----------------------------------------------------------------------------------------------- */
/* a1: raw 4:2:0/4:2:2/4:4:4 -> planar 4:4:4 uint16                                                */
/* libs/pmbb-core/src/xSeq.cpp:231-290 (xUnpackFrame); replication as xPixelOpsSTD.cpp:30-49,68-87 */
/* ----------------------------------------------------------------------------------------------- */
void qo_unpack444(const void* const planes[3], int32_t W, int32_t H, int32_t bitdepth, int32_t chroma_format, uint16_t* dst)
{
  const int32_t sx = (chroma_format == 444) ? 0 : 1;
  const int32_t sy = (chroma_format == 420) ? 1 : 0;
  for(int32_t c = 0; c < 3; c++)
  {
    const int32_t cw = c == 0 ? W : (W >> sx);
    const int32_t shx = c == 0 ? 0 : sx, shy = c == 0 ? 0 : sy;
    uint16_t* d = dst + (size_t)c * W * H;
    for(int32_t y = 0; y < H; y++)
    {
      const size_t row = (size_t)(y >> shy) * cw;
      for(int32_t x = 0; x < W; x++)
      {
        const size_t i = row + (x >> shx);
        d[(size_t)y * W + x] = bitdepth <= 8 ? ((const uint8_t*)planes[c])[i] : ((const uint16_t*)planes[c])[i];
      }
    }
  }
}

/* ----------------------------------------------------------------------------------------------- */
/* a3: global colour difference, libs/pmbb-ivqm/src/xGlobClrDiff.cpp:70-103                        */
/* ----------------------------------------------------------------------------------------------- */
void qo_gcd(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, const float coef[4], int32_t gcd[4])
{
  const int32_t maxv = qo_max_value(bitdepth);
  const double  area = (double)((int64_t)W * H);
  int64_t sd[4] = { 0, 0, 0, 0 };
  for(int32_t c = 0; c < 3; c++)
  {
    const uint16_t* t = tst + (size_t)c * W * H;
    const uint16_t* r = ref + (size_t)c * W * H;
    for(size_t i = 0; i < (size_t)W * H; i++) { sd[c] += (int32_t)t[i] - (int32_t)r[i]; } /* xDistortionSTD.cpp:12-22 */
  }
  for(int32_t c = 0; c < 4; c++)
  {
    const int32_t maxdiff = qo_round_f32(coef[c] * (float)maxv);
    const double  avg     = (double)sd[c] / area;
    gcd[c] = qo_clampi(qo_round_f64(avg), -maxdiff, maxdiff);
  }
}

/* ----------------------------------------------------------------------------------------------- */
/* a4/a5: corresponding pixel shift, one direction.                                                */
/* x86 interleaved path: libs/pmbb-ivqm/src/xCorrespPixelShiftSSE.cpp:18-70 (row SSE) and :75-127  */
/* (shift-compensated picture). Out-of-picture candidates read the edge-replicated margin          */
/* (margin = roundUp(R,2) >= R, apps/QMIV/src/xAppQMIV.cpp:353, extend() at :899) = clamped index.  */
/* The test pixel plus GCD is not clipped (xc_CLIP_CURR_TST_RANGE=false, xCommonDefIVQM.h:62).      */
/* The per-row sums live in 32-bit lanes (_mm_add_epi32) and are sign-extended to 64 bits at the    */
/* end of the row (:38-40); that is reproduced with uint32 wrap-around and an int32 cast.           */
/* ----------------------------------------------------------------------------------------------- */
void qo_cps(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, const int32_t gcd[4],
            int32_t R, const int32_t cws[4], uint64_t* row_sse, uint16_t* scp)
{
  const int32_t  maxv = qo_max_value(bitdepth);
  const size_t   pl   = (size_t)W * H;
  for(int32_t y = 0; y < H; y++)
  {
    uint32_t rowsum[3] = { 0, 0, 0 };
    for(int32_t x = 0; x < W; x++)
    {
      int32_t s[3];
      for(int32_t c = 0; c < 3; c++) { s[c] = (int32_t)tst[c * pl + (size_t)y * W + x] + gcd[c]; }
      int32_t  best_err     = INT32_MAX;
      uint32_t best_dist[3] = { 0, 0, 0 };
      int32_t  best_pel[3]  = { 0, 0, 0 };
      for(int32_t dy = -R; dy <= R; dy++)
      {
        const int32_t yy = qo_clampi(y + dy, 0, H - 1);
        for(int32_t dx = -R; dx <= R; dx++)
        {
          const int32_t xx = qo_clampi(x + dx, 0, W - 1);
          uint32_t dist[3]; int32_t pel[3]; uint32_t err = 0;
          for(int32_t c = 0; c < 3; c++)
          {
            pel[c]  = ref[c * pl + (size_t)yy * W + xx];
            const uint32_t d = (uint32_t)(s[c] - pel[c]);
            dist[c] = d * d;                          /* _mm_mullo_epi32, wraps */
            err    += dist[c] * (uint32_t)cws[c];     /* _mm_mullo_epi32 + horizontal add, wraps */
          }
          if((int32_t)err < best_err)                 /* first strict minimum in raster order */
          {
            best_err = (int32_t)err;
            for(int32_t c = 0; c < 3; c++) { best_dist[c] = dist[c]; best_pel[c] = pel[c]; }
          }
        }
      }
      for(int32_t c = 0; c < 3; c++) { rowsum[c] += best_dist[c]; }
      if(scp)
      {
        for(int32_t c = 0; c < 3; c++)
        {
          int32_t v = best_pel[c] - gcd[c];
          v = v < maxv ? v : maxv;                    /* _mm_min_epi32 */
          v = v < 0 ? 0 : (v > 65535 ? 65535 : v);    /* _mm_packus_epi32 */
          scp[c * pl + (size_t)y * W + x] = (uint16_t)v;
        }
      }
    }
    if(row_sse) { for(int32_t c = 0; c < 3; c++) { row_sse[(size_t)y * 3 + c] = (uint64_t)(int64_t)(int32_t)rowsum[c]; } }
  }
}

/* Portable planar path, libs/pmbb-ivqm/src/xCorrespPixelShiftSTD.cpp:19-84: uint64 row accumulation. */
void qo_cps_rows_std(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, const int32_t gcd[4],
                     int32_t R, const int32_t cws[4], uint64_t* row_sse)
{
  const size_t pl = (size_t)W * H;
  for(int32_t y = 0; y < H; y++)
  {
    uint64_t rowsum[3] = { 0, 0, 0 };
    for(int32_t x = 0; x < W; x++)
    {
      int32_t s[3];
      for(int32_t c = 0; c < 3; c++) { s[c] = (int32_t)tst[c * pl + (size_t)y * W + x] + gcd[c]; }
      int32_t best_err = INT32_MAX; int32_t best_pel[3] = { 0, 0, 0 };
      for(int32_t dy = -R; dy <= R; dy++)
      {
        const int32_t yy = qo_clampi(y + dy, 0, H - 1);
        for(int32_t dx = -R; dx <= R; dx++)
        {
          const int32_t xx = qo_clampi(x + dx, 0, W - 1);
          int32_t err = 0; int32_t pel[3];
          for(int32_t c = 0; c < 3; c++)
          {
            pel[c] = ref[c * pl + (size_t)yy * W + xx];
            const int32_t d = s[c] - pel[c];
            err = qo_add_wrap(err, qo_mul_wrap(qo_mul_wrap(d, d), cws[c]));
          }
          if(err < best_err) { best_err = err; for(int32_t c = 0; c < 3; c++) { best_pel[c] = pel[c]; } }
        }
      }
      for(int32_t c = 0; c < 3; c++) { const int32_t d = s[c] - best_pel[c]; rowsum[c] += (uint64_t)(int64_t)qo_mul_wrap(d, d); }
    }
    for(int32_t c = 0; c < 3; c++) { row_sse[(size_t)y * 3 + c] = rowsum[c]; }
  }
}

/* ----------------------------------------------------------------------------------------------- */
/* a8: equirectangular weights, libs/pmbb-ivqm/src/xWeightedSpherically.cpp:13-29                   */
/* ----------------------------------------------------------------------------------------------- */
void qo_ws_weights(int32_t H, int32_t lat_range, double* w, double* correction)
{
  const double pi   = 3.14159265358979323846;              /* xc_Pi, xCommonDefCORE.h:227 */
  const double heq  = 180.0 * (double)H / (double)lat_range;
  const double off  = (heq - H) / 2.0;
  qo_kbns k = { 0.0, 0.0 };
  for(int32_t h = 0; h < H; h++)
  {
    w[h] = cos((h + off - (heq / 2 - 0.5)) * pi / heq);
    qo_kbns_add(&k, w[h]);
  }
  if(correction) { *correction = H / qo_kbns_result(&k); }
}

/* ----------------------------------------------------------------------------------------------- */
/* a9/a10: SSIM under every structural similarity option of the app                                */
/* windows: libs/pmbb-ivqm/src/xStructSimSTD.cpp:19-193 (regular 11x11 centred windows: Gaussian   */
/*          float, Gaussian integer, averaged), :353-461 (block windows anchored at their top-left  */
/*          sample: Gaussian integer 8/16, averaged 8/16/32). The AVX form of the regular averaged  */
/*          window (xStructSimAVX.h:20-23 -> CalcBlckAvg11) sums the same integers.                 */
/* loops:   libs/pmbb-ivqm/src/xSSIM.cpp:161-196 (ranges, NumUnit), :381-404 (block counts),        */
/*          :215-251 (row KBNS in x order, picture KBNS over rows / NumActive)                      */
/* borders: libs/pmbb-core/src/xMarginOps.h:16-20 (Nearest, Reflect, Mirror, Constant = 65535 as   */
/*          xPicP::extend passes it, xPic.cpp:94-101, Zero); regular windows only, xSSIM.cpp:90     */
/* ERP:     libs/pmbb-ivqm/src/xIVSSIM.cpp:138-173 (row weight w[y] regular, w[y + WndSize/2] block)*/
/* ----------------------------------------------------------------------------------------------- */

/* Integer Gaussian windows (xStructSimConsts.h:111-124 for 11x11, :145-173 for 8x8 and 16x16), each
   the mirror image of its top-left quadrant in both directions; weights sum to 2^18 (16x16: 262140) and
   the sums are scaled by 2^-18 (c_InvFltrIntMul). The 11x11 quadrant is not symmetric about its
   diagonal ([4][5] = 14854, [5][4] = 14855). */
static const int32_t qo_gq11[6][6] = {
  { 0, 2, 10, 29, 57, 72 },           { 2, 15, 72, 218, 424, 530 },          { 10, 72, 340, 1032, 2010, 2510 },
  { 29, 218, 1032, 3135, 6107, 7626 }, { 57, 424, 2010, 6107, 11894, 14854 }, { 72, 530, 2510, 7626, 14855, 18550 },
};
static const int32_t qo_gq8[4][4] = {
  { 81, 308, 749, 1168 }, { 308, 1168, 2842, 4432 }, { 749, 2842, 6913, 10781 }, { 1168, 4432, 10781, 16814 },
};
static const int32_t qo_gq16[8][8] = {
  { 0, 1, 4, 10, 19, 32, 45, 54 },                 { 1, 5, 13, 32, 64, 108, 152, 181 },
  { 4, 13, 38, 91, 181, 305, 432, 514 },           { 10, 32, 91, 216, 432, 727, 1029, 1224 },
  { 19, 64, 181, 432, 865, 1456, 2061, 2451 },     { 32, 108, 305, 727, 1456, 2451, 3469, 4126 },
  { 45, 152, 432, 1029, 2061, 3469, 4909, 5839 },  { 54, 181, 514, 1224, 2451, 4126, 5839, 6947 },
};

static int32_t qo_gauss_int(int32_t N, int32_t y, int32_t x)
{
  const int32_t qy = y < N - 1 - y ? y : N - 1 - y, qx = x < N - 1 - x ? x : N - 1 - x;
  return N == 11 ? qo_gq11[qy][qx] : N == 8 ? qo_gq8[qy][qx] : qo_gq16[qy][qx];
}

/* Float Gaussian window (c_FilterRglrGaussFlt32, xStructSimConsts.h:55-68): the 11x11 Gaussian of
   sigma 1.5 normalised to unit sum, rounded to float; each product is formed in double. */
static double qo_gflt11[11][11];
static int    qo_gflt_ready = 0;
static void qo_gflt_init(void)
{
  if(qo_gflt_ready) { return; }
  double g[11][11], sum = 0.0;
  for(int32_t y = 0; y < 11; y++)
  {
    for(int32_t x = 0; x < 11; x++) { g[y][x] = exp(-(double)((x - 5) * (x - 5) + (y - 5) * (y - 5)) / 4.5); sum += g[y][x]; }
  }
  for(int32_t y = 0; y < 11; y++) { for(int32_t x = 0; x < 11; x++) { qo_gflt11[y][x] = (double)(float)(g[y][x] / sum); } }
  qo_gflt_ready = 1;
}

static int qo_ssm_regular(int32_t mode) { return mode >= QO_SSM_REGULAR_GAUSSIAN_FLT && mode <= QO_SSM_REGULAR_AVERAGED; }
static int32_t qo_ssm_window(const qo_ssim_cfg* cfg) { return qo_ssm_regular(cfg->mode) ? 11 : cfg->window; }

/* position of sample i of a length-n line after margin extension, -1 for the constant modes */
static int32_t qo_brd_index(int32_t i, int32_t n, int32_t border)
{
  if(i >= 0 && i < n) { return i; }
  switch(border)
  {
  case QO_BRD_NEAREST: return i < 0 ? 0 : n - 1;              /* ( a a a | a b c d | d d d ) */
  case QO_BRD_REFLECT: return i < 0 ? -1 - i : 2 * n - 1 - i; /* ( c b a | a b c d | d c b ) */
  case QO_BRD_MIRROR:  return i < 0 ? -i : 2 * n - 2 - i;     /* ( d c b | a b c d | c b a ) */
  default:             return -1;
  }
}
static int32_t qo_brd_sample(const uint16_t* p, int32_t W, int32_t H, int32_t x, int32_t y, int32_t border)
{
  const int32_t xi = qo_brd_index(x, W, border), yi = qo_brd_index(y, H, border);
  if(xi < 0 || yi < 0) { return border == QO_BRD_CONSTANT ? 65535 : 0; }
  return p[(size_t)yi * W + xi];
}

static double qo_ssim_formula(double avg_r, double avg_t, double var_r, double var_t, double cov, double C1, double C2, int32_t calc_l)
{
  const double cs = (2 * cov + C2) / (var_r + var_t + C2);          /* "Contrast" * "Similarity" */
  if(!calc_l) { return cs; }
  const double l = (2 * avg_r * avg_t + C1) / (avg_r * avg_r + avg_t * avg_t + C1); /* "Luminance" */
  return l * cs;
}

/* One window whose top-left input sample is (x0, y0); t = "Tst", r = "Ref". */
static double qo_ssim_window_cfg(const uint16_t* t, const uint16_t* r, int32_t W, int32_t H, int32_t x0, int32_t y0,
                                 const qo_ssim_cfg* cfg, double C1, double C2, int32_t calc_l)
{
  const int32_t N = qo_ssm_window(cfg), brd = qo_ssm_regular(cfg->mode) ? cfg->border : QO_BRD_NONE;
  if(cfg->mode == QO_SSM_REGULAR_GAUSSIAN_FLT) /* xStructSimSTD.cpp:19-88: double sums in dy, dx order */
  {
    double sr = 0, st = 0, srr = 0, stt = 0, srt = 0;
    for(int32_t dy = 0; dy < 11; dy++)
    {
      for(int32_t dx = 0; dx < 11; dx++)
      {
        const double R = (double)qo_brd_sample(r, W, H, x0 + dx, y0 + dy, brd);
        const double T = (double)qo_brd_sample(t, W, H, x0 + dx, y0 + dy, brd);
        const double C = qo_gflt11[dy][dx];
        sr += R * C; st += T * C; srr += (R * R) * C; stt += (T * T) * C; srt += (R * T) * C;
      }
    }
    return qo_ssim_formula(sr, st, srr - sr * sr, stt - st * st, srt - sr * st, C1, C2, calc_l);
  }
  const int gauss = cfg->mode == QO_SSM_REGULAR_GAUSSIAN_INT || cfg->mode == QO_SSM_BLOCK_GAUSSIAN_INT;
  int64_t sr = 0, st = 0, srr = 0, stt = 0, srt = 0;
  for(int32_t dy = 0; dy < N; dy++)
  {
    for(int32_t dx = 0; dx < N; dx++)
    {
      const int64_t R = qo_brd_sample(r, W, H, x0 + dx, y0 + dy, brd);
      const int64_t T = qo_brd_sample(t, W, H, x0 + dx, y0 + dy, brd);
      const int64_t C = gauss ? qo_gauss_int(N, dy, dx) : 1;
      sr += R * C; st += T * C; srr += R * R * C; stt += T * T * C; srt += R * T * C;
    }
  }
  const double inv = gauss ? 1.0 / (double)(1 << 18)                                    /* c_InvFltrIntMul */
                   : cfg->mode == QO_SSM_REGULAR_AVERAGED ? 1.0 / (double)121           /* c_InvFltrArea */
                   : 1.0 / (double)(N * N);                                              /* c_InvBlockArea */
  const double avg_r = (double)sr * inv, avg_t = (double)st * inv;
  const double var_r = (double)srr * inv - avg_r * avg_r;
  const double var_t = (double)stt * inv - avg_t * avg_t;
  const double cov   = (double)srt * inv - avg_r * avg_t;
  return qo_ssim_formula(avg_r, avg_t, var_r, var_t, cov, C1, C2, calc_l);
}

int qo_ssim_cfg_check(const qo_ssim_cfg* cfg, int32_t W, int32_t H)
{
  if(cfg->mode < QO_SSM_REGULAR_GAUSSIAN_FLT || cfg->mode > QO_SSM_BLOCK_AVERAGED) { return -1; }
  if(cfg->border < QO_BRD_NONE || cfg->border > QO_BRD_ZERO) { return -1; }
  const int32_t N = qo_ssm_window(cfg);
  if(qo_ssm_regular(cfg->mode) && cfg->window != 11) { return -1; }                     /* xAppQMIV.cpp:332 */
  if(cfg->mode == QO_SSM_BLOCK_AVERAGED && N != 8 && N != 16 && N != 32) { return -1; } /* xAppQMIV.cpp:104 */
  if(cfg->mode == QO_SSM_BLOCK_GAUSSIAN_INT && N != 8 && N != 16) { return -1; }        /* xStructSimSTD.cpp:399-403 */
  if(cfg->stride < 1 || cfg->stride > N) { return -1; }                                  /* xAppQMIV.cpp:331 */
  /* the averaged 11x11 window squares samples in 32-bit lanes (xStructSimSTD.cpp:167-169, and as signed
     16-bit products in its AVX form), which the constant 65535 margin overflows */
  if(cfg->mode == QO_SSM_REGULAR_AVERAGED && cfg->border == QO_BRD_CONSTANT) { return -1; }
  if(W < N || H < N) { return -1; }
  return 0;
}

/* window rows/columns of one picture: first window origin, count and the top-left offset of the
   window's input samples relative to the origin */
static void qo_ssim_range(const qo_ssim_cfg* cfg, int32_t len, int32_t* beg, int32_t* num, int32_t* org)
{
  const int32_t S = cfg->stride, N = qo_ssm_window(cfg);
  if(qo_ssm_regular(cfg->mode))
  {
    const int32_t b = cfg->border != QO_BRD_NONE ? 0 : 5, e = cfg->border != QO_BRD_NONE ? len : len - 5;
    *beg = b; *num = (e - b + S - 1) / S; *org = -5;
  }
  else { *beg = 0; *num = (len - N) / S + 1; *org = 0; }
}

static void qo_ssim_consts(int32_t bitdepth, double* C1, double* C2)
{
  const double maxv = (double)qo_max_value(bitdepth);  /* xSSIM.cpp:50-52, K1=0.01, K2=0.03 */
  const double a = 0.01 * maxv, b = 0.03 * maxv;
  *C1 = a * a; *C2 = b * b;
}

int qo_ssim_pic_cfg(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, int32_t calc_l,
                    const double* ws_weights, const qo_ssim_cfg* cfg, double out[3])
{
  if(qo_ssim_cfg_check(cfg, W, H)) { return -1; }
  qo_gflt_init();
  double C1, C2; qo_ssim_consts(bitdepth, &C1, &C2);
  int32_t bx, by, nx, ny, org;
  qo_ssim_range(cfg, W, &bx, &nx, &org);
  qo_ssim_range(cfg, H, &by, &ny, &org);
  const int32_t S = cfg->stride, wsoff = qo_ssm_regular(cfg->mode) ? 0 : (qo_ssm_window(cfg) >> 1);
  for(int32_t c = 0; c < 3; c++)
  {
    const uint16_t* t = tst + (size_t)c * W * H;
    const uint16_t* r = ref + (size_t)c * W * H;
    qo_kbns pic = { 0.0, 0.0 }, wacc = { 0.0, 0.0 };
    for(int32_t j = 0; j < ny; j++)
    {
      const int32_t y = by + j * S;
      qo_kbns row = { 0.0, 0.0 };
      for(int32_t i = 0; i < nx; i++)
      {
        const int32_t x = bx + i * S;
        qo_kbns_add(&row, qo_ssim_window_cfg(t, r, W, H, x + org, y + org, cfg, C1, C2, calc_l));
      }
      double rs = qo_kbns_result(&row);
      if(ws_weights) { const double wt = ws_weights[y + wsoff]; rs = rs * wt; qo_kbns_add(&wacc, wt); }
      qo_kbns_add(&pic, rs);
    }
    const int64_t active = (int64_t)nx * ny;
    if(ws_weights)
    {
      const double corr = qo_kbns_result(&wacc) / ny;
      out[c] = qo_kbns_result(&pic) / ((double)active * corr);
    }
    else { out[c] = qo_kbns_result(&pic) / (double)active; }
  }
  return 0;
}

static const qo_ssim_cfg qo_ssim_default = { QO_SSM_BLOCK_AVERAGED, QO_BRD_NONE, 8, 4 }; /* xSSIM.h:35-37 */

void qo_ssim_pic(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, int32_t calc_l,
                 const double* ws_weights, double out[3])
{
  if(qo_ssim_pic_cfg(tst, ref, W, H, bitdepth, calc_l, ws_weights, &qo_ssim_default, out)) { out[0] = out[1] = out[2] = 0.0; }
}

/* ----------------------------------------------------------------------------------------------- */
/* a11: MS-SSIM, libs/pmbb-ivqm/src/xSSIM.cpp:115-141, scales :405-417, exponents                  */
/* libs/pmbb-ivqm/src/xStructSimConsts.h:42-49, downsampling xPixelOpsSTD.cpp:50-67; every scale   */
/* uses the same window options, the sub-pictures extended by the same border mode (:127)          */
/* ----------------------------------------------------------------------------------------------- */
static const double qo_ms_exponents[5][5] = {
  { 1.0000, 0.0000, 0.0000, 0.0000, 0.0000 },
  { 0.1356, 0.8644, 0.0000, 0.0000, 0.0000 },
  { 0.0711, 0.4530, 0.4760, 0.0000, 0.0000 },
  { 0.0517, 0.3295, 0.3462, 0.2726, 0.0000 },
  { 0.0448, 0.2856, 0.3001, 0.2363, 0.1333 },
};

int32_t qo_num_scales(int32_t W, int32_t H)
{
  for(int32_t i = 0; i < 5; i++) { const int32_t lim = 32 << i; if(W < lim || H < lim) { return i; } }
  return 5;
}

static void qo_downsample(uint16_t* dst, const uint16_t* src, int32_t W, int32_t H) /* dst (W>>1)x(H>>1) x3 */
{
  const int32_t dw = W >> 1, dh = H >> 1;
  for(int32_t c = 0; c < 3; c++)
  {
    const uint16_t* s = src + (size_t)c * W * H;
    uint16_t*       d = dst + (size_t)c * dw * dh;
    for(int32_t y = 0; y < dh; y++)
    {
      for(int32_t x = 0; x < dw; x++)
      {
        const uint16_t* p = s + (size_t)(2 * y) * W + 2 * x;
        d[(size_t)y * dw + x] = (uint16_t)(((int32_t)p[0] + p[1] + p[W] + p[W + 1] + 2) >> 2);
      }
    }
  }
}

int qo_msssim_pic_cfg(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, const qo_ssim_cfg* cfg,
                      double out[3])
{
  const int32_t ns = qo_num_scales(W, H);
  if(ns < 1) { return -1; }
  double sub[5][3];
  int rc = qo_ssim_pic_cfg(tst, ref, W, H, bitdepth, ns == 1, NULL, cfg, sub[0]);
  uint16_t* bufT = NULL; uint16_t* bufR = NULL;
  const uint16_t* curT = tst; const uint16_t* curR = ref;
  int32_t w = W, h = H;
  for(int32_t i = 1; i < ns && rc == 0; i++)
  {
    const int32_t nw = w >> 1, nh = h >> 1;
    uint16_t* nT = (uint16_t*)malloc((size_t)nw * nh * 3 * sizeof(uint16_t));
    uint16_t* nR = (uint16_t*)malloc((size_t)nw * nh * 3 * sizeof(uint16_t));
    qo_downsample(nT, curT, w, h); qo_downsample(nR, curR, w, h);
    free(bufT); free(bufR); bufT = nT; bufR = nR; curT = nT; curR = nR; w = nw; h = nh;
    rc = qo_ssim_pic_cfg(curT, curR, w, h, bitdepth, i == ns - 1, NULL, cfg, sub[i]);
  }
  free(bufT); free(bufR);
  if(rc) { return -1; }
  for(int32_t c = 0; c < 3; c++)
  {
    double score = 1.0;
    for(int32_t i = 0; i < ns; i++)
    {
      const double v = sub[i][c] < 0 ? 0.0 : sub[i][c];   /* getVecReLU, xVec.h:297 */
      score *= pow(v, qo_ms_exponents[ns - 1][i]);
    }
    out[c] = score;
  }
  return 0;
}

int qo_msssim_pic(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, double out[3])
{
  return qo_msssim_pic_cfg(tst, ref, W, H, bitdepth, &qo_ssim_default, out);
}

/* ----------------------------------------------------------------------------------------------- */
/* a6: IV-PSNR of one direction from per-row CPS SSE, libs/pmbb-ivqm/src/xIVPSNR.cpp:163-189        */
/* ----------------------------------------------------------------------------------------------- */
static double qo_ivpsnr_quality(const uint64_t* row_sse, int32_t W, int32_t H, int32_t bitdepth, const double* ws, const int32_t cwa[4])
{
  double err[3];
  if(ws)
  {
    for(int32_t c = 0; c < 3; c++)
    {
      qo_kbns k = { 0.0, 0.0 };
      for(int32_t y = 0; y < H; y++) { qo_kbns_add(&k, (double)row_sse[(size_t)y * 3 + c] * ws[y]); }
      err[c] = qo_kbns_result(&k);
    }
  }
  else
  {
    for(int32_t c = 0; c < 3; c++)
    {
      uint64_t s = 0;
      for(int32_t y = 0; y < H; y++) { s += row_sse[(size_t)y * 3 + c]; }
      err[c] = (double)s;
    }
  }
  const int64_t area = (int64_t)W * H;
  double q[4] = { 0, 0, 0, 0 };
  for(int32_t c = 0; c < 3; c++) { q[c] = qo_psnr_from_ssd(err[c] > 0 ? err[c] : 1.0, area, bitdepth); }
  const int32_t wsum = cwa[0] + cwa[1] + cwa[2] + cwa[3];
  const double  inv  = 1.0 / (double)wsum;
  return (q[0] * (double)cwa[0] + q[1] * (double)cwa[1] + q[2] * (double)cwa[2] + q[3] * (double)cwa[3]) * inv;
}

/* ----------------------------------------------------------------------------------------------- */
/* Colour-space conversion before the metrics (f4): apps/QMIV/src/xAppQMIV.cpp:302-311 (which       */
/* conversion), :853-891 (order). The app dispatches to the integer forms; their portable versions  */
/* are libs/pmbb-core/src/xColorSpaceSTD.cpp:196-263. Fixed-point matrices with 16 fractional bits   */
/* for BT.601 (= SMPTE 170M), BT.709, SMPTE 240M and BT.2020, the same integers as the reference's   */
/* xColorSpaceCoeffYCbCr (xColorSpaceCoeff.h:59-73) so that rounding agrees.                         */
/* ----------------------------------------------------------------------------------------------- */
enum { QO_CS_RGB = 2, QO_CS_BGR = 3, QO_CS_GBR = 4, QO_CS_YCBCR = 16, QO_CS_BT601 = 17, QO_CS_SMPTE170M = 18,
       QO_CS_BT709 = 19, QO_CS_SMPTE240M = 20, QO_CS_BT2020 = 21 };
/* [space][0] = (Y<-R, Y<-G, Y<-B, Cb<-R, Cb<-G, Cr<-G, Cr<-B); [space][1] = (R<-Cr, G<-Cb, G<-Cr, B<-Cb) */
static const int32_t qo_rgb2ycc[4][7] = {
  { 19595, 38470, 7471, -11058, -21710, -27439, -5329 },   /* BT.601 */
  { 13933, 46871, 4732,  -7509, -25259, -29763, -3005 },   /* BT.709 */
  { 13894, 45941, 5701,  -7609, -25159, -29150, -3618 },   /* SMPTE 240M */
  { 17216, 44434, 3886,  -9151, -23617, -30133, -2635 },   /* BT.2020 */
};
static const int32_t qo_ycc2rgb[4][4] = {
  {  91881, -22553, -46802, 116130 },
  { 103206, -12276, -30679, 121609 },
  { 103285, -14852, -31236, 119669 },
  {  96639, -10784, -37444, 123299 },
};
static int qo_cs_is_rgb(int32_t c) { return c == QO_CS_RGB || c == QO_CS_BGR || c == QO_CS_GBR; }
static int qo_cs_is_defined_ycc(int32_t c) { return c > QO_CS_YCBCR; }
static int qo_cs_index(int32_t c) /* eClrSpcLC of a defined YCbCr space, xUtilsQMIV.cpp:43-54 */
{
  switch(c) { case QO_CS_BT601: case QO_CS_SMPTE170M: return 0; case QO_CS_BT709: return 1; case QO_CS_SMPTE240M: return 2;
              case QO_CS_BT2020: return 3; default: return -1; }
}
static inline int32_t qo_clipu(int32_t v, int32_t mx) { return v < 0 ? 0 : (v > mx ? mx : v); }

/* Converts two 4:4:4 planar pictures in place as the app's preprocessFrames. Returns nonzero for a
   combination the app refuses (xAppQMIV.cpp:302-306). */
int qo_convert_colour(uint16_t* P0, uint16_t* P1, int32_t W, int32_t H, int32_t bitdepth, int32_t cs_in, int32_t cs_metric)
{
  if(cs_in != cs_metric)
  {
    if(cs_in >= QO_CS_YCBCR && cs_metric >= QO_CS_YCBCR) { return 1; }
    if(cs_in == QO_CS_YCBCR || cs_metric == QO_CS_YCBCR) { return 1; }
  }
  const int ycc2rgb = qo_cs_is_defined_ycc(cs_in) && qo_cs_is_rgb(cs_metric);
  const int rgb2ycc = qo_cs_is_rgb(cs_in) && qo_cs_is_defined_ycc(cs_metric);
  const int reorder = qo_cs_is_rgb(cs_in) && cs_in != QO_CS_RGB && cs_metric == QO_CS_RGB;
  const size_t pl = (size_t)W * H;
  const int32_t mid = 1 << (bitdepth - 1), mx = (1 << bitdepth) - 1, add = 1 << 15;
  uint16_t* pics[2] = { P0, P1 };
  for(int i = 0; i < 2; i++)
  {
    uint16_t* a = pics[i]; uint16_t* b = a + pl; uint16_t* c = a + 2 * pl;
    if(ycc2rgb) /* xColorSpaceSTD.cpp:231-263 */
    {
      const int32_t* k = qo_ycc2rgb[qo_cs_index(cs_in)];
      for(size_t n = 0; n < pl; n++)
      {
        const int32_t iy = a[n], iu = (int32_t)b[n] - mid, iv = (int32_t)c[n] - mid;
        const int32_t sy = (iy << 16) + add;
        const int32_t r = (sy + k[0] * iv) >> 16, g = (sy + k[1] * iu + k[2] * iv) >> 16, bb = (sy + k[3] * iu) >> 16;
        a[n] = (uint16_t)qo_clipu(r, mx); b[n] = (uint16_t)qo_clipu(g, mx); c[n] = (uint16_t)qo_clipu(bb, mx);
      }
    }
    if(rgb2ycc) /* xColorSpaceSTD.cpp:196-229 */
    {
      const int32_t* k = qo_rgb2ycc[qo_cs_index(cs_metric)];
      for(size_t n = 0; n < pl; n++)
      {
        const int32_t r = a[n], g = b[n], bb = c[n];
        const int32_t ty = (k[0] * r + k[1] * g + k[2] * bb + add) >> 16;
        const int32_t tu = (k[3] * r + k[4] * g + (bb << 15) + add) >> 16;
        const int32_t tv = ((r << 15) + k[5] * g + k[6] * bb + add) >> 16;
        a[n] = (uint16_t)qo_clipu(ty, mx); b[n] = (uint16_t)qo_clipu(tu + mid, mx); c[n] = (uint16_t)qo_clipu(tv + mid, mx);
      }
    }
    if(reorder) /* xAppQMIV.cpp:878-891: BGR -> RGB swaps 0 and 2; GBR -> RGB swaps 0 and 1, then 0 and 2 */
    {
      for(size_t n = 0; n < pl; n++)
      {
        uint16_t t;
        if(cs_in == QO_CS_BGR) { t = a[n]; a[n] = c[n]; c[n] = t; }
        if(cs_in == QO_CS_GBR) { t = a[n]; a[n] = b[n]; b[n] = t; t = a[n]; a[n] = c[n]; c[n] = t; }
      }
    }
  }
  return 0;
}

/* The frame pipeline on colour-converted 4:4:4 pictures (conversion before the exactness check and
   the metrics, as xAppQMIV::preprocessFrames). */
int qo_compute_pair_cs(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask, int32_t cs_in,
                       int32_t cs_metric, qo_result* out)
{
  const int32_t W = p->width, H = p->height, BD = p->bitdepth;
  const size_t  pl = (size_t)W * H;
  uint16_t* P0 = (uint16_t*)malloc(3 * pl * sizeof(uint16_t));
  uint16_t* P1 = (uint16_t*)malloc(3 * pl * sizeof(uint16_t));
  qo_unpack444(planes0, W, H, BD, p->chroma_format, P0);
  qo_unpack444(planes1, W, H, BD, p->chroma_format, P1);
  int rc = qo_convert_colour(P0, P1, W, H, BD, cs_in, cs_metric);
  if(rc == 0)
  {
    qo_params q = *p;
    q.chroma_format = 444;
    const size_t esz = BD <= 8 ? 1 : 2;
    unsigned char* B0 = (unsigned char*)malloc(3 * pl * esz);
    unsigned char* B1 = (unsigned char*)malloc(3 * pl * esz);
    for(size_t n = 0; n < 3 * pl; n++)
    {
      if(esz == 1) { B0[n] = (unsigned char)P0[n]; B1[n] = (unsigned char)P1[n]; }
      else { ((uint16_t*)B0)[n] = P0[n]; ((uint16_t*)B1)[n] = P1[n]; }
    }
    const void* q0[3] = { B0, B0 + pl * esz, B0 + 2 * pl * esz };
    const void* q1[3] = { B1, B1 + pl * esz, B1 + 2 * pl * esz };
    rc = qo_compute_pair(&q, q0, q1, mask, out, NULL, NULL);
    free(B0); free(B1);
  }
  free(P0); free(P1);
  return rc;
}

/* ----------------------------------------------------------------------------------------------- */
/* Mask mode: the mask picture's luma weights every sample (eCmp::LM in every *M call).            */
/* ----------------------------------------------------------------------------------------------- */

/* xPixelOpsSTD::CountNonZero, libs/pmbb-core/src/xPixelOpsSTD.cpp:273-284 */
int32_t qo_count_nonzero(const uint16_t* msk, int32_t W, int32_t H)
{
  int32_t n = 0;
  for(size_t i = 0; i < (size_t)W * H; i++) { n += msk[i] != 0; }
  return n;
}

/* xGlobClrDiff::CalcGlobalColorDiffM, libs/pmbb-ivqm/src/xGlobClrDiff.cpp:60-91, with
   xDistortionSTD::CalcWeightedSD (libs/pmbb-core/src/xDistortionSTD.cpp:45-56: int32 product). */
void qo_gcd_masked(const uint16_t* tst, const uint16_t* ref, const uint16_t* msk, int32_t W, int32_t H, int32_t bitdepth,
                   int32_t mask_bitdepth, const float coef[4], int32_t nnm, int32_t gcd[4])
{
  const int32_t maxv = qo_max_value(bitdepth);
  int64_t sd[4] = { 0, 0, 0, 0 };
  for(int32_t c = 0; c < 3; c++)
  {
    const uint16_t* t = tst + (size_t)c * W * H;
    const uint16_t* r = ref + (size_t)c * W * H;
    for(size_t i = 0; i < (size_t)W * H; i++) { sd[c] += qo_mul_wrap((int32_t)t[i] - (int32_t)r[i], (int32_t)msk[i]); }
  }
  const double den = (double)((int64_t)nnm * (int64_t)qo_max_value(mask_bitdepth));
  for(int32_t c = 0; c < 4; c++)
  {
    const int32_t maxdiff = qo_round_f32(coef[c] * (float)maxv);
    gcd[c] = qo_clampi(qo_round_f64((double)sd[c] / den), -maxdiff, maxdiff);
  }
}

/* One masked CPS direction, xCorrespPixelShiftSTD::CalcDistAsymmetricRowM and
   FindBestPixelWithinBlockM, libs/pmbb-ivqm/src/xCorrespPixelShiftSTD.cpp:151-215: masked test pixels
   are skipped, masked candidates are skipped (the mask is edge-extended like the pictures), the
   winner's squared differences are weighted by the test pixel's mask value, uint64 row sums. */
void qo_cps_masked(const uint16_t* tst, const uint16_t* ref, const uint16_t* msk, int32_t W, int32_t H, const int32_t gcd[4],
                   int32_t R, const int32_t cws[4], uint64_t* row_sse)
{
  const size_t pl = (size_t)W * H;
  for(int32_t y = 0; y < H; y++)
  {
    uint64_t rowsum[3] = { 0, 0, 0 };
    for(int32_t x = 0; x < W; x++)
    {
      const int32_t m = msk[(size_t)y * W + x];
      if(m == 0) { continue; }
      int32_t s[3];
      for(int32_t c = 0; c < 3; c++) { s[c] = (int32_t)tst[c * pl + (size_t)y * W + x] + gcd[c]; }
      int32_t best_err = INT32_MAX; int32_t best_pel[3] = { 0, 0, 0 };
      for(int32_t dy = -R; dy <= R; dy++)
      {
        const int32_t yy = qo_clampi(y + dy, 0, H - 1);
        for(int32_t dx = -R; dx <= R; dx++)
        {
          const int32_t xx = qo_clampi(x + dx, 0, W - 1);
          if(msk[(size_t)yy * W + xx] == 0) { continue; }
          uint32_t err = 0; int32_t pel[3];
          for(int32_t c = 0; c < 3; c++)
          {
            pel[c] = ref[c * pl + (size_t)yy * W + xx];
            const int32_t d = s[c] - pel[c];
            err += (uint32_t)qo_mul_wrap(d, d) * (uint32_t)cws[c];
          }
          if((int32_t)err < best_err) { best_err = (int32_t)err; for(int32_t c = 0; c < 3; c++) { best_pel[c] = pel[c]; } }
        }
      }
      for(int32_t c = 0; c < 3; c++)
      {
        const int32_t d = s[c] - best_pel[c];
        rowsum[c] += (uint64_t)(int64_t)qo_mul_wrap(d, d) * (uint64_t)m;
      }
    }
    for(int32_t c = 0; c < 3; c++) { row_sse[(size_t)y * 3 + c] = rowsum[c]; }
  }
}

/* xPSNR::CalcPSNRfromMaskedSSD, libs/pmbb-ivqm/src/xPSNR.cpp:198-205 (MAX formed in int64) */
static double qo_psnr_from_masked_ssd(double ssd, int32_t nnm, int32_t bitdepth_pic, int32_t bitdepth_msk)
{
  const uint64_t mp = (uint64_t)qo_max_value(bitdepth_pic), mm = (uint64_t)qo_max_value(bitdepth_msk);
  const int64_t  MAX = (int64_t)((uint64_t)(int64_t)nnm * (mp * mp) * mm);
  return ssd > 0 ? 10.0 * log10((double)MAX / ssd) : DBL_MAX;
}

/* xIVPSNRM::xCalcQualAsymmetricPicM, libs/pmbb-ivqm/src/xIVPSNR.cpp:172-200 */
static double qo_ivpsnr_quality_masked(const uint64_t* row_sse, int32_t H, int32_t bitdepth, int32_t mask_bitdepth, int32_t nnm,
                                       const double* ws, const int32_t cwa[4])
{
  double err[3];
  for(int32_t c = 0; c < 3; c++)
  {
    if(ws)
    {
      qo_kbns k = { 0.0, 0.0 };
      for(int32_t y = 0; y < H; y++) { qo_kbns_add(&k, (double)row_sse[(size_t)y * 3 + c] * ws[y]); }
      err[c] = qo_kbns_result(&k);
    }
    else
    {
      uint64_t t = 0;
      for(int32_t y = 0; y < H; y++) { t += row_sse[(size_t)y * 3 + c]; }
      err[c] = (double)t;
    }
  }
  double q[4] = { 0, 0, 0, 0 };
  for(int32_t c = 0; c < 3; c++) { q[c] = qo_psnr_from_masked_ssd(err[c] > 0 ? err[c] : 1.0, nnm, bitdepth, mask_bitdepth); }
  const int32_t wsum = cwa[0] + cwa[1] + cwa[2] + cwa[3];
  const double  inv  = 1.0 / (double)wsum;
  return (q[0] * (double)cwa[0] + q[1] * (double)cwa[1] + q[2] * (double)cwa[2] + q[3] * (double)cwa[3]) * inv;
}

/* Mask mode of the app: apps/QMIV/src/xAppQMIV.cpp:900-906 (NumNonMasked), :930 (GCD-M), :971 (PSNR-M),
   :999 (WS-PSNR-M), :1026-1028 (IV-PSNR-M); SSIM metrics are refused with a mask (:360-365).
   mask_plane: W x H, 1 byte per sample for mask_bitdepth 8, else 2. */
int qo_compute_pair_masked(const qo_params* p, const void* const planes0[3], const void* const planes1[3], const void* mask_plane,
                           int32_t mask_bitdepth, uint32_t mask, qo_result* out, int32_t* num_non_masked)
{
  if(mask & (QO_SSIM | QO_MSSSIM | QO_IVSSIM | QO_IVMSSSIM)) { return 1; }
  const int32_t W = p->width, H = p->height, BD = p->bitdepth;
  const size_t  n = (size_t)W * H * 3, pl = (size_t)W * H;
  const int64_t area = (int64_t)W * H;
  memset(out, 0, sizeof(*out));

  uint16_t* P0 = (uint16_t*)malloc(n * sizeof(uint16_t));
  uint16_t* P1 = (uint16_t*)malloc(n * sizeof(uint16_t));
  uint16_t* M  = (uint16_t*)malloc(pl * sizeof(uint16_t));
  qo_unpack444(planes0, W, H, BD, p->chroma_format, P0);
  qo_unpack444(planes1, W, H, BD, p->chroma_format, P1);
  for(size_t i = 0; i < pl; i++) { M[i] = mask_bitdepth <= 8 ? ((const uint8_t*)mask_plane)[i] : ((const uint16_t*)mask_plane)[i]; }
  const int32_t nnm = qo_count_nonzero(M, W, H);
  *num_non_masked = nnm;

  int32_t exact[3];
  for(int32_t c = 0; c < 3; c++)
  {
    exact[c] = memcmp(P0 + (size_t)c * pl, P1 + (size_t)c * pl, pl * sizeof(uint16_t)) == 0;
    out->exact[c] = exact[c];
  }
  double* ws = NULL; double ws_corr = 1.0;
  if(p->erp) { ws = (double*)malloc((size_t)H * sizeof(double)); qo_ws_weights(H, p->lat_range, ws, &ws_corr); }
  const double inv_cwa = 1.0 / (double)(p->cwa[0] + p->cwa[1] + p->cwa[2] + p->cwa[3]);
  #define QO_PER_PIC(v) (((v)[0] * p->cwa[0] + (v)[1] * p->cwa[1] + (v)[2] * p->cwa[2]) * inv_cwa) /* xMetricQMIV.cpp:91-97 */
  const double fake = qo_psnr_from_ssd(1, area, BD); /* getFakePSNR(area, picture bit depth), xAppQMIV.cpp:974-981 */

  int32_t gcd[4] = { 0, 0, 0, 0 }, ngcd[4];
  if(mask & QO_IVPSNR) { qo_gcd_masked(P1, P0, M, W, H, BD, mask_bitdepth, p->unc, nnm, gcd); } /* swap as xGlobClrDiff.h:42 */
  for(int32_t c = 0; c < 4; c++) { out->gcd_r2t[c] = gcd[c]; ngcd[c] = -gcd[c]; }

  if(mask & (QO_PSNR | QO_WSPSNR))
  {
    /* xDistortionSTD::CalcWeightedSSD, libs/pmbb-core/src/xDistortionSTD.cpp:57-68 */
    uint64_t ssd[3] = { 0, 0, 0 };
    for(int32_t c = 0; c < 3; c++)
    {
      const uint16_t* a = P0 + (size_t)c * pl; const uint16_t* b = P1 + (size_t)c * pl;
      for(size_t i = 0; i < pl; i++) { const int32_t d = (int32_t)a[i] - (int32_t)b[i]; ssd[c] += (uint64_t)(int64_t)qo_mul_wrap(d, d) * (uint64_t)M[i]; }
    }
    /* xPSNR::calcPicPSNRM, libs/pmbb-ivqm/src/xPSNR.cpp:54-66: the mask's bit depth stands for both
       the picture's and the mask's (CalcPSNRsFromMaskedSSDs(.., Msk->getBitDepth(), Msk->getBitDepth())) */
    double psnrm[3];
    for(int32_t c = 0; c < 3; c++) { psnrm[c] = qo_psnr_from_masked_ssd((double)ssd[c], nnm, mask_bitdepth, mask_bitdepth); }
    if(mask & QO_PSNR)
    {
      for(int32_t c = 0; c < 3; c++) { out->psnr[c] = exact[c] ? fake : psnrm[c]; }
      out->psnr_pic = QO_PER_PIC(out->psnr);
    }
    if(mask & QO_WSPSNR) /* xWSPSNR.cpp:51-77 (no ERP: PSNR-M), :108-133 */
    {
      for(int32_t c = 0; c < 3; c++)
      {
        double v = psnrm[c];
        if(ws)
        {
          const uint16_t* a = P0 + (size_t)c * pl; const uint16_t* b = P1 + (size_t)c * pl;
          qo_kbns k = { 0.0, 0.0 };
          for(int32_t y = 0; y < H; y++)
          {
            uint64_t rs = 0;
            for(int32_t x = 0; x < W; x++)
            {
              const size_t i = (size_t)y * W + x;
              const int32_t d = (int32_t)b[i] - (int32_t)a[i];
              rs += (uint64_t)(int64_t)qo_mul_wrap(d, d) * (uint64_t)M[i];
            }
            qo_kbns_add(&k, (double)rs * ws[y]);
          }
          const double e = qo_kbns_result(&k) * ws_corr;
          v = qo_psnr_from_masked_ssd(e, nnm, BD, mask_bitdepth);
        }
        out->wspsnr[c] = exact[c] ? fake : v;
      }
      out->wspsnr_pic = QO_PER_PIC(out->wspsnr);
    }
  }
  if(mask & QO_IVPSNR) /* xIVPSNRM::calcPicIVPSNRM, xIVPSNR.cpp:153-170: R2T searches In1 in In0 with -GCD */
  {
    uint64_t* rows = (uint64_t*)malloc((size_t)H * 3 * sizeof(uint64_t));
    qo_cps_masked(P1, P0, M, W, H, ngcd, p->search_range, p->cws, rows);
    const double r2t = qo_ivpsnr_quality_masked(rows, H, BD, mask_bitdepth, nnm, ws, p->cwa);
    qo_cps_masked(P0, P1, M, W, H, gcd, p->search_range, p->cws, rows);
    const double t2r = qo_ivpsnr_quality_masked(rows, H, BD, mask_bitdepth, nnm, ws, p->cwa);
    free(rows);
    out->ivpsnr_r2t = r2t; out->ivpsnr_t2r = t2r;
    out->ivpsnr = t2r < r2t ? t2r : r2t;
  }
  #undef QO_PER_PIC
  free(P0); free(P1); free(M); free(ws);
  return 0;
}

/* ----------------------------------------------------------------------------------------------- */
/* Full frame pipeline, apps/QMIV/src/xAppQMIV.cpp:761-827 and the calcFrame* functions :927-1108   */
/* ----------------------------------------------------------------------------------------------- */
static int qo_compute_pair_impl(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask,
                                qo_result* out, uint16_t* scp0, uint16_t* scp1, const qo_ssim_cfg* cfg);

int qo_compute_pair(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask,
                    qo_result* out, uint16_t* scp0, uint16_t* scp1)
{
  return qo_compute_pair_impl(p, planes0, planes1, mask, out, scp0, scp1, &qo_ssim_default);
}

int qo_compute_pair_ssim(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask,
                         const qo_ssim_cfg* cfg, qo_result* out)
{
  return qo_compute_pair_impl(p, planes0, planes1, mask, out, NULL, NULL, cfg);
}

static int qo_compute_pair_impl(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask,
                                qo_result* out, uint16_t* scp0, uint16_t* scp1, const qo_ssim_cfg* cfg)
{
  const int32_t W = p->width, H = p->height, BD = p->bitdepth;
  const size_t  n = (size_t)W * H * 3;
  const int64_t area = (int64_t)W * H;
  memset(out, 0, sizeof(*out));

  uint16_t* P0 = (uint16_t*)malloc(n * sizeof(uint16_t));
  uint16_t* P1 = (uint16_t*)malloc(n * sizeof(uint16_t));
  qo_unpack444(planes0, W, H, BD, p->chroma_format, P0);
  qo_unpack444(planes1, W, H, BD, p->chroma_format, P1);

  int32_t exact[3];
  for(int32_t c = 0; c < 3; c++) /* equalCmp, xAppQMIV.cpp:894-897 */
  {
    exact[c] = memcmp(P0 + (size_t)c * W * H, P1 + (size_t)c * W * H, (size_t)W * H * sizeof(uint16_t)) == 0;
    out->exact[c] = exact[c];
  }

  double* ws = NULL; double ws_corr = 1.0;
  if(p->erp) { ws = (double*)malloc((size_t)H * sizeof(double)); qo_ws_weights(H, p->lat_range, ws, &ws_corr); }

  const double inv_cwa = 1.0 / (double)(p->cwa[0] + p->cwa[1] + p->cwa[2] + p->cwa[3]);
  #define QO_PER_PIC(v) (((v)[0] * p->cwa[0] + (v)[1] * p->cwa[1] + (v)[2] * p->cwa[2]) * inv_cwa) /* xMetricQMIV.cpp:91-97 */
  #define QO_PER_PIC4(v) (((v)[0] * (double)p->cwa[0] + (v)[1] * (double)p->cwa[1] + (v)[2] * (double)p->cwa[2] + 0.0 * (double)p->cwa[3]) * inv_cwa) /* xIVSSIM.cpp:51-52 */

  const int need_scp = (mask & (QO_IVSSIM | QO_IVMSSSIM)) || scp0 || scp1;
  const int need_gcd = (mask & (QO_IVPSNR | QO_IVSSIM | QO_IVMSSSIM)) || need_scp;
  int32_t gcd[4] = { 0, 0, 0, 0 }, ngcd[4];
  if(need_gcd) { qo_gcd(P1, P0, W, H, BD, p->unc, gcd); } /* argument swap, xGlobClrDiff.h:41 */
  for(int32_t c = 0; c < 4; c++) { out->gcd_r2t[c] = gcd[c]; ngcd[c] = -gcd[c]; }

  uint16_t* S0 = NULL; uint16_t* S1 = NULL;
  if(need_scp) /* xShftCompPic.cpp:219-228 via xAppQMIV.cpp:934-948 */
  {
    S0 = (uint16_t*)malloc(n * sizeof(uint16_t));
    S1 = (uint16_t*)malloc(n * sizeof(uint16_t));
    qo_cps(P0, P1, W, H, BD, gcd, p->search_range, p->cws, NULL, S1);
    qo_cps(P1, P0, W, H, BD, ngcd, p->search_range, p->cws, NULL, S0);
    if(scp0) { memcpy(scp0, S0, n * sizeof(uint16_t)); }
    if(scp1) { memcpy(scp1, S1, n * sizeof(uint16_t)); }
  }

  const double fake = qo_psnr_from_ssd(1, area, BD); /* xPSNR.h:55 */
  if(mask & (QO_PSNR | QO_WSPSNR))
  {
    uint64_t ssd[3] = { 0, 0, 0 };
    for(int32_t c = 0; c < 3; c++)
    {
      const uint16_t* a = P0 + (size_t)c * W * H; const uint16_t* b = P1 + (size_t)c * W * H;
      for(size_t i = 0; i < (size_t)W * H; i++) { const int64_t d = (int64_t)a[i] - b[i]; ssd[c] += (uint64_t)(d * d); }
    }
    if(mask & QO_PSNR) /* xPSNR.cpp:146-152, fake values xAppQMIV.cpp:974-981 */
    {
      for(int32_t c = 0; c < 3; c++) { out->psnr[c] = exact[c] ? fake : qo_psnr_from_ssd((double)ssd[c], area, BD); }
      out->psnr_pic = QO_PER_PIC(out->psnr);
    }
    if(mask & QO_WSPSNR) /* xWSPSNR.cpp:48-81, :112-138 */
    {
      for(int32_t c = 0; c < 3; c++)
      {
        double v;
        if(!ws) { v = qo_psnr_from_ssd((double)ssd[c], area, BD); }
        else
        {
          const uint16_t* a = P0 + (size_t)c * W * H; const uint16_t* b = P1 + (size_t)c * W * H;
          qo_kbns k = { 0.0, 0.0 };
          for(int32_t y = 0; y < H; y++)
          {
            uint64_t rs = 0;
            for(int32_t x = 0; x < W; x++) { const int64_t d = (int64_t)a[(size_t)y * W + x] - b[(size_t)y * W + x]; rs += (uint64_t)(d * d); }
            qo_kbns_add(&k, (double)rs * ws[y]);
          }
          const double e = qo_kbns_result(&k) * ws_corr;
          v = qo_psnr_from_ssd(e, area, BD);
        }
        out->wspsnr[c] = exact[c] ? fake : v;
      }
      out->wspsnr_pic = QO_PER_PIC(out->wspsnr);
    }
  }

  if(mask & QO_IVPSNR) /* xIVPSNR.cpp:109-121 */
  {
    uint64_t* rows = (uint64_t*)malloc((size_t)H * 3 * sizeof(uint64_t));
    qo_cps(P0, P1, W, H, BD, gcd, p->search_range, p->cws, rows, NULL);
    const double r2t = qo_ivpsnr_quality(rows, W, H, BD, ws, p->cwa);
    qo_cps(P1, P0, W, H, BD, ngcd, p->search_range, p->cws, rows, NULL);
    const double t2r = qo_ivpsnr_quality(rows, W, H, BD, ws, p->cwa);
    free(rows);
    out->ivpsnr_r2t = r2t; out->ivpsnr_t2r = t2r;
    out->ivpsnr = t2r < r2t ? t2r : r2t; /* std::min */
  }

  int rc = 0;
  if(mask & QO_SSIM) /* xSSIM.h:83 -> xSSIM.cpp:199-234, no ERP weighting */
  {
    rc |= qo_ssim_pic_cfg(P0, P1, W, H, BD, 1, NULL, cfg, out->ssim);
    out->ssim_pic = QO_PER_PIC(out->ssim);
  }
  if(mask & QO_MSSSIM)
  {
    rc |= qo_msssim_pic_cfg(P0, P1, W, H, BD, cfg, out->msssim);
    out->msssim_pic = QO_PER_PIC(out->msssim);
  }
  if(mask & QO_IVSSIM) /* xIVSSIM.cpp:31-61 */
  {
    double t2r[3], r2t[3];
    rc |= qo_ssim_pic_cfg(P0, S1, W, H, BD, 1, ws, cfg, t2r);
    rc |= qo_ssim_pic_cfg(P1, S0, W, H, BD, 1, ws, cfg, r2t);
    out->ivssim_t2r = QO_PER_PIC4(t2r); out->ivssim_r2t = QO_PER_PIC4(r2t);
    out->ivssim = out->ivssim_r2t < out->ivssim_t2r ? out->ivssim_r2t : out->ivssim_t2r;
  }
  if(mask & QO_IVMSSSIM) /* xIVSSIM.cpp:62-92, no ERP weighting */
  {
    double t2r[3], r2t[3];
    rc |= qo_msssim_pic_cfg(P0, S1, W, H, BD, cfg, t2r);
    rc |= qo_msssim_pic_cfg(P1, S0, W, H, BD, cfg, r2t);
    out->ivmsssim_t2r = QO_PER_PIC4(t2r); out->ivmsssim_r2t = QO_PER_PIC4(r2t);
    out->ivmsssim = out->ivmsssim_r2t < out->ivmsssim_t2r ? out->ivmsssim_r2t : out->ivmsssim_t2r;
  }
  #undef QO_PER_PIC
  #undef QO_PER_PIC4

  free(P0); free(P1); free(S0); free(S1); free(ws);
  return rc;
}
