/*
  qmiv_oracle — CPU restatement of the QMIV (pmbb-ivqm) metric hot path in plain C.

  TEST INFRASTRUCTURE ONLY. This is the checker the parity tests, __graft_entry__.smoke() and the
  cpu_baseline leg of bench.py compare the CUDA library against. It is never linked into, loaded by
  or called from the product library (qmiv_b200/libqmiv_b200.so).

  Parity pinning: the restatement is checked against the reference itself, compiled from its own
  sources by oracle/Makefile into oracle/_ref/ (tests/test_oracle_vs_reference.py), and against the
  golden fixtures in tests/golden/ that were produced by that compiled reference
  (tests/golden/make_golden.py).

  Every function cites the reference file:line it restates (paths relative to the QMIV repository).
*/
#ifndef QMIV_ORACLE_H
#define QMIV_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* metric bits, same as qmiv_gpu.h */
enum
{
  QO_PSNR = 1, QO_WSPSNR = 2, QO_IVPSNR = 4, QO_SSIM = 8, QO_MSSSIM = 16, QO_IVSSIM = 32, QO_IVMSSSIM = 64
};

typedef struct qo_params
{
  int32_t width, height, bitdepth, chroma_format; /* chroma_format: 420, 422 or 444 */
  int32_t search_range;                           /* CPS window is (2R+1)^2 */
  int32_t cws[4];                                 /* component weights used in the search */
  int32_t cwa[4];                                 /* component weights used for averaging */
  float   unc[4];                                 /* unnoticeable colour difference coefficients */
  int32_t erp, lon_range, lat_range;              /* equirectangular (WS) weighting */
  int32_t num_threads;                            /* unused by the oracle, kept for layout parity */
} qo_params;

/* Same layout as ref_result in ref_shim.cpp so the two can be compared field by field. */
typedef struct qo_result
{
  int32_t gcd_r2t[4];
  int32_t exact[4];
  double  psnr[4];   double psnr_pic;
  double  wspsnr[4]; double wspsnr_pic;
  double  ivpsnr;    double ivpsnr_r2t;   double ivpsnr_t2r;
  double  ssim[4];   double ssim_pic;
  double  msssim[4]; double msssim_pic;
  double  ivssim;    double ivssim_r2t;   double ivssim_t2r;
  double  ivmsssim;  double ivmsssim_r2t; double ivmsssim_t2r;
} qo_result;

/* Raw frame -> planar 4:4:4 uint16 (3*W*H). planes[c] is 1 byte/sample if bitdepth <= 8, else 2. */
void qo_unpack444(const void* const planes[3], int32_t W, int32_t H, int32_t bitdepth, int32_t chroma_format, uint16_t* dst);

/* xGlobClrDiff::CalcGlobalColorDiff(Tst, Ref, coef): round(mean(Tst - Ref)) clipped. 4:4:4 planar inputs. */
void qo_gcd(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, const float coef[4], int32_t gcd[4]);

/* One CPS direction: row_sse[y*3+c] (x86 SSE-path semantics) and, if scp != NULL, the
   shift-compensated picture (3*W*H). */
void qo_cps(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, const int32_t gcd[4],
            int32_t R, const int32_t cws[4], uint64_t* row_sse, uint16_t* scp);

/* Portable-path (xCorrespPixelShiftSTD, uint64 row accumulation) variant of qo_cps's row SSE. */
void qo_cps_rows_std(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, const int32_t gcd[4],
                     int32_t R, const int32_t cws[4], uint64_t* row_sse);

/* Equirectangular row weights and the WS-PSNR distortion correction. */
void qo_ws_weights(int32_t H, int32_t lat_range, double* weights, double* correction);

/* Per-channel block-averaged SSIM (8x8 windows, stride 4) of one 4:4:4 picture pair. weights may be NULL. */
void qo_ssim_pic(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, int32_t calc_l,
                 const double* ws_weights, double out[3]);

/* Per-channel MS-SSIM of one 4:4:4 picture pair. Returns 0, or -1 when the picture is too small. */
int qo_msssim_pic(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, double out[3]);

/* Structural similarity options of the app (-ssm, -ssb, -ssw, -sss; apps/QMIV/src/xAppQMIV.cpp:99-104):
   mode as xSSIM::eMode (libs/pmbb-ivqm/src/xSSIM.h:23-31), border as eMrgExt
   (libs/pmbb-core/src/xCommonDefCORE.h:322-331). The app's default is BlockAveraged, None, 8, 4. */
enum
{
  QO_SSM_REGULAR_GAUSSIAN_FLT = 0, QO_SSM_REGULAR_GAUSSIAN_INT = 1, QO_SSM_REGULAR_AVERAGED = 2,
  QO_SSM_BLOCK_GAUSSIAN_INT = 3, QO_SSM_BLOCK_AVERAGED = 4
};
enum { QO_BRD_NONE = 0, QO_BRD_NEAREST = 1, QO_BRD_REFLECT = 2, QO_BRD_MIRROR = 3, QO_BRD_CONSTANT = 4, QO_BRD_ZERO = 5 };
typedef struct qo_ssim_cfg
{
  int32_t mode, border, window, stride;
} qo_ssim_cfg;

/* Per-channel SSIM of one 4:4:4 picture pair under any structural similarity option. ws_weights (ERP,
   may be NULL) weight the window rows as xIVSSIM does. Returns 0, or -1 for an option the reference
   cannot evaluate (see qo_ssim_cfg_check). */
int qo_ssim_pic_cfg(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, int32_t calc_l,
                    const double* ws_weights, const qo_ssim_cfg* cfg, double out[3]);
int qo_msssim_pic_cfg(const uint16_t* tst, const uint16_t* ref, int32_t W, int32_t H, int32_t bitdepth, const qo_ssim_cfg* cfg,
                      double out[3]);
/* 0 when the option set is one this restatement evaluates for a W x H picture, else -1. */
int qo_ssim_cfg_check(const qo_ssim_cfg* cfg, int32_t W, int32_t H);
/* The frame pipeline with the given structural similarity options. */
int qo_compute_pair_ssim(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask,
                         const qo_ssim_cfg* cfg, qo_result* out);

/* Number of MS-SSIM scales (xSSIM::xCalcNumScales). */
int32_t qo_num_scales(int32_t W, int32_t H);

/* Full per-frame pipeline of the reference app for one raw frame pair. scp0/scp1 optional (3*W*H). */
int qo_compute_pair(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask,
                    qo_result* out, uint16_t* scp0, uint16_t* scp1);

/* Colour-space conversion of the app (-csi / -csm, codes as eClrSpcApp: RGB 2, BGR 3, GBR 4, YCbCr 16,
   BT601 17, SMPTE170M 18, BT709 19, SMPTE240M 20, BT2020 21) on two 4:4:4 planar pictures, in place,
   and the frame pipeline after it. Nonzero for combinations the app refuses. */
int qo_convert_colour(uint16_t* P0, uint16_t* P1, int32_t W, int32_t H, int32_t bitdepth, int32_t cs_in, int32_t cs_metric);
int qo_compute_pair_cs(const qo_params* p, const void* const planes0[3], const void* const planes1[3], uint32_t mask, int32_t cs_in,
                       int32_t cs_metric, qo_result* out);

/* Mask mode (GCD-M, CPS-M, PSNR-M, WS-PSNR-M, IV-PSNR-M): mask_plane is the mask's luma, W x H,
   1 byte per sample for mask_bitdepth 8, else 2. Returns nonzero for SSIM metric bits. */
int qo_compute_pair_masked(const qo_params* p, const void* const planes0[3], const void* const planes1[3], const void* mask_plane,
                           int32_t mask_bitdepth, uint32_t mask, qo_result* out, int32_t* num_non_masked);
int32_t qo_count_nonzero(const uint16_t* msk, int32_t W, int32_t H);
void qo_gcd_masked(const uint16_t* tst, const uint16_t* ref, const uint16_t* msk, int32_t W, int32_t H, int32_t bitdepth,
                   int32_t mask_bitdepth, const float coef[4], int32_t nnm, int32_t gcd[4]);
void qo_cps_masked(const uint16_t* tst, const uint16_t* ref, const uint16_t* msk, int32_t W, int32_t H, const int32_t gcd[4],
                   int32_t R, const int32_t cws[4], uint64_t* row_sse);

#ifdef __cplusplus
}
#endif
#endif
