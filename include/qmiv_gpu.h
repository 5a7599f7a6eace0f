/*
  qmiv_gpu.h — C ABI of the B200 (sm_100a) implementation of the QMIV metric hot path.

  The entry points replace the pmbb-ivqm metric-calculator calls that the QMIV app makes per frame
  (apps/QMIV/src/xAppQMIV.cpp:927-1108). Plain pointers, sizes and status codes only: no C++ or
  torch types cross this boundary. All entry points return a qmiv_status; none throws.

  Ownership: the caller owns every host buffer it passes; the library owns all device memory it
  allocates (a calc's buffers count against its context's HBM budget). Device-resident frames may
  also be passed (QMIV_MEM_DEVICE); they stay owned by the caller.
  Threading: a qmiv_calc is not re-entrant (as a reference processor with its row buffers is not,
  libs/pmbb-ivqm/src/xMetricCommon.h:23-27); different calcs may be used from different threads.

  Reference interfaces replaced (paths inside the QMIV repository):
    qmiv_calc_create        xGlobClrDiffProc / xShftCompPicProc / xIVPSNRM / xIVSSIM set-up:
                            setSearchRange, setCmpWeightsSearch/Average, setUnntcbCoef, initRowBuffers,
                            initWS, xSSIM::create, setStructSimParams
                            (apps/QMIV/src/xAppQMIV.cpp:680-744; xCorrespPixelShiftPrms.h:30-32;
                             xGlobClrDiff.h:24; xMetricCommon.cpp:12-19; xWeightedSpherically.h:21;
                             xSSIM.h:78-81)
    qmiv_calc_gcd           xGlobClrDiffProc::CalcGlobalColorDiff (xGlobClrDiff.h:41)
    qmiv_calc_scp           xShftCompPicProc::GenShftCompPics (xShftCompPic.h:44-47)
    qmiv_frame_pair_compute one frame of processAllFrames: calcFrameGCD, calcFrameSCP and the
                            calcFrame* metric calls (apps/QMIV/src/xAppQMIV.cpp:761-827):
                            xPSNR::calcPicPSNR (xPSNR.h:89), xWSPSNR::calcPicWSPSNR (xWSPSNR.h:22),
                            xIVPSNR::calcPicIVPSNR (xIVPSNR.h:36), xSSIM::calcPicSSIM / calcPicMSSSIM
                            (xSSIM.h:83-84), xIVSSIM::calcPicIVSSIM / calcPicIVMSSSIM (xIVSSIM.h:39-40)
    qmiv_batch_*            no single reference counterpart: the reference processes frames one at a
                            time (xAppQMIV.cpp:761); the batch runs many frame pairs of uneven shape
                            per launch.
    qmiv_server_*           no reference counterpart (the reference has no serving mode).
*/
#ifndef QMIV_GPU_H
#define QMIV_GPU_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define QMIV_API_VERSION 1

#if defined(__GNUC__)
#define QMIV_API __attribute__((visibility("default")))
#else
#define QMIV_API
#endif

typedef enum qmiv_status
{
  QMIV_OK                 = 0,
  QMIV_ERR_INVALID_ARG    = 1,  /* null pointer, bad size, bad parameter value */
  QMIV_ERR_UNSUPPORTED    = 2,  /* valid in the reference but not implemented here */
  QMIV_ERR_CUDA           = 3,  /* a CUDA runtime call failed (see qmiv_last_error) */
  QMIV_ERR_OUT_OF_MEMORY  = 4,  /* device allocation failed */
  QMIV_ERR_INVALID_PIXEL  = 5,  /* a sample exceeds the bit depth's range and the action is STOP */
  QMIV_ERR_BUDGET         = 6,  /* the request does not fit in the context's HBM budget */
  QMIV_ERR_TIMEOUT        = 7,  /* a bounded wait ran out */
  QMIV_ERR_NOT_READY      = 8,  /* asynchronous result not available yet */
  QMIV_ERR_CANCELLED      = 9,  /* request cancelled before it ran */
  QMIV_ERR_BUSY           = 10  /* no free slot / queue full */
} qmiv_status;

/* metric selection bits (apps/QMIV/src/xAppQMIV.cpp:60-63 metric list) */
enum
{
  QMIV_PSNR     = 1u << 0,
  QMIV_WSPSNR   = 1u << 1,
  QMIV_IVPSNR   = 1u << 2,
  QMIV_SSIM     = 1u << 3,
  QMIV_MSSSIM   = 1u << 4,
  QMIV_IVSSIM   = 1u << 5,
  QMIV_IVMSSSIM = 1u << 6,
  QMIV_ALL      = 0x7Fu
};

/* where a frame's planes live */
enum { QMIV_MEM_HOST = 0, QMIV_MEM_DEVICE = 1 };

/* invalid-pixel action (apps/QMIV/src/xAppQMIV.cpp:834-852, README "InvalidPelActn") */
enum { QMIV_PEL_SKIP = 0, QMIV_PEL_WARN = 1, QMIV_PEL_STOP = 2, QMIV_PEL_CNCL = 3 };

/* Structural similarity window modes of the app's StructSimMode option, same codes as xSSIM::eMode
   (libs/pmbb-ivqm/src/xSSIM.h:23-31): regular 11x11 windows centred on every pixel (Gaussian float,
   Gaussian integer or averaged weights), block windows of 8, 16 or 32 samples anchored at their
   top-left sample (Gaussian integer 8/16 or averaged). */
enum
{
  QMIV_SSM_REGULAR_GAUSSIAN_FLT = 0, QMIV_SSM_REGULAR_GAUSSIAN_INT = 1, QMIV_SSM_REGULAR_AVERAGED = 2,
  QMIV_SSM_BLOCK_GAUSSIAN_INT = 3, QMIV_SSM_BLOCK_AVERAGED = 4
};

/* Border extension of the regular windows (StructSimBrdExt), same codes as eMrgExt
   (libs/pmbb-core/src/xCommonDefCORE.h:322-331). QMIV_BRD_NONE evaluates only the windows inside the
   picture; the others evaluate a window at every pixel and extend the picture like xMarginOps
   (Constant = 65535). */
enum { QMIV_BRD_NONE = 0, QMIV_BRD_NEAREST = 1, QMIV_BRD_REFLECT = 2, QMIV_BRD_MIRROR = 3, QMIV_BRD_CONSTANT = 4, QMIV_BRD_ZERO = 5 };

/* Colour spaces of the app's ColorSpaceInput / ColorSpaceMetric options, same codes as its eClrSpcApp
   (apps/QMIV/src/xUtilsQMIV.h:12-27). QMIV_CS_YCBCR is the generic (unspecified) YCbCr. */
enum
{
  QMIV_CS_RGB = 2, QMIV_CS_BGR = 3, QMIV_CS_GBR = 4,
  QMIV_CS_YCBCR = 16, QMIV_CS_BT601 = 17, QMIV_CS_SMPTE170M = 18, QMIV_CS_BT709 = 19, QMIV_CS_SMPTE240M = 20, QMIV_CS_BT2020 = 21
};

typedef struct qmiv_ctx_s*    qmiv_ctx;
typedef struct qmiv_calc_s*   qmiv_calc;
typedef struct qmiv_batch_s*  qmiv_batch;
typedef struct qmiv_server_s* qmiv_server;

/* Processor parameters. qmiv_params_default() gives the reference defaults:
   R=2, weights 4:1:1:0 (xCorrespPixelShiftPrms.h:22-24), unnoticeable coef 0.01 (xGlobClrDiff.h:20),
   BlockAveraged SSIM with 8x8 windows at stride 4 and no border extension (xSSIM.h:35-37), no ERP,
   STOP on invalid pixels. The SSIM options follow xSSIM::setStructSimParams (xSSIM.cpp:86-113) with
   the app's checks (xAppQMIV.cpp:325-332). The batched and serving forms compute SSIM metrics under a
   non-default option pair by pair after the batch (the qmiv_calc path); every other metric batched. */
typedef struct qmiv_params
{
  int32_t search_range;        /* 1..5 */
  int32_t cws[4];              /* search component weights, cws[3] must be 0 */
  int32_t cwa[4];              /* averaging component weights */
  float   unc[4];              /* unnoticeable colour difference coefficients */
  int32_t erp;                 /* equirectangular (WS) weighting on/off */
  int32_t lon_range_deg;       /* 360 */
  int32_t lat_range_deg;       /* 180 */
  int32_t ssim_window;         /* 8; 11 for the regular modes; 8, 16 or 32 for the block modes */
  int32_t ssim_stride;         /* 4; 1..ssim_window */
  int32_t invalid_pel_action;  /* QMIV_PEL_* */
  int32_t ssim_mode;           /* QMIV_SSM_*, default QMIV_SSM_BLOCK_AVERAGED */
  int32_t ssim_border;         /* QMIV_BRD_*, regular modes only, default QMIV_BRD_NONE */
} qmiv_params;

/* One frame: planar Y, Cb, Cr. Samples are 1 byte for bitdepth <= 8, else 2 bytes little endian.
   pitch is in bytes. Chroma planes are (W>>1)x(H>>1) for 4:2:0, (W>>1)xH for 4:2:2, WxH for 4:4:4. */
typedef struct qmiv_frame
{
  const void* plane[3];
  int64_t     pitch[3];
  int32_t     mem;             /* QMIV_MEM_HOST or QMIV_MEM_DEVICE */
} qmiv_frame;

/* Results of one frame pair. Fields of metrics that were not requested are left at 0.
   Direction names follow the reference: R2T searches In0+GCD inside In1, T2R searches In1-GCD
   inside In0 (xIVPSNR.cpp:115-116); IV-SSIM T2R = SSIM(In0, SCP1), R2T = SSIM(In1, SCP0)
   (xIVSSIM.cpp:46-47). */
typedef struct qmiv_result
{
  int32_t  gcd_r2t[4];         /* round(mean(In1 - In0)), clipped (xGlobClrDiff.cpp:70-103) */
  int32_t  exact[4];           /* component identical in both frames (xAppQMIV.cpp:894-897) */
  int32_t  invalid_pel[2];     /* frame 0/1 held samples above the bit depth's maximum */
  uint64_t ssd[4];             /* per-component SSD of the 4:4:4 pictures */
  uint64_t cps_sse_r2t[4];     /* sum over rows of the CPS row SSE, R2T */
  uint64_t cps_sse_t2r[4];     /* sum over rows of the CPS row SSE, T2R */
  double   psnr[4];   double psnr_pic;
  double   wspsnr[4]; double wspsnr_pic;
  double   ivpsnr;    double ivpsnr_r2t;   double ivpsnr_t2r;
  double   ssim[4];   double ssim_pic;
  double   msssim[4]; double msssim_pic;
  double   ivssim;    double ivssim_r2t;   double ivssim_t2r;
  double   ivmsssim;  double ivmsssim_r2t; double ivmsssim_t2r;
} qmiv_result;

/* ---- library / context -------------------------------------------------------------------- */
QMIV_API int32_t     qmiv_api_version(void);
QMIV_API const char* qmiv_status_string(qmiv_status status);
QMIV_API const char* qmiv_last_error(void);          /* thread-local message of the last failure */
QMIV_API void        qmiv_params_default(qmiv_params* params);

/* device: CUDA ordinal. hbm_budget_bytes: cap on the device memory this context's calcs,
   batches and servers may hold (0 = no cap). */
QMIV_API qmiv_status qmiv_ctx_create(int32_t device, uint64_t hbm_budget_bytes, qmiv_ctx* out_ctx);
QMIV_API qmiv_status qmiv_ctx_destroy(qmiv_ctx ctx);
QMIV_API qmiv_status qmiv_ctx_memory(qmiv_ctx ctx, uint64_t* used_bytes, uint64_t* budget_bytes);

/* Per-stage device timing, the counterpart of the reference's per-stage tick accounting at
   VerboseLevel >= 3 (apps/QMIV/src/xAppQMIV.cpp:763-826, AvgTime table :1151-1219). When enabled,
   every calc/batch of the context brackets each stage's launches with CUDA events on the stream
   they run on; qmiv_ctx_stage_times returns the accumulated milliseconds and launch counts per
   stage (indices QMIV_STAGE_*) and, if reset != 0, clears them. */
enum
{
  QMIV_STAGE_H2D = 0,        /* host frame upload */
  QMIV_STAGE_PREPASS = 1,    /* per-row SD/SSD */
  QMIV_STAGE_REDUCE = 2,     /* totals + GCD */
  QMIV_STAGE_CPS = 3,        /* corresponding-pixel-shift search, both directions */
  QMIV_STAGE_SSIM_WIN = 4,   /* SSIM windows (+ pyramid downsampling) */
  QMIV_STAGE_SSIM_ROWS = 5,  /* per-row SSIM sums */
  QMIV_STAGE_FINALIZE = 6,   /* FP64 pooling chains */
  QMIV_STAGE_D2H = 7,        /* result read-back */
  QMIV_NUM_STAGES = 8
};
QMIV_API qmiv_status qmiv_ctx_set_profiling(qmiv_ctx ctx, int32_t enable);
QMIV_API qmiv_status qmiv_ctx_stage_times(qmiv_ctx ctx, double ms[8], uint64_t launches[8], int32_t reset);

/* ---- plain form: one frame pair per call -------------------------------------------------- */
QMIV_API qmiv_status qmiv_calc_create(qmiv_ctx ctx, int32_t width, int32_t height, int32_t bitdepth, int32_t chroma_format,
                             const qmiv_params* params, qmiv_calc* out_calc);
QMIV_API qmiv_status qmiv_calc_destroy(qmiv_calc calc);

/* Full per-frame pipeline (GCD, SCP if needed, requested metrics). Blocks until done. */
QMIV_API qmiv_status qmiv_frame_pair_compute(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1,
                                    uint32_t metric_mask, qmiv_result* out);

/* Asynchronous form: enqueue on the calc's stream; qmiv_frame_pair_wait() returns the result.
   One submission in flight per calc; host frames must stay valid until the wait returns. */
QMIV_API qmiv_status qmiv_frame_pair_submit(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1,
                                   uint32_t metric_mask);
QMIV_API qmiv_status qmiv_frame_pair_wait(qmiv_calc calc, int32_t timeout_ms, qmiv_result* out);

/* Mask mode, the app's -im option (apps/QMIV/src/xAppQMIV.cpp:900-1030): every sample is weighted by
   the mask picture's luma value M(x, y) (plane[0] of `mask`, W x H, 1 byte per sample for
   mask_bitdepth 8, else 2; mask_bitdepth 8..14). Replaces the reference's *M processor calls:
     xGlobClrDiffProc::CalcGlobalColorDiffM   (xGlobClrDiff.h:42)     -> out->gcd_r2t
     xPSNR::calcPicPSNRM                      (xPSNR.cpp:54-66)       -> out->psnr[], psnr_pic
     xWSPSNR::calcPicWSPSNRM                  (xWSPSNR.cpp:51-77)     -> out->wspsnr[], wspsnr_pic
     xIVPSNRM::calcPicIVPSNRM                 (xIVPSNR.cpp:153-170)   -> out->ivpsnr, _r2t, _t2r
   with the reference's arithmetic, including two of its conventions: PSNR-M takes the mask's bit
   depth for the picture's maximum (xPSNR.cpp:61), and IV-PSNR-M labels the search of In1 in In0
   "R2T" (xIVPSNR.cpp:161). out->ssd holds the weighted SSDs, cps_sse_* the weighted CPS sums.
   metric_mask may hold QMIV_PSNR, QMIV_WSPSNR and QMIV_IVPSNR; the SSIM family is refused with
   QMIV_ERR_UNSUPPORTED as the app refuses it (xAppQMIV.cpp:360-365). num_non_masked (may be NULL)
   receives the count of non-zero mask samples (xAppQMIV.cpp:904); an all-zero mask is
   QMIV_ERR_INVALID_ARG. Blocks until done. */
QMIV_API qmiv_status qmiv_frame_pair_compute_masked(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1,
                                                    const qmiv_frame* mask, int32_t mask_bitdepth, uint32_t metric_mask,
                                                    qmiv_result* out, int32_t* num_non_masked);

/* The app's colour-space conversion (ColorSpaceInput -csi, ColorSpaceMetric -csm;
   apps/QMIV/src/xAppQMIV.cpp:299-311, :853-891) for this calc's later qmiv_frame_pair_compute /
   _submit calls: YCbCr (BT.601, SMPTE 170M, BT.709, SMPTE 240M, BT.2020) to RGB, RGB to YCbCr, or BGR /
   GBR reordered to RGB, applied to the 4:4:4 pictures before the exactness check and every metric,
   with the reference's integer arithmetic. Equal spaces (the default, QMIV_CS_YCBCR for both) convert
   nothing. YCbCr to YCbCr is QMIV_ERR_UNSUPPORTED and the generic YCbCr in a conversion
   QMIV_ERR_INVALID_ARG, as the app refuses them. While a conversion is set, qmiv_calc_gcd / _scp /
   _cps_rows are QMIV_ERR_UNSUPPORTED. */
QMIV_API qmiv_status qmiv_calc_set_color_space(qmiv_calc calc, int32_t color_space_input, int32_t color_space_metric);

/* xGlobClrDiffProc::CalcGlobalColorDiff(Tst=In0, Ref=In1) -> round(mean(In1 - In0)), clipped. */
QMIV_API qmiv_status qmiv_calc_gcd(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, int32_t gcd_r2t[4]);

/* xShftCompPicProc::GenShftCompPics as called by the app (xAppQMIV.cpp:934-948): writes the
   shift-compensated pictures SCP0 (In0 resampled onto In1's grid) and SCP1 (In1 onto In0's), planar
   4:4:4, WxH per component, 2-byte samples, into the caller's host or device buffers
   (dst_mem = QMIV_MEM_*). Either destination may be NULL. gcd_r2t may be NULL (computed here). */
QMIV_API qmiv_status qmiv_calc_scp(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, const int32_t* gcd_r2t,
                          uint16_t* scp0, uint16_t* scp1, int32_t dst_mem);

/* Use a caller-supplied GCD (R2T convention) instead of computing it, for the reference's
   calcPicIVPSNR(Tst, Ref, GlobalColorDiffRef2Tst) (xIVPSNR.h:36) and GenShftCompPics(..., GCD)
   (xShftCompPic.h:44-47) forms. NULL restores the computed GCD. Applies to later calls. */
QMIV_API qmiv_status qmiv_calc_set_gcd(qmiv_calc calc, const int32_t* gcd_r2t);

/* Per-row CPS SSE of the last computed pair: rows_r2t/rows_t2r receive H*3 uint64 values
   (row-major, component fastest) with the reference's 32-bit-lane accumulation semantics
   (xCorrespPixelShiftSSE.cpp:29-40). Either pointer may be NULL. */
QMIV_API qmiv_status qmiv_calc_cps_rows(qmiv_calc calc, uint64_t* rows_r2t, uint64_t* rows_t2r);

/* Device stream (cudaStream_t) the calc enqueues on, for callers that order their own work. */
QMIV_API qmiv_status qmiv_calc_stream(qmiv_calc calc, void** cuda_stream);

/* ---- allocation-free form ------------------------------------------------------------------ */
/* No counterpart in the reference. For callers that must not allocate device memory: code running
   inside a host application's own memory manager or a plugin sandbox that forbids cudaMalloc, paths
   that run under a strict no-allocation policy after start-up, and callers whose allocator is not
   theirs to use (allocating there could deadlock or break a memory budget). It computes PSNR,
   WS-PSNR and IV-PSNR (the metrics in `metric_mask`, others are rejected) of one frame pair whose
   planes are already in device memory, enqueued on `cuda_stream` (0 = default stream), and blocks
   until the result is in `out`; it synchronises that stream and copies from pageable host memory, so
   it must not be called on a stream that is being captured into a CUDA graph. It calls no
   cudaMalloc, cudaFree or other allocating routine: its scratch is one fixed file-scope device array
   (about 350 KB per GPU), which limits the picture height to QMIV_STATIC_MAX_HEIGHT rows; taller
   pictures are rejected with QMIV_ERR_UNSUPPORTED. The array comes with the library's device code:
   with CUDA's lazy module loading (the default) it is placed on a GPU at this entry point's first
   call there, and it stays until the process exits, so a caller that may not allocate after
   start-up makes one call on each GPU during start-up. Each call looks up the array's address in the
   context current at the call. All calls share the one array: calls that overlap on the GPU (from
   different threads or streams) race, so serialise them. */
#define QMIV_STATIC_MAX_HEIGHT 4352
QMIV_API qmiv_status qmiv_frame_pair_compute_static(const qmiv_frame* in0, const qmiv_frame* in1, int32_t width,
                                                    int32_t height, int32_t bitdepth, int32_t chroma_format,
                                                    const qmiv_params* params, uint32_t metric_mask,
                                                    void* cuda_stream, qmiv_result* out);

/* ---- batched form: many frame pairs of uneven shape per launch ---------------------------- */
typedef struct qmiv_pair_desc
{
  qmiv_frame in0, in1;
  int32_t    width, height, bitdepth, chroma_format;
  int32_t    search_range;     /* 1..5 */
  uint32_t   metric_mask;
} qmiv_pair_desc;

/* max_pairs: pairs per qmiv_batch_compute call; max_pixels: sum of W*H over one call's pairs.
   params: shared weights/coefficients (search_range is taken per pair). flags: QMIV_BATCH_*. */
enum
{
  QMIV_BATCH_GRAPH    = 1,  /* replay the launch sequence from CUDA graphs keyed by the call's shape signature */
  QMIV_BATCH_AUTOTUNE = 4   /* time the CPS tile shapes on the first pair of every (W, H, bit depth, R) and keep the faster */
};
QMIV_API qmiv_status qmiv_batch_create(qmiv_ctx ctx, int32_t max_pairs, int64_t max_pixels, const qmiv_params* params,
                              int32_t flags, qmiv_batch* out_batch);
QMIV_API qmiv_status qmiv_batch_destroy(qmiv_batch batch);
QMIV_API qmiv_status qmiv_batch_compute(qmiv_batch batch, const qmiv_pair_desc* pairs, int32_t num_pairs, qmiv_result* out);
/* Mask mode for many frame pairs at once: replaces the app's per-frame *M processor calls
   (apps/QMIV/src/xAppQMIV.cpp:900-1030; the reference runs them one frame at a time). pairs[i] as for
   qmiv_batch_compute, whose metric_mask may hold QMIV_PSNR, QMIV_WSPSNR and QMIV_IVPSNR; masks[i] the
   luma plane of pair i's mask picture (plane[0], pitch[0], mem; 1-byte samples for mask_bitdepths[i]
   = 8, 2-byte above, up to 14). Every stage runs as one launch per group of up to 32 pairs with the
   same sample sizes and search range; each result equals qmiv_frame_pair_compute_masked's for that pair.
   num_non_masked may be NULL. Returns the first failing pair's status (the others' results are still
   filled). Blocks until the results are on the host. */
QMIV_API qmiv_status qmiv_batch_compute_masked(qmiv_batch batch, const qmiv_pair_desc* pairs, const qmiv_frame* masks,
                                      const int32_t* mask_bitdepths, int32_t num_pairs, qmiv_result* out,
                                      int32_t* num_non_masked);

/* Asynchronous form of qmiv_batch_compute with two calls in flight: qmiv_batch_submit enqueues a
   call's uploads and launches and returns at once with a ticket; qmiv_batch_wait(ticket) waits for
   that call and writes its results. A third submission before a wait, or qmiv_batch_compute while
   the first slot is held, returns QMIV_ERR_BUSY. Host frames must stay valid until the wait returns.
   With host frames, the uploads of one call overlap the kernels of the other. */
QMIV_API qmiv_status qmiv_batch_submit(qmiv_batch batch, const qmiv_pair_desc* pairs, int32_t num_pairs, uint64_t* ticket);
QMIV_API qmiv_status qmiv_batch_wait(qmiv_batch batch, uint64_t ticket, qmiv_result* results);
/* Device stream (cudaStream_t) the batch enqueues on. */
QMIV_API qmiv_status qmiv_batch_stream(qmiv_batch batch, void** cuda_stream);
/* Tile shapes picked by the autotuner for (width, height, bitdepth, R): for inspection and tests. */
QMIV_API qmiv_status qmiv_batch_tuning(qmiv_batch batch, int32_t width, int32_t height, int32_t bitdepth, int32_t search_range,
                              int32_t* cps_tile_w, int32_t* cps_tile_h, int32_t* cps_rows_per_thread);

/* ---- serving loop: sequences of frame pairs admitted by HBM budget, continuously batched ------ */
/* No reference counterpart: the reference app processes one sequence per process.
   A request is a sequence of frame pairs of one shape and metric set. At admission its frames are
   made resident on the device (host frames are copied into memory counted against the context's
   HBM budget; device frames are used in place and must stay valid until the request completes);
   a request whose frames do not fit waits until completed requests free memory, and a request
   larger than the whole budget is rejected at submission. Worker threads, each with its own batched
   engine and stream, repeatedly take the next pending pairs of all admitted requests (in arrival
   order, up to max_batch_pairs / max_batch_pixels per launch sequence), so requests that arrive
   while others are on the GPU join the next batch and their work overlaps on the device. A pair's
   result does not depend on the batch it ran in. */

typedef struct qmiv_request
{
  int32_t           width, height, bitdepth, chroma_format;
  int32_t           search_range;   /* 1..5 */
  uint32_t          metric_mask;
  int32_t           num_pairs;
  const qmiv_frame* in0;            /* [num_pairs] */
  const qmiv_frame* in1;            /* [num_pairs] */
} qmiv_request;

typedef struct qmiv_request_stats
{
  double  submit_ms, admit_ms, done_ms;  /* since the server's creation (steady clock) */
  double  latency_ms;                    /* done - submit */
  int32_t batches;                       /* launch sequences the request's pairs ran in */
  /* sequence means over the request's pairs, as the reference's per-sequence averages:
     compensated sum in frame order / number of frames (apps/QMIV/src/xMetricQMIV.cpp:98-102) */
  double  mean_psnr_pic, mean_wspsnr_pic, mean_ivpsnr, mean_ssim_pic, mean_msssim_pic, mean_ivssim, mean_ivmsssim;
} qmiv_request_stats;

/* workers: engines running concurrently (1..4). params as for qmiv_batch_create. */
QMIV_API qmiv_status qmiv_server_create(qmiv_ctx ctx, const qmiv_params* params, int32_t max_batch_pairs,
                               int64_t max_batch_pixels, int32_t workers, qmiv_server* out_server);
/* Waits for every admitted and queued request, then stops the workers. */
QMIV_API qmiv_status qmiv_server_destroy(qmiv_server server);
QMIV_API qmiv_status qmiv_server_submit(qmiv_server server, const qmiv_request* request, uint64_t* ticket);
/* Waits up to timeout_ms (< 0: no limit) for a request; results: [num_pairs] or null; stats may be
   null. A ticket is released by a successful wait. QMIV_ERR_TIMEOUT leaves it pending. */
QMIV_API qmiv_status qmiv_server_wait(qmiv_server server, uint64_t ticket, int32_t timeout_ms, qmiv_result* results,
                             qmiv_request_stats* stats);
/* Latency percentiles (nearest rank) of the requests completed since the last reset (or creation), and
   pairs completed per second from the reset to the last completion. */
QMIV_API qmiv_status qmiv_server_stats(qmiv_server server, double* p50_ms, double* p99_ms, double* pairs_per_s,
                              int64_t* completed_requests, int32_t reset);

#ifdef __cplusplus
}
#endif
#endif /* QMIV_GPU_H */
