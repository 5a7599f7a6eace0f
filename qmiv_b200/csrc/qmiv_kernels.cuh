// Kernel argument blocks and host-side launch wrappers of the QMIV metric kernels.
#pragma once
#include "qmiv_device.cuh"

namespace qmiv {

// ---------------------------------------------------------------------------------------------
// prepass: per raw row of every plane, SD (In1 - In0) and SSD, plus the largest sample per frame
// ---------------------------------------------------------------------------------------------
struct PrepassArgs
{
  Img       in0, in1;
  int32_t   rows[3];       // raw rows per plane
  int32_t   cols[3];       // raw samples per row per plane
  uint32_t  clip;          // conceal: samples above are clipped (65535 = no clipping)
  int64_t*  row_sd;        // [rows[0] + rows[1] + rows[2]]
  uint64_t* row_ssd;       // same indexing
  PairOut*  out;           // max_sample (atomicMax)
};

// ---------------------------------------------------------------------------------------------
// reduce: totals, GCD, path flags
// ---------------------------------------------------------------------------------------------
struct ReduceArgs
{
  int32_t         rows[3];
  int32_t         mult[3];     // 4:4:4 multiplicity of a raw chroma sample (1 << (sx + sy))
  int64_t         area;
  int32_t         maxv;
  int32_t         maxdiff[4];  // round(unc * Max) per component, computed on the host in float
  int32_t         need_gcd;
  int32_t         gcd_override_on;  // use gcd_override instead of the computed GCD
  int32_t         gcd_override[4];
  int32_t         fp32_ok;     // fp32 exact-key CPS path is valid for in-range samples
  int32_t         clip_on;     // conceal active
  const int64_t*  row_sd;
  const uint64_t* row_ssd;
  PairOut*        out;
};

// ---------------------------------------------------------------------------------------------
// CPS search, both directions in one pass
// ---------------------------------------------------------------------------------------------
struct CpsArgs
{
  Img            in0, in1;
  int32_t        W, H;
  int32_t        maxv;
  uint32_t       clip;
  int32_t        wi[3];        // search weights
  float          wf[3];
  const PairOut* gcd_src;      // gcd + flags
  uint32_t*      rows;         // [2][H][3], zeroed, 32-bit wrap-around sums
  void*          scp0;         // In0 resampled (T2R search result), planar 3 x W*H, may be null
  void*          scp1;         // In1 resampled (R2T search result)
  // SSIM moments of (test picture, its SCP) per direction, for IV-SSIM without storing the SCP:
  // mom[0] = (In0, SCP1) (T2R), mom[1] = (In1, SCP0) (R2T); null to skip
  Moments        mom[2];
};

// ---------------------------------------------------------------------------------------------
// block SSIM
// ---------------------------------------------------------------------------------------------
// moments of an image pair (+ fused 2x2 downsampling of both inputs for the next MS-SSIM scale)
struct SsimMomArgs
{
  Img      a, b;               // a = "Tst" picture, b = "Ref" picture of xSSIM::xCalcPicSSIM
  int32_t  W, H;
  uint32_t clip;
  Moments  mom;
  MutImg   down_a, down_b;     // outputs ((W>>1) x (H>>1), 4:4:4) or null planes
};

// windows from moments, ordered row sums (xSSIM.cpp:353-369), for up to 6 (pair, component) jobs
struct SsimPoolJob
{
  double          C1, C2;      // (0.01 Max)^2, (0.03 Max)^2 of the pair's bit depth
  const uint32_t* mom;         // the five moment planes of one component
  size_t          plane;       // elements between moment planes
  int32_t         pitch;
  int32_t         nx, ny;      // windows per row / column
  int32_t         calc_l;
  int32_t         wide;        // window sums can exceed 32 bits (bit depth > 12)
  int32_t         pad_;
  double*         row_sum;     // [ny]
  double*         win;         // scratch window values [ceil(ny / 32)][nx][32] (pool_win_elems)
};

struct SsimPoolArgs
{
  int32_t     njobs;
  SsimPoolJob job[9];
};

// ---------------------------------------------------------------------------------------------
// SSIM under any structural similarity option (qmiv_ssim_gen.cu): window values of up to 9
// (picture pair, component) jobs into their band-transposed scratch, then k_ssim_rows
// ---------------------------------------------------------------------------------------------
struct SsimGenJob
{
  Img      a, b;       // a = "Tst", b = "Ref" (xSSIM::xCalcPicSSIM argument order)
  int32_t  comp;
  int32_t  W, H;       // picture size in 4:4:4 samples
  int32_t  x0, y0;     // input position of the first window's top-left sample
  int32_t  nx, ny;     // windows per row / column
  int32_t  calc_l;
  uint32_t clip;       // conceal: samples above are clipped (65535 = no clipping)
  int32_t  esz;        // bytes per sample of a and b
  double   C1, C2;
  double*  win;        // [ceil(ny / 32)][nx][32] (pool_win_elems)
};

constexpr int kGenMaxJobs = 9;
struct SsimGenArgs
{
  int32_t    njobs;
  int32_t    S, border, coef;   // stride, QMIV_BRD_*, offset of the window's coefficients (set by the launcher)
  double     inv;               // scale of the integer sums: 2^-18, 1 / 121 or 1 / N^2 (set by the launcher)
  int32_t    tw, th, cw;        // tile width / height in samples, columns per phase (set by the launcher)
  int32_t    wr;                // window rows per CTA of the row-walking form (set by the launcher)
  SsimGenJob job[kGenMaxJobs];
};

// ---------------------------------------------------------------------------------------------
// finalize: every serial KBNS chain of one frame pair, one thread per chain
// ---------------------------------------------------------------------------------------------
struct SsimSlot
{
  const double* row_sum;       // [3][ny]
  int32_t       nx, ny;
  int32_t       use_ws;        // ERP row weights w[ws_base + ws_step j] (xIVSSIM.cpp:148-165)
  int32_t       ws_base, ws_step;
};

enum { kChainWsPsnr = 0, kChainIvPsnr = 1, kChainSsim = 2 };
struct FinChain
{
  int32_t kind;  // kChain*
  int32_t a, b;  // component / direction / slot
};

struct FinalizeArgs
{
  int32_t         H;
  int32_t         rows[3];
  int32_t         sy[3], mult_row[3];   // 4:4:4 row y of plane c = raw row (y >> sy) times mult_row
  const uint64_t* row_ssd;              // prepass rows
  const double*   ws;                   // [H] equirectangular weights or null
  int32_t         do_wspsnr;
  const uint32_t* cps_rows;             // [2][H][3] or null
  int32_t         nslots;
  SsimSlot        slot[kMaxSsimSlots];
  int32_t         nchains;              // filled by launch_finalize
  FinChain        chain[3 + 6 + 3 * kMaxSsimSlots];
  PairOut*        out;
};

// one (pair, chain) CTA of the multi-pair finalize; chain == nchains of the pair is its exact CPS sums
struct FinJob
{
  int32_t pair, chain;
};
constexpr size_t kFinalizeMaxSmem = 200 * 1024;

// launch wrappers (return cudaError_t of the launch)
template <typename T> cudaError_t launch_prepass(const PrepassArgs& a, cudaStream_t s);
cudaError_t launch_reduce(const ReduceArgs& a, cudaStream_t s);
template <typename T> cudaError_t launch_cps(const CpsArgs& a, int R, cudaStream_t s);
template <typename T> cudaError_t launch_ssim_moments(const SsimMomArgs& a, cudaStream_t s);
cudaError_t launch_ssim_pool(const SsimPoolArgs& a, cudaStream_t s);
cudaError_t launch_ssim_rows(const SsimPoolArgs& a, cudaStream_t s);   // row sums of ready window values
// SSIM windows of one option set for up to kGenMaxJobs jobs: mode QMIV_SSM_*, window N, stride S,
// border QMIV_BRD_* (regular modes)
cudaError_t launch_ssim_gen(SsimGenArgs& a, int mode, int N, int S, int border, cudaStream_t s);
template <typename T>
cudaError_t launch_downsample2(const Img& a, const Img& b, const MutImg& da, const MutImg& db, int dw, int dh, uint32_t clip,
                               cudaStream_t s);
cudaError_t launch_finalize(const FinalizeArgs& a, cudaStream_t s);
int         finalize_plan(FinalizeArgs& a);          // fills a.chain / a.nchains, returns the CTA count
size_t      finalize_smem(const FinalizeArgs& a);

// multi-pair forms: argument blocks in device memory, one launch for every pair of a batch
template <typename T> cudaError_t launch_prepass_multi(const PrepassArgs* d_jobs, int njobs, int max_rows, cudaStream_t s);
cudaError_t launch_reduce_multi(const ReduceArgs* d_jobs, int njobs, cudaStream_t s);
template <typename T>
cudaError_t launch_ssim_moments_multi(const SsimMomArgs* d_jobs, int njobs, int max_nbx, int max_nby, cudaStream_t s);
cudaError_t launch_ssim_pool_multi(const SsimPoolJob* d_jobs, int njobs, int max_nx, int max_ny, cudaStream_t s);
size_t      pool_win_elems(int nx, int ny);   // doubles of SsimPoolJob::win
// 16-byte alignment of the moment rows and the scratch, which the pooling kernels copy with cp.async
bool        pool_job_aligned(const SsimPoolJob& J);
cudaError_t launch_finalize_multi(const FinalizeArgs* d_pairs, const FinJob* d_jobs, int njobs, size_t smem, cudaStream_t s);

// CPS work-list form: one 64-byte aligned descriptor (tensor maps + tile geometry) per frame pair,
// pairs grouped by (search range, sample size, tile height); pair p owns work-list tiles
// [prefix[p], prefix[p + 1]).
struct CpsPairPlan
{
  int32_t  ntiles;
  uint32_t raw_bytes;   // raw-box region of the pair
  size_t   smem;        // dynamic shared memory of the pair alone
};
size_t      cps_desc_bytes();
int         cps_pick_wy(int R, int esz, int sx, int sy);   // warps per tile column: 8 (128x32) or 4 (128x16), 0 = none
bool        cps_tile_fits(int R, int wy, int esz, int sx, int sy);
cudaError_t cps_describe(void* desc, const CpsArgs& a, int R, int esz, int wy, CpsPairPlan* plan);
cudaError_t launch_cps_multi(const void* d_descs, const int32_t* d_prefix, int npairs, int ntiles, int R, int wy,
                             int esz, uint32_t raw_cap, size_t smem, cudaStream_t s);

// Exactness check of the fp32 key path for a given bit depth, weights and GCD clip range.
bool cps_fp32_exact(int32_t maxv, const int32_t w[3], const int32_t maxdiff[3]);

}  // namespace qmiv
