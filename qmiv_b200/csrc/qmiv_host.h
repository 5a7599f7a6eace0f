// Host-side internals of the QMIV B200 library (not part of the public ABI).
#pragma once
#include "qmiv_gpu.h"
#include "qmiv_kernels.cuh"

#include <cstdint>
#include <mutex>
#include <string>
#include <memory>
#include <map>
#include <vector>

struct qmiv_ctx_s
{
  int32_t    device = 0;
  uint64_t   budget = 0;  // 0 = unlimited
  uint64_t   used   = 0;
  std::mutex mu;
  bool reserve(size_t n);
  void unreserve(size_t n);
  // per-stage timing (QMIV_STAGE_*)
  bool     profiling = false;
  double   stage_ms[QMIV_NUM_STAGES] = {};
  uint64_t stage_n[QMIV_NUM_STAGES] = {};
  void add_stage(int stage, double ms)
  {
    std::lock_guard<std::mutex> lk(mu);
    stage_ms[stage] += ms;
    stage_n[stage] += 1;
  }
};

namespace qmiv {

extern thread_local std::string g_last_error;
qmiv_status fail(qmiv_status st, const std::string& msg);
qmiv_status cuda_fail(cudaError_t e, const char* what);

#define QMIV_CUDA(call)                                           \
  do {                                                            \
    const cudaError_t qmiv_e_ = (call);                           \
    if(qmiv_e_ != cudaSuccess) { return cuda_fail(qmiv_e_, #call); } \
  } while(0)

#define QMIV_TRY(call)                                            \
  do {                                                            \
    const qmiv_status qmiv_s_ = (call);                           \
    if(qmiv_s_ != QMIV_OK) { return qmiv_s_; }                    \
  } while(0)

// Device allocation counted against the owning context's HBM budget.
struct DevMem
{
  void*       p     = nullptr;
  size_t      bytes = 0;
  qmiv_ctx_s* ctx   = nullptr;
  DevMem() = default;
  DevMem(const DevMem&) = delete;
  DevMem& operator=(const DevMem&) = delete;
  ~DevMem() { release(); }
  qmiv_status alloc(qmiv_ctx_s* c, size_t n);
  qmiv_status ensure(qmiv_ctx_s* c, size_t n);
  void        release();
  template <typename T> T* as() const { return static_cast<T*>(p); }
};

// SSIM result slots of PairOut::ssim
constexpr int kSlotSsim = 0, kSlotIvT2R = 1, kSlotIvR2T = 2, kSlotMs = 3, kSlotIvmsT2R = 8, kSlotIvmsR2T = 13;

struct FinishInfo
{
  int32_t  W, H, bitdepth;
  uint32_t mask;
  int32_t  erp;
  double   ws_corr;
  int32_t  cwa[4];
  int32_t  num_scales;
};

double  psnr_from_ssd(double ssd, int64_t area, int32_t bitdepth);
int32_t num_scales(int32_t W, int32_t H);
int32_t round_f32_half_away(float f);
// equirectangular row weights w[0..H) and the WS-PSNR correction H / sum(w)
void    ws_weights(int32_t H, int32_t lat_range, double* w, double& correction);
void    ws_weights(int32_t H, int32_t lat_range, std::vector<double>& w, double& correction);
void    finish_result(const PairOut& o, const FinishInfo& fi, qmiv_result* r);
// Status of a finished pair from its device flags: a CPS tile load that did not complete, then
// invalid samples under QMIV_PEL_STOP.
qmiv_status pair_status(const PairOut& o, int32_t invalid_pel_action);

// Geometry of one frame-pair shape.
struct Shape
{
  int32_t W = 0, H = 0, bitdepth = 0, chroma_format = 0;
  int32_t sx = 0, sy = 0;        // chroma subsampling shifts
  int32_t cw = 0, ch = 0;        // chroma plane size
  size_t  esz = 0;               // bytes per sample (1 or 2)
  int32_t maxv = 0;
  qmiv_status init(int32_t W, int32_t H, int32_t bitdepth, int32_t chroma_format);
  size_t  plane_cols(int c) const { return c == 0 ? (size_t)W : (size_t)cw; }
  size_t  plane_rows(int c) const { return c == 0 ? (size_t)H : (size_t)ch; }
  size_t  frame_bytes() const { return esz * ((size_t)W * H + 2 * (size_t)cw * ch); }
  // device copy of a host frame: rows padded to 16 bytes and planes to 256 bytes, so that TMA can
  // load the planes directly
  size_t  staged_pitch(int c) const { return (plane_cols(c) * esz + 15) & ~(size_t)15; }
  size_t  staged_plane_bytes(int c) const { return (staged_pitch(c) * plane_rows(c) + 255) & ~(size_t)255; }
  size_t  staged_frame_bytes() const { return staged_plane_bytes(0) + staged_plane_bytes(1) + staged_plane_bytes(2); }
};

qmiv_status validate_params(const qmiv_params& p);

// The device view of a frame of shape S: device planes are used in place, host planes are copied into
// `staging` (S.staged_frame_bytes(), rows padded to 16 bytes) on stream s.
qmiv_status resolve_frame(const Shape& S, const qmiv_frame* f, char* staging, Img& out, cudaStream_t s);

// Structural similarity options of a parameter set (xSSIM::setStructSimParams, xSSIM.cpp:86-113).
constexpr uint32_t kSsimFamily = QMIV_SSIM | QMIV_MSSSIM | QMIV_IVSSIM | QMIV_IVMSSSIM;
inline bool    ssim_regular(int32_t mode) { return mode >= QMIV_SSM_REGULAR_GAUSSIAN_FLT && mode <= QMIV_SSM_REGULAR_AVERAGED; }
// BlockAveraged 8x8 windows at stride 4: the moment-based path (qmiv_ssim.cu)
inline bool    ssim_is_default(const qmiv_params& p) { return p.ssim_mode == QMIV_SSM_BLOCK_AVERAGED && p.ssim_window == 8 && p.ssim_stride == 4; }
inline int32_t ssim_window_size(const qmiv_params& p) { return ssim_regular(p.ssim_mode) ? 11 : p.ssim_window; }
// Windows along a picture line of length len (xSSIM::xInitLoopRanges, xSSIM.cpp:161-196, counts
// :381-404) and the line position of the first window's first input sample.
void ssim_line(const qmiv_params& p, int32_t len, int32_t& first_sample, int32_t& count);

// Known metric bits, and the SSIM family only where it is exact: up to 14 bits for the default
// windows (exact 32-bit sub-block moments: 16 * (2^14 - 1)^2 < 2^32) and for every option whose
// reference arithmetic squares samples in 32 bits; plain SSIM up to 16 bits under the regular Gaussian
// windows, whose reference sums are double or 64-bit (xStructSimSTD.cpp:19-154).
qmiv_status check_metrics(const Shape& S, uint32_t mask, const qmiv_params& p);

// The device pipeline of one frame pair of a fixed shape, with its scratch buffers.
// Per-stage device timing: begin and end events on the launching stream, read once the stream has
// synchronised and added to the context's totals (qmiv_ctx_stage_times). begin returns -1 (and end then
// does nothing) while the context does not profile.
class StageClock
{
public:
  int  begin(qmiv_ctx_s* ctx, cudaStream_t s);
  void end(cudaStream_t s, int stage, int tok);
  void harvest(qmiv_ctx_s* ctx);
  ~StageClock();

private:
  std::vector<cudaEvent_t> pool_;
  size_t used_ = 0;
  std::vector<std::pair<int, int>> pending_;     // (stage, index of the begin event)
};

class PairPipeline
{
public:
  qmiv_status configure(qmiv_ctx_s* ctx, const Shape& shape, const qmiv_params& prm, int32_t search_range);
  // Reserve every buffer the metrics in `mask` need (lazily grows).
  qmiv_status prepare(uint32_t mask, bool want_scp, bool host_frames);
  // Resolve a frame: device frames are used in place, host frames are copied to staging.
  qmiv_status resolve(const qmiv_frame* f, int which, Img& out, cudaStream_t s);
  // Enqueue the full pipeline; results land in the pinned host PairOut after the stream syncs.
  qmiv_status enqueue(const Img& in0, const Img& in1, uint32_t mask, bool want_scp, bool want_gcd, cudaStream_t s);
  const PairOut& host_out() const { return *h_out; }
  FinishInfo finish_info(uint32_t mask) const;
  // SCP planes (T samples, planar 3 x W*H) of the last run, or null
  const void* scp(int which) const;
  const uint32_t* cps_rows() const { return cps_rows_.as<uint32_t>(); }
  const double* ws_device() const { return ws_.as<double>(); }   // ERP row weights, after prepare()
  double ws_corr() const { return ws_corr_; }
  const int32_t* maxdiff() const { return maxdiff_; }
  const Shape& shape() const { return shape_; }
  int32_t search_range() const { return R_; }
  void set_gcd_override(const int32_t* g)
  {
    gcd_override_on_ = g != nullptr;
    for(int c = 0; c < 4; c++) { gcd_override_[c] = g ? g[c] : 0; }
  }
  bool get_gcd_override(int32_t g[4]) const
  {
    for(int c = 0; c < 4; c++) { g[c] = gcd_override_[c]; }
    return gcd_override_on_;
  }
  // stage timing: events recorded on the launching stream, harvested after the stream synced
  int  prof_begin(cudaStream_t s);
  void prof_end(cudaStream_t s, int stage, int token);
  void harvest_profile();
  ~PairPipeline();

private:
  template <typename T> qmiv_status enqueue_t(const Img& in0, const Img& in1, uint32_t mask, bool want_scp, bool want_gcd, cudaStream_t s);
  // SSIM family under a non-default structural similarity option (qmiv_ssim_gen.cu windows on the
  // pictures and their SCPs)
  template <typename T>
  qmiv_status enqueue_ssim_gen(const Img& in0, const Img& in1, const Img& scp0, const Img& scp1, uint32_t mask, uint32_t clip,
                               FinalizeArgs& fa, cudaStream_t s);
  bool need_scp_for(uint32_t mask, bool want_scp) const
  {
    return want_scp || (mask & QMIV_IVMSSSIM) || (gen_ && (mask & QMIV_IVSSIM));
  }

  qmiv_ctx_s*  ctx_ = nullptr;
  Shape        shape_;
  qmiv_params  prm_{};
  int32_t      R_ = 2;
  int32_t      maxdiff_[4] = { 0, 0, 0, 0 };
  bool         fp32_ok_ = true;
  int32_t      ns_ = 0;
  int32_t      nx_[5] = {}, ny_[5] = {}, nxp_ = 0;
  bool         gen_ = false;                       // non-default structural similarity option
  int32_t      gnx_[5] = {}, gny_[5] = {};         // its windows per row / column at each MS-SSIM scale
  int32_t      gfirst_ = 0, gws_base_ = 0;         // first window's first input sample; ERP weight of window row 0
  std::vector<double> ws_host_;
  double       ws_corr_ = 1.0;
  double       C1_ = 0, C2_ = 0;

  // SSIM moments (qmiv_device.cuh, Moments) of one pair at scale s, in slot k of mom_
  Moments mom_at(int slot, int scale) const
  {
    Moments m{};
    m.nbx = ((shape_.W >> scale) + 3) / 4;
    m.nby = ((shape_.H >> scale) + 3) / 4;
    m.pitch = (m.nbx + 7) & ~7;
    m.p = mom_.as<uint32_t>() + (size_t)slot * mom_slot_elems();
    return m;
  }
  size_t mom_slot_elems() const
  {
    const size_t nbx = ((size_t)shape_.W + 3) / 4, nby = ((size_t)shape_.H + 3) / 4;
    return 3 * 5 * nby * ((nbx + 7) & ~(size_t)7);
  }

  DevMem row_sd_, row_ssd_, cps_rows_, out_, ws_, scp_, pyr_, mom_, rowsum_, win_, staging_;
  PairOut* h_out = nullptr;
  bool ws_uploaded_ = false;
  bool gcd_override_on_ = false;
  int32_t gcd_override_[4] = { 0, 0, 0, 0 };
  StageClock clock_;
};

// Colour-space conversion of one calc (qmiv_colour.cu): the converted 4:4:4 planes of the current pair
// and the 4:4:4 pipeline that computes the metrics on them.
class ColourStage
{
public:
  qmiv_status configure(int32_t cs_in, int32_t cs_metric);
  // Converts both frames into 4:4:4 planes (out0 / out1 describe them) on stream s.
  qmiv_status convert(qmiv_ctx_s* ctx, const Shape& S, const qmiv_params& prm, const Img& in0, const Img& in1, Img& out0, Img& out1,
                      cudaStream_t s);
  // bit0 / bit1: frame 0 / 1 held samples above maxv (valid after the stream synced)
  int32_t invalid_flags(int32_t maxv) const;
  ~ColourStage();

  bool         active = false;
  PairPipeline pipe444;

private:
  int32_t  mode = 0, space = 0, perm[3] = { 0, 1, 2 };
  bool     configured_ = false;
  Shape    shape444_;
  DevMem   planes_, max_;
  uint32_t* h_max_ = nullptr;
};

// Mask mode of one calc (qmiv_masked.cu): its scratch and the synchronous run.
// Mask mode for many frame pairs of uneven shape (qmiv_batch_compute_masked): every stage one launch
// per group of pairs with the same sample sizes, search range and search form.
class MaskedBatch
{
public:
  qmiv_status run(qmiv_ctx_s* ctx, const qmiv_params& prm, cudaStream_t s, const qmiv_pair_desc* pairs,
                  const qmiv_frame* masks, const int32_t* mask_bitdepths, int32_t n, qmiv_result* out,
                  int32_t* num_non_masked);
  ~MaskedBatch();

private:
  DevMem arena_;
  void*  h_ = nullptr;        // pinned block of the results
  size_t h_bytes_ = 0;
  StageClock clock_;
  std::map<std::pair<int32_t, int32_t>, DevMem> ws_dev_;   // ERP row weights by (height, latitude range)
};

class MaskedPipeline
{
public:
  qmiv_status run(qmiv_calc_s* calc, const qmiv_frame* in0, const qmiv_frame* in1, const qmiv_frame* mask,
                  int32_t mask_bitdepth, uint32_t metrics, qmiv_result* out, int32_t* num_non_masked);
  ~MaskedPipeline();

private:
  DevMem out_, rows_, stage_;
  void*  h_out_ = nullptr;
};

}  // namespace qmiv

struct qmiv_calc_s
{
  qmiv_ctx_s*          ctx = nullptr;
  qmiv::Shape          shape;
  qmiv_params          prm{};
  qmiv::PairPipeline   pipe;
  cudaStream_t         stream = nullptr;
  cudaEvent_t          done = nullptr;
  bool                 pending = false;
  uint32_t             pending_mask = 0;
  bool                 has_last = false;
  std::unique_ptr<qmiv::MaskedPipeline> masked;   // created by the first masked call
  std::unique_ptr<qmiv::ColourStage>    colour;   // set by qmiv_calc_set_color_space
  bool                 pending_colour = false;   // the submission in flight went through the colour stage
};
