// Plain form: one frame pair per call (qmiv_calc_* entry points) on top of PairPipeline, the
// device pipeline of one frame pair that the batched form reuses.
#include "qmiv_host.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>

namespace qmiv {

// ---------------------------------------------------------------------------------------------
// shape / parameter validation
// ---------------------------------------------------------------------------------------------
qmiv_status Shape::init(int32_t W_, int32_t H_, int32_t bd, int32_t cf)
{
  if(W_ <= 0 || H_ <= 0) { return fail(QMIV_ERR_INVALID_ARG, "picture size must be positive"); }
  if(bd < 1 || bd > 16) { return fail(QMIV_ERR_INVALID_ARG, "bit depth must be in 1..16"); }
  if(cf != 420 && cf != 422 && cf != 444) { return fail(QMIV_ERR_UNSUPPORTED, "chroma format must be 420, 422 or 444"); }
  W = W_; H = H_; bitdepth = bd; chroma_format = cf;
  sx = cf == 444 ? 0 : 1;
  sy = cf == 420 ? 1 : 0;
  if((sx && (W & 1)) || (sy && (H & 1))) { return fail(QMIV_ERR_INVALID_ARG, "subsampled chroma needs even picture dimensions"); }
  cw = W >> sx; ch = H >> sy;
  esz = bd <= 8 ? 1 : 2;
  maxv = (1 << bd) - 1;
  return QMIV_OK;
}

qmiv_status check_metrics(const Shape& S, uint32_t mask, const qmiv_params& p)
{
  if((mask & ~(uint32_t)QMIV_ALL) != 0) { return fail(QMIV_ERR_INVALID_ARG, "unknown metric bits"); }
  if((mask & (QMIV_SSIM | QMIV_MSSSIM | QMIV_IVSSIM | QMIV_IVMSSSIM)) && S.bitdepth > 14)
  {
    // plain SSIM only: the reference's SIMD 2x2 downsampling (MS-SSIM) adds sample pairs in signed 16-bit
    // lanes (xPixelOpsSSE.cpp:186-189), and the IV metrics' search errors overflow int32, above 14 bits
    const bool wide_ok = (p.ssim_mode == QMIV_SSM_REGULAR_GAUSSIAN_FLT || p.ssim_mode == QMIV_SSM_REGULAR_GAUSSIAN_INT) &&
                         !(mask & (QMIV_MSSSIM | QMIV_IVSSIM | QMIV_IVMSSSIM));
    if(!wide_ok)
    {
      return fail(QMIV_ERR_UNSUPPORTED, "SSIM metrics at a bit depth above 14 need the RegularGaussianFlt or RegularGaussianInt "
                                        "option (plain SSIM only)");
    }
  }
  return QMIV_OK;
}

qmiv_status validate_params(const qmiv_params& p)
{
  if(p.search_range < 1 || p.search_range > 5) { return fail(QMIV_ERR_UNSUPPORTED, "search range must be 1..5"); }
  if(p.cws[3] != 0) { return fail(QMIV_ERR_UNSUPPORTED, "the fourth search weight must be 0"); }
  for(int c = 0; c < 3; c++) { if(p.cws[c] < 0 || p.cwa[c] < 0) { return fail(QMIV_ERR_INVALID_ARG, "weights must be >= 0"); } }
  if(p.cwa[0] + p.cwa[1] + p.cwa[2] + p.cwa[3] <= 0) { return fail(QMIV_ERR_INVALID_ARG, "averaging weights sum to 0"); }
  // structural similarity options: the app's checks (xAppQMIV.cpp:325-332) and the sets the reference's
  // windows evaluate (xStructSimSTD.cpp:399-403 returns NaN for Gaussian 32x32 blocks)
  if(p.ssim_mode < QMIV_SSM_REGULAR_GAUSSIAN_FLT || p.ssim_mode > QMIV_SSM_BLOCK_AVERAGED) { return fail(QMIV_ERR_INVALID_ARG, "unknown SSIM mode"); }
  if(p.ssim_border < QMIV_BRD_NONE || p.ssim_border > QMIV_BRD_ZERO) { return fail(QMIV_ERR_INVALID_ARG, "unknown SSIM border mode"); }
  if(ssim_regular(p.ssim_mode) && p.ssim_window != 11) { return fail(QMIV_ERR_INVALID_ARG, "regular SSIM modes use 11x11 windows"); }
  if(p.ssim_mode == QMIV_SSM_BLOCK_AVERAGED && p.ssim_window != 8 && p.ssim_window != 16 && p.ssim_window != 32)
  {
    return fail(QMIV_ERR_UNSUPPORTED, "BlockAveraged SSIM windows are 8, 16 or 32");
  }
  if(p.ssim_mode == QMIV_SSM_BLOCK_GAUSSIAN_INT && p.ssim_window != 8 && p.ssim_window != 16)
  {
    return fail(QMIV_ERR_UNSUPPORTED, "BlockGaussianInt SSIM windows are 8 or 16");
  }
  if(p.ssim_stride < 1 || p.ssim_stride > ssim_window_size(p)) { return fail(QMIV_ERR_INVALID_ARG, "SSIM stride must be in 1..window"); }
  // the averaged 11x11 window squares samples in 32-bit lanes (xStructSimSTD.cpp:167-169; signed 16-bit
  // products in its AVX form), which the constant margin of 65535 overflows
  if(p.ssim_mode == QMIV_SSM_REGULAR_AVERAGED && p.ssim_border == QMIV_BRD_CONSTANT)
  {
    return fail(QMIV_ERR_UNSUPPORTED, "RegularAveraged SSIM with the Constant border overflows in the reference");
  }
  if(p.erp && (p.lat_range_deg <= 0 || p.lat_range_deg > 180)) { return fail(QMIV_ERR_INVALID_ARG, "lat range must be in 1..180"); }
  if(p.invalid_pel_action < QMIV_PEL_SKIP || p.invalid_pel_action > QMIV_PEL_CNCL) { return fail(QMIV_ERR_INVALID_ARG, "bad invalid pixel action"); }
  return QMIV_OK;
}

void ssim_line(const qmiv_params& p, int32_t len, int32_t& first_sample, int32_t& count)
{
  const int32_t S = p.ssim_stride, N = ssim_window_size(p);
  if(ssim_regular(p.ssim_mode))
  {
    const bool margin = p.ssim_border != QMIV_BRD_NONE;
    const int32_t beg = margin ? 0 : 5, end = margin ? len : len - 5;   // c_FilterRange = 5
    count = end > beg ? (end - beg + S - 1) / S : 0;
    first_sample = beg - 5;
  }
  else
  {
    count = len >= N ? (len - N) / S + 1 : 0;
    first_sample = 0;
  }
}

// ---------------------------------------------------------------------------------------------
// PairPipeline
// ---------------------------------------------------------------------------------------------
PairPipeline::~PairPipeline()
{
  if(h_out) { cudaFreeHost(h_out); h_out = nullptr; }
}

int StageClock::begin(qmiv_ctx_s* ctx, cudaStream_t s)
{
  if(!ctx || !ctx->profiling) { return -1; }
  while(pool_.size() < used_ + 2)
  {
    cudaEvent_t e;
    if(cudaEventCreate(&e) != cudaSuccess) { return -1; }
    pool_.push_back(e);
  }
  const int tok = (int)used_;
  used_ += 2;
  cudaEventRecord(pool_[tok], s);
  return tok;
}

void StageClock::end(cudaStream_t s, int stage, int tok)
{
  if(tok < 0) { return; }
  cudaEventRecord(pool_[tok + 1], s);
  pending_.emplace_back(stage, tok);
}

void StageClock::harvest(qmiv_ctx_s* ctx)
{
  for(const auto& p : pending_)
  {
    float ms = 0.f;
    if(ctx && cudaEventElapsedTime(&ms, pool_[p.second], pool_[p.second + 1]) == cudaSuccess) { ctx->add_stage(p.first, ms); }
  }
  pending_.clear();
  used_ = 0;
}

StageClock::~StageClock()
{
  for(cudaEvent_t e : pool_) { cudaEventDestroy(e); }
}

int PairPipeline::prof_begin(cudaStream_t s) { return clock_.begin(ctx_, s); }
void PairPipeline::prof_end(cudaStream_t s, int stage, int tok) { clock_.end(s, stage, tok); }
void PairPipeline::harvest_profile() { clock_.harvest(ctx_); }

qmiv_status PairPipeline::configure(qmiv_ctx_s* ctx, const Shape& shape, const qmiv_params& prm, int32_t search_range)
{
  ctx_ = ctx; shape_ = shape; prm_ = prm; R_ = search_range;
  for(int c = 0; c < 4; c++) { maxdiff_[c] = round_f32_half_away(prm.unc[c] * (float)shape.maxv); }  // xGlobClrDiff.cpp:76
  fp32_ok_ = cps_fp32_exact(shape.maxv, prm.cws, maxdiff_);
  ns_ = num_scales(shape.W, shape.H);
  int32_t w = shape.W, h = shape.H;
  for(int s = 0; s < 5; s++)
  {
    nx_[s] = w >= 8 ? (w - 8) / 4 + 1 : 0;   // xSSIM::xCalcNumBlocks for 8/4
    ny_[s] = h >= 8 ? (h - 8) / 4 + 1 : 0;
    w >>= 1; h >>= 1;
  }
  nxp_ = (nx_[0] + 31) & ~31;
  gen_ = !ssim_is_default(prm);
  for(int s = 0; s < 5; s++)
  {
    int32_t f = 0;
    ssim_line(prm, shape.W >> s, f, gnx_[s]);
    ssim_line(prm, shape.H >> s, gfirst_, gny_[s]);
  }
  // ERP weight of window row j: its centre row (regular) or top row + WndSize / 2 (xIVSSIM.cpp:153)
  gws_base_ = ssim_regular(prm.ssim_mode) ? gfirst_ + 5 : ssim_window_size(prm) / 2;
  const double maxd = (double)shape.maxv;  // xSSIM.cpp:165-167
  const double k1 = 0.01 * maxd, k2 = 0.03 * maxd;
  C1_ = k1 * k1; C2_ = k2 * k2;
  if(prm.erp) { ws_weights(shape.H, prm.lat_range_deg, ws_host_, ws_corr_); }
  ws_uploaded_ = false;
  if(!h_out) { QMIV_CUDA(cudaMallocHost((void**)&h_out, sizeof(PairOut))); }
  std::memset(h_out, 0, sizeof(PairOut));
  return QMIV_OK;
}

qmiv_status PairPipeline::prepare(uint32_t mask, bool want_scp, bool host_frames)
{
  const Shape& S = shape_;
  const size_t rows_total = (size_t)S.H + 2 * (size_t)S.ch;
  QMIV_TRY(row_sd_.ensure(ctx_, rows_total * sizeof(int64_t)));
  QMIV_TRY(row_ssd_.ensure(ctx_, rows_total * sizeof(uint64_t)));
  QMIV_TRY(out_.ensure(ctx_, sizeof(PairOut)));
  const bool need_scp = need_scp_for(mask, want_scp);
  const bool need_search = need_scp || (mask & (QMIV_IVPSNR | QMIV_IVSSIM));
  const bool need_ssim = mask & (QMIV_SSIM | QMIV_MSSSIM | QMIV_IVSSIM | QMIV_IVMSSSIM);
  const bool need_ms = mask & (QMIV_MSSSIM | QMIV_IVMSSSIM);
  if(need_search) { QMIV_TRY(cps_rows_.ensure(ctx_, (size_t)2 * S.H * 3 * sizeof(uint32_t))); }
  if(need_scp) { QMIV_TRY(scp_.ensure(ctx_, (size_t)2 * 3 * S.W * S.H * S.esz)); }
  if(need_ssim && !gen_)
  {
    // moment slots: 0, 1 = IV-SSIM directions (written by the search), 2 = SSIM / MS-SSIM pair,
    // 3, 4 = IV-MS-SSIM pairs
    const int slots = (mask & QMIV_IVMSSSIM) ? 5 : (mask & (QMIV_SSIM | QMIV_MSSSIM)) ? 3 : 2;
    QMIV_TRY(mom_.ensure(ctx_, (size_t)slots * mom_slot_elems() * sizeof(uint32_t)));
  }
  if(prm_.erp)
  {
    QMIV_TRY(ws_.ensure(ctx_, (size_t)S.H * sizeof(double)));
    if(!ws_uploaded_) { QMIV_CUDA(cudaMemcpy(ws_.p, ws_host_.data(), S.H * sizeof(double), cudaMemcpyHostToDevice)); ws_uploaded_ = true; }
  }
  if(need_ssim && !gen_)
  {
    if(nx_[0] < 1 || ny_[0] < 1) { return fail(QMIV_ERR_INVALID_ARG, "picture smaller than one 8x8 SSIM window"); }
    QMIV_TRY(rowsum_.ensure(ctx_, (size_t)kMaxSsimSlots * 3 * ny_[0] * sizeof(double)));
    // window values of up to 9 pool jobs (one flush) at scale 0, reused by later flushes
    QMIV_TRY(win_.ensure(ctx_, (size_t)9 * pool_win_elems(nx_[0], ny_[0]) * sizeof(double)));
  }
  if(need_ssim && gen_)
  {
    const int32_t N = ssim_window_size(prm_);
    if(S.W < N || S.H < N || gnx_[0] < 1 || gny_[0] < 1) { return fail(QMIV_ERR_INVALID_ARG, "picture smaller than one SSIM window"); }
    QMIV_TRY(rowsum_.ensure(ctx_, (size_t)kMaxSsimSlots * 3 * gny_[0] * sizeof(double)));
    QMIV_TRY(win_.ensure(ctx_, (size_t)kGenMaxJobs * pool_win_elems(gnx_[0], gny_[0]) * sizeof(double)));
  }
  if(need_ms)
  {
    if(ns_ < 1) { return fail(QMIV_ERR_INVALID_ARG, "picture too small for MS-SSIM (needs >= 32x32)"); }
    size_t lv = 0;
    for(int s = 1; s < ns_; s++) { lv += (size_t)(S.W >> s) * (S.H >> s) * 3; }
    QMIV_TRY(pyr_.ensure(ctx_, 4 * lv * S.esz));
  }
  if(host_frames) { QMIV_TRY(staging_.ensure(ctx_, 2 * S.staged_frame_bytes())); }
  return QMIV_OK;
}

qmiv_status resolve_frame(const Shape& S, const qmiv_frame* f, char* staging, Img& out, cudaStream_t s)
{
  if(!f) { return fail(QMIV_ERR_INVALID_ARG, "frame is null"); }
  size_t off = 0;
  for(int c = 0; c < 3; c++)
  {
    if(!f->plane[c]) { return fail(QMIV_ERR_INVALID_ARG, "frame plane is null"); }
    const size_t row_bytes = S.plane_cols(c) * S.esz;
    if(f->pitch[c] < (int64_t)row_bytes || (f->pitch[c] % (int64_t)S.esz) != 0) { return fail(QMIV_ERR_INVALID_ARG, "bad plane pitch"); }
    out.sx[c] = c ? (int8_t)S.sx : 0;
    out.sy[c] = c ? (int8_t)S.sy : 0;
    if(f->mem == QMIV_MEM_DEVICE)
    {
      out.p[c] = f->plane[c];
      out.pitch[c] = (int32_t)(f->pitch[c] / (int64_t)S.esz);
    }
    else if(f->mem == QMIV_MEM_HOST)
    {
      if(!staging) { return fail(QMIV_ERR_INVALID_ARG, "staging not prepared"); }
      char* dst = staging + off;
      if((size_t)f->pitch[c] == row_bytes && S.staged_pitch(c) == row_bytes)
      {
        QMIV_CUDA(cudaMemcpyAsync(dst, f->plane[c], row_bytes * S.plane_rows(c), cudaMemcpyHostToDevice, s));
      }
      else
      {
        QMIV_CUDA(cudaMemcpy2DAsync(dst, S.staged_pitch(c), f->plane[c], (size_t)f->pitch[c], row_bytes, S.plane_rows(c),
                                    cudaMemcpyHostToDevice, s));
      }
      out.p[c] = dst;
      out.pitch[c] = (int32_t)(S.staged_pitch(c) / S.esz);
      off += S.staged_plane_bytes(c);
    }
    else { return fail(QMIV_ERR_INVALID_ARG, "frame mem must be QMIV_MEM_HOST or QMIV_MEM_DEVICE"); }
  }
  return QMIV_OK;
}

qmiv_status PairPipeline::resolve(const qmiv_frame* f, int which, Img& out, cudaStream_t s)
{
  if(!f) { return fail(QMIV_ERR_INVALID_ARG, "frame is null"); }
  const int tok = f->mem == QMIV_MEM_HOST ? prof_begin(s) : -1;
  char* stage = staging_.p ? staging_.as<char>() + (size_t)which * shape_.staged_frame_bytes() : nullptr;
  QMIV_TRY(resolve_frame(shape_, f, stage, out, s));
  prof_end(s, QMIV_STAGE_H2D, tok);
  return QMIV_OK;
}

const void* PairPipeline::scp(int which) const
{
  if(!scp_.p) { return nullptr; }
  return scp_.as<char>() + (size_t)which * 3 * shape_.W * shape_.H * shape_.esz;
}

FinishInfo PairPipeline::finish_info(uint32_t mask) const
{
  FinishInfo fi{};
  fi.W = shape_.W; fi.H = shape_.H; fi.bitdepth = shape_.bitdepth; fi.mask = mask;
  fi.erp = prm_.erp; fi.ws_corr = ws_corr_;
  for(int c = 0; c < 4; c++) { fi.cwa[c] = prm_.cwa[c]; }
  fi.num_scales = ns_;
  return fi;
}

qmiv_status PairPipeline::enqueue(const Img& in0, const Img& in1, uint32_t mask, bool want_scp, bool want_gcd, cudaStream_t s)
{
  return shape_.esz == 1 ? enqueue_t<uint8_t>(in0, in1, mask, want_scp, want_gcd, s)
                         : enqueue_t<uint16_t>(in0, in1, mask, want_scp, want_gcd, s);
}

static Img img444(const void* base, int32_t W, int32_t H, size_t esz)
{
  Img im{};
  for(int c = 0; c < 3; c++)
  {
    im.p[c] = static_cast<const char*>(base) + (size_t)c * W * H * esz;
    im.pitch[c] = W; im.sx[c] = 0; im.sy[c] = 0;
  }
  return im;
}
static MutImg mut444(void* base, int32_t W, int32_t H, size_t esz)
{
  MutImg im{};
  for(int c = 0; c < 3; c++) { im.p[c] = static_cast<char*>(base) + (size_t)c * W * H * esz; im.pitch[c] = W; }
  return im;
}

template <typename T>
qmiv_status PairPipeline::enqueue_t(const Img& in0, const Img& in1, uint32_t mask, bool want_scp, bool want_gcd, cudaStream_t s)
{
  const Shape& S = shape_;
  const bool need_scp = need_scp_for(mask, want_scp);
  const bool need_search = need_scp || (mask & (QMIV_IVPSNR | QMIV_IVSSIM));
  const uint32_t clip = prm_.invalid_pel_action == QMIV_PEL_CNCL ? (uint32_t)S.maxv : 0xffffu;
  PairOut* dout = out_.as<PairOut>();

  QMIV_CUDA(cudaMemsetAsync(dout, 0, sizeof(PairOut), s));
  if(need_search) { QMIV_CUDA(cudaMemsetAsync(cps_rows_.p, 0, (size_t)2 * S.H * 3 * sizeof(uint32_t), s)); }

  // 1. prepass + reduce (GCD)
  PrepassArgs pa{};
  pa.in0 = in0; pa.in1 = in1;
  for(int c = 0; c < 3; c++) { pa.rows[c] = (int32_t)S.plane_rows(c); pa.cols[c] = (int32_t)S.plane_cols(c); }
  pa.clip = clip; pa.row_sd = row_sd_.as<int64_t>(); pa.row_ssd = row_ssd_.as<uint64_t>(); pa.out = dout;
  { const int t = prof_begin(s); QMIV_CUDA(launch_prepass<T>(pa, s)); prof_end(s, QMIV_STAGE_PREPASS, t); }

  ReduceArgs ra{};
  for(int c = 0; c < 3; c++) { ra.rows[c] = pa.rows[c]; ra.mult[c] = c ? (1 << (S.sx + S.sy)) : 1; }
  ra.area = (int64_t)S.W * S.H; ra.maxv = S.maxv;
  for(int c = 0; c < 4; c++) { ra.maxdiff[c] = maxdiff_[c]; }
  ra.need_gcd = need_search || want_gcd; ra.fp32_ok = fp32_ok_; ra.clip_on = prm_.invalid_pel_action == QMIV_PEL_CNCL;
  if(gcd_override_on_)
  {
    int32_t mag[4];
    for(int c = 0; c < 4; c++) { ra.gcd_override[c] = gcd_override_[c]; mag[c] = gcd_override_[c] < 0 ? -gcd_override_[c] : gcd_override_[c]; }
    ra.gcd_override_on = 1;
    ra.fp32_ok = cps_fp32_exact(S.maxv, prm_.cws, mag);
  }
  ra.row_sd = pa.row_sd; ra.row_ssd = pa.row_ssd; ra.out = dout;
  { const int t = prof_begin(s); QMIV_CUDA(launch_reduce(ra, s)); prof_end(s, QMIV_STAGE_REDUCE, t); }

  // 2. CPS search, both directions, SCP pictures when needed
  if(need_search)
  {
    CpsArgs ca{};
    ca.in0 = in0; ca.in1 = in1; ca.W = S.W; ca.H = S.H; ca.maxv = S.maxv; ca.clip = clip;
    for(int c = 0; c < 3; c++) { ca.wi[c] = prm_.cws[c]; ca.wf[c] = (float)prm_.cws[c]; }
    ca.gcd_src = dout; ca.rows = cps_rows_.as<uint32_t>();
    ca.scp0 = need_scp ? const_cast<void*>(scp(0)) : nullptr;
    ca.scp1 = need_scp ? const_cast<void*>(scp(1)) : nullptr;
    if((mask & QMIV_IVSSIM) && !gen_) { ca.mom[0] = mom_at(0, 0); ca.mom[1] = mom_at(1, 0); }  // (In0, SCP1), (In1, SCP0)
    const int t = prof_begin(s);
    QMIV_CUDA(launch_cps<T>(ca, R_, s));
    prof_end(s, QMIV_STAGE_CPS, t);
  }

  // 3. SSIM family
  FinalizeArgs fa{};
  fa.nslots = kMaxSsimSlots;
  if(gen_ && (mask & kSsimFamily))
  {
    const Img scp0 = need_scp ? img444(scp(0), S.W, S.H, S.esz) : Img{};
    const Img scp1 = need_scp ? img444(scp(1), S.W, S.H, S.esz) : Img{};
    QMIV_TRY(enqueue_ssim_gen<T>(in0, in1, scp0, scp1, mask, clip, fa, s));
  }
  else
  {
    double* rowsum = rowsum_.as<double>();
    // window pooling of up to three pictures pairs (x 3 components) from their moments, one launch
    SsimPoolArgs pool{};
    auto add_pool = [&](const Moments& m, int scale, int slot, int calc_l, int use_ws) {
      for(int c = 0; c < 3; c++)
      {
        SsimPoolJob& J = pool.job[pool.njobs];
        J.win = win_.as<double>() + (size_t)pool.njobs * pool_win_elems(nx_[0], ny_[0]);
        pool.njobs++;
        J.mom = m.p + (size_t)c * 5 * m.plane(); J.plane = m.plane(); J.pitch = m.pitch;
        J.C1 = C1_; J.C2 = C2_;
        J.nx = nx_[scale]; J.ny = ny_[scale]; J.calc_l = calc_l; J.wide = shape_.bitdepth > 12 ? 1 : 0;
        J.row_sum = rowsum + (size_t)slot * 3 * ny_[0] + (size_t)c * ny_[scale];  // finalize reads [c][ny_scale]
      }
      fa.slot[slot].row_sum = rowsum + (size_t)slot * 3 * ny_[0];
      fa.slot[slot].nx = nx_[scale]; fa.slot[slot].ny = ny_[scale]; fa.slot[slot].use_ws = use_ws;
      fa.slot[slot].ws_base = 4; fa.slot[slot].ws_step = 4;  // window row j covers rows 4j..4j+7 (xIVSSIM.cpp:153)
    };
    auto flush_pool = [&]() -> qmiv_status {
      if(pool.njobs == 0) { return QMIV_OK; }
      const int t = prof_begin(s);
      QMIV_CUDA(launch_ssim_pool(pool, s));
      prof_end(s, QMIV_STAGE_SSIM_ROWS, t);
      pool.njobs = 0;
      return QMIV_OK;
    };
    auto moments = [&](const Img& a, const Img& b, int W, int H, const Moments& m, const MutImg* down_a,
                       const MutImg* down_b) -> qmiv_status {
      SsimMomArgs ma{};
      ma.a = a; ma.b = b; ma.W = W; ma.H = H; ma.clip = clip; ma.mom = m;
      if(down_a) { ma.down_a = *down_a; }
      if(down_b) { ma.down_b = *down_b; }
      const int t = prof_begin(s);
      QMIV_CUDA(launch_ssim_moments<T>(ma, s));
      prof_end(s, QMIV_STAGE_SSIM_WIN, t);
      return QMIV_OK;
    };

    const Img scp0 = need_scp ? img444(scp(0), S.W, S.H, S.esz) : Img{};
    const Img scp1 = need_scp ? img444(scp(1), S.W, S.H, S.esz) : Img{};
    const int use_ws = prm_.erp ? 1 : 0;
    if(mask & QMIV_IVSSIM)  // moments written by the search: (In0, SCP1) = T2R, (In1, SCP0) = R2T (xIVSSIM.cpp:46-47)
    {
      add_pool(mom_at(0, 0), 0, kSlotIvT2R, 1, use_ws);
      add_pool(mom_at(1, 0), 0, kSlotIvR2T, 1, use_ws);
    }
    if(mask & QMIV_SSIM)  // xSSIM.h:83
    {
      QMIV_TRY(moments(in0, in1, S.W, S.H, mom_at(2, 0), nullptr, nullptr));
      if(pool.njobs + 3 > 9) { QMIV_TRY(flush_pool()); }
      add_pool(mom_at(2, 0), 0, kSlotSsim, 1, 0);
    }
    QMIV_TRY(flush_pool());
    if(mask & (QMIV_MSSSIM | QMIV_IVMSSSIM))                                                                      // xSSIM.cpp:230-256
    {
      // pyramid levels 1..ns-1 of In0, In1, SCP0, SCP1
      size_t lv = 0;
      for(int s2 = 1; s2 < ns_; s2++) { lv += (size_t)(S.W >> s2) * (S.H >> s2) * 3; }
      auto level_base = [&](int img, int scale) -> char* {
        size_t o = (size_t)img * lv;
        for(int s2 = 1; s2 < scale; s2++) { o += (size_t)(S.W >> s2) * (S.H >> s2) * 3; }
        return pyr_.as<char>() + o * S.esz;
      };
      auto level_img = [&](int img, int scale) -> Img {
        if(scale == 0) { return img == 0 ? in0 : img == 1 ? in1 : img == 2 ? scp0 : scp1; }
        return img444(level_base(img, scale), S.W >> scale, S.H >> scale, S.esz);
      };
      for(int sc = 0; sc < ns_; sc++)
      {
        const int Ws = S.W >> sc, Hs = S.H >> sc;
        const bool last = sc == ns_ - 1;
        bool written[4] = { false, false, false, false };
        auto down = [&](int img, MutImg& m) -> const MutImg* {
          if(last || written[img]) { return nullptr; }
          written[img] = true;
          m = mut444(level_base(img, sc + 1), S.W >> (sc + 1), S.H >> (sc + 1), S.esz);
          return &m;
        };
        MutImg m0, m1, m2, m3, m4, m5;
        if(mask & QMIV_MSSSIM)
        {
          const MutImg* d0 = down(0, m0); const MutImg* d1 = down(1, m1);
          QMIV_TRY(moments(level_img(0, sc), level_img(1, sc), Ws, Hs, mom_at(2, sc), d0, d1));
          add_pool(mom_at(2, sc), sc, kSlotMs + sc, last ? 1 : 0, 0);
        }
        if(mask & QMIV_IVMSSSIM)  // xIVSSIM.cpp:77-78, no ERP weighting
        {
          const MutImg* d0 = down(0, m2); const MutImg* d3 = down(3, m3);
          QMIV_TRY(moments(level_img(0, sc), level_img(3, sc), Ws, Hs, mom_at(3, sc), d0, d3));
          add_pool(mom_at(3, sc), sc, kSlotIvmsT2R + sc, last ? 1 : 0, 0);
          const MutImg* d1 = down(1, m4); const MutImg* d2 = down(2, m5);
          QMIV_TRY(moments(level_img(1, sc), level_img(2, sc), Ws, Hs, mom_at(4, sc), d1, d2));
          add_pool(mom_at(4, sc), sc, kSlotIvmsR2T + sc, last ? 1 : 0, 0);
        }
        QMIV_TRY(flush_pool());
      }
    }
  }

  // 4. pooling chains
  fa.H = S.H;
  for(int c = 0; c < 3; c++) { fa.rows[c] = (int32_t)S.plane_rows(c); fa.sy[c] = c ? S.sy : 0; fa.mult_row[c] = c ? (1 << S.sx) : 1; }
  fa.row_ssd = row_ssd_.as<uint64_t>();
  fa.ws = prm_.erp ? ws_.as<double>() : nullptr;
  fa.do_wspsnr = (mask & QMIV_WSPSNR) ? 1 : 0;
  fa.cps_rows = need_search ? cps_rows_.as<uint32_t>() : nullptr;
  fa.out = dout;
  { const int t = prof_begin(s); QMIV_CUDA(launch_finalize(fa, s)); prof_end(s, QMIV_STAGE_FINALIZE, t); }
  { const int t = prof_begin(s); QMIV_CUDA(cudaMemcpyAsync(h_out, dout, sizeof(PairOut), cudaMemcpyDeviceToHost, s)); prof_end(s, QMIV_STAGE_D2H, t); }
  return QMIV_OK;
}

// Structural similarity options other than BlockAveraged 8/4 (xSSIM.cpp:199-234 SSIM and MS-SSIM,
// xIVSSIM.cpp:31-92 IV-SSIM and IV-MS-SSIM): window values of every (picture pair, component) job
// from k_ssim_gen, row sums from k_ssim_rows, MS-SSIM levels from k_downsample2.
template <typename T>
qmiv_status PairPipeline::enqueue_ssim_gen(const Img& in0, const Img& in1, const Img& scp0, const Img& scp1, uint32_t mask,
                                           uint32_t clip, FinalizeArgs& fa, cudaStream_t s)
{
  const Shape& S = shape_;
  const int32_t N = ssim_window_size(prm_);
  double* rowsum = rowsum_.as<double>();
  const size_t wstride = pool_win_elems(gnx_[0], gny_[0]);
  SsimGenArgs ga{};
  SsimPoolArgs rows{};
  auto add = [&](const Img& a, const Img& b, int scale, int slot, int calc_l, int use_ws) {
    for(int c = 0; c < 3; c++)
    {
      SsimGenJob& J = ga.job[ga.njobs];
      J = SsimGenJob{};
      J.a = a; J.b = b; J.comp = c; J.W = S.W >> scale; J.H = S.H >> scale;
      J.x0 = gfirst_; J.y0 = gfirst_; J.nx = gnx_[scale]; J.ny = gny_[scale];
      J.calc_l = calc_l; J.clip = clip; J.esz = (int32_t)S.esz; J.C1 = C1_; J.C2 = C2_;
      J.win = win_.as<double>() + (size_t)ga.njobs * wstride;
      SsimPoolJob& P = rows.job[rows.njobs];
      P = SsimPoolJob{};
      P.win = J.win; P.nx = J.nx; P.ny = J.ny;
      P.row_sum = rowsum + (size_t)slot * 3 * gny_[0] + (size_t)c * gny_[scale];   // finalize reads [c][ny_scale]
      ga.njobs++; rows.njobs++;
    }
    SsimSlot& sl = fa.slot[slot];
    sl.row_sum = rowsum + (size_t)slot * 3 * gny_[0];
    sl.nx = gnx_[scale]; sl.ny = gny_[scale]; sl.use_ws = use_ws;
    sl.ws_base = gws_base_; sl.ws_step = prm_.ssim_stride;
  };
  auto flush = [&]() -> qmiv_status {
    if(ga.njobs == 0) { return QMIV_OK; }
    int t = prof_begin(s);
    QMIV_CUDA(launch_ssim_gen(ga, prm_.ssim_mode, N, prm_.ssim_stride, prm_.ssim_border, s));
    prof_end(s, QMIV_STAGE_SSIM_WIN, t);
    t = prof_begin(s);
    QMIV_CUDA(launch_ssim_rows(rows, s));
    prof_end(s, QMIV_STAGE_SSIM_ROWS, t);
    ga.njobs = 0; rows.njobs = 0;
    return QMIV_OK;
  };

  const int use_ws = prm_.erp ? 1 : 0;
  if(mask & QMIV_IVSSIM)   // T2R = SSIM(In0, SCP1), R2T = SSIM(In1, SCP0) with ERP row weights (xIVSSIM.cpp:46-47)
  {
    add(in0, scp1, 0, kSlotIvT2R, 1, use_ws);
    add(in1, scp0, 0, kSlotIvR2T, 1, use_ws);
  }
  if(mask & QMIV_SSIM) { add(in0, in1, 0, kSlotSsim, 1, 0); }   // xSSIM.h:83
  QMIV_TRY(flush());
  if(mask & (QMIV_MSSSIM | QMIV_IVMSSSIM))   // xSSIM.cpp:115-141, every scale with the same option
  {
    size_t lv = 0;
    for(int s2 = 1; s2 < ns_; s2++) { lv += (size_t)(S.W >> s2) * (S.H >> s2) * 3; }
    auto level_base = [&](int img, int scale) -> char* {
      size_t o = (size_t)img * lv;
      for(int s2 = 1; s2 < scale; s2++) { o += (size_t)(S.W >> s2) * (S.H >> s2) * 3; }
      return pyr_.as<char>() + o * S.esz;
    };
    auto level_img = [&](int img, int scale) -> Img {
      if(scale == 0) { return img == 0 ? in0 : img == 1 ? in1 : img == 2 ? scp0 : scp1; }
      return img444(level_base(img, scale), S.W >> scale, S.H >> scale, S.esz);
    };
    auto down = [&](int ia, int ib, int scale) -> qmiv_status {   // level scale - 1 -> scale of pictures ia, ib
      const int t = prof_begin(s);
      QMIV_CUDA(launch_downsample2<T>(level_img(ia, scale - 1), level_img(ib, scale - 1),
                                      mut444(level_base(ia, scale), S.W >> scale, S.H >> scale, S.esz),
                                      mut444(level_base(ib, scale), S.W >> scale, S.H >> scale, S.esz), S.W >> scale,
                                      S.H >> scale, clip, s));
      prof_end(s, QMIV_STAGE_SSIM_WIN, t);
      return QMIV_OK;
    };
    for(int sc = 0; sc < ns_; sc++)
    {
      const int last = sc == ns_ - 1 ? 1 : 0;
      if(sc > 0)
      {
        if(mask & QMIV_MSSSIM) { QMIV_TRY(down(0, 1, sc)); }
        if(mask & QMIV_IVMSSSIM)
        {
          if(!(mask & QMIV_MSSSIM)) { QMIV_TRY(down(0, 1, sc)); }
          QMIV_TRY(down(2, 3, sc));
        }
      }
      if(mask & QMIV_MSSSIM) { add(level_img(0, sc), level_img(1, sc), sc, kSlotMs + sc, last, 0); }
      if(mask & QMIV_IVMSSSIM)   // no ERP weighting (xIVSSIM.cpp:77-78)
      {
        add(level_img(0, sc), level_img(3, sc), sc, kSlotIvmsT2R + sc, last, 0);
        add(level_img(1, sc), level_img(2, sc), sc, kSlotIvmsR2T + sc, last, 0);
      }
      QMIV_TRY(flush());
    }
  }
  return QMIV_OK;
}

}  // namespace qmiv

using namespace qmiv;

// =============================================================================================
// calc entry points
// =============================================================================================
static qmiv_status wait_event(cudaEvent_t ev, int32_t timeout_ms)
{
  if(timeout_ms < 0) { QMIV_CUDA(cudaEventSynchronize(ev)); return QMIV_OK; }
  const auto t0 = std::chrono::steady_clock::now();
  for(;;)
  {
    const cudaError_t e = cudaEventQuery(ev);
    if(e == cudaSuccess) { return QMIV_OK; }
    if(e != cudaErrorNotReady) { return cuda_fail(e, "cudaEventQuery"); }
    const auto el = std::chrono::duration_cast<std::chrono::milliseconds>(std::chrono::steady_clock::now() - t0).count();
    if(el >= timeout_ms) { return fail(QMIV_ERR_TIMEOUT, "result not ready within the timeout"); }
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

static qmiv_status calc_submit(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, uint32_t mask, bool want_scp,
                               bool want_gcd = false)
{
  if(!calc || !in0 || !in1) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  if(calc->pending) { return fail(QMIV_ERR_BUSY, "a submission is already in flight on this calc"); }
  QMIV_TRY(check_metrics(calc->pipe.shape(), mask, calc->prm));
  QMIV_CUDA(cudaSetDevice(calc->ctx->device));
  const bool host = in0->mem == QMIV_MEM_HOST || in1->mem == QMIV_MEM_HOST;
  const bool colour = calc->colour && calc->colour->active;
  QMIV_TRY(calc->pipe.prepare(colour ? 0u : mask, colour ? false : want_scp, host));
  Img a{}, b{};
  QMIV_TRY(calc->pipe.resolve(in0, 0, a, calc->stream));
  QMIV_TRY(calc->pipe.resolve(in1, 1, b, calc->stream));
  if(colour)
  {
    // metrics on the converted 4:4:4 pictures (xAppQMIV.cpp:853-891 before :893-1108)
    ColourStage& cs = *calc->colour;
    Img c0{}, c1{};
    QMIV_TRY(cs.convert(calc->ctx, calc->shape, calc->prm, a, b, c0, c1, calc->stream));
    QMIV_TRY(cs.pipe444.prepare(mask, want_scp, false));
    QMIV_TRY(cs.pipe444.enqueue(c0, c1, mask, want_scp, want_gcd, calc->stream));
  }
  else { QMIV_TRY(calc->pipe.enqueue(a, b, mask, want_scp, want_gcd, calc->stream)); }
  QMIV_CUDA(cudaEventRecord(calc->done, calc->stream));
  calc->pending = true;
  calc->pending_mask = mask;
  calc->pending_colour = colour;
  return QMIV_OK;
}

static qmiv_status calc_collect(qmiv_calc calc, int32_t timeout_ms, qmiv_result* out)
{
  if(!calc->pending) { return fail(QMIV_ERR_INVALID_ARG, "nothing submitted"); }
  QMIV_TRY(wait_event(calc->done, timeout_ms));
  calc->pending = false;
  calc->has_last = !calc->pending_colour;
  calc->pipe.harvest_profile();
  if(calc->pending_colour)
  {
    ColourStage& cs = *calc->colour;
    cs.pipe444.harvest_profile();
    const PairOut& o = cs.pipe444.host_out();
    const int32_t inv = cs.invalid_flags(calc->shape.maxv);   // the original frames, before conversion
    if(out)
    {
      finish_result(o, cs.pipe444.finish_info(calc->pending_mask), out);
      out->invalid_pel[0] = (inv & 1) != 0;
      out->invalid_pel[1] = (inv & 2) != 0;
    }
    if(calc->prm.invalid_pel_action == QMIV_PEL_STOP && inv)
    {
      return fail(QMIV_ERR_INVALID_PIXEL, "input frame contains samples above the bit depth's maximum");
    }
    return pair_status(o, calc->prm.invalid_pel_action);
  }
  const PairOut& o = calc->pipe.host_out();
  if(out) { finish_result(o, calc->pipe.finish_info(calc->pending_mask), out); }
  return pair_status(o, calc->prm.invalid_pel_action);
}

extern "C" {

qmiv_status qmiv_calc_create(qmiv_ctx ctx, int32_t width, int32_t height, int32_t bitdepth, int32_t chroma_format,
                             const qmiv_params* params, qmiv_calc* out_calc)
{
  if(!ctx || !out_calc) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  *out_calc = nullptr;
  qmiv_params prm;
  if(params) { prm = *params; } else { qmiv_params_default(&prm); }
  QMIV_TRY(validate_params(prm));
  Shape shape;
  QMIV_TRY(shape.init(width, height, bitdepth, chroma_format));
  QMIV_CUDA(cudaSetDevice(ctx->device));
  qmiv_calc c = new qmiv_calc_s();
  c->ctx = ctx; c->shape = shape; c->prm = prm;
  qmiv_status st = c->pipe.configure(ctx, shape, prm, prm.search_range);
  if(st == QMIV_OK)
  {
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if(e == cudaSuccess) { e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming); }
    if(e != cudaSuccess) { st = cuda_fail(e, "stream/event creation"); }
  }
  if(st != QMIV_OK) { qmiv_calc_destroy(c); return st; }
  *out_calc = c;
  return QMIV_OK;
}

qmiv_status qmiv_calc_destroy(qmiv_calc calc)
{
  if(!calc) { return fail(QMIV_ERR_INVALID_ARG, "calc is null"); }
  cudaSetDevice(calc->ctx->device);
  if(calc->stream) { cudaStreamSynchronize(calc->stream); }
  if(calc->done) { cudaEventDestroy(calc->done); }
  if(calc->stream) { cudaStreamDestroy(calc->stream); }
  delete calc;
  return QMIV_OK;
}

qmiv_status qmiv_frame_pair_compute(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, uint32_t metric_mask, qmiv_result* out)
{
  QMIV_TRY(calc_submit(calc, in0, in1, metric_mask, false));
  return calc_collect(calc, -1, out);
}

qmiv_status qmiv_frame_pair_submit(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, uint32_t metric_mask)
{
  return calc_submit(calc, in0, in1, metric_mask, false);
}

qmiv_status qmiv_frame_pair_wait(qmiv_calc calc, int32_t timeout_ms, qmiv_result* out)
{
  if(!calc) { return fail(QMIV_ERR_INVALID_ARG, "calc is null"); }
  return calc_collect(calc, timeout_ms, out);
}

qmiv_status qmiv_calc_set_color_space(qmiv_calc calc, int32_t color_space_input, int32_t color_space_metric)
{
  if(!calc) { return fail(QMIV_ERR_INVALID_ARG, "calc is null"); }
  if(calc->pending) { return fail(QMIV_ERR_BUSY, "a submission is in flight on this calc"); }
  std::unique_ptr<ColourStage> cs(new ColourStage());
  QMIV_TRY(cs->configure(color_space_input, color_space_metric));
  if(cs->active && calc->shape.bitdepth > 14) { return fail(QMIV_ERR_UNSUPPORTED, "colour conversion needs bit depth <= 14"); }
  calc->colour = cs->active ? std::move(cs) : nullptr;
  return QMIV_OK;
}

static bool colour_set(qmiv_calc calc) { return calc && calc->colour && calc->colour->active; }

qmiv_status qmiv_calc_gcd(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, int32_t gcd_r2t[4])
{
  if(colour_set(calc)) { return fail(QMIV_ERR_UNSUPPORTED, "not available with a colour conversion set"); }
  if(!gcd_r2t) { return fail(QMIV_ERR_INVALID_ARG, "gcd_r2t is null"); }
  qmiv_result r;
  QMIV_TRY(calc_submit(calc, in0, in1, 0, false, true));
  QMIV_TRY(calc_collect(calc, -1, &r));
  for(int c = 0; c < 4; c++) { gcd_r2t[c] = r.gcd_r2t[c]; }
  return QMIV_OK;
}

qmiv_status qmiv_calc_scp(qmiv_calc calc, const qmiv_frame* in0, const qmiv_frame* in1, const int32_t* gcd_r2t,
                          uint16_t* scp0, uint16_t* scp1, int32_t dst_mem)
{
  if(dst_mem != QMIV_MEM_HOST && dst_mem != QMIV_MEM_DEVICE) { return fail(QMIV_ERR_INVALID_ARG, "bad dst_mem"); }
  if(!calc) { return fail(QMIV_ERR_INVALID_ARG, "calc is null"); }
  if(colour_set(calc)) { return fail(QMIV_ERR_UNSUPPORTED, "not available with a colour conversion set"); }
  int32_t saved[4];
  const bool had = calc->pipe.get_gcd_override(saved);
  if(gcd_r2t) { calc->pipe.set_gcd_override(gcd_r2t); }
  qmiv_status st = calc_submit(calc, in0, in1, 0, true);
  if(st == QMIV_OK) { st = calc_collect(calc, -1, nullptr); }
  calc->pipe.set_gcd_override(had ? saved : nullptr);
  QMIV_TRY(st);
  const Shape& S = calc->shape;
  const size_t n = (size_t)3 * S.W * S.H;
  for(int k = 0; k < 2; k++)
  {
    uint16_t* dst = k ? scp1 : scp0;
    if(!dst) { continue; }
    const void* src = calc->pipe.scp(k);
    if(S.esz == 2)
    {
      QMIV_CUDA(cudaMemcpy(dst, src, n * 2, dst_mem == QMIV_MEM_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice));
    }
    else
    {
      std::vector<uint8_t> tmp(n);
      QMIV_CUDA(cudaMemcpy(tmp.data(), src, n, cudaMemcpyDeviceToHost));
      if(dst_mem == QMIV_MEM_HOST) { for(size_t i = 0; i < n; i++) { dst[i] = tmp[i]; } }
      else
      {
        std::vector<uint16_t> w(tmp.begin(), tmp.end());
        QMIV_CUDA(cudaMemcpy(dst, w.data(), n * 2, cudaMemcpyHostToDevice));
      }
    }
  }
  return QMIV_OK;
}

qmiv_status qmiv_calc_cps_rows(qmiv_calc calc, uint64_t* rows_r2t, uint64_t* rows_t2r)
{
  if(!calc) { return fail(QMIV_ERR_INVALID_ARG, "calc is null"); }
  if(colour_set(calc)) { return fail(QMIV_ERR_UNSUPPORTED, "not available with a colour conversion set"); }
  if(!calc->has_last || !calc->pipe.cps_rows()) { return fail(QMIV_ERR_INVALID_ARG, "no CPS result available"); }
  const Shape& S = calc->shape;
  std::vector<uint32_t> tmp((size_t)2 * S.H * 3);
  QMIV_CUDA(cudaMemcpy(tmp.data(), calc->pipe.cps_rows(), tmp.size() * 4, cudaMemcpyDeviceToHost));
  for(int d = 0; d < 2; d++)
  {
    uint64_t* dst = d ? rows_t2r : rows_r2t;
    if(!dst) { continue; }
    for(size_t i = 0; i < (size_t)S.H * 3; i++) { dst[i] = (uint64_t)(int64_t)(int32_t)tmp[(size_t)d * S.H * 3 + i]; }
  }
  return QMIV_OK;
}

qmiv_status qmiv_calc_set_gcd(qmiv_calc calc, const int32_t* gcd_r2t)
{
  if(!calc) { return fail(QMIV_ERR_INVALID_ARG, "calc is null"); }
  if(calc->pending) { return fail(QMIV_ERR_BUSY, "a submission is in flight on this calc"); }
  calc->pipe.set_gcd_override(gcd_r2t);
  return QMIV_OK;
}

qmiv_status qmiv_calc_stream(qmiv_calc calc, void** cuda_stream)
{
  if(!calc || !cuda_stream) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  *cuda_stream = (void*)calc->stream;
  return QMIV_OK;
}

}  // extern "C"
