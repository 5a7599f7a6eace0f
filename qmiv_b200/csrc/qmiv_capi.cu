// C ABI of the QMIV B200 library (include/qmiv_gpu.h): contexts, calcs (plain form), and the host
// finishing step that turns the device's exact integer / FP64 pooled values into dB and indices
// with the same libm calls as the reference (log10 in xPSNR.cpp:186-192, std::pow in
// xSSIM.cpp:251-253, cos in xWeightedSpherically.cpp:13-29).
#include "qmiv_gpu.h"
#include "qmiv_host.h"

#include <cfloat>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>

using namespace qmiv;

namespace qmiv {

thread_local std::string g_last_error;

qmiv_status fail(qmiv_status st, const std::string& msg)
{
  g_last_error = msg;
  return st;
}

qmiv_status cuda_fail(cudaError_t e, const char* what)
{
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? QMIV_ERR_OUT_OF_MEMORY : QMIV_ERR_CUDA;
}

// ---------------------------------------------------------------------------------------------
// device memory accounted against the context budget
// ---------------------------------------------------------------------------------------------
qmiv_status DevMem::alloc(qmiv_ctx_s* ctx_, size_t n)
{
  release();
  if(n == 0) { return QMIV_OK; }
  const size_t rounded = (n + 255) & ~(size_t)255;
  if(!ctx_->reserve(rounded)) { return fail(QMIV_ERR_BUDGET, "HBM budget exceeded"); }
  const cudaError_t e = cudaMalloc(&p, rounded);
  if(e != cudaSuccess) { ctx_->unreserve(rounded); p = nullptr; return cuda_fail(e, "cudaMalloc"); }
  ctx = ctx_; bytes = rounded;
  return QMIV_OK;
}

void DevMem::release()
{
  if(p) { cudaFree(p); ctx->unreserve(bytes); }
  p = nullptr; bytes = 0;
}

qmiv_status DevMem::ensure(qmiv_ctx_s* ctx_, size_t n)
{
  if(p && bytes >= n) { return QMIV_OK; }
  return alloc(ctx_, n);
}

// ---------------------------------------------------------------------------------------------
// host finishing helpers
// ---------------------------------------------------------------------------------------------
static const double kMsExponents[5][5] = {  // libs/pmbb-ivqm/src/xStructSimConsts.h:42-49
  { 1.0000, 0.0000, 0.0000, 0.0000, 0.0000 },
  { 0.1356, 0.8644, 0.0000, 0.0000, 0.0000 },
  { 0.0711, 0.4530, 0.4760, 0.0000, 0.0000 },
  { 0.0517, 0.3295, 0.3462, 0.2726, 0.0000 },
  { 0.0448, 0.2856, 0.3001, 0.2363, 0.1333 },
};

double psnr_from_ssd(double ssd, int64_t area, int32_t bitdepth)  // xPSNR.cpp:186-192
{
  const uint64_t maxv = (uint64_t)((1 << bitdepth) - 1);
  const uint64_t MAX  = (uint64_t)area * (maxv * maxv);
  return ssd > 0 ? 10.0 * log10((double)MAX / ssd) : DBL_MAX;
}

int32_t num_scales(int32_t W, int32_t H)  // xSSIM.cpp:520-532
{
  for(int32_t i = 0; i < 5; i++) { const int32_t lim = 32 << i; if(W < lim || H < lim) { return i; } }
  return 5;
}

int32_t round_f32_half_away(float f)  // xHelpersFLT.h:32
{
  volatile float t = f + copysignf(0.5f, f);
  return (int32_t)t;
}

void ws_weights(int32_t H, int32_t lat_range, double* w, double& correction)  // xWeightedSpherically.cpp:13-29
{
  const double pi  = 3.14159265358979323846;
  const double heq = 180.0 * (double)H / (double)lat_range;
  const double off = (heq - H) / 2.0;
  double s = 0.0, c = 0.0;  // KBNS (xKBNS.h:36-43)
  for(int32_t h = 0; h < H; h++)
  {
    w[h] = cos((h + off - (heq / 2 - 0.5)) * pi / heq);
    const double t = s + w[h];
    if(std::fabs(s) >= std::fabs(w[h])) { c += ((s - t) + w[h]); } else { c += ((w[h] - t) + s); }
    s = t;
  }
  correction = H / (s + c);
}

void ws_weights(int32_t H, int32_t lat_range, std::vector<double>& w, double& correction)
{
  w.resize(H);
  ws_weights(H, lat_range, w.data(), correction);
}

// per-picture average of a per-component metric, xMetricQMIV.cpp:91-97
static double per_pic3(const double v[4], const int32_t w[4])
{
  const double inv = 1.0 / (double)(w[0] + w[1] + w[2] + w[3]);
  return (v[0] * w[0] + v[1] * w[1] + v[2] * w[2]) * inv;
}
// weighted 4-lane average of the IV metrics, xIVPSNR.cpp:184-187 / xIVSSIM.cpp:47-52
static double per_pic4(const double v[4], const int32_t w[4])
{
  const double inv = 1.0 / (double)(w[0] + w[1] + w[2] + w[3]);
  return (v[0] * (double)w[0] + v[1] * (double)w[1] + v[2] * (double)w[2] + v[3] * (double)w[3]) * inv;
}

qmiv_status pair_status(const PairOut& o, int32_t invalid_pel_action)
{
  if(o.flags & 8) { return fail(QMIV_ERR_TIMEOUT, "a CPS tile load did not complete within its wait bound"); }
  if(invalid_pel_action == QMIV_PEL_STOP && (o.flags & 3))
  {
    return fail(QMIV_ERR_INVALID_PIXEL, "input frame contains samples above the bit depth's maximum");
  }
  return QMIV_OK;
}

void finish_result(const PairOut& o, const FinishInfo& fi, qmiv_result* r)
{
  std::memset(r, 0, sizeof(*r));
  const int64_t area = (int64_t)fi.W * fi.H;
  for(int c = 0; c < 4; c++) { r->gcd_r2t[c] = o.gcd[c]; }
  for(int c = 0; c < 3; c++)
  {
    r->exact[c] = o.ssd[c] == 0;
    r->ssd[c]   = o.ssd[c];
    r->cps_sse_r2t[c] = o.cps_sum[0][c];
    r->cps_sse_t2r[c] = o.cps_sum[1][c];
  }
  r->invalid_pel[0] = (o.flags & 1) != 0;
  r->invalid_pel[1] = (o.flags & 2) != 0;
  const uint32_t m = fi.mask;
  const double fake = psnr_from_ssd(1, area, fi.bitdepth);  // xPSNR.h:55, xAppQMIV.cpp:974-981
  const int32_t* cwa = fi.cwa;

  if(m & QMIV_PSNR)
  {
    for(int c = 0; c < 3; c++) { r->psnr[c] = r->exact[c] ? fake : psnr_from_ssd((double)o.ssd[c], area, fi.bitdepth); }
    r->psnr_pic = per_pic3(r->psnr, cwa);
  }
  if(m & QMIV_WSPSNR)  // xWSPSNR.cpp:48-81, :112-138
  {
    for(int c = 0; c < 3; c++)
    {
      const double v = fi.erp ? psnr_from_ssd(o.ws_ssd[c] * fi.ws_corr, area, fi.bitdepth)
                              : psnr_from_ssd((double)o.ssd[c], area, fi.bitdepth);
      r->wspsnr[c] = r->exact[c] ? fake : v;
    }
    r->wspsnr_pic = per_pic3(r->wspsnr, cwa);
  }
  if(m & QMIV_IVPSNR)  // xIVPSNR.cpp:109-121, :163-189
  {
    double q[2];
    for(int d = 0; d < 2; d++)
    {
      double qc[4] = { 0, 0, 0, 0 };
      for(int c = 0; c < 3; c++)
      {
        const double err = fi.erp ? o.cps_ws[d][c] : (double)o.cps_sum[d][c];
        qc[c] = psnr_from_ssd(err > 0 ? err : 1.0, area, fi.bitdepth);
      }
      q[d] = per_pic4(qc, cwa);
    }
    r->ivpsnr_r2t = q[0]; r->ivpsnr_t2r = q[1];
    r->ivpsnr = (q[1] < q[0]) ? q[1] : q[0];  // std::min(R2T, T2R)
  }
  if(m & QMIV_SSIM)
  {
    for(int c = 0; c < 3; c++) { r->ssim[c] = o.ssim[kSlotSsim][c]; }
    r->ssim_pic = per_pic3(r->ssim, cwa);
  }
  auto ms_compose = [&](int first_slot, double out[4]) {  // xSSIM.cpp:248-253
    out[3] = 0.0;
    for(int c = 0; c < 3; c++)
    {
      double score = 1.0;
      for(int s = 0; s < fi.num_scales; s++)
      {
        double v = o.ssim[first_slot + s][c];
        v = v < 0 ? 0.0 : v;
        score *= std::pow(v, kMsExponents[fi.num_scales - 1][s]);
      }
      out[c] = score;
    }
  };
  if(m & QMIV_MSSSIM)
  {
    ms_compose(kSlotMs, r->msssim);
    r->msssim_pic = per_pic3(r->msssim, cwa);
  }
  if(m & QMIV_IVSSIM)  // xIVSSIM.cpp:46-56
  {
    double t2r[4] = { o.ssim[kSlotIvT2R][0], o.ssim[kSlotIvT2R][1], o.ssim[kSlotIvT2R][2], 0.0 };
    double r2t[4] = { o.ssim[kSlotIvR2T][0], o.ssim[kSlotIvR2T][1], o.ssim[kSlotIvR2T][2], 0.0 };
    r->ivssim_t2r = per_pic4(t2r, cwa);
    r->ivssim_r2t = per_pic4(r2t, cwa);
    r->ivssim = (r->ivssim_r2t < r->ivssim_t2r) ? r->ivssim_r2t : r->ivssim_t2r;  // std::min(T2R, R2T)
  }
  if(m & QMIV_IVMSSSIM)  // xIVSSIM.cpp:62-92
  {
    double t2r[4], r2t[4];
    ms_compose(kSlotIvmsT2R, t2r);
    ms_compose(kSlotIvmsR2T, r2t);
    r->ivmsssim_t2r = per_pic4(t2r, cwa);
    r->ivmsssim_r2t = per_pic4(r2t, cwa);
    r->ivmsssim = (r->ivmsssim_r2t < r->ivmsssim_t2r) ? r->ivmsssim_r2t : r->ivmsssim_t2r;
  }
}

}  // namespace qmiv

// =============================================================================================
// context
// =============================================================================================
bool qmiv_ctx_s::reserve(size_t n)
{
  std::lock_guard<std::mutex> lk(mu);
  if(budget != 0 && used + n > budget) { return false; }
  used += n;
  return true;
}
void qmiv_ctx_s::unreserve(size_t n)
{
  std::lock_guard<std::mutex> lk(mu);
  used -= n;
}

extern "C" {

int32_t qmiv_api_version(void) { return QMIV_API_VERSION; }

const char* qmiv_status_string(qmiv_status s)
{
  switch(s)
  {
  case QMIV_OK: return "ok";
  case QMIV_ERR_INVALID_ARG: return "invalid argument";
  case QMIV_ERR_UNSUPPORTED: return "unsupported";
  case QMIV_ERR_CUDA: return "CUDA error";
  case QMIV_ERR_OUT_OF_MEMORY: return "out of device memory";
  case QMIV_ERR_INVALID_PIXEL: return "invalid pixel value";
  case QMIV_ERR_BUDGET: return "HBM budget exceeded";
  case QMIV_ERR_TIMEOUT: return "timeout";
  case QMIV_ERR_NOT_READY: return "not ready";
  case QMIV_ERR_CANCELLED: return "cancelled";
  case QMIV_ERR_BUSY: return "busy";
  }
  return "unknown status";
}

const char* qmiv_last_error(void) { return qmiv::g_last_error.c_str(); }

void qmiv_params_default(qmiv_params* p)
{
  if(!p) { return; }
  std::memset(p, 0, sizeof(*p));
  p->search_range = 2;
  p->cws[0] = 4; p->cws[1] = 1; p->cws[2] = 1; p->cws[3] = 0;
  p->cwa[0] = 4; p->cwa[1] = 1; p->cwa[2] = 1; p->cwa[3] = 0;
  p->unc[0] = 0.01f; p->unc[1] = 0.01f; p->unc[2] = 0.01f; p->unc[3] = 0.0f;
  p->erp = 0; p->lon_range_deg = 360; p->lat_range_deg = 180;
  p->ssim_window = 8; p->ssim_stride = 4;
  p->invalid_pel_action = QMIV_PEL_STOP;
  p->ssim_mode = QMIV_SSM_BLOCK_AVERAGED; p->ssim_border = QMIV_BRD_NONE;
}

qmiv_status qmiv_ctx_create(int32_t device, uint64_t hbm_budget_bytes, qmiv_ctx* out_ctx)
{
  if(!out_ctx) { return fail(QMIV_ERR_INVALID_ARG, "out_ctx is null"); }
  *out_ctx = nullptr;
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if(e != cudaSuccess) { return cuda_fail(e, "cudaGetDeviceCount"); }
  if(device < 0 || device >= n) { return fail(QMIV_ERR_INVALID_ARG, "device ordinal out of range"); }
  e = cudaSetDevice(device);
  if(e != cudaSuccess) { return cuda_fail(e, "cudaSetDevice"); }
  qmiv_ctx c = new qmiv_ctx_s();
  c->device = device; c->budget = hbm_budget_bytes; c->used = 0;
  *out_ctx = c;
  return QMIV_OK;
}

qmiv_status qmiv_ctx_destroy(qmiv_ctx ctx)
{
  if(!ctx) { return fail(QMIV_ERR_INVALID_ARG, "ctx is null"); }
  delete ctx;
  return QMIV_OK;
}

qmiv_status qmiv_ctx_set_profiling(qmiv_ctx ctx, int32_t enable)
{
  if(!ctx) { return fail(QMIV_ERR_INVALID_ARG, "ctx is null"); }
  std::lock_guard<std::mutex> lk(ctx->mu);
  ctx->profiling = enable != 0;
  return QMIV_OK;
}

qmiv_status qmiv_ctx_stage_times(qmiv_ctx ctx, double ms[8], uint64_t launches[8], int32_t reset)
{
  if(!ctx) { return fail(QMIV_ERR_INVALID_ARG, "ctx is null"); }
  std::lock_guard<std::mutex> lk(ctx->mu);
  for(int i = 0; i < QMIV_NUM_STAGES; i++)
  {
    if(ms) { ms[i] = ctx->stage_ms[i]; }
    if(launches) { launches[i] = ctx->stage_n[i]; }
    if(reset) { ctx->stage_ms[i] = 0.0; ctx->stage_n[i] = 0; }
  }
  return QMIV_OK;
}

qmiv_status qmiv_ctx_memory(qmiv_ctx ctx, uint64_t* used_bytes, uint64_t* budget_bytes)
{
  if(!ctx) { return fail(QMIV_ERR_INVALID_ARG, "ctx is null"); }
  std::lock_guard<std::mutex> lk(ctx->mu);
  if(used_bytes) { *used_bytes = ctx->used; }
  if(budget_bytes) { *budget_bytes = ctx->budget; }
  return QMIV_OK;
}

}  // extern "C"
