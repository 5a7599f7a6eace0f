// Allocation-free entry point qmiv_frame_pair_compute_static (declared in include/qmiv_gpu.h).
//
// Some callers cannot allocate device memory: code running inside a host application's memory
// manager or a plugin sandbox that forbids cudaMalloc, and paths held to a no-allocation rule after
// start-up. This entry point serves them. It runs the same kernels as the plain form for PSNR,
// WS-PSNR and IV-PSNR of one device-resident frame pair, with all of its scratch in one file-scope
// device array of fixed size, and calls no cudaMalloc, cudaFree or other allocating routine.
//
// In host code the array's name is a host-side stand-in, not a device address. Every call looks up
// the array's device address with cudaGetSymbolAddress for the device (and context) current at the
// call and passes it to the kernels; the lookup allocates nothing once the library's module is
// loaded on that device, so a context created by the caller or a context re-created after
// cudaDeviceReset is always given its own copy's address. With CUDA's lazy module loading the module,
// and with it the array, is loaded on a device at the first call there: callers that may not allocate
// later make one call during start-up. Every call shares the array; calls that overlap on the GPU
// race, so callers must serialise them.
#include "qmiv_host.h"

#include <cstring>

using namespace qmiv;

namespace {

constexpr int32_t kMaxH = QMIV_STATIC_MAX_HEIGHT;
constexpr size_t  kAlign = 256;
constexpr size_t align_up(size_t n) { return (n + kAlign - 1) & ~(kAlign - 1); }

// scratch layout (bytes): per-row SD / SSD of up to three planes of kMaxH rows, the 32-bit CPS row
// sums of both directions, the device result block, and the ERP row weights
constexpr size_t kOffRowSd  = 0;
constexpr size_t kOffRowSsd = kOffRowSd + align_up(sizeof(int64_t) * 3 * kMaxH);
constexpr size_t kOffCps    = kOffRowSsd + align_up(sizeof(uint64_t) * 3 * kMaxH);
constexpr size_t kOffOut    = kOffCps + align_up(sizeof(uint32_t) * 2 * 3 * kMaxH);
constexpr size_t kOffWs     = kOffOut + align_up(sizeof(PairOut));
constexpr size_t kScratchBytes = kOffWs + align_up(sizeof(double) * kMaxH);

static __device__ __align__(256) unsigned char g_static_scratch[kScratchBytes];

// device address of g_static_scratch in the current device's context
qmiv_status scratch_address(char** out)
{
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
  if(e != cudaSuccess || p == nullptr) { return cuda_fail(e == cudaSuccess ? cudaErrorInvalidSymbol : e, "cudaGetSymbolAddress"); }
  *out = static_cast<char*>(p);
  return QMIV_OK;
}

template <typename T>
qmiv_status enqueue_static(char* base, const Shape& S, const qmiv_params& prm, const Img& in0, const Img& in1,
                           uint32_t mask, int32_t ws_rows, cudaStream_t s)
{
  int64_t*  row_sd  = reinterpret_cast<int64_t*>(base + kOffRowSd);
  uint64_t* row_ssd = reinterpret_cast<uint64_t*>(base + kOffRowSsd);
  uint32_t* cps     = reinterpret_cast<uint32_t*>(base + kOffCps);
  PairOut*  dout    = reinterpret_cast<PairOut*>(base + kOffOut);
  double*   ws      = reinterpret_cast<double*>(base + kOffWs);
  const bool search = (mask & QMIV_IVPSNR) != 0;
  const uint32_t clip = prm.invalid_pel_action == QMIV_PEL_CNCL ? (uint32_t)S.maxv : 0xffffu;

  // the array keeps the previous call's contents: clear what must start at zero
  QMIV_CUDA(cudaMemsetAsync(dout, 0, sizeof(PairOut), s));
  if(search) { QMIV_CUDA(cudaMemsetAsync(cps, 0, sizeof(uint32_t) * 2 * 3 * S.H, s)); }

  PrepassArgs pa{};
  pa.in0 = in0; pa.in1 = in1;
  for(int c = 0; c < 3; c++) { pa.rows[c] = (int32_t)S.plane_rows(c); pa.cols[c] = (int32_t)S.plane_cols(c); }
  pa.clip = clip; pa.row_sd = row_sd; pa.row_ssd = row_ssd; pa.out = dout;
  QMIV_CUDA(launch_prepass<T>(pa, s));

  int32_t maxdiff[4];
  for(int c = 0; c < 4; c++) { maxdiff[c] = round_f32_half_away(prm.unc[c] * (float)S.maxv); }
  ReduceArgs ra{};
  for(int c = 0; c < 3; c++) { ra.rows[c] = pa.rows[c]; ra.mult[c] = c ? (1 << (S.sx + S.sy)) : 1; }
  ra.area = (int64_t)S.W * S.H; ra.maxv = S.maxv;
  for(int c = 0; c < 4; c++) { ra.maxdiff[c] = maxdiff[c]; }
  ra.need_gcd = search; ra.fp32_ok = cps_fp32_exact(S.maxv, prm.cws, maxdiff);
  ra.clip_on = prm.invalid_pel_action == QMIV_PEL_CNCL;
  ra.row_sd = row_sd; ra.row_ssd = row_ssd; ra.out = dout;
  QMIV_CUDA(launch_reduce(ra, s));

  if(search)
  {
    CpsArgs ca{};
    ca.in0 = in0; ca.in1 = in1; ca.W = S.W; ca.H = S.H; ca.maxv = S.maxv; ca.clip = clip;
    for(int c = 0; c < 3; c++) { ca.wi[c] = prm.cws[c]; ca.wf[c] = (float)prm.cws[c]; }
    ca.gcd_src = dout; ca.rows = cps; ca.scp0 = nullptr; ca.scp1 = nullptr;
    QMIV_CUDA(launch_cps<T>(ca, prm.search_range, s));
  }

  FinalizeArgs fa{};
  fa.H = S.H;
  for(int c = 0; c < 3; c++) { fa.rows[c] = (int32_t)S.plane_rows(c); fa.sy[c] = c ? S.sy : 0; fa.mult_row[c] = c ? (1 << S.sx) : 1; }
  fa.row_ssd = row_ssd;
  fa.ws = ws_rows ? ws : nullptr;
  fa.do_wspsnr = (mask & QMIV_WSPSNR) ? 1 : 0;
  fa.cps_rows = search ? cps : nullptr;
  fa.nslots = 0;
  fa.out = dout;
  QMIV_CUDA(launch_finalize(fa, s));
  return QMIV_OK;
}

}  // namespace

extern "C" qmiv_status qmiv_frame_pair_compute_static(const qmiv_frame* in0, const qmiv_frame* in1, int32_t width,
                                                      int32_t height, int32_t bitdepth, int32_t chroma_format,
                                                      const qmiv_params* params, uint32_t metric_mask,
                                                      void* cuda_stream, qmiv_result* out)
{
  if(!in0 || !in1 || !out) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  if(in0->mem != QMIV_MEM_DEVICE || in1->mem != QMIV_MEM_DEVICE)
  {
    return fail(QMIV_ERR_INVALID_ARG, "the allocation-free entry point takes device-resident frames only");
  }
  if(metric_mask == 0 || (metric_mask & ~(uint32_t)(QMIV_PSNR | QMIV_WSPSNR | QMIV_IVPSNR)) != 0)
  {
    return fail(QMIV_ERR_UNSUPPORTED, "the allocation-free entry point computes PSNR, WS-PSNR and IV-PSNR only");
  }
  if(height > kMaxH) { return fail(QMIV_ERR_UNSUPPORTED, "picture taller than QMIV_STATIC_MAX_HEIGHT rows"); }
  qmiv_params prm;
  if(params) { prm = *params; } else { qmiv_params_default(&prm); }
  QMIV_TRY(validate_params(prm));
  Shape S;
  QMIV_TRY(S.init(width, height, bitdepth, chroma_format));

  char* base = nullptr;
  QMIV_TRY(scratch_address(&base));
  cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);

  // frames: device pointers used in place
  Img im[2];
  const qmiv_frame* fr[2] = { in0, in1 };
  for(int k = 0; k < 2; k++)
  {
    for(int c = 0; c < 3; c++)
    {
      if(!fr[k]->plane[c]) { return fail(QMIV_ERR_INVALID_ARG, "frame plane is null"); }
      const int64_t row_bytes = (int64_t)(S.plane_cols(c) * S.esz);
      if(fr[k]->pitch[c] < row_bytes || fr[k]->pitch[c] % (int64_t)S.esz) { return fail(QMIV_ERR_INVALID_ARG, "bad plane pitch"); }
      im[k].p[c] = fr[k]->plane[c];
      im[k].pitch[c] = (int32_t)(fr[k]->pitch[c] / (int64_t)S.esz);
      im[k].sx[c] = c ? (int8_t)S.sx : 0;
      im[k].sy[c] = c ? (int8_t)S.sy : 0;
    }
  }

  // ERP row weights: computed into a fixed host array (no heap) and copied into the scratch array
  static thread_local double ws_host[kMaxH];
  double ws_corr = 1.0;
  const bool need_ws = prm.erp && (metric_mask & (QMIV_WSPSNR | QMIV_IVPSNR));
  if(need_ws)
  {
    ws_weights(S.H, prm.lat_range_deg, ws_host, ws_corr);
    QMIV_CUDA(cudaMemcpyAsync(base + kOffWs, ws_host, sizeof(double) * S.H, cudaMemcpyHostToDevice, s));
  }

  const qmiv_status st = S.esz == 1 ? enqueue_static<uint8_t>(base, S, prm, im[0], im[1], metric_mask, need_ws ? S.H : 0, s)
                                    : enqueue_static<uint16_t>(base, S, prm, im[0], im[1], metric_mask, need_ws ? S.H : 0, s);
  QMIV_TRY(st);
  PairOut host;
  QMIV_CUDA(cudaMemcpyAsync(&host, base + kOffOut, sizeof(PairOut), cudaMemcpyDeviceToHost, s));
  QMIV_CUDA(cudaStreamSynchronize(s));

  FinishInfo fi{};
  fi.W = S.W; fi.H = S.H; fi.bitdepth = S.bitdepth; fi.mask = metric_mask;
  fi.erp = prm.erp; fi.ws_corr = ws_corr;
  for(int c = 0; c < 4; c++) { fi.cwa[c] = prm.cwa[c]; }
  fi.num_scales = num_scales(S.W, S.H);
  finish_result(host, fi, out);
  return pair_status(host, prm.invalid_pel_action);
}
