// Batched form (qmiv_batch_*): many frame pairs of uneven shape per call on the multi-pair engine.
#include "qmiv_engine.h"

#include <memory>

using namespace qmiv;

struct qmiv_batch_s
{
  qmiv_ctx_s*  ctx = nullptr;
  qmiv_params  prm{};
  int32_t      max_pairs = 0, flags = 0;
  int64_t      max_pixels = 0;
  Engine       engine;                          // synchronous calls and the first submission slot
  std::unique_ptr<Engine> engine2;              // second submission slot, created on first use
  uint64_t     ticket[2] = { 0, 0 };            // submission held by each slot, 0 = none
  uint64_t     next_ticket = 1;
  Engine& slot(int k) { return k == 0 ? engine : *engine2; }
  std::unique_ptr<MaskedBatch> masked;          // mask-mode calls, created on first use
};

extern "C" {

qmiv_status qmiv_batch_create(qmiv_ctx ctx, int32_t max_pairs, int64_t max_pixels, const qmiv_params* params,
                              int32_t flags, qmiv_batch* out_batch)
{
  if(!ctx || !out_batch || max_pairs <= 0 || max_pixels <= 0) { return fail(QMIV_ERR_INVALID_ARG, "bad batch arguments"); }
  if(flags & ~(QMIV_BATCH_GRAPH | QMIV_BATCH_AUTOTUNE)) { return fail(QMIV_ERR_INVALID_ARG, "unknown batch flags"); }
  *out_batch = nullptr;
  qmiv_params prm;
  if(params) { prm = *params; } else { qmiv_params_default(&prm); }
  QMIV_TRY(validate_params(prm));
  qmiv_batch b = new qmiv_batch_s();
  b->ctx = ctx; b->prm = prm; b->max_pairs = max_pairs; b->max_pixels = max_pixels; b->flags = flags;
  const qmiv_status st = b->engine.init(ctx, prm, max_pairs, max_pixels, flags);
  if(st != QMIV_OK) { delete b; return st; }
  *out_batch = b;
  return QMIV_OK;
}

qmiv_status qmiv_batch_destroy(qmiv_batch b)
{
  if(!b) { return fail(QMIV_ERR_INVALID_ARG, "batch is null"); }
  for(int k = 0; k < 2; k++)
  {
    if(b->ticket[k]) { b->slot(k).collect(nullptr); }    // let submissions in flight finish first
  }
  delete b;
  return QMIV_OK;
}

qmiv_status qmiv_batch_compute(qmiv_batch b, const qmiv_pair_desc* pairs, int32_t n, qmiv_result* out)
{
  if(!b || (!pairs && n > 0) || (!out && n > 0)) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  if(b->ticket[0]) { return fail(QMIV_ERR_BUSY, "an asynchronous submission holds the batch's first slot"); }
  return b->engine.run(pairs, n, out);
}

qmiv_status qmiv_batch_submit(qmiv_batch b, const qmiv_pair_desc* pairs, int32_t n, uint64_t* ticket)
{
  if(!b || (!pairs && n > 0) || !ticket) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  int k = b->ticket[0] == 0 ? 0 : (b->ticket[1] == 0 ? 1 : -1);
  if(k < 0) { return fail(QMIV_ERR_BUSY, "two submissions are in flight; wait for one first"); }
  if(k == 1 && !b->engine2)
  {
    std::unique_ptr<Engine> e(new Engine());
    QMIV_TRY(e->init(b->ctx, b->prm, b->max_pairs, b->max_pixels, b->flags));
    b->engine2 = std::move(e);
  }
  QMIV_TRY(b->slot(k).submit(pairs, n));
  b->ticket[k] = b->next_ticket++;
  *ticket = b->ticket[k];
  return QMIV_OK;
}

qmiv_status qmiv_batch_wait(qmiv_batch b, uint64_t ticket, qmiv_result* out)
{
  if(!b || ticket == 0) { return fail(QMIV_ERR_INVALID_ARG, "bad argument"); }
  for(int k = 0; k < 2; k++)
  {
    if(b->ticket[k] == ticket)
    {
      b->ticket[k] = 0;
      return b->slot(k).collect(out);
    }
  }
  return fail(QMIV_ERR_INVALID_ARG, "unknown ticket");
}

qmiv_status qmiv_batch_compute_masked(qmiv_batch b, const qmiv_pair_desc* pairs, const qmiv_frame* masks,
                                      const int32_t* mask_bitdepths, int32_t n, qmiv_result* out, int32_t* num_non_masked)
{
  if(!b || !pairs || !masks || !mask_bitdepths || n <= 0) { return fail(QMIV_ERR_INVALID_ARG, "null argument or no pairs"); }
  if(n > b->max_pairs) { return fail(QMIV_ERR_INVALID_ARG, "more pairs than the batch was created for"); }
  if(b->ticket[0] || b->ticket[1]) { return fail(QMIV_ERR_BUSY, "a submission is in flight; wait for it first"); }
  QMIV_CUDA(cudaSetDevice(b->ctx->device));
  if(!b->masked) { b->masked.reset(new MaskedBatch()); }
  return b->masked->run(b->ctx, b->prm, b->engine.stream(), pairs, masks, mask_bitdepths, n, out, num_non_masked);
}

qmiv_status qmiv_batch_stream(qmiv_batch b, void** cuda_stream)
{
  if(!b || !cuda_stream) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  *cuda_stream = (void*)b->engine.stream();
  return QMIV_OK;
}

qmiv_status qmiv_batch_tuning(qmiv_batch b, int32_t width, int32_t height, int32_t bitdepth, int32_t search_range,
                              int32_t* cps_tile_w, int32_t* cps_tile_h, int32_t* cps_rows_per_thread)
{
  if(!b) { return fail(QMIV_ERR_INVALID_ARG, "batch is null"); }
  if(!b->engine.tuning(width, height, bitdepth, search_range, cps_tile_w, cps_tile_h, cps_rows_per_thread))
  {
    return fail(QMIV_ERR_INVALID_ARG, "no pair of this kind has been computed by the batch yet");
  }
  return QMIV_OK;
}

}  // extern "C"
