// Batched form (qmiv_batch_*): many frame pairs of uneven shape per call on the multi-pair engine.
#include "qmiv_engine.h"

using namespace qmiv;

struct qmiv_batch_s
{
  qmiv_ctx_s* ctx = nullptr;
  Engine      engine;
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
  b->ctx = ctx;
  const qmiv_status st = b->engine.init(ctx, prm, max_pairs, max_pixels, flags);
  if(st != QMIV_OK) { delete b; return st; }
  *out_batch = b;
  return QMIV_OK;
}

qmiv_status qmiv_batch_destroy(qmiv_batch b)
{
  if(!b) { return fail(QMIV_ERR_INVALID_ARG, "batch is null"); }
  delete b;
  return QMIV_OK;
}

qmiv_status qmiv_batch_compute(qmiv_batch b, const qmiv_pair_desc* pairs, int32_t n, qmiv_result* out)
{
  if(!b || (!pairs && n > 0) || (!out && n > 0)) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  return b->engine.run(pairs, n, out);
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
