// Batched form: many frame pairs of uneven shape per call.
#include "qmiv_host.h"

#include <map>
#include <memory>
#include <tuple>

using namespace qmiv;

struct qmiv_batch_s
{
  qmiv_ctx_s*  ctx = nullptr;
  qmiv_params  prm{};
  int32_t      max_pairs = 0;
  int64_t      max_pixels = 0;
  int32_t      flags = 0;
  cudaStream_t stream = nullptr;           // the batch's stream: a call starts and ends on it
  std::vector<cudaStream_t> lanes;         // worker streams the pairs are spread over
  std::vector<cudaEvent_t>  lane_done;
  cudaEvent_t               start = nullptr;
  // one pipeline per (pair index) so that every pair of a call has its own scratch
  std::vector<std::unique_ptr<PairPipeline>> pipes;
  std::vector<std::tuple<int32_t, int32_t, int32_t, int32_t, int32_t>> keys;
};

static constexpr int kBatchLanes = 4;

extern "C" {

qmiv_status qmiv_batch_create(qmiv_ctx ctx, int32_t max_pairs, int64_t max_pixels, const qmiv_params* params,
                              int32_t flags, qmiv_batch* out_batch)
{
  if(!ctx || !out_batch || max_pairs <= 0 || max_pixels <= 0) { return fail(QMIV_ERR_INVALID_ARG, "bad batch arguments"); }
  *out_batch = nullptr;
  qmiv_params prm;
  if(params) { prm = *params; } else { qmiv_params_default(&prm); }
  QMIV_TRY(validate_params(prm));
  QMIV_CUDA(cudaSetDevice(ctx->device));
  qmiv_batch b = new qmiv_batch_s();
  b->ctx = ctx; b->prm = prm; b->max_pairs = max_pairs; b->max_pixels = max_pixels; b->flags = flags;
  cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if(e == cudaSuccess) { e = cudaEventCreateWithFlags(&b->start, cudaEventDisableTiming); }
  const int lanes = (flags & QMIV_BATCH_SERIAL) ? 1 : kBatchLanes;
  for(int k = 0; k < lanes && e == cudaSuccess; k++)
  {
    cudaStream_t s; cudaEvent_t d;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if(e == cudaSuccess) { b->lanes.push_back(s); e = cudaEventCreateWithFlags(&d, cudaEventDisableTiming); }
    if(e == cudaSuccess) { b->lane_done.push_back(d); }
  }
  if(e != cudaSuccess) { qmiv_batch_destroy(b); return cuda_fail(e, "batch stream/event creation"); }
  b->pipes.resize(max_pairs);
  b->keys.resize(max_pairs);
  *out_batch = b;
  return QMIV_OK;
}

qmiv_status qmiv_batch_destroy(qmiv_batch b)
{
  if(!b) { return fail(QMIV_ERR_INVALID_ARG, "batch is null"); }
  cudaSetDevice(b->ctx->device);
  if(b->stream) { cudaStreamSynchronize(b->stream); }
  for(cudaStream_t s : b->lanes) { cudaStreamSynchronize(s); cudaStreamDestroy(s); }
  for(cudaEvent_t d : b->lane_done) { cudaEventDestroy(d); }
  if(b->start) { cudaEventDestroy(b->start); }
  b->pipes.clear();
  if(b->stream) { cudaStreamDestroy(b->stream); }
  delete b;
  return QMIV_OK;
}

qmiv_status qmiv_batch_compute(qmiv_batch b, const qmiv_pair_desc* pairs, int32_t n, qmiv_result* out)
{
  if(!b || (!pairs && n > 0) || !out) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  if(n > b->max_pairs) { return fail(QMIV_ERR_INVALID_ARG, "more pairs than max_pairs"); }
  int64_t px = 0;
  for(int i = 0; i < n; i++) { px += (int64_t)pairs[i].width * pairs[i].height; }
  if(px > b->max_pixels) { return fail(QMIV_ERR_INVALID_ARG, "more pixels than max_pixels"); }
  QMIV_CUDA(cudaSetDevice(b->ctx->device));
  // fork: every lane starts after the work already queued on the batch's stream
  QMIV_CUDA(cudaEventRecord(b->start, b->stream));
  for(cudaStream_t s : b->lanes) { QMIV_CUDA(cudaStreamWaitEvent(s, b->start, 0)); }
  for(int i = 0; i < n; i++)
  {
    cudaStream_t lane = b->lanes[i % b->lanes.size()];
    const qmiv_pair_desc& d = pairs[i];
    const auto key = std::make_tuple(d.width, d.height, d.bitdepth, d.chroma_format, d.search_range);
    if(!b->pipes[i] || b->keys[i] != key)
    {
      Shape shape;
      QMIV_TRY(shape.init(d.width, d.height, d.bitdepth, d.chroma_format));
      qmiv_params prm = b->prm; prm.search_range = d.search_range;
      QMIV_TRY(validate_params(prm));
      b->pipes[i].reset(new PairPipeline());
      QMIV_TRY(b->pipes[i]->configure(b->ctx, shape, prm, d.search_range));
      b->keys[i] = key;
    }
    PairPipeline& p = *b->pipes[i];
    const bool host = d.in0.mem == QMIV_MEM_HOST || d.in1.mem == QMIV_MEM_HOST;
    QMIV_TRY(p.prepare(d.metric_mask, false, host));
    Img a{}, c{};
    QMIV_TRY(p.resolve(&d.in0, 0, a, lane));
    QMIV_TRY(p.resolve(&d.in1, 1, c, lane));
    QMIV_TRY(p.enqueue(a, c, d.metric_mask, false, false, lane));
  }
  // join: the batch's stream waits for every lane
  for(size_t k = 0; k < b->lanes.size(); k++)
  {
    QMIV_CUDA(cudaEventRecord(b->lane_done[k], b->lanes[k]));
    QMIV_CUDA(cudaStreamWaitEvent(b->stream, b->lane_done[k], 0));
  }
  QMIV_CUDA(cudaStreamSynchronize(b->stream));
  qmiv_status st = QMIV_OK;
  for(int i = 0; i < n; i++)
  {
    b->pipes[i]->harvest_profile();
    const PairOut& o = b->pipes[i]->host_out();
    finish_result(o, b->pipes[i]->finish_info(pairs[i].metric_mask), &out[i]);
    const qmiv_status ps = pair_status(o, b->prm.invalid_pel_action);
    if(ps != QMIV_OK && st == QMIV_OK) { st = ps; }
  }
  return st;
}

qmiv_status qmiv_batch_stream(qmiv_batch b, void** cuda_stream)
{
  if(!b || !cuda_stream) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  *cuda_stream = (void*)b->stream;
  return QMIV_OK;
}

qmiv_status qmiv_batch_tuning(qmiv_batch b, int32_t width, int32_t height, int32_t bitdepth, int32_t search_range,
                              int32_t* cps_tile_w, int32_t* cps_tile_h, int32_t* cps_rows_per_thread)
{
  if(!b) { return fail(QMIV_ERR_INVALID_ARG, "batch is null"); }
  (void)width; (void)height; (void)bitdepth; (void)search_range;
  if(cps_tile_w) { *cps_tile_w = 32; }
  if(cps_tile_h) { *cps_tile_h = 32; }
  if(cps_rows_per_thread) { *cps_rows_per_thread = 8; }
  return QMIV_OK;
}

}  // extern "C"
