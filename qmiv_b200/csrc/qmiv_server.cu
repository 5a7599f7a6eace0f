// Serving loop (qmiv_server_*): requests (sequences of frame pairs) admitted by HBM budget and
// continuously batched over worker engines.
//
//   submit   validates the request and queues it (rejects one larger than the whole budget)
//   ingest   one thread admits queued requests in arrival order while their resident frames fit the
//            budget (host frames need device copies counted against the context's budget; device
//            frames are used in place), then uploads a request's host frames pair by pair on its own
//            copy stream, outside the scheduler lock, and publishes each pair once its copies have
//            landed; a request that does not fit waits for finished requests to release theirs
//   batch    each worker takes the next landed pairs of all admitted requests, in arrival order,
//            up to max_batch_pairs / max_batch_pixels, and runs them through its own engine
//            (own stream), so two workers keep two launch sequences in flight while the ingest
//            thread keeps the host link busy
//   finish   when a request's last pair is done its resident frames are freed, the sequence means
//            are formed, and waiters are woken
#include "qmiv_engine.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

using namespace qmiv;

namespace {

using Clock = std::chrono::steady_clock;

struct Request
{
  uint64_t     ticket = 0;
  qmiv_request desc{};
  std::vector<qmiv_frame> in0, in1;       // caller frames (or resident copies after admission)
  char*        resident = nullptr;        // device copies of host frames (from the server's memory pool)
  size_t       resident_bytes = 0;        // bytes the request needs there (counted against the budget)
  int32_t      next = 0;                  // next pair to schedule
  int32_t      landed = 0;                // pairs whose frames are in device memory
  int32_t      done = 0;                  // pairs finished
  int32_t      batches = 0;
  bool         admitted = false, finished = false;
  qmiv_status  status = QMIV_OK;
  std::vector<qmiv_result> results;
  double       submit_ms = 0, admit_ms = 0, done_ms = 0;
};

// Neumaier compensated sum in order, then / n (xMetricQMIV.cpp:98-102 with xKBNS.h:36-43)
double seq_mean(const std::vector<qmiv_result>& r, double qmiv_result::*field)
{
  double s = 0.0, c = 0.0;
  for(const qmiv_result& x : r)
  {
    const double v = x.*field;
    const double t = s + v;
    if(std::fabs(s) >= std::fabs(v)) { c += (s - t) + v; } else { c += (v - t) + s; }
    s = t;
  }
  return (s + c) / (double)r.size();
}

}  // namespace

struct qmiv_server_s
{
  qmiv_ctx_s*  ctx = nullptr;
  qmiv_params  prm{};
  int32_t      max_batch_pairs = 0;
  int64_t      max_batch_pixels = 0;
  Clock::time_point t0;
  std::mutex   mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<Request>> queued;      // not admitted yet
  std::vector<std::shared_ptr<Request>> admitted;   // in arrival order
  std::unordered_map<uint64_t, std::shared_ptr<Request>> by_ticket;
  uint64_t     next_ticket = 1;
  bool         stopping = false;
  std::vector<std::unique_ptr<Engine>> engines;
  std::vector<std::thread> workers;
  std::thread  ingest_thread;
  static constexpr int kInFlight = 8;     // pairs whose uploads are in flight at once
  cudaStream_t copy_stream[2] = { nullptr, nullptr };
  cudaEvent_t  copy_event[kInFlight] = {};
  cudaEvent_t  alloc_event = nullptr;     // orders a fresh allocation before the second copy stream
  // Resident frames come from a stream-ordered pool that keeps its memory: allocating and freeing a
  // request's frames never synchronises the device (cudaFree would wait for every worker's kernels).
  cudaMemPool_t pool = nullptr;
  // statistics since the last reset
  std::vector<double> latencies;
  int64_t      pairs_done = 0;
  double       window_start_ms = 0;
  double       last_done_ms = 0;

  double now_ms() const { return std::chrono::duration<double, std::milli>(Clock::now() - t0).count(); }
  void   worker(int w);
  void   ingest();
  // admits the front of the queue; false while the budget is full (mu held)
  bool   admit_front_locked(std::shared_ptr<Request>& out);
  qmiv_status upload_pair(Request& r, const Shape& S, int i, cudaStream_t cs, cudaEvent_t ev);
  // resident memory of a request: budget first, then the pool (ingest thread); release at finish
  qmiv_status alloc_resident(Request& r);
  void        free_resident(Request& r);
};

static size_t frame_device_bytes(const Shape& S) { return 2 * S.staged_frame_bytes(); }

// Admits the front of the queue: allocates its resident frames if it has host frames. Returns false
// (and admits nothing) while the budget is full and admitted requests will still release memory.
bool qmiv_server_s::admit_front_locked(std::shared_ptr<Request>& out)
{
  std::shared_ptr<Request> r = queued.front();
  if(r->resident_bytes > 0 && alloc_resident(*r) != QMIV_OK)
  {
    bool busy = false;
    for(auto& a : admitted) { busy = busy || !a->finished; }
    if(busy) { return false; }   // budget full: wait for admitted requests to free memory, keep the order
    // nothing admitted will free memory: the request cannot fit beside the engines' working memory
    r->status = fail(QMIV_ERR_BUDGET, "request frames do not fit the HBM budget beside the engines' working memory");
    r->resident_bytes = 0;
  }
  queued.pop_front();
  r->admitted = true;
  r->admit_ms = now_ms();
  if(r->resident_bytes == 0) { r->landed = r->desc.num_pairs; }   // device frames, or failed: nothing to upload
  admitted.push_back(r);
  out = r;
  return true;
}

qmiv_status qmiv_server_s::alloc_resident(Request& r)
{
  if(!ctx->reserve(r.resident_bytes)) { return fail(QMIV_ERR_BUDGET, "HBM budget exceeded"); }
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, r.resident_bytes, pool, copy_stream[0]);
  if(e == cudaSuccess) { e = cudaEventRecord(alloc_event, copy_stream[0]); }
  if(e == cudaSuccess) { e = cudaStreamWaitEvent(copy_stream[1], alloc_event, 0); }
  if(e != cudaSuccess)
  {
    if(p) { cudaFreeAsync(p, copy_stream[0]); }
    cudaGetLastError();
    ctx->unreserve(r.resident_bytes);
    return cuda_fail(e, "server frame memory");
  }
  r.resident = static_cast<char*>(p);
  return QMIV_OK;
}

// Called when every pair of the request is done (the workers' engines have synchronised their
// streams), so the memory is free for the next allocation in copy-stream order.
void qmiv_server_s::free_resident(Request& r)
{
  if(r.resident)
  {
    cudaFreeAsync(r.resident, copy_stream[0]);
    ctx->unreserve(r.resident_bytes);
    r.resident = nullptr;
  }
}

// Enqueues the copies of pair i's host frames into the request's resident memory on copy stream `cs`
// and records `ev` after them. Frame descriptors are rewritten to the device copies, which workers
// read only once the pair is published.
qmiv_status qmiv_server_s::upload_pair(Request& r, const Shape& S, int i, cudaStream_t cs, cudaEvent_t ev)
{
  char* base = r.resident;
  for(int f = 0; f < 2; f++)
  {
    qmiv_frame& fr = f ? r.in1[i] : r.in0[i];
    if(fr.mem != QMIV_MEM_HOST) { continue; }
    size_t off = ((size_t)i * 2 + f) * S.staged_frame_bytes();
    for(int c = 0; c < 3; c++)
    {
      char* dst = base + off;
      const size_t row = S.plane_cols(c) * S.esz;
      QMIV_CUDA(cudaMemcpy2DAsync(dst, S.staged_pitch(c), fr.plane[c], (size_t)fr.pitch[c], row, S.plane_rows(c),
                                  cudaMemcpyHostToDevice, cs));
      fr.plane[c] = dst;
      fr.pitch[c] = (int64_t)S.staged_pitch(c);
      off += S.staged_plane_bytes(c);
    }
    fr.mem = QMIV_MEM_DEVICE;
  }
  QMIV_CUDA(cudaEventRecord(ev, cs));
  return QMIV_OK;
}

// Admission and upload thread. Up to kInFlight pairs, across request boundaries, have their copies
// in flight, alternating between two copy streams (both copy engines busy); pairs are published in
// order as their copies land.
void qmiv_server_s::ingest()
{
  cudaSetDevice(ctx->device);
  struct Flight
  {
    std::shared_ptr<Request> r;
    int                      i;
    cudaEvent_t              ev;
  };
  std::deque<Flight> flight;
  std::vector<cudaEvent_t> free_ev(copy_event, copy_event + kInFlight);
  std::shared_ptr<Request> cur;     // the admitted request whose pairs are being issued
  Shape S;
  int next_pair = 0;
  uint64_t issued = 0;
  // publishes the oldest pair in flight once its copies have landed
  auto retire = [&]() {
    Flight f = flight.front();
    flight.pop_front();
    const cudaError_t e = cudaEventSynchronize(f.ev);
    free_ev.push_back(f.ev);
    {
      std::lock_guard<std::mutex> lk(mu);
      if(e != cudaSuccess && f.r->status == QMIV_OK) { f.r->status = cuda_fail(e, "server frame upload"); }
      f.r->landed = std::max(f.r->landed, f.i + 1);
    }
    cv_work.notify_all();
  };
  for(;;)
  {
    if(!cur)
    {
      std::unique_lock<std::mutex> lk(mu);
      if(queued.empty())
      {
        if(!flight.empty()) { lk.unlock(); retire(); continue; }
        if(stopping) { return; }
        cv_work.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
      std::shared_ptr<Request> r;
      if(!admit_front_locked(r))
      {
        if(!flight.empty()) { lk.unlock(); retire(); continue; }
        cv_done.wait_for(lk, std::chrono::milliseconds(2));   // a finishing request releases memory
        continue;
      }
      lk.unlock();
      cv_work.notify_all();
      if(r->landed == r->desc.num_pairs) { continue; }     // nothing to upload
      cur = r;
      S.init(r->desc.width, r->desc.height, r->desc.bitdepth, r->desc.chroma_format);
      next_pair = 0;
    }
    if(flight.size() == (size_t)kInFlight) { retire(); continue; }
    cudaEvent_t ev = free_ev.back();
    free_ev.pop_back();
    const qmiv_status st = upload_pair(*cur, S, next_pair, copy_stream[issued++ & 1], ev);
    if(st != QMIV_OK)
    {
      // the pairs in flight land first; then the request is failed and marked fully landed
      free_ev.push_back(ev);
      while(!flight.empty()) { retire(); }
      {
        std::lock_guard<std::mutex> lk(mu);
        if(cur->status == QMIV_OK) { cur->status = st; }
        cur->landed = cur->desc.num_pairs;
      }
      cv_work.notify_all();
      cur.reset();
      continue;
    }
    flight.push_back(Flight{ cur, next_pair, ev });
    if(++next_pair == cur->desc.num_pairs) { cur.reset(); }
  }
}

void qmiv_server_s::worker(int w)
{
  cudaSetDevice(ctx->device);
  Engine& eng = *engines[w];
  std::vector<qmiv_pair_desc> descs;
  std::vector<std::pair<std::shared_ptr<Request>, int>> owners;
  std::vector<qmiv_result> out;
  for(;;)
  {
    descs.clear();
    owners.clear();
    {
      std::unique_lock<std::mutex> lk(mu);
      for(;;)
      {
        // next landed pairs of the admitted requests, in arrival order
        int64_t px = 0;
        for(auto& r : admitted)
        {
          if(r->status != QMIV_OK) { continue; }
          const int64_t ppx = (int64_t)r->desc.width * r->desc.height;
          bool counted = false;
          while(r->next < r->landed && (int)descs.size() < max_batch_pairs && px + ppx <= max_batch_pixels)
          {
            qmiv_pair_desc d{};
            d.in0 = r->in0[r->next]; d.in1 = r->in1[r->next];
            d.width = r->desc.width; d.height = r->desc.height; d.bitdepth = r->desc.bitdepth;
            d.chroma_format = r->desc.chroma_format; d.search_range = r->desc.search_range; d.metric_mask = r->desc.metric_mask;
            descs.push_back(d);
            owners.emplace_back(r, r->next);
            r->next++;
            px += ppx;
            if(!counted) { r->batches++; counted = true; }
          }
          if((int)descs.size() >= max_batch_pairs) { break; }
        }
        // requests that failed at admission or upload finish without running (once no pair of
        // theirs is still running on a worker)
        for(auto& r : admitted)
        {
          if(r->status != QMIV_OK && !r->finished && r->landed == r->desc.num_pairs && r->done == r->next)
          {
            r->finished = true;
            r->done_ms = now_ms();
            free_resident(*r);
            cv_done.notify_all();
          }
        }
        if(!descs.empty()) { break; }
        if(stopping && queued.empty())
        {
          bool busy = false;
          for(auto& r : admitted) { busy = busy || !r->finished; }
          if(!busy) { return; }
        }
        cv_work.wait_for(lk, std::chrono::milliseconds(1));
      }
    }
    out.assign(descs.size(), qmiv_result{});
    const qmiv_status st = eng.run(descs.data(), (int32_t)descs.size(), out.data());
    {
      std::lock_guard<std::mutex> lk(mu);
      const double t = now_ms();
      for(size_t k = 0; k < owners.size(); k++)
      {
        Request& r = *owners[k].first;
        r.results[owners[k].second] = out[k];
        if(st != QMIV_OK && r.status == QMIV_OK) { r.status = st; }
        r.done++;
        pairs_done++;
        if(r.done == r.desc.num_pairs && !r.finished)
        {
          r.finished = true;
          r.done_ms = t;
          free_resident(r);
          latencies.push_back(r.done_ms - r.submit_ms);
          last_done_ms = t;
        }
      }
      // drop finished requests from the admitted list (their tickets stay until waited on)
      std::vector<std::shared_ptr<Request>> keep;
      for(auto& r : admitted) { if(!r->finished) { keep.push_back(r); } }
      admitted.swap(keep);
    }
    cv_done.notify_all();
    cv_work.notify_all();
  }
}

extern "C" {

qmiv_status qmiv_server_create(qmiv_ctx ctx, const qmiv_params* params, int32_t max_batch_pairs, int64_t max_batch_pixels,
                               int32_t workers, qmiv_server* out_server)
{
  if(!ctx || !out_server || max_batch_pairs <= 0 || max_batch_pixels <= 0 || workers < 1 || workers > 4)
  {
    return fail(QMIV_ERR_INVALID_ARG, "bad server arguments");
  }
  *out_server = nullptr;
  qmiv_params prm;
  if(params) { prm = *params; } else { qmiv_params_default(&prm); }
  QMIV_TRY(validate_params(prm));
  std::unique_ptr<qmiv_server_s> s(new qmiv_server_s());
  s->ctx = ctx; s->prm = prm; s->max_batch_pairs = max_batch_pairs; s->max_batch_pixels = max_batch_pixels;
  s->t0 = Clock::now();
  for(int w = 0; w < workers; w++)
  {
    s->engines.emplace_back(new Engine());
    QMIV_TRY(s->engines.back()->init(ctx, prm, max_batch_pairs, max_batch_pixels, QMIV_BATCH_GRAPH | QMIV_BATCH_AUTOTUNE));
  }
  QMIV_CUDA(cudaSetDevice(ctx->device));
  for(int k = 0; k < 2; k++) { QMIV_CUDA(cudaStreamCreateWithFlags(&s->copy_stream[k], cudaStreamNonBlocking)); }
  for(int k = 0; k < qmiv_server_s::kInFlight; k++) { QMIV_CUDA(cudaEventCreateWithFlags(&s->copy_event[k], cudaEventDisableTiming)); }
  QMIV_CUDA(cudaEventCreateWithFlags(&s->alloc_event, cudaEventDisableTiming));
  cudaMemPoolProps pp{};
  pp.allocType = cudaMemAllocationTypePinned;
  pp.location.type = cudaMemLocationTypeDevice;
  pp.location.id = ctx->device;
  QMIV_CUDA(cudaMemPoolCreate(&s->pool, &pp));
  uint64_t keep = UINT64_MAX;   // the pool keeps what it has reserved: no release to the driver between requests
  QMIV_CUDA(cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep));
  qmiv_server_s* sp = s.get();
  for(int w = 0; w < workers; w++) { s->workers.emplace_back([sp, w] { sp->worker(w); }); }
  s->ingest_thread = std::thread([sp] { sp->ingest(); });
  *out_server = s.release();
  return QMIV_OK;
}

qmiv_status qmiv_server_destroy(qmiv_server s)
{
  if(!s) { return fail(QMIV_ERR_INVALID_ARG, "server is null"); }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  if(s->ingest_thread.joinable()) { s->ingest_thread.join(); }
  for(std::thread& t : s->workers) { t.join(); }
  for(auto& kv : s->by_ticket) { s->free_resident(*kv.second); }   // requests never waited on
  if(s->copy_stream[0]) { cudaStreamSynchronize(s->copy_stream[0]); }
  if(s->pool) { cudaMemPoolDestroy(s->pool); }
  if(s->alloc_event) { cudaEventDestroy(s->alloc_event); }
  for(int k = 0; k < qmiv_server_s::kInFlight; k++) { if(s->copy_event[k]) { cudaEventDestroy(s->copy_event[k]); } }
  for(int k = 0; k < 2; k++) { if(s->copy_stream[k]) { cudaStreamDestroy(s->copy_stream[k]); } }
  delete s;
  return QMIV_OK;
}

qmiv_status qmiv_server_submit(qmiv_server s, const qmiv_request* req, uint64_t* ticket)
{
  if(!s || !req || !ticket) { return fail(QMIV_ERR_INVALID_ARG, "null argument"); }
  if(req->num_pairs <= 0 || !req->in0 || !req->in1) { return fail(QMIV_ERR_INVALID_ARG, "a request needs at least one pair"); }
  if((req->metric_mask & ~(uint32_t)QMIV_ALL) != 0) { return fail(QMIV_ERR_INVALID_ARG, "unknown metric bits"); }
  if((int64_t)req->width * req->height > s->max_batch_pixels) { return fail(QMIV_ERR_INVALID_ARG, "picture larger than max_batch_pixels"); }
  Shape S;
  QMIV_TRY(S.init(req->width, req->height, req->bitdepth, req->chroma_format));
  qmiv_params p = s->prm;
  p.search_range = req->search_range;
  QMIV_TRY(validate_params(p));
  QMIV_TRY(check_metrics(S, req->metric_mask, p));
  std::shared_ptr<Request> r(new Request());
  r->desc = *req;
  r->in0.assign(req->in0, req->in0 + req->num_pairs);
  r->in1.assign(req->in1, req->in1 + req->num_pairs);
  size_t host_frames = 0;
  for(int i = 0; i < req->num_pairs; i++)
  {
    if(r->in0[i].mem == QMIV_MEM_HOST || r->in1[i].mem == QMIV_MEM_HOST) { host_frames++; }
  }
  // resident copies: a full pair slot for every pair with a host frame
  r->resident_bytes = host_frames ? (size_t)req->num_pairs * frame_device_bytes(S) : 0;
  uint64_t used = 0, budget = 0;
  qmiv_ctx_memory(s->ctx, &used, &budget);
  if(budget != 0 && r->resident_bytes > budget) { return fail(QMIV_ERR_BUDGET, "request larger than the whole HBM budget"); }
  r->results.assign(req->num_pairs, qmiv_result{});
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if(s->stopping) { return fail(QMIV_ERR_INVALID_ARG, "server is stopping"); }
    r->ticket = s->next_ticket++;
    r->submit_ms = s->now_ms();
    s->queued.push_back(r);
    s->by_ticket[r->ticket] = r;
    *ticket = r->ticket;
  }
  s->cv_work.notify_all();
  return QMIV_OK;
}

qmiv_status qmiv_server_wait(qmiv_server s, uint64_t ticket, int32_t timeout_ms, qmiv_result* results,
                             qmiv_request_stats* stats)
{
  if(!s) { return fail(QMIV_ERR_INVALID_ARG, "server is null"); }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->by_ticket.find(ticket);
  if(it == s->by_ticket.end()) { return fail(QMIV_ERR_INVALID_ARG, "unknown ticket"); }
  std::shared_ptr<Request> r = it->second;
  auto ready = [&] { return r->finished; };
  if(timeout_ms < 0) { s->cv_done.wait(lk, ready); }
  else if(!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
  {
    return fail(QMIV_ERR_TIMEOUT, "request not finished within the timeout");
  }
  s->by_ticket.erase(it);
  if(results) { for(int i = 0; i < r->desc.num_pairs; i++) { results[i] = r->results[i]; } }
  if(stats)
  {
    qmiv_request_stats& st = *stats;
    st.submit_ms = r->submit_ms; st.admit_ms = r->admit_ms; st.done_ms = r->done_ms;
    st.latency_ms = r->done_ms - r->submit_ms;
    st.batches = r->batches;
    st.mean_psnr_pic = seq_mean(r->results, &qmiv_result::psnr_pic);
    st.mean_wspsnr_pic = seq_mean(r->results, &qmiv_result::wspsnr_pic);
    st.mean_ivpsnr = seq_mean(r->results, &qmiv_result::ivpsnr);
    st.mean_ssim_pic = seq_mean(r->results, &qmiv_result::ssim_pic);
    st.mean_msssim_pic = seq_mean(r->results, &qmiv_result::msssim_pic);
    st.mean_ivssim = seq_mean(r->results, &qmiv_result::ivssim);
    st.mean_ivmsssim = seq_mean(r->results, &qmiv_result::ivmsssim);
  }
  return r->status;
}

qmiv_status qmiv_server_stats(qmiv_server s, double* p50_ms, double* p99_ms, double* pairs_per_s,
                              int64_t* completed_requests, int32_t reset)
{
  if(!s) { return fail(QMIV_ERR_INVALID_ARG, "server is null"); }
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> l = s->latencies;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) -> double {
    if(l.empty()) { return 0.0; }
    size_t k = (size_t)std::ceil(q * (double)l.size());   // nearest rank
    k = k == 0 ? 0 : k - 1;
    return l[std::min(k, l.size() - 1)];
  };
  if(p50_ms) { *p50_ms = pct(0.50); }
  if(p99_ms) { *p99_ms = pct(0.99); }
  const double span = s->last_done_ms - s->window_start_ms;
  if(pairs_per_s) { *pairs_per_s = span > 0 ? (double)s->pairs_done / (span / 1e3) : 0.0; }
  if(completed_requests) { *completed_requests = (int64_t)l.size(); }
  if(reset)
  {
    s->latencies.clear();
    s->pairs_done = 0;
    s->window_start_ms = s->now_ms();
    s->last_done_ms = s->window_start_ms;
  }
  return QMIV_OK;
}

}  // extern "C"
