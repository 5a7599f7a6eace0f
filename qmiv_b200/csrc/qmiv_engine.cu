// Batched form: many frame pairs of uneven size, bit depth, search range and metric set per call,
// every stage of the pipeline one launch for all pairs.
//
//   descriptors   one host-to-device copy of every pair's argument blocks (tensor maps included)
//   prepass       one launch per sample size, a CTA row per pair          (k_prepass_multi)
//   reduce        one CTA per pair                                        (k_reduce_multi)
//   CPS           one persistent launch per (R, sample size, tile height) over a work list of the
//                 tiles of all its pairs                                   (k_cps_multi)
//   SSIM          per scale: moments of all pairs, then every window row of every (pair, component)
//   finalize      one CTA per (pair, pooling chain)                       (k_finalize_multi)
//   results       one device-to-host copy of all pairs' PairOut
//
// Host frames are uploaded on two copy streams in sub-batches of about kChunkBytes; each sub-batch's
// stages start as soon as its frames have landed, so uploads overlap compute.
// With QMIV_BATCH_GRAPH (device frames) the launch sequence, descriptor copy to result copy, is
// captured once per call signature (the pairs' shapes, search ranges and metric sets) and replayed;
// frame addresses travel in the descriptors, so a replay only rewrites the pinned descriptor mirror.
// With QMIV_BATCH_AUTOTUNE the CPS tile height of every (W, H, bit depth, R) is picked by timing the
// candidate kernels on the first pair of that kind; qmiv_batch_tuning reports the choice.
#include "qmiv_engine.h"

#include <algorithm>
#include <cassert>
#include <cmath>
#include <cstdio>
#include <cstring>

namespace qmiv {

namespace {

constexpr size_t kRegionAlign = 256;
constexpr size_t kChunkBytes = 64u << 20;   // host frames uploaded per sub-batch
inline size_t align_sz(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Img of a planar 4:4:4 picture of W x H samples at base
Img img444(const void* base, int32_t W, int32_t H, size_t esz)
{
  Img im{};
  for(int c = 0; c < 3; c++)
  {
    im.p[c] = static_cast<const char*>(base) + (size_t)c * W * H * esz;
    im.pitch[c] = W; im.sx[c] = 0; im.sy[c] = 0;
  }
  return im;
}
MutImg mut444(void* base, int32_t W, int32_t H, size_t esz)
{
  MutImg im{};
  for(int c = 0; c < 3; c++) { im.p[c] = static_cast<char*>(base) + (size_t)c * W * H * esz; im.pitch[c] = W; }
  return im;
}

}  // namespace

// ---------------------------------------------------------------------------------------------
// kinds and the autotuner
// ---------------------------------------------------------------------------------------------
qmiv_status Engine::kind_for(const qmiv_pair_desc& d, PairKind*& out)
{
  const KindKey key{ d.width, d.height, d.bitdepth, d.chroma_format, d.search_range };
  auto it = kinds_.find(key);
  if(it != kinds_.end()) { out = it->second.get(); return QMIV_OK; }
  std::unique_ptr<PairKind> k(new PairKind());
  QMIV_TRY(k->S.init(d.width, d.height, d.bitdepth, d.chroma_format));
  k->prm = prm_;
  k->prm.search_range = d.search_range;
  QMIV_TRY(validate_params(k->prm));
  k->R = d.search_range;
  for(int c = 0; c < 4; c++) { k->maxdiff[c] = round_f32_half_away(prm_.unc[c] * (float)k->S.maxv); }  // xGlobClrDiff.cpp:76
  k->fp32_ok = cps_fp32_exact(k->S.maxv, prm_.cws, k->maxdiff);
  k->ns = num_scales(k->S.W, k->S.H);
  int32_t w = k->S.W, h = k->S.H;
  for(int s = 0; s < 5; s++)
  {
    k->nx[s] = w >= 8 ? (w - 8) / 4 + 1 : 0;  // xSSIM::xCalcNumBlocks for 8/4
    k->ny[s] = h >= 8 ? (h - 8) / 4 + 1 : 0;
    w >>= 1; h >>= 1;
  }
  const double maxd = (double)k->S.maxv;  // xSSIM.cpp:165-167
  const double k1 = 0.01 * maxd, k2 = 0.03 * maxd;
  k->C1 = k1 * k1;
  k->C2 = k2 * k2;
  if(prm_.erp)
  {
    ws_weights(k->S.H, prm_.lat_range_deg, k->ws_host, k->ws_corr);
    QMIV_TRY(k->ws_dev.alloc(ctx_, (size_t)k->S.H * sizeof(double)));
    QMIV_CUDA(cudaMemcpy(k->ws_dev.p, k->ws_host.data(), k->S.H * sizeof(double), cudaMemcpyHostToDevice));
  }
  k->wy = cps_pick_wy(k->R, (int)k->S.esz, k->S.sx, k->S.sy);
  if(k->wy == 0) { return fail(QMIV_ERR_UNSUPPORTED, "no CPS tile shape fits shared memory for this search range"); }
  out = k.get();
  kinds_[key] = std::move(k);
  return QMIV_OK;
}

// Times the candidate CPS tile shapes (128 x 32 with 16 warps, 128 x 24 with 12, 128 x 16 with 8 at
// two CTAs per SM; those that fit shared memory) on one real pair of the kind (GCD 0, results
// discarded) and keeps the fastest. The candidates take turns over several rounds and each keeps its
// fastest launch, so a clock ramp or another stream's burst during one round does not decide.
qmiv_status Engine::autotune(PairKind& k, const Img& in0, const Img& in1, cudaStream_t s)
{
  k.tuned = true;
  constexpr int kCands = 3, kRounds = 5;
  const int cands[kCands] = { 8, 6, 4 };
  int wys[kCands], n = 0;
  for(int c = 0; c < kCands; c++)
  {
    if(cps_tile_fits(k.R, cands[c], (int)k.S.esz, k.S.sx, k.S.sy)) { wys[n++] = cands[c]; }
  }
  if(n < 2) { return QMIV_OK; }   // one candidate only: nothing to tune
  const Shape& S = k.S;
  const size_t out_b = align_sz(sizeof(PairOut), kRegionAlign);
  const size_t rows_b = align_sz((size_t)2 * S.H * 3 * sizeof(uint32_t), kRegionAlign);
  const size_t desc_b = align_sz(cps_desc_bytes(), kRegionAlign);
  QMIV_TRY(tune_scratch_.ensure(ctx_, out_b + rows_b + kCands * (desc_b + kRegionAlign)));
  char* base = tune_scratch_.as<char>();
  PairOut* dout = reinterpret_cast<PairOut*>(base);
  uint32_t* rows = reinterpret_cast<uint32_t*>(base + out_b);
  QMIV_CUDA(cudaMemsetAsync(base, 0, out_b + rows_b, s));
  CpsArgs ca{};
  ca.in0 = in0; ca.in1 = in1; ca.W = S.W; ca.H = S.H; ca.maxv = S.maxv; ca.clip = 0xffffu;
  for(int c = 0; c < 3; c++) { ca.wi[c] = prm_.cws[c]; ca.wf[c] = (float)prm_.cws[c]; }
  ca.gcd_src = dout; ca.rows = rows;
  alignas(64) static thread_local unsigned char host_desc[4096];
  if(cps_desc_bytes() > sizeof(host_desc)) { return QMIV_OK; }
  CpsPairPlan plan[kCands]{};
  void* ddesc[kCands];
  int32_t* dprefix[kCands];
  bool ok[kCands] = {};
  for(int c = 0; c < n; c++)
  {
    ddesc[c] = base + out_b + rows_b + c * (desc_b + kRegionAlign);
    dprefix[c] = reinterpret_cast<int32_t*>(static_cast<char*>(ddesc[c]) + desc_b);
    if(cps_describe(host_desc, ca, k.R, (int)S.esz, wys[c], &plan[c]) != cudaSuccess) { continue; }
    const int32_t prefix[2] = { 0, plan[c].ntiles };
    QMIV_CUDA(cudaMemcpyAsync(ddesc[c], host_desc, cps_desc_bytes(), cudaMemcpyHostToDevice, s));
    QMIV_CUDA(cudaMemcpyAsync(dprefix[c], prefix, sizeof(prefix), cudaMemcpyHostToDevice, s));
    QMIV_CUDA(cudaStreamSynchronize(s));   // host_desc is reused for the next candidate
    ok[c] = true;
  }
  cudaEvent_t e0, e1;
  QMIV_CUDA(cudaEventCreate(&e0));
  QMIV_CUDA(cudaEventCreate(&e1));
  float best_ms[kCands];
  for(int c = 0; c < kCands; c++) { best_ms[c] = 1e30f; }
  cudaError_t e = cudaSuccess;
  for(int round = 0; round <= kRounds && e == cudaSuccess; round++)   // round 0 warms every candidate up
  {
    for(int c = 0; c < n && e == cudaSuccess; c++)
    {
      if(!ok[c]) { continue; }
      e = cudaEventRecord(e0, s);
      if(e == cudaSuccess) { e = launch_cps_multi(ddesc[c], dprefix[c], 1, plan[c].ntiles, k.R, wys[c], (int)S.esz, plan[c].raw_bytes, plan[c].smem, s); }
      if(e == cudaSuccess) { e = cudaEventRecord(e1, s); }
      if(e == cudaSuccess) { e = cudaEventSynchronize(e1); }
      if(e == cudaSuccess && round > 0)
      {
        float t = 0.f;
        cudaEventElapsedTime(&t, e0, e1);
        best_ms[c] = std::min(best_ms[c], t);
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if(e != cudaSuccess) { return cuda_fail(e, "CPS autotuning launch"); }
  int best = -1;
  for(int c = 0; c < n; c++)
  {
    for(int q = 0; q < kCands; q++) { if(cands[q] == wys[c]) { k.tune_ms[q] = ok[c] ? best_ms[c] : 0.f; } }
    if(ok[c] && (best < 0 || best_ms[c] < best_ms[best])) { best = c; }
  }
  if(best >= 0) { k.wy = wys[best]; }
  return QMIV_OK;
}

// ---------------------------------------------------------------------------------------------
// life cycle
// ---------------------------------------------------------------------------------------------
qmiv_status Engine::init(qmiv_ctx_s* ctx, const qmiv_params& prm, int32_t max_pairs, int64_t max_pixels, int32_t flags)
{
  ctx_ = ctx; prm_ = prm; max_pairs_ = max_pairs; max_pixels_ = max_pixels; flags_ = flags;
  QMIV_CUDA(cudaSetDevice(ctx->device));
  QMIV_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  return QMIV_OK;
}

Engine::~Engine()
{
  if(ctx_) { cudaSetDevice(ctx_->device); }
  if(stream_) { cudaStreamSynchronize(stream_); }
  for(cudaStream_t cs : copy_stream_)
  {
    if(cs) { cudaStreamSynchronize(cs); cudaStreamDestroy(cs); }
  }
  for(cudaEvent_t e : chunk_ready_) { cudaEventDestroy(e); }
  clear_graphs();
  if(host_mirror_) { cudaFreeHost(host_mirror_); }
  if(host_out_) { cudaFreeHost(host_out_); }
  if(stream_) { cudaStreamDestroy(stream_); }
}

void Engine::clear_graphs()
{
  for(auto& g : graphs_) { if(g.second) { cudaGraphExecDestroy(g.second); } }
  graphs_.clear();
}

qmiv_status Engine::ensure_host(size_t mirror_bytes, int n)
{
  if(mirror_bytes > host_mirror_bytes_)
  {
    if(host_mirror_) { cudaFreeHost(host_mirror_); host_mirror_ = nullptr; }
    const size_t b = std::max(mirror_bytes, host_mirror_bytes_ * 2);
    QMIV_CUDA(cudaMallocHost(&host_mirror_, b));
    host_mirror_bytes_ = b;
    clear_graphs();
  }
  if(n > host_out_n_)
  {
    if(host_out_) { cudaFreeHost(host_out_); host_out_ = nullptr; }
    QMIV_CUDA(cudaMallocHost((void**)&host_out_, sizeof(PairOut) * (size_t)n));
    host_out_n_ = n;
    clear_graphs();
  }
  return QMIV_OK;
}

// ---------------------------------------------------------------------------------------------
// one call
// ---------------------------------------------------------------------------------------------
qmiv_status Engine::run(const qmiv_pair_desc* pairs, int32_t n, qmiv_result* results)
{
  QMIV_TRY(submit(pairs, n));
  return collect(results);
}

qmiv_status Engine::submit(const qmiv_pair_desc* pairs, int32_t n)
{
  if(pend_n_ >= 0) { return fail(QMIV_ERR_BUSY, "the engine has a call in flight"); }
  if(!pairs && n > 0) { return fail(QMIV_ERR_INVALID_ARG, "null pairs"); }
  if(n > max_pairs_) { return fail(QMIV_ERR_INVALID_ARG, "more pairs than max_pairs"); }
  int64_t px = 0;
  for(int i = 0; i < n; i++) { px += (int64_t)pairs[i].width * pairs[i].height; }
  if(px > max_pixels_) { return fail(QMIV_ERR_INVALID_ARG, "more pixels than max_pixels"); }
  if(n == 0) { pend_n_ = 0; return QMIV_OK; }
  QMIV_CUDA(cudaSetDevice(ctx_->device));
  cudaStream_t s = stream_;

  // ---- per-pair kinds, masks, arena layout ---------------------------------------------------
  std::vector<PairKind*> kind(n);
  std::vector<int> gen_idx;
  std::vector<PairSlot>& P = slots_;
  P.assign(n, PairSlot{});
  std::string sig;
  size_t arena = 0;
  auto take = [&](size_t bytes) { const size_t o = arena; arena += align_sz(bytes, kRegionAlign); return o; };
  // zeroed region first: all PairOut, then all CPS row sums
  const size_t outs_off = take(sizeof(PairOut) * (size_t)n);
  for(int i = 0; i < n; i++)
  {
    const qmiv_pair_desc& d = pairs[i];
    QMIV_TRY(kind_for(d, kind[i]));
    QMIV_TRY(check_metrics(kind[i]->S, d.metric_mask, prm_));
    PairSlot& p = P[i];
    const Shape& S = kind[i]->S;
    p.mask = d.metric_mask;
    if(!ssim_is_default(prm_) && (p.mask & kSsimFamily))
    {
      int32_t f, nx, ny;
      ssim_line(prm_, S.W, f, nx);
      ssim_line(prm_, S.H, f, ny);
      if(S.W < ssim_window_size(prm_) || S.H < ssim_window_size(prm_) || nx < 1 || ny < 1)
      {
        return fail(QMIV_ERR_INVALID_ARG, "picture smaller than one SSIM window");
      }
      gen_idx.push_back(i);
      p.mask &= ~kSsimFamily;
    }
    p.need_scp = (p.mask & QMIV_IVMSSSIM) != 0;
    p.need_search = p.need_scp || (p.mask & (QMIV_IVPSNR | QMIV_IVSSIM));
    p.need_ssim = (p.mask & (QMIV_SSIM | QMIV_MSSSIM | QMIV_IVSSIM | QMIV_IVMSSSIM)) != 0;
    p.need_ms = (p.mask & (QMIV_MSSSIM | QMIV_IVMSSSIM)) != 0;
    p.host = d.in0.mem == QMIV_MEM_HOST || d.in1.mem == QMIV_MEM_HOST;
    if(p.need_ssim && (kind[i]->nx[0] < 1 || kind[i]->ny[0] < 1)) { return fail(QMIV_ERR_INVALID_ARG, "picture smaller than one 8x8 SSIM window"); }
    if(p.need_ms && kind[i]->ns < 1) { return fail(QMIV_ERR_INVALID_ARG, "picture too small for MS-SSIM (needs >= 32x32)"); }
    p.out = outs_off + sizeof(PairOut) * (size_t)i;
    char k[96];
    std::snprintf(k, sizeof(k), "%d,%d,%d,%d,%d,%u,%d;", S.W, S.H, S.bitdepth, S.chroma_format, kind[i]->R, p.mask, p.host ? 1 : 0);
    sig += k;
  }
  for(int i = 0; i < n; i++)
  {
    if(P[i].need_search) { P[i].cps_rows = take((size_t)2 * kind[i]->S.H * 3 * sizeof(uint32_t)); }
  }
  const size_t zero_bytes = arena;
  for(int i = 0; i < n; i++)
  {
    PairSlot& p = P[i];
    const PairKind& K = *kind[i];
    const Shape& S = K.S;
    const size_t rows_total = (size_t)S.H + 2 * (size_t)S.ch;
    p.row_sd = take(rows_total * sizeof(int64_t));
    p.row_ssd = take(rows_total * sizeof(uint64_t));
    if(p.need_scp) { p.scp = take((size_t)2 * 3 * S.W * S.H * S.esz); }
    if(p.need_ssim)
    {
      const int slots = (p.mask & QMIV_IVMSSSIM) ? 5 : (p.mask & (QMIV_SSIM | QMIV_MSSSIM)) ? 3 : 2;
      p.mom_slot = mom_slot_elems(S);
      p.mom = take((size_t)slots * p.mom_slot * sizeof(uint32_t));
      p.rowsum = take((size_t)kMaxSsimSlots * 3 * K.ny[0] * sizeof(double));
      // window values of the pair's scale-0 pool jobs, reused by the MS-SSIM scales
      const int jobs0 = 3 * (((p.mask & QMIV_IVSSIM) ? 2 : 0) + ((p.mask & QMIV_SSIM) ? 1 : 0) +
                             ((p.mask & QMIV_MSSSIM) ? 1 : 0) + ((p.mask & QMIV_IVMSSSIM) ? 2 : 0));
      p.win = take((size_t)jobs0 * pool_win_elems(K.nx[0], K.ny[0]) * sizeof(double));
    }
    if(p.need_ms)
    {
      size_t lv = 0;
      for(int s2 = 1; s2 < K.ns; s2++) { lv += (size_t)(S.W >> s2) * (S.H >> s2) * 3; }
      p.pyr_lv = lv;
      p.pyr = take(4 * lv * S.esz);
    }
    if(p.host) { p.staging = take(2 * S.staged_frame_bytes()); }
  }
  if(arena > arena_.bytes)
  {
    QMIV_CUDA(cudaStreamSynchronize(s));
    clear_graphs();
    QMIV_TRY(arena_.alloc(ctx_, std::max(arena, arena_.bytes + arena_.bytes / 2)));
  }
  char* dbase = arena_.as<char>();
  PairOut* douts = reinterpret_cast<PairOut*>(dbase + outs_off);

  // ---- sub-batches: with host frames the pairs are cut into sub-batches of about kChunkBytes of
  // frames whose stages start when their uploads have landed; device frames: one sub-batch -------
  bool any_host = false;
  for(int i = 0; i < n; i++) { any_host = any_host || P[i].host; }
  std::vector<std::pair<int, int>> chunks;  // (first pair, pairs)
  if(any_host)
  {
    int first = 0;
    size_t bytes = 0;
    for(int i = 0; i < n; i++)
    {
      bytes += 2 * kind[i]->S.frame_bytes();
      if(bytes >= kChunkBytes || i == n - 1) { chunks.emplace_back(first, i + 1 - first); first = i + 1; bytes = 0; }
    }
    for(cudaStream_t& cs : copy_stream_)
    {
      if(!cs) { QMIV_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)); }
    }
    while(chunk_ready_.size() < chunks.size())
    {
      cudaEvent_t e;
      QMIV_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      chunk_ready_.push_back(e);
    }
  }
  else { chunks.emplace_back(0, n); }

  // ---- frames ----------------------------------------------------------------------------------
  std::vector<Img> in0(n), in1(n);
  for(size_t ck = 0; ck < chunks.size(); ck++)
  {
    const int cf = chunks[ck].first, cn = chunks[ck].second;
    cudaStream_t cs = copy_stream_[ck & 1];
    const int tok = any_host ? prof_begin(cs) : -1;
    for(int i = cf; i < cf + cn; i++)
    {
      const Shape& S = kind[i]->S;
      for(int f = 0; f < 2; f++)
      {
        const qmiv_frame* fr = f ? &pairs[i].in1 : &pairs[i].in0;
        Img& out = f ? in1[i] : in0[i];
        size_t off = P[i].staging + (size_t)f * S.staged_frame_bytes();
        for(int c = 0; c < 3; c++)
        {
          if(!fr->plane[c]) { return fail(QMIV_ERR_INVALID_ARG, "frame plane is null"); }
          const size_t row_bytes = S.plane_cols(c) * S.esz;
          if(fr->pitch[c] < (int64_t)row_bytes || (fr->pitch[c] % (int64_t)S.esz) != 0) { return fail(QMIV_ERR_INVALID_ARG, "bad plane pitch"); }
          out.sx[c] = c ? (int8_t)S.sx : 0;
          out.sy[c] = c ? (int8_t)S.sy : 0;
          if(fr->mem == QMIV_MEM_DEVICE)
          {
            out.p[c] = fr->plane[c];
            out.pitch[c] = (int32_t)(fr->pitch[c] / (int64_t)S.esz);
          }
          else if(fr->mem == QMIV_MEM_HOST)
          {
            char* dst = dbase + off;
            if((size_t)fr->pitch[c] == row_bytes && S.staged_pitch(c) == row_bytes)
            {
              // contiguous plane on both sides: one linear copy
              QMIV_CUDA(cudaMemcpyAsync(dst, fr->plane[c], row_bytes * S.plane_rows(c), cudaMemcpyHostToDevice, cs));
            }
            else
            {
              QMIV_CUDA(cudaMemcpy2DAsync(dst, S.staged_pitch(c), fr->plane[c], (size_t)fr->pitch[c], row_bytes, S.plane_rows(c),
                                          cudaMemcpyHostToDevice, cs));
            }
            out.p[c] = dst;
            out.pitch[c] = (int32_t)(S.staged_pitch(c) / S.esz);
            off += S.staged_plane_bytes(c);
          }
          else { return fail(QMIV_ERR_INVALID_ARG, "frame mem must be QMIV_MEM_HOST or QMIV_MEM_DEVICE"); }
        }
      }
    }
    if(any_host)
    {
      prof_end(cs, QMIV_STAGE_H2D, tok);
      QMIV_CUDA(cudaEventRecord(chunk_ready_[ck], cs));
    }
  }

  // ---- autotune new kinds on their first pair --------------------------------------------------
  if(flags_ & QMIV_BATCH_AUTOTUNE)
  {
    bool uploaded = !any_host;
    for(int i = 0; i < n; i++)
    {
      if(kind[i]->tuned || !P[i].need_search) { continue; }
      if(!uploaded)
      {
        for(cudaStream_t cs : copy_stream_) { QMIV_CUDA(cudaStreamSynchronize(cs)); }
        uploaded = true;
      }
      QMIV_TRY(autotune(*kind[i], in0[i], in1[i], s));
    }
  }

  // ---- descriptor tables (host mirror) ----------------------------------------------------------
  std::vector<Tables> TT(chunks.size());
  std::vector<size_t> tbase(chunks.size());
  size_t tbytes = 0;
  for(size_t ck = 0; ck < chunks.size(); ck++)
  {
    QMIV_TRY(build_tables(chunks[ck].first, chunks[ck].second, kind, TT[ck]));
    tbase[ck] = tbytes;
    tbytes += TT[ck].bytes;
  }
  QMIV_TRY(ensure_host(tbytes, n));
  const void* old_desc = arena_desc_.p;
  QMIV_TRY(arena_desc_.ensure(ctx_, tbytes));
  if(arena_desc_.p != old_desc) { clear_graphs(); }
  std::memset(host_mirror_, 0, tbytes);
  for(size_t ck = 0; ck < chunks.size(); ck++)
  {
    fill_tables(chunks[ck].second, kind, in0, in1, dbase, TT[ck], static_cast<char*>(host_mirror_) + tbase[ck],
                arena_desc_.as<char>() + tbase[ck]);
  }

  // ---- launches -----------------------------------------------------------------------------------
  // graphs (device frames only): a signature's first call runs eagerly (it also configures every
  // kernel), the second captures, later calls replay
  const bool graph = (flags_ & QMIV_BATCH_GRAPH) != 0 && !ctx_->profiling && !any_host && seen_[sig]++ > 0;
  auto enqueue = [&]() -> qmiv_status {
    QMIV_CUDA(cudaMemcpyAsync(arena_desc_.p, host_mirror_, tbytes, cudaMemcpyHostToDevice, s));
    QMIV_CUDA(cudaMemsetAsync(dbase, 0, zero_bytes, s));
    for(size_t ck = 0; ck < chunks.size(); ck++)
    {
      if(any_host) { QMIV_CUDA(cudaStreamWaitEvent(s, chunk_ready_[ck], 0)); }
      QMIV_TRY(launch_all(TT[ck], s));
    }
    QMIV_CUDA(cudaMemcpyAsync(host_out_, douts, sizeof(PairOut) * (size_t)n, cudaMemcpyDeviceToHost, s));
    return QMIV_OK;
  };
  if(graph)
  {
    cudaGraphExec_t& ex = graphs_[sig];
    if(!ex)
    {
      cudaGraph_t g = nullptr;
      QMIV_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
      const qmiv_status st = enqueue();
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      if(st != QMIV_OK) { if(g) { cudaGraphDestroy(g); } graphs_.erase(sig); return st; }
      if(ce != cudaSuccess) { graphs_.erase(sig); return cuda_fail(ce, "cudaStreamEndCapture"); }
      const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if(ie != cudaSuccess) { graphs_.erase(sig); return cuda_fail(ie, "cudaGraphInstantiate"); }
    }
    QMIV_CUDA(cudaGraphLaunch(ex, s));
  }
  else { QMIV_TRY(enqueue()); }
  pend_kind_ = kind;
  pend_mask_.resize(n);
  for(int i = 0; i < n; i++) { pend_mask_[i] = P[i].mask; }
  pend_gen_ = gen_idx;
  pend_gen_desc_.clear();
  for(int i : gen_idx) { pend_gen_desc_.push_back(pairs[i]); }
  pend_n_ = n;
  return QMIV_OK;
}

qmiv_status Engine::collect(qmiv_result* results)
{
  if(pend_n_ < 0) { return fail(QMIV_ERR_INVALID_ARG, "nothing submitted"); }
  const int n = pend_n_;
  pend_n_ = -1;
  if(n == 0) { return QMIV_OK; }
  QMIV_CUDA(cudaSetDevice(ctx_->device));
  QMIV_CUDA(cudaStreamSynchronize(stream_));
  harvest_profile();

  // ---- results ------------------------------------------------------------------------------------
  qmiv_status st = QMIV_OK;
  for(int i = 0; i < n; i++)
  {
    const PairKind& K = *pend_kind_[i];
    FinishInfo fi{};
    fi.W = K.S.W; fi.H = K.S.H; fi.bitdepth = K.S.bitdepth; fi.mask = pend_mask_[i];
    fi.erp = prm_.erp; fi.ws_corr = K.ws_corr;
    for(int c = 0; c < 4; c++) { fi.cwa[c] = prm_.cwa[c]; }
    fi.num_scales = K.ns;
    if(results) { finish_result(host_out_[i], fi, &results[i]); }
    const qmiv_status ps = pair_status(host_out_[i], prm_.invalid_pel_action);
    if(ps != QMIV_OK && st == QMIV_OK) { st = ps; }
  }
  if(results && st == QMIV_OK && !pend_gen_.empty()) { st = collect_gen(results); }
  return st;
}

qmiv_status Engine::collect_gen(qmiv_result* results)
{
  for(size_t g = 0; g < pend_gen_.size(); g++)
  {
    const int i = pend_gen_[g];
    const qmiv_pair_desc& d = pend_gen_desc_[g];
    const uint32_t mask = d.metric_mask & kSsimFamily;
    const KindKey key{ d.width, d.height, d.bitdepth, d.chroma_format, d.search_range };
    std::unique_ptr<PairPipeline>& pp = gen_pipes_[key];
    if(!pp)
    {
      pp.reset(new PairPipeline());
      qmiv_params prm = prm_;
      prm.search_range = d.search_range;
      QMIV_TRY(pp->configure(ctx_, pend_kind_[i]->S, prm, d.search_range));
    }
    const bool host = d.in0.mem == QMIV_MEM_HOST || d.in1.mem == QMIV_MEM_HOST;
    QMIV_TRY(pp->prepare(mask, false, host));
    Img a, b;
    QMIV_TRY(pp->resolve(&d.in0, 0, a, stream_));
    QMIV_TRY(pp->resolve(&d.in1, 1, b, stream_));
    QMIV_TRY(pp->enqueue(a, b, mask, false, false, stream_));
    QMIV_CUDA(cudaStreamSynchronize(stream_));
    qmiv_result r{};
    finish_result(pp->host_out(), pp->finish_info(mask), &r);
    qmiv_result& o = results[i];
    for(int c = 0; c < 4; c++) { o.ssim[c] = r.ssim[c]; o.msssim[c] = r.msssim[c]; }
    o.ssim_pic = r.ssim_pic; o.msssim_pic = r.msssim_pic;
    o.ivssim = r.ivssim; o.ivssim_r2t = r.ivssim_r2t; o.ivssim_t2r = r.ivssim_t2r;
    o.ivmsssim = r.ivmsssim; o.ivmsssim_r2t = r.ivmsssim_r2t; o.ivmsssim_t2r = r.ivmsssim_t2r;
    if(mask & (QMIV_IVSSIM | QMIV_IVMSSSIM))   // the search's side outputs, as the plain form reports them
    {
      for(int c = 0; c < 4; c++) { o.gcd_r2t[c] = r.gcd_r2t[c]; o.cps_sse_r2t[c] = r.cps_sse_r2t[c]; o.cps_sse_t2r[c] = r.cps_sse_t2r[c]; }
    }
  }
  return QMIV_OK;
}

// ---------------------------------------------------------------------------------------------
// descriptor tables
// ---------------------------------------------------------------------------------------------
size_t Engine::mom_slot_elems(const Shape& S)
{
  const size_t nbx = ((size_t)S.W + 3) / 4, nby = ((size_t)S.H + 3) / 4;
  return 3 * 5 * nby * ((nbx + 7) & ~(size_t)7);
}

Moments Engine::mom_at(const Shape& S, const PairSlot& p, char* dbase, int slot, int scale)
{
  Moments m{};
  m.nbx = ((S.W >> scale) + 3) / 4;
  m.nby = ((S.H >> scale) + 3) / 4;
  m.pitch = (m.nbx + 7) & ~7;
  m.p = reinterpret_cast<uint32_t*>(dbase + p.mom) + (size_t)slot * p.mom_slot;
  return m;
}

uint32_t Engine::clip_of(const PairKind& K) const
{
  return prm_.invalid_pel_action == QMIV_PEL_CNCL ? (uint32_t)K.S.maxv : 0xffffu;
}

// Counts every table entry of pairs [first, first + n) and lays the tables out.
qmiv_status Engine::build_tables(int first, int n, const std::vector<PairKind*>& kind, Tables& T)
{
  T = Tables{};
  T.first = first;
  T.n = n;
  for(int i = first; i < first + n; i++)
  {
    const int g = kind[i]->S.esz == 1 ? 0 : 1;
    T.prepass_idx[g].push_back(i);
    const int rows = kind[i]->S.H + 2 * kind[i]->S.ch;
    T.prepass_max_rows[g] = std::max(T.prepass_max_rows[g], rows);
  }
  for(int i = first; i < first + n; i++)
  {
    if(!slots_[i].need_search) { continue; }
    const PairKind& K = *kind[i];
    T.cps_groups[CpsGroupKey{ K.R, (int)K.S.esz, K.wy }].push_back(i);
  }
  int max_ns = 0;
  for(int i = first; i < first + n; i++) { if(slots_[i].need_ms) { max_ns = std::max(max_ns, kind[i]->ns); } }
  T.phases = std::max(1, max_ns);

  size_t off = 0;
  auto place = [&](size_t bytes, size_t align) { off = align_sz(off, align); const size_t o = off; off += bytes; return o; };
  T.prepass_off[0] = place(sizeof(PrepassArgs) * T.prepass_idx[0].size(), 64);
  T.prepass_off[1] = place(sizeof(PrepassArgs) * T.prepass_idx[1].size(), 64);
  T.reduce_off = place(sizeof(ReduceArgs) * (size_t)n, 64);
  size_t ncps = 0;
  for(auto& g : T.cps_groups) { ncps += g.second.size(); }
  T.cps_off = place(cps_desc_bytes() * ncps, 64);
  T.prefix_off = place(sizeof(int32_t) * (ncps + T.cps_groups.size()), 16);
  T.fin_off = place(sizeof(FinalizeArgs) * (size_t)n, 64);
  size_t mom_jobs = 0, pool_jobs = 0, fin_jobs = 0;
  for(int i = first; i < first + n; i++)
  {
    const PairSlot& p = slots_[i];
    const size_t ns = p.need_ms ? (size_t)kind[i]->ns : 0;
    mom_jobs += ((p.mask & QMIV_SSIM) ? 1 : 0) + ns * (((p.mask & QMIV_MSSSIM) ? 1 : 0) + ((p.mask & QMIV_IVMSSSIM) ? 2 : 0));
    pool_jobs += 3 * (((p.mask & QMIV_IVSSIM) ? 2 : 0) + ((p.mask & QMIV_SSIM) ? 1 : 0) +
                      ns * (((p.mask & QMIV_MSSSIM) ? 1 : 0) + ((p.mask & QMIV_IVMSSSIM) ? 2 : 0)));
    fin_jobs += 3 + 6 + 3 * kMaxSsimSlots + 1;
  }
  T.mom_off = place(sizeof(SsimMomArgs) * mom_jobs, 64);
  T.pool_off = place(sizeof(SsimPoolJob) * pool_jobs, 64);
  T.finjob_off = place(sizeof(FinJob) * fin_jobs, 16);
  T.bytes = align_sz(off, 256);
  return QMIV_OK;
}

void Engine::fill_tables(int n, const std::vector<PairKind*>& kind, const std::vector<Img>& in0,
                         const std::vector<Img>& in1, char* dbase, Tables& T, char* h, char* d)
{
  const int first = T.first;
  // prepass + reduce
  for(int g = 0; g < 2; g++)
  {
    PrepassArgs* pa = reinterpret_cast<PrepassArgs*>(h + T.prepass_off[g]);
    for(size_t j = 0; j < T.prepass_idx[g].size(); j++)
    {
      const int i = T.prepass_idx[g][j];
      const PairKind& K = *kind[i];
      const PairSlot& p = slots_[i];
      PrepassArgs& a = pa[j];
      a.in0 = in0[i]; a.in1 = in1[i];
      for(int c = 0; c < 3; c++) { a.rows[c] = (int32_t)K.S.plane_rows(c); a.cols[c] = (int32_t)K.S.plane_cols(c); }
      a.clip = clip_of(K);
      a.row_sd = reinterpret_cast<int64_t*>(dbase + p.row_sd);
      a.row_ssd = reinterpret_cast<uint64_t*>(dbase + p.row_ssd);
      a.out = reinterpret_cast<PairOut*>(dbase + p.out);
    }
  }
  ReduceArgs* ra = reinterpret_cast<ReduceArgs*>(h + T.reduce_off);
  for(int i = first; i < first + n; i++)
  {
    const PairKind& K = *kind[i];
    const PairSlot& p = slots_[i];
    ReduceArgs& a = ra[i - first];
    for(int c = 0; c < 3; c++) { a.rows[c] = (int32_t)K.S.plane_rows(c); a.mult[c] = c ? (1 << (K.S.sx + K.S.sy)) : 1; }
    a.area = (int64_t)K.S.W * K.S.H; a.maxv = K.S.maxv;
    for(int c = 0; c < 4; c++) { a.maxdiff[c] = K.maxdiff[c]; }
    a.need_gcd = p.need_search ? 1 : 0;
    a.fp32_ok = K.fp32_ok ? 1 : 0;
    a.clip_on = prm_.invalid_pel_action == QMIV_PEL_CNCL;
    a.row_sd = reinterpret_cast<int64_t*>(dbase + p.row_sd);
    a.row_ssd = reinterpret_cast<uint64_t*>(dbase + p.row_ssd);
    a.out = reinterpret_cast<PairOut*>(dbase + p.out);
  }
  // CPS work lists
  {
    char* cdesc = h + T.cps_off;
    int32_t* prefix = reinterpret_cast<int32_t*>(h + T.prefix_off);
    size_t di = 0, pi = 0;
    T.cps_launch.clear();
    for(auto& g : T.cps_groups)
    {
      CpsLaunch L{};
      L.R = g.first.R; L.esz = g.first.esz; L.wy = g.first.wy;
      L.d_desc = d + T.cps_off + di * cps_desc_bytes();
      L.d_prefix = reinterpret_cast<const int32_t*>(d + T.prefix_off) + pi;
      L.npairs = (int)g.second.size();
      int tiles = 0;
      for(int i : g.second)
      {
        const PairKind& K = *kind[i];
        const PairSlot& p = slots_[i];
        CpsArgs ca{};
        ca.in0 = in0[i]; ca.in1 = in1[i]; ca.W = K.S.W; ca.H = K.S.H; ca.maxv = K.S.maxv; ca.clip = clip_of(K);
        for(int c = 0; c < 3; c++) { ca.wi[c] = prm_.cws[c]; ca.wf[c] = (float)prm_.cws[c]; }
        ca.gcd_src = reinterpret_cast<PairOut*>(dbase + p.out);
        ca.rows = reinterpret_cast<uint32_t*>(dbase + p.cps_rows);
        if(p.need_scp)
        {
          ca.scp0 = dbase + p.scp;
          ca.scp1 = dbase + p.scp + (size_t)3 * K.S.W * K.S.H * K.S.esz;
        }
        if(p.mask & QMIV_IVSSIM) { ca.mom[0] = mom_at(K.S, p, dbase, 0, 0); ca.mom[1] = mom_at(K.S, p, dbase, 1, 0); }
        CpsPairPlan plan{};
        cps_describe(cdesc + di * cps_desc_bytes(), ca, K.R, (int)K.S.esz, K.wy, &plan);
        prefix[pi++] = tiles;
        tiles += plan.ntiles;
        L.raw_cap = std::max(L.raw_cap, plan.raw_bytes);
        L.smem = std::max(L.smem, plan.smem);
        di++;
      }
      prefix[pi++] = tiles;
      L.ntiles = tiles;
      T.cps_launch.push_back(L);
    }
  }
  // SSIM moments / pool jobs per phase, finalize
  SsimMomArgs* mj = reinterpret_cast<SsimMomArgs*>(h + T.mom_off);
  SsimPoolJob* pj = reinterpret_cast<SsimPoolJob*>(h + T.pool_off);
  FinalizeArgs* fa = reinterpret_cast<FinalizeArgs*>(h + T.fin_off);
  size_t nm = 0, np = 0;
  T.phase.assign(T.phases, Phase{});
  for(int ph = 0; ph < T.phases; ph++)
  {
    Phase& PH = T.phase[ph];
    for(int esz = 0; esz < 2; esz++)
    {
      PH.mom_first[esz] = nm;
      for(int i = first; i < first + n; i++)
      {
        if((kind[i]->S.esz == 1 ? 0 : 1) != esz) { continue; }
        add_moment_jobs(i, *kind[i], ph, in0[i], in1[i], dbase, mj, nm, PH);
      }
      PH.mom_count[esz] = nm - PH.mom_first[esz];
    }
    PH.pool_first = np;
    for(int i = first; i < first + n; i++) { add_pool_jobs(i, *kind[i], ph, dbase, pj, np, PH, fa[i - first]); }
    PH.pool_count = np - PH.pool_first;
  }
  FinJob* fj = reinterpret_cast<FinJob*>(h + T.finjob_off);
  size_t nf = 0;
  T.fin_smem = 0;
  for(int i = first; i < first + n; i++)
  {
    const PairKind& K = *kind[i];
    const PairSlot& p = slots_[i];
    FinalizeArgs& a = fa[i - first];
    a.nslots = kMaxSsimSlots;
    a.H = K.S.H;
    for(int c = 0; c < 3; c++) { a.rows[c] = (int32_t)K.S.plane_rows(c); a.sy[c] = c ? K.S.sy : 0; a.mult_row[c] = c ? (1 << K.S.sx) : 1; }
    a.row_ssd = reinterpret_cast<const uint64_t*>(dbase + p.row_ssd);
    a.ws = prm_.erp ? K.ws_dev.as<double>() : nullptr;
    a.do_wspsnr = (p.mask & QMIV_WSPSNR) ? 1 : 0;
    a.cps_rows = p.need_search ? reinterpret_cast<const uint32_t*>(dbase + p.cps_rows) : nullptr;
    a.out = reinterpret_cast<PairOut*>(dbase + p.out);
    const int blocks = finalize_plan(a);
    for(int b = 0; b < blocks; b++) { fj[nf++] = FinJob{ i - first, b }; }
    T.fin_smem = std::max(T.fin_smem, finalize_smem(a));
  }
  T.fin_jobs = (int)nf;
  T.d_fin = reinterpret_cast<const FinalizeArgs*>(d + T.fin_off);
  T.d_finjobs = reinterpret_cast<const FinJob*>(d + T.finjob_off);
  T.d_prepass[0] = reinterpret_cast<const PrepassArgs*>(d + T.prepass_off[0]);
  T.d_prepass[1] = reinterpret_cast<const PrepassArgs*>(d + T.prepass_off[1]);
  T.d_reduce = reinterpret_cast<const ReduceArgs*>(d + T.reduce_off);
  T.d_mom = reinterpret_cast<const SsimMomArgs*>(d + T.mom_off);
  T.d_pool = reinterpret_cast<const SsimPoolJob*>(d + T.pool_off);
}

// SSIM moments of phase (scale) ph of pair i: plain SSIM at scale 0, MS-SSIM / IV-MS-SSIM scales
// with the next pyramid level written on the way (xSSIM.cpp:230-256)
void Engine::add_moment_jobs(int i, const PairKind& K, int ph, const Img& a0, const Img& a1, char* dbase,
                             SsimMomArgs* mj, size_t& nm, Phase& PH)
{
  const PairSlot& p = slots_[i];
  const Shape& S = K.S;
  const int ns = p.need_ms ? K.ns : 0;
  const Img scp0 = p.need_scp ? img444(dbase + p.scp, S.W, S.H, S.esz) : Img{};
  const Img scp1 = p.need_scp ? img444(dbase + p.scp + (size_t)3 * S.W * S.H * S.esz, S.W, S.H, S.esz) : Img{};
  auto level_base = [&](int img, int scale) -> char* {
    size_t o = (size_t)img * p.pyr_lv;
    for(int s2 = 1; s2 < scale; s2++) { o += (size_t)(S.W >> s2) * (S.H >> s2) * 3; }
    return dbase + p.pyr + o * S.esz;
  };
  auto level_img = [&](int img, int scale) -> Img {
    if(scale == 0) { return img == 0 ? a0 : img == 1 ? a1 : img == 2 ? scp0 : scp1; }
    return img444(level_base(img, scale), S.W >> scale, S.H >> scale, S.esz);
  };
  const uint32_t clip = clip_of(K);
  auto push = [&](const Img& x, const Img& y, int W, int H, const Moments& m, const MutImg* dx, const MutImg* dy) {
    SsimMomArgs& a = mj[nm++];
    a.a = x; a.b = y; a.W = W; a.H = H; a.clip = clip; a.mom = m;
    if(dx) { a.down_a = *dx; }
    if(dy) { a.down_b = *dy; }
    PH.mom_max_nbx = std::max(PH.mom_max_nbx, m.nbx);
    PH.mom_max_nby = std::max(PH.mom_max_nby, m.nby);
  };
  if(ph == 0 && (p.mask & QMIV_SSIM)) { push(a0, a1, S.W, S.H, mom_at(S, p, dbase, 2, 0), nullptr, nullptr); }
  if(ph < ns)
  {
    const int sc = ph;
    const int Ws = S.W >> sc, Hs = S.H >> sc;
    const bool last = sc == ns - 1;
    bool written[4] = { false, false, false, false };
    MutImg m[6];
    int mi = 0;
    auto down = [&](int img) -> const MutImg* {
      if(last || written[img]) { return nullptr; }
      written[img] = true;
      m[mi] = mut444(level_base(img, sc + 1), S.W >> (sc + 1), S.H >> (sc + 1), S.esz);
      return &m[mi++];
    };
    if(p.mask & QMIV_MSSSIM)
    {
      const MutImg* d0 = down(0); const MutImg* d1 = down(1);
      push(level_img(0, sc), level_img(1, sc), Ws, Hs, mom_at(S, p, dbase, 2, sc), d0, d1);
    }
    if(p.mask & QMIV_IVMSSSIM)  // xIVSSIM.cpp:77-78, no ERP weighting
    {
      const MutImg* d0 = down(0); const MutImg* d3 = down(3);
      push(level_img(0, sc), level_img(3, sc), Ws, Hs, mom_at(S, p, dbase, 3, sc), d0, d3);
      const MutImg* d1 = down(1); const MutImg* d2 = down(2);
      push(level_img(1, sc), level_img(2, sc), Ws, Hs, mom_at(S, p, dbase, 4, sc), d1, d2);
    }
  }
}

void Engine::add_pool_jobs(int i, const PairKind& K, int ph, char* dbase, SsimPoolJob* pj, size_t& np, Phase& PH,
                           FinalizeArgs& fa)
{
  const PairSlot& p = slots_[i];
  if(!p.need_ssim) { return; }
  const Shape& S = K.S;
  const int ns = p.need_ms ? K.ns : 0;
  double* rowsum = reinterpret_cast<double*>(dbase + p.rowsum);
  double* win = reinterpret_cast<double*>(dbase + p.win);
  int jobs_here = 0;
  auto add = [&](const Moments& m, int scale, int slot, int calc_l, int use_ws) {
    for(int c = 0; c < 3; c++)
    {
      SsimPoolJob& J = pj[np++];
      J.win = win + (size_t)(jobs_here++) * pool_win_elems(K.nx[0], K.ny[0]);
      J.C1 = K.C1; J.C2 = K.C2;
      J.mom = m.p + (size_t)c * 5 * m.plane(); J.plane = m.plane(); J.pitch = m.pitch;
      J.nx = K.nx[scale]; J.ny = K.ny[scale]; J.calc_l = calc_l; J.wide = S.bitdepth > 12 ? 1 : 0;
      J.row_sum = rowsum + (size_t)slot * 3 * K.ny[0] + (size_t)c * K.ny[scale];  // finalize reads [c][ny_scale]
      assert(pool_job_aligned(J));
      PH.pool_max_nx = std::max(PH.pool_max_nx, J.nx);
      PH.pool_max_ny = std::max(PH.pool_max_ny, J.ny);
    }
    fa.slot[slot].row_sum = rowsum + (size_t)slot * 3 * K.ny[0];
    fa.slot[slot].nx = K.nx[scale]; fa.slot[slot].ny = K.ny[scale]; fa.slot[slot].use_ws = use_ws;
    fa.slot[slot].ws_base = 4; fa.slot[slot].ws_step = 4;  // window row j covers rows 4j..4j+7 (xIVSSIM.cpp:153)
  };
  const int use_ws = prm_.erp ? 1 : 0;
  if(ph == 0 && (p.mask & QMIV_IVSSIM))  // (In0, SCP1) = T2R, (In1, SCP0) = R2T (xIVSSIM.cpp:46-47)
  {
    add(mom_at(S, p, dbase, 0, 0), 0, kSlotIvT2R, 1, use_ws);
    add(mom_at(S, p, dbase, 1, 0), 0, kSlotIvR2T, 1, use_ws);
  }
  if(ph == 0 && (p.mask & QMIV_SSIM)) { add(mom_at(S, p, dbase, 2, 0), 0, kSlotSsim, 1, 0); }
  if(ph < ns)
  {
    const int sc = ph;
    const bool last = sc == ns - 1;
    if(p.mask & QMIV_MSSSIM) { add(mom_at(S, p, dbase, 2, sc), sc, kSlotMs + sc, last ? 1 : 0, 0); }
    if(p.mask & QMIV_IVMSSSIM)
    {
      add(mom_at(S, p, dbase, 3, sc), sc, kSlotIvmsT2R + sc, last ? 1 : 0, 0);
      add(mom_at(S, p, dbase, 4, sc), sc, kSlotIvmsR2T + sc, last ? 1 : 0, 0);
    }
  }
}

qmiv_status Engine::launch_all(const Tables& T, cudaStream_t s)
{
  {
    const int t = prof_begin(s);
    QMIV_CUDA(launch_prepass_multi<uint8_t>(T.d_prepass[0], (int)T.prepass_idx[0].size(), T.prepass_max_rows[0], s));
    QMIV_CUDA(launch_prepass_multi<uint16_t>(T.d_prepass[1], (int)T.prepass_idx[1].size(), T.prepass_max_rows[1], s));
    prof_end(s, QMIV_STAGE_PREPASS, t);
  }
  {
    const int t = prof_begin(s);
    QMIV_CUDA(launch_reduce_multi(T.d_reduce, T.n, s));
    prof_end(s, QMIV_STAGE_REDUCE, t);
  }
  for(const CpsLaunch& L : T.cps_launch)
  {
    const int t = prof_begin(s);
    QMIV_CUDA(launch_cps_multi(L.d_desc, L.d_prefix, L.npairs, L.ntiles, L.R, L.wy, L.esz, L.raw_cap, L.smem, s));
    prof_end(s, QMIV_STAGE_CPS, t);
  }
  for(int ph = 0; ph < T.phases; ph++)
  {
    const Phase& PH = T.phase[ph];
    if(PH.mom_count[0] + PH.mom_count[1] > 0)
    {
      const int t = prof_begin(s);
      QMIV_CUDA(launch_ssim_moments_multi<uint8_t>(T.d_mom + PH.mom_first[0], (int)PH.mom_count[0], PH.mom_max_nbx, PH.mom_max_nby, s));
      QMIV_CUDA(launch_ssim_moments_multi<uint16_t>(T.d_mom + PH.mom_first[1], (int)PH.mom_count[1], PH.mom_max_nbx, PH.mom_max_nby, s));
      prof_end(s, QMIV_STAGE_SSIM_WIN, t);
    }
    if(PH.pool_count > 0)
    {
      const int t = prof_begin(s);
      QMIV_CUDA(launch_ssim_pool_multi(T.d_pool + PH.pool_first, (int)PH.pool_count, PH.pool_max_nx, PH.pool_max_ny, s));
      prof_end(s, QMIV_STAGE_SSIM_ROWS, t);
    }
  }
  {
    const int t = prof_begin(s);
    QMIV_CUDA(launch_finalize_multi(T.d_fin, T.d_finjobs, T.fin_jobs, T.fin_smem, s));
    prof_end(s, QMIV_STAGE_FINALIZE, t);
  }
  return QMIV_OK;
}

// ---- stage timing (not while a graph is replayed) -------------------------------------------------
int Engine::prof_begin(cudaStream_t s) { return clock_.begin(ctx_, s); }
void Engine::prof_end(cudaStream_t s, int stage, int tok) { clock_.end(s, stage, tok); }
void Engine::harvest_profile() { clock_.harvest(ctx_); }

bool Engine::tuning(int32_t W, int32_t H, int32_t bd, int32_t R, int32_t* tile_w, int32_t* tile_h, int32_t* rows) const
{
  for(const auto& kv : kinds_)
  {
    const KindKey& k = kv.first;
    if(k.W == W && k.H == H && k.bd == bd && k.R == R)
    {
      if(tile_w) { *tile_w = 128; }
      if(tile_h) { *tile_h = 4 * kv.second->wy; }
      if(rows) { *rows = 4; }
      return true;
    }
  }
  return false;
}

}  // namespace qmiv
