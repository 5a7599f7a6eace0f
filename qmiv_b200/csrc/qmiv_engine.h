// Batched multi-pair engine (qmiv_engine.cu): the pipeline of qmiv_calc.cu for many frame pairs at
// once, one launch per stage, optionally replayed from CUDA graphs.
#pragma once
#include "qmiv_host.h"

#include <map>
#include <memory>
#include <string>
#include <tuple>
#include <vector>

namespace qmiv {

// Constants of one kind of frame pair (size, bit depth, chroma format, search range).
struct PairKind
{
  Shape       S;
  qmiv_params prm{};
  int32_t     R = 2;
  int32_t     maxdiff[4] = { 0, 0, 0, 0 };
  bool        fp32_ok = true;
  int32_t     ns = 0, nx[5] = {}, ny[5] = {};
  double      C1 = 0, C2 = 0;
  std::vector<double> ws_host;
  double      ws_corr = 1.0;
  DevMem      ws_dev;
  int32_t     wy = 8;          // CPS tile height / 4
  bool        tuned = false;
  float       tune_ms[3] = { 0.f, 0.f, 0.f };   // fastest launch of 128 x 32, 128 x 24, 128 x 16 tiles
};

struct KindKey
{
  int32_t W, H, bd, cf, R;
  bool operator<(const KindKey& o) const { return std::tie(W, H, bd, cf, R) < std::tie(o.W, o.H, o.bd, o.cf, o.R); }
};

// Byte offsets of one pair's buffers in the batch arena.
struct PairSlot
{
  uint32_t mask = 0;
  bool     need_scp = false, need_search = false, need_ssim = false, need_ms = false, host = false;
  size_t   out = 0, cps_rows = 0, row_sd = 0, row_ssd = 0, scp = 0, mom = 0, mom_slot = 0, rowsum = 0, win = 0;
  size_t   pyr = 0, pyr_lv = 0, staging = 0;
};

struct CpsGroupKey
{
  int R, esz, wy;
  bool operator<(const CpsGroupKey& o) const { return std::tie(R, esz, wy) < std::tie(o.R, o.esz, o.wy); }
};

struct CpsLaunch
{
  int            R = 2, esz = 2, wy = 8, npairs = 0, ntiles = 0;
  const void*    d_desc = nullptr;
  const int32_t* d_prefix = nullptr;
  uint32_t       raw_cap = 0;
  size_t         smem = 0;
};

// SSIM work of one scale: moment jobs per sample size, then pool jobs
struct Phase
{
  size_t mom_first[2] = { 0, 0 }, mom_count[2] = { 0, 0 };
  int    mom_max_nbx = 0, mom_max_nby = 0;
  size_t pool_first = 0, pool_count = 0;
  int    pool_max_nx = 0, pool_max_ny = 0;
};

// Argument tables of one set of pairs: host layout, device pointers, launch shapes.
struct Tables
{
  size_t bytes = 0;
  int    n = 0;
  int    first = 0;                 // global index of the set's first pair
  std::vector<int> prepass_idx[2];
  int    prepass_max_rows[2] = { 0, 0 };
  size_t prepass_off[2] = { 0, 0 }, reduce_off = 0, cps_off = 0, prefix_off = 0, fin_off = 0;
  size_t mom_off = 0, pool_off = 0, finjob_off = 0;
  std::map<CpsGroupKey, std::vector<int>> cps_groups;
  std::vector<CpsLaunch> cps_launch;
  int    phases = 1;
  std::vector<Phase> phase;
  int    fin_jobs = 0;
  size_t fin_smem = 0;
  const PrepassArgs*  d_prepass[2] = { nullptr, nullptr };
  const ReduceArgs*   d_reduce = nullptr;
  const SsimMomArgs*  d_mom = nullptr;
  const SsimPoolJob*  d_pool = nullptr;
  const FinalizeArgs* d_fin = nullptr;
  const FinJob*       d_finjobs = nullptr;
};

class Engine
{
public:
  qmiv_status init(qmiv_ctx_s* ctx, const qmiv_params& prm, int32_t max_pairs, int64_t max_pixels, int32_t flags);
  // Computes every pair and waits for the results.
  qmiv_status run(const qmiv_pair_desc* pairs, int32_t n, qmiv_result* results);
  // The two halves of run(): enqueue every upload and launch on the engine's streams, then wait and
  // finish the results. One call in flight per engine; host frames must stay valid until collect().
  qmiv_status submit(const qmiv_pair_desc* pairs, int32_t n);
  qmiv_status collect(qmiv_result* results);
  bool        busy() const { return pend_n_ >= 0; }
  cudaStream_t stream() const { return stream_; }
  bool tuning(int32_t W, int32_t H, int32_t bd, int32_t R, int32_t* tile_w, int32_t* tile_h, int32_t* rows) const;
  size_t device_bytes() const { return arena_.bytes + arena_desc_.bytes + tune_scratch_.bytes; }
  ~Engine();

private:
  qmiv_status kind_for(const qmiv_pair_desc& d, PairKind*& out);
  qmiv_status autotune(PairKind& k, const Img& in0, const Img& in1, cudaStream_t s);
  qmiv_status ensure_host(size_t mirror_bytes, int n);
  void        clear_graphs();
  // argument tables of pairs [first, first + n): layout, then contents (host mirror h, device d)
  qmiv_status build_tables(int first, int n, const std::vector<PairKind*>& kind, Tables& T);
  void        fill_tables(int n, const std::vector<PairKind*>& kind, const std::vector<Img>& in0,
                          const std::vector<Img>& in1, char* dbase, Tables& T, char* h, char* d);
  void        add_moment_jobs(int i, const PairKind& K, int ph, const Img& a0, const Img& a1, char* dbase, SsimMomArgs* mj,
                              size_t& nm, Phase& PH);
  void        add_pool_jobs(int i, const PairKind& K, int ph, char* dbase, SsimPoolJob* pj, size_t& np, Phase& PH,
                            FinalizeArgs& fa);
  qmiv_status launch_all(const Tables& T, cudaStream_t s);
  uint32_t    clip_of(const PairKind& K) const;
  static size_t  mom_slot_elems(const Shape& S);
  static Moments mom_at(const Shape& S, const PairSlot& p, char* dbase, int slot, int scale);
  int  prof_begin(cudaStream_t s);
  void prof_end(cudaStream_t s, int stage, int token);
  void harvest_profile();

  qmiv_ctx_s*  ctx_ = nullptr;
  qmiv_params  prm_{};
  int32_t      max_pairs_ = 0;
  int64_t      max_pixels_ = 0;
  int32_t      flags_ = 0;
  cudaStream_t stream_ = nullptr;
  cudaStream_t copy_stream_[2] = { nullptr, nullptr };  // host-frame uploads, sub-batches alternate
  std::vector<cudaEvent_t> chunk_ready_;
  std::map<KindKey, std::unique_ptr<PairKind>> kinds_;
  std::vector<PairSlot> slots_;
  DevMem       arena_, arena_desc_, tune_scratch_;
  void*        host_mirror_ = nullptr;
  size_t       host_mirror_bytes_ = 0;
  PairOut*     host_out_ = nullptr;
  int          host_out_n_ = 0;
  std::map<std::string, cudaGraphExec_t> graphs_;
  std::map<std::string, int> seen_;
  StageClock   clock_;
  int          pend_n_ = -1;                   // pairs of the call in flight, -1 = none
  std::vector<PairKind*> pend_kind_;
  std::vector<uint32_t>  pend_mask_;
  // SSIM metrics under a structural similarity option other than BlockAveraged 8/4: the batch computes
  // every other metric, then collect() computes these pair by pair through a PairPipeline of the
  // pair's kind (the qmiv_calc path) and merges them into the results
  std::vector<int>            pend_gen_;       // indices of the call's pairs with such metrics
  std::vector<qmiv_pair_desc> pend_gen_desc_;
  std::map<KindKey, std::unique_ptr<PairPipeline>> gen_pipes_;
  qmiv_status collect_gen(qmiv_result* results);
};

}  // namespace qmiv
