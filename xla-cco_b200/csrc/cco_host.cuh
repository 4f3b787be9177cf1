// Host-side internals shared by the C-ABI translation units: error reporting,
// the per-device memory pool, the problem object and the lane-set runtime
// (lane records, evaluation plans, the CUDA-graph tick driver) that both the
// one-shot relaxations and the serving pool run on.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <vector>

#include "cco.h"
#include "cco_internal.cuh"
#include "cco_flow.cuh"
#include "cco_md.cuh"
#include "cco_opt.cuh"

struct cco_problem {
  int device = 0;
  int d = 0, N = 0, M = 0;
  cco::ProbDev host{};         // pointers are device pointers
  cco::ProbDev* dev = nullptr; // device copy
  cco::SegHdr* seg1 = nullptr;
  cco::SegHdr* seg2 = nullptr;
  double* w_run = nullptr;
  int* run2ref = nullptr;
  cco::GemmRun* grun = nullptr;
  cco::GemmBlock* gblk = nullptr;
  double4* krow = nullptr;     // run-order rows (n_0, n_1, n_2, w) for the Hessian kernels
  size_t smem1 = 0, smem2 = 0, smemG = 0;
};

namespace cco {

// Closed-form Hessians of `batch` configurations (cco_hessian.cu): rho_run is
// each configuration's run-order density from the evaluation kernels, H is
// [batch][N d][N d].
cudaError_t hessian_launch(const cco_problem* p, cudaStream_t st, int batch, const double* s,
                           const double2* rho_run, double* H);

// Records the message for cco_last_error and returns `code`.
int fail(int code, const char* fmt, ...);
int cuda_fail(cudaError_t e, const char* what);

#define CCO_CUDA(call)                                       \
  do {                                                       \
    cudaError_t e_ = (call);                                 \
    if (e_ != cudaSuccess) return ::cco::cuda_fail(e_, #call); \
  } while (0)

// Stream-ordered allocations come from one memory pool per device that keeps
// its memory (release threshold = max).
cudaError_t device_pool(cudaMemPool_t* out);

template <class T>
cudaError_t pool_alloc(T** ptr, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool;
  const cudaError_t e = device_pool(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(reinterpret_cast<void**>(ptr), bytes, pool, st);
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& src, cudaStream_t st) {
  cudaError_t e = pool_alloc(dst, sizeof(T) * std::max<size_t>(src.size(), 1), st);
  if (e == cudaSuccess && !src.empty())
    e = cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, st);
  return e;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------ lane records
enum class Method { Descent, Lbfgs, Flow, Md };

// What every record of one launch shares: the minimizer and, for L-BFGS,
// the memory m and whether the scalar kernel's triangles live in the record.
struct RecordShape {
  Method method = Method::Lbfgs;
  int m = 0, tri_len = 0;
  int keep_s0 = 0;   // L-BFGS mixed precision: records hold s0
  int waves = 0;   // MD segment runs: tracked waves per lane
};

inline size_t record_doubles(const RecordShape& R, const cco_problem* p) {
  const int ld = pad4(p->N * p->d);
  size_t n = 0;
  if (R.method == Method::Descent) n = ds_record_doubles(ld, p->M, p->host.ntile1);
  else if (R.method == Method::Flow) n = fl_record_doubles(ld, p->M, p->host.ntile1);
  else if (R.method == Method::Md) n = md_record_doubles(ld, p->M, p->host.ntile1, R.waves);
  else n = lb_record_doubles(R.m, R.tri_len, ld, p->M, p->host.ntile1, R.keep_s0);
  return (n + 31) & ~(size_t)31;   // records start on 256-byte boundaries
}

inline size_t record_bytes(const RecordShape& R, const cco_problem* p) {
  return record_doubles(R, p) * sizeof(double);
}

// Evaluation view of a lane record: probe positions in, energy, gradient and
// densities out, status read by the evaluation kernels.
inline EvalLane eval_lane(const RecordShape& R, const LaneRef& L, const cco_problem* p,
                          int prob_index) {
  EvalLane e{};
  double2* dens;
  e.prec = nullptr;
  e.fixed_prec = PREC_FP64;
  if (R.method == Method::Descent) {
    const DsView v = ds_view(L.rec, L.ld);
    e.s = v.ps;
    e.g = v.pg;
    e.f = v.pf;
    dens = v.dens;
  } else if (R.method == Method::Flow) {
    const FlView v = fl_view(L.rec, L.ld);
    e.s = v.ps;
    e.g = v.pg;
    e.f = v.pf;
    dens = v.dens;
  } else if (R.method == Method::Md) {
    const MdView v = md_view(L.rec, L.ld, R.waves);
    e.s = v.ps;
    e.g = v.pg;
    e.f = v.pf;
    dens = v.dens;
  } else {
    const LbView v = lb_view(L.rec, R.m, R.tri_len, L.ld, R.keep_s0);
    e.s = v.ps;
    e.g = v.pg;
    e.f = v.pf;
    e.prec = &v.st->prec;
    dens = v.dens;
  }
  e.rho = dens;
  e.rhow = dens + p->M;
  e.part = dens + 2 * (size_t)p->M;
  e.status = rec_status(L.rec);
  e.prob = prob_index;
  return e;
}

// Evaluation plan of a list of lanes, built on the host and uploaded.
struct EvalSet {
  ProbDev* probs = nullptr;
  EvalLane* lanes = nullptr;
  EvalItem* it1 = nullptr;
  EvalItem* it2 = nullptr;
  EvalItem* itG = nullptr;
  EvalPlan plan{};

  cudaError_t build(const RecordShape& R, const std::vector<LaneRef>& refs,
                    const std::vector<const cco_problem*>& probs_of, int lo, int hi,
                    cudaStream_t st, bool may_fp32 = false) {
    long long tiles1 = 0, seg_tiles = 0;
    for (int i = lo; i < hi; ++i) {
      tiles1 += probs_of[i]->host.ntile2;
      if (!probs_of[i]->host.gemm) seg_tiles += probs_of[i]->host.ntile1;
    }
    const int split = pass2_split(tiles1);
    // pass-1 segment chunks: enough CTAs for the per-segment FP64 tiles
    int chunks = 1;
    while (!may_fp32 && chunks < 8 && seg_tiles * chunks < kPass2TargetCtas) chunks *= 2;
    std::vector<const cco_problem*> uniq;
    std::vector<ProbDev> pv;
    std::vector<EvalLane> lv;
    std::vector<EvalItem> g1[3], g2[3];   // items grouped by d
    std::vector<EvalItem> gG[3][kGemmFoldMaxCq];   // GEMM items by d and window width
    size_t smem1 = 0, smem2 = 0, smem2f = 0, smemG = 0;
    int max_d = 1, max_m = 1;
    for (int i = lo; i < hi; ++i) {
      const cco_problem* p = probs_of[i];
      int u = 0;
      while (u < (int)uniq.size() && uniq[u] != p) ++u;
      if (u == (int)uniq.size()) {
        uniq.push_back(p);
        pv.push_back(p->host);
        smem1 = std::max(smem1, p->smem1);
        smem2 = std::max(smem2, eval_smem2(p->host, split));
        smem2f = std::max(smem2f, eval_smem2(p->host, split, true));
        smemG = std::max(smemG, p->smemG);
        max_d = std::max(max_d, p->d);
        max_m = std::max(max_m, p->M);
      }
      const int j = i - lo;
      lv.push_back(eval_lane(R, refs[i], p, u));
      if (p->host.gemm) {
        const int ntG = p->host.ntile1 * p->host.ngblk;
        for (int t = 0; t < ntG; ++t) gG[p->d - 1][p->host.gcq - 1].push_back(EvalItem{j, t});
      }
      // the per-segment pass 1: FP32 lanes, and problems without the GEMM form
      if (!p->host.gemm || may_fp32) {
        const int C = pass1_chunks(p->host, chunks);
        for (int t = 0; t < p->host.ntile1 * C; ++t) g1[p->d - 1].push_back(EvalItem{j, t});
      }
      const int nt2 = pass2_tiles(p->host, split);
      for (int t = 0; t < nt2; ++t) g2[p->d - 1].push_back(EvalItem{j, t});
    }
    std::vector<EvalItem> i1, i2, iG;
    plan.d_off1[0] = plan.d_off2[0] = plan.d_offG[0] = 0;
    for (int D = 0; D < 3; ++D) {
      i1.insert(i1.end(), g1[D].begin(), g1[D].end());
      i2.insert(i2.end(), g2[D].begin(), g2[D].end());
      for (int c = 0; c < kGemmFoldMaxCq; ++c) {
        if (D >= 1) plan.q_offG[D - 1][c] = (int)iG.size();
        iG.insert(iG.end(), gG[D][c].begin(), gG[D][c].end());
      }
      if (D >= 1) plan.q_offG[D - 1][kGemmFoldMaxCq] = (int)iG.size();
      plan.d_off1[D + 1] = (int)i1.size();
      plan.d_off2[D + 1] = (int)i2.size();
      plan.d_offG[D + 1] = (int)iG.size();
    }
    plan.dyn_prec = may_fp32 ? 1 : 0;
    cudaError_t e = upload(&probs, pv, st);
    if (e == cudaSuccess) e = upload(&lanes, lv, st);
    if (e == cudaSuccess) e = upload(&it1, i1, st);
    if (e == cudaSuccess) e = upload(&it2, i2, st);
    if (e == cudaSuccess) e = upload(&itG, iG, st);
    plan.probs = probs;
    plan.lanes = lanes;
    plan.items1 = it1;
    plan.items2 = it2;
    plan.itemsG = itG;
    plan.n_itemsG = (int)iG.size();
    plan.smemG = smemG;
    plan.n_lanes = hi - lo;
    plan.n_items1 = (int)i1.size();
    plan.n_items2 = (int)i2.size();
    plan.max_d = max_d;
    plan.smem1 = smem1;
    plan.smem2 = smem2;
    plan.smem2_f32 = smem2f;
    plan.red_chunks = reduce_chunks(max_m);
    plan.split2 = split;
    plan.chunks1 = chunks;
    plan.want_grad = true;
    return e;
  }
  void release(cudaStream_t st) {
    if (probs) cudaFreeAsync(probs, st);
    if (lanes) cudaFreeAsync(lanes, st);
    if (it1) cudaFreeAsync(it1, st);
    if (it2) cudaFreeAsync(it2, st);
    if (itG) cudaFreeAsync(itG, st);
    itG = nullptr;
    probs = nullptr;
    lanes = nullptr;
    it1 = it2 = nullptr;
  }
};

// ------------------------------------------------------------ tick schedule
// A tick evaluates every RUNNING lane once and runs its minimizer update.
// Ticks are captured into CUDA graphs of `graph_ticks` ticks, with the lanes
// split into `branches` independent graph branches so that one branch's
// FP64-bound evaluation overlaps another branch's HBM-bound update.
struct Schedule {
  int branches = 2;
  int graph_ticks = 16;
  // overlap: branch b > 0 starts half a tick late (after branch 0's first
  // evaluation) and every branch's update kernels run on a high-priority
  // stream, so the HBM-bound update of one branch takes SM slots as the
  // FP64-bound evaluation of another frees them
  int overlap = 0;
};
constexpr int kMaxBranches = 8;
constexpr int kInflight = 3;    // graphs in flight before the host checks completion
constexpr int kMaxInflight = 16;   // CCO_INFLIGHT bound (and the round bounds' slack)

// Lane ranges [bounds[b], bounds[b + 1]) of the branches, balanced by the
// evaluation work (N M) of each lane.
std::vector<int> branch_bounds(const std::vector<const cco_problem*>& probs, int nbr);

// Tuned schedules, cached per shape class (minimizer, lane count and total
// N M bucketed by powers of two, largest d).
bool schedule_cached(const std::vector<const cco_problem*>& probs, Method method, Schedule* out);
void schedule_store(const std::vector<const cco_problem*>& probs, Method method,
                    const Schedule& s);
void schedule_clear();

// The lanes of one launch: their problems, records and the minimizer
// arguments (lanes = d_refs, B = all lanes) that every branch slices.
struct LaneTable {
  RecordShape shape;
  std::vector<const cco_problem*> probs;
  std::vector<LaneRef> refs;
  LaneRef* d_refs = nullptr;
  DescentArgs ds{};
  LbArgs lb{};
  FlArgs fl{};
  MdArgs md{};
  int upload_refs(cudaStream_t st);
  void release(cudaStream_t st);
};

// ------------------------------------------------------------ persistent lanes
// Problems small enough that one CTA evaluates them in a few microseconds run
// their whole descent in one persistent launch (cco_persist.cu) instead of
// graph ticks. The choice depends on the problem alone, so a lane gives the
// same bits alone and in any batch.
constexpr double kPersistMaxFlops = 2.5e5;          // N M F_pair(d) per evaluation
constexpr size_t kPersistMaxSmem = 200 * 1024;      // dynamic shared memory of the launch
bool persist_eligible(const cco_problem* p);
size_t persist_smem(const cco_problem* p);
// One launch per dimension present (bit d-1 of `dims`) over a.B lanes;
// *d_overrun is set to 1 if a lane reached max_ticks while still RUNNING.
cudaError_t persist_descent(const DescentArgs& a, const EvalPlan& plan, size_t smem, int dims,
                            int64_t max_ticks, int* d_overrun, cudaStream_t st);

// One schedule of a lane table captured as an executable graph of
// sch.graph_ticks ticks.
struct TickPlan {
  Method method = Method::Lbfgs;
  Schedule sch;
  int nbr = 1;
  std::vector<int> bounds;
  EvalSet ev[kMaxBranches];
  DescentArgs ds[kMaxBranches];
  LbArgs lb[kMaxBranches];
  FlArgs fl[kMaxBranches];
  MdArgs md[kMaxBranches];
  cudaGraphExec_t exec = nullptr;
  int build(const LaneTable& T, const Schedule& sch, cudaStream_t st);
  cudaError_t tick(cudaStream_t s, int b, const EvalSide* side = nullptr) const;
  cudaError_t update(cudaStream_t s, int b) const;
  int launches_per_tick() const;
  void release(cudaStream_t st);
};

struct RunStats {
  int64_t ticks = 0, launches = 0;
  Schedule schedule;     // of the first (full) table
  int compactions = 0;   // lane-table compactions
};

// Runs tick graphs until no lane of T is RUNNING (CCO_ERR_ROUNDS past
// max_ticks), compacting the lane table as lanes finish. The schedule is
// forced by CCO_BRANCHES / CCO_GRAPH_TICKS / CCO_OVERLAP, cached for the shape class, or
// tuned online on the live lanes; CCO_COMPACT=0 keeps the full table.
int run_lane_table(LaneTable& T, cudaStream_t st, int64_t max_ticks, RunStats* stats);

// L-BFGS settings -> kernel arguments and record shape.
int lbfgs_args(const cco_lbfgs_settings* cfg, LbArgs* A, RecordShape* shape);

}  // namespace cco
