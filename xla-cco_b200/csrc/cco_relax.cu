// Batched relaxations on lane records: the uniform entry points
// (cco_relax_descent / cco_relax_lbfgs, one problem for every lane), the
// mixed ones (a problem per lane), the CUDA-graph tick driver and the
// schedule autotuner they share with the serving pool (cco_serve.cu).
//
// Reference: relax (src/xla_cco/minimize/__init__.py:102-151) runs host
// rounds of jitted chunks over the RUNNING lanes, padded to a power of two,
// with a host sync per round. Here every lane is a device state machine
// (cco_opt.cu); the host only launches captured graphs of ticks and checks,
// a few graphs behind, whether any lane is still RUNNING.
#include <cmath>
#include <cstdlib>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "cco.h"
#include "cco_host.cuh"

using namespace cco;

namespace cco {

std::vector<int> branch_bounds(const std::vector<const cco_problem*>& probs, int nbr) {
  const int B = (int)probs.size();
  std::vector<double> cum(B + 1, 0.0);
  for (int i = 0; i < B; ++i) cum[i + 1] = cum[i] + (double)probs[i]->N * probs[i]->M;
  std::vector<int> b(nbr + 1, 0);
  b[nbr] = B;
  for (int k = 1; k < nbr; ++k) {
    const double target = cum[B] * k / nbr;
    int i = (int)(std::lower_bound(cum.begin(), cum.end(), target) - cum.begin());
    i = std::max(i, b[k - 1] + 1);
    i = std::min(i, B - (nbr - k));
    b[k] = i;
  }
  return b;
}

namespace {

// ------------------------------------------------------------ schedule cache
// Tuned schedules are cached per shape class: the minimizer, the lane count
// and the total evaluation work (sum of N M), each bucketed by powers of two,
// and the largest d.
using ShapeKey = std::tuple<int, int, int, int>;
std::mutex g_sched_mu;
std::map<ShapeKey, Schedule> g_sched;

ShapeKey shape_key(const std::vector<const cco_problem*>& probs, Method method) {
  double work = 0.0;
  int maxd = 1;
  for (const cco_problem* p : probs) {
    work += (double)p->N * p->M;
    maxd = std::max(maxd, p->d);
  }
  const int lb = (int)std::floor(std::log2((double)probs.size()));
  const int lw = (int)std::floor(std::log2(std::max(work, 1.0)));
  return ShapeKey((int)method, lb, lw, maxd);
}

int env_int(const char* name, int fallback) {
  const char* v = getenv(name);
  return v ? atoi(v) : fallback;
}

}  // namespace

bool schedule_cached(const std::vector<const cco_problem*>& probs, Method method, Schedule* out) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  auto it = g_sched.find(shape_key(probs, method));
  if (it == g_sched.end()) return false;
  *out = it->second;
  return true;
}

void schedule_store(const std::vector<const cco_problem*>& probs, Method method,
                    const Schedule& s) {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  g_sched[shape_key(probs, method)] = s;
}

void schedule_clear() {
  std::lock_guard<std::mutex> lk(g_sched_mu);
  g_sched.clear();
}

// ------------------------------------------------------------ tick plans
int TickPlan::build(const LaneTable& T, const Schedule& sch, cudaStream_t st) {
  release(st);
  this->sch = sch;
  const int B = (int)T.refs.size();
  nbr = std::max(1, std::min(sch.branches, std::min(kMaxBranches, B)));
  bounds = branch_bounds(T.probs, nbr);
  for (int b = 0; b < nbr; ++b) {
    const int lo = bounds[b], hi = bounds[b + 1];
    const bool may_fp32 = T.shape.method == Method::Lbfgs && T.lb.prec0 == PREC_FP32;
    CCO_CUDA(ev[b].build(T.shape, T.refs, T.probs, lo, hi, st, may_fp32));
    int nblk = 1, nch = 1;
    for (int i = lo; i < hi; ++i) {
      nblk = std::max(nblk, lb_nblk(T.refs[i].ld));
      nch = std::max(nch, lb_achunks(T.refs[i].ld));
    }
    if (T.shape.method == Method::Flow) {
      FlArgs a = T.fl;
      a.B = hi - lo;
      a.lanes = T.d_refs + lo;
      fl[b] = a;
    } else if (T.shape.method == Method::Md) {
      MdArgs a = T.md;
      a.B = hi - lo;
      a.lanes = T.d_refs + lo;
      md[b] = a;
    } else if (T.shape.method == Method::Descent) {
      DescentArgs a = T.ds;
      a.B = hi - lo;
      a.lanes = T.d_refs + lo;
      ds[b] = a;
    } else {
      LbArgs a = T.lb;
      a.B = hi - lo;
      a.lanes = T.d_refs + lo;
      a.nblkB = nblk;
      a.nchA = nch;
      lb[b] = a;
    }
  }
  // capture graph_ticks ticks of every branch; branches fork from and join
  // back into the first capture stream
  cudaStream_t cap[kMaxBranches] = {};
  cudaEvent_t fork = nullptr, join[kMaxBranches] = {};
  EvalSide side[kMaxBranches] = {};   // per-dimension side streams of each branch
  cudaError_t e = cudaSuccess;
  for (int b = 0; b < nbr && e == cudaSuccess; ++b)
    e = cudaStreamCreateWithFlags(&cap[b], cudaStreamNonBlocking);
  for (int b = 0; b < nbr && e == cudaSuccess; ++b) {
    if (eval_dims(ev[b].plan) < 2) continue;   // one dimension: no side streams
    for (int u = 0; u < 2 && e == cudaSuccess; ++u) {
      e = cudaStreamCreateWithFlags(&side[b].aux[u], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&side[b].join[u], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&side[b].fork, cudaEventDisableTiming);
  }
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
  for (int b = 0; b < nbr && e == cudaSuccess; ++b)
    e = cudaEventCreateWithFlags(&join[b], cudaEventDisableTiming);
  // overlap schedules: per-branch high-priority update streams (kernel nodes
  // take the capturing stream's priority; the graph runs with node priorities)
  const bool overlap = sch.overlap && nbr > 1;
  cudaStream_t up[kMaxBranches] = {};
  cudaEvent_t ev_done[kMaxBranches] = {}, up_done[kMaxBranches] = {};
  cudaEvent_t phase = nullptr;
  if (overlap && e == cudaSuccess) {
    int least = 0, greatest = 0;
    e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
    for (int b = 0; b < nbr && e == cudaSuccess; ++b) {
      e = cudaStreamCreateWithPriority(&up[b], cudaStreamNonBlocking, greatest);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev_done[b], cudaEventDisableTiming);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&up_done[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&phase, cudaEventDisableTiming);
  }
  // the capture streams must see the uploads made on `st`
  cudaEvent_t ready = nullptr;
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ready, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(ready, st);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(cap[0], ready, 0);
  cudaGraph_t graph = nullptr;
  if (e == cudaSuccess) e = cudaStreamBeginCapture(cap[0], cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    e = cudaEventRecord(fork, cap[0]);
    for (int b = 1; b < nbr && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(cap[b], fork, 0);
    for (int t = 0; t < sch.graph_ticks && e == cudaSuccess; ++t)
      for (int b = 0; b < nbr && e == cudaSuccess; ++b) {
        const EvalSide* sd = side[b].fork ? &side[b] : nullptr;
        if (!overlap) {
          e = tick(cap[b], b, sd);
          continue;
        }
        if (t == 0 && b > 0) e = cudaStreamWaitEvent(cap[b], phase, 0);
        if (e == cudaSuccess) e = eval_launch(ev[b].plan, cap[b], sd);
        if (e == cudaSuccess && t == 0 && b == 0) e = cudaEventRecord(phase, cap[0]);
        if (e == cudaSuccess) e = cudaEventRecord(ev_done[b], cap[b]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(up[b], ev_done[b], 0);
        if (e == cudaSuccess) e = update(up[b], b);
        if (e == cudaSuccess) e = cudaEventRecord(up_done[b], up[b]);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(cap[b], up_done[b], 0);
      }
    for (int b = 1; b < nbr && e == cudaSuccess; ++b) {
      e = cudaEventRecord(join[b], cap[b]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(cap[0], join[b], 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(cap[0], &graph);
    if (e == cudaSuccess) e = e2;
  }
  if (e == cudaSuccess)
    e = cudaGraphInstantiate(&exec, graph, overlap ? cudaGraphInstantiateFlagUseNodePriority : 0);
  if (graph) cudaGraphDestroy(graph);
  for (int b = 0; b < nbr; ++b) {
    if (cap[b]) cudaStreamDestroy(cap[b]);
    if (join[b]) cudaEventDestroy(join[b]);
    if (up[b]) cudaStreamDestroy(up[b]);
    if (ev_done[b]) cudaEventDestroy(ev_done[b]);
    if (up_done[b]) cudaEventDestroy(up_done[b]);
    for (int u = 0; u < 2; ++u) {
      if (side[b].aux[u]) cudaStreamDestroy(side[b].aux[u]);
      if (side[b].join[u]) cudaEventDestroy(side[b].join[u]);
    }
    if (side[b].fork) cudaEventDestroy(side[b].fork);
  }
  if (fork) cudaEventDestroy(fork);
  if (phase) cudaEventDestroy(phase);
  if (ready) cudaEventDestroy(ready);
  if (e != cudaSuccess) return cuda_fail(e, "tick graph capture");
  return CCO_OK;
}

cudaError_t TickPlan::tick(cudaStream_t s, int b, const EvalSide* side) const {
  cudaError_t e = eval_launch(ev[b].plan, s, side);
  if (e != cudaSuccess) return e;
  return update(s, b);
}

cudaError_t TickPlan::update(cudaStream_t s, int b) const {
  if (method == Method::Flow) return flow_update(fl[b], s);
  if (method == Method::Md) return md_update(md[b], s);
  return method == Method::Descent ? descent_update(ds[b], s) : lbfgs_update(lb[b], s);
}

int TickPlan::launches_per_tick() const {
  // the evaluation kernels each branch's plan issues + the update kernels
  // (L-BFGS: probe, pass A, scalar, pass B; MD segments: + the wave sums and
  // the per-wave observables)
  const int md_waves = method == Method::Md && md[0].w > md[0].nc ? 1 : 0;
  const int md_obs = method == Method::Md && md[0].w > 0 ? 1 : 0;
  const int upd = method == Method::Lbfgs ? 4 : 1 + md_waves + md_obs;
  int n = 0;
  for (int b = 0; b < nbr; ++b) n += eval_kernels(ev[b].plan) + upd;
  return n;
}

void TickPlan::release(cudaStream_t st) {
  if (exec) cudaGraphExecDestroy(exec);
  exec = nullptr;
  for (int b = 0; b < kMaxBranches; ++b) ev[b].release(st);
}

// ------------------------------------------------------------ lane tables
int LaneTable::upload_refs(cudaStream_t st) {
  if (d_refs) cudaFreeAsync(d_refs, st);
  d_refs = nullptr;
  CCO_CUDA(upload(&d_refs, refs, st));
  return CCO_OK;
}

void LaneTable::release(cudaStream_t st) {
  if (d_refs) cudaFreeAsync(d_refs, st);
  d_refs = nullptr;
}

// ------------------------------------------------------------ the tick driver
namespace {

// Candidate schedules of the online tuner: 1, 2, 3, 4, 6 or 8 branches of
// at least 8 lanes. (On the 256-lane d = 2 relax: 260, 268, 254 and 256 ms
// per relaxation at 3, 4, 6 and 8 branches. The overlap form, CCO_OVERLAP=1,
// measured slower than plain branches - 906 vs 955 relaxations/s at two
// branches - and is not a candidate.)
std::vector<Schedule> candidates(int B) {
  std::vector<Schedule> c;
  for (int nb : {1, 2, 3, 4, 6, 8}) {
    if (nb > kMaxBranches || (nb > 1 && B / nb < 8)) break;
    Schedule s;
    s.branches = nb;
    s.graph_ticks = 16;
    c.push_back(s);
  }
  return c;
}

// Pinned host buffer owned by the calling thread, grown on demand
// (cudaHostAlloc is slow and may synchronize, so it stays out of most calls).
int64_t* pinned_status(size_t count) {
  static thread_local int64_t* buf = nullptr;
  static thread_local size_t cap = 0;
  if (count > cap) {
    if (buf) cudaFreeHost(buf);
    buf = nullptr;
    cap = 0;
    const size_t n = std::max<size_t>(count, 4096);
    if (cudaHostAlloc(reinterpret_cast<void**>(&buf), n * sizeof(int64_t), cudaHostAllocDefault) !=
        cudaSuccess)
      return nullptr;
    cap = n;
  }
  return buf;
}

// Online tuning: graphs of each candidate on the live lanes C, timed with
// events, then the fastest per tick. Every candidate advances every lane by
// the same ticks, so results do not depend on which schedule wins.
int tune_schedule(const LaneTable& C, cudaStream_t st, int64_t max_ticks, int64_t* ticks,
                  int64_t* launches, Schedule* out) {
  // Two rounds, the second in reverse order, each candidate timed once per
  // round: the lanes' work drifts while they advance (histories fill, rescale
  // passes restart them), and the mean of a forward and a backward visit
  // cancels a drift that is linear in time.
  const std::vector<Schedule> cand = candidates((int)C.refs.size());
  const size_t nc = cand.size();
  std::vector<cudaEvent_t> t0(2 * nc, nullptr), t1(2 * nc, nullptr);
  std::vector<int> ran(2 * nc, 0);
  int rc = CCO_OK;
  cudaError_t e = cudaSuccess;
  for (size_t c = 0; c < 2 * nc && e == cudaSuccess; ++c) {
    e = cudaEventCreate(&t0[c]);
    if (e == cudaSuccess) e = cudaEventCreate(&t1[c]);
  }
  for (size_t v = 0; v < 2 * nc && rc == CCO_OK && e == cudaSuccess && *ticks < max_ticks; ++v) {
    const size_t c = v < nc ? v : 2 * nc - 1 - v;
    TickPlan P;
    P.method = C.shape.method;
    rc = P.build(C, cand[c], st);
    if (rc != CCO_OK) break;
    e = cudaEventRecord(t0[v], st);
    if (e == cudaSuccess) e = cudaGraphLaunch(P.exec, st);
    if (e == cudaSuccess) e = cudaEventRecord(t1[v], st);
    ran[v] = e == cudaSuccess;
    *ticks += cand[c].graph_ticks;
    *launches += (int64_t)cand[c].graph_ticks * P.launches_per_tick();
    P.release(st);
  }
  if (rc == CCO_OK && e == cudaSuccess) e = cudaStreamSynchronize(st);
  std::vector<float> sum(nc, 0.f);
  std::vector<int> cnt(nc, 0);
  for (size_t v = 0; v < 2 * nc && e == cudaSuccess && rc == CCO_OK; ++v) {
    if (!ran[v]) continue;
    const size_t c = v < nc ? v : 2 * nc - 1 - v;
    float x = 0.f;
    if (cudaEventElapsedTime(&x, t0[v], t1[v]) == cudaSuccess) {
      sum[c] += x / cand[c].graph_ticks;
      cnt[c] += 1;
    } else {
      cudaGetLastError();
    }
  }
  std::vector<float> ms(nc, 1e30f);
  int best = 0;
  for (size_t c = 0; c < nc; ++c) {
    if (cnt[c] > 0) ms[c] = sum[c] / cnt[c];
    if (ms[c] < ms[best]) best = (int)c;
  }
  for (size_t c = 0; c < 2 * nc; ++c) {
    if (t0[c]) cudaEventDestroy(t0[c]);
    if (t1[c]) cudaEventDestroy(t1[c]);
  }
  if (rc != CCO_OK) return rc;
  if (e != cudaSuccess) return cuda_fail(e, "schedule tuning");
  Schedule s = cand[best];
  // graphs of about 8 ms of device work: with three in flight the device has
  // ~20 ms queued, so a host thread descheduled on a busy host does not leave
  // it idle; the graphs that run past the last lane's completion cost little
  // (their kernels exit at once for finished lanes)
  const double tick_ms = ms[best] < 1e29f ? ms[best] : 0.2;
  const int gt = (int)std::lround(8.0 / std::max(tick_ms, 1e-3));
  s.graph_ticks = std::max(4, std::min(32, gt));
  *out = s;
  return CCO_OK;
}

}  // namespace

// The tick driver. Graphs run on a lane table C that starts as all of T and
// is compacted - rebuilt from the lanes a status snapshot shows RUNNING -
// whenever at most half of it still runs, so finished lanes stop costing
// launch slots (the reference's per-round compaction of active lanes,
// minimize/__init__.py:75-99, without moving any lane's state). Each
// compaction looks up or re-tunes the schedule for the smaller table.
int run_lane_table(LaneTable& T, cudaStream_t st, int64_t max_ticks, RunStats* stats) {
  const int B = (int)T.refs.size();
  const int inflight = std::max(1, std::min(kMaxInflight, env_int("CCO_INFLIGHT", kInflight)));
  const int kSlots = inflight + 1;
  int64_t* d_status = nullptr;
  int64_t* h_status = pinned_status((size_t)kSlots * B);
  if (!h_status) return fail(CCO_ERR_OOM, "pinned status buffer");
  CCO_CUDA(pool_alloc(&d_status, sizeof(int64_t) * kSlots * B, st));
  cudaEvent_t ev[kMaxInflight + 1];
  int ver[kMaxInflight + 1] = {}, rows[kMaxInflight + 1] = {};
  for (int i = 0; i < kSlots; ++i) CCO_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  int64_t ticks = 0, launches = 0;
  int rc = CCO_OK;
  cudaError_t e = cudaSuccess;
  bool done = false;

  const int force_br = env_int("CCO_BRANCHES", 0), force_gt = env_int("CCO_GRAPH_TICKS", 0);
  const int force_ov = env_int("CCO_OVERLAP", -1);
  const bool tune = env_int("CCO_AUTOTUNE", 1) != 0;
  const bool compact = env_int("CCO_COMPACT", 1) != 0;

  LaneTable C;           // the live table (owns its own device copy of refs)
  C.shape = T.shape;
  C.ds = T.ds;
  C.lb = T.lb;
  C.fl = T.fl;
  C.md = T.md;
  C.refs = T.refs;
  C.probs = T.probs;
  Schedule chosen, first;
  bool first_set = false;
  TickPlan P;
  P.method = T.shape.method;
  int version = 0;
  // An L-BFGS table is tuned only once its lanes' histories have filled: in
  // the first ticks the HBM-bound update is short, so schedules that overlap
  // it with the FP64-bound evaluation of another branch cannot show their
  // gain. Until then it runs the default schedule.
  constexpr int64_t kTuneAfterTicks = 128;
  bool defer_tune = false;

  // (re)start on table C: schedule, graph
  auto start = [&]() -> int {
    int r = C.upload_refs(st);
    if (r != CCO_OK) return r;
    C.ds.lanes = C.d_refs;
    C.ds.B = (int)C.refs.size();
    C.lb.lanes = C.d_refs;
    C.lb.B = (int)C.refs.size();
    C.fl.lanes = C.d_refs;
    C.fl.B = (int)C.refs.size();
    C.md.lanes = C.d_refs;
    C.md.B = (int)C.refs.size();
    Schedule s;
    if (force_br > 0 || force_gt > 0 || force_ov >= 0) {
      if (force_br > 0) s.branches = force_br;
      if (force_gt > 0) s.graph_ticks = force_gt;
      if (force_ov >= 0) s.overlap = force_ov;
    } else if (!schedule_cached(C.probs, C.shape.method, &s) && tune) {
      defer_tune = C.shape.method == Method::Lbfgs && ticks < kTuneAfterTicks;
      if (!defer_tune) {
        r = tune_schedule(C, st, max_ticks, &ticks, &launches, &s);
        if (r != CCO_OK) return r;
        schedule_store(C.probs, C.shape.method, s);
      }
    }
    chosen = s;
    if (!first_set) {
      first = s;
      first_set = true;
    }
    ++version;
    return P.build(C, chosen, st);
  };
  rc = start();

  int launched = 0, checked = 0;
  auto land = [&]() -> int {
    const int slot = checked % kSlots;
    CCO_CUDA(cudaEventSynchronize(ev[slot]));
    ++checked;
    const int64_t* h = h_status + (size_t)slot * B;
    int running = 0;
    for (int i = 0; i < rows[slot]; ++i) running += h[i] == CCO_STATUS_RUNNING;
    if (running == 0) {
      done = true;
      return CCO_OK;
    }
    const int n = (int)C.refs.size();
    if (!compact || ver[slot] != version || n < 2 || 2 * running > n) return CCO_OK;
    // compaction: keep the lanes this snapshot of the current table shows running
    std::vector<LaneRef> refs;
    std::vector<const cco_problem*> probs;
    for (int i = 0; i < n; ++i)
      if (h[i] == CCO_STATUS_RUNNING) {
        refs.push_back(C.refs[i]);
        probs.push_back(C.probs[i]);
      }
    // The graphs still in flight on the old table keep running while the new
    // plan is captured: stream order puts the new graphs after them, the old
    // plan's buffers are freed stream-ordered, and their status snapshots
    // (older version, old row order) only feed the all-finished test.
    C.refs.swap(refs);
    C.probs.swap(probs);
    P.release(st);
    return start();
  };

  while (rc == CCO_OK && e == cudaSuccess && !done) {
    if (ticks >= max_ticks) break;
    e = cudaGraphLaunch(P.exec, st);
    if (e != cudaSuccess) break;
    ticks += chosen.graph_ticks;
    launches += (int64_t)chosen.graph_ticks * P.launches_per_tick() + 1;
    const int slot = launched % kSlots;
    const int n = (int)C.refs.size();
    e = gather_status(C.d_refs, n, d_status + (size_t)slot * B, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(h_status + (size_t)slot * B, d_status + (size_t)slot * B,
                          sizeof(int64_t) * n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[slot], st);
    ver[slot] = version;
    rows[slot] = n;
    ++launched;
    if (e == cudaSuccess && launched - checked > inflight) rc = land();
    if (rc == CCO_OK && e == cudaSuccess && !done && defer_tune && ticks >= kTuneAfterTicks) {
      P.release(st);   // the deferred tuning, on the same table
      rc = start();
    }
  }
  // drain the launches still in flight, oldest first
  while (rc == CCO_OK && e == cudaSuccess && !done && checked < launched) rc = land();
  if (rc == CCO_OK) {
    if (e != cudaSuccess) rc = cuda_fail(e, "relax ticks");
    else if (!done) rc = fail(CCO_ERR_ROUNDS, "relax did not finish within the round bound (%lld ticks)", (long long)max_ticks);
  }
  P.release(st);
  C.release(st);
  for (int i = 0; i < kSlots; ++i) cudaEventDestroy(ev[i]);
  cudaFreeAsync(d_status, st);
  cudaStreamSynchronize(st);
  if (stats) {
    stats->ticks = ticks;
    stats->launches = launches;
    stats->schedule = first;
    stats->compactions = version - 1;
  }
  return rc;
}

}  // namespace cco

// ------------------------------------------------------------ entry points
namespace {

bool out_ok(const cco_relax_out* o) {
  return o && o->s && o->energy && o->grad_norm && o->n_evals && o->n_iters && o->status;
}

int check_traj(const cco_relax_out* out, bool rec) {
  if (rec && (!out->traj_s || !out->traj_energy || !out->traj_step || !out->traj_iteration ||
              !out->traj_count))
    return fail(CCO_ERR_ARG, "trajectory recording needs the traj_* outputs");
  return CCO_OK;
}

// Lane table of a one-shot relaxation: records carved from one allocation,
// positions packed in the caller's order, trajectory rows `cap` per lane.
int make_table(cco_problem* const* probs, int B, const RecordShape& shape, int64_t cap,
               cudaStream_t st, LaneTable* T, double** records) {
  if (B < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  T->shape = shape;
  T->probs.resize(B);
  T->refs.resize(B);
  size_t total = 0;
  int device = -1;
  for (int i = 0; i < B; ++i) {
    const cco_problem* p = probs[i];
    if (!p) return fail(CCO_ERR_ARG, "null problem for lane %d", i);
    if (device < 0) device = p->device;
    if (p->device != device) return fail(CCO_ERR_ARG, "lanes must share one device");
    T->probs[i] = p;
    total += record_doubles(shape, p);
  }
  CCO_CUDA(pool_alloc(records, total * sizeof(double), st));
  size_t o = 0;
  int64_t soff = 0;
  for (int i = 0; i < B; ++i) {
    const cco_problem* p = T->probs[i];
    LaneRef& r = T->refs[i];
    r.rec = *records + o;
    r.nd = p->N * p->d;
    r.ld = pad4(r.nd);
    r.soff = soff;
    r.toff = cap * soff;
    r.idx = i;
    r.n = p->N;
    o += record_doubles(shape, p);
    soff += r.nd;
  }
  return T->upload_refs(st);
}

// The descent lanes of a table split by problem size: the small ones run one
// persistent launch (on a side stream when graph ticks run beside it), the
// others form `large`, the table of the graph driver.
struct PersistRun {
  LaneTable large;
  EvalSet ev;
  LaneRef* d_small = nullptr;
  int* d_over = nullptr;
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  int64_t launches = 0;
  bool any = false;

  int start(const LaneTable& T, cudaStream_t st, int64_t max_ticks) {
    large.shape = T.shape;
    large.ds = T.ds;
    std::vector<LaneRef> small;
    std::vector<const cco_problem*> sprobs;
    size_t smem = 0;
    int dims = 0;
    for (size_t i = 0; i < T.refs.size(); ++i) {
      const cco_problem* p = T.probs[i];
      if (persist_eligible(p)) {
        small.push_back(T.refs[i]);
        sprobs.push_back(p);
        smem = std::max(smem, persist_smem(p));
        dims |= 1 << (p->d - 1);
      } else {
        large.refs.push_back(T.refs[i]);
        large.probs.push_back(p);
      }
    }
    if (!large.refs.empty()) {
      const int rc = large.upload_refs(st);
      if (rc != CCO_OK) return rc;
    }
    if (small.empty()) return CCO_OK;
    any = true;
    CCO_CUDA(upload(&d_small, small, st));
    CCO_CUDA(ev.build(T.shape, small, sprobs, 0, (int)small.size(), st));
    CCO_CUDA(pool_alloc(&d_over, sizeof(int), st));
    CCO_CUDA(cudaMemsetAsync(d_over, 0, sizeof(int), st));
    DescentArgs a = T.ds;
    a.B = (int)small.size();
    a.lanes = d_small;
    cudaStream_t run = st;
    if (!large.refs.empty()) {   // beside the graph ticks of the large lanes
      CCO_CUDA(cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking));
      CCO_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
      CCO_CUDA(cudaEventCreateWithFlags(&join, cudaEventDisableTiming));
      CCO_CUDA(cudaEventRecord(fork, st));
      CCO_CUDA(cudaStreamWaitEvent(side, fork, 0));
      run = side;
    }
    CCO_CUDA(persist_descent(a, ev.plan, smem, dims, max_ticks, d_over, run));
    launches = __builtin_popcount(dims);
    if (side) CCO_CUDA(cudaEventRecord(join, side));
    return CCO_OK;
  }

  // Joins the persistent launch into st; CCO_ERR_ROUNDS if a lane overran.
  int finish(cudaStream_t st) {
    if (!any) return CCO_OK;
    if (side) CCO_CUDA(cudaStreamWaitEvent(st, join, 0));
    int over = 0;
    CCO_CUDA(cudaMemcpyAsync(&over, d_over, sizeof(int), cudaMemcpyDeviceToHost, st));
    CCO_CUDA(cudaStreamSynchronize(st));
    if (over) return fail(CCO_ERR_ROUNDS, "relax did not finish within the round bound");
    return CCO_OK;
  }

  void release(cudaStream_t st) {
    if (side && join) cudaStreamWaitEvent(st, join, 0);
    ev.release(st);
    large.release(st);
    if (d_small) cudaFreeAsync(d_small, st);
    if (d_over) cudaFreeAsync(d_over, st);
    if (side) cudaStreamDestroy(side);
    if (fork) cudaEventDestroy(fork);
    if (join) cudaEventDestroy(join);
    side = nullptr;
    fork = join = nullptr;
  }
};

int relax_descent_set(cco_problem* const* probs, int B, cudaStream_t st, const double* s0,
                      const cco_descent_settings* cfg, cco_relax_out* out) {
  if (!cfg || !s0) return fail(CCO_ERR_ARG, "null argument");
  if (!out_ok(out)) return fail(CCO_ERR_ARG, "incomplete output struct");
  if (cfg->max_evals < 0) return fail(CCO_ERR_ARG, "max_evals must be >= 0");
  if (B < 1 || !probs[0]) return fail(CCO_ERR_ARG, "need at least one configuration");
  const bool rec = cfg->record_every > 0 && cfg->max_records > 0;
  if (check_traj(out, rec) != CCO_OK) return CCO_ERR_ARG;
  DeviceGuard guard(probs[0]->device);
  RecordShape shape;
  shape.method = Method::Descent;
  LaneTable T;
  DescentArgs& a = T.ds;
  a.step_init = cfg->step_init;
  a.step_min = cfg->step_min;
  a.shrink = cfg->shrink;
  a.grow = cfg->grow;
  a.rel_tol = cfg->rel_tol;
  a.energy_tol = cfg->energy_tol;
  a.max_iters = cfg->max_evals / 2;
  a.rec_every = rec ? cfg->record_every : 1;
  a.rec_cap = rec ? cfg->max_records : 0;
  if (rec) {
    a.traj_s = out->traj_s;
    a.traj_e = out->traj_energy;
    a.traj_step = out->traj_step;
    a.traj_it = out->traj_iteration;
    a.traj_count = out->traj_count;
  }
  double* records = nullptr;
  int rc = make_table(probs, B, shape, a.rec_cap, st, &T, &records);
  if (rc != CCO_OK) {
    if (records) cudaFreeAsync(records, st);
    return rc;
  }
  a.B = B;
  a.lanes = T.d_refs;
  CCO_CUDA(descent_init(a, s0, st));
  const int64_t max_ticks = 1 + a.max_iters + 4 * (kMaxInflight + 1) * 32;
  RunStats rs;
  PersistRun pr;
  rc = pr.start(T, st, max_ticks);
  if (rc == CCO_OK && !pr.large.refs.empty()) rc = run_lane_table(pr.large, st, max_ticks, &rs);
  if (rc == CCO_OK) rc = pr.finish(st);
  if (rc == CCO_OK) {
    cudaError_t e = descent_finalize(a, out->s, out->energy, out->grad_norm, out->n_evals,
                                     out->n_iters, out->status, out->latency_ns, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "descent_finalize");
  }
  out->ticks = rs.ticks;
  out->launches = rs.launches + 3 + pr.launches;
  out->branches = rs.schedule.branches;
  out->overlap = rs.schedule.overlap;
  out->graph_ticks = rs.schedule.graph_ticks;
  pr.release(st);
  T.release(st);
  cudaFreeAsync(records, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "relax descent");
  return rc;
}

std::mutex g_cfg_mu;
size_t g_scalar_smem_configured = 0;

int relax_lbfgs_set(cco_problem* const* probs, int B, cudaStream_t st, const double* s0,
                    const cco_lbfgs_settings* cfg, cco_relax_out* out) {
  if (!cfg || !s0) return fail(CCO_ERR_ARG, "null argument");
  if (!out_ok(out)) return fail(CCO_ERR_ARG, "incomplete output struct");
  if (cfg->n_rescales < 1 || cfg->n_rescales > CCO_MAX_RESCALES)
    return fail(CCO_ERR_ARG, "need 1..%d rescale passes", CCO_MAX_RESCALES);
  if (cfg->memory < 1) return fail(CCO_ERR_ARG, "memory must be >= 1");
  if (cfg->memory > 256) return fail(CCO_ERR_ARG, "memory must be <= 256 on this build");
  if (cfg->max_linesearch_steps < 1) return fail(CCO_ERR_ARG, "max_linesearch_steps must be >= 1");
  if (cfg->precision != 0 && cfg->precision != 1) return fail(CCO_ERR_ARG, "precision must be 0 or 1");
  if (B < 1 || !probs[0]) return fail(CCO_ERR_ARG, "need at least one configuration");
  const bool rec = cfg->record_every > 0 && cfg->max_records > 0;
  if (check_traj(out, rec) != CCO_OK) return CCO_ERR_ARG;
  DeviceGuard guard(probs[0]->device);
  LaneTable T;
  LbArgs& A = T.lb;
  int rc = lbfgs_args(cfg, &A, &T.shape);
  if (rc != CCO_OK) return rc;
  if (rec) {
    A.traj_s = out->traj_s;
    A.traj_e = out->traj_energy;
    A.traj_step = out->traj_step;
    A.traj_it = out->traj_iteration;
    A.traj_count = out->traj_count;
  }
  A.rec_every = rec ? cfg->record_every : 1;
  A.rec_cap = rec ? cfg->max_records : 0;
  double* records = nullptr;
  rc = make_table(probs, B, T.shape, A.rec_cap, st, &T, &records);
  if (rc != CCO_OK) {
    if (records) cudaFreeAsync(records, st);
    return rc;
  }
  A.B = B;
  A.lanes = T.d_refs;
  int nblk = 1, nch = 1;
  for (const LaneRef& r : T.refs) {
    nblk = std::max(nblk, lb_nblk(r.ld));
    nch = std::max(nch, lb_achunks(r.ld));
  }
  A.nblkB = nblk;
  A.nchA = nch;
  CCO_CUDA(lbfgs_init(A, s0, st));
  const int64_t max_ticks =
      1 + (int64_t)cfg->n_rescales * (cfg->max_evals_per_pass + cfg->max_linesearch_steps + 1) +
      4 * (kMaxInflight + 1) * 32;
  RunStats rs;
  rc = run_lane_table(T, st, max_ticks, &rs);
  if (rc == CCO_OK) {
    cudaError_t e = lbfgs_finalize(A, out->s, out->energy, out->grad_norm, out->n_evals,
                                   out->n_iters, out->status, out->latency_ns, out->n_evals_fp32,
                                   st);
    if (e != cudaSuccess) rc = cuda_fail(e, "lbfgs_finalize");
  }
  out->ticks = rs.ticks;
  out->launches = rs.launches + 3;
  out->branches = rs.schedule.branches;
  out->overlap = rs.schedule.overlap;
  out->graph_ticks = rs.schedule.graph_ticks;
  T.release(st);
  cudaFreeAsync(records, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "relax lbfgs");
  return rc;
}

}  // namespace

namespace cco {

// Settings -> kernel arguments shared by the one-shot relaxation and the
// serving pool; also sizes the scalar kernel's shared-memory triangles.
int lbfgs_args(const cco_lbfgs_settings* cfg, LbArgs* A, RecordShape* shape) {
  *A = LbArgs{};
  const int m = (int)cfg->memory;
  A->m = m;
  A->n_pass = cfg->n_rescales;
  for (int i = 0; i < CCO_MAX_RESCALES; ++i)
    A->rescales[i] = i < cfg->n_rescales ? cfg->rescales[i] : 1.0;
  A->energy_tol = cfg->energy_tol;
  A->grad_tol = cfg->grad_tol;
  A->budget = cfg->max_evals_per_pass;
  A->patience = cfg->stagnation_patience;
  A->max_ls = cfg->max_linesearch_steps;
  A->rec_every = 1;
  A->rec_cap = 0;
  A->prec0 = cfg->precision == 1 ? PREC_FP32 : PREC_FP64;
  A->keep_s0 = cfg->precision == 1 ? 1 : 0;
  const size_t tri_bytes = lbfgs_update_smem(m);
  const bool in_smem = tri_bytes <= 200 * 1024;
  A->smem_tri = in_smem ? tri_bytes : 0;
  A->tri_len = in_smem ? 0 : m * (m + 1);
  if (in_smem) {
    std::lock_guard<std::mutex> lk(g_cfg_mu);
    if (g_scalar_smem_configured < 200 * 1024) {
      CCO_CUDA(lbfgs_configure(200 * 1024));
      g_scalar_smem_configured = 200 * 1024;
    }
  }
  shape->method = Method::Lbfgs;
  shape->m = m;
  shape->tri_len = A->tri_len;
  shape->keep_s0 = A->keep_s0;
  return CCO_OK;
}

}  // namespace cco

extern "C" int cco_relax_descent(cco_problem* p, void* stream, int batch, const double* s0,
                                 const cco_descent_settings* cfg, int chunk_iters,
                                 cco_relax_out* out) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  std::vector<cco_problem*> probs(batch, p);
  return relax_descent_set(probs.data(), batch, (cudaStream_t)stream, s0, cfg, out);
}

extern "C" int cco_relax_lbfgs(cco_problem* p, void* stream, int batch, const double* s0,
                               const cco_lbfgs_settings* cfg, int chunk_iters,
                               cco_relax_out* out) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  std::vector<cco_problem*> probs(batch, p);
  return relax_lbfgs_set(probs.data(), batch, (cudaStream_t)stream, s0, cfg, out);
}

extern "C" int cco_relax_descent_mixed(cco_problem* const* problems, void* stream, int batch,
                                       const double* s0, const cco_descent_settings* cfg,
                                       int chunk_iters, cco_relax_out* out) {
  if (!problems) return fail(CCO_ERR_ARG, "null problem array");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  return relax_descent_set(problems, batch, (cudaStream_t)stream, s0, cfg, out);
}

extern "C" int cco_relax_lbfgs_mixed(cco_problem* const* problems, void* stream, int batch,
                                     const double* s0, const cco_lbfgs_settings* cfg,
                                     int chunk_iters, cco_relax_out* out) {
  if (!problems) return fail(CCO_ERR_ARG, "null problem array");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  return relax_lbfgs_set(problems, batch, (cudaStream_t)stream, s0, cfg, out);
}

namespace {

// B, B^-T and (B B^T)^-1 of a d x d basis into 3x3 row-major slots (Gauss-
// Jordan with partial pivoting). False if the basis is singular.
bool basis_mats(const double* basis, int d, double* out27) {
  double a[3][6] = {};
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      a[i][j] = basis[i * d + j];
      a[i][d + j] = i == j ? 1.0 : 0.0;
    }
  for (int c = 0; c < d; ++c) {
    int piv = c;
    for (int i = c + 1; i < d; ++i)
      if (std::fabs(a[i][c]) > std::fabs(a[piv][c])) piv = i;
    if (a[piv][c] == 0.0 || !std::isfinite(a[piv][c])) return false;
    if (piv != c)
      for (int j = 0; j < 2 * d; ++j) std::swap(a[c][j], a[piv][j]);
    const double inv = 1.0 / a[c][c];
    for (int j = 0; j < 2 * d; ++j) a[c][j] *= inv;
    for (int i = 0; i < d; ++i)
      if (i != c) {
        const double f = a[i][c];
        for (int j = 0; j < 2 * d; ++j) a[i][j] -= f * a[c][j];
      }
  }
  for (int q = 0; q < 27; ++q) out27[q] = 0.0;
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      out27[i * 3 + j] = basis[i * d + j];
      out27[9 + i * 3 + j] = a[j][d + i];  // (B^-1)^T
    }
  // (B B^T)^-1 = B^-T B^-1
  for (int i = 0; i < d; ++i)
    for (int j = 0; j < d; ++j) {
      double acc = 0.0;
      for (int k = 0; k < d; ++k) acc += a[k][d + i] * a[k][d + j];
      out27[18 + i * 3 + j] = acc;
    }
  return true;
}

}  // namespace

extern "C" int cco_gradient_flow(cco_problem* const* problems, void* stream, int batch,
                                 const double* s0, const double* bases, const double* dt0,
                                 const cco_flow_settings* cfg, cco_flow_out* out) {
  if (!problems || !s0 || !bases || !cfg || !out) return fail(CCO_ERR_ARG, "null argument");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  if (!out->s || !out->energy || !out->t || !out->length || !out->dt || !out->n_steps ||
      !out->n_evals || !out->status)
    return fail(CCO_ERR_ARG, "incomplete output struct");
  if (!(cfg->atol > 0.0) || !(cfg->rtol > 0.0) || !(cfg->dt_init > 0.0) || cfg->max_steps <= 0)
    return fail(CCO_ERR_ARG, "atol, rtol, dt_init and max_steps must be positive");
  if (cfg->arclength && std::isfinite(cfg->t_max))
    return fail(CCO_ERR_ARG, "t_max is supported only with parametrization='time'");
  if (cfg->record_every < 0 || cfg->max_records < 0)
    return fail(CCO_ERR_ARG, "record_every and max_records must be >= 0");
  if ((cfg->record_every > 0) != (cfg->max_records > 1))
    return fail(CCO_ERR_ARG, "recording needs record_every > 0 and max_records >= 2");
  const bool rec = cfg->record_every > 0;
  if (rec && (!out->traj_s || !out->traj_t || !out->traj_length || !out->traj_energy ||
              !out->traj_count))
    return fail(CCO_ERR_ARG, "trajectory recording needs the traj_* outputs");
  for (int i = 0; i < batch; ++i)
    if (!problems[i]) return fail(CCO_ERR_ARG, "null problem for lane %d", i);
  std::vector<double> mats((size_t)batch * 27);
  size_t bo = 0;
  for (int i = 0; i < batch; ++i) {
    const int d = problems[i]->d;
    if (!basis_mats(bases + bo, d, mats.data() + (size_t)i * 27))
      return fail(CCO_ERR_ARG, "singular basis for lane %d", i);
    bo += (size_t)d * d;
  }
  DeviceGuard guard(problems[0]->device);
  cudaStream_t st = (cudaStream_t)stream;
  RecordShape shape;
  shape.method = Method::Flow;
  LaneTable T;
  FlArgs& a = T.fl;
  a.rtol = cfg->rtol;
  a.atol = cfg->atol;
  a.dt_init = cfg->dt_init;
  a.dt_min = cfg->dt_min;
  a.dt_max = cfg->dt_max;
  a.t_max = cfg->t_max;
  a.energy_tol = cfg->energy_tol;
  a.grad_tol = cfg->grad_tol;
  a.max_steps = cfg->max_steps;
  a.arclength = cfg->arclength ? 1 : 0;
  a.rec_every = rec ? cfg->record_every : 0;
  a.rec_cap = rec ? cfg->max_records : 0;
  if (rec) {
    a.traj_s = out->traj_s;
    a.traj_t = out->traj_t;
    a.traj_len = out->traj_length;
    a.traj_e = out->traj_energy;
    a.traj_count = out->traj_count;
  }
  double* records = nullptr;
  int rc = make_table(problems, batch, shape, a.rec_cap, st, &T, &records);
  if (rc != CCO_OK) {
    if (records) cudaFreeAsync(records, st);
    return rc;
  }
  a.B = batch;
  a.lanes = T.d_refs;
  double* d_mats = nullptr;
  double* d_dt0 = nullptr;
  CCO_CUDA(upload(&d_mats, mats, st));
  if (dt0) {
    std::vector<double> v(dt0, dt0 + batch);
    CCO_CUDA(upload(&d_dt0, v, st));
  }
  CCO_CUDA(flow_init(a, s0, d_mats, d_dt0, st));
  const int64_t max_ticks = 2 + 6 * 4 * cfg->max_steps + 4 * (kMaxInflight + 1) * 32;
  RunStats rs;
  rc = run_lane_table(T, st, max_ticks, &rs);
  if (rc == CCO_OK) {
    cudaError_t e = flow_finalize(a, out->s, out->energy, out->t, out->length, out->dt,
                                  out->n_steps, out->n_evals, out->status, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "flow_finalize");
  }
  out->ticks = rs.ticks;
  out->launches = rs.launches + 3;
  T.release(st);
  cudaFreeAsync(d_mats, st);
  if (d_dt0) cudaFreeAsync(d_dt0, st);
  cudaFreeAsync(records, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "gradient flow");
  return rc;
}

extern "C" int cco_md_run(cco_problem* const* problems, void* stream, int batch,
                          const double* r0, const double* v0, const double* bases,
                          const uint32_t* keys, const double* acc0, const cco_md_settings* cfg,
                          cco_md_out* out) {
  if (!problems || !r0 || !v0 || !bases || !keys || !cfg || !out)
    return fail(CCO_ERR_ARG, "null argument");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  if (!out->r || !out->v || !out->energy || !out->kinetic || !out->max_drift || !out->n_resets ||
      !out->reset_acc || !out->keys || !out->status)
    return fail(CCO_ERR_ARG, "incomplete output struct");
  if (!(std::isfinite(cfg->dt) && cfg->dt > 0.0))
    return fail(CCO_ERR_ARG, "dt must be finite and positive, got %g", cfg->dt);
  if (cfg->n_steps < 0) return fail(CCO_ERR_ARG, "n_steps must be >= 0");
  if (cfg->scheme != MD_VERLET && cfg->scheme != MD_BAOAB) return fail(CCO_ERR_ARG, "unknown scheme");
  if (cfg->andersen < 0 || cfg->andersen > 2) return fail(CCO_ERR_ARG, "unknown Andersen mode");
  if (cfg->andersen != ANDERSEN_OFF && !(cfg->andersen_p >= 0.0 && cfg->andersen_p <= 1.0))
    return fail(CCO_ERR_ARG, "p must lie in [0, 1], got %g", cfg->andersen_p);
  if (cfg->scheme == MD_BAOAB && !(std::isfinite(cfg->gamma) && cfg->gamma >= 0.0))
    return fail(CCO_ERR_ARG, "gamma must be finite and >= 0, got %g", cfg->gamma);
  if (!(cfg->temperature >= 0.0)) return fail(CCO_ERR_ARG, "temperature must be >= 0");
  for (int i = 0; i < batch; ++i)
    if (!problems[i]) return fail(CCO_ERR_ARG, "null problem for lane %d", i);
  std::vector<double> mats((size_t)batch * 27);
  size_t bo = 0;
  for (int i = 0; i < batch; ++i) {
    const int d = problems[i]->d;
    double m27[27];
    if (!basis_mats(bases + bo, d, m27)) return fail(CCO_ERR_ARG, "singular basis for lane %d", i);
    // B, B^-1 (= (B^-T)^T), B^-T
    for (int q = 0; q < 9; ++q) mats[(size_t)i * 27 + q] = m27[q];
    for (int a = 0; a < 3; ++a)
      for (int b = 0; b < 3; ++b) {
        mats[(size_t)i * 27 + 9 + a * 3 + b] = m27[9 + b * 3 + a];
        mats[(size_t)i * 27 + 18 + a * 3 + b] = m27[9 + a * 3 + b];
      }
    bo += (size_t)d * d;
  }
  DeviceGuard guard(problems[0]->device);
  cudaStream_t st = (cudaStream_t)stream;
  RecordShape shape;
  shape.method = Method::Md;
  LaneTable T;
  MdArgs& a = T.md;
  a.dt = cfg->dt;
  a.gamma = cfg->gamma;
  a.temperature = cfg->temperature;
  a.andersen_p = cfg->andersen_p;
  a.drift_tol = cfg->drift_tol;
  a.n_steps = cfg->n_steps;
  a.scheme = cfg->scheme;
  a.andersen = cfg->scheme == MD_VERLET ? cfg->andersen : ANDERSEN_OFF;
  double* records = nullptr;
  int rc = make_table(problems, batch, shape, 0, st, &T, &records);
  if (rc != CCO_OK) {
    if (records) cudaFreeAsync(records, st);
    return rc;
  }
  a.B = batch;
  a.lanes = T.d_refs;
  double* d_mats = nullptr;
  uint32_t* d_keys = nullptr;
  double* d_acc = nullptr;
  CCO_CUDA(upload(&d_mats, mats, st));
  CCO_CUDA(upload(&d_keys, std::vector<uint32_t>(keys, keys + 2 * (size_t)batch), st));
  if (acc0) CCO_CUDA(upload(&d_acc, std::vector<double>(acc0, acc0 + batch), st));
  CCO_CUDA(md_init(a, r0, v0, d_mats, d_keys, d_acc, st));
  const int64_t max_ticks = 2 + cfg->n_steps + 4 * (kMaxInflight + 1) * 32;
  RunStats rs;
  rc = run_lane_table(T, st, max_ticks, &rs);
  if (rc == CCO_OK) {
    cudaError_t e = md_finalize(a, out->r, out->v, out->f, out->energy, out->kinetic,
                                out->max_drift, out->n_resets, out->reset_acc, out->keys,
                                out->status, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "md_finalize");
  }
  out->ticks = rs.ticks;
  out->launches = rs.launches + 3;
  T.release(st);
  cudaFreeAsync(d_mats, st);
  cudaFreeAsync(d_keys, st);
  if (d_acc) cudaFreeAsync(d_acc, st);
  cudaFreeAsync(records, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "md run");
  return rc;
}

extern "C" int cco_md_segment(cco_problem* p, void* stream, int batch, const double* basis,
                              const cco_md_segment_settings* cfg, const cco_md_waves* wv,
                              cco_md_state* io, int64_t* ticks) {
  if (!p || !basis || !cfg || !wv || !io) return fail(CCO_ERR_ARG, "null argument");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one lane");
  if (!(std::isfinite(cfg->dt) && cfg->dt > 0.0))
    return fail(CCO_ERR_ARG, "dt must be finite and positive, got %g", cfg->dt);
  if (cfg->n_steps < 0) return fail(CCO_ERR_ARG, "n_steps must be >= 0");
  if (cfg->scheme != MD_VERLET && cfg->scheme != MD_BAOAB) return fail(CCO_ERR_ARG, "unknown scheme");
  if (cfg->andersen < 0 || cfg->andersen > 2) return fail(CCO_ERR_ARG, "unknown Andersen mode");
  if (!(cfg->andersen_p >= 0.0 && cfg->andersen_p <= 1.0))
    return fail(CCO_ERR_ARG, "andersen_p must lie in [0, 1], got %g", cfg->andersen_p);
  if (!(cfg->gamma >= 0.0 && std::isfinite(cfg->gamma)))
    return fail(CCO_ERR_ARG, "gamma must be finite and >= 0, got %g", cfg->gamma);
  if (cfg->wind_every < 1) return fail(CCO_ERR_ARG, "wind_every must be >= 1");
  if (!(cfg->phase_floor >= 0.0) || !(cfg->drift_tol > 0.0))
    return fail(CCO_ERR_ARG, "need phase_floor >= 0 and drift_tol > 0");
  if (cfg->n_record_steps < 0 || cfg->n_record_steps > 256 ||
      (cfg->n_record_steps > 0 && !cfg->record_steps))
    return fail(CCO_ERR_ARG, "record_steps: at most 256");
  for (int j = 0; j < cfg->n_record_steps; ++j)
    if (cfg->record_steps[j] < 1 || (j > 0 && cfg->record_steps[j] <= cfg->record_steps[j - 1]))
      return fail(CCO_ERR_ARG, "record_steps must be strictly increasing integers >= 1");
  if (cfg->record_rho_every < 0 || cfg->max_rho_records < 0 ||
      (cfg->record_rho_every > 0 && cfg->max_rho_records < 1))
    return fail(CCO_ERR_ARG, "a rho trace needs record_rho_every > 0 and max_rho_records >= 1");
  const int d = p->d, w = wv->n_waves, nc = wv->n_constrained;
  if (w < 1 || nc < 1 || nc > w || !wv->n_vectors || !wv->kvec || !wv->constrained_rows)
    return fail(CCO_ERR_ARG, "need 1 <= n_constrained <= n_waves and the wave arrays");
  const bool rec = cfg->n_record_steps > 0, trace = cfg->record_rho_every > 0;
  if (!io->r || !io->v || !io->f || !io->phi || !io->temperature || !io->time || !io->reset_acc ||
      !io->e0 || !io->max_drift || !io->sum_kinetic || !io->sum_phi || !io->sum_phi2 ||
      !io->keys || !io->step || !io->status || !io->n_sum || !io->rho_prev || !io->wind_abs ||
      !io->wind_net || !io->sum_s || !io->n_valid || !io->snap_count || !io->trace_count)
    return fail(CCO_ERR_ARG, "incomplete state struct");
  if (rec && (!io->snap_step || !io->snap_time || !io->snap_phi || !io->snap_kinetic ||
              !io->snap_wind_abs || !io->snap_wind_net || !io->snap_rho || !io->snap_r))
    return fail(CCO_ERR_ARG, "snapshot buffers missing");
  if (trace && (!io->trace_rho || !io->trace_time)) return fail(CCO_ERR_ARG, "trace buffers missing");
  double m27[27];
  if (!basis_mats(basis, d, m27)) return fail(CCO_ERR_ARG, "singular basis");
  std::vector<double> mats(27);
  for (int q = 0; q < 9; ++q) mats[q] = m27[q];
  for (int x = 0; x < 3; ++x)
    for (int y = 0; y < 3; ++y) {
      mats[9 + x * 3 + y] = m27[9 + y * 3 + x];
      mats[18 + x * 3 + y] = m27[9 + x * 3 + y];
    }
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  // run position of each constrained wave's density
  std::vector<int> r2r(p->M), pos(p->M), cpos(nc);
  CCO_CUDA(cudaMemcpy(r2r.data(), p->run2ref, sizeof(int) * p->M, cudaMemcpyDeviceToHost));
  for (int k = 0; k < p->M; ++k) pos[r2r[k]] = k;
  for (int c = 0; c < nc; ++c) {
    const int row = wv->constrained_rows[c];
    if (row < 0 || row >= p->M) return fail(CCO_ERR_ARG, "constrained wave %d: row %d outside the problem", c, row);
    cpos[c] = pos[row];
  }
  RecordShape shape;
  shape.method = Method::Md;
  shape.waves = w;
  LaneTable T;
  MdArgs& a = T.md;
  a.dt = cfg->dt;
  a.gamma = cfg->gamma;
  a.temperature = 0.0;
  a.andersen_p = cfg->andersen_p;
  a.drift_tol = 0.0;
  a.n_steps = cfg->n_steps;
  a.scheme = cfg->scheme;
  a.andersen = cfg->scheme == MD_VERLET ? cfg->andersen : ANDERSEN_OFF;
  a.w = w;
  a.nc = nc;
  a.wind_every = cfg->wind_every;
  a.corrected = (a.scheme == MD_BAOAB || a.andersen != ANDERSEN_OFF) ? 1 : 0;
  const bool guard_on = a.scheme == MD_VERLET && a.andersen == ANDERSEN_OFF && std::isfinite(cfg->drift_tol);
  a.drift_coef = guard_on ? cfg->drift_tol * 0.5 * d * (p->N - 1) : -1.0;
  a.phase_floor = cfg->phase_floor;
  a.n_rec = cfg->n_record_steps;
  a.trace_every = trace ? cfg->record_rho_every : 0;
  a.trace_cap = trace ? cfg->max_rho_records : 0;
  MdSegIO& o = a.io;
  o.r = io->r; o.v = io->v; o.f = io->f; o.phi = io->phi; o.temperature = io->temperature;
  o.time = io->time; o.reset_acc = io->reset_acc; o.keys = io->keys; o.step = io->step;
  o.status = io->status; o.n_valid = io->n_valid; o.n_sum = io->n_sum; o.rho_prev = io->rho_prev;
  o.wind_abs = io->wind_abs; o.wind_net = io->wind_net; o.sum_s = io->sum_s; o.e0 = io->e0;
  o.max_drift = io->max_drift; o.sum_kinetic = io->sum_kinetic; o.sum_phi = io->sum_phi;
  o.sum_phi2 = io->sum_phi2; o.snap_step = io->snap_step; o.snap_count = io->snap_count;
  o.snap_time = io->snap_time; o.snap_wind_abs = io->snap_wind_abs;
  o.snap_wind_net = io->snap_wind_net; o.snap_rho = io->snap_rho; o.snap_r = io->snap_r;
  o.snap_phi = io->snap_phi; o.snap_kinetic = io->snap_kinetic; o.trace_rho = io->trace_rho;
  o.trace_time = io->trace_time; o.trace_count = io->trace_count;
  std::vector<cco_problem*> probs(batch, p);
  double* records = nullptr;
  int rc = make_table(probs.data(), batch, shape, 0, st, &T, &records);
  if (rc != CCO_OK) {
    if (records) cudaFreeAsync(records, st);
    return rc;
  }
  a.B = batch;
  a.lanes = T.d_refs;
  double *d_mats = nullptr, *d_wn = nullptr, *d_wk = nullptr;
  int* d_cpos = nullptr;
  int64_t* d_rec = nullptr;
  cudaError_t e = upload(&d_mats, mats, st);
  if (e == cudaSuccess) e = upload(&d_wn, std::vector<double>(wv->n_vectors, wv->n_vectors + (size_t)w * d), st);
  if (e == cudaSuccess) e = upload(&d_wk, std::vector<double>(wv->kvec, wv->kvec + (size_t)w * d), st);
  if (e == cudaSuccess) e = upload(&d_cpos, cpos, st);
  if (e == cudaSuccess && rec)
    e = upload(&d_rec, std::vector<int64_t>(cfg->record_steps, cfg->record_steps + cfg->n_record_steps), st);
  a.wave_n = d_wn;
  a.wave_k = d_wk;
  a.cpos = d_cpos;
  a.rec_steps = d_rec;
  if (e == cudaSuccess) e = md_seg_init(a, d_mats, st);
  if (e != cudaSuccess) rc = cuda_fail(e, "md segment setup");
  RunStats rs;
  if (rc == CCO_OK) rc = run_lane_table(T, st, 2 + cfg->n_steps + 4 * (kMaxInflight + 1) * 32, &rs);
  if (rc == CCO_OK) {
    e = md_seg_finalize(a, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "md segment finalize");
  }
  if (ticks) *ticks = rs.ticks;
  T.release(st);
  for (void* q : {(void*)d_mats, (void*)d_wn, (void*)d_wk, (void*)d_cpos, (void*)d_rec, (void*)records})
    if (q) cudaFreeAsync(q, st);
  e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "md segment");
  return rc;
}

extern "C" int cco_schedule_reset(void) {
  schedule_clear();
  return CCO_OK;
}
