// Serving pool: continuous batching of L-BFGS relaxations on one device.
//
// A driver thread keeps a running set of lanes (one lane record per request,
// cco_opt.cuh) and launches captured graphs of ticks over it. Between graphs
// it admits queued requests while their records fit max_lanes and the HBM
// budget, retires lanes whose status left RUNNING (a per-graph status
// snapshot read kServeInflight graphs behind), and recaptures the graph when
// the set changed. A lane's state never moves while it runs, and nothing a
// lane computes depends on the other lanes, so a result is bit-identical to
// the same configuration relaxed alone by cco_relax_lbfgs.
//
// Every host wait is bounded by device work that itself ends (each kernel
// does a fixed amount of work per lane), and the driver wakes at least every
// few milliseconds when idle.
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "cco.h"
#include "cco_host.cuh"

using namespace cco;

namespace {

int64_t steady_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Request {
  int64_t id = 0;
  cco_problem* p = nullptr;
  std::vector<double> s0;
  size_t bytes = 0;
  int64_t submit_ns = 0, admit_ns = 0, done_ns = 0;
  // results
  std::vector<double> s;
  double energy = 0.0, grad_norm = 0.0;
  int64_t n_evals = 0, n_iters = 0, status = CCO_STATUS_RUNNING, device_ns = 0, n_fp32 = 0;
  int error = CCO_OK;
  bool done = false;
  bool cancel = false;      // asked by the client
  // driver-side state
  double* rec = nullptr;    // device lane record while admitted
  bool retiring = false;    // finalize issued
  bool cancel_sent = false; // cancel kernel issued
};

// Pinned host buffer that grows on demand.
struct Pinned {
  void* ptr = nullptr;
  size_t cap = 0;
  cudaError_t reserve(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    size_t n = std::max<size_t>(bytes, 1 << 16);
    n = std::max(n, 2 * bytes);
    cudaError_t e = cudaHostAlloc(&ptr, n, cudaHostAllocDefault);
    if (e == cudaSuccess) cap = n;
    return e;
  }
  ~Pinned() {
    if (ptr) cudaFreeHost(ptr);
  }
};

constexpr int kServeInflight = 3;
constexpr int kServeSlots = kServeInflight + 1;
constexpr int kRetireSlots = 8;

// One launched graph: its status snapshot and the lanes it covered.
struct Flight {
  cudaEvent_t ev = nullptr;
  std::vector<Request*> lanes;
  Pinned h_status;
  int64_t* d_status = nullptr;
  size_t d_cap = 0;
};

// One batch of retiring lanes: finalize outputs on their way to the host.
struct Retire {
  cudaEvent_t ev = nullptr;
  std::vector<Request*> reqs;
  std::vector<int64_t> soff;
  Pinned host;
};

// A tick plan kept alive until the last graph launched from it has run.
struct OldPlan {
  std::unique_ptr<TickPlan> plan;
  cudaEvent_t ev = nullptr;
};

}  // namespace

struct cco_server {
  int device = 0;
  cco_lbfgs_settings settings{};
  LbArgs args{};
  RecordShape shape;
  size_t budget = 0;
  int max_lanes = 4096;
  int graph_ticks = 8;
  int branches = 0;

  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<Request*> incoming;
  std::unordered_map<int64_t, std::unique_ptr<Request>> reqs;
  int64_t next_id = 1;
  bool stop = false;
  int error = CCO_OK;
  std::thread driver;

  // statistics (guarded by mu)
  int64_t n_submitted = 0, n_admitted = 0, n_completed = 0, n_cancelled = 0;
  int64_t n_pending = 0, n_running = 0;
  int64_t bytes_in_use = 0, peak_bytes = 0, peak_lanes = 0;
  int64_t graphs = 0, ticks = 0, rebuilds = 0;
};

namespace {

// Marks a request done (caller holds S->mu).
void complete_locked(cco_server* S, Request* r) {
  r->done = true;
  r->done_ns = steady_ns();
  S->n_completed += 1;
  if (r->status == CCO_STATUS_CANCELLED) S->n_cancelled += 1;
}

class Driver {
 public:
  explicit Driver(cco_server* S) : S_(S) {}

  void run() {
    cudaError_t e = cudaSetDevice(S_->device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking);
    for (int i = 0; i < kServeSlots && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&fl_[i].ev, cudaEventDisableTiming);
    for (int i = 0; i < kRetireSlots && e == cudaSuccess; ++i)
      e = cudaEventCreateWithFlags(&rt_[i].ev, cudaEventDisableTiming);
    table_.shape = S_->shape;
    table_.lb = S_->args;
    int rc = e == cudaSuccess ? CCO_OK : cuda_fail(e, "serving driver start");
    while (rc == CCO_OK) {
      bool stopping = false;
      rc = intake(&stopping);
      if (rc != CCO_OK) break;
      if (stopping && active_.empty() && pending_.empty() && rt_count_ == 0) break;
      rc = collect_retired(false);
      if (rc == CCO_OK) rc = admit();
      if (rc == CCO_OK && dirty_) rc = rebuild();
      if (rc != CCO_OK) break;
      if (plan_ && !live_.empty() && fl_count_ < kServeInflight) {
        rc = launch();
        continue;
      }
      if (fl_count_ > 0) {
        rc = land_oldest();
        continue;
      }
      if (rt_count_ > 0) {
        rc = collect_retired(true);
        continue;
      }
      // idle: wait for a submission or a cancel
      std::unique_lock<std::mutex> lk(S_->mu);
      S_->cv_work.wait_for(lk, std::chrono::milliseconds(5), [&] {
        return S_->stop || !S_->incoming.empty() || cancel_pending_locked();
      });
    }
    // drain the device and end what is left
    if (st_) cudaStreamSynchronize(st_);
    {
      std::lock_guard<std::mutex> lk(S_->mu);
      if (rc != CCO_OK) S_->error = rc;
      auto finish = [&](Request* r) {
        if (r->done) return;
        r->status = CCO_STATUS_CANCELLED;
        r->error = rc;
        complete_locked(S_, r);
      };
      for (Request* r : pending_) finish(r);
      for (Request* r : active_) finish(r);
      for (Request* r : S_->incoming) finish(r);
      S_->incoming.clear();
      S_->n_pending = 0;
      S_->n_running = 0;
    }
    S_->cv_done.notify_all();
    for (Request* r : active_)
      if (r->rec) cudaFreeAsync(r->rec, st_);
    active_.clear();
    if (plan_) plan_->release(st_);
    for (auto& o : old_) {
      o.plan->release(st_);
      if (o.ev) cudaEventDestroy(o.ev);
    }
    table_.release(st_);
    for (int i = 0; i < kServeSlots; ++i) {
      if (fl_[i].d_status) cudaFreeAsync(fl_[i].d_status, st_);
      if (fl_[i].ev) cudaEventDestroy(fl_[i].ev);
    }
    for (int i = 0; i < kRetireSlots; ++i)
      if (rt_[i].ev) cudaEventDestroy(rt_[i].ev);
    if (st_) {
      cudaStreamSynchronize(st_);
      cudaStreamDestroy(st_);
    }
  }

 private:
  cco_server* S_;
  cudaStream_t st_ = nullptr;
  std::deque<Request*> pending_;     // queued, not admitted (arrival order)
  std::vector<Request*> active_;     // admitted, not yet handed back
  std::vector<Request*> live_;       // lanes of the current table
  LaneTable table_;
  std::unique_ptr<TickPlan> plan_;
  std::vector<OldPlan> old_;
  bool dirty_ = false;
  size_t used_ = 0;      // bytes of the resident records
  int resident_ = 0;     // admitted lanes whose records are not yet freed
  Flight fl_[kServeSlots];
  int fl_head_ = 0, fl_count_ = 0;
  Retire rt_[kRetireSlots];
  int rt_head_ = 0, rt_count_ = 0;

  // (driver thread, S_->mu held)
  bool cancel_pending_locked() {
    for (Request* r : active_)
      if (r->cancel && !r->cancel_sent && !r->retiring) return true;
    for (Request* r : pending_)
      if (r->cancel) return true;
    return false;
  }

  int intake(bool* stopping) {
    std::vector<Request*> to_cancel;
    {
      std::lock_guard<std::mutex> lk(S_->mu);
      while (!S_->incoming.empty()) {
        pending_.push_back(S_->incoming.front());
        S_->incoming.pop_front();
      }
      *stopping = S_->stop;
      if (S_->stop) {
        for (Request* r : pending_) r->cancel = true;
        for (Request* r : active_) r->cancel = true;
      }
      // queued requests cancelled before admission end here
      for (auto it = pending_.begin(); it != pending_.end();) {
        if ((*it)->cancel) {
          (*it)->status = CCO_STATUS_CANCELLED;
          complete_locked(S_, *it);
          it = pending_.erase(it);
        } else {
          ++it;
        }
      }
      S_->n_pending = (int64_t)pending_.size();
      for (Request* r : active_)
        if (r->cancel && !r->cancel_sent && !r->retiring) to_cancel.push_back(r);
    }
    S_->cv_done.notify_all();
    // running requests: the cancel kernel ends the lane between graphs (the
    // kernels skip it from then on) and the next snapshot retires it
    for (Request* r : to_cancel) {
      CCO_CUDA(cancel_lbfgs_lane(r->rec, st_));
      r->cancel_sent = true;
    }
    return CCO_OK;
  }

  int admit() {
    std::vector<Request*> fresh;
    while (!pending_.empty() && resident_ < S_->max_lanes) {
      Request* r = pending_.front();
      if (used_ + r->bytes > S_->budget) break;   // first come, first served
      double* rec = nullptr;
      const cudaError_t e = pool_alloc(&rec, r->bytes, st_);
      if (e != cudaSuccess) {
        cudaGetLastError();
        if (resident_ == 0) {
          // nothing to wait for: this request cannot fit the device
          std::lock_guard<std::mutex> lk(S_->mu);
          r->status = CCO_STATUS_CANCELLED;
          r->error = CCO_ERR_OOM;
          complete_locked(S_, r);
          pending_.pop_front();
          continue;
        }
        break;   // retry once running lanes free memory
      }
      pending_.pop_front();
      r->rec = rec;
      r->admit_ns = steady_ns();
      used_ += r->bytes;
      ++resident_;
      active_.push_back(r);
      fresh.push_back(r);
    }
    if (fresh.empty()) return CCO_OK;
    // start the fresh lanes: packed s0 upload and the init kernel
    std::vector<LaneRef> refs;
    std::vector<double> s0;
    for (Request* r : fresh) {
      LaneRef ref{};
      ref.rec = r->rec;
      ref.nd = r->p->N * r->p->d;
      ref.ld = pad4(ref.nd);
      ref.n = r->p->N;
      ref.soff = (int64_t)s0.size();
      ref.toff = 0;
      s0.insert(s0.end(), r->s0.begin(), r->s0.end());
      refs.push_back(ref);
    }
    LaneRef* d_refs = nullptr;
    double* d_s0 = nullptr;
    CCO_CUDA(upload(&d_refs, refs, st_));
    CCO_CUDA(upload(&d_s0, s0, st_));
    LbArgs a = S_->args;
    a.B = (int)fresh.size();
    a.lanes = d_refs;
    CCO_CUDA(lbfgs_init(a, d_s0, st_));
    CCO_CUDA(cudaFreeAsync(d_refs, st_));
    CCO_CUDA(cudaFreeAsync(d_s0, st_));
    for (Request* r : fresh) std::vector<double>().swap(r->s0);
    dirty_ = true;
    std::lock_guard<std::mutex> lk(S_->mu);
    S_->n_admitted += (int64_t)fresh.size();
    S_->n_pending = (int64_t)pending_.size();
    S_->bytes_in_use = (int64_t)used_;
    S_->peak_bytes = std::max(S_->peak_bytes, (int64_t)used_);
    S_->peak_lanes = std::max(S_->peak_lanes, (int64_t)resident_);
    return CCO_OK;
  }

  // New lane table and graph for the lanes that are admitted and not retiring.
  int rebuild() {
    dirty_ = false;
    live_.clear();
    for (Request* r : active_)
      if (!r->retiring) live_.push_back(r);
    if (plan_) {
      // keep the old plan until its launched graphs have run
      OldPlan o;
      o.plan = std::move(plan_);
      CCO_CUDA(cudaEventCreateWithFlags(&o.ev, cudaEventDisableTiming));
      CCO_CUDA(cudaEventRecord(o.ev, st_));
      old_.push_back(std::move(o));
    }
    reap_old_plans();
    {
      std::lock_guard<std::mutex> lk(S_->mu);
      S_->n_running = (int64_t)live_.size();
    }
    if (live_.empty()) {
      table_.release(st_);
      return CCO_OK;
    }
    table_.probs.clear();
    table_.refs.clear();
    for (Request* r : live_) {
      LaneRef ref{};
      ref.rec = r->rec;
      ref.nd = r->p->N * r->p->d;
      ref.ld = pad4(ref.nd);
      ref.n = r->p->N;
      table_.probs.push_back(r->p);
      table_.refs.push_back(ref);
    }
    int rc = table_.upload_refs(st_);
    if (rc != CCO_OK) return rc;
    table_.lb = S_->args;
    table_.lb.B = (int)live_.size();
    table_.lb.lanes = table_.d_refs;
    Schedule sch;
    sch.graph_ticks = S_->graph_ticks;
    sch.branches = S_->branches > 0 ? S_->branches : (live_.size() >= 64 ? 2 : 1);
    plan_.reset(new TickPlan());
    plan_->method = Method::Lbfgs;
    rc = plan_->build(table_, sch, st_);
    std::lock_guard<std::mutex> lk(S_->mu);
    S_->rebuilds += 1;
    return rc;
  }

  void reap_old_plans() {
    for (auto it = old_.begin(); it != old_.end();) {
      if (cudaEventQuery(it->ev) == cudaSuccess) {
        it->plan->release(st_);
        cudaEventDestroy(it->ev);
        it = old_.erase(it);
      } else {
        cudaGetLastError();
        ++it;
      }
    }
  }

  int launch() {
    Flight& f = fl_[(fl_head_ + fl_count_) % kServeSlots];
    const size_t n = live_.size();
    if (f.d_cap < n) {
      if (f.d_status) CCO_CUDA(cudaFreeAsync(f.d_status, st_));
      f.d_status = nullptr;
      f.d_cap = std::max<size_t>(n, 256);
      CCO_CUDA(pool_alloc(&f.d_status, sizeof(int64_t) * f.d_cap, st_));
    }
    CCO_CUDA(f.h_status.reserve(sizeof(int64_t) * n));
    CCO_CUDA(cudaGraphLaunch(plan_->exec, st_));
    CCO_CUDA(gather_status(table_.d_refs, (int)n, f.d_status, st_));
    CCO_CUDA(cudaMemcpyAsync(f.h_status.ptr, f.d_status, sizeof(int64_t) * n,
                             cudaMemcpyDeviceToHost, st_));
    CCO_CUDA(cudaEventRecord(f.ev, st_));
    f.lanes = live_;
    ++fl_count_;
    std::lock_guard<std::mutex> lk(S_->mu);
    S_->graphs += 1;
    S_->ticks += plan_->sch.graph_ticks;
    return CCO_OK;
  }

  // Waits for the oldest graph and retires the lanes its snapshot shows done.
  int land_oldest() {
    Flight& f = fl_[fl_head_];
    CCO_CUDA(cudaEventSynchronize(f.ev));
    const int64_t* h = static_cast<const int64_t*>(f.h_status.ptr);
    std::vector<Request*> done;
    for (size_t i = 0; i < f.lanes.size(); ++i) {
      Request* r = f.lanes[i];
      if (h[i] != CCO_STATUS_RUNNING && !r->retiring) {
        r->retiring = true;
        done.push_back(r);
      }
    }
    f.lanes.clear();
    fl_head_ = (fl_head_ + 1) % kServeSlots;
    --fl_count_;
    if (!done.empty()) {
      dirty_ = true;
      return retire(done);
    }
    return CCO_OK;
  }

  // Finalize kernel into packed device outputs, one copy to pinned memory,
  // then the records go back to the pool (stream-ordered).
  int retire(const std::vector<Request*>& done) {
    while (rt_count_ == kRetireSlots) {
      const int rc = collect_retired(true);
      if (rc != CCO_OK) return rc;
    }
    Retire& R = rt_[(rt_head_ + rt_count_) % kRetireSlots];
    const size_t n = done.size();
    std::vector<LaneRef> refs;
    R.soff.clear();
    int64_t total = 0;
    for (Request* r : done) {
      LaneRef ref{};
      ref.rec = r->rec;
      ref.nd = r->p->N * r->p->d;
      ref.ld = pad4(ref.nd);
      ref.n = r->p->N;
      ref.soff = total;
      R.soff.push_back(total);
      total += ref.nd;
      refs.push_back(ref);
    }
    // device outputs: s (total), energy, grad_norm (n each), then
    // n_evals, n_iters, status, latency, FP32 evaluations (n each, int64)
    const size_t bytes = sizeof(double) * ((size_t)total + 7 * n);
    double* d_out = nullptr;
    LaneRef* d_refs = nullptr;
    CCO_CUDA(upload(&d_refs, refs, st_));
    CCO_CUDA(pool_alloc(&d_out, bytes, st_));
    CCO_CUDA(R.host.reserve(bytes));
    LbArgs a = S_->args;
    a.B = (int)n;
    a.lanes = d_refs;
    double* s_out = d_out;
    double* e_out = d_out + total;
    double* g_out = e_out + n;
    int64_t* i_out = reinterpret_cast<int64_t*>(g_out + n);
    CCO_CUDA(lbfgs_finalize(a, s_out, e_out, g_out, i_out, i_out + n, i_out + 2 * n,
                            i_out + 3 * n, i_out + 4 * n, st_));
    CCO_CUDA(cudaMemcpyAsync(R.host.ptr, d_out, bytes, cudaMemcpyDeviceToHost, st_));
    CCO_CUDA(cudaEventRecord(R.ev, st_));
    CCO_CUDA(cudaFreeAsync(d_out, st_));
    CCO_CUDA(cudaFreeAsync(d_refs, st_));
    for (Request* r : done) {
      CCO_CUDA(cudaFreeAsync(r->rec, st_));
      r->rec = nullptr;
      used_ -= r->bytes;
      --resident_;
    }
    R.reqs = done;
    ++rt_count_;
    std::lock_guard<std::mutex> lk(S_->mu);
    S_->bytes_in_use = (int64_t)used_;
    return CCO_OK;
  }

  // Hands finished retire batches to their requests (wait: block on the oldest).
  int collect_retired(bool wait) {
    while (rt_count_ > 0) {
      Retire& R = rt_[rt_head_];
      if (wait) {
        CCO_CUDA(cudaEventSynchronize(R.ev));
      } else {
        const cudaError_t q = cudaEventQuery(R.ev);
        if (q == cudaErrorNotReady) {
          cudaGetLastError();
          return CCO_OK;
        }
        if (q != cudaSuccess) return cuda_fail(q, "serving retire");
      }
      const size_t n = R.reqs.size();
      int64_t total = 0;
      for (Request* r : R.reqs) total += r->p->N * r->p->d;
      const double* hs = static_cast<const double*>(R.host.ptr);
      const double* he = hs + total;
      const double* hg = he + n;
      const int64_t* hi = reinterpret_cast<const int64_t*>(hg + n);
      {
        std::lock_guard<std::mutex> lk(S_->mu);
        for (size_t i = 0; i < n; ++i) {
          Request* r = R.reqs[i];
          const int nd = r->p->N * r->p->d;
          r->s.assign(hs + R.soff[i], hs + R.soff[i] + nd);
          r->energy = he[i];
          r->grad_norm = hg[i];
          r->n_evals = hi[i];
          r->n_iters = hi[n + i];
          r->status = hi[2 * n + i];
          r->device_ns = hi[3 * n + i];
          r->n_fp32 = hi[4 * n + i];
          complete_locked(S_, r);
        }
        std::vector<Request*> keep;
        for (Request* r : active_)
          if (!r->done) keep.push_back(r);
        active_.swap(keep);
      }
      S_->cv_done.notify_all();
      R.reqs.clear();
      rt_head_ = (rt_head_ + 1) % kRetireSlots;
      --rt_count_;
      wait = false;
    }
    return CCO_OK;
  }
};

void drive(cco_server* S) {
  Driver d(S);
  d.run();
}

}  // namespace

extern "C" int cco_server_create(int device, const cco_lbfgs_settings* settings,
                                 const cco_server_config* config, cco_server** out) {
  if (!settings || !out) return fail(CCO_ERR_ARG, "null argument");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    return fail(CCO_ERR_NODEVICE, "no CUDA device visible");
  }
  if (device < 0 || device >= n) return fail(CCO_ERR_ARG, "device %d out of range", device);
  if (settings->n_rescales < 1 || settings->n_rescales > CCO_MAX_RESCALES)
    return fail(CCO_ERR_ARG, "need 1..%d rescale passes", CCO_MAX_RESCALES);
  if (settings->memory < 1 || settings->memory > 256)
    return fail(CCO_ERR_ARG, "memory must be in 1..256");
  if (settings->max_linesearch_steps < 1)
    return fail(CCO_ERR_ARG, "max_linesearch_steps must be >= 1");
  if (settings->precision != 0 && settings->precision != 1)
    return fail(CCO_ERR_ARG, "precision must be 0 or 1");
  if (settings->record_every > 0 && settings->max_records > 0)
    return fail(CCO_ERR_ARG, "the serving pool does not record trajectories");
  if (config && (config->max_lanes < 0 || config->graph_ticks < 0 || config->branches < 0 ||
                 config->hbm_budget_bytes < 0))
    return fail(CCO_ERR_ARG, "negative server configuration");
  std::unique_ptr<cco_server> S(new cco_server());
  S->device = device;
  S->settings = *settings;
  {
    DeviceGuard guard(device);
    const int rc = lbfgs_args(settings, &S->args, &S->shape);
    if (rc != CCO_OK) return rc;
    size_t free_b = 0, total_b = 0;
    CCO_CUDA(cudaMemGetInfo(&free_b, &total_b));
    const int64_t want = config && config->hbm_budget_bytes > 0 ? config->hbm_budget_bytes
                                                                : (int64_t)150 << 30;
    S->budget = std::min<size_t>((size_t)want, (size_t)(0.9 * (double)free_b));
  }
  if (config) {
    if (config->max_lanes > 0) S->max_lanes = (int)std::min<int64_t>(config->max_lanes, 1 << 20);
    if (config->graph_ticks > 0) S->graph_ticks = std::min(config->graph_ticks, 256);
    if (config->branches > 0) S->branches = std::min(config->branches, kMaxBranches);
  }
  cco_server* raw = S.release();
  raw->driver = std::thread(drive, raw);
  *out = raw;
  return CCO_OK;
}

extern "C" int cco_server_destroy(cco_server* S) {
  if (!S) return CCO_OK;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  if (S->driver.joinable()) S->driver.join();
  delete S;
  return CCO_OK;
}

extern "C" int cco_server_submit(cco_server* S, cco_problem* p, const double* s0,
                                 int64_t* ticket) {
  if (!S || !p || !s0 || !ticket) return fail(CCO_ERR_ARG, "null argument");
  if (p->device != S->device) return fail(CCO_ERR_ARG, "problem lives on another device");
  std::unique_ptr<Request> r(new Request());
  r->p = p;
  r->bytes = record_bytes(S->shape, p);
  if (r->bytes > S->budget)
    return fail(CCO_ERR_ADMISSION, "request needs %zu bytes of lane state, the budget is %zu",
                r->bytes, S->budget);
  const size_t nd = (size_t)p->N * p->d;
  r->s0.assign(s0, s0 + nd);
  r->submit_ns = steady_ns();
  {
    std::lock_guard<std::mutex> lk(S->mu);
    if (S->error != CCO_OK) return fail(S->error, "the serving driver failed earlier");
    if (S->stop) return fail(CCO_ERR_ARG, "server is shutting down");
    r->id = S->next_id++;
    *ticket = r->id;
    S->incoming.push_back(r.get());
    S->reqs[r->id] = std::move(r);
    S->n_submitted += 1;
  }
  S->cv_work.notify_all();
  return CCO_OK;
}

extern "C" int cco_server_poll(cco_server* S, int64_t ticket, int timeout_ms,
                               cco_request_result* out) {
  if (!S || !out) return fail(CCO_ERR_ARG, "null argument");
  std::unique_lock<std::mutex> lk(S->mu);
  auto it = S->reqs.find(ticket);
  if (it == S->reqs.end()) return fail(CCO_ERR_ARG, "unknown ticket %lld", (long long)ticket);
  Request* r = it->second.get();
  if (!r->done && timeout_ms != 0) {
    auto pred = [&] { return r->done; };
    if (timeout_ms < 0) {
      // bounded slices: the driver completes every request before it exits
      while (!r->done) S->cv_done.wait_for(lk, std::chrono::milliseconds(50), pred);
    } else {
      S->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred);
    }
  }
  if (!r->done) return CCO_ERR_TIMEOUT;
  double* s_dst = out->s;
  out->energy = r->energy;
  out->grad_norm = r->grad_norm;
  out->n_evals = r->n_evals;
  out->n_iters = r->n_iters;
  out->status = r->status;
  out->submit_ns = r->submit_ns;
  out->admit_ns = r->admit_ns;
  out->done_ns = r->done_ns;
  out->device_ns = r->device_ns;
  out->error = r->error;
  out->pad_ = 0;
  out->n_evals_fp32 = r->n_fp32;
  if (s_dst && !r->s.empty()) std::memcpy(s_dst, r->s.data(), sizeof(double) * r->s.size());
  S->reqs.erase(it);
  return CCO_OK;
}

extern "C" int cco_server_cancel(cco_server* S, int64_t ticket) {
  if (!S) return fail(CCO_ERR_ARG, "null server");
  {
    std::lock_guard<std::mutex> lk(S->mu);
    auto it = S->reqs.find(ticket);
    if (it == S->reqs.end()) return fail(CCO_ERR_ARG, "unknown ticket %lld", (long long)ticket);
    if (!it->second->done) it->second->cancel = true;
  }
  S->cv_work.notify_all();
  return CCO_OK;
}

extern "C" int cco_server_get_stats(cco_server* S, cco_server_stats* out) {
  if (!S || !out) return fail(CCO_ERR_ARG, "null argument");
  std::lock_guard<std::mutex> lk(S->mu);
  out->submitted = S->n_submitted;
  out->admitted = S->n_admitted;
  out->completed = S->n_completed;
  out->cancelled = S->n_cancelled;
  out->pending = S->n_pending + (int64_t)S->incoming.size();
  out->running = S->n_running;
  out->bytes_in_use = S->bytes_in_use;
  out->peak_bytes = S->peak_bytes;
  out->peak_lanes = S->peak_lanes;
  out->budget_bytes = (int64_t)S->budget;
  out->graphs = S->graphs;
  out->ticks = S->ticks;
  out->rebuilds = S->rebuilds;
  return CCO_OK;
}
