// Batched minimizers as per-lane device state machines (sm_100a, FP64).
//
// A relaxation advances in ticks; each tick evaluates the energy and gradient
// of every RUNNING lane at its probe point (cco_eval.cu) and then runs one
// update CTA per lane that consumes the result. Finished lanes keep their
// state untouched (status != RUNNING makes every kernel skip them), which is
// the reference's bit-exact lane freeze (src/xla_cco/minimize/_loop.py:105-153)
// and its compaction (minimize/__init__.py:75-99) without a host round trip:
// the lane order never changes, so results come back in input order.
//
// Descent (src/xla_cco/minimize/descent.py:92-197): one iteration per tick.
// L-BFGS (src/xla_cco/minimize/lbfgs.py:163-329): one line-search probe per
// tick. The direction is the two-loop recursion of optax's scale_by_lbfgs
// written through inner products: with a_p = s_p.g, b_p = y_p.g,
// SY[p][q] = s_p.y_q (p older than q) and YY = y.y maintained as pairs arrive,
//   alpha_p = rho_p (a_p - sum_{q>p} alpha_q SY[p][q])             (loop 1)
//   beta_p  = rho_p (gamma (b_p - sum_q alpha_q YY[p][q])
//                    + sum_{q<p} (alpha_q - beta_q) SY[q][p])       (loop 2)
//   dir     = -gamma g + sum_q gamma alpha_q y_q - sum_q (alpha_q - beta_q) s_q
// which is algebraically the two-loop recursion. Each iteration streams the
// history twice (dots, then the combination) with no serial reduction chain
// over the history, so the update is HBM-bound instead of latency-bound.
#include <cmath>

#include "cco_opt.cuh"
#include "cco_opt_bodies.cuh"

namespace cco {

namespace {

constexpr int kPassBMaxPairs = 512;  // direction coefficients staged in smem up to this
constexpr int kScalarMaxPairs = 256; // L-BFGS memory supported by the scalar kernel

__global__ void k_descent_init(DescentArgs a, const double* __restrict__ s0) {
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const DsView v = ds_view(R.rec, R.ld);
  for (int e = threadIdx.x; e < R.ld; e += blockDim.x) {
    const double x = e < R.nd ? s0[R.soff + e] : 0.0;
    v.ps[e] = x;
    v.s[e] = x;
    v.g[e] = 0.0;
    v.pg[e] = 0.0;
  }
  if (threadIdx.x == 0) {
    DsState S = {};
    S.phase = PH_INIT;
    S.status = CCO_STATUS_RUNNING;
    S.step = a.step_init;
    S.t0 = gtimer();
    *v.st = S;
    if (a.traj_count) a.traj_count[R.idx] = 0;
  }
}

}  // namespace

namespace {

__global__ void __launch_bounds__(kUpdThreads) k_descent_update(DescentArgs a) {
  descent_update_lane(a, blockIdx.x);
}

__global__ void k_descent_finalize(DescentArgs a, double* s_out, double* e_out, double* gn_out,
                                   int64_t* ne_out, int64_t* ni_out, int64_t* st_out,
                                   int64_t* lat_out) {
  __shared__ double red[32];
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const DsView v = ds_view(R.rec, R.ld);
  double ss = 0.0;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    const double x = v.g[e];
    ss += x * x;
    s_out[R.soff + e] = wrap01(v.s[e]);
  }
  ss = block_sum(ss, red);
  if (threadIdx.x == 0) {
    const DsState S = *v.st;
    e_out[lane] = S.f;
    gn_out[lane] = sqrt(ss);
    ne_out[lane] = S.n_evals;
    ni_out[lane] = S.it;
    st_out[lane] = S.status;
    if (lat_out) lat_out[lane] = S.t1 - S.t0;
  }
}

// ============================================================ L-BFGS

enum : int { LS_CONTINUE = 0, LS_ACCEPT_PROBE = 1, LS_ACCEPT_LO = 2, LS_FAIL = 3 };

constexpr double kC1 = 1e-4, kC2 = 0.9, kApproxEps = 1e-6, kGrow = 2.0;

__device__ __forceinline__ bool sufficient(const LbState& L, double a, double f, double d) {
  if (!isfinite(f) || !isfinite(d)) return false;
  const double armijo = f - (L.f0 + kC1 * a * L.dphi0);
  const double approx = fmax(d - (2.0 * kC1 - 1.0) * L.dphi0, f - L.f0 - kApproxEps * fabs(L.f0));
  return fmin(armijo, approx) <= 0.0;
}

__device__ __forceinline__ bool curvature_ok(const LbState& L, double d) {
  return fabs(d) <= kC2 * fabs(L.dphi0);
}

// Safeguarded cubic step between lo and hi (Nocedal & Wright eq. 3.59),
// bisection when the cubic is undefined or leaves the inner 80% of the bracket.
__device__ double zoom_trial(const LbState& L) {
  const double al = L.a_lo, ah = L.a_hi;
  const double dlt = ah - al;
  const double lo_b = fmin(al, ah) + 0.1 * fabs(dlt);
  const double hi_b = fmax(al, ah) - 0.1 * fabs(dlt);
  if (isfinite(L.f_hi) && isfinite(L.d_hi) && dlt != 0.0) {
    const double d1 = L.d_lo + L.d_hi - 3.0 * (L.f_lo - L.f_hi) / (al - ah);
    const double disc = d1 * d1 - L.d_lo * L.d_hi;
    if (disc >= 0.0 && isfinite(disc)) {
      const double d2 = copysign(sqrt(disc), dlt);
      const double den = L.d_hi - L.d_lo + 2.0 * d2;
      const double a = ah - dlt * (L.d_hi + d2 - d1) / den;
      if (isfinite(a) && a >= lo_b && a <= hi_b) return a;
    }
  }
  return al + 0.5 * dlt;
}

// One probe result (alpha, f, d) -> decision. Sets *new_lo when the probe
// becomes the best point with sufficient decrease (its gradient is kept).
__device__ int ls_decide(LbState& L, double f, double d, int64_t max_ls, int* new_lo) {
  const double a = L.alpha;
  const bool suff = sufficient(L, a, f, d);
  *new_lo = 0;
  int out = LS_CONTINUE;
  if (L.phase == PH_EXPAND) {
    if (!suff || (L.ls_steps > 1 && f >= L.f_prev)) {
      L.a_lo = L.a_prev; L.f_lo = L.f_prev; L.d_lo = L.d_prev;   // (have_lo unchanged)
      L.a_hi = a; L.f_hi = f; L.d_hi = d;
      L.phase = PH_ZOOM;
    } else if (curvature_ok(L, d)) {
      return LS_ACCEPT_PROBE;
    } else if (d >= 0.0) {
      L.a_hi = L.a_prev; L.f_hi = L.f_prev; L.d_hi = L.d_prev;
      L.a_lo = a; L.f_lo = f; L.d_lo = d; L.have_lo = 1; *new_lo = 1;
      L.phase = PH_ZOOM;
    } else {
      L.a_prev = a; L.f_prev = f; L.d_prev = d;
      L.a_lo = a; L.f_lo = f; L.d_lo = d; L.have_lo = 1; *new_lo = 1;
      L.alpha = kGrow * a;
    }
  } else {
    if (!suff || f >= L.f_lo) {
      L.a_hi = a; L.f_hi = f; L.d_hi = d;
    } else {
      if (curvature_ok(L, d)) return LS_ACCEPT_PROBE;
      if (d * (L.a_hi - L.a_lo) >= 0.0) { L.a_hi = L.a_lo; L.f_hi = L.f_lo; L.d_hi = L.d_lo; }
      L.a_lo = a; L.f_lo = f; L.d_lo = d; L.have_lo = 1; *new_lo = 1;
    }
  }
  if (L.phase == PH_ZOOM) L.alpha = zoom_trial(L);
  if (L.ls_steps >= max_ls) out = L.have_lo ? LS_ACCEPT_LO : LS_FAIL;
  return out;
}

__device__ __forceinline__ int tri(int p, int q) { return q * (q + 1) / 2 + p; }  // p <= q

struct LbShared {
  LbState L;
  double red[32];
  int outcome, new_lo, advance, reeval, restart;
};

// Lane vectors and history rows have a padded length ld (a multiple of 4
// doubles, 16-byte aligned rows); padding entries stay zero, so every vector
// loop runs over ld/2 double2 words without a tail.
__device__ __forceinline__ double2 ld2(const double* p, int i) {
  return reinterpret_cast<const double2*>(p)[i];
}
__device__ __forceinline__ void st2(double* p, int i, double2 v) {
  reinterpret_cast<double2*>(p)[i] = v;
}

// An element loop over a lane's double2 words with U words per thread in
// flight: all U are loaded before any is stored, since the compiler cannot
// move a load across a store that may alias it. Thread t still handles the
// words t, t + blockDim.x, ..., each exactly as a one-at-a-time loop would.
template <int U, class Load, class Store>
__device__ __forceinline__ void lb_words(int h2, Load load, Store store) {
  for (int e0 = threadIdx.x; e0 < h2; e0 += U * blockDim.x) {
    decltype(load(0)) t[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * (int)blockDim.x;
      if (e < h2) t[u] = load(e);
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int e = e0 + u * (int)blockDim.x;
      if (e < h2) store(e, t[u]);
    }
  }
}

__device__ __forceinline__ LbView lane_view(const LbArgs& A, const LaneRef& R) {
  return lb_view(R.rec, A.m, A.tri_len, R.ld, A.keep_s0);
}

__device__ void lb_record(const LbArgs& A, int lane, const LaneRef& R, LbShared& sh,
                          const double* s) {
  if (A.traj_count == nullptr) return;
  __shared__ int64_t row;
  if (threadIdx.x == 0) {
    const int64_t c = A.traj_count[R.idx];
    const int64_t it = sh.L.it;
    row = ((it % A.rec_every) == 0 && c < A.rec_cap) ? c : -1;
    if (row >= 0) {
      A.traj_e[R.idx * A.rec_cap + row] = sh.L.f;
      A.traj_step[R.idx * A.rec_cap + row] = sh.L.last_step;
      A.traj_it[R.idx * A.rec_cap + row] = it;
      A.traj_count[R.idx] = c + 1;
    }
  }
  __syncthreads();
  if (row >= 0) {
    double* o = A.traj_s + R.toff + (size_t)row * R.nd;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) o[e] = wrap01(s[e]);
  }
  __syncthreads();
}

// End of an L-BFGS iteration (lbfgs.py:267-313): accept or keep the point,
// push the new (s, y) pair, update counters and statuses, and advance the
// rescale pass (history reset) when the pass ends. A lane that keeps running
// is flagged for a new direction (passes A, scalar, B of this tick).
__device__ void lb_end_iteration(const LbArgs& A, int lane, const LaneRef& R, const LbView& v,
                                 LbShared& sh) {
  LbState& L = sh.L;
  const int ld = R.ld, h2 = ld >> 1, m = A.m;
  double* x = v.x;
  double* s = v.s;
  double* g = v.g;
  const int outcome = sh.outcome;
  const bool fail = outcome == LS_FAIL;
  const double Rs = L.R;
  const double f_old = L.f;
  double ss_acc = 0.0;   // this thread's part of |g|^2 when the point moves
  __syncthreads();
  if (!fail) {
    const bool probe = outcome == LS_ACCEPT_PROBE;
    const double al = probe ? L.alpha : L.a_lo;
    const int sl = L.hhead;
    double* Sr = v.Sh + (size_t)sl * ld;
    double* Yr = v.Yh + (size_t)sl * ld;
    struct Words {
      double2 xo, dv, go, gn;
    };
    const double* gsrc = probe ? v.pg : v.glo;
    lb_words<4>(
        h2,
        [&](int e) { return Words{ld2(x, e), ld2(v.dir, e), ld2(g, e), ld2(gsrc, e)}; },
        [&](int e, const Words& w) {
          const double2 xn = make_double2(w.xo.x + al * w.dv.x, w.xo.y + al * w.dv.y);
          const double2 gn = probe ? make_double2(w.gn.x / Rs, w.gn.y / Rs) : w.gn;
          st2(Sr, e, make_double2(xn.x - w.xo.x, xn.y - w.xo.y));
          st2(Yr, e, make_double2(gn.x - w.go.x, gn.y - w.go.y));
          st2(x, e, xn);
          st2(s, e, make_double2(xn.x / Rs, xn.y / Rs));
          st2(g, e, gn);
          ss_acc += gn.x * gn.x + gn.y * gn.y;   // |g|^2, words in the same order as below
        });
    __syncthreads();
    if (threadIdx.x == 0) {
      L.f = L.f_lo;  // accepted energy (an accepted probe is stashed in f_lo)
      L.hhead = (L.hhead + 1) % m;
      L.hk = min(L.hk + 1, m);
      L.newpair = 1;
      L.last_step = al;
    }
  } else if (threadIdx.x == 0) {
    L.last_step = L.alpha;
  }
  __syncthreads();
  // |g_s| = |g_x| R; an accepted point summed its new g while storing it
  // (thread t over the words t, t + blockDim.x, ... in both cases)
  double ss = ss_acc;
  if (fail)
    for (int e = threadIdx.x; e < h2; e += blockDim.x) {
      const double2 gv = ld2(g, e);
      ss += gv.x * gv.x + gv.y * gv.y;
    }
  ss = block_sum(ss, sh.red);
  if (threadIdx.x == 0) {
    L.stag = (L.f < f_old) ? 0 : L.stag + 1;
    const int64_t ev = L.ls_steps > 1 ? L.ls_steps : 1;
    L.pass_evals += ev;
    L.n_evals += ev;
    L.it += 1;
    const double gnorm = sqrt(ss) * Rs;
    int glob = gnorm < A.grad_tol ? CCO_STATUS_GRAD_TOL : CCO_STATUS_RUNNING;
    if (L.f < A.energy_tol) glob = CCO_STATUS_ENERGY_TOL;
    int local = L.pass_evals >= A.budget ? CCO_STATUS_BUDGET : CCO_STATUS_RUNNING;
    if (L.stag >= A.patience) local = CCO_STATUS_STAGNATED;
    if (fail) local = CCO_STATUS_LINESEARCH_FAIL;
    // mixed precision: an FP32 lane never ends, and never ends a pass, on an
    // FP32 judgement. Once its energy is low, or on any outcome that would
    // stop it (energy or gradient tolerance, budget, stagnation, a failed
    // line search), it switches to FP64 at the current point; the FP64
    // re-evaluation and the FP64 iterations after it decide the status.
    bool sw = false;
    if (L.prec == PREC_FP32) {
      const bool low = L.f < kFp32SwitchPerParticle * (double)R.n;
      if (low || glob != CCO_STATUS_RUNNING || local != CCO_STATUS_RUNNING) {
        sw = true;
        glob = CCO_STATUS_RUNNING;
        local = CCO_STATUS_RUNNING;
      }
    }
    const bool last = L.pass_idx >= A.n_pass - 1;
    const bool pass_end = local != CCO_STATUS_RUNNING && glob == CCO_STATUS_RUNNING;
    const bool advance = pass_end && !last;
    int status = glob != CCO_STATUS_RUNNING ? glob : CCO_STATUS_RUNNING;
    if (pass_end && last) status = local;
    // a lane that started in FP32 and ends above the energy tolerance runs
    // again from s0 in FP64: the plain run of its configuration, bit for bit
    const bool restart = status != CCO_STATUS_RUNNING && L.mode == 1 && A.energy_tol > 0.0 &&
                         !(L.f < A.energy_tol);
    L.status = status;
    if (status != CCO_STATUS_RUNNING && !restart) L.t1 = gtimer();
    sh.advance = advance && !restart;
    sh.reeval = sw;
    sh.restart = restart;
    if (sw) {
      // fresh FP64 start at the current point: no history, one re-evaluation
      L.prec = PREC_FP64;
      L.phase = PH_REEVAL;
      L.hk = 0;
      L.hhead = 0;
      L.newpair = 0;
      L.stag = 0;
    }
  }
  __syncthreads();
  if (sh.reeval) {
    for (int e = threadIdx.x; e < h2; e += blockDim.x) st2(v.ps, e, ld2(s, e));
  }
  if (sh.advance) {
    const int nx = min(L.pass_idx + 1, A.n_pass - 1);
    const double rn = A.rescales[nx];
    for (int e = threadIdx.x; e < h2; e += blockDim.x) {
      const double2 sv = ld2(s, e), gv = ld2(g, e);
      st2(x, e, make_double2(sv.x * rn, sv.y * rn));
      st2(g, e, make_double2(gv.x * Rs / rn, gv.y * Rs / rn));
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      L.pass_idx += 1;
      L.R = rn;
      L.pass_evals = 0;
      L.stag = 0;
      L.hk = 0;
      L.hhead = 0;
      L.newpair = 0;
    }
  }
  __syncthreads();
  if (sh.restart) {
    // the fresh lane of k_lbfgs_init, keeping the clock and the counts spent
    for (int e = threadIdx.x; e < 7 * R.ld; e += blockDim.x) v.x[e] = 0.0;
    __syncthreads();
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) v.ps[e] = v.s0[e];
    if (threadIdx.x == 0) {
      LbState F = {};
      F.phase = PH_INIT;
      F.status = CCO_STATUS_RUNNING;
      F.R = A.rescales[0];
      F.prec = PREC_FP64;
      F.mode = 2;
      F.t0 = L.t0;
      F.n_fp32 = L.n_fp32;
      F.evals_prior = L.evals_prior + L.n_evals;
      L = F;
      if (A.traj_count) A.traj_count[R.idx] = 0;   // the trajectory of the run that counts
    }
    __syncthreads();
    return;
  }
  lb_record(A, lane, R, sh, s);
  if (threadIdx.x == 0 && L.status == CCO_STATUS_RUNNING && L.phase != PH_REEVAL)
    L.need_dir = 1;
}

// Lane start: probe positions = s0, every vector zero (padding included).
__global__ void k_lbfgs_init(LbArgs A, const double* __restrict__ s0) {
  const int lane = blockIdx.x;
  const LaneRef R = A.lanes[lane];
  const LbView v = lane_view(A, R);
  for (int e = threadIdx.x; e < 7 * R.ld; e += blockDim.x) v.x[e] = 0.0;
  __syncthreads();
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) v.ps[e] = s0[R.soff + e];
  if (v.s0)
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) v.s0[e] = s0[R.soff + e];
  if (threadIdx.x == 0) {
    LbState L = {};
    L.phase = PH_INIT;
    L.status = CCO_STATUS_RUNNING;
    L.R = A.rescales[0];
    // mixed precision starts lanes of d >= 2 (N d > N) in FP32
    L.prec = (A.prec0 == PREC_FP32 && R.nd > R.n) ? PREC_FP32 : PREC_FP64;
    L.mode = L.prec == PREC_FP32 ? 1 : 0;
    L.t0 = gtimer();
    *v.st = L;
    if (A.traj_count) A.traj_count[R.idx] = 0;
  }
}

// Probe kernel: one CTA per lane. Starts the line search of a direction
// built by the previous tick's passes, consumes this tick's probe and either
// places the next probe or ends the iteration.
__global__ void __launch_bounds__(kUpdThreads, 2) k_lbfgs_probe(LbArgs A) {
  __shared__ LbShared sh;
  const int lane = blockIdx.x;
  const LaneRef R = A.lanes[lane];
  const LbView v = lane_view(A, R);
  if (threadIdx.x == 0) sh.L = *v.st;
  __syncthreads();
  if (sh.L.status != CCO_STATUS_RUNNING) return;
  LbState& L = sh.L;
  const int h2 = R.ld >> 1;
  if (threadIdx.x == 0 && L.prec == PREC_FP32) L.n_fp32 += 1;   // this tick's evaluation
  if (L.phase == PH_REEVAL) {
    // the FP64 evaluation of the current point after a precision switch
    const double Rs = L.R;
    for (int e = threadIdx.x; e < h2; e += blockDim.x) {
      const double2 gv = ld2(v.pg, e);
      st2(v.g, e, make_double2(gv.x / Rs, gv.y / Rs));
    }
    if (threadIdx.x == 0) {
      L.f = *v.pf;
      L.n_evals += 1;
      L.pass_evals += 1;
      L.phase = PH_EXPAND;
      if (L.f < A.energy_tol) {
        L.status = CCO_STATUS_ENERGY_TOL;
        L.t1 = gtimer();
      } else {
        L.need_dir = 1;
      }
    }
  } else if (L.phase == PH_INIT) {
    // init_one (lbfgs.py:163-197): x = R0 s0, g_x = g_s / R0, one evaluation
    const double R0 = L.R;
    for (int e = threadIdx.x; e < h2; e += blockDim.x) {
      const double2 sv = ld2(v.ps, e), gv = ld2(v.pg, e);
      st2(v.s, e, sv);
      st2(v.x, e, make_double2(sv.x * R0, sv.y * R0));
      st2(v.g, e, make_double2(gv.x / R0, gv.y / R0));
    }
    if (threadIdx.x == 0) {
      L.f = *v.pf;
      L.n_evals = 1;
      L.status = L.f < A.energy_tol ? CCO_STATUS_ENERGY_TOL : CCO_STATUS_RUNNING;
      L.last_step = 0.0;
      L.phase = PH_EXPAND;
      if (L.status != CCO_STATUS_RUNNING && L.prec == PREC_FP32) {
        // an FP32 start below the tolerance is judged again in FP64
        L.status = CCO_STATUS_RUNNING;
        L.prec = PREC_FP64;
        L.phase = PH_REEVAL;
      } else if (L.status != CCO_STATUS_RUNNING) {
        L.t1 = gtimer();
      } else {
        L.need_dir = 1;
      }
    }
    __syncthreads();
    lb_record(A, lane, R, sh, v.s);
  } else {
    if (L.need_dir) {
      // the direction and the first probe (alpha = 1) were written by pass B;
      // g.dir is the sum of its block partials (a wide lane's many partials:
      // strided per thread, then the block tree)
      const double* dpart = v.scal + 4 * A.m + 1;
      const int nb = lb_nblk(R.ld);
      double dpw = 0.0;
      if (lb_wide(R.ld)) {
        for (int b = threadIdx.x; b < nb; b += blockDim.x) dpw += dpart[b];
        dpw = block_sum(dpw, sh.red);
      }
      if (threadIdx.x == 0) {
        double dp = 0.0;
        if (lb_wide(R.ld))
          dp = dpw;
        else
          for (int b = 0; b < nb; ++b) dp += dpart[b];
        L.f0 = L.f;
        L.dphi0 = dp;
        L.phase = PH_EXPAND;
        L.ls_steps = 0;
        L.alpha = 1.0;
        L.a_prev = 0.0; L.f_prev = L.f; L.d_prev = dp;
        L.a_lo = 0.0; L.f_lo = L.f; L.d_lo = dp;
        L.a_hi = 0.0; L.f_hi = L.f; L.d_hi = dp;
        L.have_lo = 0;
        L.newpair = 0;
        L.need_dir = 0;
      }
      __syncthreads();
    }
    // one probe of the line search
    const double Rs = L.R;
    double dp = 0.0;
    {
      // eight words per thread in flight, added in the order of a one-word loop
      constexpr int U = 8;
      for (int e0 = threadIdx.x; e0 < h2; e0 += U * blockDim.x) {
        double2 pv[U], dv[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int e = e0 + u * (int)blockDim.x;
          if (e < h2) {
            pv[u] = ld2(v.pg, e);
            dv[u] = ld2(v.dir, e);
          }
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (e0 + u * (int)blockDim.x < h2) dp += (pv[u].x / Rs) * dv[u].x + (pv[u].y / Rs) * dv[u].y;
      }
    }
    dp = block_sum(dp, sh.red);
    if (threadIdx.x == 0) {
      L.ls_steps += 1;
      int nl = 0;
      const double fp = *v.pf;
      sh.outcome = ls_decide(L, fp, dp, A.max_ls, &nl);
      sh.new_lo = nl;
      if (sh.outcome == LS_ACCEPT_PROBE) L.f_lo = fp;  // read by end_iteration
    }
    __syncthreads();
    if (sh.new_lo) {
      lb_words<8>(
          h2, [&](int e) { return ld2(v.pg, e); },
          [&](int e, double2 pv) { st2(v.glo, e, make_double2(pv.x / Rs, pv.y / Rs)); });
    }
    if (sh.outcome == LS_CONTINUE) {
      const double al = L.alpha;
      struct Words {
        double2 xv, dv;
      };
      lb_words<4>(
          h2, [&](int e) { return Words{ld2(v.x, e), ld2(v.dir, e)}; },
          [&](int e, const Words& w) {
            st2(v.ps, e,
                make_double2((w.xv.x + al * w.dv.x) / Rs, (w.xv.y + al * w.dv.y) / Rs));
          });
    } else {
      __syncthreads();
      lb_end_iteration(A, lane, R, v, sh);
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) *v.st = sh.L;
}

// Pass A (grid: pair blocks x element chunks, lanes): a_p = s_p.g, b_p = y_p.g
// for every stored pair and, after a push, the newest pair's column s_p.y_n,
// y_p.y_n. One warp per (pair, chunk) with four double2 words per lane in
// flight; a lane of one chunk writes the dots, a wide lane its partials.
__global__ void __launch_bounds__(kUpdThreads) k_lbfgs_passA(LbArgs A) {
  const int lane = blockIdx.y;
  const LaneRef R = A.lanes[lane];
  const int chunk = blockIdx.x % A.nchA, pblk = blockIdx.x / A.nchA;
  const int nch = lb_achunks(R.ld);
  if (chunk >= nch) return;
  const LbView v = lane_view(A, R);
  const LbState* Lp = v.st;
  const int k = Lp->hk;
  if (Lp->status != CCO_STATUS_RUNNING || !Lp->need_dir || k == 0) return;
  const int warp = threadIdx.x >> 5, wl = threadIdx.x & 31;
  const int p = pblk * (kUpdThreads / 32) + warp;
  if (p >= k) return;
  const int ld = R.ld, m = A.m;
  const int e_lo = chunk * kLbWide;
  const int h2 = nch == 1 ? (ld >> 1) : min(ld >> 1, e_lo + kLbWide);   // end of this chunk
  const int head = Lp->hhead;
  const bool np = Lp->newpair != 0;
  const int sp = (head - k + p + m) % m, sn = (head - 1 + m) % m;
  const double* g = v.g;
  const double* sr = v.Sh + (size_t)sp * ld;
  const double* yr = v.Yh + (size_t)sp * ld;
  const double* yn = v.Yh + (size_t)sn * ld;
  double ag = 0.0, bg = 0.0, sy = 0.0, yy = 0.0;
  int e = (nch == 1 ? 0 : e_lo) + wl;
  for (; e + 96 < h2; e += 128) {
    double2 sv[4], yv[4], gv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      sv[u] = ld2(sr, e + 32 * u);
      yv[u] = ld2(yr, e + 32 * u);
      gv[u] = ld2(g, e + 32 * u);
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      ag += sv[u].x * gv[u].x + sv[u].y * gv[u].y;
      bg += yv[u].x * gv[u].x + yv[u].y * gv[u].y;
    }
    if (np) {
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const double2 w = ld2(yn, e + 32 * u);
        sy += sv[u].x * w.x + sv[u].y * w.y;
        yy += yv[u].x * w.x + yv[u].y * w.y;
      }
    }
  }
  for (; e < h2; e += 32) {
    const double2 sv = ld2(sr, e), yv = ld2(yr, e), gv = ld2(g, e);
    ag += sv.x * gv.x + sv.y * gv.y;
    bg += yv.x * gv.x + yv.y * gv.y;
    if (np) {
      const double2 w = ld2(yn, e);
      sy += sv.x * w.x + sv.y * w.y;
      yy += yv.x * w.x + yv.y * w.y;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ag += __shfl_xor_sync(0xffffffffu, ag, o);
    bg += __shfl_xor_sync(0xffffffffu, bg, o);
    sy += __shfl_xor_sync(0xffffffffu, sy, o);
    yy += __shfl_xor_sync(0xffffffffu, yy, o);
  }
  if (wl == 0) {
    double* sc = v.scal;
    if (nch == 1) {
      sc[p] = ag;
      sc[m + p] = bg;
      if (np) {
        v.SY[(size_t)sn * m + sp] = sy;   // row = newer slot
        v.YY[(size_t)sp * m + sn] = yy;
        v.YY[(size_t)sn * m + sp] = yy;
      }
    } else {
      double* ap = sc + lb_apart_off(m, ld) + (size_t)chunk * 4 * m;
      ap[p] = ag;
      ap[m + p] = bg;
      if (np) {
        ap[2 * m + p] = sy;
        ap[3 * m + p] = yy;
      }
    }
  }
}

// The dots of a wide lane: its pass-A chunk partials summed in chunk order.
__device__ void lb_sum_apart(const LbArgs& A, const LaneRef& R, const LbView& v, int k,
                             int head, bool np) {
  const int m = A.m, nch = lb_achunks(R.ld);
  const double* ap = v.scal + lb_apart_off(m, R.ld);
  const int sn = (head - 1 + m) % m;
  for (int p = threadIdx.x; p < k; p += blockDim.x) {
    double ag = ap[p], bg = ap[m + p], sy = 0.0, yy = 0.0;
    if (np) {
      sy = ap[2 * m + p];
      yy = ap[3 * m + p];
    }
    for (int c = 1; c < nch; ++c) {
      const double* q = ap + (size_t)c * 4 * m;
      ag += q[p];
      bg += q[m + p];
      if (np) {
        sy += q[2 * m + p];
        yy += q[3 * m + p];
      }
    }
    v.scal[p] = ag;
    v.scal[m + p] = bg;
    if (np) {
      const int sp = (head - k + p + m) % m;
      v.SY[(size_t)sn * m + sp] = sy;
      v.YY[(size_t)sp * m + sn] = yy;
      v.YY[(size_t)sn * m + sp] = yy;
    }
  }
  __syncthreads();
}

// Scalar kernel (one CTA per lane): gamma and the coefficients of the
// direction from the inner products. The lower triangles of SY (s_older .
// y_newer) and YY are gathered from the slot matrices into shared memory in
// logical (oldest-first) order with every thread keeping eight loads in
// flight - the slot matrices are usually L2 misses by now, so the gather is
// latency-bound and needs the parallelism. Loop 1 then runs column-oriented
// (one shuffle per step) and loop 2 row-oriented; both read contiguous
// shared-memory rows.
__global__ void __launch_bounds__(kUpdThreads) k_lbfgs_scalar(LbArgs A) {
  extern __shared__ double dsm[];
  __shared__ double av[kScalarMaxPairs], bv[kScalarMaxPairs], alp[kScalarMaxPairs],
      bet[kScalarMaxPairs], rh[kScalarMaxPairs];
  __shared__ int sl[kScalarMaxPairs];
  __shared__ double red[32];
  __shared__ double gam_s;
  const int lane = blockIdx.x;
  const LaneRef R = A.lanes[lane];
  const LbView v = lane_view(A, R);
  const LbState* Lp = v.st;
  if (Lp->status != CCO_STATUS_RUNNING || !Lp->need_dir) return;
  const int k = Lp->hk, m = A.m, head = Lp->hhead;
  double* sc = v.scal;
  const int warp = threadIdx.x >> 5, wl = threadIdx.x & 31;
  if (k > 0 && lb_wide(R.ld)) lb_sum_apart(A, R, v, k, head, Lp->newpair != 0);
  // two packings by newer rows (tri(p, q) = q (q + 1) / 2 + p, p <= q):
  // triSY (SY[p][q] = s_p . y_q, p older than q) and triYY (the symmetric YY).
  // Two triangles (2 m (m + 1) / 2 doubles, 81 KB at m = 100) let two CTAs
  // share an SM, so a 256-lane update runs in one wave.
  const size_t tri_n = (size_t)m * (m + 1) / 2;
  double* triSY = A.smem_tri ? dsm : v.tri;
  double* triYY = triSY + tri_n;
  if (k > 0) {
    const double* SYt = v.SY;
    const double* YYs = v.YY;
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
      sl[p] = (head - k + p + m) % m;
      av[p] = sc[p];
      bv[p] = sc[m + p];
    }
    __syncthreads();
    const int total = k * (k + 1) / 2;
    constexpr int U = 8;
    for (int t0 = threadIdx.x; t0 < total; t0 += U * blockDim.x) {
      double xs[U], xy[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int t = t0 + u * blockDim.x;
        // row of packed index t: an FP32 estimate, made exact by the two
        // integer corrections below (t < m (m + 1) / 2 is far below 2^24)
        int q = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
        while (q * (q + 1) / 2 > t) --q;
        while ((q + 1) * (q + 2) / 2 <= t) ++q;
        const int p = t - q * (q + 1) / 2;
        if (t < total) {
          xs[u] = SYt[(size_t)sl[q] * m + sl[p]];
          xy[u] = YYs[(size_t)sl[q] * m + sl[p]];
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int t = t0 + u * blockDim.x;
        if (t < total) {
          triSY[t] = xs[u];
          triYY[t] = xy[u];
        }
      }
    }
    __syncthreads();
    for (int p = threadIdx.x; p < k; p += blockDim.x) {
      const double ys = triSY[tri(p, p)];
      rh[p] = ys == 0.0 ? 0.0 : 1.0 / ys;
    }
    if (threadIdx.x == 0) {
      const int n = k - 1;
      const double num = triSY[tri(n, n)], den = triYY[tri(n, n)];
      gam_s = den > 0.0 ? num / den : 1.0;
    }
  } else {
    // gamma (optax scale_by_lbfgs) on a fresh pass: min(1, 1/|g|)
    double ss = 0.0;
    for (int e = threadIdx.x; e < (R.ld >> 1); e += blockDim.x) {
      const double2 gv = ld2(v.g, e);
      ss += gv.x * gv.x + gv.y * gv.y;
    }
    ss = block_sum(ss, red);
    if (threadIdx.x == 0) gam_s = fmin(1.0, 1.0 / sqrt(ss));
  }
  __syncthreads();
  const double gam = gam_s;
  if (threadIdx.x == 0) sc[2 * m] = gam;
  if (k == 0) return;
  constexpr int R8 = kScalarMaxPairs / 32;
  // Loops 1 and 2 run on warp 0 with lane l holding the entries p = 32 i + l
  // in register i. Both are unrolled over i so that every register index is
  // a compile-time constant: the step's critical path is one multiply, one
  // shuffle and one FMA.
  if (warp == 0) {
    // loop 1 (newest first): alpha_q = rho_q t_q, then t_p -= alpha_q SY[p][q], p < q
    double tv[R8];
#pragma unroll
    for (int i = 0; i < R8; ++i) tv[i] = (32 * i + wl < k) ? av[32 * i + wl] : 0.0;
#pragma unroll
    for (int oi = R8 - 1; oi >= 0; --oi) {
      if (32 * oi < k) {
        const int top = min(31, k - 1 - 32 * oi);
        for (int own = top; own >= 0; --own) {
          const int q = 32 * oi + own;
          const double* row = triSY + q * (q + 1) / 2;
          const double aq = __shfl_sync(0xffffffffu, rh[q] * tv[oi], own);
          if (wl == 0) alp[q] = aq;
#pragma unroll
          for (int i = 0; i <= oi; ++i) {
            const int p = 32 * i + wl;
            if (p < q) tv[i] -= aq * row[p];
          }
        }
      }
    }
  }
  __syncthreads();
  // t2_p = b_p - sum_q alpha_q YY[p][q] (a thread per p; triYY row r holds
  // YY[p][r] for p <= r, so q < p reads row p and q >= p reads column p)
  for (int p = threadIdx.x; p < k; p += blockDim.x) {
    const double* rp = triYY + p * (p + 1) / 2;
    double acc = 0.0;
    for (int q = 0; q < p; ++q) acc += alp[q] * rp[q];
    for (int q = p; q < k; ++q) acc += alp[q] * triYY[q * (q + 1) / 2 + p];
    bet[p] = bv[p] - acc;   // holds t2_p until loop 2 overwrites it
  }
  __syncthreads();
  if (warp == 0) {
    // loop 2 (oldest first, column-oriented): beta_p = rho_p (gamma t2_p + u_p),
    // then u_q += (alpha_p - beta_p) SY[p][q] for every newer q. Every lane
    // forms the candidate from its own u and the owner's is shuffled out, as
    // in loop 1 (no divergent owner branch).
    double u[R8];
#pragma unroll
    for (int i = 0; i < R8; ++i) u[i] = 0.0;
#pragma unroll
    for (int oi = 0; oi < R8; ++oi) {
      if (32 * oi < k) {
        const int top = min(31, k - 1 - 32 * oi);
        for (int own = 0; own <= top; ++own) {
          const int p = 32 * oi + own;
          const double* col = triSY + p;   // col[q (q + 1) / 2] = SY[p][q]
          const double bp = __shfl_sync(0xffffffffu, rh[p] * (gam * bet[p] + u[oi]), own);
          const double dq = alp[p] - bp;
          if (wl == 0) bet[p] = bp;
#pragma unroll
          for (int i = oi; i < R8; ++i) {
            const int q = 32 * i + wl;
            if (q > p && q < k) u[i] += dq * col[q * (q + 1) / 2];
          }
        }
      }
    }
    __syncwarp();
    for (int q = wl; q < k; q += 32) {
      sc[2 * m + 1 + q] = gam * alp[q];        // cy_q
      sc[3 * m + 1 + q] = bet[q] - alp[q];     // cs_q
    }
  }
}

// Pass B (grid: element blocks x lanes): dir = -gamma g + sum cy_q y_q +
// sum cs_q s_q, the first probe s = (x + dir) / R and this block's part of
// g.dir. One double2 word per thread, eight pairs (16 loads) in flight.
__global__ void __launch_bounds__(kUpdThreads) k_lbfgs_passB(LbArgs A) {
  __shared__ double cyv[kPassBMaxPairs], csv[kPassBMaxPairs];
  __shared__ double red[32];
  const int lane = blockIdx.y;
  const LaneRef R = A.lanes[lane];
  if ((int)blockIdx.x >= lb_nblk(R.ld)) return;   // this lane has fewer element blocks
  const LbView v = lane_view(A, R);
  const LbState* Lp = v.st;
  if (Lp->status != CCO_STATUS_RUNNING || !Lp->need_dir) return;
  const int k = Lp->hk, m = A.m, head = Lp->hhead;
  const int ld = R.ld, h2 = ld >> 1;
  const double Rs = Lp->R;
  double* sc = v.scal;
  const double gam = sc[2 * m];
  const bool in_smem = k <= kPassBMaxPairs;
  if (in_smem) {
    for (int q = threadIdx.x; q < k; q += blockDim.x) {
      cyv[q] = sc[2 * m + 1 + q];
      csv[q] = sc[3 * m + 1 + q];
    }
  }
  __syncthreads();
  const double* cy = in_smem ? cyv : sc + 2 * m + 1;
  const double* cs = in_smem ? csv : sc + 3 * m + 1;
  const double* Sh = v.Sh;
  const double* Yh = v.Yh;
  double dp = 0.0;
  if (lb_wide(ld)) {
    // warp w sums the pairs [w k / G, (w + 1) k / G) for the block's 32 words;
    // warp 0 adds the G group sums in order and finishes the words
    __shared__ double2 gsum[kPassBGroups][32];
    const int w = threadIdx.x >> 5, wl = threadIdx.x & 31;
    const int e = blockIdx.x * 32 + wl;
    const int q1 = (w + 1) * k / kPassBGroups;
    double ax = 0.0, ay = 0.0;
    if (e < h2) {
      int q = w * k / kPassBGroups;
      for (; q + 8 <= q1; q += 8) {
        double2 yv[8], sv[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          const size_t r = (size_t)((head - k + q + u + m) % m) * ld;
          yv[u] = ld2(Yh + r, e);
          sv[u] = ld2(Sh + r, e);
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
          ax += cy[q + u] * yv[u].x + cs[q + u] * sv[u].x;
          ay += cy[q + u] * yv[u].y + cs[q + u] * sv[u].y;
        }
      }
      for (; q < q1; ++q) {
        const size_t r = (size_t)((head - k + q + m) % m) * ld;
        const double2 yv = ld2(Yh + r, e), sv = ld2(Sh + r, e);
        ax += cy[q] * yv.x + cs[q] * sv.x;
        ay += cy[q] * yv.y + cs[q] * sv.y;
      }
    }
    gsum[w][wl] = make_double2(ax, ay);
    __syncthreads();
    if (w == 0 && e < h2) {
      double2 t = gsum[0][wl];
#pragma unroll
      for (int g = 1; g < kPassBGroups; ++g) {
        t.x += gsum[g][wl].x;
        t.y += gsum[g][wl].y;
      }
      const double2 gv = ld2(v.g, e), xv = ld2(v.x, e);
      const double2 de = make_double2(t.x - gam * gv.x, t.y - gam * gv.y);
      st2(v.dir, e, de);
      dp = gv.x * de.x + gv.y * de.y;
      st2(v.ps, e, make_double2((xv.x + 1.0 * de.x) / Rs, (xv.y + 1.0 * de.y) / Rs));
    }
    dp = block_sum(dp, red);
    if (threadIdx.x == 0) sc[4 * m + 1 + blockIdx.x] = dp;
    return;
  }
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < h2) {
    double ax = 0.0, ay = 0.0;
    int q = 0;
    for (; q + 8 <= k; q += 8) {
      double2 yv[8], sv[8];
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        const size_t r = (size_t)((head - k + q + u + m) % m) * ld;
        yv[u] = ld2(Yh + r, e);
        sv[u] = ld2(Sh + r, e);
      }
#pragma unroll
      for (int u = 0; u < 8; ++u) {
        ax += cy[q + u] * yv[u].x + cs[q + u] * sv[u].x;
        ay += cy[q + u] * yv[u].y + cs[q + u] * sv[u].y;
      }
    }
    for (; q < k; ++q) {
      const size_t r = (size_t)((head - k + q + m) % m) * ld;
      const double2 yv = ld2(Yh + r, e), sv = ld2(Sh + r, e);
      ax += cy[q] * yv.x + cs[q] * sv.x;
      ay += cy[q] * yv.y + cs[q] * sv.y;
    }
    const double2 gv = ld2(v.g, e), xv = ld2(v.x, e);
    const double2 de = make_double2(ax - gam * gv.x, ay - gam * gv.y);
    st2(v.dir, e, de);
    dp = gv.x * de.x + gv.y * de.y;
    st2(v.ps, e, make_double2((xv.x + 1.0 * de.x) / Rs, (xv.y + 1.0 * de.y) / Rs));
  }
  dp = block_sum(dp, red);
  if (threadIdx.x == 0) sc[4 * m + 1 + blockIdx.x] = dp;
}

__global__ void k_lbfgs_finalize(LbArgs A, double* s_out, double* e_out, double* gn_out,
                                 int64_t* ne_out, int64_t* ni_out, int64_t* st_out,
                                 int64_t* lat_out, int64_t* n32_out) {
  __shared__ double red[32];
  const int lane = blockIdx.x;
  const LaneRef R = A.lanes[lane];
  const LbView v = lane_view(A, R);
  double ss = 0.0;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    const double gv = v.g[e];
    ss += gv * gv;
    s_out[R.soff + e] = wrap01(v.s[e]);
  }
  ss = block_sum(ss, red);
  if (threadIdx.x == 0) {
    const LbState L = *v.st;
    e_out[lane] = L.f;
    gn_out[lane] = sqrt(ss) * L.R;
    ne_out[lane] = L.n_evals + L.evals_prior;
    ni_out[lane] = L.it;
    st_out[lane] = L.status;
    if (lat_out) lat_out[lane] = L.t1 - L.t0;
    if (n32_out) n32_out[lane] = L.n_fp32;
  }
}

__global__ void k_count_running(const LaneRef* lanes, int B, int* out) {
  __shared__ double red[32];
  double c = 0.0;
  for (int i = threadIdx.x; i < B; i += blockDim.x)
    c += (*rec_status(lanes[i].rec) == CCO_STATUS_RUNNING) ? 1.0 : 0.0;
  c = block_sum(c, red);
  if (threadIdx.x == 0) *out = (int)c;
}

__global__ void k_gather_status(const LaneRef* lanes, int B, int64_t* out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x)
    out[i] = *rec_status(lanes[i].rec);
}

__global__ void k_cancel_lbfgs(double* rec) {
  LbState* L = reinterpret_cast<LbState*>(rec);
  if (L->status == CCO_STATUS_RUNNING) {
    L->status = CCO_STATUS_CANCELLED;
    L->t1 = gtimer();
  }
}

}  // namespace

cudaError_t descent_init(const DescentArgs& a, const double* s0, cudaStream_t st) {
  k_descent_init<<<a.B, kUpdThreads, 0, st>>>(a, s0);
  return cudaGetLastError();
}
cudaError_t descent_update(const DescentArgs& a, cudaStream_t st) {
  k_descent_update<<<a.B, kUpdThreads, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t descent_finalize(const DescentArgs& a, double* s_out, double* e_out, double* gn_out,
                             int64_t* ne_out, int64_t* ni_out, int64_t* st_out, int64_t* lat_out,
                             cudaStream_t st) {
  k_descent_finalize<<<a.B, kUpdThreads, 0, st>>>(a, s_out, e_out, gn_out, ne_out, ni_out,
                                                  st_out, lat_out);
  return cudaGetLastError();
}

size_t lbfgs_update_smem(int m) { return 2 * ((size_t)m * (m + 1) / 2) * sizeof(double); }
cudaError_t lbfgs_configure(size_t smem) {
  return cudaFuncSetAttribute(k_lbfgs_scalar, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)smem);
}
cudaError_t lbfgs_init(const LbArgs& a, const double* s0, cudaStream_t st) {
  k_lbfgs_init<<<a.B, kUpdThreads, 0, st>>>(a, s0);
  return cudaGetLastError();
}
// One tick of the minimizer: the probe kernel for every lane, then the three
// direction stages, which exit at once for lanes that are mid line search.
cudaError_t lbfgs_update(const LbArgs& a, cudaStream_t st) {
  k_lbfgs_probe<<<a.B, kUpdThreads, 0, st>>>(a);
  const dim3 ga((a.m + kUpdThreads / 32 - 1) / (kUpdThreads / 32) * a.nchA, a.B);
  k_lbfgs_passA<<<ga, kUpdThreads, 0, st>>>(a);
  k_lbfgs_scalar<<<a.B, kUpdThreads, a.smem_tri, st>>>(a);
  const dim3 gb(a.nblkB, a.B);
  k_lbfgs_passB<<<gb, kUpdThreads, 0, st>>>(a);
  return cudaGetLastError();
}
cudaError_t lbfgs_finalize(const LbArgs& a, double* s_out, double* e_out, double* gn_out,
                           int64_t* ne_out, int64_t* ni_out, int64_t* st_out, int64_t* lat_out,
                           int64_t* n32_out, cudaStream_t st) {
  k_lbfgs_finalize<<<a.B, kUpdThreads, 0, st>>>(a, s_out, e_out, gn_out, ne_out, ni_out, st_out,
                                                lat_out, n32_out);
  return cudaGetLastError();
}
cudaError_t count_running(const LaneRef* lanes, int B, int* out, cudaStream_t st) {
  k_count_running<<<1, 256, 0, st>>>(lanes, B, out);
  return cudaGetLastError();
}
cudaError_t gather_status(const LaneRef* lanes, int B, int64_t* out, cudaStream_t st) {
  int blocks = (B + 255) / 256;
  k_gather_status<<<blocks < 1 ? 1 : blocks, 256, 0, st>>>(lanes, B, out);
  return cudaGetLastError();
}

cudaError_t cancel_lbfgs_lane(double* rec, cudaStream_t st) {
  k_cancel_lbfgs<<<1, 1, 0, st>>>(rec);
  return cudaGetLastError();
}

}  // namespace cco
