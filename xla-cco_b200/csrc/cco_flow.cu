// Gradient flow on sm_100a: adaptive Dormand-Prince 5(4) per lane (FP64).
//
// Reference: gradient_flow (src/xla_cco/minimize/flow.py:258-364,401-451)
// integrates ds/dt = -grad_s Phi (B B^T)^-1 (or the unit-speed arclength
// form) with the Dormand-Prince 5(4) pair, FSAL, a step controller (safety
// 0.9, factor clipped to [0.2, 5], exponent -1/5) and a local error measured
// as RMS Cartesian displacement error over atol + rtol * RMS Cartesian step;
// the flow time and arclength ride along under the same relative control.
//
// B200 formulation: each lane is a stage machine that advances one stage per
// tick - the tick's evaluation (cco_eval.cu) is the stage's energy and
// gradient at the probe position ps, and k_flow_update turns it into the
// stage velocity and places the next probe. An attempted step is six ticks
// (stages 2..7; stage 1 is the previous step's last, FSAL). Lanes of
// different N, d, basis and k-set share the launches; a finished lane is
// frozen and skipped.
#include <cmath>

#include "cco_flow.cuh"

namespace cco {

namespace {

// Dormand & Prince (1980) 5(4) tableau: stage matrix, 5th-order weights and
// the difference of the 5th- and embedded 4th-order weights (with FSAL).
__constant__ double kA[7][6] = {
    {0, 0, 0, 0, 0, 0},
    {1.0 / 5, 0, 0, 0, 0, 0},
    {3.0 / 40, 9.0 / 40, 0, 0, 0, 0},
    {44.0 / 45, -56.0 / 15, 32.0 / 9, 0, 0, 0},
    {19372.0 / 6561, -25360.0 / 2187, 64448.0 / 6561, -212.0 / 729, 0, 0},
    {9017.0 / 3168, -355.0 / 33, 46732.0 / 5247, 49.0 / 176, -5103.0 / 18656, 0},
    {0, 0, 0, 0, 0, 0}};
__constant__ double kB5[7] = {35.0 / 384, 0.0, 500.0 / 1113, 125.0 / 192, -2187.0 / 6784,
                              11.0 / 84, 0.0};
__constant__ double kB4[7] = {5179.0 / 57600, 0.0, 7571.0 / 16695, 393.0 / 640,
                              -92097.0 / 339200, 187.0 / 2100, 1.0 / 40};
constexpr double kSafety = 0.9, kShrinkMin = 0.2, kGrowMax = 5.0;

__device__ __forceinline__ int64_t gtimer() {
  uint64_t v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  return (int64_t)v;
}

// Stop code; precedence energy > gradient > time/budget > step floor
// (flow.py:_status).
__device__ int flow_status(const FlArgs& a, double f, bool all_zero, double gnorm, double t,
                           double dt, int64_t steps, int64_t tries) {
  int code = dt < a.dt_min ? CCO_STATUS_STEP_FLOOR : CCO_STATUS_RUNNING;
  const bool over = (t >= a.t_max) || (steps >= a.max_steps);
  if (over || tries >= 4 * a.max_steps) code = CCO_STATUS_BUDGET;
  if (all_zero || gnorm < a.grad_tol) code = CCO_STATUS_GRAD_TOL;
  if (f < a.energy_tol) code = CCO_STATUS_ENERGY_TOL;
  return code;
}

struct FlShared {
  FlState S;
  double red[32];
  int all_zero;
};

// Stage velocity from the probe gradient pg into kv: v = -g (B B^T)^-1,
// scaled by 1/|g B^-T| in arclength mode; returns |g B^-T| and whether g is
// exactly zero (block-wide, every thread).
__device__ double stage_velocity(const FlArgs& a, const LaneRef& R, const FlState& S,
                                 const double* pg, double* kv, double* red, int* all_zero) {
  const int d = R.nd / R.n;
  double ss = 0.0;
  int nz = 0;
  for (int j = threadIdx.x; j < R.n; j += blockDim.x) {
    double gj[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < d; ++b) {
      gj[b] = pg[(size_t)j * d + b];
      nz |= gj[b] != 0.0;
    }
    for (int c = 0; c < d; ++c) {
      double v = 0.0, gc = 0.0;
      for (int b = 0; b < d; ++b) {
        v += gj[b] * S.Minv[b * 3 + c];
        gc += gj[b] * S.BinvT[b * 3 + c];
      }
      kv[(size_t)j * d + c] = -v;
      ss += gc * gc;
    }
  }
  ss = block_sum(ss, red);
  nz = __syncthreads_or(nz);
  *all_zero = !nz;
  const double gn = sqrt(ss);
  if (a.arclength) {
    const double inv = gn > 0.0 ? 1.0 / gn : 0.0;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) kv[e] = kv[e] * inv;
    __syncthreads();
  }
  return gn;
}

__device__ __forceinline__ void stage_rate(const FlArgs& a, double gn, double* rate) {
  if (a.arclength) {
    rate[0] = gn > 0.0 ? 1.0 / gn : 0.0;
    rate[1] = 1.0;
  } else {
    rate[0] = 1.0;
    rate[1] = gn;
  }
}

// ps = s + dt * sum_j A[i][j] k_j (j < i): the position of stage i (0-based).
__device__ void place_stage(const LaneRef& R, const FlView& v, int i, double dt) {
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    double incr = 0.0;
    for (int j = 0; j < i; ++j) incr += kA[i][j] * v.k[(size_t)j * R.ld + e];
    v.ps[e] = v.s[e] + dt * incr;
  }
}

__device__ void flow_record(const FlArgs& a, const LaneRef& R, FlState& S, const double* s) {
  if (a.traj_count == nullptr) return;
  __shared__ int64_t row;
  if (threadIdx.x == 0) {
    row = S.count < a.rec_cap ? S.count : -1;
    if (row >= 0) {
      const size_t o = (size_t)R.idx * a.rec_cap + row;
      a.traj_t[o] = S.t;
      a.traj_len[o] = S.length;
      a.traj_e[o] = S.f;
      S.count += 1;
    }
  }
  __syncthreads();
  if (row >= 0) {
    double* out = a.traj_s + R.toff + (size_t)row * R.nd;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) out[e] = s[e];
  }
  __syncthreads();
}

// Start of an attempted step: the step size (clipped to t_max in time mode)
// and the stage-2 probe.
__device__ void begin_step(const FlArgs& a, const LaneRef& R, const FlView& v, FlShared& sh) {
  if (threadIdx.x == 0) {
    double dt = sh.S.dt;
    if (!a.arclength) dt = fmin(dt, a.t_max - sh.S.t);
    sh.S.dt_step = dt;
    sh.S.stage = 1;
  }
  __syncthreads();
  place_stage(R, v, 1, sh.S.dt_step);
}

__global__ void k_flow_init(FlArgs a, const double* __restrict__ s0, const double* __restrict__ mats,
                            const double* __restrict__ dt0) {
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const FlView v = fl_view(R.rec, R.ld);
  for (int e = threadIdx.x; e < 12 * R.ld; e += blockDim.x) v.s[e] = 0.0;
  __syncthreads();
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    const double x = s0[R.soff + e];
    v.s[e] = x;
    v.ps[e] = x;
  }
  if (threadIdx.x == 0) {
    FlState S = {};
    S.status = CCO_STATUS_RUNNING;
    S.stage = 0;
    const double first = dt0 ? dt0[R.idx] : a.dt_init;
    S.dt = fmin(first, a.dt_max);
    for (int q = 0; q < 9; ++q) {
      S.B[q] = mats[(size_t)R.idx * 27 + q];
      S.BinvT[q] = mats[(size_t)R.idx * 27 + 9 + q];
      S.Minv[q] = mats[(size_t)R.idx * 27 + 18 + q];
    }
    S.t0 = gtimer();
    *v.st = S;
    if (a.traj_count) a.traj_count[R.idx] = 0;
  }
}

__global__ void __launch_bounds__(kUpdThreads) k_flow_update(FlArgs a) {
  __shared__ FlShared sh;
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const FlView v = fl_view(R.rec, R.ld);
  if (threadIdx.x == 0) sh.S = *v.st;
  __syncthreads();
  if (sh.S.status != CCO_STATUS_RUNNING) return;
  FlState& S = sh.S;
  const int stage = S.stage;
  const size_t ld = R.ld;
  if (stage == 0) {
    // the evaluation at s0: stage-1 velocity, energy, first status
    int zero = 0;
    const double gn = stage_velocity(a, R, S, v.pg, v.k, sh.red, &zero);
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) v.g[e] = v.pg[e];
    if (threadIdx.x == 0) {
      S.f = *v.pf;
      S.gnorm = gn;
      stage_rate(a, gn, S.rate[0]);
      S.n_evals = 1;
      S.count = 0;
      S.status = flow_status(a, S.f, zero, gn, 0.0, S.dt, 0, 0);
      if (S.status != CCO_STATUS_RUNNING) S.t1 = gtimer();
    }
    __syncthreads();
    flow_record(a, R, S, v.s);
    if (S.status == CCO_STATUS_RUNNING) begin_step(a, R, v, sh);
  } else if (stage < 6) {
    // stage velocity k_{stage+1} at the probe, then the next probe
    int zero = 0;
    const double gn = stage_velocity(a, R, S, v.pg, v.k + stage * ld, sh.red, &zero);
    if (threadIdx.x == 0) stage_rate(a, gn, S.rate[stage]);
    if (stage < 5) {
      place_stage(R, v, stage + 1, S.dt_step);
      if (threadIdx.x == 0) S.stage = stage + 1;
    } else {
      // 5th-order solution s_new = s + dt sum b5_j k_j (j = 1..6) is the last probe
      const double dt = S.dt_step;
      for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
        double incr = 0.0;
        for (int j = 0; j < 6; ++j) incr += kB5[j] * v.k[(size_t)j * ld + e];
        const double x = v.s[e] + dt * incr;
        v.sn[e] = x;
        v.ps[e] = x;
      }
      if (threadIdx.x == 0) S.stage = 6;
    }
  } else {
    // stage 7 (FSAL) at s_new: error estimate, accept or reject, controller
    int zero = 0;
    const double gn7 = stage_velocity(a, R, S, v.pg, v.k + 6 * ld, sh.red, &zero);
    const double dt = S.dt_step;
    const int d = R.nd / R.n;
    double e2 = 0.0, m2 = 0.0;
    for (int j = threadIdx.x; j < R.n; j += blockDim.x) {
      double es[3] = {0.0, 0.0, 0.0}, ms[3] = {0.0, 0.0, 0.0};
      for (int b = 0; b < d; ++b) {
        const size_t e = (size_t)j * d + b;
        double acc = 0.0;
        for (int q = 0; q < 7; ++q) acc += (kB5[q] - kB4[q]) * v.k[(size_t)q * ld + e];
        es[b] = dt * acc;
        ms[b] = v.sn[e] - v.s[e];
      }
      for (int c = 0; c < d; ++c) {
        double ec = 0.0, mc = 0.0;
        for (int b = 0; b < d; ++b) {
          ec += es[b] * S.B[b * 3 + c];
          mc += ms[b] * S.B[b * 3 + c];
        }
        e2 += ec * ec;
        m2 += mc * mc;
      }
    }
    e2 = block_sum(e2, sh.red);
    m2 = block_sum(m2, sh.red);
    __shared__ int accept_s;
    if (threadIdx.x == 0) {
      double rate7[2];
      stage_rate(a, gn7, rate7);
      const double cnt = (double)R.nd;
      const double move = sqrt(m2 / cnt);
      double err = sqrt(e2 / cnt) / (a.atol + a.rtol * move);
      double tl[2], etl[2];
      for (int c = 0; c < 2; ++c) {
        double sb = 0.0, se = 0.0;
        for (int q = 0; q < 6; ++q) sb += kB5[q] * S.rate[q][c];
        for (int q = 0; q < 6; ++q) se += (kB5[q] - kB4[q]) * S.rate[q][c];
        se += (kB5[6] - kB4[6]) * rate7[c];
        tl[c] = dt * sb;
        etl[c] = dt * se;
        err = fmax(err, fabs(etl[c]) / (a.atol + a.rtol * fabs(tl[c])));
      }
      const bool accept = err <= 1.0;
      double factor = fmin(fmax(kSafety * pow(err, -1.0 / 5.0), kShrinkMin), kGrowMax);
      if (!isfinite(factor)) factor = kShrinkMin;
      const double dt_next = fmin(dt * factor, a.dt_max);
      if (accept) {
        S.f = *v.pf;
        S.gnorm = gn7;
        S.t += tl[0];
        S.length += tl[1];
        S.var += dt;
        S.rate[0][0] = rate7[0];
        S.rate[0][1] = rate7[1];
        S.n_steps += 1;
      }
      S.n_tries += 1;
      S.n_evals += 6;
      S.dt = dt_next;
      accept_s = accept;
    }
    __syncthreads();
    const bool accept = accept_s;
    if (accept) {
      // s = s_new, g = g_new, k1 = k7 (FSAL)
      for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
        v.s[e] = v.sn[e];
        v.g[e] = v.pg[e];
        v.k[e] = v.k[6 * ld + e];
      }
    }
    // the status uses the current (accepted or kept) gradient
    int nz = 0;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) nz |= v.g[e] != 0.0;
    nz = __syncthreads_or(nz);
    if (threadIdx.x == 0) {
      S.status = flow_status(a, S.f, !nz, S.gnorm, S.t, S.dt, S.n_steps, S.n_tries);
      if (S.status != CCO_STATUS_RUNNING) S.t1 = gtimer();
    }
    __syncthreads();
    const int64_t every = a.rec_every > 0 ? a.rec_every : 1;
    if (accept && a.rec_every > 0 && (S.n_steps % every) == 0) flow_record(a, R, S, v.s);
    if (S.status == CCO_STATUS_RUNNING) begin_step(a, R, v, sh);
  }
  __syncthreads();
  if (threadIdx.x == 0) *v.st = sh.S;
}

// Final state; the trajectory gets the final state appended (overwriting the
// last row when full), as flow.py:_finish.
__global__ void k_flow_finalize(FlArgs a, double* s_out, double* e_out, double* t_out,
                                double* len_out, double* dt_out, int64_t* steps_out,
                                int64_t* evals_out, int64_t* status_out) {
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const FlView v = fl_view(R.rec, R.ld);
  const FlState S = *v.st;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) s_out[R.soff + e] = v.s[e];
  __shared__ int64_t row;
  if (threadIdx.x == 0) {
    e_out[R.idx] = S.f;
    t_out[R.idx] = S.t;
    len_out[R.idx] = S.length;
    dt_out[R.idx] = S.dt;
    steps_out[R.idx] = S.n_steps;
    evals_out[R.idx] = S.n_evals;
    status_out[R.idx] = S.status;
    row = -1;
    if (a.traj_count) {
      const int64_t last = S.count - 1;
      const size_t o = (size_t)R.idx * a.rec_cap;
      const bool last_is_final =
          last >= 0 && a.traj_len[o + last] == S.length && a.traj_t[o + last] == S.t;
      const int64_t idx = last_is_final ? last : min(S.count, a.rec_cap - 1);
      a.traj_t[o + idx] = S.t;
      a.traj_len[o + idx] = S.length;
      a.traj_e[o + idx] = S.f;
      a.traj_count[R.idx] = idx + 1;
      row = idx;
    }
  }
  __syncthreads();
  if (row >= 0) {
    double* out = a.traj_s + R.toff + (size_t)row * R.nd;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) out[e] = v.s[e];
  }
}

}  // namespace

cudaError_t flow_init(const FlArgs& a, const double* s0, const double* mats, const double* dt0,
                      cudaStream_t st) {
  k_flow_init<<<a.B, kUpdThreads, 0, st>>>(a, s0, mats, dt0);
  return cudaGetLastError();
}

cudaError_t flow_update(const FlArgs& a, cudaStream_t st) {
  k_flow_update<<<a.B, kUpdThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t flow_finalize(const FlArgs& a, double* s_out, double* e_out, double* t_out,
                          double* len_out, double* dt_out, int64_t* steps_out,
                          int64_t* evals_out, int64_t* status_out, cudaStream_t st) {
  k_flow_finalize<<<a.B, kUpdThreads, 0, st>>>(a, s_out, e_out, t_out, len_out, dt_out,
                                               steps_out, evals_out, status_out);
  return cudaGetLastError();
}

}  // namespace cco
