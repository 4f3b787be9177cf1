// Device bodies of the descent minimizer shared by the launched update kernel
// (cco_opt.cu) and the persistent small-lane kernel (cco_persist.cu): the
// %globaltimer clock, the [0, 1) wrap, the status and recording rules and
// one iteration of a lane.
#pragma once

#include <cmath>

#include "cco_opt.cuh"

namespace cco {

namespace {

__device__ __forceinline__ int64_t gtimer() {
  uint64_t v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  return (int64_t)v;
}

__device__ __forceinline__ double wrap01(double v) {
  const double w = v - floor(v);
  const double below_one = 0x1.fffffffffffffp-1;
  return w < below_one ? w : below_one;
}

// ============================================================ descent

__device__ int descent_status(double f, bool nonzero, double step, int64_t it,
                              const DescentArgs& a) {
  int code = it >= a.max_iters ? CCO_STATUS_BUDGET : CCO_STATUS_RUNNING;
  if (step <= a.step_min) code = CCO_STATUS_STEP_FLOOR;
  if (!nonzero) code = CCO_STATUS_GRAD_TOL;
  if (f < a.energy_tol) code = CCO_STATUS_ENERGY_TOL;
  return code;
}

__device__ void descent_record(const DescentArgs& a, int lane, const LaneRef& R, int64_t it,
                               const double* s, double f, double step) {
  if (a.traj_count == nullptr) return;
  __shared__ int64_t row;
  if (threadIdx.x == 0) {
    const int64_t c = a.traj_count[R.idx];
    row = ((it % a.rec_every) == 0 && c < a.rec_cap) ? c : -1;
    if (row >= 0) {
      a.traj_e[R.idx * a.rec_cap + row] = f;
      a.traj_step[R.idx * a.rec_cap + row] = step;
      a.traj_it[R.idx * a.rec_cap + row] = it;
      a.traj_count[R.idx] = c + 1;
    }
  }
  __syncthreads();
  if (row >= 0) {
    double* o = a.traj_s + R.toff + (size_t)row * R.nd;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) o[e] = wrap01(s[e]);
  }
}

// Gradient norm and the exact all-zero test of the accepted gradient.
__device__ void descent_norm(const LaneRef& R, const DsView& v, double* red) {
  double ss = 0.0;
  int nz = 0;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    const double x = v.g[e];
    ss += x * x;
    nz |= (x != 0.0);
  }
  ss = block_sum(ss, red);
  nz = __syncthreads_or(nz);
  if (threadIdx.x == 0) {
    v.st->norm = sqrt(ss);
    v.st->nonzero = nz;
  }
}

// One descent iteration of lane `lane` (the whole CTA): the update kernel's
// body, also run by the persistent small-lane kernel (cco_persist.cu).
__device__ void descent_update_lane(const DescentArgs& a, int lane) {
  __shared__ double red[32];
  __shared__ int s_reject, s_status;
  const LaneRef R = a.lanes[lane];
  const DsView v = ds_view(R.rec, R.ld);
  DsState* S = v.st;
  if (S->status != CCO_STATUS_RUNNING) return;
  const int nd = R.nd;
  if (S->phase == PH_INIT) {
    // init_one (descent.py:121-141): one evaluation at s0, no iteration
    for (int e = threadIdx.x; e < nd; e += blockDim.x) v.g[e] = v.pg[e];
    descent_norm(R, v, red);
    __syncthreads();
    if (threadIdx.x == 0) {
      S->f = *v.pf;
      S->phase = PH_ITER;
      s_status = descent_status(S->f, S->nonzero != 0, S->step, 0, a);
      S->status = s_status;
      if (s_status != CCO_STATUS_RUNNING) S->t1 = gtimer();
    }
    __syncthreads();
    descent_record(a, lane, R, 0, v.s, S->f, S->step);
  } else {
    // step_fn (descent.py:153-175) with the probe evaluated at xn
    if (threadIdx.x == 0) {
      const double f = S->f, f2 = *v.pf;
      const double step = S->step, norm = S->norm;
      const double df = f - f2;
      const double df2 = step * norm;
      const bool reject = fabs(df - df2) / df2 > a.rel_tol;  // NaN accepts
      S->step = reject ? step * a.shrink : step * a.grow;
      if (!reject) S->f = f2;
      S->it += 1;
      S->n_evals += 2;
      s_reject = reject;
    }
    __syncthreads();
    if (!s_reject) {
      for (int e = threadIdx.x; e < nd; e += blockDim.x) {
        v.s[e] = v.ps[e];
        v.g[e] = v.pg[e];
      }
      descent_norm(R, v, red);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      s_status = descent_status(S->f, S->nonzero != 0, S->step, S->it, a);
      S->status = s_status;
      if (s_status != CCO_STATUS_RUNNING) S->t1 = gtimer();
    }
    __syncthreads();
    descent_record(a, lane, R, S->it, v.s, S->f, S->step);
  }
  __syncthreads();
  if (s_status == CCO_STATUS_RUNNING) {
    // next probe: xn = s - (g / |g|) * step  (0 * g when |g| = 0)
    const double norm = S->norm, step = S->step;
    for (int e = threadIdx.x; e < nd; e += blockDim.x) {
      const double gn = norm > 0.0 ? __ddiv_rn(v.g[e], norm) : 0.0 * v.g[e];
      v.ps[e] = __dsub_rn(v.s[e], __dmul_rn(gn, step));
    }
  }
}

}  // namespace

}  // namespace cco
