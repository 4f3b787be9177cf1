// Gradient flow lanes (device side): adaptive Dormand-Prince 5(4) as a
// per-lane stage machine. See cco_flow.cu.
#pragma once

#include "cco_opt.cuh"

namespace cco {

// Flow record: [0, kFlHead) FlState, the lane's basis B, B^-T and (B B^T)^-1
// (row-major 3x3 slots) and the probe energy pf at [kFlHead - 1]; then
// s, g (accepted point and its gradient), k1..k7 (stage velocities), s_new,
// ps, pg (probe positions and gradient), ld each; then the evaluation scratch.
struct FlState {
  int64_t status, n_steps, n_tries, n_evals, count;
  int64_t t0, t1;                  // %globaltimer at start / completion
  double t, length, var, dt, dt_step, f, gnorm, f_new;
  double rate[7][2];               // per stage: d(t, length)/d(variable)
  double B[9], BinvT[9], Minv[9];  // basis, its inverse transpose, (B B^T)^-1
  int32_t stage, pad_;
};
constexpr int kFlHead = 72;
static_assert(sizeof(FlState) <= (kFlHead - 1) * sizeof(double), "FlState outgrew its slot");

struct FlView {
  FlState* st;
  double *pf, *s, *g, *k, *sn, *ps, *pg;   // k: 7 stage vectors, ld apart
  double2* dens;
};

__host__ __device__ __forceinline__ FlView fl_view(double* rec, int ld) {
  FlView v;
  v.st = reinterpret_cast<FlState*>(rec);
  v.pf = rec + kFlHead - 1;
  v.s = rec + kFlHead;
  v.g = v.s + ld;
  v.k = v.s + 2 * (size_t)ld;
  v.sn = v.s + 9 * (size_t)ld;
  v.ps = v.s + 10 * (size_t)ld;
  v.pg = v.s + 11 * (size_t)ld;
  v.dens = reinterpret_cast<double2*>(v.s + 12 * (size_t)ld);
  return v;
}

__host__ __device__ __forceinline__ size_t fl_record_doubles(int ld, int M, int nt1) {
  return kFlHead + 12 * (size_t)ld + 2 * (size_t)M * (2 + nt1);
}

struct FlArgs {
  int B;
  const LaneRef* lanes;
  double rtol, atol, dt_init, dt_min, dt_max, t_max, energy_tol, grad_tol;
  int64_t max_steps;
  int arclength;                 // 1: unit Cartesian speed, 0: physical time
  int d_unused;
  int64_t rec_every, rec_cap;
  // trajectory (null when off): rows by LaneRef::idx, traj_s by toff
  double *traj_s, *traj_t, *traj_len, *traj_e;
  int64_t* traj_count;
};

// bases: [B][3][3] host-uploaded per lane (B, B^-T, (B B^T)^-1 in that order:
// 27 doubles per lane); dt0: [B] first step per lane, or null for dt_init.
cudaError_t flow_init(const FlArgs& a, const double* s0, const double* mats, const double* dt0,
                      cudaStream_t st);
cudaError_t flow_update(const FlArgs& a, cudaStream_t st);
cudaError_t flow_finalize(const FlArgs& a, double* s_out, double* e_out, double* t_out,
                          double* len_out, double* dt_out, int64_t* steps_out,
                          int64_t* evals_out, int64_t* status_out, cudaStream_t st);

}  // namespace cco
