// Molecular-dynamics lanes (device side): velocity Verlet with optional
// Andersen resets, and Langevin BAOAB, one force evaluation per tick.
// See cco_md.cu.
#pragma once

#include "cco_opt.cuh"

namespace cco {

// MD record: [0, kMdHead) MdState (with the basis matrices) and the probe
// energy pf at [kMdHead - 1]; then r, v, f (Cartesian), ps (fractional probe
// r B^-1) and pg (its gradient), ld each; then, for segment runs with w
// tracked waves, the wave section (rho_prev 2w, winding |.| w, winding net w,
// valid steps w, sum of S w, fresh densities 2w); then the evaluation scratch.
struct MdState {
  int64_t status, step, n_resets;
  int64_t t0, t1;
  double phi, ke, e0, max_drift, acc;
  double B[9], Binv[9], BinvT[9];
  uint32_t key[2];
  int32_t phase, pad_;
  int64_t step_end;            // the lane stops when step reaches it
  int64_t n_sum, snap_count, trace_count;
  double temperature, time;    // segment runs: per-lane T, elapsed time
  double sum_kinetic, sum_phi, sum_phi2;
  double drift_limit;          // |E - e0| bound (< 0: no guard)
  // observables of the step just finished, for k_md_observe (segment runs)
  double obs_rcm[3];           // centre of mass at that step
  int32_t obs_pending;         // 1: k_md_observe has this step's waves to do
  int32_t obs_wind;            // the step was a wind step (unconstrained waves fresh)
  int32_t obs_snap, obs_trace; // snapshot slot and trace row (-1: none)
};
constexpr int kMdHead = 64;
static_assert(sizeof(MdState) <= (kMdHead - 1) * sizeof(double), "MdState outgrew its slot");

struct MdView {
  MdState* st;
  double *pf, *r, *v, *f, *ps, *pg;
  double *rho_prev, *wind_abs, *wind_net, *n_valid, *sum_s, *fresh;
  double2* dens;
};

__host__ __device__ __forceinline__ MdView md_view(double* rec, int ld, int w = 0) {
  MdView v;
  v.st = reinterpret_cast<MdState*>(rec);
  v.pf = rec + kMdHead - 1;
  v.r = rec + kMdHead;
  v.v = v.r + ld;
  v.f = v.r + 2 * (size_t)ld;
  v.ps = v.r + 3 * (size_t)ld;
  v.pg = v.r + 4 * (size_t)ld;
  v.rho_prev = v.r + 5 * (size_t)ld;
  v.wind_abs = v.rho_prev + 2 * (size_t)w;
  v.wind_net = v.wind_abs + w;
  v.n_valid = v.wind_net + w;
  v.sum_s = v.n_valid + w;
  v.fresh = v.sum_s + w;
  v.dens = reinterpret_cast<double2*>(v.fresh + 2 * (size_t)w);
  return v;
}

__host__ __device__ __forceinline__ size_t md_wave_doubles(int w) { return 8 * (size_t)w; }

__host__ __device__ __forceinline__ size_t md_record_doubles(int ld, int M, int nt1, int w = 0) {
  return kMdHead + 5 * (size_t)ld + md_wave_doubles(w) + 2 * (size_t)M * (2 + nt1);
}

enum : int { MD_VERLET = 0, MD_BAOAB = 1 };
enum : int { ANDERSEN_OFF = 0, ANDERSEN_COUNT = 1, ANDERSEN_BERNOULLI = 2 };

// Device arrays of a segment run's batched state ([batch] first everywhere;
// w waves, n particles, d axes, R snapshot slots, Q trace rows).
struct MdSegIO {
  double *r, *v, *f, *phi, *temperature, *time, *reset_acc;
  uint32_t* keys;                        // [B][2]
  int64_t *step, *status, *n_valid, *n_sum;
  double *rho_prev, *wind_abs, *wind_net, *sum_s;   // [B][w][2], [B][w] ...
  double *e0, *max_drift, *sum_kinetic, *sum_phi, *sum_phi2;
  int64_t *snap_step, *snap_count;       // [B][R], [B]
  double *snap_time, *snap_wind_abs, *snap_wind_net, *snap_rho, *snap_r, *snap_phi,
      *snap_kinetic;                     // [B][R], [B][R][w], ..., [B][R][w][2], [B][R][n][d]
  double *trace_rho, *trace_time;        // [B][Q][w][2], [B][Q]
  int64_t* trace_count;                  // [B]
};

struct MdArgs {
  int B;
  const LaneRef* lanes;
  double dt, gamma, temperature, andersen_p, drift_tol;
  int64_t n_steps;
  int scheme, andersen;
  // segment runs (w > 0): tracked waves and observables
  int w = 0, nc = 0, wind_every = 1, corrected = 0;
  double drift_coef = -1.0;              // drift bound = coef * T (< 0: none)
  double phase_floor = 0.0;
  const double* wave_n = nullptr;        // [w][d] reciprocal-basis coefficients
  const double* wave_k = nullptr;        // [w][d] Cartesian wavevectors
  const int* cpos = nullptr;             // [nc] run position of constrained wave c
  int n_rec = 0, trace_every = 0, trace_cap = 0;
  const int64_t* rec_steps = nullptr;    // [n_rec] ascending
  MdSegIO io{};
};

// mats: [B][27] host-uploaded B, B^-1, B^-T per lane; keys: [B][2];
// acc0: [B] Andersen accumulators (count mode).
cudaError_t md_init(const MdArgs& a, const double* r0, const double* v0, const double* mats,
                    const uint32_t* keys, const double* acc0, cudaStream_t st);
cudaError_t md_update(const MdArgs& a, cudaStream_t st);
cudaError_t md_finalize(const MdArgs& a, double* r_out, double* v_out, double* f_out,
                        double* phi_out, double* ke_out, double* drift_out, int64_t* resets_out,
                        double* acc_out, uint32_t* keys_out, int64_t* status_out,
                        cudaStream_t st);
// Segment runs: lanes start from (and end in) the batched state a.io.
cudaError_t md_seg_init(const MdArgs& a, const double* mats, cudaStream_t st);
cudaError_t md_seg_finalize(const MdArgs& a, cudaStream_t st);

}  // namespace cco
