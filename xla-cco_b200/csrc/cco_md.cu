// Molecular-dynamics steps on sm_100a (FP64): velocity Verlet with Andersen
// resets and Langevin BAOAB, mass 1, Cartesian positions r = s B.
//
// Reference: verlet_step, andersen_reset, baoab_step
// (src/xla_cco/dynamics/integrators.py:83-176) with the force
// F = -dPhi/ds B^-T of value_grad_density(r B^-1) (dynamics/run.py:219-244).
// Each lane advances one step per tick: the tick's evaluation is the force at
// the drifted positions, k_md_update finishes the step (last half kick,
// Andersen reset, energy bookkeeping) and starts the next (first half kick
// and drift, with the BAOAB thermostat between the two half drifts).
//
// Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
// numbers: as easy as 1, 2, 3", SC11). A lane holds a key K_s during step s;
// every draw of the step is Philox(K_s, (0, 0, stream, index)) and a step that
// drew ends with K_{s+1} = Philox(K_s, (0, 0, NEXT, 0)).xy - the device run equals
// the host step functions chained with the keys they return, and nothing
// depends on launch shapes. Normals by Box-Muller on two 53-bit uniforms.
// JAX's threefry streams are not reproduced: the reference's draws differ,
// their distributions do not.
//
// Segment runs (the reference's simulate, dynamics/run.py:398-540) add the
// per-step observables of w tracked waves: the constrained waves' densities
// are the force evaluation's own (rho in run order, cpos maps them), the
// others are summed fresh by k_md_waves on wind steps; both are multiplied
// by exp(-i k . R_cm) unless the scheme is plain Verlet; then the winding
// update, running sums, the drift guard (plain Verlet), snapshots at the
// recorded steps and the dense rho trace (_step, _record, winding_update in
// dynamics/run.py and dynamics/observables.py:98-125).
#include <cmath>

#include "cco_md.cuh"

namespace cco {

namespace {

__device__ __forceinline__ int64_t gtimer() {
  uint64_t v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  return (int64_t)v;
}

// Philox4x32 with 10 rounds (Random123 constants).
__device__ __forceinline__ uint4 philox(uint2 key, uint4 c) {
  constexpr uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  constexpr uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    c = make_uint4(hi1 ^ c.y ^ key.x, lo1, hi0 ^ c.w ^ key.y, lo0);
    key.x += W0;
    key.y += W1;
  }
  return c;
}

enum : uint32_t { RNG_NOISE = 1, RNG_COIN = 3, RNG_PICK = 4, RNG_ROW = 5, RNG_NEXT = 7 };

__device__ __forceinline__ uint4 draw(const MdState& S, uint32_t stream, uint32_t index) {
  return philox(make_uint2(S.key[0], S.key[1]), make_uint4(0u, 0u, stream, index));
}

// 53-bit uniform in [0, 1) from two words
__device__ __forceinline__ double u53(uint32_t a, uint32_t b) {
  return (double)(((uint64_t)(a >> 5) << 26) | (b >> 6)) * 0x1p-53;
}

__device__ __forceinline__ double normal(uint4 w) {
  const double u1 = 1.0 - u53(w.x, w.y);  // (0, 1]
  const double u2 = u53(w.z, w.w);
  return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

// positions -> fractional probe s = r B^-1 for every particle
__device__ void to_fractional(const LaneRef& R, const MdView& w, const MdState& S, int d) {
  for (int j = threadIdx.x; j < R.n; j += blockDim.x)
    for (int c = 0; c < d; ++c) {
      double acc = 0.0;
      for (int b = 0; b < d; ++b) acc += w.r[(size_t)j * d + b] * S.Binv[b * 3 + c];
      w.ps[(size_t)j * d + c] = acc;
    }
}

// F = -g B^-T from the probe gradient
__device__ void forces(const LaneRef& R, const MdView& w, const MdState& S, int d) {
  for (int j = threadIdx.x; j < R.n; j += blockDim.x) {
    double g[3] = {0.0, 0.0, 0.0};
    for (int b = 0; b < d; ++b) g[b] = w.pg[(size_t)j * d + b];
    for (int c = 0; c < d; ++c) {
      double acc = 0.0;
      for (int b = 0; b < d; ++b) acc += g[b] * S.BinvT[b * 3 + c];
      w.f[(size_t)j * d + c] = -acc;
    }
  }
}

__device__ double kinetic(const LaneRef& R, const MdView& w, double* red) {
  double s = 0.0;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) s += w.v[e] * w.v[e];
  return 0.5 * block_sum(s, red);
}

// First half of step `next`: B (half kick) and the drift; BAOAB splits the
// drift around the O (Ornstein-Uhlenbeck) update.
__device__ void begin_step(const MdArgs& a, const LaneRef& R, const MdView& w, const MdState& S,
                           int d, double c, double noise) {
  const double half = 0.5 * a.dt;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    double v = w.v[e] + half * w.f[e];
    double r = w.r[e];
    if (a.scheme == MD_BAOAB) {
      r = r + half * v;
      const double xi = normal(draw(S, RNG_NOISE, (uint32_t)e));
      v = c * v + noise * xi;
      r = r + half * v;
    } else {
      r = r + a.dt * v;
    }
    w.v[e] = v;
    w.r[e] = r;
  }
  __syncthreads();
  to_fractional(R, w, S, d);
}

__global__ void k_md_init(MdArgs a, const double* __restrict__ r0, const double* __restrict__ v0,
                          const double* __restrict__ mats, const uint32_t* __restrict__ keys,
                          const double* __restrict__ acc0) {
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const MdView w = md_view(R.rec, R.ld, a.w);
  for (int e = threadIdx.x; e < 5 * R.ld; e += blockDim.x) w.r[e] = 0.0;
  __shared__ MdState S;
  if (threadIdx.x == 0) {
    MdState x = {};
    x.status = CCO_STATUS_RUNNING;
    for (int q = 0; q < 9; ++q) {
      x.B[q] = mats[(size_t)R.idx * 27 + q];
      x.Binv[q] = mats[(size_t)R.idx * 27 + 9 + q];
      x.BinvT[q] = mats[(size_t)R.idx * 27 + 18 + q];
    }
    x.key[0] = keys[2 * R.idx];
    x.key[1] = keys[2 * R.idx + 1];
    x.acc = acc0 ? acc0[R.idx] : 0.0;
    x.step_end = a.n_steps;
    x.temperature = a.temperature;
    x.drift_limit = a.drift_tol > 0.0 ? a.drift_tol : -1.0;
    x.e0 = NAN;
    x.t0 = gtimer();
    S = x;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    w.r[e] = r0[R.soff + e];
    w.v[e] = v0[R.soff + e];
  }
  __syncthreads();
  to_fractional(R, w, S, R.nd / R.n);
  if (threadIdx.x == 0) *w.st = S;
}

// NaN-propagating maximum (jnp.maximum).
__device__ __forceinline__ double max_nan(double a, double b) {
  return (a != a || b != b) ? NAN : fmax(a, b);
}

// Mean Cartesian position (unwrapped r, mass 1) into rcm[0..d).
__device__ void center_of_mass(const LaneRef& R, const MdView& w, int d, double* rcm,
                               double* red) {
  for (int c = 0; c < d; ++c) {
    double s = 0.0;
    for (int j = threadIdx.x; j < R.n; j += blockDim.x) s += w.r[(size_t)j * d + c];
    s = block_sum(s, red);
    if (threadIdx.x == 0) rcm[c] = s / R.n;
    __syncthreads();
  }
}

// Density of wave c as the observables see it: the force pass's rho for a
// constrained wave, the fresh sum otherwise; times exp(-i k . R_cm) when
// the scheme corrects the centre of mass.
__device__ __forceinline__ double2 wave_rho(const MdArgs& a, const MdView& w, int c, int d,
                                            const double* rcm) {
  double2 r;
  if (c < a.nc) r = w.dens[a.cpos[c]];
  else r = make_double2(w.fresh[2 * c], w.fresh[2 * c + 1]);
  if (a.corrected) {
    double ph = 0.0;
    for (int q = 0; q < d; ++q) ph += a.wave_k[(size_t)c * d + q] * rcm[q];
    double sn, cs;
    sincos(ph, &sn, &cs);
    r = make_double2(r.x * cs + r.y * sn, r.y * cs - r.x * sn);
  }
  return r;
}

// Index of `step` among the ascending recorded steps, or -1.
__device__ __forceinline__ int record_slot(const MdArgs& a, int64_t step) {
  int lo = 0, hi = a.n_rec - 1;
  while (lo <= hi) {
    const int mid = (lo + hi) >> 1;
    const int64_t v = a.rec_steps[mid];
    if (v == step) return mid;
    if (v < step) lo = mid + 1;
    else hi = mid - 1;
  }
  return -1;
}

// Observables after a finished step of a segment run (S holds the new step,
// time, phi, ke; running sums and counters are advanced here).
__device__ void observe_step(const MdArgs& a, const LaneRef& R, const MdView& w, MdState& S,
                             int d, double* red) {
  __shared__ double rcm[3];
  if (a.corrected) center_of_mass(R, w, d, rcm, red);
  const size_t lane = (size_t)R.idx;
  if (threadIdx.x == 0) {
    const int js = a.n_rec > 0 ? record_slot(a, S.step) : -1;
    const int jt = (a.trace_every > 0 && a.trace_cap > 0 && S.step % a.trace_every == 0 &&
                    S.trace_count < a.trace_cap) ? (int)S.trace_count : -1;
    for (int q = 0; q < 3; ++q) S.obs_rcm[q] = a.corrected && q < d ? rcm[q] : 0.0;
    S.obs_pending = 1;
    S.obs_wind = S.step % a.wind_every == 0 ? 1 : 0;
    S.obs_snap = js;
    S.obs_trace = jt;
    if (js >= 0) {
      const size_t o = lane * a.n_rec + js;
      a.io.snap_step[o] = S.step;
      a.io.snap_time[o] = S.time;
      a.io.snap_phi[o] = S.phi;
      a.io.snap_kinetic[o] = S.ke;
      S.snap_count += 1;
    }
    if (jt >= 0) {
      a.io.trace_time[lane * a.trace_cap + jt] = S.time;
      S.trace_count += 1;
    }
  }
  __syncthreads();
  // the positions of a snapshot, before the next step's drift moves them
  if (S.obs_snap >= 0)
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x)
      a.io.snap_r[(lane * a.n_rec + S.obs_snap) * R.nd + e] = w.r[e];
}

// Rows of rho_prev marked pending (NaN) get the current densities (the first
// tick of a segment run evaluated the force at the current positions).
__device__ void repair_pending(const MdArgs& a, const LaneRef& R, const MdView& w, int d,
                               double* red) {
  __shared__ double rcm[3];
  if (a.corrected) center_of_mass(R, w, d, rcm, red);
  for (int c = threadIdx.x; c < a.w; c += blockDim.x)
    if (w.rho_prev[2 * c] != w.rho_prev[2 * c]) {
      const double2 r = wave_rho(a, w, c, d, rcm);
      w.rho_prev[2 * c] = r.x;
      w.rho_prev[2 * c + 1] = r.y;
    }
}

__global__ void __launch_bounds__(kUpdThreads) k_md_update(MdArgs a, double c, double noise_var) {
  __shared__ MdState S;
  __shared__ double red[32];
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const MdView w = md_view(R.rec, R.ld, a.w);
  if (threadIdx.x == 0) {
    S = *w.st;
    S.obs_pending = 0;   // the previous step's waves were observed by the last tick
  }
  __syncthreads();
  if (S.status != CCO_STATUS_RUNNING) {
    if (threadIdx.x == 0 && w.st->obs_pending) w.st->obs_pending = 0;
    return;
  }
  const int d = R.nd / R.n;
  forces(R, w, S, d);
  __syncthreads();
  if (S.phase == 0) {
    // forces at the start: energy reference for the drift (kept when the
    // segment already has one), pending densities of a segment run
    const double ke = kinetic(R, w, red);
    if (a.w > 0) repair_pending(a, R, w, d, red);
    if (threadIdx.x == 0) {
      S.phi = *w.pf;
      S.ke = ke;
      if (a.w == 0 || S.e0 != S.e0) S.e0 = S.phi + ke;
      if (a.w == 0) S.max_drift = 0.0;
      S.phase = 1;
      if (S.step >= S.step_end) {
        S.status = CCO_STATUS_BUDGET;
        S.t1 = gtimer();
      }
    }
  } else {
    // finish the step: last half kick, then Andersen (Verlet only)
    const double half = 0.5 * a.dt;
    for (int e = threadIdx.x; e < R.nd; e += blockDim.x) w.v[e] = w.v[e] + half * w.f[e];
    __shared__ int fire, pick;
    if (threadIdx.x == 0) {
      S.step += 1;
      S.time += a.dt;
      fire = 0;
      pick = 0;
      if (a.scheme == MD_VERLET && a.andersen != ANDERSEN_OFF) {
        if (a.andersen == ANDERSEN_COUNT) {
          const double acc = S.acc + a.andersen_p;
          fire = acc >= 1.0;
          S.acc = fire ? acc - 1.0 : acc;
        } else {
          const uint4 u = draw(S, RNG_COIN, 0);
          fire = u53(u.x, u.y) < a.andersen_p;
        }
        const uint4 q = draw(S, RNG_PICK, 0);
        pick = min((int)(u53(q.x, q.y) * R.n), R.n - 1);
        S.n_resets += fire;
      }
    }
    __syncthreads();
    if (fire && threadIdx.x < d)
      w.v[(size_t)pick * d + threadIdx.x] =
          sqrt(S.temperature) * normal(draw(S, RNG_ROW, threadIdx.x));
    __syncthreads();
    const double ke = kinetic(R, w, red);
    if (threadIdx.x == 0) {
      if (a.scheme == MD_BAOAB || a.andersen != ANDERSEN_OFF) {
        // a step that drew numbers hands on the next key (plain Verlet draws none)
        const uint4 k = draw(S, RNG_NEXT, 0);
        S.key[0] = k.x;
        S.key[1] = k.y;
      }
      S.phi = *w.pf;
      S.ke = ke;
      const double drift = fabs(S.phi + ke - S.e0);
      S.max_drift = max_nan(S.max_drift, drift);
      if (S.drift_limit >= 0.0 && !(drift <= S.drift_limit)) S.status = CCO_STATUS_DRIFT;
      if (a.w > 0) {
        S.sum_kinetic += ke;
        S.sum_phi += S.phi;
        S.sum_phi2 += S.phi * S.phi;
        S.n_sum += 1;
      }
    }
    __syncthreads();
    if (a.w > 0) observe_step(a, R, w, S, d, red);
    if (threadIdx.x == 0) {
      if (S.status == CCO_STATUS_RUNNING && S.step >= S.step_end) S.status = CCO_STATUS_BUDGET;
      if (S.status != CCO_STATUS_RUNNING) S.t1 = gtimer();
    }
  }
  __syncthreads();
  if (S.status == CCO_STATUS_RUNNING) {
    const double noise = sqrt(noise_var * S.temperature);
    begin_step(a, R, w, S, d, c, noise);
  }
  __syncthreads();
  if (threadIdx.x == 0) *w.st = S;
}

// Per-wave observables of the step k_md_update just finished (segment runs),
// one thread per wave over (lane, wave chunk) blocks: the wave's density
// times exp(-i k . R_cm), the winding increment (atan2 of the phase change),
// running sums, and the snapshot and trace rows. Waves are independent, so
// spreading a lane's waves over blocks changes no result.
__global__ void __launch_bounds__(kUpdThreads) k_md_observe(MdArgs a) {
  const LaneRef R = a.lanes[blockIdx.x];
  const MdView w = md_view(R.rec, R.ld, a.w);
  const MdState* S = w.st;
  if (!S->obs_pending) return;
  const int c = blockIdx.y * blockDim.x + threadIdx.x;
  if (c >= a.w) return;
  const int d = R.nd / R.n;
  const int js = S->obs_snap, jt = S->obs_trace;
  const bool wind = S->obs_wind != 0;
  const size_t lane = (size_t)R.idx;
  const double2 old = make_double2(w.rho_prev[2 * c], w.rho_prev[2 * c + 1]);
  const bool active = c < a.nc || wind;
  double2 nw = old;
  if (active) nw = wave_rho(a, w, c, d, S->obs_rcm);
  const double delta = atan2(nw.y * old.x - nw.x * old.y, nw.x * old.x + nw.y * old.y);
  const double s_old = (old.x * old.x + old.y * old.y) / R.n;
  const double s_new = (nw.x * nw.x + nw.y * nw.y) / R.n;
  const bool ok = active && s_old > a.phase_floor && s_new > a.phase_floor;
  const double2 rp = active ? nw : old;
  w.rho_prev[2 * c] = rp.x;
  w.rho_prev[2 * c + 1] = rp.y;
  if (ok) {
    w.wind_abs[c] += fabs(delta);
    w.wind_net[c] += delta;
    w.n_valid[c] += 1.0;
  }
  w.sum_s[c] += (rp.x * rp.x + rp.y * rp.y) / R.n;
  if (js >= 0) {
    const size_t o = (lane * a.n_rec + js) * a.w + c;
    a.io.snap_wind_abs[o] = w.wind_abs[c];
    a.io.snap_wind_net[o] = w.wind_net[c];
    a.io.snap_rho[2 * o] = rp.x;
    a.io.snap_rho[2 * o + 1] = rp.y;
  }
  if (jt >= 0) {
    const size_t o = (lane * a.trace_cap + jt) * a.w + c;
    a.io.trace_rho[2 * o] = rp.x;
    a.io.trace_rho[2 * o + 1] = rp.y;
  }
}

// Fresh densities of the unconstrained waves at the probe positions (the
// positions the tick's force pass evaluated) on wind steps and on the first
// tick. Grid: (lanes, wave chunks of blockDim.x); particles staged in tiles.
__global__ void __launch_bounds__(kUpdThreads) k_md_waves(MdArgs a) {
  __shared__ double tile[kUpdThreads * 3];
  const LaneRef R = a.lanes[blockIdx.x];
  const MdView w = md_view(R.rec, R.ld, a.w);
  const MdState* S = w.st;
  if (S->status != CCO_STATUS_RUNNING) return;
  if (S->phase != 0 && (S->step + 1) % a.wind_every != 0) return;
  const int d = R.nd / R.n;
  const int u = a.nc + blockIdx.y * blockDim.x + threadIdx.x;
  double nv[3] = {0.0, 0.0, 0.0};
  if (u < a.w)
    for (int q = 0; q < d; ++q) nv[q] = a.wave_n[(size_t)u * d + q];
  double re = 0.0, im = 0.0;
  for (int j0 = 0; j0 < R.n; j0 += blockDim.x) {
    const int nj = min((int)blockDim.x, R.n - j0);
    __syncthreads();
    for (int e = threadIdx.x; e < nj * d; e += blockDim.x) tile[e] = w.ps[(size_t)j0 * d + e];
    __syncthreads();
    if (u < a.w)
      for (int jj = 0; jj < nj; ++jj) {
        double sn, cs;
        if (d == 1) sincos_2pi_dot<1>(nv, tile + jj, &sn, &cs);
        else if (d == 2) sincos_2pi_dot<2>(nv, tile + jj * 2, &sn, &cs);
        else sincos_2pi_dot<3>(nv, tile + jj * 3, &sn, &cs);
        re += cs;
        im += sn;
      }
  }
  if (u < a.w) {
    w.fresh[2 * u] = re;
    w.fresh[2 * u + 1] = im;
  }
}

// Segment runs: each lane's record from the batched state.
__global__ void k_md_seg_init(MdArgs a, const double* __restrict__ mats) {
  const LaneRef R = a.lanes[blockIdx.x];
  const MdView w = md_view(R.rec, R.ld, a.w);
  const MdSegIO& io = a.io;
  const size_t i = (size_t)R.idx;
  __shared__ MdState S;
  if (threadIdx.x == 0) {
    MdState x = {};
    x.status = io.status[i];
    for (int q = 0; q < 9; ++q) {
      x.B[q] = mats[q];
      x.Binv[q] = mats[9 + q];
      x.BinvT[q] = mats[18 + q];
    }
    x.key[0] = io.keys[2 * i];
    x.key[1] = io.keys[2 * i + 1];
    x.acc = io.reset_acc[i];
    x.step = io.step[i];
    x.step_end = x.step + a.n_steps;
    x.time = io.time[i];
    x.temperature = io.temperature[i];
    x.phi = io.phi[i];
    x.e0 = io.e0[i];
    x.max_drift = io.max_drift[i];
    x.sum_kinetic = io.sum_kinetic[i];
    x.sum_phi = io.sum_phi[i];
    x.sum_phi2 = io.sum_phi2[i];
    x.n_sum = io.n_sum[i];
    x.snap_count = io.snap_count[i];
    x.trace_count = io.trace_count[i];
    x.drift_limit = a.drift_coef >= 0.0 ? a.drift_coef * x.temperature : -1.0;
    x.t0 = gtimer();
    S = x;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    w.r[e] = io.r[R.soff + e];
    w.v[e] = io.v[R.soff + e];
    w.f[e] = io.f[R.soff + e];
  }
  for (int c = threadIdx.x; c < a.w; c += blockDim.x) {
    const size_t o = i * a.w + c;
    w.rho_prev[2 * c] = io.rho_prev[2 * o];
    w.rho_prev[2 * c + 1] = io.rho_prev[2 * o + 1];
    w.wind_abs[c] = io.wind_abs[o];
    w.wind_net[c] = io.wind_net[o];
    w.n_valid[c] = (double)io.n_valid[o];
    w.sum_s[c] = io.sum_s[o];
  }
  __syncthreads();
  to_fractional(R, w, S, R.nd / R.n);
  if (threadIdx.x == 0) *w.st = S;
}

// Segment runs: the batched state from each lane's record. A lane that
// finished its steps is STATUS_RUNNING again (only a drift stops a lane).
__global__ void k_md_seg_finalize(MdArgs a) {
  const LaneRef R = a.lanes[blockIdx.x];
  const MdView w = md_view(R.rec, R.ld, a.w);
  const MdSegIO& io = a.io;
  const size_t i = (size_t)R.idx;
  const MdState S = *w.st;
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    io.r[R.soff + e] = w.r[e];
    io.v[R.soff + e] = w.v[e];
    io.f[R.soff + e] = w.f[e];
  }
  for (int c = threadIdx.x; c < a.w; c += blockDim.x) {
    const size_t o = i * a.w + c;
    io.rho_prev[2 * o] = w.rho_prev[2 * c];
    io.rho_prev[2 * o + 1] = w.rho_prev[2 * c + 1];
    io.wind_abs[o] = w.wind_abs[c];
    io.wind_net[o] = w.wind_net[c];
    io.n_valid[o] = (int64_t)w.n_valid[c];
    io.sum_s[o] = w.sum_s[c];
  }
  if (threadIdx.x == 0) {
    io.status[i] = S.status == CCO_STATUS_BUDGET ? CCO_STATUS_RUNNING : S.status;
    io.keys[2 * i] = S.key[0];
    io.keys[2 * i + 1] = S.key[1];
    io.reset_acc[i] = S.acc;
    io.step[i] = S.step;
    io.time[i] = S.time;
    io.phi[i] = S.phi;
    io.e0[i] = S.e0;
    io.max_drift[i] = S.max_drift;
    io.sum_kinetic[i] = S.sum_kinetic;
    io.sum_phi[i] = S.sum_phi;
    io.sum_phi2[i] = S.sum_phi2;
    io.n_sum[i] = S.n_sum;
    io.snap_count[i] = S.snap_count;
    io.trace_count[i] = S.trace_count;
  }
}

__global__ void k_md_finalize(MdArgs a, double* r_out, double* v_out, double* f_out,
                              double* phi_out, double* ke_out, double* drift_out,
                              int64_t* resets_out, double* acc_out, uint32_t* keys_out,
                              int64_t* status_out) {
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const MdView w = md_view(R.rec, R.ld, a.w);
  for (int e = threadIdx.x; e < R.nd; e += blockDim.x) {
    r_out[R.soff + e] = w.r[e];
    v_out[R.soff + e] = w.v[e];
    if (f_out) f_out[R.soff + e] = w.f[e];
  }
  if (threadIdx.x == 0) {
    const MdState S = *w.st;
    phi_out[R.idx] = S.phi;
    ke_out[R.idx] = S.ke;
    drift_out[R.idx] = S.max_drift;
    resets_out[R.idx] = S.n_resets;
    acc_out[R.idx] = S.acc;
    keys_out[2 * R.idx] = S.key[0];   // the key of the next step
    keys_out[2 * R.idx + 1] = S.key[1];
    status_out[R.idx] = S.status;
  }
}

}  // namespace

cudaError_t md_init(const MdArgs& a, const double* r0, const double* v0, const double* mats,
                    const uint32_t* keys, const double* acc0, cudaStream_t st) {
  k_md_init<<<a.B, kUpdThreads, 0, st>>>(a, r0, v0, mats, keys, acc0);
  return cudaGetLastError();
}

cudaError_t md_update(const MdArgs& a, cudaStream_t st) {
  // c = exp(-gamma dt), 1 - c^2 = -expm1(-2 gamma dt) without cancellation;
  // the noise amplitude is sqrt((1 - c^2) T) with each lane's T
  const double c = std::exp(-a.gamma * a.dt);
  const double noise_var = -std::expm1(-2.0 * a.gamma * a.dt);
  if (a.w > a.nc) {
    const dim3 grid(a.B, (a.w - a.nc + kUpdThreads - 1) / kUpdThreads);
    k_md_waves<<<grid, kUpdThreads, 0, st>>>(a);
  }
  k_md_update<<<a.B, kUpdThreads, 0, st>>>(a, c, noise_var);
  if (a.w > 0) {
    const dim3 grid(a.B, (a.w + kUpdThreads - 1) / kUpdThreads);
    k_md_observe<<<grid, kUpdThreads, 0, st>>>(a);
  }
  return cudaGetLastError();
}

cudaError_t md_seg_init(const MdArgs& a, const double* mats, cudaStream_t st) {
  k_md_seg_init<<<a.B, kUpdThreads, 0, st>>>(a, mats);
  return cudaGetLastError();
}

cudaError_t md_seg_finalize(const MdArgs& a, cudaStream_t st) {
  k_md_seg_finalize<<<a.B, kUpdThreads, 0, st>>>(a);
  return cudaGetLastError();
}

cudaError_t md_finalize(const MdArgs& a, double* r_out, double* v_out, double* f_out,
                        double* phi_out, double* ke_out, double* drift_out, int64_t* resets_out,
                        double* acc_out, uint32_t* keys_out, int64_t* status_out,
                        cudaStream_t st) {
  k_md_finalize<<<a.B, kUpdThreads, 0, st>>>(a, r_out, v_out, f_out, phi_out, ke_out, drift_out,
                                             resets_out, acc_out, keys_out, status_out);
  return cudaGetLastError();
}

}  // namespace cco
