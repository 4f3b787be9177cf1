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
  const MdView w = md_view(R.rec, R.ld);
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

__global__ void __launch_bounds__(kUpdThreads) k_md_update(MdArgs a, double c, double noise) {
  __shared__ MdState S;
  __shared__ double red[32];
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const MdView w = md_view(R.rec, R.ld);
  if (threadIdx.x == 0) S = *w.st;
  __syncthreads();
  if (S.status != CCO_STATUS_RUNNING) return;
  const int d = R.nd / R.n;
  forces(R, w, S, d);
  __syncthreads();
  if (S.phase == 0) {
    // forces at the start: energy reference for the drift
    const double ke = kinetic(R, w, red);
    if (threadIdx.x == 0) {
      S.phi = *w.pf;
      S.ke = ke;
      S.e0 = S.phi + ke;
      S.max_drift = 0.0;
      S.phase = 1;
      if (a.n_steps <= 0) {
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
          sqrt(a.temperature) * normal(draw(S, RNG_ROW, threadIdx.x));
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
      S.max_drift = fmax(S.max_drift, drift);
      if (a.drift_tol > 0.0 && !(drift <= a.drift_tol)) S.status = CCO_STATUS_DRIFT;
      else if (S.step >= a.n_steps) S.status = CCO_STATUS_BUDGET;
      if (S.status != CCO_STATUS_RUNNING) S.t1 = gtimer();
    }
  }
  __syncthreads();
  if (S.status == CCO_STATUS_RUNNING) begin_step(a, R, w, S, d, c, noise);
  __syncthreads();
  if (threadIdx.x == 0) *w.st = S;
}

__global__ void k_md_finalize(MdArgs a, double* r_out, double* v_out, double* f_out,
                              double* phi_out, double* ke_out, double* drift_out,
                              int64_t* resets_out, double* acc_out, uint32_t* keys_out,
                              int64_t* status_out) {
  const int lane = blockIdx.x;
  const LaneRef R = a.lanes[lane];
  const MdView w = md_view(R.rec, R.ld);
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
  // c = exp(-gamma dt), 1 - c^2 = -expm1(-2 gamma dt) without cancellation
  const double c = std::exp(-a.gamma * a.dt);
  const double noise = std::sqrt(-std::expm1(-2.0 * a.gamma * a.dt) * a.temperature);
  k_md_update<<<a.B, kUpdThreads, 0, st>>>(a, c, noise);
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
