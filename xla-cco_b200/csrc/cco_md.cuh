// Molecular-dynamics lanes (device side): velocity Verlet with optional
// Andersen resets, and Langevin BAOAB, one force evaluation per tick.
// See cco_md.cu.
#pragma once

#include "cco_opt.cuh"

namespace cco {

// MD record: [0, kMdHead) MdState (with the basis matrices) and the probe
// energy pf at [kMdHead - 1]; then r, v, f (Cartesian), ps (fractional probe
// r B^-1) and pg (its gradient), ld each; then the evaluation scratch.
struct MdState {
  int64_t status, step, n_resets;
  int64_t t0, t1;
  double phi, ke, e0, max_drift, acc;
  double B[9], Binv[9], BinvT[9];
  uint32_t key[2];
  int32_t phase, pad_;
};
constexpr int kMdHead = 48;
static_assert(sizeof(MdState) <= (kMdHead - 1) * sizeof(double), "MdState outgrew its slot");

struct MdView {
  MdState* st;
  double *pf, *r, *v, *f, *ps, *pg;
  double2* dens;
};

__host__ __device__ __forceinline__ MdView md_view(double* rec, int ld) {
  MdView w;
  w.st = reinterpret_cast<MdState*>(rec);
  w.pf = rec + kMdHead - 1;
  w.r = rec + kMdHead;
  w.v = w.r + ld;
  w.f = w.r + 2 * (size_t)ld;
  w.ps = w.r + 3 * (size_t)ld;
  w.pg = w.r + 4 * (size_t)ld;
  w.dens = reinterpret_cast<double2*>(w.r + 5 * (size_t)ld);
  return w;
}

__host__ __device__ __forceinline__ size_t md_record_doubles(int ld, int M, int nt1) {
  return kMdHead + 5 * (size_t)ld + 2 * (size_t)M * (2 + nt1);
}

enum : int { MD_VERLET = 0, MD_BAOAB = 1 };
enum : int { ANDERSEN_OFF = 0, ANDERSEN_COUNT = 1, ANDERSEN_BERNOULLI = 2 };

struct MdArgs {
  int B;
  const LaneRef* lanes;
  double dt, gamma, temperature, andersen_p, drift_tol;
  int64_t n_steps;
  int scheme, andersen;
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

}  // namespace cco
