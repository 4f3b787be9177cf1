// Per-lane minimizer state machines (device side). See cco_opt.cu.
#pragma once

#include "cco_internal.cuh"

namespace cco {

enum : int { PH_INIT = 0, PH_ITER = 1, PH_EXPAND = 1, PH_ZOOM = 2 };

// ------------------------------------------------------------ descent
// Lane layouts: lanes may differ in N and d (mixed batches, the serving
// pool). Every per-lane array is addressed through device offset arrays:
//   voff[i]  offset (doubles) of lane i in each lane-vector array
//   soff[i]  offset of lane i in the caller's packed positions (N_i d_i each)
//   toff[i]  offset of lane i's trajectory rows in traj_s
//   lnd[i]   N_i d_i
struct DescentArgs {
  int B;
  const int64_t *voff, *soff, *toff;
  const int* lnd;
  double step_init, step_min, shrink, grow, rel_tol, energy_tol;
  int64_t max_iters;      // max_evals // 2
  int64_t rec_every, rec_cap;
  // lane state (SoA)
  double *s, *g;          // [B][nd] accepted point and its gradient
  double* ps;             // [B][nd] probe positions (evaluation input)
  const double* pg;       // [B][nd] probe gradient (evaluation output)
  const double* pf;       // [B]     probe energy
  double *f, *step, *norm;
  int64_t *it, *n_evals, *status;
  int* phase;
  int* nonzero;           // [B] any(g != 0)
  int64_t *t0, *t1;       // [B] %globaltimer at start / completion
  // trajectory (null when off)
  double *traj_s, *traj_e, *traj_step;
  int64_t *traj_it, *traj_count;
};

// ------------------------------------------------------------ L-BFGS
struct LbState {
  double f, R;
  double f0, dphi0, alpha;
  double a_prev, f_prev, d_prev;
  double a_lo, f_lo, d_lo;
  double a_hi, f_hi, d_hi;
  double gamma, last_step;
  int64_t it, n_evals, pass_evals, stag, status;
  int64_t t0, t1;         // %globaltimer at start / completion
  int32_t phase, ls_steps, pass_idx, hk, hhead, have_lo, newpair, need_dir;
};

struct LbArgs {
  int B, m, n_pass;
  // lane layouts (see DescentArgs); lld[i] = N_i d_i rounded up to 4 doubles
  // (16-byte rows, zero padding); hoff[i] = offset of lane i in Sh and Yh
  const int64_t *voff, *soff, *toff, *hoff;
  const int *lnd, *lld;
  double rescales[CCO_MAX_RESCALES];
  double energy_tol, grad_tol;
  int64_t budget, patience, max_ls;
  int64_t rec_every, rec_cap;
  LbState* st;            // [B]
  double *x, *s, *g, *dir, *glo;   // [B][nd]
  double* ps;             // [B][nd] probe s = (x + alpha dir) / R (evaluation input)
  const double* pg;       // [B][nd] probe dPhi/ds (evaluation output)
  const double* pf;       // [B]
  double *Sh, *Yh;        // [B][m][nd] history rings
  double *SYs, *YYs;      // [B][m][m] slot inner products (SYs: row = newer slot)
  double* tri_g;          // [B][m (m+1) + 7m] packed triangles when they do not fit in smem
  double* scal;           // [B][scal_stride] a_p, b_p, gamma, cy, cs, pass-B partials
  int scal_stride, nblkB; // row length of scal; pass-B element blocks per lane
  size_t smem_tri;        // 0: triangles in global memory
  double *traj_s, *traj_e, *traj_step;
  int64_t *traj_it, *traj_count;
};

cudaError_t descent_init(const DescentArgs& a, const double* s0, cudaStream_t st);
cudaError_t descent_update(const DescentArgs& a, cudaStream_t st);
cudaError_t descent_finalize(const DescentArgs& a, double* s_out, double* e_out,
                             double* gn_out, int64_t* ne_out, int64_t* ni_out,
                             int64_t* st_out, int64_t* lat_out, cudaStream_t st);

size_t lbfgs_update_smem(int m);
cudaError_t lbfgs_configure(size_t smem);
cudaError_t lbfgs_init(const LbArgs& a, const double* s0, cudaStream_t st);
cudaError_t lbfgs_update(const LbArgs& a, cudaStream_t st);
cudaError_t lbfgs_finalize(const LbArgs& a, double* s_out, double* e_out, double* gn_out,
                           int64_t* ne_out, int64_t* ni_out, int64_t* st_out, int64_t* lat_out,
                           cudaStream_t st);

// Count lanes whose status is RUNNING (status stride in int64 units).
cudaError_t count_running(const int64_t* status, size_t stride, int B, int* out,
                          cudaStream_t st);

}  // namespace cco
