// Per-lane minimizer state machines (device side). See cco_opt.cu.
//
// Every lane owns one contiguous record in device memory holding its whole
// state: the state machine scalars, its vectors, its L-BFGS history and the
// scratch of its energy evaluations (densities and pass-1 partials). Kernels
// reach a lane through a LaneRef table, so a batch may mix lanes of different
// N, d and k-set, and the serving pool can add and retire lanes between
// launches without moving any lane's state.
#pragma once

#include "cco_internal.cuh"

namespace cco {

enum : int { PH_INIT = 0, PH_ITER = 1, PH_EXPAND = 1, PH_ZOOM = 2, PH_REEVAL = 3 };

// Mixed-precision L-BFGS: a lane of a d >= 2 problem starts with FP32
// evaluations and switches to FP64 for good once its energy falls below
// kFp32SwitchPerParticle * N, or on any outcome that would stop it (the FP32
// energy is too coarse to judge). At the switch the history is cleared and the
// current point is evaluated again in FP64 before the next direction, so every
// energy the line search compares and the final judgement come from FP64
// evaluations. A lane that nevertheless ends above the energy tolerance is
// restarted from its initial positions in FP64 and then repeats, bit for bit,
// the plain FP64 run of the same configuration: the mixed form's success mask
// equals the plain one's wherever plain FP64 fails. Lanes of 1-D problems run
// FP64 throughout (their slow, marginal approach to 1e-20 is where an FP32
// prefix changed outcomes).
constexpr double kFp32SwitchPerParticle = 1e-6;

// One lane of a launch.
struct LaneRef {
  double* rec;      // lane record (layouts below)
  int nd, ld;       // N d, and N d rounded up to a multiple of 4 doubles
  int64_t soff;     // offset of the lane in the caller's packed positions
  int64_t toff;     // offset of the lane's trajectory rows in traj_s
  int32_t idx;      // the lane's index in the call: its row of traj_e/step/it/count
  int32_t n;        // particles N
};

__host__ __device__ __forceinline__ int pad4(int nd) { return (nd + 3) & ~3; }

// Both state structs start with the status word, so a lane's status is the
// first int64 of its record whatever the minimizer.
__host__ __device__ __forceinline__ int64_t* rec_status(double* rec) {
  return reinterpret_cast<int64_t*>(rec);
}

// ------------------------------------------------------------ descent
// Record: [0, 16) DsState and the probe energy pf at [15]; then s, g, ps, pg
// (ld each); then the evaluation scratch (double2: rho M, rhow M, part nt1 M).
struct DsState {
  int64_t status, it, n_evals, t0, t1;   // t0/t1: %globaltimer at start / completion
  double f, step, norm;
  int32_t phase, nonzero;
};
constexpr int kDsHead = 16;

struct DsView {
  DsState* st;
  double *pf, *s, *g, *ps, *pg;
  double2* dens;
};

__host__ __device__ __forceinline__ DsView ds_view(double* rec, int ld) {
  DsView v;
  v.st = reinterpret_cast<DsState*>(rec);
  v.pf = rec + kDsHead - 1;
  v.s = rec + kDsHead;
  v.g = v.s + ld;
  v.ps = v.s + 2 * (size_t)ld;
  v.pg = v.s + 3 * (size_t)ld;
  v.dens = reinterpret_cast<double2*>(v.s + 4 * (size_t)ld);
  return v;
}

__host__ __device__ __forceinline__ size_t ds_record_doubles(int ld, int M, int nt1) {
  return kDsHead + 4 * (size_t)ld + 2 * (size_t)M * (2 + nt1);
}

struct DescentArgs {
  int B;
  const LaneRef* lanes;
  double step_init, step_min, shrink, grow, rel_tol, energy_tol;
  int64_t max_iters;      // max_evals // 2
  int64_t rec_every, rec_cap;
  // trajectory (null when off): traj_e/step/it/count rows by LaneRef::idx, traj_s by toff
  double *traj_s, *traj_e, *traj_step;
  int64_t *traj_it, *traj_count;
};

// ------------------------------------------------------------ L-BFGS
struct LbState {
  int64_t status, it, n_evals, pass_evals, stag;
  int64_t t0, t1;         // %globaltimer at start / completion
  double f, R;
  double f0, dphi0, alpha;
  double a_prev, f_prev, d_prev;
  double a_lo, f_lo, d_lo;
  double a_hi, f_hi, d_hi;
  double gamma, last_step;
  int32_t phase, ls_steps, pass_idx, hk, hhead, have_lo, newpair, need_dir;
  int32_t prec;           // evaluation arithmetic (PREC_FP64 / PREC_FP32)
  int32_t n_fp32;         // evaluations done in FP32
  int32_t mode;           // 0: FP64 lane; 1: started in FP32; 2: restarted in FP64 from s0
  int32_t pad_;
  int64_t evals_prior;    // evaluations before a restart (counted in the result)
};
constexpr int kLbHead = 32;   // LbState (30 doubles) and pf at [31]
static_assert(sizeof(LbState) <= (kLbHead - 1) * sizeof(double), "LbState outgrew its slot");
static_assert(sizeof(DsState) <= (kDsHead - 1) * sizeof(double), "DsState outgrew its slot");

constexpr int kUpdThreads = 256;

// Wide lanes (more than kLbWide double2 words) split the two history passes
// finer, so that a lone wide lane still spreads its stream over many SMs:
// pass A over element chunks of kLbWide words (each warp's partial dots are
// summed in chunk order by the scalar kernel), pass B over kPassBGroups pair
// groups of 32-word element blocks (the groups' sums are added in group
// order). Which form a lane takes depends on its size alone, so its bits do
// not depend on the batch it runs in.
constexpr int kLbWide = 1024;
constexpr int kPassBGroups = kUpdThreads / 32;
__host__ __device__ __forceinline__ bool lb_wide(int ld) { return (ld >> 1) > kLbWide; }
// Pass-A element chunks of a lane.
__host__ __device__ __forceinline__ int lb_achunks(int ld) {
  return lb_wide(ld) ? ((ld >> 1) + kLbWide - 1) / kLbWide : 1;
}
// Pass-B element blocks of a lane: one double2 word per thread, or 32 words
// per block (a word per warp lane, a pair group per warp) for wide lanes.
__host__ __device__ __forceinline__ int lb_nblk(int ld) {
  return lb_wide(ld) ? ((ld >> 1) + 31) / 32 : ((ld >> 1) + kUpdThreads - 1) / kUpdThreads;
}
// Scalar row: a_p, b_p (m each), gamma + cy (1 + m), cs (m), pass-B partials,
// then (wide lanes) the pass-A partials: [chunk][a, b, sy, yy][m].
__host__ __device__ __forceinline__ size_t lb_scal_len(int m, int ld) {
  const size_t apart = lb_wide(ld) ? (size_t)4 * m * lb_achunks(ld) : 0;
  return ((size_t)4 * m + 1 + lb_nblk(ld) + apart + 3) & ~(size_t)3;
}
__host__ __device__ __forceinline__ size_t lb_apart_off(int m, int ld) {
  return (size_t)4 * m + 1 + lb_nblk(ld);
}

// Record: [0, 32) LbState, pf at [31]; SY (m m, row = newer slot), YY (m m);
// the packed triangles of the scalar kernel (tri_len = m (m + 1) when
// they do not fit in shared memory, else 0); the scalar row; x, s, g, dir, glo, ps, pg (ld each); the
// history rings S and Y (m ld each); s0 (ld, mixed precision only); the evaluation scratch.
struct LbView {
  LbState* st;
  double *pf, *SY, *YY, *tri, *scal;
  double *x, *s, *g, *dir, *glo, *ps, *pg, *Sh, *Yh;
  double* s0;             // the lane's initial positions (mixed precision only, else null)
  double2* dens;
};

// keep_s0: the record holds a copy of the lane's initial positions (ld
// doubles after the history), which mixed-precision lanes restart from.
__host__ __device__ __forceinline__ LbView lb_view(double* rec, int m, int tri_len, int ld,
                                                   int keep_s0 = 0) {
  LbView v;
  const size_t mm = (size_t)m * m;
  v.st = reinterpret_cast<LbState*>(rec);
  v.pf = rec + kLbHead - 1;
  v.SY = rec + kLbHead;
  v.YY = v.SY + mm;
  v.tri = v.YY + mm;
  v.scal = v.tri + tri_len;
  v.x = v.scal + lb_scal_len(m, ld);
  v.s = v.x + ld;
  v.g = v.x + 2 * (size_t)ld;
  v.dir = v.x + 3 * (size_t)ld;
  v.glo = v.x + 4 * (size_t)ld;
  v.ps = v.x + 5 * (size_t)ld;
  v.pg = v.x + 6 * (size_t)ld;
  v.Sh = v.x + 7 * (size_t)ld;
  v.Yh = v.Sh + (size_t)m * ld;
  v.s0 = keep_s0 ? v.Yh + (size_t)m * ld : nullptr;
  v.dens = reinterpret_cast<double2*>(v.Yh + (size_t)(m + (keep_s0 ? 1 : 0)) * ld);
  return v;
}

__host__ __device__ __forceinline__ size_t lb_record_doubles(int m, int tri_len, int ld, int M,
                                                             int nt1, int keep_s0 = 0) {
  return kLbHead + 2 * (size_t)m * m + tri_len + lb_scal_len(m, ld) +
         (7 + 2 * (size_t)m + (keep_s0 ? 1 : 0)) * ld + 2 * (size_t)M * (2 + nt1);
}

struct LbArgs {
  int B, m, n_pass, tri_len;
  const LaneRef* lanes;
  double rescales[CCO_MAX_RESCALES];
  double energy_tol, grad_tol;
  int64_t budget, patience, max_ls;
  int64_t rec_every, rec_cap;
  int prec0;              // PREC_FP32: lanes of d >= 2 start in FP32 (mixed precision)
  int keep_s0;            // records hold s0 (mixed precision: restart of a failed lane)
  int nblkB;              // grid width of pass B (max over the lanes)
  int nchA;               // pass-A element chunks (max over the lanes)
  size_t smem_tri;        // 0: triangles in the record (global memory)
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
                           int64_t* n32_out, cudaStream_t st);

// Count lanes whose status is RUNNING.
cudaError_t count_running(const LaneRef* lanes, int B, int* out, cudaStream_t st);
// Copy every lane's status into out[B].
cudaError_t gather_status(const LaneRef* lanes, int B, int64_t* out, cudaStream_t st);
// Ends an L-BFGS lane with CCO_STATUS_CANCELLED if it is still RUNNING.
cudaError_t cancel_lbfgs_lane(double* rec, cudaStream_t st);

}  // namespace cco
