// Internal declarations shared by the CUDA translation units of libcco.
//
// HBM layout of one problem (built once by cco_problem_create):
//   seg1[nseg1], seg2[nseg2]  32-byte segment headers (runs of consecutive
//                             last-axis n, split at <= 8 / <= 256 rows)
//   w_run[M]                  weights in run order
//   run2ref[M]                run-order row -> caller row
// Per evaluated configuration (lane):
//   s[N][d] in, phi out, g[N][d] out, rho[M] / rhow[M] (complex, run order),
//   part[ntile1][M] pass-1 partial densities (one row per particle tile).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "cco.h"

namespace cco {

constexpr int kSeg1Len = 8;     // pass-1 segment length (register accumulators)
constexpr int kSeg2Len = 256;   // pass-2 segment length (phase re-seed interval)
constexpr int kPass1Threads = 128;
constexpr int kPass1Tile = 64;  // particles per pass-1 CTA
constexpr int kPass1Stride = kPass1Tile + 1;  // padded table row (bank spread)
constexpr int kPass2Threads = 128;
constexpr int kPass2Tile = kPass2Threads;     // one particle per pass-2 thread
constexpr int kMaxLevels = 3;
constexpr size_t kPass1TableBudget = 56 * 1024;   // bytes of pass-1 tables per CTA
constexpr size_t kPass2TableBudget = 44 * 1024;   // bytes of pass-2 tables per CTA
constexpr size_t kPass2RhoStage = 24 * 1024;      // density staged in pass-2 smem up to this
constexpr size_t kPass2RhoStage1D = 64 * 1024;    // the same for 1-D problems (no phase tables)

// One segment: rows kstart .. kstart+len-1 (run order) share the prefix
// n_0..n_{d-2}; the last axis runs n_{d-1} = n[d-1] + i.
// dig[a] packs the absolute table rows of the digits of |n_a| (start value
// for the last axis) in that pass's table layout: level l in bits 8l..8l+7,
// sign (n_a < 0) in bit 24.
struct SegHdr {
  int dig[3];
  int kstart;
  int n[3];
  int len;
};
static_assert(sizeof(SegHdr) == 32, "segment header is two 16-byte loads");

// Pass 1 as a complex GEMM (problems where it is efficient, FP64 lanes): the
// density of a particle tile on the grid (run r, last-axis n) is
// C[r][n] = sum_j A[r][j] Z[n][j] with A the run's prefix phase and Z the
// last-axis power z_j^n. The last axis is folded: a block's columns are
// c = |n|, and the four real products of A z^c give both C(c) and C(-c).
// Runs are grouped kGemmRows at a time (sorted by folded length) and each
// group's folded range is cut into windows of 16 cq columns (cq per problem,
// 1..kGemmFoldMaxCq); a (group, window) is a block, one CTA per (lane, tile,
// block).
constexpr int kGemmRows = 24, kGemmChunk = 32, kGemmThreads = 128;
constexpr int kGemmFoldMaxCq = 3;
// odd row stride of the last-axis table: table writes spread over banks
__host__ __device__ constexpr int gemm_fold_zstride(int cq) { return 16 * cq + 1; }
constexpr int kGemmMaxPrefix = 128;   // table entries per prefix axis
constexpr int kGemmMaxRun = 16;       // longest power chain between FP64 sincospi seeds
struct GemmRun {
  int n0, n1, a, b, kstart, pad_;   // prefix (n0[, n1]), last-axis range [a, b]
};
struct GemmBlock {
  int run0, nrun, lo, nb;            // runs [run0, run0 + nrun), columns lo .. lo + nb - 1
  int m0, c0, m1, c1;                // the group's prefix windows [m, m + c) per axis
};

// Per-particle phase tables of one pass: row r holds z_a^(e * base^l) for one
// (axis a, level l, entry e); level 0 always holds z^0 .. z^(base-1).
struct TabLayout {
  int nlev[3];
  int base[3];
  int nent[3][kMaxLevels];
  int row[3][kMaxLevels];
  int nrows;
  int zrow;   // row of z^1 of the last axis
};

// Device-resident problem descriptor.
struct ProbDev {
  int d, N, M, nseg1, nseg2;
  TabLayout t1, t2;          // pass-1 / pass-2 table layouts
  int ntile1, ntile2;        // particle tiles of pass 1 / pass 2 (pass 2 at split 1)
  int sl2;                   // logical slices of the pass-2 segment pairs (power of 2, <= 8)
  int gemm;                  // 1: FP64 pass 1 runs as the GEMM below
  int ngblk, gm0, gc0, gm1, gc1;   // GEMM blocks; gc0, gc1: the widest group prefix windows
  int gs0, gs1;              // their shared-memory row strides (odd)
  int gL, gu0, gu1, guz;     // table fill: gL entries per unit; units per particle per table
  int gcq, gpad_;            // d = 2: folded window of 16 gcq columns
  const GemmBlock* gblk;
  const GemmRun* grun;
  double vol;                // V
  double gpref;              // 2 (2 pi) / V
  const SegHdr* seg1;
  const SegHdr* seg2;        // sorted by length (pairs processed together)
  const double* w_run;
  const int* run2ref;
};

// One configuration evaluated by a launch.
struct EvalLane {
  const double* s;        // [N][d]
  double* f;              // [1]
  double* g;              // [N][d] or null
  double2* rho;           // [M] run order
  double2* rhow;          // [M] weighted density (pass-2 input)
  double2* part;          // [ntile1][M]
  const int64_t* status;  // evaluate iff null or *status == RUNNING
  const int32_t* prec;    // arithmetic of this evaluation: *prec, or `fixed_prec` when null
  int prob;
  int fixed_prec;         // PREC_FP64 or PREC_FP32
};

// Evaluation arithmetic of a lane. PREC_FP32: phase tables seeded in FP64
// and stored in FP32, phase recurrences, pass-1 accumulation (compensated)
// and the back-projection in FP32; the tile reduction, rho, w rho and Phi in
// FP64; pass-2 segment sums folded into FP64 gradients.
enum : int32_t { PREC_FP64 = 0, PREC_FP32 = 1 };
__device__ __forceinline__ int lane_prec(const EvalLane& ln) {
  return ln.prec ? *ln.prec : ln.fixed_prec;
}

struct EvalItem {
  int lane;
  int tile;
};

// ---------------------------------------------------------------- phases
// sin and cos of 2 pi m s for an integer-valued m and any s. The product m s
// is formed without rounding (p + e == m s, e by fma) and its nearest integer
// removed exactly before sincospi, so the phase keeps full precision however
// large |m s| is. Passing the rounded product instead puts |m s| eps of
// absolute error into the argument: 1.4e-12 rad at |m s| ~ 4000, which
// makes Phi ~ M (1.4e-12)^2 ~ 1e-20 the roundoff floor of a wide 1-D k-set.
__device__ __forceinline__ void sincos_2pi_ms(double m, double s, double* sn, double* cs) {
  const double p = m * s;
  const double e = fma(m, s, -p);
  sincospi(2.0 * ((p - rint(p)) + e), sn, cs);
}

// The same for n . s = sum_a n_a s_a (integer-valued n_a): exact products,
// compensated sum, nearest integer removed before sincospi.
template <int D>
__device__ __forceinline__ void sincos_2pi_dot(const double* n, const double* s, double* sn,
                                               double* cs) {
  double hi = 0.0, lo = 0.0;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const double p = n[a] * s[a];
    const double e = fma(n[a], s[a], -p);
    const double t = hi + p;
    const double z = t - hi;
    lo += ((hi - (t - z)) + (p - z)) + e;
    hi = t;
  }
  sincospi(2.0 * ((hi - rint(hi)) + lo), sn, cs);
}

// ---------------------------------------------------------------- complex
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ bool lane_active(const int64_t* status) {
  return status == nullptr || *status == CCO_STATUS_RUNNING;
}

// Deterministic block sum (fixed shuffle tree, then fixed warp order).
// `red` holds >= 32 doubles; every thread gets the total.
__device__ __forceinline__ double block_sum(double v, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < nw; ++w) t += red[w];
  return t;
}

// ---------------------------------------------------------------- launches
// Three launches per evaluation: partial densities, reduction + energy,
// gradient. Items index (lane, tile); lanes whose status is not RUNNING exit.
struct EvalPlan {
  const ProbDev* probs;     // device
  const EvalLane* lanes;    // device
  const EvalItem* items1;   // device, grouped by d: d = D items at [d_off1[D-1], d_off1[D])
  const EvalItem* items2;   // device, grouped the same way (d_off2)
  int n_lanes, n_items1, n_items2;
  int d_off1[4], d_off2[4];
  const EvalItem* itemsG;   // GEMM pass-1 items (lane, tile * ngblk + block), grouped by d
  int n_itemsG;
  int d_offG[4];
  // within dimension D's GEMM items (D = 2, 3): those of window width 16 cq at
  // [q_offG[D - 2][cq - 1], q_offG[D - 2][cq]) (one kernel per (D, cq))
  int q_offG[2][kGemmFoldMaxCq + 1];
  size_t smemG;
  int dyn_prec;             // 1: lanes may be FP32 (the FP32 pass kernels launch too), 0: FP64 only
  int max_d;                // largest d in the plan (template dispatch)
  int red_chunks;           // k-chunks of the reduction: ceil(max M / kReduceChunk)
  int split2;               // pass-2 threads per particle (1, 2, 4 or 8)
  int chunks1;              // pass-1 segment chunks per tile (FP64 per-segment form; 1 = none)
  size_t smem1, smem2;      // dynamic shared memory of pass 1 / pass 2 (FP64 kernels)
  size_t smem2_f32;         // pass 2, FP32 kernels
  bool want_grad;
};

// A launch with few pass-1 tiles (a lone wide lane: one CTA per SM at most)
// splits each tile's segments over up to 8 CTAs. Only problems with at least
// 2 kPass1ChunkSegs segments are split, where one thread already owns one
// segment (no in-CTA particle slices), so every segment's sum is computed
// exactly as unsplit: the chunking changes where the work runs, not the bits.
// A tile is cut into no more chunks than it takes to give each thread of a
// 128-thread CTA one segment (ceil(nseg / 128)).
constexpr int kPass1ChunkSegs = 128;
__host__ __device__ __forceinline__ int pass1_chunks(const ProbDev& p, int plan_chunks) {
  if (p.nseg1 < 2 * kPass1ChunkSegs) return 1;
  const int most = (p.nseg1 + kPass1ChunkSegs - 1) / kPass1ChunkSegs;
  return plan_chunks < most ? plan_chunks : most;
}

// The reduction of the pass-1 partials runs one block per kReduceChunk
// k-vectors of a lane; a second kernel sums the chunks' energies in a fixed
// order, so the energy's rounding depends on M alone.
constexpr int kReduceChunk = 256;
__host__ __device__ __forceinline__ int reduce_chunks(int M) {
  return (M + kReduceChunk - 1) / kReduceChunk;
}

// Side streams of one launching stream: when a plan holds lanes of several
// dimensions, each dimension's pass kernels run on their own stream (forked
// from and joined back into the launching stream with these events), so the
// small per-dimension grids of a mixed plan overlap instead of running back
// to back. The kernels and their results are the same either way.
struct EvalSide {
  cudaStream_t aux[2];
  cudaEvent_t fork, join[2];
};
cudaError_t eval_launch(const EvalPlan& plan, cudaStream_t stream,
                        const EvalSide* side = nullptr);
// Kernels one eval_launch of a plan issues: per dimension the per-segment and
// GEMM pass-1 kernels and the pass-2 kernel that have items, plus the reduction (and
// the energy kernel when there is no pass 2).
inline int eval_kernels(const EvalPlan& p) {
  int n = p.n_lanes > 0 ? (p.want_grad ? 1 : 2) : 0;   // reduce (+ energy without pass 2)
  const int per = p.dyn_prec ? 2 : 1;   // FP64 and FP32 pass kernels
  for (int D = 1; D <= 3; ++D) {
    n += per * (p.d_off1[D] > p.d_off1[D - 1]);
    if (D >= 2)
      for (int c = 0; c < kGemmFoldMaxCq; ++c) n += p.q_offG[D - 2][c + 1] > p.q_offG[D - 2][c];
    if (p.want_grad) n += per * (p.d_off2[D] > p.d_off2[D - 1]);
  }
  return n;
}

// Dimensions whose pass kernels a plan launches (side streams pay off from 2).
inline int eval_dims(const EvalPlan& p) {
  int n = 0;
  for (int D = 1; D <= 3; ++D)
    n += p.d_off1[D] > p.d_off1[D - 1] || p.d_offG[D] > p.d_offG[D - 1] ||
         p.d_off2[D] > p.d_off2[D - 1];
  return n;
}
size_t eval_smem1(const ProbDev& p);
size_t eval_smemG(const ProbDev& p);   // GEMM pass 1 (0 when the problem has none)
// Pass-2 dynamic shared memory at `split` for the FP64 kernels, or with
// f32 for the FP32 ones (which keep phase tables for 1-D problems too).
size_t eval_smem2(const ProbDev& p, int split, bool f32 = false);
// Pass-2 tiles of one configuration when `split` threads share a particle.
int pass2_tiles(const ProbDev& p, int split);
// Threads per particle in pass 2 for a launch whose configurations have
// `tiles_at_split1` tiles in total at split 1: the smallest power of two
// (<= 8) that gives kPass2TargetCtas CTAs (CCO_PASS2_SPLIT overrides).
// It changes how work is spread, never the arithmetic.
constexpr long long kPass2TargetCtas = 148 * 3;
int pass2_split(long long tiles_at_split1);
cudaError_t eval_configure();   // opt-in to large dynamic shared memory

// Copy the run-order density of lane i out in the caller's row order.
cudaError_t rho_scatter(const double2* rho_run, const int* run2ref, int M,
                        int batch, size_t lane_stride, double* re, double* im,
                        cudaStream_t stream);

}  // namespace cco
