// Stealthy energy, gradient and collective density on sm_100a (FP64).
//
// Reference math (src/xla_cco/energy.py:45-50,195-225,301-324):
//   rho_k  = sum_j exp(2 pi i n_k . s_j)
//   Phi    = (1/V) sum_k w_k |rho_k|^2
//   dPhi/ds_j = (2 (2 pi) / V) sum_k w_k (Im rho_k cos th_kj - Re rho_k sin th_kj) n_k
//
// B200 formulation. The k-set is stored as runs of consecutive last-axis n
// with a fixed prefix (n_0..n_{d-2}); along a run the phase advances by one
// complex multiply, exp(i th_{k+1,j}) = exp(i th_kj) z_j, z_j = exp(2 pi i
// s_{j,d-1}). A segment start takes its phase from per-particle tables in
// shared memory: z_a^|n| = prod_l T_a,l[digit_l(|n|)]. Table entries come
// from FP64 sincospi of the exact integer exponent (the product e s reduced
// without rounding, sincos_2pi_ms), re-seeded every 8 entries
// with products in between, so a phase carries O(10 eps) error on top of the
// <= segment-length products along a run - inside the reference's eps |theta|
// trig error. No theta matrix ever reaches HBM: traffic per evaluation is s
// in, g out and the M-row density, so both passes are FP64-pipe bound.
//
//   pass 1 (k_pass1): CTA = (configuration, 64-particle tile), 128 threads.
//     A thread owns a segment of <= 8 rows and streams the tile's particles
//     four at a time (four independent phase chains), accumulating 8 complex
//     sums in registers: no cross-thread reduction. Small k-sets split the
//     particles into slices summed in a fixed order. Output: one partial
//     density row per tile.
//   reduce  (k_reduce): sums the tile rows in tile order (deterministic),
//     forms rho, w rho and Phi (fixed-order block sum).
//   pass 2 (k_pass2): CTA = (configuration, 128-particle tile), one particle
//     per thread; the CTA walks the segments two at a time (two independent
//     chains per thread; density reads are warp-uniform broadcasts, fetched
//     two rows ahead). Per row: one complex multiply, the coefficient
//     w(Im rho cos - Re rho sin) and two accumulations; prefix axes are
//     weighted once per segment.
#include <cstdio>
#include <cstdlib>

#include "cco_eval_bodies.cuh"
#include "cco_internal.cuh"

namespace cco {

namespace {

// One kernel per (dimension, window width): each holds one body, so the
// instruction cache serves one folded product loop.
template <int D, int CQ>
__global__ void __launch_bounds__(kGemmThreads, 4) k_pass1_gemm(EvalPlan plan) {
  extern __shared__ double2 smem[];
  __shared__ ProbDev sp;
  const EvalItem it = plan.itemsG[plan.q_offG[D - 2][CQ - 1] + blockIdx.x];
  const EvalLane ln = plan.lanes[it.lane];
  if (!lane_active(ln.status)) return;
  if (plan.dyn_prec && lane_prec(ln) == PREC_FP32) return;   // the FP32 body handles it
  if (threadIdx.x == 0) sp = plan.probs[ln.prob];
  __syncthreads();
  if constexpr (D == 2)
    pass1_gemm_body_d2<CQ>(sp, ln, it.tile / sp.ngblk, it.tile % sp.ngblk, smem);
  else
    pass1_gemm_body<D, CQ>(sp, ln, it.tile / sp.ngblk, it.tile % sp.ngblk, smem);
}

template <int D>
void launch_gemm(const EvalPlan& plan, cudaStream_t s) {
  const int* q = plan.q_offG[D - 2];
  if (q[1] > q[0]) k_pass1_gemm<D, 1><<<q[1] - q[0], kGemmThreads, plan.smemG, s>>>(plan);
  if (q[2] > q[1]) k_pass1_gemm<D, 2><<<q[2] - q[1], kGemmThreads, plan.smemG, s>>>(plan);
  if (q[3] > q[2]) k_pass1_gemm<D, 3><<<q[3] - q[2], kGemmThreads, plan.smemG, s>>>(plan);
}

template <int D>
cudaError_t configure_gemm() {
  cudaError_t e = cudaFuncSetAttribute(k_pass1_gemm<D, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       227 * 1024 - 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_pass1_gemm<D, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024 - 1024);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_pass1_gemm<D, 3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             227 * 1024 - 1024);
  return e;
}

// One kernel per dimension D and arithmetic keeps each kernel's code small:
// the instruction cache holds one body instead of all of them. F32 = false
// evaluates the FP64 lanes of a launch, F32 = true its FP32 lanes (a plan with
// FP32 lanes launches both). An FP64 lane therefore always runs the same
// kernel, in a mixed-precision run and in a plain one, and gets the same bits.
template <int D, bool F32>
__global__ void __launch_bounds__(kPass1Threads, 4) k_pass1(EvalPlan plan) {
  extern __shared__ double2 smem[];
  __shared__ ProbDev sp;
  const EvalItem it = plan.items1[plan.d_off1[D - 1] + blockIdx.x];
  const EvalLane ln = plan.lanes[it.lane];
  if (!lane_active(ln.status)) return;
  if ((lane_prec(ln) == PREC_FP32) != F32) return;   // the other kernel's lane
  if (threadIdx.x == 0) sp = plan.probs[ln.prob];
  __syncthreads();
  if (F32) {
    pass1_body_f32<D>(sp, ln, it.tile, smem);
  } else if (!sp.gemm) {   // GEMM problems: k_pass1_gemm
    const int C = pass1_chunks(sp, plan.chunks1);
    pass1_body<D>(sp, ln, it.tile / C, smem, it.tile % C, C);
  }
}

// Reduction (grid: k-chunks x lanes): rho_k = sum over tiles of the pass-1
// partials in tile order, the weighted density for pass 2, and this chunk's
// part of sum w |rho|^2, stored over the chunk's first partial (which only
// this block reads).
__global__ void __launch_bounds__(kReduceChunk) k_reduce(EvalPlan plan) {
  __shared__ double red[32];
  const EvalLane ln = plan.lanes[blockIdx.y];
  if (!lane_active(ln.status)) return;
  const ProbDev& P = plan.probs[ln.prob];
  const int M = P.M, nt = P.ntile1;
  const int k0 = blockIdx.x * kReduceChunk;
  if (k0 >= M) return;
  const int k = k0 + threadIdx.x;
  double e = 0.0;
  if (k < M) {
    const double2* __restrict__ col = ln.part + k;
    double2 t = col[0];
    int q = 1;
    // sixteen tile rows in flight per step, added in tile order (the same sums
    // as one row at a time; a lone lane of many tiles is latency-bound here)
    for (; q + 16 <= nt; q += 16) {
      double2 o[16];
#pragma unroll
      for (int u = 0; u < 16; ++u) o[u] = col[(size_t)(q + u) * M];
#pragma unroll
      for (int u = 0; u < 16; ++u) {
        t.x += o[u].x;
        t.y += o[u].y;
      }
    }
    for (; q < nt; ++q) {
      const double2 o = col[(size_t)q * M];
      t.x += o.x;
      t.y += o.y;
    }
    ln.rho[k] = t;
    const double wk = P.w_run[k];
    if (lane_prec(ln) == PREC_FP32)
      reinterpret_cast<float2*>(ln.rhow)[k] = make_float2((float)(wk * t.x), (float)(wk * t.y));
    else
      ln.rhow[k] = make_double2(wk * t.x, wk * t.y);
    e = wk * (t.x * t.x + t.y * t.y);
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) ln.part[k0] = make_double2(e, 0.0);
}

// Energy of one lane (one warp): the chunk energies summed in a fixed order.
__device__ __forceinline__ void lane_energy(const EvalPlan& plan, const EvalLane& ln) {
  const ProbDev& P = plan.probs[ln.prob];
  const int nc = reduce_chunks(P.M);
  double e = 0.0;
  for (int c = threadIdx.x; c < nc; c += 32) e += ln.part[(size_t)c * kReduceChunk].x;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if (threadIdx.x == 0) *ln.f = e / P.vol;
}

// Energy-only evaluations (no pass 2): one warp per lane. With the gradient,
// the first warp of each lane's first pass-2 tile sums it instead (one launch
// fewer per evaluation, the same sum).
__global__ void k_energy(EvalPlan plan) {
  const EvalLane ln = plan.lanes[blockIdx.x];
  if (!lane_active(ln.status)) return;
  lane_energy(plan, ln);
}

template <int D, bool F32>
__global__ void __launch_bounds__(kPass2Threads, 4) k_pass2(EvalPlan plan) {
  extern __shared__ double2 smem[];
  __shared__ ProbDev sp;
  const EvalItem it = plan.items2[plan.d_off2[D - 1] + blockIdx.x];
  const EvalLane ln = plan.lanes[it.lane];
  if (!lane_active(ln.status)) return;
  if ((lane_prec(ln) == PREC_FP32) != F32) return;   // the other kernel's lane
  if (it.tile == 0 && threadIdx.x < 32) lane_energy(plan, ln);
  if (ln.g == nullptr) return;
  if (threadIdx.x == 0) sp = plan.probs[ln.prob];
  __syncthreads();
  if (D == 1 && !F32) {
    if ((size_t)sp.M * sizeof(double2) <= kPass2RhoStage1D)
      pass2_body_1d<true>(sp, ln, it.tile, plan.split2, smem);
    else
      pass2_body_1d<false>(sp, ln, it.tile, plan.split2, smem);
    return;
  }
  const bool staged = (size_t)sp.M * sizeof(double2) <= kPass2RhoStage;
  if (F32) {
    if (staged)
      pass2_body_f32<D, true>(sp, ln, it.tile, plan.split2, smem);
    else
      pass2_body_f32<D, false>(sp, ln, it.tile, plan.split2, smem);
    return;
  }
  if (staged)
    pass2_body<D, true>(sp, ln, it.tile, plan.split2, smem);
  else
    pass2_body<D, false>(sp, ln, it.tile, plan.split2, smem);
}

__global__ void k_rho_scatter(const double2* __restrict__ rho, const int* __restrict__ run2ref,
                              int M, int batch, size_t lane_stride, double* re, double* im) {
  const size_t total = (size_t)M * batch;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total;
       t += (size_t)gridDim.x * blockDim.x) {
    const int b = (int)(t / M), k = (int)(t - (size_t)b * M);
    const double2 v = rho[(size_t)b * lane_stride + k];
    const size_t o = (size_t)b * M + run2ref[k];
    if (re) re[o] = v.x;
    if (im) im[o] = v.y;
  }
}

}  // namespace

int pass1_slices(int nseg, int nj) {
  int ns = 1;
  while (2 * ns * nseg <= kPass1Threads && 2 * ns <= nj) ns *= 2;
  return ns;
}

size_t eval_smem1(const ProbDev& p) {
  const int ns = pass1_slices(p.nseg1, kPass1Tile);
  const size_t red = ns > 1 ? (size_t)ns * p.nseg1 * kSeg1Len : 0;
  return ((size_t)p.t1.nrows * kPass1Stride + red) * sizeof(double2);
}

size_t eval_smemG(const ProbDev& p) {
  if (!p.gemm) return 0;
  if (p.d == 2)   // two table sets (prefix, last axis) and two root sets
    return (size_t)kGemmChunk * (2 * (p.gs0 + gemm_fold_zstride(p.gcq)) + 2 * p.d) *
           sizeof(double2);
  const int s1 = p.d == 3 ? p.gs1 : 0;
  return (size_t)kGemmChunk * (p.gs0 + s1 + gemm_fold_zstride(p.gcq) + kGemmRows + 2 * p.d) *
         sizeof(double2);
}

size_t eval_smem2(const ProbDev& p, int split, bool f32) {
  if (p.d == 1 && !f32) {   // pass2_body_1d: the staged density and the slice combine
    const size_t rho = (size_t)p.M * sizeof(double2);
    const size_t comb = split > 1 ? (size_t)kPass2Tile * sizeof(double) : 0;
    return (rho <= kPass2RhoStage1D ? rho : 0) + comb;
  }
  const size_t rho = (size_t)p.M * sizeof(double2);
  const size_t comb = split > 1 ? (size_t)kPass2Tile * p.d * sizeof(double) : 0;
  return (size_t)p.t2.nrows * (kPass2Tile / split) * sizeof(double2) +
         (rho <= kPass2RhoStage ? rho : 0) + comb;
}

int pass2_tiles(const ProbDev& p, int split) {
  const int tw = kPass2Tile / split;
  return (p.N + tw - 1) / tw;
}

int pass2_split(long long tiles_at_split1) {
  if (const char* env = getenv("CCO_PASS2_SPLIT")) {
    const int s = atoi(env);
    if (s == 1 || s == 2 || s == 4 || s == 8) return s;
  }
  int split = 1;
  while (split < 8 && tiles_at_split1 * split < kPass2TargetCtas) split *= 2;
  return split;
}

namespace {

template <int D, bool F32>
cudaError_t configure_d() {
  cudaError_t e = cudaFuncSetAttribute(k_pass1<D, F32>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024 - 1024);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_pass2<D, F32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              227 * 1024 - 1024);
}

template <int D, bool F32>
void launch_d(const EvalPlan& plan, bool pass2, cudaStream_t stream) {
  if (!pass2) {
    const int n = plan.d_off1[D] - plan.d_off1[D - 1];
    if (n > 0) k_pass1<D, F32><<<n, kPass1Threads, plan.smem1, stream>>>(plan);
  } else {
    const int n = plan.d_off2[D] - plan.d_off2[D - 1];
    if (n > 0) k_pass2<D, F32><<<n, kPass2Threads, F32 ? plan.smem2_f32 : plan.smem2, stream>>>(plan);
  }
}

}  // namespace

cudaError_t eval_configure() {
  cudaError_t e = configure_gemm<2>();
  if (e == cudaSuccess) e = configure_gemm<3>();
  if (e == cudaSuccess) e = configure_d<1, false>();
  if (e == cudaSuccess) e = configure_d<2, false>();
  if (e == cudaSuccess) e = configure_d<3, false>();
  if (e == cudaSuccess) e = configure_d<1, true>();
  if (e == cudaSuccess) e = configure_d<2, true>();
  if (e == cudaSuccess) e = configure_d<3, true>();
  return e;
}

namespace {

// The pass kernels of dimension D on stream s (pass 1: per-segment and GEMM forms).
// FP64 lanes run the F32 = false kernels whatever the plan; a plan that may
// hold FP32 lanes (dyn_prec) launches the F32 = true kernels as well.
void launch_dim(const EvalPlan& plan, bool pass2, int D, cudaStream_t s) {
  if (D == 1) {
    launch_d<1, false>(plan, pass2, s);
    if (plan.dyn_prec) launch_d<1, true>(plan, pass2, s);
  } else if (D == 2) {
    launch_d<2, false>(plan, pass2, s);
    if (plan.dyn_prec) launch_d<2, true>(plan, pass2, s);
    if (!pass2) launch_gemm<2>(plan, s);
  } else {
    launch_d<3, false>(plan, pass2, s);
    if (plan.dyn_prec) launch_d<3, true>(plan, pass2, s);
    if (!pass2) launch_gemm<3>(plan, s);
  }
}

// One pass over every dimension present: in order on `stream`, or, with side
// streams and more than one dimension, the first dimension on `stream` and the
// others on side streams forked from it and joined back before returning.
cudaError_t launch_pass_all(const EvalPlan& plan, bool pass2, cudaStream_t stream,
                            const EvalSide* side) {
  bool has[4] = {false, false, false, false};
  int nd = 0;
  for (int D = 1; D <= 3; ++D) {
    has[D] = pass2 ? plan.d_off2[D] > plan.d_off2[D - 1]
                   : (plan.d_off1[D] > plan.d_off1[D - 1] || plan.d_offG[D] > plan.d_offG[D - 1]);
    nd += has[D];
  }
  if (!side || nd < 2) {
    for (int D = 1; D <= 3; ++D)
      if (has[D]) launch_dim(plan, pass2, D, stream);
    return cudaGetLastError();
  }
  cudaError_t e = cudaEventRecord(side->fork, stream);
  cudaStream_t sd[4] = {stream, stream, stream, stream};
  int used = 0;
  bool first = true;
  for (int D = 1; D <= 3 && e == cudaSuccess; ++D) {
    if (!has[D]) continue;
    if (first) {
      first = false;
      continue;
    }
    sd[D] = side->aux[used++];
    e = cudaStreamWaitEvent(sd[D], side->fork, 0);
  }
  if (e != cudaSuccess) return e;
  for (int D = 1; D <= 3; ++D)
    if (has[D]) launch_dim(plan, pass2, D, sd[D]);
  for (int u = 0; u < used && e == cudaSuccess; ++u) {
    e = cudaEventRecord(side->join[u], side->aux[u]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(stream, side->join[u], 0);
  }
  return e == cudaSuccess ? cudaGetLastError() : e;
}

}  // namespace

cudaError_t eval_launch(const EvalPlan& plan, cudaStream_t stream, const EvalSide* side) {
  cudaError_t e = launch_pass_all(plan, false, stream, side);
  if (e != cudaSuccess) return e;
  if (plan.n_lanes > 0) {
    k_reduce<<<dim3(plan.red_chunks, plan.n_lanes), kReduceChunk, 0, stream>>>(plan);
    if (!plan.want_grad) k_energy<<<plan.n_lanes, 32, 0, stream>>>(plan);
  }
  if (plan.want_grad) {
    e = launch_pass_all(plan, true, stream, side);
    if (e != cudaSuccess) return e;
  }
  return cudaGetLastError();
}

cudaError_t rho_scatter(const double2* rho_run, const int* run2ref, int M, int batch,
                        size_t lane_stride, double* re, double* im, cudaStream_t stream) {
  const size_t total = (size_t)M * batch;
  int blocks = (int)((total + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  if (blocks < 1) blocks = 1;
  k_rho_scatter<<<blocks, 256, 0, stream>>>(rho_run, run2ref, M, batch, lane_stride, re, im);
  return cudaGetLastError();
}

}  // namespace cco
