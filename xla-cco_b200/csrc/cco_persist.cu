// cco_persist.cu - persistent relaxation of small problems: one CTA runs one
// lane's whole descent, evaluation and update, in a single launch.
//
// A tick of the graph driver (cco_relax.cu) is five to eight dependent kernel
// launches; for a problem of a few thousand (k, particle) pairs - the
// reference README's d=3 N=100 chi=0.05 relax has 1300 - their launch
// latency is the whole cost of an iteration. Here a CTA of 128 threads (the
// evaluation bodies' size) owns one lane and loops: pass 1 over the lane's
// particle tiles (per-segment or GEMM form), the tile-order reduction to rho,
// w rho and Phi, pass 2 over its tiles, and the descent update, with block
// barriers between the stages and no host round trip. Lanes never wait on
// one another, so there is no inter-CTA synchronization; the loop ends when
// the lane's status leaves RUNNING or after the same tick bound as the graph
// driver (then the launch reports an overrun, the host CCO_ERR_ROUNDS).
//
// Which path a lane takes depends on its problem alone (persist_eligible), so
// a lane relaxed alone and in any batch takes the same path and gives the
// same bits.
#include <cuda_runtime.h>

#include "cco_eval_bodies.cuh"
#include "cco_host.cuh"
#include "cco_internal.cuh"
#include "cco_opt_bodies.cuh"

namespace cco {

namespace {

constexpr int kPersistThreads = 128;   // kPass1Threads = kPass2Threads = kGemmThreads

// rho_k = sum over tiles of the pass-1 rows in tile order, w rho and Phi
// (one lane, the whole CTA; fixed-order block sum).
__device__ void persist_reduce(const ProbDev& P, const EvalLane& ln, double* red) {
  const int M = P.M, nt = P.ntile1;
  double e = 0.0;
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    double2 t = ln.part[k];
    for (int q = 1; q < nt; ++q) {
      const double2 o = ln.part[(size_t)q * M + k];
      t.x += o.x;
      t.y += o.y;
    }
    ln.rho[k] = t;
    const double wk = P.w_run[k];
    ln.rhow[k] = make_double2(wk * t.x, wk * t.y);
    e += wk * (t.x * t.x + t.y * t.y);
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) *ln.f = e / P.vol;
}

// Energy, gradient and density of the lane's probe positions (FP64).
template <int D>
__device__ void persist_eval(const ProbDev& P, const EvalLane& ln, double2* smem, double* red) {
  if constexpr (D >= 2) {
    if (P.gemm) {
      const int items = P.ntile1 * P.ngblk;
      for (int it = 0; it < items; ++it) {
        if constexpr (D == 2) pass1_gemm_d2(P, ln, it / P.ngblk, it % P.ngblk, smem);
        else pass1_gemm_d3(P, ln, it / P.ngblk, it % P.ngblk, smem);
        __syncthreads();
      }
    }
  }
  if (!P.gemm) {
    for (int t = 0; t < P.ntile1; ++t) {
      pass1_body<D>(P, ln, t, smem);
      __syncthreads();
    }
  }
  persist_reduce(P, ln, red);
  __syncthreads();
  const int nt2 = (P.N + kPass2Tile - 1) / kPass2Tile;
  for (int t = 0; t < nt2; ++t) {
    if constexpr (D == 1) {
      if ((size_t)P.M * sizeof(double2) <= kPass2RhoStage1D) pass2_body_1d<true>(P, ln, t, 1, smem);
      else pass2_body_1d<false>(P, ln, t, 1, smem);
    } else {
      if ((size_t)P.M * sizeof(double2) <= kPass2RhoStage) pass2_body<D, true>(P, ln, t, 1, smem);
      else pass2_body<D, false>(P, ln, t, 1, smem);
    }
    __syncthreads();
  }
}

// CTA i relaxes lane i of the table (lanes of another dimension leave at once).
template <int D>
__global__ void __launch_bounds__(kPersistThreads) k_persist_descent(DescentArgs a, EvalPlan plan,
                                                                     int64_t max_ticks,
                                                                     int* overrun) {
  extern __shared__ double2 smem[];
  __shared__ ProbDev sp;
  __shared__ double red[32];
  const int lane = blockIdx.x;
  const EvalLane ln = plan.lanes[lane];
  if (threadIdx.x == 0) sp = plan.probs[ln.prob];
  __syncthreads();
  if (sp.d != D) return;
  const LaneRef R = a.lanes[lane];
  for (int64_t t = 0;; ++t) {
    if (*rec_status(R.rec) != CCO_STATUS_RUNNING) break;   // written before the last barrier
    if (t >= max_ticks) {
      if (threadIdx.x == 0) atomicExch(overrun, 1);
      break;
    }
    persist_eval<D>(sp, ln, smem, red);
    __syncthreads();
    descent_update_lane(a, lane);
    __syncthreads();
  }
}

}  // namespace

bool persist_eligible(const cco_problem* p) {
  const double flops = (double)p->N * p->M * (p->d == 1 ? 7.0 : p->d == 2 ? 21.0 : 35.0);
  return flops <= kPersistMaxFlops && persist_smem(p) <= kPersistMaxSmem;
}

size_t persist_smem(const cco_problem* p) {
  size_t s = std::max(p->smem1, eval_smem2(p->host, 1));
  if (p->host.gemm) s = std::max(s, p->smemG);
  return s;
}

cudaError_t persist_descent(const DescentArgs& a, const EvalPlan& plan, size_t smem, int dims,
                            int64_t max_ticks, int* d_overrun, cudaStream_t st) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_persist_descent<1>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, kPersistMaxSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_persist_descent<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kPersistMaxSmem);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_persist_descent<3>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kPersistMaxSmem);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  if (dims & 1) k_persist_descent<1><<<a.B, kPersistThreads, smem, st>>>(a, plan, max_ticks, d_overrun);
  if (dims & 2) k_persist_descent<2><<<a.B, kPersistThreads, smem, st>>>(a, plan, max_ticks, d_overrun);
  if (dims & 4) k_persist_descent<3><<<a.B, kPersistThreads, smem, st>>>(a, plan, max_ticks, d_overrun);
  return cudaGetLastError();
}

}  // namespace cco
