// Stealthy energy, gradient and collective density on sm_100a (FP64).
//
// Reference math (src/xla_cco/energy.py:45-50,195-225,301-324):
//   rho_k  = sum_j exp(2 pi i n_k . s_j)
//   Phi    = (1/V) sum_k w_k |rho_k|^2
//   dPhi/ds_j = (2 (2 pi) / V) sum_k w_k (Im rho_k cos th_kj - Re rho_k sin th_kj) n_k
//
// B200 formulation. The k-set is stored as runs of consecutive last-axis n
// with a fixed prefix (n_0..n_{d-2}); along a run the phase advances by one
// complex multiply, exp(i th_{k+1,j}) = exp(i th_kj) z_j with
// z_j = exp(2 pi i s_{j,d-1}). A run start takes its phase from per-particle
// digit tables in shared memory: z_a^|n| = prod_l T_a,l[digit_l(|n|)], level 0
// built by products of z (<= base factors) and higher levels from FP64 sincospi
// of the exact exponent, so a phase carries O((base + run length) eps) error,
// well inside the reference's eps |theta| trig error. No theta matrix ever
// reaches HBM; HBM traffic per evaluation is s in, g out and the M-row
// density, so the kernels are FP64-pipe bound (SURVEY roofline).
//
//   pass 1 (k_pass1): CTA = (configuration, 128-particle tile). A thread owns
//     a segment of <= 8 rows and streams the tile's particles, accumulating
//     8 complex sums in registers (no cross-thread reduction). Small k-sets
//     split the particles into slices reduced in a fixed order. Output: one
//     partial density row per tile.
//   reduce  (k_reduce): sums the tile rows in tile order (deterministic),
//     forms rho, w rho and Phi (fixed-order block sum).
//   pass 2 (k_pass2): CTA = (configuration, 128-particle tile); a thread owns
//     2 particles and walks every segment (uniform across the CTA, density
//     reads are broadcasts): per row one complex multiply, the coefficient
//     w(Im rho cos - Re rho sin), and two FMA-class accumulations; prefix axes
//     are weighted once per segment.
#include <cstdio>

#include "cco_internal.cuh"

namespace cco {

namespace {

struct Rows {
  int r[3][kMaxLevels];
  int nlev[3];
};

template <int D>
__device__ __forceinline__ Rows load_rows(const ProbDev& P) {
  Rows R;
#pragma unroll
  for (int a = 0; a < D; ++a) {
    R.nlev[a] = P.nlev[a];
#pragma unroll
    for (int l = 0; l < kMaxLevels; ++l) R.r[a][l] = P.row[a][l];
  }
  return R;
}

// Digit tables of the tile's particles: row r holds one power of z_a for all
// tj particles (stride >= tj). Particles past nj get s = 0 and are never read
// back into a result.
template <int D>
__device__ void build_tables(const ProbDev& P, const double* __restrict__ s,
                             int j0, int nj, int tj, int stride, double2* tab) {
  for (int u = threadIdx.x; u < D * tj; u += blockDim.x) {
    const int a = u / tj, j = u - a * tj;
    const double sv = (j < nj) ? s[(size_t)(j0 + j) * D + a] : 0.0;
    double sn, cs;
    sincospi(2.0 * sv, &sn, &cs);
    const double2 z = make_double2(cs, sn);
    double2 p = make_double2(1.0, 0.0);
    const int r0 = P.row[a][0];
    const int n0 = P.nent[a][0];
    for (int e = 0; e < n0; ++e) {
      tab[(r0 + e) * stride + j] = p;
      p = cmul(p, z);
    }
    int scale = P.base[a];
    for (int l = 1; l < P.nlev[a]; ++l) {
      const int rl = P.row[a][l];
      const int nl = P.nent[a][l];
      for (int e = 0; e < nl; ++e) {
        const double t = (double)(e * scale) * sv;
        sincospi(2.0 * t, &sn, &cs);
        tab[(rl + e) * stride + j] = make_double2(cs, sn);
      }
      scale *= P.base[a];
    }
  }
}

// exp(2 pi i n . s_j) at a segment start, from the digit tables.
template <int D>
__device__ __forceinline__ double2 start_phase(const Rows& R, const SegHdr& h,
                                               const double2* tab, int stride, int j) {
  double2 ph = make_double2(1.0, 0.0);
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const int dg = h.dig[a];
    double2 f = tab[(R.r[a][0] + (dg & 255)) * stride + j];
#pragma unroll
    for (int l = 1; l < kMaxLevels; ++l) {
      if (l < R.nlev[a]) f = cmul(f, tab[(R.r[a][l] + ((dg >> (8 * l)) & 255)) * stride + j]);
    }
    if (dg >> 24) f.y = -f.y;
    ph = (a == 0) ? f : cmul(ph, f);
  }
  return ph;
}

template <int D>
__device__ void pass1_body(const ProbDev& P, const EvalLane& ln, int tile, double2* smem) {
  const int tj = kPass1Tile, stride = kPass1Tile + 1;
  const int j0 = tile * tj;
  const int nj = min(tj, P.N - j0);
  double2* tab = smem;
  build_tables<D>(P, ln.s, j0, nj, tj, stride, tab);
  const Rows R = load_rows<D>(P);
  __syncthreads();
  const int nseg = P.nseg1;
  int nslice = 1;
  while (2 * nslice * nseg <= (int)blockDim.x && 2 * nslice <= nj) nslice *= 2;
  const int units = nseg * nslice;
  double2* red = tab + (size_t)P.nrows * stride;
  const int zrow = R.r[D - 1][0] + 1;
  double2* out = ln.part + (size_t)tile * P.M;
  for (int u = threadIdx.x; u < units; u += blockDim.x) {
    const int sg = u % nseg, slice = u / nseg;
    const SegHdr h = P.seg1[sg];
    double2 acc[kSeg1Len];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) acc[i] = make_double2(0.0, 0.0);
    int j = slice;
    for (; j + nslice < nj; j += 2 * nslice) {
      const int jb = j + nslice;
      double2 pa = start_phase<D>(R, h, tab, stride, j);
      double2 pb = start_phase<D>(R, h, tab, stride, jb);
      const double2 za = tab[zrow * stride + j];
      const double2 zb = tab[zrow * stride + jb];
#pragma unroll
      for (int i = 0; i < kSeg1Len; ++i) {
        if (i < h.len) {
          acc[i].x += pa.x;
          acc[i].y += pa.y;
          acc[i].x += pb.x;
          acc[i].y += pb.y;
          pa = cmul(pa, za);
          pb = cmul(pb, zb);
        }
      }
    }
    if (j < nj) {
      double2 pa = start_phase<D>(R, h, tab, stride, j);
      const double2 za = tab[zrow * stride + j];
#pragma unroll
      for (int i = 0; i < kSeg1Len; ++i) {
        if (i < h.len) {
          acc[i].x += pa.x;
          acc[i].y += pa.y;
          pa = cmul(pa, za);
        }
      }
    }
    if (nslice == 1) {
#pragma unroll
      for (int i = 0; i < kSeg1Len; ++i)
        if (i < h.len) out[h.kstart + i] = acc[i];
    } else {
#pragma unroll
      for (int i = 0; i < kSeg1Len; ++i) red[((size_t)slice * nseg + sg) * kSeg1Len + i] = acc[i];
    }
  }
  if (nslice > 1) {
    __syncthreads();
    for (int v = threadIdx.x; v < nseg * kSeg1Len; v += blockDim.x) {
      const int sg = v / kSeg1Len, i = v - sg * kSeg1Len;
      const SegHdr h = P.seg1[sg];
      if (i < h.len) {
        double2 t = red[v];
        for (int q = 1; q < nslice; ++q) {
          const double2 o = red[(size_t)q * nseg * kSeg1Len + v];
          t.x += o.x;
          t.y += o.y;
        }
        out[h.kstart + i] = t;
      }
    }
  }
}

template <int D>
__device__ void pass2_body(const ProbDev& P, const EvalLane& ln, int tile, double2* tab) {
  constexpr int JB = kPass2PerThread;
  const int tj = kPass2Tile, stride = kPass2Tile;
  const int j0 = tile * tj;
  const int nj = min(tj, P.N - j0);
  build_tables<D>(P, ln.s, j0, nj, tj, stride, tab);
  const Rows R = load_rows<D>(P);
  __syncthreads();
  const int zrow = R.r[D - 1][0] + 1;
  int jl[JB];
  double2 z[JB];
  double G[JB][D];
#pragma unroll
  for (int b = 0; b < JB; ++b) {
    jl[b] = threadIdx.x + b * blockDim.x;
    z[b] = tab[zrow * stride + jl[b]];
#pragma unroll
    for (int a = 0; a < D; ++a) G[b][a] = 0.0;
  }
  const double2* __restrict__ rw = ln.rhow;
  for (int sg = 0; sg < P.nseg2; ++sg) {
    const SegHdr h = P.seg2[sg];
    double2 ph[JB];
    double S[JB], T[JB];
#pragma unroll
    for (int b = 0; b < JB; ++b) {
      ph[b] = start_phase<D>(R, h, tab, stride, jl[b]);
      S[b] = 0.0;
      T[b] = 0.0;
    }
    double nn = (double)h.n[D - 1];
    const double2* rk = rw + h.kstart;
    for (int i = 0; i < h.len; ++i) {
      const double2 r = __ldg(rk + i);
#pragma unroll
      for (int b = 0; b < JB; ++b) {
        const double c = r.y * ph[b].x - r.x * ph[b].y;
        S[b] += c;
        T[b] += c * nn;
        ph[b] = cmul(ph[b], z[b]);
      }
      nn += 1.0;
    }
#pragma unroll
    for (int b = 0; b < JB; ++b) {
#pragma unroll
      for (int a = 0; a < D - 1; ++a) G[b][a] += (double)h.n[a] * S[b];
      G[b][D - 1] += T[b];
    }
  }
#pragma unroll
  for (int b = 0; b < JB; ++b) {
    if (jl[b] < nj) {
      double* gj = ln.g + (size_t)(j0 + jl[b]) * D;
#pragma unroll
      for (int a = 0; a < D; ++a) gj[a] = P.gpref * G[b][a];
    }
  }
}

__global__ void __launch_bounds__(kPass1Threads) k_pass1(EvalPlan plan) {
  extern __shared__ double2 smem[];
  __shared__ ProbDev sp;
  const EvalItem it = plan.items1[blockIdx.x];
  const EvalLane ln = plan.lanes[it.lane];
  if (!lane_active(ln.status)) return;
  if (threadIdx.x == 0) sp = plan.probs[ln.prob];
  __syncthreads();
  switch (sp.d) {
    case 1: pass1_body<1>(sp, ln, it.tile, smem); break;
    case 2: pass1_body<2>(sp, ln, it.tile, smem); break;
    default: pass1_body<3>(sp, ln, it.tile, smem); break;
  }
}

__global__ void __launch_bounds__(256) k_reduce(EvalPlan plan) {
  __shared__ double red[32];
  const EvalLane ln = plan.lanes[blockIdx.x];
  if (!lane_active(ln.status)) return;
  const ProbDev& P = plan.probs[ln.prob];
  const int M = P.M, nt = P.ntile1;
  const double* __restrict__ w = P.w_run;
  double e = 0.0;
  for (int k = threadIdx.x; k < M; k += blockDim.x) {
    double2 t = ln.part[k];
    for (int q = 1; q < nt; ++q) {
      const double2 o = ln.part[(size_t)q * M + k];
      t.x += o.x;
      t.y += o.y;
    }
    ln.rho[k] = t;
    const double wk = w[k];
    ln.rhow[k] = make_double2(wk * t.x, wk * t.y);
    e += wk * (t.x * t.x + t.y * t.y);
  }
  e = block_sum(e, red);
  if (threadIdx.x == 0) *ln.f = e / P.vol;
}

__global__ void __launch_bounds__(kPass2Threads) k_pass2(EvalPlan plan) {
  extern __shared__ double2 smem[];
  __shared__ ProbDev sp;
  const EvalItem it = plan.items2[blockIdx.x];
  const EvalLane ln = plan.lanes[it.lane];
  if (!lane_active(ln.status) || ln.g == nullptr) return;
  if (threadIdx.x == 0) sp = plan.probs[ln.prob];
  __syncthreads();
  switch (sp.d) {
    case 1: pass2_body<1>(sp, ln, it.tile, smem); break;
    case 2: pass2_body<2>(sp, ln, it.tile, smem); break;
    default: pass2_body<3>(sp, ln, it.tile, smem); break;
  }
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

size_t eval_smem1(const ProbDev& p) {
  int nslice = 1;
  while (2 * nslice * p.nseg1 <= kPass1Threads && 2 * nslice <= kPass1Tile) nslice *= 2;
  size_t red = nslice > 1 ? (size_t)nslice * p.nseg1 * kSeg1Len : 0;
  return ((size_t)p.nrows * (kPass1Tile + 1) + red) * sizeof(double2);
}

size_t eval_smem2(const ProbDev& p) { return (size_t)p.nrows * kPass2Tile * sizeof(double2); }

cudaError_t eval_configure() {
  cudaError_t e = cudaFuncSetAttribute(k_pass1, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       227 * 1024 - 1024);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_pass2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              227 * 1024 - 1024);
}

cudaError_t eval_launch(const EvalPlan& plan, cudaStream_t stream) {
  if (plan.n_items1 > 0)
    k_pass1<<<plan.n_items1, kPass1Threads, plan.smem1, stream>>>(plan);
  if (plan.n_lanes > 0) k_reduce<<<plan.n_lanes, 256, 0, stream>>>(plan);
  if (plan.want_grad && plan.n_items2 > 0)
    k_pass2<<<plan.n_items2, kPass2Threads, plan.smem2, stream>>>(plan);
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
