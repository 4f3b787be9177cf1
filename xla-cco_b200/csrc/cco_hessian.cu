// cco_hessian.cu - closed-form Hessian of the stealthy energy on the device.
//
//   d2 Phi / ds_ja ds_lb = pref sum_k w_k n_ka n_kb [cos(th_kj - th_kl)
//                           - delta_jl (Re rho_k cos th_kj + Im rho_k sin th_kj)]
//   th_kj = 2 pi n_k . s_j,  pref = 2 (2 pi)^2 / V        (src/xla_cco/energy.py:272-299)
//
// The reference forms the (N, M) cos / sin matrices and two (N, M) x (M, N)
// products per (a, b). Here no (N, M) array exists: a CTA owns one tile pair
// (particles J x particles L, L >= J; the Hessian is symmetric, the lower
// tiles are written as mirrors), walks the k-set in chunks, forms the chunk's
// phases of both particle tiles in shared memory and accumulates
//   acc_ab[j][l] += q_kab (cos th_kj cos th_kl + sin th_kj sin th_kl),
//   q_kab = w_k n_ka n_kb   (a <= b; the (a, b) and (b, a) blocks are equal)
// in registers, 4 x 4 particle pairs per thread. The delta_jl term needs rho,
// which the evaluation kernels compute first; a second kernel subtracts it
// from the diagonal blocks.
//
// Phases use the argument n . s reduced exactly (fma products, compensated
// sum, nearest integer removed) before sincospi, so |n . s| in the thousands
// costs no accuracy.
#include <cuda_runtime.h>

#include "cco_host.cuh"
#include "cco_internal.cuh"

namespace cco {
namespace {

constexpr int kHessTile = 64;      // particles per tile side
constexpr int kHessK = 16;         // k rows per shared-memory chunk
constexpr int kHessThreads = 256;  // 16 x 16 threads, 4 x 4 particle pairs each

// (a, b) component pairs (a <= b) a CTA accumulates: group g of dimension D.
// D = 1: (0,0); D = 2: (0,0) (0,1) (1,1); D = 3: two groups of three.
template <int D>
struct Combos;
template <>
struct Combos<1> {
  static constexpr int kGroups = 1, kPer = 1;
  __device__ static void ab(int, int, int& a, int& b) { a = 0; b = 0; }
};
template <>
struct Combos<2> {
  static constexpr int kGroups = 1, kPer = 3;
  __device__ static void ab(int, int c, int& a, int& b) {
    a = c == 2 ? 1 : 0;
    b = c == 0 ? 0 : 1;
  }
};
template <>
struct Combos<3> {
  static constexpr int kGroups = 2, kPer = 3;
  __device__ static void ab(int g, int c, int& a, int& b) {
    // group 0: (0,0) (0,1) (0,2); group 1: (1,1) (1,2) (2,2)
    if (g == 0) { a = 0; b = c; }
    else { a = c == 2 ? 2 : 1; b = c == 0 ? 1 : 2; }
  }
};

// exp(2 pi i n . s) with n . s reduced exactly before the transcendental.
template <int D>
__device__ __forceinline__ double2 exact_phase(const double4& nk, const double* sj) {
  const double nv[3] = {nk.x, nk.y, nk.z};
  double sn, cs;
  sincos_2pi_dot<D>(nv, sj, &sn, &cs);
  return make_double2(cs, sn);
}

// Linear index over the upper triangle of T x T tile pairs -> (J, L), L >= J.
__device__ __forceinline__ void tile_pair(int t, int T, int& J, int& L) {
  J = 0;
  while (t >= T - J) {
    t -= T - J;
    ++J;
  }
  L = J + t;
}

template <int D>
__global__ void __launch_bounds__(kHessThreads, 1)
k_hess_tiles(const double* __restrict__ s, size_t s_stride, const double4* __restrict__ krow,
             int N, int M, double pref, double* __restrict__ H, size_t h_stride) {
  using C = Combos<D>;
  constexpr int NC = C::kPer;
  __shared__ double2 zj[kHessK][kHessTile];
  __shared__ double2 zl[kHessK][kHessTile];
  __shared__ double q[kHessK][NC];
  const int T = (N + kHessTile - 1) / kHessTile;
  int J, L;
  tile_pair(blockIdx.x, T, J, L);
  const int g = blockIdx.y, lane = blockIdx.z;
  const double* sl = s + (size_t)lane * s_stride;
  double* Hl = H + (size_t)lane * h_stride;
  const bool diag_tile = J == L;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  int ca[NC], cb[NC];
#pragma unroll
  for (int c = 0; c < NC; ++c) C::ab(g, c, ca[c], cb[c]);

  double acc[4][4][NC];
#pragma unroll
  for (int u = 0; u < 4; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int c = 0; c < NC; ++c) acc[u][v][c] = 0.0;

  const int fill = (diag_tile ? 1 : 2) * kHessK * kHessTile;
  for (int k0 = 0; k0 < M; k0 += kHessK) {
    __syncthreads();
    for (int idx = threadIdx.x; idx < fill; idx += kHessThreads) {
      const int which = idx / (kHessK * kHessTile);
      const int r = idx - which * (kHessK * kHessTile);
      const int kk = r / kHessTile, p = r - kk * kHessTile;
      const int k = k0 + kk, part = (which ? L : J) * kHessTile + p;
      double2 z = make_double2(0.0, 0.0);
      if (k < M && part < N) z = exact_phase<D>(krow[k], sl + (size_t)part * D);
      if (which) zl[kk][p] = z;
      else zj[kk][p] = z;
    }
    for (int idx = threadIdx.x; idx < kHessK * NC; idx += kHessThreads) {
      const int kk = idx / NC, c = idx - kk * NC;
      const int k = k0 + kk;
      double v = 0.0;
      if (k < M) {
        const double4 r = krow[k];
        const double nv[3] = {r.x, r.y, r.z};
        v = r.w * nv[ca[c]] * nv[cb[c]];
      }
      q[kk][c] = v;
    }
    __syncthreads();
    const double2(*zr)[kHessTile] = diag_tile ? zj : zl;
#pragma unroll 2
    for (int kk = 0; kk < kHessK; ++kk) {
      double2 a[4], b[4];
      double qc[NC];
#pragma unroll
      for (int u = 0; u < 4; ++u) a[u] = zj[kk][ty + 16 * u];
#pragma unroll
      for (int v = 0; v < 4; ++v) b[v] = zr[kk][tx + 16 * v];
#pragma unroll
      for (int c = 0; c < NC; ++c) qc[c] = q[kk][c];
#pragma unroll
      for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
          const double t = fma(a[u].x, b[v].x, a[u].y * b[v].y);
#pragma unroll
          for (int c = 0; c < NC; ++c) acc[u][v][c] = fma(qc[c], t, acc[u][v][c]);
        }
    }
  }
  const size_t nd = (size_t)N * D;
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    const int j = J * kHessTile + ty + 16 * u;
    if (j >= N) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      const int l = L * kHessTile + tx + 16 * v;
      if (l >= N) continue;
#pragma unroll
      for (int c = 0; c < NC; ++c) {
        const double val = pref * acc[u][v][c];
        const int a = ca[c], b = cb[c];
        Hl[(size_t)(j * D + a) * nd + l * D + b] = val;
        if (a != b) Hl[(size_t)(j * D + b) * nd + l * D + a] = val;
        if (!diag_tile) {
          Hl[(size_t)(l * D + b) * nd + j * D + a] = val;
          if (a != b) Hl[(size_t)(l * D + a) * nd + j * D + b] = val;
        }
      }
    }
  }
}

// Diagonal blocks: H[(j,a),(j,b)] -= pref sum_k q_kab (Re rho_k cos th_kj + Im rho_k sin th_kj).
// One thread per particle; rho is the evaluation's run-order density.
template <int D>
__global__ void k_hess_diag(const double* __restrict__ s, size_t s_stride,
                            const double4* __restrict__ krow, const double2* __restrict__ rho,
                            int N, int M, double pref, double* __restrict__ H, size_t h_stride) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x, lane = blockIdx.y;
  if (j >= N) return;
  const double* sj = s + (size_t)lane * s_stride + (size_t)j * D;
  const double2* rl = rho + (size_t)lane * M;
  double acc[D][D];
#pragma unroll
  for (int a = 0; a < D; ++a)
#pragma unroll
    for (int b = 0; b < D; ++b) acc[a][b] = 0.0;
  for (int k = 0; k < M; ++k) {
    const double4 r = krow[k];
    const double2 z = exact_phase<D>(r, sj);
    const double2 rh = rl[k];
    const double core = r.w * fma(rh.x, z.x, rh.y * z.y);
    const double nv[3] = {r.x, r.y, r.z};
#pragma unroll
    for (int a = 0; a < D; ++a)
#pragma unroll
      for (int b = a; b < D; ++b) acc[a][b] = fma(core * nv[a], nv[b], acc[a][b]);
  }
  const size_t nd = (size_t)N * D;
  double* Hl = H + (size_t)lane * h_stride;
#pragma unroll
  for (int a = 0; a < D; ++a)
#pragma unroll
    for (int b = a; b < D; ++b) {
      Hl[(size_t)(j * D + a) * nd + j * D + b] -= pref * acc[a][b];
      if (a != b) Hl[(size_t)(j * D + b) * nd + j * D + a] -= pref * acc[a][b];
    }
}

template <int D>
cudaError_t launch_hessian(const cco_problem* p, cudaStream_t st, int batch, const double* s,
                           const double2* rho, double* H) {
  const int N = p->N, M = p->M;
  const int T = (N + kHessTile - 1) / kHessTile;
  const size_t nd = (size_t)N * D;
  const double pref = 2.0 * (2.0 * M_PI) * (2.0 * M_PI) / p->host.vol;
  dim3 grid((unsigned)(T * (T + 1) / 2), Combos<D>::kGroups, (unsigned)batch);
  k_hess_tiles<D><<<grid, kHessThreads, 0, st>>>(s, nd, p->krow, N, M, pref, H, nd * nd);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  dim3 g2((unsigned)((N + 127) / 128), (unsigned)batch);
  k_hess_diag<D><<<g2, 128, 0, st>>>(s, nd, p->krow, rho, N, M, pref, H, nd * nd);
  return cudaGetLastError();
}

}  // namespace

cudaError_t hessian_launch(const cco_problem* p, cudaStream_t st, int batch, const double* s,
                           const double2* rho_run, double* H) {
  if (p->d == 1) return launch_hessian<1>(p, st, batch, s, rho_run, H);
  if (p->d == 2) return launch_hessian<2>(p, st, batch, s, rho_run, H);
  return launch_hessian<3>(p, st, batch, s, rho_run, H);
}

}  // namespace cco
