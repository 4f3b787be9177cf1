// Minimum-image pair statistics of a batch of configurations: the pair
// distance histogram and the nearest-neighbour distances that the ground-state
// driver writes as g2 and Hp tables.
//
// Reference: src/xla_cco/analysis/pairs.py:41-128 (nearest_neighbor_distances,
// pair_distance_histogram) with the distance rule of _block_distances
// (:173-188): ds = s_j - s_i, ds -= round(ds), the 3^d image shifts of ds
// mapped through the basis, the smallest |r|^2, then sqrt; a particle's own
// zero shift is excluded. Binning follows np.histogram (_bin_counts,
// :191-199): bins are [e_k, e_k+1), the last one closed.
//
// Layout: one CTA per (row tile, column tile, configuration). The column
// tile's positions are staged in shared memory; each thread owns one row.
// The histogram keeps per-CTA bins in shared memory (32-bit) and adds them
// into the 64-bit result once, so the counts are exact and independent of
// the launch order.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <vector>

#include "cco.h"
#include "cco_host.cuh"

namespace cco {
namespace {

constexpr int kPairTile = 128;        // rows per CTA = columns per staged tile
constexpr int kSmemBins = 8192;       // bins kept in shared memory (32 KB)

struct PairGeom {
  double B[9];   // basis rows (lattice vectors), row-major d x d
  int n, n_bins;
};

template <int D>
__device__ __forceinline__ double min_image_r2(const double* si, const double* sj,
                                               const PairGeom& g, bool self) {
  double ds[D];
#pragma unroll
  for (int c = 0; c < D; ++c) {
    const double t = __dadd_rn(sj[c], -si[c]);
    ds[c] = __dadd_rn(t, -rint(t));
  }
  double best = INFINITY;
  constexpr int kShifts = D == 1 ? 3 : (D == 2 ? 9 : 27);
#pragma unroll
  for (int q = 0; q < kShifts; ++q) {
    int rem = q;
    double x[D];
    bool zero = true;
#pragma unroll
    for (int c = 0; c < D; ++c) {
      const int sh = rem % 3 - 1;
      rem /= 3;
      zero &= sh == 0;
      x[c] = __dadd_rn(ds[c], (double)sh);
    }
    if (self && zero) continue;
    double r2 = 0.0;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < D; ++c) v = __dadd_rn(v, __dmul_rn(x[c], g.B[c * D + a]));
      r2 = __dadd_rn(r2, __dmul_rn(v, v));
    }
    best = fmin(best, r2);
  }
  return best;
}

// np.histogram bin of r: (number of edges <= r) - 1; the last edge belongs
// to the last bin; -1 when outside [edges[0], edges[n_bins]] or not finite.
__device__ __forceinline__ int bin_of(double r, const double* __restrict__ edges, int n_bins) {
  if (!(r >= edges[0]) || !(r <= edges[n_bins])) return -1;
  if (r == edges[n_bins]) return n_bins - 1;
  int lo = 0, hi = n_bins;   // invariant: edges[lo] <= r < edges[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(edges + mid) <= r) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int D>
__global__ void __launch_bounds__(kPairTile) k_pair_hist(const double* __restrict__ s, PairGeom g,
                                                         const double* __restrict__ edges,
                                                         unsigned long long* counts, int tiles) {
  const int ti = blockIdx.x / tiles, tj = blockIdx.x % tiles;
  if (tj < ti) return;   // upper triangle of tiles: every pair i < j once
  extern __shared__ unsigned int bins[];
  __shared__ double col[kPairTile * D];
  const bool local = g.n_bins <= kSmemBins;
  if (local)
    for (int b = threadIdx.x; b < g.n_bins; b += blockDim.x) bins[b] = 0u;
  const double* sc = s + (size_t)blockIdx.y * g.n * D;
  const int j0 = tj * kPairTile;
  const int nj = min(kPairTile, g.n - j0);
  for (int u = threadIdx.x; u < nj * D; u += blockDim.x) col[u] = sc[(size_t)j0 * D + u];
  __syncthreads();
  const int i = ti * kPairTile + threadIdx.x;
  if (i < g.n) {
    double si[D];
#pragma unroll
    for (int c = 0; c < D; ++c) si[c] = sc[(size_t)i * D + c];
    for (int jj = 0; jj < nj; ++jj) {
      const int j = j0 + jj;
      if (j <= i) continue;
      const double r = sqrt(min_image_r2<D>(si, col + jj * D, g, false));
      const int b = bin_of(r, edges, g.n_bins);
      if (b < 0) continue;
      if (local) atomicAdd(bins + b, 1u);
      else atomicAdd(counts + b, 1ull);
    }
  }
  if (!local) return;
  __syncthreads();
  for (int b = threadIdx.x; b < g.n_bins; b += blockDim.x)
    if (bins[b]) atomicAdd(counts + b, (unsigned long long)bins[b]);
}

template <int D>
__global__ void __launch_bounds__(kPairTile) k_nearest(const double* __restrict__ s, PairGeom g,
                                                       double* __restrict__ out) {
  __shared__ double col[kPairTile * D];
  const double* sc = s + (size_t)blockIdx.y * g.n * D;
  const int i = blockIdx.x * kPairTile + threadIdx.x;
  double si[D];
#pragma unroll
  for (int c = 0; c < D; ++c) si[c] = i < g.n ? sc[(size_t)i * D + c] : 0.0;
  double best = INFINITY;
  for (int j0 = 0; j0 < g.n; j0 += kPairTile) {
    const int nj = min(kPairTile, g.n - j0);
    __syncthreads();
    for (int u = threadIdx.x; u < nj * D; u += blockDim.x) col[u] = sc[(size_t)j0 * D + u];
    __syncthreads();
    if (i < g.n)
      for (int jj = 0; jj < nj; ++jj)
        best = fmin(best, min_image_r2<D>(si, col + jj * D, g, j0 + jj == i));
  }
  if (i < g.n) out[(size_t)blockIdx.y * g.n + i] = sqrt(best);
}

int pair_args(int device, int batch, int n, int d, const double* s, const double* basis,
              PairGeom* g) {
  if (d < 1 || d > 3) return fail(CCO_ERR_ARG, "d must be 1, 2 or 3, got %d", d);
  if (batch < 1 || n < 1) return fail(CCO_ERR_ARG, "need batch >= 1 and n >= 1");
  if (batch > 65535) return fail(CCO_ERR_ARG, "batch %d above 65535: split it", batch);
  if (!s || !basis) return fail(CCO_ERR_ARG, "null positions or basis");
  int ndev = 0;
  if (cco_device_count(&ndev) != CCO_OK) return CCO_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return fail(CCO_ERR_ARG, "device %d out of range", device);
  *g = PairGeom{};
  for (int k = 0; k < d * d; ++k) {
    if (!std::isfinite(basis[k])) return fail(CCO_ERR_ARG, "non-finite basis entry %d", k);
    g->B[k] = basis[k];
  }
  g->n = n;
  return CCO_OK;
}

}  // namespace
}  // namespace cco

using namespace cco;

extern "C" {

int cco_pair_histogram(int device, void* stream, int batch, int n, int d, const double* s,
                       const double* basis, int n_edges, const double* edges, int64_t* counts) {
  PairGeom g;
  const int rc = pair_args(device, batch, n, d, s, basis, &g);
  if (rc != CCO_OK) return rc;
  if (n_edges < 2 || !edges || !counts) return fail(CCO_ERR_ARG, "need >= 2 edges and a counts array");
  for (int k = 0; k < n_edges; ++k) {
    if (!std::isfinite(edges[k]) || edges[k] < 0.0)
      return fail(CCO_ERR_ARG, "edges must be finite and non-negative");
    if (k > 0 && !(edges[k] > edges[k - 1])) return fail(CCO_ERR_ARG, "edges must be strictly increasing");
  }
  g.n_bins = n_edges - 1;
  DeviceGuard guard(device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* d_edges = nullptr;
  std::vector<double> he(edges, edges + n_edges);
  CCO_CUDA(upload(&d_edges, he, st));
  CCO_CUDA(cudaMemsetAsync(counts, 0, sizeof(int64_t) * g.n_bins, st));
  const int tiles = (n + kPairTile - 1) / kPairTile;
  const dim3 grid(tiles * tiles, batch);
  const size_t smem = g.n_bins <= kSmemBins ? sizeof(unsigned int) * g.n_bins : 0;
  auto* c = reinterpret_cast<unsigned long long*>(counts);
  if (d == 1) k_pair_hist<1><<<grid, kPairTile, smem, st>>>(s, g, d_edges, c, tiles);
  else if (d == 2) k_pair_hist<2><<<grid, kPairTile, smem, st>>>(s, g, d_edges, c, tiles);
  else k_pair_hist<3><<<grid, kPairTile, smem, st>>>(s, g, d_edges, c, tiles);
  CCO_CUDA(cudaGetLastError());
  CCO_CUDA(cudaFreeAsync(d_edges, st));
  return CCO_OK;
}

int cco_nearest_neighbor(int device, void* stream, int batch, int n, int d, const double* s,
                         const double* basis, double* out) {
  PairGeom g;
  const int rc = pair_args(device, batch, n, d, s, basis, &g);
  if (rc != CCO_OK) return rc;
  if (!out) return fail(CCO_ERR_ARG, "null output");
  DeviceGuard guard(device);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const dim3 grid((n + kPairTile - 1) / kPairTile, batch);
  if (d == 1) k_nearest<1><<<grid, kPairTile, 0, st>>>(s, g, out);
  else if (d == 2) k_nearest<2><<<grid, kPairTile, 0, st>>>(s, g, out);
  else k_nearest<3><<<grid, kPairTile, 0, st>>>(s, g, out);
  CCO_CUDA(cudaGetLastError());
  return CCO_OK;
}

}  // extern "C"
