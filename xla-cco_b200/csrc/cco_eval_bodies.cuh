// Device bodies of the evaluation: phase tables, the pass-1 density (per
// segment and GEMM forms, FP64 and FP32) and the pass-2 gradient. Included
// by cco_eval.cu (the launched kernels) and cco_persist.cu (the persistent
// small-lane kernel); each file compiles its own copy.
#pragma once

#include "cco_internal.cuh"

namespace cco {

namespace {

template <int D>
struct Levels {
  int n[D];
};

template <int D>
__device__ __forceinline__ Levels<D> levels(const TabLayout& T) {
  Levels<D> L;
#pragma unroll
  for (int a = 0; a < D; ++a) L.n[a] = T.nlev[a];
  return L;
}

// Table entries (a, l, e) = z_a^(e base_a^l) of the tile's particles; units of
// up to 8 entries, each seeded by FP64 sincospi of the exact exponent. Level 0
// continues by products with z (error <= 8 eps), higher levels use one
// sincospi per entry. Particles past nj get s = 0 and are never read back.
__device__ __forceinline__ void put(double2* p, double2 v) { *p = v; }
__device__ __forceinline__ void put(float2* p, double2 v) {
  *p = make_float2((float)v.x, (float)v.y);
}

template <int D, class C>
__device__ void build_tables(const TabLayout& T, const double* __restrict__ s, int j0, int nj,
                             int tj, int stride, C* tab) {
  int units = 0;
#pragma unroll
  for (int a = 0; a < D; ++a)
    for (int l = 0; l < T.nlev[a]; ++l) units += (T.nent[a][l] + 7) >> 3;
  for (int u = threadIdx.x; u < units * tj; u += blockDim.x) {
    const int j = u % tj;
    int q = u / tj, a = 0, l = 0, scale = 1;
    for (;;) {
      const int c = (T.nent[a][l] + 7) >> 3;
      if (q < c) break;
      q -= c;
      scale *= T.base[a];
      if (++l >= T.nlev[a]) { l = 0; scale = 1; ++a; }
    }
    const double sv = (j < nj) ? s[(size_t)(j0 + j) * D + a] : 0.0;
    const int e0 = q * 8, e1 = min(e0 + 8, T.nent[a][l]);
    double sn, cs;
    C* out = tab + (size_t)T.row[a][l] * stride + j;
    if (l == 0) {
      sincospi(2.0 * sv, &sn, &cs);
      const double2 z = make_double2(cs, sn);
      sincos_2pi_ms((double)e0, sv, &sn, &cs);
      double2 p = make_double2(cs, sn);
      for (int e = e0; e < e1; ++e) {
        put(out + (size_t)e * stride, p);
        p = cmul(p, z);
      }
    } else {
      for (int e = e0; e < e1; ++e) {
        sincos_2pi_ms((double)(e * scale), sv, &sn, &cs);
        put(out + (size_t)e * stride, make_double2(cs, sn));
      }
    }
  }
}

// exp(2 pi i n . s_j) at a segment start, from the tables.
template <int D, class C>
__device__ __forceinline__ C start_phase(const Levels<D>& L, const SegHdr& h, const C* tab,
                                         int stride, int j) {
  C ph = tab[j];   // replaced at a = 0
#pragma unroll
  for (int a = 0; a < D; ++a) {
    const int dg = h.dig[a];
    C f = tab[(dg & 255) * stride + j];
    if (L.n[a] > 1) f = cmul(f, tab[((dg >> 8) & 255) * stride + j]);
    if (L.n[a] > 2) f = cmul(f, tab[((dg >> 16) & 255) * stride + j]);
    if (dg >> 24) f.y = -f.y;
    ph = (a == 0) ? f : cmul(ph, f);
  }
  return ph;
}

// Pass-1 accumulation of one segment over the particles j = j, j + ns, ...
// FULL: the segment has exactly kSeg1Len rows (no per-row predicate).
template <int D, bool FULL>
__device__ __forceinline__ void seg_sum(const Levels<D>& L, const SegHdr& h, const double2* tab,
                                        int zrow, int j, int ns, int nj, double2 (&acc)[kSeg1Len]) {
  constexpr int S = kPass1Stride;
  const int len = h.len;
  for (; j + 3 * ns < nj; j += 4 * ns) {
    double2 p0 = start_phase<D>(L, h, tab, S, j);
    double2 p1 = start_phase<D>(L, h, tab, S, j + ns);
    double2 p2 = start_phase<D>(L, h, tab, S, j + 2 * ns);
    double2 p3 = start_phase<D>(L, h, tab, S, j + 3 * ns);
    const double2 z0 = tab[zrow * S + j], z1 = tab[zrow * S + j + ns];
    const double2 z2 = tab[zrow * S + j + 2 * ns], z3 = tab[zrow * S + j + 3 * ns];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) {
      if (FULL || i < len) {
        acc[i].x += (p0.x + p1.x) + (p2.x + p3.x);
        acc[i].y += (p0.y + p1.y) + (p2.y + p3.y);
        p0 = cmul(p0, z0);
        p1 = cmul(p1, z1);
        p2 = cmul(p2, z2);
        p3 = cmul(p3, z3);
      }
    }
  }
  for (; j < nj; j += ns) {
    double2 p0 = start_phase<D>(L, h, tab, S, j);
    const double2 z0 = tab[zrow * S + j];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) {
      if (FULL || i < len) {
        acc[i].x += p0.x;
        acc[i].y += p0.y;
        p0 = cmul(p0, z0);
      }
    }
  }
}

// Chunk c of C covers the segments [c nseg / C, (c + 1) nseg / C) (C > 1 only
// when nseg >= 2 kPass1ChunkSegs, where ns = 1).
template <int D>
__device__ void pass1_body(const ProbDev& P, const EvalLane& ln, int tile, double2* tab,
                           int chunk = 0, int chunks = 1) {
  const TabLayout& T = P.t1;
  const int j0 = tile * kPass1Tile;
  const int nj = min(kPass1Tile, P.N - j0);
  build_tables<D>(T, ln.s, j0, nj, kPass1Tile, kPass1Stride, tab);
  const Levels<D> L = levels<D>(T);
  const int zrow = T.zrow;
  __syncthreads();
  const int nseg = P.nseg1;
  int ns = 1;
  while (2 * ns * nseg <= (int)blockDim.x && 2 * ns <= nj) ns *= 2;
  const int seg_lo = (int)((long long)chunk * nseg / chunks);
  const int seg_hi = (int)((long long)(chunk + 1) * nseg / chunks);
  const int nsc = seg_hi - seg_lo;
  const int units = nsc * ns;
  double2* red = tab + (size_t)T.nrows * kPass1Stride;
  double2* out = ln.part + (size_t)tile * P.M;
  for (int u = threadIdx.x; u < units; u += blockDim.x) {
    const int sg = seg_lo + u % nsc, slice = u / nsc;
    const SegHdr h = P.seg1[sg];
    double2 acc[kSeg1Len];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) acc[i] = make_double2(0.0, 0.0);
    if (h.len == kSeg1Len)
      seg_sum<D, true>(L, h, tab, zrow, slice, ns, nj, acc);
    else
      seg_sum<D, false>(L, h, tab, zrow, slice, ns, nj, acc);
    if (ns == 1) {
#pragma unroll
      for (int i = 0; i < kSeg1Len; ++i)
        if (i < h.len) out[h.kstart + i] = acc[i];
    } else {
#pragma unroll
      for (int i = 0; i < kSeg1Len; ++i) red[((size_t)slice * nseg + sg) * kSeg1Len + i] = acc[i];
    }
  }
  if (ns > 1) {
    __syncthreads();
    for (int v = threadIdx.x; v < nseg * kSeg1Len; v += blockDim.x) {
      const int sg = v / kSeg1Len, i = v - sg * kSeg1Len;
      const SegHdr h = P.seg1[sg];
      if (i < h.len) {
        double2 t = red[v];
        for (int q = 1; q < ns; ++q) {
          const double2 o = red[(size_t)q * nseg * kSeg1Len + v];
          t.x += o.x;
          t.y += o.y;
        }
        out[h.kstart + i] = t;
      }
    }
  }
}

// One row of the back-projection for one chain.
__device__ __forceinline__ void bp_step(double2 r, double2& ph, double2 z, double di, double& S,
                                        double& Tn) {
  const double c = r.y * ph.x - r.x * ph.y;
  S += c;
  Tn += c * di;
  ph = cmul(ph, z);
}

// Pairwise (tree) sum of D-vectors pushed in order: push i merges with the
// partial sums of its completed subtrees, so a power-of-two count n of
// leaves always sums as the same balanced tree, whichever threads produced
// the leaves. Depth <= 4 (16 leaves).
template <int D>
struct Pairwise {
  double st[4][D];
  int n = 0;
  __device__ __forceinline__ void push(const double (&v)[D]) {
    double cur[D];
#pragma unroll
    for (int a = 0; a < D; ++a) cur[a] = v[a];
    int lvl = 0;
    for (int c = n; c & 1; c >>= 1, ++lvl) {
#pragma unroll
      for (int a = 0; a < D; ++a) cur[a] = st[lvl][a] + cur[a];
    }
#pragma unroll
    for (int a = 0; a < D; ++a) st[lvl][a] = cur[a];
    ++n;
  }
  // total of a power-of-two count of leaves
  __device__ __forceinline__ void total(double (&out)[D]) const {
    int lvl = 0;
    while ((1 << lvl) < n) ++lvl;
#pragma unroll
    for (int a = 0; a < D; ++a) out[a] = st[lvl][a];
  }
};

// One row of the back-projection for one chain in prefix form: S += c and
// Q += S, so that after an L-row segment sum_i i c_i = L S - Q. This takes one
// FP64 add per row where the direct form (T += c i) needs an FMA plus the
// row index's own increments.
__device__ __forceinline__ void bp_stepq(double2 r, double2& ph, double2 z, double& S,
                                         double& Q) {
  const double c = r.y * ph.x - r.x * ph.y;
  S += c;
  Q += S;
  ph = cmul(ph, z);
}

// Gradient contribution of logical slice q: segment pairs q, q + sl, ...
template <int D>
__device__ __forceinline__ void pass2_slice(const ProbDev& P, const Levels<D>& L,
                                            const double2* __restrict__ rw, const double2* tab,
                                            int stride, int j, double2 z, int q, int sl,
                                            double (&G)[D]) {
  const int nseg = P.nseg2;
#pragma unroll
  for (int a = 0; a < D; ++a) G[a] = 0.0;
  for (int sg = 2 * q; sg < nseg; sg += 2 * sl) {
    const SegHdr hA = P.seg2[sg];
    const SegHdr hB = P.seg2[min(sg + 1, nseg - 1)];
    double2 pA = start_phase<D>(L, hA, tab, stride, j);
    double2 pB = start_phase<D>(L, hB, tab, stride, j);
    double SA = 0.0, QA = 0.0, SB = 0.0, QB = 0.0;
    const double2* rA = rw + hA.kstart;
    const double2* rB = rw + hB.kstart;
    // la >= lb (segments sorted by length); an odd last segment pairs with nothing
    const int la = hA.len, lb = (sg + 1 < nseg) ? hB.len : 0;
    int i = 0;
    for (; i + 2 <= lb; i += 2) {
      const double2 a0 = rA[i], a1 = rA[i + 1];
      const double2 b0 = rB[i], b1 = rB[i + 1];
      bp_stepq(a0, pA, z, SA, QA);
      bp_stepq(b0, pB, z, SB, QB);
      bp_stepq(a1, pA, z, SA, QA);
      bp_stepq(b1, pB, z, SB, QB);
    }
    if (i < lb) {
      bp_stepq(rA[i], pA, z, SA, QA);
      bp_stepq(rB[i], pB, z, SB, QB);
      ++i;
    }
    for (; i + 2 <= la; i += 2) {
      const double2 a0 = rA[i], a1 = rA[i + 1];
      bp_stepq(a0, pA, z, SA, QA);
      bp_stepq(a1, pA, z, SA, QA);
    }
    if (i < la) bp_stepq(rA[i], pA, z, SA, QA);
    // the last axis: sum over rows of (n_start + i) c_i = (n_start + L) S - Q
#pragma unroll
    for (int a = 0; a < D - 1; ++a) G[a] += (double)hA.n[a] * SA + (double)hB.n[a] * SB;
    G[D - 1] += ((double)(hA.n[D - 1] + la) * SA - QA) + ((double)(hB.n[D - 1] + lb) * SB - QB);
  }
}

// Pass 2 of one particle tile. The segment pairs of a problem form P.sl2
// logical slices (slice q: pairs q, q + sl2, ...) whose gradients are summed
// as a balanced tree, so the result depends on the problem alone. `split`
// (a launch choice) sets how many threads share one particle: a CTA holds
// kPass2Tile / split particles and each of a particle's split threads
// evaluates a contiguous block of slices; the tree's top levels are then
// finished in shared memory. STAGED: the lane's weighted density (M rows) is
// copied once into shared memory after the tables and every row read is a
// shared-memory broadcast; otherwise rows are read through L1.
template <int D, bool STAGED>
__device__ void pass2_body(const ProbDev& P, const EvalLane& ln, int tile, int split,
                           double2* tab) {
  const TabLayout& T = P.t2;
  const int tw = kPass2Tile / split;
  const int j0 = tile * tw;
  const int nj = min(tw, P.N - j0);
  const double2* __restrict__ rw = ln.rhow;
  double2* after = tab + (size_t)T.nrows * tw;
  if (STAGED) {
    for (int k = threadIdx.x; k < P.M; k += blockDim.x) after[k] = rw[k];
    rw = after;
    after += P.M;
  }
  double* comb = reinterpret_cast<double*>(after);   // [split][tw][D]
  build_tables<D>(T, ln.s, j0, nj, tw, tw, tab);
  const Levels<D> L = levels<D>(T);
  __syncthreads();
  const int j = threadIdx.x % tw, qp = threadIdx.x / tw;
  const double2 z = tab[T.zrow * tw + j];
  const int sl = P.sl2;
  const int per = sl > split ? sl / split : 1;    // slices per thread
  const int nblk = sl / per;                      // threads of a particle that have slices
  if (qp < nblk) {
    Pairwise<D> acc;
    for (int q = qp * per; q < (qp + 1) * per; ++q) {
      double G[D];
      pass2_slice<D>(P, L, rw, tab, tw, j, z, q, sl, G);
      acc.push(G);
    }
    double G[D];
    acc.total(G);
    if (nblk > 1) {
#pragma unroll
      for (int a = 0; a < D; ++a) comb[((size_t)qp * tw + j) * D + a] = G[a];
    } else if (j < nj) {
      double* gj = ln.g + (size_t)(j0 + j) * D;
#pragma unroll
      for (int a = 0; a < D; ++a) gj[a] = P.gpref * G[a];
    }
  }
  if (nblk > 1) {
    __syncthreads();
    if (qp == 0 && j < nj) {
      Pairwise<D> acc;
      for (int b = 0; b < nblk; ++b) {
        double G[D];
#pragma unroll
        for (int a = 0; a < D; ++a) G[a] = comb[((size_t)b * tw + j) * D + a];
        acc.push(G);
      }
      double G[D];
      acc.total(G);
      double* gj = ln.g + (size_t)(j0 + j) * D;
#pragma unroll
      for (int a = 0; a < D; ++a) gj[a] = P.gpref * G[a];
    }
  }
}

// ------------------------------------------------------------ 1-D pass 2
// A 1-D k-set is one run n = n_min, n_min + 1, ... (1..M without K1), cut into
// segments of <= kSeg2Len rows. Each thread seeds a segment's phase z_j^n0
// directly (one exactly reduced sincospi per segment and particle, ~2% of the
// row work at M = 2000) and walks the rows by products with z_j, so the pass
// needs no phase tables and the whole weighted density is staged in shared
// memory (broadcast reads) for M <= kPass2RhoStage1D / 16.
__device__ __forceinline__ void pass2_slice_1d(const ProbDev& P, const double2* __restrict__ rw,
                                               double sj, double2 z, int q, int sl, double& G) {
  const int nseg = P.nseg2;
  G = 0.0;
  for (int sg = 2 * q; sg < nseg; sg += 2 * sl) {
    const SegHdr hA = P.seg2[sg];
    const SegHdr hB = P.seg2[min(sg + 1, nseg - 1)];
    double sn, cs;
    sincos_2pi_ms((double)hA.n[0], sj, &sn, &cs);
    double2 pA = make_double2(cs, sn);
    sincos_2pi_ms((double)hB.n[0], sj, &sn, &cs);
    double2 pB = make_double2(cs, sn);
    double SA = 0.0, TA = 0.0, SB = 0.0, TB = 0.0;
    const double2* rA = rw + hA.kstart;
    const double2* rB = rw + hB.kstart;
    const int la = hA.len, lb = (sg + 1 < nseg) ? hB.len : 0;
    int i = 0;
    double di = 0.0;
    for (; i + 2 <= lb; i += 2) {
      const double2 a0 = rA[i], a1 = rA[i + 1];
      const double2 b0 = rB[i], b1 = rB[i + 1];
      bp_step(a0, pA, z, di, SA, TA);
      bp_step(b0, pB, z, di, SB, TB);
      bp_step(a1, pA, z, di + 1.0, SA, TA);
      bp_step(b1, pB, z, di + 1.0, SB, TB);
      di += 2.0;
    }
    if (i < lb) {
      bp_step(rA[i], pA, z, di, SA, TA);
      bp_step(rB[i], pB, z, di, SB, TB);
      ++i;
      di += 1.0;
    }
    for (; i + 2 <= la; i += 2) {
      const double2 a0 = rA[i], a1 = rA[i + 1];
      bp_step(a0, pA, z, di, SA, TA);
      bp_step(a1, pA, z, di + 1.0, SA, TA);
      di += 2.0;
    }
    if (i < la) bp_step(rA[i], pA, z, di, SA, TA);
    G += ((double)hA.n[0] * SA + TA) + ((double)hB.n[0] * SB + TB);
  }
}

// Pass 2 of one particle tile of a 1-D problem (FP64): the slices and their
// tree sum as in pass2_body, the phases from pass2_slice_1d.
template <bool STAGED>
__device__ void pass2_body_1d(const ProbDev& P, const EvalLane& ln, int tile, int split,
                              double2* smem) {
  const int tw = kPass2Tile / split;
  const int j0 = tile * tw;
  const int nj = min(tw, P.N - j0);
  const double2* __restrict__ rw = ln.rhow;
  double2* after = smem;
  if (STAGED) {
    for (int k = threadIdx.x; k < P.M; k += blockDim.x) after[k] = rw[k];
    rw = after;
    after += P.M;
  }
  double* comb = reinterpret_cast<double*>(after);   // [split][tw]
  __syncthreads();
  const int j = threadIdx.x % tw, qp = threadIdx.x / tw;
  const double sj = (j < nj) ? ln.s[j0 + j] : 0.0;
  double sn, cs;
  sincospi(2.0 * sj, &sn, &cs);
  const double2 z = make_double2(cs, sn);
  const int sl = P.sl2;
  const int per = sl > split ? sl / split : 1;
  const int nblk = sl / per;
  if (qp < nblk) {
    Pairwise<1> acc;
    for (int q = qp * per; q < (qp + 1) * per; ++q) {
      double G[1];
      pass2_slice_1d(P, rw, sj, z, q, sl, G[0]);
      acc.push(G);
    }
    double G[1];
    acc.total(G);
    if (nblk > 1) comb[(size_t)qp * tw + j] = G[0];
    else if (j < nj) ln.g[j0 + j] = P.gpref * G[0];
  }
  if (nblk > 1) {
    __syncthreads();
    if (qp == 0 && j < nj) {
      Pairwise<1> acc;
      for (int b = 0; b < nblk; ++b) {
        double G[1] = {comb[(size_t)b * tw + j]};
        acc.push(G);
      }
      double G[1];
      acc.total(G);
      ln.g[j0 + j] = P.gpref * G[0];
    }
  }
}

// ------------------------------------------------------------ FP32 bodies
// Kahan-compensated FP32 complex accumulation: s holds the sum, c minus the
// low-order part lost so far (value = s - c).
__device__ __forceinline__ void kahan_add(float2& s, float2& c, float2 v) {
  const float yx = v.x - c.x, yy = v.y - c.y;
  const float tx = s.x + yx, ty = s.y + yy;
  c.x = (tx - s.x) - yx;
  c.y = (ty - s.y) - yy;
  s.x = tx;
  s.y = ty;
}

template <int D, bool FULL>
__device__ __forceinline__ void seg_sum_f32(const Levels<D>& L, const SegHdr& h, const float2* tab,
                                            int zrow, int j, int ns, int nj,
                                            float2 (&acc)[kSeg1Len], float2 (&cmp)[kSeg1Len]) {
  constexpr int S = kPass1Stride;
  const int len = h.len;
  for (; j + 3 * ns < nj; j += 4 * ns) {
    float2 p0 = start_phase<D>(L, h, tab, S, j);
    float2 p1 = start_phase<D>(L, h, tab, S, j + ns);
    float2 p2 = start_phase<D>(L, h, tab, S, j + 2 * ns);
    float2 p3 = start_phase<D>(L, h, tab, S, j + 3 * ns);
    const float2 z0 = tab[zrow * S + j], z1 = tab[zrow * S + j + ns];
    const float2 z2 = tab[zrow * S + j + 2 * ns], z3 = tab[zrow * S + j + 3 * ns];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) {
      if (FULL || i < len) {
        kahan_add(acc[i], cmp[i],
                  make_float2((p0.x + p1.x) + (p2.x + p3.x), (p0.y + p1.y) + (p2.y + p3.y)));
        p0 = cmul(p0, z0);
        p1 = cmul(p1, z1);
        p2 = cmul(p2, z2);
        p3 = cmul(p3, z3);
      }
    }
  }
  for (; j < nj; j += ns) {
    float2 p0 = start_phase<D>(L, h, tab, S, j);
    const float2 z0 = tab[zrow * S + j];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) {
      if (FULL || i < len) {
        kahan_add(acc[i], cmp[i], p0);
        p0 = cmul(p0, z0);
      }
    }
  }
}

// Pass 1 in FP32 (same decomposition as pass1_body); partial rows leave in FP64.
template <int D>
__device__ void pass1_body_f32(const ProbDev& P, const EvalLane& ln, int tile, double2* smem) {
  const TabLayout& T = P.t1;
  float2* tab = reinterpret_cast<float2*>(smem);
  const int j0 = tile * kPass1Tile;
  const int nj = min(kPass1Tile, P.N - j0);
  build_tables<D>(T, ln.s, j0, nj, kPass1Tile, kPass1Stride, tab);
  const Levels<D> L = levels<D>(T);
  const int zrow = T.zrow;
  __syncthreads();
  const int nseg = P.nseg1;
  int ns = 1;
  while (2 * ns * nseg <= (int)blockDim.x && 2 * ns <= nj) ns *= 2;
  const int units = nseg * ns;
  // slice partials after the tables, on a 16-byte boundary
  double2* red = smem + ((size_t)T.nrows * kPass1Stride + 1) / 2;
  double2* out = ln.part + (size_t)tile * P.M;
  for (int u = threadIdx.x; u < units; u += blockDim.x) {
    const int sg = u % nseg, slice = u / nseg;
    const SegHdr h = P.seg1[sg];
    float2 acc[kSeg1Len], cmp[kSeg1Len];
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) {
      acc[i] = make_float2(0.f, 0.f);
      cmp[i] = make_float2(0.f, 0.f);
    }
    if (h.len == kSeg1Len)
      seg_sum_f32<D, true>(L, h, tab, zrow, slice, ns, nj, acc, cmp);
    else
      seg_sum_f32<D, false>(L, h, tab, zrow, slice, ns, nj, acc, cmp);
#pragma unroll
    for (int i = 0; i < kSeg1Len; ++i) {
      const double2 v = make_double2((double)acc[i].x - (double)cmp[i].x,
                                     (double)acc[i].y - (double)cmp[i].y);
      if (ns == 1) {
        if (i < h.len) out[h.kstart + i] = v;
      } else {
        red[((size_t)slice * nseg + sg) * kSeg1Len + i] = v;
      }
    }
  }
  if (ns > 1) {
    __syncthreads();
    for (int v = threadIdx.x; v < nseg * kSeg1Len; v += blockDim.x) {
      const int sg = v / kSeg1Len, i = v - sg * kSeg1Len;
      const SegHdr h = P.seg1[sg];
      if (i < h.len) {
        double2 t = red[v];
        for (int q = 1; q < ns; ++q) {
          const double2 o = red[(size_t)q * nseg * kSeg1Len + v];
          t.x += o.x;
          t.y += o.y;
        }
        out[h.kstart + i] = t;
      }
    }
  }
}

__device__ __forceinline__ void bp_step_f32(float2 r, float2& ph, float2 z, float di, float& S,
                                            float& Tn) {
  const float c = r.y * ph.x - r.x * ph.y;
  S += c;
  Tn += c * di;
  ph = cmul(ph, z);
}

// Slice q of pass 2 in FP32: each segment's sums S, T (<= 256 rows) in FP32,
// folded into the FP64 gradient once per segment.
template <int D>
__device__ __forceinline__ void pass2_slice_f32(const ProbDev& P, const Levels<D>& L,
                                                const float2* __restrict__ rw, const float2* tab,
                                                int stride, int j, float2 z, int q, int sl,
                                                double (&G)[D]) {
  const int nseg = P.nseg2;
#pragma unroll
  for (int a = 0; a < D; ++a) G[a] = 0.0;
  for (int sg = 2 * q; sg < nseg; sg += 2 * sl) {
    const SegHdr hA = P.seg2[sg];
    const SegHdr hB = P.seg2[min(sg + 1, nseg - 1)];
    float2 pA = start_phase<D>(L, hA, tab, stride, j);
    float2 pB = start_phase<D>(L, hB, tab, stride, j);
    float SA = 0.f, TA = 0.f, SB = 0.f, TB = 0.f;
    const float2* rA = rw + hA.kstart;
    const float2* rB = rw + hB.kstart;
    const int la = hA.len, lb = (sg + 1 < nseg) ? hB.len : 0;
    int i = 0;
    float di = 0.f;
    for (; i + 2 <= lb; i += 2) {
      const float2 a0 = rA[i], a1 = rA[i + 1];
      const float2 b0 = rB[i], b1 = rB[i + 1];
      bp_step_f32(a0, pA, z, di, SA, TA);
      bp_step_f32(b0, pB, z, di, SB, TB);
      bp_step_f32(a1, pA, z, di + 1.f, SA, TA);
      bp_step_f32(b1, pB, z, di + 1.f, SB, TB);
      di += 2.f;
    }
    if (i < lb) {
      bp_step_f32(rA[i], pA, z, di, SA, TA);
      bp_step_f32(rB[i], pB, z, di, SB, TB);
      ++i;
      di += 1.f;
    }
    for (; i + 2 <= la; i += 2) {
      const float2 a0 = rA[i], a1 = rA[i + 1];
      bp_step_f32(a0, pA, z, di, SA, TA);
      bp_step_f32(a1, pA, z, di + 1.f, SA, TA);
      di += 2.f;
    }
    if (i < la) bp_step_f32(rA[i], pA, z, di, SA, TA);
#pragma unroll
    for (int a = 0; a < D - 1; ++a) G[a] += (double)hA.n[a] * SA + (double)hB.n[a] * SB;
    G[D - 1] += ((double)hA.n[D - 1] * SA + TA) + ((double)hB.n[D - 1] * SB + TB);
  }
}

// Pass 2 in FP32 (decomposition of pass2_body). The weighted density of an
// FP32 lane is an FP32 array (written by the reduction over the lane's FP64
// w rho buffer).
template <int D, bool STAGED>
__device__ void pass2_body_f32(const ProbDev& P, const EvalLane& ln, int tile, int split,
                               double2* smem) {
  const TabLayout& T = P.t2;
  float2* tab = reinterpret_cast<float2*>(smem);
  const int tw = kPass2Tile / split;
  const int j0 = tile * tw;
  const int nj = min(tw, P.N - j0);
  const float2* __restrict__ rw = reinterpret_cast<const float2*>(ln.rhow);
  float2* after = tab + (size_t)T.nrows * tw;
  if (STAGED) {
    for (int k = threadIdx.x; k < P.M; k += blockDim.x) after[k] = rw[k];
    rw = after;
    after += P.M;
  }
  double* comb = reinterpret_cast<double*>(after + ((after - tab) & 1));   // 8-byte aligned
  build_tables<D>(T, ln.s, j0, nj, tw, tw, tab);
  const Levels<D> L = levels<D>(T);
  __syncthreads();
  const int j = threadIdx.x % tw, qp = threadIdx.x / tw;
  const float2 z = tab[T.zrow * tw + j];
  const int sl = P.sl2;
  const int per = sl > split ? sl / split : 1;
  const int nblk = sl / per;
  if (qp < nblk) {
    Pairwise<D> acc;
    for (int q = qp * per; q < (qp + 1) * per; ++q) {
      double G[D];
      pass2_slice_f32<D>(P, L, rw, tab, tw, j, z, q, sl, G);
      acc.push(G);
    }
    double G[D];
    acc.total(G);
    if (nblk > 1) {
#pragma unroll
      for (int a = 0; a < D; ++a) comb[((size_t)qp * tw + j) * D + a] = G[a];
    } else if (j < nj) {
      double* gj = ln.g + (size_t)(j0 + j) * D;
#pragma unroll
      for (int a = 0; a < D; ++a) gj[a] = P.gpref * G[a];
    }
  }
  if (nblk > 1) {
    __syncthreads();
    if (qp == 0 && j < nj) {
      Pairwise<D> acc;
      for (int b = 0; b < nblk; ++b) {
        double G[D];
#pragma unroll
        for (int a = 0; a < D; ++a) G[a] = comb[((size_t)b * tw + j) * D + a];
        acc.push(G);
      }
      double G[D];
      acc.total(G);
      double* gj = ln.g + (size_t)(j0 + j) * D;
#pragma unroll
      for (int a = 0; a < D; ++a) gj[a] = P.gpref * G[a];
    }
  }
}

// ------------------------------------------------------------ GEMM pass 1
// Powers dst[e] = exp(2 pi i (base + e) s) for e in [e0, e0 + cnt): FP64
// sincospi of the exact exponent at e0, products with z = exp(2 pi i s) after it.
__device__ __forceinline__ void fill_powers(double2* dst, int e0, int cnt, int base, double s,
                                            double2 z) {
  double sn, cs;
  sincos_2pi_ms((double)(base + e0), s, &sn, &cs);
  double2 p = make_double2(cs, sn);
  for (int e = 0; e < cnt; ++e) {
    dst[e0 + e] = p;
    p = cmul(p, z);
  }
}

// z = exp(2 pi i s) per (particle, axis) of the chunk starting at particle jb.
template <int D>
__device__ __forceinline__ void chunk_roots(double2* zs, const double* s, int jb, int kc) {
  for (int u = threadIdx.x; u < kGemmChunk * D; u += blockDim.x) {
    const int j = u / D;
    double sn = 0.0, cs = 1.0;
    if (j < kc) sincospi(2.0 * s[(size_t)jb * D + u], &sn, &cs);
    zs[u] = make_double2(cs, sn);
  }
}

// The outputs of a folded block: cell (run 3 tr + i, column lo + tn + 16 q)
// holds C(c) = (P1 - P2) + i (P3 + P4) and C(-c) = (P1 + P2) + i (P4 - P3);
// each lands in its run's row if the run contains that n.
template <int CQ>
__device__ __forceinline__ void gemm_fold_store(const ProbDev& P, const EvalLane& ln, int tile,
                                                const GemmBlock& B, int tr, int tn,
                                                const double (&p1)[3][CQ],
                                                const double (&p2)[3][CQ],
                                                const double (&p3)[3][CQ],
                                                const double (&p4)[3][CQ]) {
  double2* out = ln.part + (size_t)tile * P.M;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int r = 3 * tr + i;
    if (r < B.nrun) {
      const GemmRun g = P.grun[B.run0 + r];
#pragma unroll
      for (int q = 0; q < CQ; ++q) {
        const int col = tn + 16 * q;
        const int cv = B.lo + col;
        if (col < B.nb) {
          if (cv >= g.a && cv <= g.b)
            out[g.kstart + (cv - g.a)] = make_double2(p1[i][q] - p2[i][q], p3[i][q] + p4[i][q]);
          if (cv > 0 && -cv >= g.a && -cv <= g.b)
            out[g.kstart + (-cv - g.a)] = make_double2(p1[i][q] + p2[i][q], p4[i][q] - p3[i][q]);
        }
      }
    }
  }
}

// Pass 1 of one (lane, tile, block) of a 3-D k-set as a complex GEMM over
// the tile's particles, kGemmChunk at a time: the tables of the chunk (prefix
// powers per axis, last-axis powers for the block's window) and the A rows
// (A = T0 T1, the runs' prefix phases) are built in shared memory. The last
// axis is folded as in the d = 2 body: columns are c = |n2| and the four sums
// P1..P4 of a cell give C(c) and C(-c). Each thread accumulates 3 runs x CQ
// columns (tn, tn + 16, ...). Each k-set row is written once. The roots z of
// the next chunk are formed while the A rows are built.
template <int D, int CQ>
__device__ void pass1_gemm_body(const ProbDev& P, const EvalLane& ln, int tile, int blk,
                                double2* smem) {
  constexpr int KC = kGemmChunk, ZS = gemm_fold_zstride(CQ), W = 16 * CQ;
  const GemmBlock B = P.gblk[blk];
  const int j0 = tile * kPass1Tile;
  const int nj = min(kPass1Tile, P.N - j0);
  const int c0 = B.c0, c1 = D == 3 ? B.c1 : 0;   // this group's prefix windows
  const int s0 = P.gs0, s1 = D == 3 ? P.gs1 : 0;
  double2* T0 = smem;                       // [KC][s0]
  double2* T1 = T0 + KC * s0;               // [KC][s1]
  double2* Z = T1 + KC * s1;                // [KC][ZS]
  double2* A = Z + KC * ZS;                 // [KC][kGemmRows]
  double2* R = A + KC * kGemmRows;          // [2][KC * D] roots, double-buffered
  const int tr = threadIdx.x >> 4, tn = threadIdx.x & 15;
  double p1[3][CQ], p2[3][CQ], p3[3][CQ], p4[3][CQ];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int q = 0; q < CQ; ++q) p1[i][q] = p2[i][q] = p3[i][q] = p4[i][q] = 0.0;
  const int L = P.gL, u0 = P.gu0, u1 = D == 3 ? P.gu1 : 0, uz = P.guz;
  chunk_roots<D>(R, ln.s, j0, min(KC, nj));
  int buf = 0;
  for (int jc = 0; jc < nj; jc += KC) {
    const int kc = min(KC, nj - jc);
    const double2* zs = R + buf * KC * D;
    __syncthreads();   // the previous chunk's products and this chunk's roots are done
    for (int u = threadIdx.x; u < KC * (u0 + u1 + uz); u += blockDim.x) {
      const int j = u % KC, q = u / KC;
      const double* sj = ln.s + (size_t)(j0 + jc + j) * D;
      const bool live = j < kc;
      if (q < u0) {
        if (L * q < c0)
          fill_powers(T0 + j * s0, L * q, min(L, c0 - L * q), B.m0, live ? sj[0] : 0.0,
                      zs[j * D]);
      } else if (q < u0 + u1) {
        const int qq = q - u0;
        if (L * qq < c1)
          fill_powers(T1 + j * s1, L * qq, min(L, c1 - L * qq), B.m1, live ? sj[1] : 0.0,
                      zs[j * D + 1]);
      } else {
        const int qq = q - u0 - u1;
        fill_powers(Z + j * ZS, L * qq, min(L, W - L * qq), B.lo, live ? sj[D - 1] : 0.0,
                    zs[j * D + D - 1]);
      }
    }
    __syncthreads();
    for (int u = threadIdx.x; u < KC * kGemmRows; u += blockDim.x) {
      const int j = u / kGemmRows, r = u - j * kGemmRows;
      double2 v = make_double2(0.0, 0.0);
      if (j < kc && r < B.nrun) {
        const GemmRun g = P.grun[B.run0 + r];
        v = T0[j * s0 + (g.n0 - B.m0)];
        if (D == 3) v = cmul(v, T1[j * s1 + (g.n1 - B.m1)]);
      }
      A[j * kGemmRows + r] = v;
    }
    if (jc + KC < nj) chunk_roots<D>(R + (buf ^ 1) * KC * D, ln.s, j0 + jc + KC, min(KC, nj - jc - KC));
    buf ^= 1;
    __syncthreads();
    const int kr = 6 * (threadIdx.x >> 5) < B.nrun ? kc : 0;   // warps past the runs skip
    for (int j = 0; j < kr; ++j) {
      double2 a[3], z[CQ];
#pragma unroll
      for (int i = 0; i < 3; ++i) a[i] = A[j * kGemmRows + 3 * tr + i];
#pragma unroll
      for (int q = 0; q < CQ; ++q) z[q] = Z[j * ZS + tn + 16 * q];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int q = 0; q < CQ; ++q) {
          p1[i][q] = fma(a[i].x, z[q].x, p1[i][q]);
          p2[i][q] = fma(a[i].y, z[q].y, p2[i][q]);
          p3[i][q] = fma(a[i].x, z[q].y, p3[i][q]);
          p4[i][q] = fma(a[i].y, z[q].x, p4[i][q]);
        }
    }
  }
  gemm_fold_store<CQ>(P, ln, tile, B, tr, tn, p1, p2, p3, p4);
}

// d = 2: the A rows are a gather from the prefix table (A[r][j] = T0[j][n0(r)]),
// so there is no A phase. The last axis is folded: the block's columns are
// c = |n|, and with A = a + ib and z^c = u + iv the four sums P1 = sum a u,
// P2 = sum b v, P3 = sum a v, P4 = sum b u give C(c) = (P1 - P2) + i (P3 + P4)
// and C(-c) = A conj(z^c) summed = (P1 + P2) + i (P4 - P3): four FMAs per
// cell and particle for two k-set rows. Each thread accumulates 3 runs x CQ
// columns (tn, tn + 16, ...). The tables are double-buffered: while the CTA
// multiplies chunk c it fills chunk c + 1 (and the roots of chunk c + 2), one
// barrier per chunk. Rows past the group's runs read the zero column c0.
// CQ: columns per thread (tn, tn + 16, ...), the problem's window is 16 CQ.
template <int CQ>
__device__ void pass1_gemm_body_d2(const ProbDev& P, const EvalLane& ln, int tile, int blk,
                                   double2* smem) {
  constexpr int KC = kGemmChunk, D = 2, ZS = gemm_fold_zstride(CQ), W = 16 * CQ;
  const GemmBlock B = P.gblk[blk];
  const int j0 = tile * kPass1Tile;
  const int nj = min(kPass1Tile, P.N - j0);
  const int c0 = B.c0, s0 = P.gs0;           // s0 > P.gc0 >= c0: column P.gc0 holds zeros
  const int zc = P.gc0;
  const int buf = KC * (s0 + ZS);            // one table set
  double2* R = smem + 2 * buf;               // [2][KC * D] roots
  const int tr = threadIdx.x >> 4, tn = threadIdx.x & 15;
  const bool rows_live = 6 * (threadIdx.x >> 5) < B.nrun;   // this warp's rows 6w .. 6w + 5
  int off[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const int r = 3 * tr + i;
    off[i] = r < B.nrun ? P.grun[B.run0 + r].n0 - B.m0 : zc;
  }
  double p1[3][CQ], p2[3][CQ], p3[3][CQ], p4[3][CQ];
#pragma unroll
  for (int i = 0; i < 3; ++i)
#pragma unroll
    for (int q = 0; q < CQ; ++q) p1[i][q] = p2[i][q] = p3[i][q] = p4[i][q] = 0.0;
  const int L = P.gL, u0 = P.gu0, uz = P.guz;
  const int nch = (nj + KC - 1) / KC;
  auto fill = [&](int c) {   // tables of chunk c into buffer c & 1 (roots in R[c & 1])
    double2* T0 = smem + (c & 1) * buf;
    double2* Z = T0 + KC * s0;
    const double2* zs = R + (c & 1) * KC * D;
    const int jc = c * KC, kc = min(KC, nj - jc);
    for (int u = threadIdx.x; u < KC * (u0 + uz); u += blockDim.x) {
      const int j = u % KC, q = u / KC;
      const double* sj = ln.s + (size_t)(j0 + jc + j) * D;
      const bool live = j < kc;
      if (q < u0) {
        if (L * q < c0)   // the problem's widest window sets the units; this one may be narrower
          fill_powers(T0 + j * s0, L * q, min(L, c0 - L * q), B.m0, live ? sj[0] : 0.0, zs[j * D]);
      } else {
        const int qq = q - u0;
        fill_powers(Z + j * ZS, L * qq, min(L, W - L * qq), B.lo, live ? sj[1] : 0.0,
                    zs[j * D + 1]);
      }
    }
    if (threadIdx.x < KC) T0[threadIdx.x * s0 + zc] = make_double2(0.0, 0.0);
  };
  chunk_roots<D>(R, ln.s, j0, min(KC, nj));
  if (nch > 1) chunk_roots<D>(R + KC * D, ln.s, j0 + KC, min(KC, nj - KC));
  __syncthreads();
  fill(0);
  __syncthreads();
  for (int c = 0; c < nch; ++c) {
    if (c + 1 < nch) fill(c + 1);
    if (c + 2 < nch)   // roots of chunk c + 2 replace those of chunk c (used by fill(c), done)
      chunk_roots<D>(R + (c & 1) * KC * D, ln.s, j0 + (c + 2) * KC, min(KC, nj - (c + 2) * KC));
    const double2* T0 = smem + (c & 1) * buf;
    const double2* Z = T0 + KC * s0;
    const int kc = rows_live ? min(KC, nj - c * KC) : 0;
    for (int j = 0; j < kc; ++j) {
      double2 a[3], z[CQ];
#pragma unroll
      for (int i = 0; i < 3; ++i) a[i] = T0[j * s0 + off[i]];
#pragma unroll
      for (int q = 0; q < CQ; ++q) z[q] = Z[j * ZS + tn + 16 * q];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int q = 0; q < CQ; ++q) {
          p1[i][q] = fma(a[i].x, z[q].x, p1[i][q]);
          p2[i][q] = fma(a[i].y, z[q].y, p2[i][q]);
          p3[i][q] = fma(a[i].x, z[q].y, p3[i][q]);
          p4[i][q] = fma(a[i].y, z[q].x, p4[i][q]);
        }
    }
    __syncthreads();
  }
  gemm_fold_store<CQ>(P, ln, tile, B, tr, tn, p1, p2, p3, p4);
}

// The folded 3-D body at the problem's window width.
__device__ __forceinline__ void pass1_gemm_d3(const ProbDev& P, const EvalLane& ln, int tile,
                                              int blk, double2* smem) {
  if (P.gcq == 1) pass1_gemm_body<3, 1>(P, ln, tile, blk, smem);
  else if (P.gcq == 2) pass1_gemm_body<3, 2>(P, ln, tile, blk, smem);
  else pass1_gemm_body<3, 3>(P, ln, tile, blk, smem);
}

// The folded d = 2 body at the problem's window width.
__device__ __forceinline__ void pass1_gemm_d2(const ProbDev& P, const EvalLane& ln, int tile,
                                              int blk, double2* smem) {
  if (P.gcq == 1) pass1_gemm_body_d2<1>(P, ln, tile, blk, smem);
  else if (P.gcq == 2) pass1_gemm_body_d2<2>(P, ln, tile, blk, smem);
  else pass1_gemm_body_d2<3>(P, ln, tile, blk, smem);
}

}  // namespace

}  // namespace cco
