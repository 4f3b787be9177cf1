// C ABI of libcco: problems, evaluation and the batched relax drivers.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "cco_host.cuh"
#include "cco_internal.cuh"
#include "cco_opt.cuh"

using namespace cco;

namespace {
thread_local std::string g_last_error;
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxPoolDevices] = {};
}  // namespace

namespace cco {

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

int cuda_fail(cudaError_t e, const char* what) {
  if (e == cudaErrorMemoryAllocation) return fail(CCO_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return fail(CCO_ERR_DEVICE, "%s: %s", what, cudaGetErrorString(e));
}

// One pool per device that keeps its memory (release threshold = max): a
// relaxation's lane records are reused by the next call instead of being
// unmapped at every synchronize, as the default pool (threshold 0) would do.
cudaError_t device_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxPoolDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    e = cudaMemPoolCreate(&pool, &props);
    if (e != cudaSuccess) return e;
    uint64_t keep = UINT64_MAX;
    e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) return e;
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

}  // namespace cco


namespace {

// ----------------------------------------------------------- problem build
// Digit layout of one axis for |n| <= R with `nlev` levels: base b with
// b^nlev > R; level 0 holds z^0..z^(b-1) (the run axis needs z^1, so b >= 2
// there), the top level holds R / b^(nlev-1) + 1 entries.
void set_axis(TabLayout& T, int a, int R, int nlev, bool run_axis) {
  const int nv = R + 1;
  int b = 1;
  if (nlev == 1) {
    b = std::max(nv, run_axis ? 2 : 1);
  } else {
    b = std::max(2, (int)std::floor(std::pow((double)nv, 1.0 / nlev)));
    auto pw = [&](int x) { long long r = 1; for (int l = 0; l < nlev; ++l) r *= x; return r; };
    while (pw(b) < nv) ++b;
  }
  T.nlev[a] = nlev;
  T.base[a] = b;
  long long scale = 1;
  for (int l = 0; l < kMaxLevels; ++l) {
    if (l >= nlev) T.nent[a][l] = 0;
    else if (l == nlev - 1) T.nent[a][l] = (int)(R / scale) + 1;
    else T.nent[a][l] = b;
    if (l == 0 && nlev == 1) T.nent[a][0] = b;
    scale *= b;
  }
}

void assign_rows(TabLayout& T, int d) {
  int row = 0;
  for (int a = 0; a < 3; ++a)
    for (int l = 0; l < kMaxLevels; ++l) {
      T.row[a][l] = row;
      if (a < d && l < T.nlev[a]) row += T.nent[a][l];
    }
  T.nrows = row;
  T.zrow = T.row[d - 1][0] + 1;
}

// Fewest table lookups whose rows fit `max_rows`: start with one level per
// axis (one load per lookup) and add a level to the axis with the most rows
// until the table fits (or every axis has kMaxLevels levels).
TabLayout make_layout(const int* R, int d, int max_rows) {
  TabLayout T{};
  int lev[3] = {1, 1, 1};
  for (;;) {
    for (int a = 0; a < d; ++a) set_axis(T, a, R[a], lev[a], a == d - 1);
    assign_rows(T, d);
    if (T.nrows <= max_rows) break;
    int best = -1, most = 0;
    for (int a = 0; a < d; ++a) {
      int rows = 0;
      for (int l = 0; l < lev[a]; ++l) rows += T.nent[a][l];
      if (lev[a] < kMaxLevels && rows > most) { most = rows; best = a; }
    }
    if (best < 0) break;
    ++lev[best];
  }
  return T;
}

// Absolute table rows of the digits of v on axis a (+ sign bit 24).
int pack_rows(int v, const TabLayout& T, int a) {
  const int neg = v < 0;
  int x = v < 0 ? -v : v;
  int out = 0;
  for (int l = 0; l < T.nlev[a]; ++l) {
    int dl;
    if (l == T.nlev[a] - 1) dl = x;
    else {
      dl = x % T.base[a];
      x /= T.base[a];
    }
    out |= ((T.row[a][l] + dl) & 255) << (8 * l);
  }
  return out | (neg << 24);
}

}  // namespace

extern "C" {

int cco_abi_version(void) { return CCO_ABI_VERSION; }

const char* cco_error_string(int code) {
  switch (code) {
    case CCO_OK: return "ok";
    case CCO_ERR_ARG: return "invalid argument";
    case CCO_ERR_OOM: return "out of device memory";
    case CCO_ERR_ADMISSION: return "refused by the HBM admission budget";
    case CCO_ERR_DEVICE: return "CUDA error";
    case CCO_ERR_TIMEOUT: return "timed out";
    case CCO_ERR_ROUNDS: return "relax did not finish within the round bound";
    case CCO_ERR_NODEVICE: return "no CUDA device";
    default: return "unknown error";
  }
}

const char* cco_last_error(void) { return g_last_error.c_str(); }

int cco_device_count(int* n_devices) {
  if (!n_devices) return fail(CCO_ERR_ARG, "n_devices is null");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0) {
    *n_devices = 0;
    cudaGetLastError();
    return fail(CCO_ERR_NODEVICE, "no CUDA device visible (%s)",
                e == cudaSuccess ? "count 0" : cudaGetErrorString(e));
  }
  *n_devices = n;
  return CCO_OK;
}

int cco_problem_create(int device, int d, int n_particles, int m, const int32_t* n_vectors,
                       const double* weights, double volume, cco_problem** out) {
  if (!out) return fail(CCO_ERR_ARG, "out is null");
  *out = nullptr;
  if (d < 1 || d > 3) return fail(CCO_ERR_ARG, "d must be 1, 2 or 3, got %d", d);
  if (n_particles < 1) return fail(CCO_ERR_ARG, "n_particles must be >= 1");
  if (m < 1) return fail(CCO_ERR_ARG, "empty k-set: no k-vectors in the shell");
  if (!n_vectors || !weights) return fail(CCO_ERR_ARG, "null k-set arrays");
  if (!(volume > 0.0) || !std::isfinite(volume)) return fail(CCO_ERR_ARG, "volume must be finite and > 0");
  int ndev = 0;
  if (cco_device_count(&ndev) != CCO_OK) return CCO_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return fail(CCO_ERR_ARG, "device %d out of range", device);

  // validate rows
  std::vector<int> R(3, 0);
  for (int k = 0; k < m; ++k) {
    bool nz = false;
    for (int a = 0; a < d; ++a) {
      const int v = n_vectors[(size_t)k * d + a];
      if (v < -65535 || v > 65535) return fail(CCO_ERR_ARG, "|n| too large at row %d", k);
      R[a] = std::max(R[a], std::abs(v));
      nz |= v != 0;
    }
    if (!nz) return fail(CCO_ERR_ARG, "row %d is the zero vector (padding rows are handled by the caller)", k);
    if (!std::isfinite(weights[k])) return fail(CCO_ERR_ARG, "non-finite weight at row %d", k);
  }
  // run order: prefix lexicographic, then the last axis ascending
  std::vector<int> order(m);
  for (int k = 0; k < m; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    for (int a = 0; a < d; ++a) {
      const int u = n_vectors[(size_t)x * d + a], v = n_vectors[(size_t)y * d + a];
      if (u != v) return u < v;
    }
    return false;
  });
  for (int k = 1; k < m; ++k) {
    bool same = true;
    for (int a = 0; a < d; ++a)
      same &= n_vectors[(size_t)order[k] * d + a] == n_vectors[(size_t)order[k - 1] * d + a];
    if (same) return fail(CCO_ERR_ARG, "duplicate k row (rows %d and %d)", order[k - 1], order[k]);
  }
  ProbDev P{};
  P.d = d;
  P.N = n_particles;
  P.M = m;
  {
    const int Rv[3] = {R[0], R[1], R[2]};
    P.t1 = make_layout(Rv, d, (int)(kPass1TableBudget / (kPass1Stride * sizeof(double2))));
    P.t2 = make_layout(Rv, d, (int)(kPass2TableBudget / (kPass2Tile * sizeof(double2))));
  }
  if (P.t1.nrows > 255 || P.t2.nrows > 255)
    return fail(CCO_ERR_ARG, "k-set phase tables too large (%d / %d rows)", P.t1.nrows, P.t2.nrows);
  P.ntile1 = (n_particles + kPass1Tile - 1) / kPass1Tile;
  P.ntile2 = (n_particles + kPass2Tile - 1) / kPass2Tile;
  P.vol = volume;
  P.gpref = (2.0 * (2.0 * M_PI)) / volume;

  // runs -> segments (headers carry each pass's absolute table rows)
  std::vector<SegHdr> s1, s2;
  std::vector<GemmRun> runs;
  auto emit = [&](std::vector<SegHdr>& dst, const TabLayout& T, int kstart, int len, int maxlen) {
    for (int off = 0; off < len; off += maxlen) {
      SegHdr h{};
      h.kstart = kstart + off;
      h.len = std::min(maxlen, len - off);
      const int* nv = n_vectors + (size_t)order[h.kstart] * d;
      for (int a = 0; a < d; ++a) {
        h.n[a] = nv[a];
        h.dig[a] = pack_rows(nv[a], T, a);
      }
      dst.push_back(h);
    }
  };
  int start = 0;
  for (int k = 1; k <= m; ++k) {
    bool brk = (k == m);
    if (!brk) {
      const int* p = n_vectors + (size_t)order[k - 1] * d;
      const int* c = n_vectors + (size_t)order[k] * d;
      for (int a = 0; a < d - 1; ++a) brk |= p[a] != c[a];
      brk |= c[d - 1] != p[d - 1] + 1;
    }
    if (brk) {
      emit(s1, P.t1, start, k - start, kSeg1Len);
      emit(s2, P.t2, start, k - start, kSeg2Len);
      const int* nv = n_vectors + (size_t)order[start] * d;
      GemmRun g{};
      g.n0 = d >= 2 ? nv[0] : 0;
      g.n1 = d >= 3 ? nv[1] : 0;
      g.a = nv[d - 1];
      g.b = nv[d - 1] + (k - start) - 1;
      g.kstart = start;
      runs.push_back(g);
      start = k;
    }
  }
  // GEMM pass 1: runs grouped kGemmRows at a time by length, each group's
  // last-axis range cut into column windows. Used when the blocks cost at
  // most 8 FMAs per k-set row and particle (4 for d = 3): m >= cells / 2
  // (m >= cells), cells counted with the warps' 6-row granularity (a folded
  // cell serves two rows)
  // (CCO_PASS1_GEMM=0 turns it off).
  std::vector<GemmRun> grun;
  std::vector<GemmBlock> gblk;
  {
    const char* env = getenv("CCO_PASS1_GEMM");
    const bool allow = d >= 2 && !(env && atoi(env) == 0);
    // The last axis is folded: columns are c = |n|, a run [a, b] covers
    // [ca, cb] (its folded range), and one cell (run, c) yields C(c) and C(-c).
    // Its window width is 16 cq columns (cq = 1..3), the width that computes
    // the fewest cells for this k-set (the widest on ties: fewer blocks).
    auto fa = [](const GemmRun& g) {
      return (g.a <= 0 && g.b >= 0) ? 0 : std::min(std::abs(g.a), std::abs(g.b));
    };
    auto fb = [](const GemmRun& g) { return std::max(std::abs(g.a), std::abs(g.b)); };
    std::vector<GemmRun> sorted = runs;
    std::stable_sort(sorted.begin(), sorted.end(), [&](const GemmRun& x, const GemmRun& y) {
      return (fb(x) - fa(x)) > (fb(y) - fa(y));
    });
    int c0 = 0, c1 = 0;      // widest group prefix windows
    double computed = 0.0;   // grid cells the blocks multiply (4 FMAs per particle each)
    auto group = [&](int cols) {
      grun.clear();
      gblk.clear();
      c0 = c1 = 0;
      computed = 0.0;
      for (size_t r0 = 0; r0 < sorted.size(); r0 += kGemmRows) {
        const int nrun = (int)std::min<size_t>(kGemmRows, sorted.size() - r0);
        int lo = 1 << 30, hi = -(1 << 30);
        int gm0 = 1 << 30, gM0 = -(1 << 30), gm1 = 1 << 30, gM1 = -(1 << 30);
        for (int r = 0; r < nrun; ++r) {
          const GemmRun& g = sorted[r0 + r];
          lo = std::min(lo, fa(g));
          hi = std::max(hi, fb(g));
          gm0 = std::min(gm0, g.n0);
          gM0 = std::max(gM0, g.n0);
          gm1 = std::min(gm1, g.n1);
          gM1 = std::max(gM1, g.n1);
        }
        // each group's prefix tables cover only its own prefixes
        const int gc0 = gM0 - gm0 + 1, gc1 = d >= 3 ? gM1 - gm1 + 1 : 0;
        c0 = std::max(c0, gc0);
        c1 = std::max(c1, gc1);
        const int run0 = (int)grun.size();
        for (int r = 0; r < nrun; ++r) grun.push_back(sorted[r0 + r]);
        // warps whose 6 rows lie past the group's runs skip their products
        computed += (double)((nrun + 5) / 6 * 6) * cols * ((hi - lo) / cols + 1);
        for (int w = lo; w <= hi; w += cols) {
          GemmBlock b{};
          b.run0 = run0;
          b.nrun = nrun;
          b.lo = w;
          b.nb = std::min(cols, hi - w + 1);
          b.m0 = gm0;
          b.c0 = gc0;
          b.m1 = d >= 3 ? gm1 : 0;
          b.c1 = gc1;
          gblk.push_back(b);
        }
      }
    };
    int best = 1;
    double best_cells = 0.0;
    for (int cq = 1; cq <= kGemmFoldMaxCq; ++cq) {
      group(16 * cq);
      if (cq == 1 || computed <= best_cells) {
        best = cq;
        best_cells = computed;
      }
    }
    const int cols = 16 * best;
    P.gcq = best;
    group(cols);
    const double cells = computed;
    // d = 3 builds an A phase per chunk and only broke even with the
    // per-segment kernel at about 3.5 FMAs per row (d=3 N=4000 chi=0.45: 1.480
    // vs 1.481 ms per 32-lane evaluation; at 6.2 FMAs, N=2000 chi=0.20, it lost
    // 4%), so 3-D k-sets take the GEMM form only at <= 4 FMAs per row
    const double need = d == 3 ? 1.0 : 0.5;
    P.gemm = allow && !runs.empty() && c0 <= kGemmMaxPrefix && c1 <= kGemmMaxPrefix &&
             (double)m >= need * cells;
    P.ngblk = (int)gblk.size();
    P.gm0 = 0;
    P.gc0 = c0;
    P.gm1 = 0;
    P.gc1 = c1;
    P.gs0 = (c0 + 1) | 1;   // odd, with a spare column c0 (zeros in the d = 2 kernel)
    P.gs1 = c1 > 0 ? (c1 | 1) : 0;
    // fill units: the fewest rounds of one unit per thread, then the
    // shortest chains (each unit seeds with sincospi, then multiplies)
    const int per_round = kGemmThreads / kGemmChunk;
    bool found = false;
    for (int rounds = 1; !found; ++rounds)
      for (int L = 8; L <= kGemmMaxRun && !found; ++L) {
        const int u0 = (c0 + L - 1) / L, u1 = (c1 + L - 1) / L, uz = (cols + L - 1) / L;
        if (u0 + u1 + uz <= per_round * rounds) {
          P.gL = L;
          P.gu0 = u0;
          P.gu1 = u1;
          P.guz = uz;
          found = true;
        }
      }
  }
  // longest segments first: pass-1 warps share trip counts, pass 2 pairs
  // segments of similar length
  auto by_len = [](const SegHdr& x, const SegHdr& y) { return x.len > y.len; };
  std::stable_sort(s1.begin(), s1.end(), by_len);
  std::stable_sort(s2.begin(), s2.end(), by_len);
  P.nseg1 = (int)s1.size();
  P.nseg2 = (int)s2.size();
  {
    // logical pass-2 slices: at least one segment pair each, at most 8 (a
    // launch of few lanes spreads a particle's slices over up to 8 threads)
    const int npairs = (P.nseg2 + 1) / 2;
    int sl = 1;
    while (sl < 8 && 2 * sl <= npairs) sl *= 2;
    P.sl2 = sl;
  }

  const size_t smem1 = eval_smem1(P);
  const size_t smem2 = std::max(std::max(eval_smem2(P, 1), eval_smem2(P, 8)),
                                std::max(eval_smem2(P, 1, true), eval_smem2(P, 8, true)));
  if (smem1 > 220 * 1024 || smem2 > 220 * 1024)
    return fail(CCO_ERR_ARG, "k-set phase tables too large for shared memory (%d / %d rows)",
                P.t1.nrows, P.t2.nrows);

  DeviceGuard guard(device);
  static std::once_flag once;
  static cudaError_t cfg_err = cudaSuccess;
  std::call_once(once, [] { cfg_err = eval_configure(); });
  if (cfg_err != cudaSuccess) return cuda_fail(cfg_err, "eval_configure");

  auto* pr = new cco_problem();
  pr->device = device;
  pr->d = d;
  pr->N = n_particles;
  pr->M = m;
  std::vector<double> w_run(m);
  std::vector<int> r2r(m);
  std::vector<double4> krow(m);
  for (int k = 0; k < m; ++k) {
    w_run[k] = weights[order[k]];
    r2r[k] = order[k];
    const int32_t* nv = n_vectors + (size_t)order[k] * d;
    krow[k] = make_double4(nv[0], d > 1 ? nv[1] : 0, d > 2 ? nv[2] : 0, w_run[k]);
  }
  cudaError_t e = cudaSuccess;
  e = cudaMalloc(&pr->seg1, s1.size() * sizeof(SegHdr));
  if (e == cudaSuccess) e = cudaMalloc(&pr->seg2, s2.size() * sizeof(SegHdr));
  if (e == cudaSuccess) e = cudaMalloc(&pr->w_run, m * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&pr->run2ref, m * sizeof(int));
  if (e == cudaSuccess) e = cudaMalloc(&pr->dev, sizeof(ProbDev));
  if (e == cudaSuccess) e = cudaMemcpy(pr->seg1, s1.data(), s1.size() * sizeof(SegHdr), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pr->seg2, s2.data(), s2.size() * sizeof(SegHdr), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pr->w_run, w_run.data(), m * sizeof(double), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(pr->run2ref, r2r.data(), m * sizeof(int), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMalloc(&pr->krow, m * sizeof(double4));
  if (e == cudaSuccess) e = cudaMemcpy(pr->krow, krow.data(), m * sizeof(double4), cudaMemcpyHostToDevice);
  if (P.gemm) {
    if (e == cudaSuccess) e = cudaMalloc(&pr->grun, grun.size() * sizeof(GemmRun));
    if (e == cudaSuccess) e = cudaMalloc(&pr->gblk, gblk.size() * sizeof(GemmBlock));
    if (e == cudaSuccess) e = cudaMemcpy(pr->grun, grun.data(), grun.size() * sizeof(GemmRun), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(pr->gblk, gblk.data(), gblk.size() * sizeof(GemmBlock), cudaMemcpyHostToDevice);
  }
  P.grun = pr->grun;
  P.gblk = pr->gblk;
  P.seg1 = pr->seg1;
  P.seg2 = pr->seg2;
  P.w_run = pr->w_run;
  P.run2ref = pr->run2ref;
  if (e == cudaSuccess) e = cudaMemcpy(pr->dev, &P, sizeof(ProbDev), cudaMemcpyHostToDevice);
  pr->host = P;
  pr->smem1 = smem1;
  pr->smem2 = smem2;
  pr->smemG = eval_smemG(P);
  if (e != cudaSuccess) {
    cco_problem_destroy(pr);
    return cuda_fail(e, "cco_problem_create upload");
  }
  *out = pr;
  return CCO_OK;
}

int cco_problem_destroy(cco_problem* p) {
  if (!p) return CCO_OK;
  DeviceGuard guard(p->device);
  cudaFree(p->seg1);
  cudaFree(p->seg2);
  cudaFree(p->w_run);
  cudaFree(p->run2ref);
  if (p->grun) cudaFree(p->grun);
  if (p->gblk) cudaFree(p->gblk);
  if (p->krow) cudaFree(p->krow);
  cudaFree(p->dev);
  delete p;
  return CCO_OK;
}

int cco_problem_info(const cco_problem* p, int* d, int* n_particles, int* m, int* n_seg1,
                     int* n_seg2, int* table_rows) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (d) *d = p->d;
  if (n_particles) *n_particles = p->N;
  if (m) *m = p->M;
  if (n_seg1) *n_seg1 = p->host.nseg1;
  if (n_seg2) *n_seg2 = p->host.nseg2;
  if (table_rows) *table_rows = p->host.t1.nrows * 256 + p->host.t2.nrows;
  return CCO_OK;
}

int cco_problem_pass1_form(const cco_problem* p, int* gemm_blocks) {
  if (!p || !gemm_blocks) return fail(CCO_ERR_ARG, "null argument");
  *gemm_blocks = p->host.gemm ? p->host.ngblk : 0;
  return CCO_OK;
}

}  // extern "C"

// ------------------------------------------------------------ eval workspace
namespace {

__global__ void k_make_lanes(EvalLane* lanes, EvalItem* it1, EvalItem* it2, EvalItem* itG,
                             int B, int nt1, int nt2, int ntG, int total, const double* s,
                             size_t s_stride, double* f,
                             size_t f_stride, double* g, size_t g_stride, double2* rho,
                             double2* rhow, double2* part, int M, const int64_t* status,
                             size_t status_stride, int prec) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    if (i < B) {
      EvalLane L;
      L.s = s + (size_t)i * s_stride;
      L.f = f + (size_t)i * f_stride;
      L.g = g ? g + (size_t)i * g_stride : nullptr;
      L.rho = rho + (size_t)i * M;
      L.rhow = rhow + (size_t)i * M;
      L.part = part + (size_t)i * nt1 * M;
      L.status = status ? status + (size_t)i * status_stride : nullptr;
      L.prec = nullptr;
      L.fixed_prec = prec;
      L.prob = 0;
      lanes[i] = L;
    }
    const int j = i - B;
    if (j >= 0) {
      if (j < B * nt1) it1[j] = EvalItem{j / nt1, j % nt1};
      if (j < B * nt2) it2[j] = EvalItem{j / nt2, j % nt2};
      if (itG && j < B * ntG) itG[j] = EvalItem{j / ntG, j % ntG};
    }
  }
}

// Device buffers of one batched evaluation: densities, partials and the plan.
struct EvalWS {
  EvalLane* lanes = nullptr;
  EvalItem* it1 = nullptr;
  EvalItem* it2 = nullptr;
  EvalItem* itG = nullptr;   // GEMM pass-1 items (problems with p->host.gemm)
  double2* rho = nullptr;
  double2* rhow = nullptr;
  double2* part = nullptr;
  EvalPlan plan{};
  int prec = PREC_FP64;   // arithmetic of every lane of this workspace

  static int gemm_tiles(const cco_problem* p) {
    return p->host.gemm ? p->host.ntile1 * p->host.ngblk : 0;
  }

  // pass-2 threads per particle and tiles per configuration for a batch of B
  static int split_for(const cco_problem* p, int B) {
    return pass2_split((long long)B * p->host.ntile2);
  }
  cudaError_t alloc(const cco_problem* p, int B, cudaStream_t st) {
    const int M = p->M, nt1 = p->host.ntile1, nt2 = pass2_tiles(p->host, split_for(p, B));
    cudaError_t e = pool_alloc(&lanes, sizeof(EvalLane) * B, st);
    if (e == cudaSuccess) e = pool_alloc(&it1, sizeof(EvalItem) * (size_t)B * nt1, st);
    if (e == cudaSuccess) e = pool_alloc(&it2, sizeof(EvalItem) * (size_t)B * nt2, st);
    if (e == cudaSuccess && gemm_tiles(p) > 0)
      e = pool_alloc(&itG, sizeof(EvalItem) * (size_t)B * gemm_tiles(p), st);
    if (e == cudaSuccess) e = pool_alloc(&rho, sizeof(double2) * (size_t)B * M, st);
    if (e == cudaSuccess) e = pool_alloc(&rhow, sizeof(double2) * (size_t)B * M, st);
    if (e == cudaSuccess) e = pool_alloc(&part, sizeof(double2) * (size_t)B * nt1 * M, st);
    return e;
  }
  cudaError_t build(const cco_problem* p, int B, const double* s, size_t s_stride, double* f,
                    size_t f_stride, double* g, size_t g_stride, const int64_t* status,
                    size_t status_stride, cudaStream_t st) {
    const int split = split_for(p, B);
    const int nt1 = p->host.ntile1, nt2 = pass2_tiles(p->host, split);
    const int ntG = itG ? gemm_tiles(p) : 0;
    const int total = B * std::max(std::max(nt1, nt2), ntG) + B;
    const int blocks = std::min(1024, (total + 255) / 256);
    k_make_lanes<<<blocks, 256, 0, st>>>(lanes, it1, it2, itG, B, nt1, nt2, ntG, total, s,
                                         s_stride, f, f_stride, g, g_stride, rho, rhow, part,
                                         p->M, status, status_stride, prec);
    plan.probs = p->dev;
    plan.lanes = lanes;
    plan.items1 = it1;
    plan.items2 = it2;
    plan.itemsG = itG;
    plan.n_lanes = B;
    // the per-segment pass 1 covers FP32 lanes, and FP64 lanes of problems
    // without the GEMM form
    plan.n_items1 = (ntG > 0 && prec == PREC_FP64) ? 0 : B * nt1;
    plan.n_items2 = B * nt2;
    plan.n_itemsG = (prec == PREC_FP64) ? B * ntG : 0;
    for (int D = 0; D <= 3; ++D) {
      plan.d_off1[D] = D >= p->d ? plan.n_items1 : 0;
      plan.d_off2[D] = D >= p->d ? plan.n_items2 : 0;
      plan.d_offG[D] = D >= p->d ? plan.n_itemsG : 0;
    }
    // one problem: its GEMM items are all of its window width
    for (int D = 2; D <= 3; ++D)
      for (int c = 0; c <= kGemmFoldMaxCq; ++c)
        plan.q_offG[D - 2][c] = (D == p->d && c >= p->host.gcq) ? plan.n_itemsG : 0;
    plan.smemG = p->smemG;
    plan.dyn_prec = prec == PREC_FP32 ? 1 : 0;
    plan.max_d = p->d;
    plan.smem1 = p->smem1;
    plan.smem2 = eval_smem2(p->host, split);
    plan.smem2_f32 = eval_smem2(p->host, split, true);
    plan.split2 = split;
    plan.chunks1 = 1;
    plan.red_chunks = reduce_chunks(p->M);
    plan.want_grad = g != nullptr;
    return cudaGetLastError();
  }
  void release(cudaStream_t st) {
    cudaFreeAsync(lanes, st);
    cudaFreeAsync(it1, st);
    cudaFreeAsync(it2, st);
    if (itG) cudaFreeAsync(itG, st);
    cudaFreeAsync(rho, st);
    cudaFreeAsync(rhow, st);
    cudaFreeAsync(part, st);
    lanes = nullptr;
    itG = nullptr;
  }
};

}  // namespace

extern "C" int cco_energy_grad(cco_problem* p, void* stream, int batch, const double* s,
                               double* phi, double* grad, double* rho_re, double* rho_im) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (batch < 0) return fail(CCO_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return CCO_OK;
  if (!s || !phi) return fail(CCO_ERR_ARG, "null s or phi");
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  EvalWS ws;
  CCO_CUDA(ws.alloc(p, batch, st));
  const size_t nd = (size_t)p->N * p->d;
  CCO_CUDA(ws.build(p, batch, s, nd, phi, 1, grad, nd, nullptr, 0, st));
  CCO_CUDA(eval_launch(ws.plan, st));
  if (rho_re || rho_im)
    CCO_CUDA(rho_scatter(ws.rho, p->run2ref, p->M, batch, p->M, rho_re, rho_im, st));
  ws.release(st);
  CCO_CUDA(cudaGetLastError());
  return CCO_OK;
}

extern "C" int cco_energy_grad_fp32(cco_problem* p, void* stream, int batch, const double* s,
                                    double* phi, double* grad) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (batch < 0) return fail(CCO_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return CCO_OK;
  if (!s || !phi) return fail(CCO_ERR_ARG, "null s or phi");
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  EvalWS ws;
  ws.prec = PREC_FP32;
  CCO_CUDA(ws.alloc(p, batch, st));
  const size_t nd = (size_t)p->N * p->d;
  CCO_CUDA(ws.build(p, batch, s, nd, phi, 1, grad, nd, nullptr, 0, st));
  CCO_CUDA(eval_launch(ws.plan, st));
  ws.release(st);
  CCO_CUDA(cudaGetLastError());
  return CCO_OK;
}

extern "C" int cco_hessian(cco_problem* p, void* stream, int batch, const double* s,
                           double* hess) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (batch < 0) return fail(CCO_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return CCO_OK;
  if (!s || !hess) return fail(CCO_ERR_ARG, "null s or hess");
  if (batch > 65535) return fail(CCO_ERR_ARG, "batch %d > 65535: split it", batch);
  DeviceGuard guard(p->device);
  cudaStream_t st = (cudaStream_t)stream;
  EvalWS ws;
  double* phi = nullptr;
  CCO_CUDA(ws.alloc(p, batch, st));
  CCO_CUDA(pool_alloc(&phi, sizeof(double) * batch, st));
  const size_t nd = (size_t)p->N * p->d;
  CCO_CUDA(ws.build(p, batch, s, nd, phi, 1, nullptr, 0, nullptr, 0, st));
  CCO_CUDA(eval_launch(ws.plan, st));   // the density the diagonal blocks need
  CCO_CUDA(hessian_launch(p, st, batch, s, ws.rho, hess));
  ws.release(st);
  cudaFreeAsync(phi, st);
  CCO_CUDA(cudaGetLastError());
  return CCO_OK;
}

// ------------------------------------------------- evaluation without allocation
namespace {

// Scratch of cco_energy_grad_noalloc: one fixed device array in the library,
// resident on every GPU that loads it until the process exits. Host code must
// never pass this name to a kernel: on the host it is only a stand-in for the
// symbol; the device address is resolved per device below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[CCO_NOALLOC_SCRATCH_BYTES];

constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_addr[kNoallocMaxDevices] = {};

// Device address of the scratch on `device`, resolved on the first call with
// that device current (the caller holds a DeviceGuard for it).
int noalloc_scratch(int device, unsigned char** out) {
  if (device < 0 || device >= kNoallocMaxDevices)
    return fail(CCO_ERR_ARG, "device %d out of range for the fixed scratch", device);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (g_noalloc_addr[device] == nullptr) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(fixed scratch)");
    g_noalloc_addr[device] = addr;
  }
  *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
  return CCO_OK;
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" int cco_energy_grad_noalloc(cco_problem* p, void* stream, int batch, const double* s,
                                       double* phi, double* grad) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (batch < 0) return fail(CCO_ERR_ARG, "batch must be >= 0");
  if (batch == 0) return CCO_OK;
  if (!s || !phi) return fail(CCO_ERR_ARG, "null s or phi");
  const size_t B = (size_t)batch, M = (size_t)p->M;
  const size_t nt1 = (size_t)p->host.ntile1;
  const size_t nt2 = (size_t)pass2_tiles(p->host, EvalWS::split_for(p, batch));
  const size_t b_lanes = round256(sizeof(EvalLane) * B);
  const size_t b_it1 = round256(sizeof(EvalItem) * B * nt1);
  const size_t b_it2 = round256(sizeof(EvalItem) * B * nt2);
  const size_t b_itG = round256(sizeof(EvalItem) * B * (size_t)EvalWS::gemm_tiles(p));
  const size_t b_rho = round256(sizeof(double2) * B * M);
  const size_t b_part = round256(sizeof(double2) * B * nt1 * M);
  const size_t need = b_lanes + b_it1 + b_it2 + 2 * b_rho + b_part + b_itG;
  if (need > CCO_NOALLOC_SCRATCH_BYTES)
    return fail(CCO_ERR_ARG,
                "batch %d needs %zu bytes of fixed scratch, the limit is %zu: split the batch",
                batch, need, (size_t)CCO_NOALLOC_SCRATCH_BYTES);
  DeviceGuard guard(p->device);
  unsigned char* base = nullptr;
  const int rc = noalloc_scratch(p->device, &base);
  if (rc != CCO_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  EvalWS ws;  // carved from the fixed scratch; never released
  ws.lanes = reinterpret_cast<EvalLane*>(base);
  ws.it1 = reinterpret_cast<EvalItem*>(base + b_lanes);
  ws.it2 = reinterpret_cast<EvalItem*>(base + b_lanes + b_it1);
  ws.rho = reinterpret_cast<double2*>(base + b_lanes + b_it1 + b_it2);
  ws.rhow = reinterpret_cast<double2*>(base + b_lanes + b_it1 + b_it2 + b_rho);
  ws.part = reinterpret_cast<double2*>(base + b_lanes + b_it1 + b_it2 + 2 * b_rho);
  ws.itG = b_itG > 0 ? reinterpret_cast<EvalItem*>(base + b_lanes + b_it1 + b_it2 + 2 * b_rho + b_part)
                     : nullptr;
  const size_t nd = (size_t)p->N * p->d;
  CCO_CUDA(ws.build(p, batch, s, nd, phi, 1, grad, nd, nullptr, 0, st));
  CCO_CUDA(eval_launch(ws.plan, st));
  return CCO_OK;
}

