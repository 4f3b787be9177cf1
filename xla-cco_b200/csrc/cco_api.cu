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

#include "cco_internal.cuh"
#include "cco_opt.cuh"

using namespace cco;

namespace {

thread_local std::string g_last_error;

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

#define CCO_CUDA(call)                                 \
  do {                                                 \
    cudaError_t e_ = (call);                           \
    if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
  } while (0)

// Stream-ordered allocations come from one memory pool per device that keeps
// its memory (release threshold = max): a relaxation's ~GB of lane state is
// reused by the next call instead of being unmapped at every synchronize, as
// the default pool (threshold 0) would do.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mu;
cudaMemPool_t g_pool[kMaxPoolDevices] = {};

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

template <class T>
cudaError_t pool_alloc(T** ptr, size_t bytes, cudaStream_t st) {
  cudaMemPool_t pool;
  const cudaError_t e = device_pool(&pool);
  if (e != cudaSuccess) return e;
  return cudaMallocFromPoolAsync(reinterpret_cast<void**>(ptr), bytes, pool, st);
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

}  // namespace

struct cco_problem {
  int device = 0;
  int d = 0, N = 0, M = 0;
  ProbDev host{};         // pointers are device pointers
  ProbDev* dev = nullptr; // device copy
  SegHdr* seg1 = nullptr;
  SegHdr* seg2 = nullptr;
  double* w_run = nullptr;
  int* run2ref = nullptr;
  size_t smem1 = 0, smem2 = 0;
};

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
      start = k;
    }
  }
  // longest segments first: pass-1 warps share trip counts, pass 2 pairs
  // segments of similar length
  auto by_len = [](const SegHdr& x, const SegHdr& y) { return x.len > y.len; };
  std::stable_sort(s1.begin(), s1.end(), by_len);
  std::stable_sort(s2.begin(), s2.end(), by_len);
  P.nseg1 = (int)s1.size();
  P.nseg2 = (int)s2.size();

  const size_t smem1 = eval_smem1(P), smem2 = eval_smem2(P);
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
  for (int k = 0; k < m; ++k) {
    w_run[k] = weights[order[k]];
    r2r[k] = order[k];
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
  P.seg1 = pr->seg1;
  P.seg2 = pr->seg2;
  P.w_run = pr->w_run;
  P.run2ref = pr->run2ref;
  if (e == cudaSuccess) e = cudaMemcpy(pr->dev, &P, sizeof(ProbDev), cudaMemcpyHostToDevice);
  pr->host = P;
  pr->smem1 = smem1;
  pr->smem2 = smem2;
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

}  // extern "C"

// ------------------------------------------------------------ eval workspace
namespace {

__global__ void k_make_lanes(EvalLane* lanes, EvalItem* it1, EvalItem* it2, int B, int nt1,
                             int nt2, int total, const double* s, size_t s_stride, double* f,
                             size_t f_stride, double* g, size_t g_stride, double2* rho,
                             double2* rhow, double2* part, int M, const int64_t* status,
                             size_t status_stride) {
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
      L.prob = 0;
      L.pad_ = 0;
      lanes[i] = L;
    }
    const int j = i - B;
    if (j >= 0) {
      if (j < B * nt1) it1[j] = EvalItem{j / nt1, j % nt1};
      if (j < B * nt2) it2[j] = EvalItem{j / nt2, j % nt2};
    }
  }
}

// Device buffers of one batched evaluation: densities, partials and the plan.
struct EvalWS {
  EvalLane* lanes = nullptr;
  EvalItem* it1 = nullptr;
  EvalItem* it2 = nullptr;
  double2* rho = nullptr;
  double2* rhow = nullptr;
  double2* part = nullptr;
  EvalPlan plan{};

  cudaError_t alloc(const cco_problem* p, int B, cudaStream_t st) {
    const int M = p->M, nt1 = p->host.ntile1, nt2 = p->host.ntile2;
    cudaError_t e = pool_alloc(&lanes, sizeof(EvalLane) * B, st);
    if (e == cudaSuccess) e = pool_alloc(&it1, sizeof(EvalItem) * (size_t)B * nt1, st);
    if (e == cudaSuccess) e = pool_alloc(&it2, sizeof(EvalItem) * (size_t)B * nt2, st);
    if (e == cudaSuccess) e = pool_alloc(&rho, sizeof(double2) * (size_t)B * M, st);
    if (e == cudaSuccess) e = pool_alloc(&rhow, sizeof(double2) * (size_t)B * M, st);
    if (e == cudaSuccess) e = pool_alloc(&part, sizeof(double2) * (size_t)B * nt1 * M, st);
    return e;
  }
  cudaError_t build(const cco_problem* p, int B, const double* s, size_t s_stride, double* f,
                    size_t f_stride, double* g, size_t g_stride, const int64_t* status,
                    size_t status_stride, cudaStream_t st) {
    const int nt1 = p->host.ntile1, nt2 = p->host.ntile2;
    const int total = B * std::max(nt1, nt2) + B;
    const int blocks = std::min(1024, (total + 255) / 256);
    k_make_lanes<<<blocks, 256, 0, st>>>(lanes, it1, it2, B, nt1, nt2, total, s, s_stride, f, f_stride,
                                         g, g_stride, rho, rhow, part, p->M, status,
                                         status_stride);
    plan.probs = p->dev;
    plan.lanes = lanes;
    plan.items1 = it1;
    plan.items2 = it2;
    plan.n_lanes = B;
    plan.n_items1 = B * nt1;
    plan.n_items2 = B * nt2;
    plan.max_d = p->d;
    plan.smem1 = p->smem1;
    plan.smem2 = p->smem2;
    plan.want_grad = g != nullptr;
    return cudaGetLastError();
  }
  void release(cudaStream_t st) {
    cudaFreeAsync(lanes, st);
    cudaFreeAsync(it1, st);
    cudaFreeAsync(it2, st);
    cudaFreeAsync(rho, st);
    cudaFreeAsync(rhow, st);
    cudaFreeAsync(part, st);
    lanes = nullptr;
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
  const size_t nt1 = (size_t)p->host.ntile1, nt2 = (size_t)p->host.ntile2;
  const size_t b_lanes = round256(sizeof(EvalLane) * B);
  const size_t b_it1 = round256(sizeof(EvalItem) * B * nt1);
  const size_t b_it2 = round256(sizeof(EvalItem) * B * nt2);
  const size_t b_rho = round256(sizeof(double2) * B * M);
  const size_t b_part = round256(sizeof(double2) * B * nt1 * M);
  const size_t need = b_lanes + b_it1 + b_it2 + 2 * b_rho + b_part;
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
  const size_t nd = (size_t)p->N * p->d;
  CCO_CUDA(ws.build(p, batch, s, nd, phi, 1, grad, nd, nullptr, 0, st));
  CCO_CUDA(eval_launch(ws.plan, st));
  return CCO_OK;
}

// ------------------------------------------------------------ relax drivers
namespace {

// Runs ticks (one evaluation + one update per running lane) in captured CUDA
// graphs of kGraphTicks ticks until no lane is RUNNING or the tick bound is
// reached. The lanes are split into `nbr` independent branches of the graph:
// a branch's FP64-bound evaluation overlaps another branch's HBM-bound
// minimizer update on the device. Completion is checked kInflight graphs
// behind, so host or driver hiccups (a clock sampler, a busy CPU) do not
// leave the device idle; lanes already finished make the surplus graphs
// near-empty launches.
constexpr int kGraphTicks = 16;
constexpr int kInflight = 3;
constexpr int kMaxBranches = 4;

int branch_count(int B) {
  int nbr = 2;
  if (const char* env = getenv("CCO_BRANCHES")) nbr = atoi(env);
  nbr = std::max(1, std::min(nbr, kMaxBranches));
  while (nbr > 1 && B / nbr < 32) --nbr;
  return nbr;
}

template <class TickFn>
int run_ticks(cudaStream_t st, int nbr, TickFn tick, const int64_t* status, size_t stride, int B,
              int64_t max_ticks, int64_t* ticks_out) {
  constexpr int kSlots = kInflight + 1;
  int* d_count = nullptr;
  // pinned completion counters: allocated once per host thread (cudaMallocHost
  // is slow and may synchronize, so it stays out of every call)
  static thread_local int* h_count = nullptr;
  CCO_CUDA(pool_alloc(&d_count, kSlots * sizeof(int), st));
  if (h_count == nullptr) CCO_CUDA(cudaMallocHost(&h_count, kSlots * sizeof(int)));
  cudaEvent_t ev[kSlots];
  for (int i = 0; i < kSlots; ++i) CCO_CUDA(cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming));
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int rc = CCO_OK;
  // capture kGraphTicks ticks of every branch; branches fork from and join
  // back into the first capture stream
  cudaStream_t cap[kMaxBranches];
  cudaEvent_t fork, join[kMaxBranches];
  for (int b = 0; b < nbr; ++b) CCO_CUDA(cudaStreamCreateWithFlags(&cap[b], cudaStreamNonBlocking));
  CCO_CUDA(cudaEventCreateWithFlags(&fork, cudaEventDisableTiming));
  for (int b = 0; b < nbr; ++b) CCO_CUDA(cudaEventCreateWithFlags(&join[b], cudaEventDisableTiming));
  cudaError_t e = cudaStreamBeginCapture(cap[0], cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    e = cudaEventRecord(fork, cap[0]);
    for (int b = 1; b < nbr && e == cudaSuccess; ++b) e = cudaStreamWaitEvent(cap[b], fork, 0);
    for (int t = 0; t < kGraphTicks && e == cudaSuccess; ++t)
      for (int b = 0; b < nbr && e == cudaSuccess; ++b) e = tick(cap[b], b);
    for (int b = 1; b < nbr && e == cudaSuccess; ++b) {
      e = cudaEventRecord(join[b], cap[b]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(cap[0], join[b], 0);
    }
    cudaError_t e2 = cudaStreamEndCapture(cap[0], &graph);
    if (e == cudaSuccess) e = e2;
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  int64_t ticks = 0;
  int launched = 0, checked = 0;
  bool done = false;
  while (e == cudaSuccess && !done) {
    if (ticks >= max_ticks) break;
    e = cudaGraphLaunch(exec, st);
    if (e != cudaSuccess) break;
    ticks += kGraphTicks;
    const int slot = launched % kSlots;
    e = count_running(status, stride, B, d_count + slot, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_count + slot, d_count + slot, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaEventRecord(ev[slot], st);
    ++launched;
    if (e == cudaSuccess && launched - checked > kInflight) {
      const int old = checked % kSlots;
      e = cudaEventSynchronize(ev[old]);
      ++checked;
      if (e == cudaSuccess && h_count[old] == 0) done = true;
    }
  }
  // drain the launches still in flight, oldest first
  while (e == cudaSuccess && !done && checked < launched) {
    const int old = checked % kSlots;
    e = cudaEventSynchronize(ev[old]);
    ++checked;
    if (e == cudaSuccess && h_count[old] == 0) done = true;
  }
  if (e != cudaSuccess) rc = cuda_fail(e, "relax ticks");
  else if (!done) rc = fail(CCO_ERR_ROUNDS, "relax did not finish within the round bound (%lld ticks)", (long long)max_ticks);
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  for (int b = 0; b < nbr; ++b) {
    cudaStreamDestroy(cap[b]);
    cudaEventDestroy(join[b]);
  }
  cudaEventDestroy(fork);
  for (int i = 0; i < kSlots; ++i) cudaEventDestroy(ev[i]);
  cudaFreeAsync(d_count, st);
  cudaStreamSynchronize(st);
  if (ticks_out) *ticks_out = ticks;
  return rc;
}

// Lanes of one relaxation: each lane has its own problem (mixed N, d and
// k-set) or all lanes share one. Positions are packed in the caller's
// buffers (soff, N_i d_i each); the device lane vectors use padded lengths
// (voff, ld_i).
struct LaneSet {
  int B = 0, device = 0;
  std::vector<const cco_problem*> prob;   // [B]
  std::vector<int> nd, ld;                 // [B]
  std::vector<int64_t> soff, voff;         // [B]
  int64_t s_total = 0, v_total = 0;
  int max_ld = 0;
  std::vector<const cco_problem*> uniq;    // distinct problems
  std::vector<int> pidx;                   // [B] index into uniq
};

int make_laneset(cco_problem* const* probs, int B, int pad, LaneSet* L) {
  if (B < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  L->B = B;
  L->prob.resize(B);
  L->nd.resize(B);
  L->ld.resize(B);
  L->soff.resize(B);
  L->voff.resize(B);
  L->pidx.resize(B);
  for (int i = 0; i < B; ++i) {
    const cco_problem* p = probs[i];
    if (!p) return fail(CCO_ERR_ARG, "null problem for lane %d", i);
    if (i == 0) L->device = p->device;
    if (p->device != L->device) return fail(CCO_ERR_ARG, "lanes must share one device");
    const int nd = p->N * p->d;
    const int ld = (nd + pad - 1) / pad * pad;
    L->prob[i] = p;
    L->nd[i] = nd;
    L->ld[i] = ld;
    L->soff[i] = L->s_total;
    L->voff[i] = L->v_total;
    L->s_total += nd;
    L->v_total += ld;
    L->max_ld = std::max(L->max_ld, ld);
    int u = 0;
    while (u < (int)L->uniq.size() && L->uniq[u] != p) ++u;
    if (u == (int)L->uniq.size()) L->uniq.push_back(p);
    L->pidx[i] = u;
  }
  return CCO_OK;
}

template <class T>
cudaError_t upload(T** dst, const std::vector<T>& src, cudaStream_t st) {
  cudaError_t e = pool_alloc(dst, sizeof(T) * std::max<size_t>(src.size(), 1), st);
  if (e == cudaSuccess && !src.empty())
    e = cudaMemcpyAsync(*dst, src.data(), sizeof(T) * src.size(), cudaMemcpyHostToDevice, st);
  return e;
}

// Evaluation plan of lanes [lo, hi) of a lane set, built on the host.
struct EvalSet {
  ProbDev* probs = nullptr;
  EvalLane* lanes = nullptr;
  EvalItem* it1 = nullptr;
  EvalItem* it2 = nullptr;
  double2* dens = nullptr;   // rho, w rho and the pass-1 partials of every lane
  EvalPlan plan{};

  cudaError_t build(const LaneSet& L, int lo, int hi, double* s_base, double* f_base,
                    double* g_base, const int64_t* status_base, size_t status_stride,
                    cudaStream_t st) {
    std::vector<ProbDev> pv;
    size_t smem1 = 0, smem2 = 0;
    int max_d = 1;
    for (const cco_problem* p : L.uniq) {
      pv.push_back(p->host);
      smem1 = std::max(smem1, p->smem1);
      smem2 = std::max(smem2, p->smem2);
      max_d = std::max(max_d, p->d);
    }
    size_t dn = 0;
    for (int i = lo; i < hi; ++i) dn += (size_t)L.prob[i]->M * (2 + L.prob[i]->host.ntile1);
    cudaError_t e = pool_alloc(&dens, sizeof(double2) * std::max<size_t>(dn, 1), st);
    std::vector<EvalLane> lv;
    std::vector<EvalItem> i1, i2;
    size_t o = 0;
    for (int i = lo; i < hi; ++i) {
      const cco_problem* p = L.prob[i];
      const size_t M = p->M;
      EvalLane ln{};
      ln.s = s_base + L.voff[i];
      ln.f = f_base + i;
      ln.g = g_base ? g_base + L.voff[i] : nullptr;
      ln.rho = dens + o;
      ln.rhow = dens + o + M;
      ln.part = dens + o + 2 * M;
      o += M * (2 + p->host.ntile1);
      ln.status = status_base ? status_base + (size_t)i * status_stride : nullptr;
      ln.prob = L.pidx[i];
      const int j = i - lo;
      for (int t = 0; t < p->host.ntile1; ++t) i1.push_back(EvalItem{j, t});
      for (int t = 0; t < p->host.ntile2; ++t) i2.push_back(EvalItem{j, t});
      lv.push_back(ln);
    }
    if (e == cudaSuccess) e = upload(&probs, pv, st);
    if (e == cudaSuccess) e = upload(&lanes, lv, st);
    if (e == cudaSuccess) e = upload(&it1, i1, st);
    if (e == cudaSuccess) e = upload(&it2, i2, st);
    plan.probs = probs;
    plan.lanes = lanes;
    plan.items1 = it1;
    plan.items2 = it2;
    plan.n_lanes = hi - lo;
    plan.n_items1 = (int)i1.size();
    plan.n_items2 = (int)i2.size();
    plan.max_d = max_d;
    plan.smem1 = smem1;
    plan.smem2 = smem2;
    plan.want_grad = g_base != nullptr;
    return e;
  }
  void release(cudaStream_t st) {
    cudaFreeAsync(probs, st);
    cudaFreeAsync(lanes, st);
    cudaFreeAsync(it1, st);
    cudaFreeAsync(it2, st);
    cudaFreeAsync(dens, st);
  }
};

bool out_ok(const cco_relax_out* o) {
  return o && o->s && o->energy && o->grad_norm && o->n_evals && o->n_iters && o->status;
}

// Device copies of the lane layout arrays (offsets and lengths).
struct LaneArrays {
  int64_t *voff = nullptr, *soff = nullptr, *toff = nullptr, *hoff = nullptr;
  int *lnd = nullptr, *lld = nullptr;
  cudaError_t build(const LaneSet& L, int64_t cap, int m, cudaStream_t st) {
    std::vector<int64_t> th(L.B), hh(L.B);
    int64_t t = 0, h = 0;
    for (int i = 0; i < L.B; ++i) {
      th[i] = t;
      hh[i] = h;
      t += cap * L.nd[i];
      h += (int64_t)m * L.ld[i];
    }
    cudaError_t e = upload(&voff, L.voff, st);
    if (e == cudaSuccess) e = upload(&soff, L.soff, st);
    if (e == cudaSuccess) e = upload(&toff, th, st);
    if (e == cudaSuccess) e = upload(&hoff, hh, st);
    if (e == cudaSuccess) e = upload(&lnd, L.nd, st);
    if (e == cudaSuccess) e = upload(&lld, L.ld, st);
    return e;
  }
  int64_t hist_total(const LaneSet& L, int m) const {
    int64_t h = 0;
    for (int i = 0; i < L.B; ++i) h += (int64_t)m * L.ld[i];
    return h;
  }
  void release(cudaStream_t st) {
    cudaFreeAsync(voff, st);
    cudaFreeAsync(soff, st);
    cudaFreeAsync(toff, st);
    cudaFreeAsync(hoff, st);
    cudaFreeAsync(lnd, st);
    cudaFreeAsync(lld, st);
  }
};

int check_traj(const cco_relax_out* out, bool rec) {
  if (rec && (!out->traj_s || !out->traj_energy || !out->traj_step || !out->traj_iteration ||
              !out->traj_count))
    return fail(CCO_ERR_ARG, "trajectory recording needs the traj_* outputs");
  return CCO_OK;
}

int relax_descent_set(const LaneSet& L, cudaStream_t st, const double* s0,
                      const cco_descent_settings* cfg, cco_relax_out* out) {
  if (!cfg || !s0) return fail(CCO_ERR_ARG, "null argument");
  if (!out_ok(out)) return fail(CCO_ERR_ARG, "incomplete output struct");
  if (cfg->max_evals < 0) return fail(CCO_ERR_ARG, "max_evals must be >= 0");
  const bool rec = cfg->record_every > 0 && cfg->max_records > 0;
  if (check_traj(out, rec) != CCO_OK) return CCO_ERR_ARG;
  DeviceGuard guard(L.device);
  const int B = L.B;
  const size_t V = L.v_total;
  DescentArgs a{};
  a.B = B;
  a.step_init = cfg->step_init;
  a.step_min = cfg->step_min;
  a.shrink = cfg->shrink;
  a.grow = cfg->grow;
  a.rel_tol = cfg->rel_tol;
  a.energy_tol = cfg->energy_tol;
  a.max_iters = cfg->max_evals / 2;
  a.rec_every = rec ? cfg->record_every : 1;
  a.rec_cap = rec ? cfg->max_records : 0;
  LaneArrays la;
  CCO_CUDA(la.build(L, a.rec_cap, 0, st));
  a.voff = la.voff;
  a.soff = la.soff;
  a.toff = la.toff;
  a.lnd = la.lnd;
  double* vec = nullptr;   // s, g, ps, pg
  double* sc = nullptr;    // f, step, norm, pf
  int64_t* ic = nullptr;   // it, n_evals, status, t0, t1
  int* ph = nullptr;       // phase, nonzero
  CCO_CUDA(pool_alloc(&vec, sizeof(double) * V * 4, st));
  CCO_CUDA(pool_alloc(&sc, sizeof(double) * B * 4, st));
  CCO_CUDA(pool_alloc(&ic, sizeof(int64_t) * B * 5, st));
  CCO_CUDA(pool_alloc(&ph, sizeof(int) * B * 2, st));
  a.s = vec;
  a.g = vec + V;
  a.ps = vec + 2 * V;
  double* pg = vec + 3 * V;
  a.pg = pg;
  a.f = sc;
  a.step = sc + B;
  a.norm = sc + 2 * B;
  double* pf = sc + 3 * B;
  a.pf = pf;
  a.it = ic;
  a.n_evals = ic + B;
  a.status = ic + 2 * B;
  a.t0 = ic + 3 * B;
  a.t1 = ic + 4 * B;
  a.phase = ph;
  a.nonzero = ph + B;
  if (rec) {
    a.traj_s = out->traj_s;
    a.traj_e = out->traj_energy;
    a.traj_step = out->traj_step;
    a.traj_it = out->traj_iteration;
    a.traj_count = out->traj_count;
  }
  const int nbr = branch_count(B);
  EvalSet ws[kMaxBranches];
  DescentArgs ab[kMaxBranches];
  for (int b = 0; b < nbr; ++b) {
    const int lo = b * B / nbr, hi = (b + 1) * B / nbr;
    DescentArgs r = a;
    r.B = hi - lo;
    r.voff += lo; r.soff += lo; r.toff += lo; r.lnd += lo;
    r.pf += lo; r.f += lo; r.step += lo; r.norm += lo;
    r.it += lo; r.n_evals += lo; r.status += lo; r.phase += lo; r.nonzero += lo;
    r.t0 += lo; r.t1 += lo;
    if (rec) {
      r.traj_e += (size_t)lo * a.rec_cap;
      r.traj_step += (size_t)lo * a.rec_cap;
      r.traj_it += (size_t)lo * a.rec_cap;
      r.traj_count += lo;
    }
    ab[b] = r;
    CCO_CUDA(ws[b].build(L, lo, hi, a.ps, pf, pg, a.status, 1, st));
  }
  CCO_CUDA(descent_init(a, s0, st));
  auto tick = [&](cudaStream_t s, int b) -> cudaError_t {
    cudaError_t e = eval_launch(ws[b].plan, s);
    if (e == cudaSuccess) e = descent_update(ab[b], s);
    return e;
  };
  const int64_t max_ticks = 1 + a.max_iters + (kInflight + 1) * kGraphTicks;
  int64_t ticks = 0;
  int rc = run_ticks(st, nbr, tick, a.status, 1, B, max_ticks, &ticks);
  if (rc == CCO_OK) {
    cudaError_t e = descent_finalize(a, out->s, out->energy, out->grad_norm, out->n_evals,
                                     out->n_iters, out->status, out->latency_ns, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "descent_finalize");
  }
  out->ticks = ticks;
  out->launches = ticks * 4 * nbr + ticks / kGraphTicks + 2;
  for (int b = 0; b < nbr; ++b) ws[b].release(st);
  la.release(st);
  cudaFreeAsync(vec, st);
  cudaFreeAsync(sc, st);
  cudaFreeAsync(ic, st);
  cudaFreeAsync(ph, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "relax descent");
  return rc;
}

int relax_lbfgs_set(const LaneSet& L, cudaStream_t st, const double* s0,
                    const cco_lbfgs_settings* cfg, cco_relax_out* out) {
  if (!cfg || !s0) return fail(CCO_ERR_ARG, "null argument");
  if (!out_ok(out)) return fail(CCO_ERR_ARG, "incomplete output struct");
  if (cfg->n_rescales < 1 || cfg->n_rescales > CCO_MAX_RESCALES)
    return fail(CCO_ERR_ARG, "need 1..%d rescale passes", CCO_MAX_RESCALES);
  if (cfg->memory < 1) return fail(CCO_ERR_ARG, "memory must be >= 1");
  if (cfg->memory > 256) return fail(CCO_ERR_ARG, "memory must be <= 256 on this build");
  if (cfg->max_linesearch_steps < 1) return fail(CCO_ERR_ARG, "max_linesearch_steps must be >= 1");
  const bool rec = cfg->record_every > 0 && cfg->max_records > 0;
  if (check_traj(out, rec) != CCO_OK) return CCO_ERR_ARG;
  DeviceGuard guard(L.device);
  const int B = L.B;
  const size_t V = L.v_total;
  const int m = (int)cfg->memory;
  LbArgs A{};
  A.B = B;
  A.m = m;
  A.n_pass = cfg->n_rescales;
  for (int i = 0; i < CCO_MAX_RESCALES; ++i) A.rescales[i] = i < cfg->n_rescales ? cfg->rescales[i] : 1.0;
  A.energy_tol = cfg->energy_tol;
  A.grad_tol = cfg->grad_tol;
  A.budget = cfg->max_evals_per_pass;
  A.patience = cfg->stagnation_patience;
  A.max_ls = cfg->max_linesearch_steps;
  A.rec_every = rec ? cfg->record_every : 1;
  A.rec_cap = rec ? cfg->max_records : 0;
  const size_t tri_bytes = lbfgs_update_smem(m);
  const bool in_smem = tri_bytes <= 200 * 1024;
  A.smem_tri = in_smem ? tri_bytes : 0;
  if (in_smem) {
    static std::mutex mu;
    static size_t configured = 0;
    std::lock_guard<std::mutex> lk(mu);
    if (tri_bytes > configured) {
      CCO_CUDA(lbfgs_configure(200 * 1024));
      configured = 200 * 1024;
    }
  }
  LaneArrays la;
  CCO_CUDA(la.build(L, A.rec_cap, m, st));
  A.voff = la.voff;
  A.soff = la.soff;
  A.toff = la.toff;
  A.hoff = la.hoff;
  A.lnd = la.lnd;
  A.lld = la.lld;
  const size_t H = la.hist_total(L, m);
  LbState* stv = nullptr;
  double* vec = nullptr;   // x, s, g, dir, glo, ps, pg
  double* hist = nullptr;  // S, Y
  double* dots = nullptr;  // SY, YY
  double* pf = nullptr;
  double* trig = nullptr;
  double* scal = nullptr;
  CCO_CUDA(pool_alloc(&stv, sizeof(LbState) * B, st));
  CCO_CUDA(pool_alloc(&vec, sizeof(double) * V * 7, st));
  CCO_CUDA(cudaMemsetAsync(vec, 0, sizeof(double) * V * 7, st));
  CCO_CUDA(pool_alloc(&hist, sizeof(double) * H * 2, st));
  CCO_CUDA(pool_alloc(&dots, sizeof(double) * (size_t)B * m * m * 2, st));
  CCO_CUDA(pool_alloc(&pf, sizeof(double) * B, st));
  if (!in_smem) CCO_CUDA(pool_alloc(&trig, tri_bytes * B, st));
  A.nblkB = (int)((L.max_ld / 2 + 255) / 256);
  A.scal_stride = (4 * m + 1 + A.nblkB + 1) & ~1;
  CCO_CUDA(pool_alloc(&scal, sizeof(double) * (size_t)A.scal_stride * B, st));
  A.scal = scal;
  A.st = stv;
  A.x = vec;
  A.s = vec + V;
  A.g = vec + 2 * V;
  A.dir = vec + 3 * V;
  A.glo = vec + 4 * V;
  A.ps = vec + 5 * V;
  double* pg = vec + 6 * V;
  A.pg = pg;
  A.pf = pf;
  A.Sh = hist;
  A.Yh = hist + H;
  A.SYs = dots;
  A.YYs = dots + (size_t)B * m * m;
  A.tri_g = trig;
  if (rec) {
    A.traj_s = out->traj_s;
    A.traj_e = out->traj_energy;
    A.traj_step = out->traj_step;
    A.traj_it = out->traj_iteration;
    A.traj_count = out->traj_count;
  }
  const size_t st_stride = sizeof(LbState) / sizeof(int64_t);
  const int64_t* status0 = &stv->status;
  const int nbr = branch_count(B);
  EvalSet ws[kMaxBranches];
  LbArgs Ab[kMaxBranches];
  for (int b = 0; b < nbr; ++b) {
    const int lo = b * B / nbr, hi = (b + 1) * B / nbr;
    LbArgs r = A;
    r.B = hi - lo;
    r.st += lo;
    r.pf += lo;
    r.voff += lo; r.soff += lo; r.toff += lo; r.hoff += lo; r.lnd += lo; r.lld += lo;
    r.SYs += (size_t)lo * m * m;
    r.YYs += (size_t)lo * m * m;
    if (r.tri_g) r.tri_g += (size_t)lo * ((size_t)m * (m + 1));
    r.scal += (size_t)lo * A.scal_stride;
    if (rec) {
      r.traj_e += (size_t)lo * A.rec_cap;
      r.traj_step += (size_t)lo * A.rec_cap;
      r.traj_it += (size_t)lo * A.rec_cap;
      r.traj_count += lo;
    }
    Ab[b] = r;
    CCO_CUDA(ws[b].build(L, lo, hi, A.ps, pf, pg, status0, st_stride, st));
  }
  CCO_CUDA(lbfgs_init(A, s0, st));
  auto tick = [&](cudaStream_t s, int b) -> cudaError_t {
    cudaError_t e = eval_launch(ws[b].plan, s);
    if (e == cudaSuccess) e = lbfgs_update(Ab[b], s);
    return e;
  };
  const int64_t max_ticks =
      1 + (int64_t)cfg->n_rescales * (cfg->max_evals_per_pass + cfg->max_linesearch_steps + 1) +
      (kInflight + 1) * kGraphTicks;
  int64_t ticks = 0;
  int rc = run_ticks(st, nbr, tick, status0, st_stride, B, max_ticks, &ticks);
  if (rc == CCO_OK) {
    cudaError_t e = lbfgs_finalize(A, out->s, out->energy, out->grad_norm, out->n_evals,
                                   out->n_iters, out->status, out->latency_ns, st);
    if (e != cudaSuccess) rc = cuda_fail(e, "lbfgs_finalize");
  }
  out->ticks = ticks;
  out->launches = ticks * 7 * nbr + ticks / kGraphTicks + 2;
  for (int b = 0; b < nbr; ++b) ws[b].release(st);
  la.release(st);
  cudaFreeAsync(stv, st);
  cudaFreeAsync(vec, st);
  cudaFreeAsync(hist, st);
  cudaFreeAsync(dots, st);
  cudaFreeAsync(pf, st);
  if (trig) cudaFreeAsync(trig, st);
  cudaFreeAsync(scal, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (rc == CCO_OK && e != cudaSuccess) rc = cuda_fail(e, "relax lbfgs");
  return rc;
}

}  // namespace

extern "C" int cco_relax_descent(cco_problem* p, void* stream, int batch, const double* s0,
                                 const cco_descent_settings* cfg, int chunk_iters,
                                 cco_relax_out* out) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  std::vector<cco_problem*> probs(batch, p);
  LaneSet L;
  if (make_laneset(probs.data(), batch, 1, &L) != CCO_OK) return CCO_ERR_ARG;
  return relax_descent_set(L, (cudaStream_t)stream, s0, cfg, out);
}

extern "C" int cco_relax_lbfgs(cco_problem* p, void* stream, int batch, const double* s0,
                               const cco_lbfgs_settings* cfg, int chunk_iters,
                               cco_relax_out* out) {
  if (!p) return fail(CCO_ERR_ARG, "null problem");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  if (batch < 1) return fail(CCO_ERR_ARG, "need at least one configuration");
  std::vector<cco_problem*> probs(batch, p);
  LaneSet L;
  if (make_laneset(probs.data(), batch, 4, &L) != CCO_OK) return CCO_ERR_ARG;
  return relax_lbfgs_set(L, (cudaStream_t)stream, s0, cfg, out);
}

extern "C" int cco_relax_descent_mixed(cco_problem* const* problems, void* stream, int batch,
                                       const double* s0, const cco_descent_settings* cfg,
                                       int chunk_iters, cco_relax_out* out) {
  if (!problems) return fail(CCO_ERR_ARG, "null problem array");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  LaneSet L;
  if (make_laneset(problems, batch, 1, &L) != CCO_OK) return CCO_ERR_ARG;
  return relax_descent_set(L, (cudaStream_t)stream, s0, cfg, out);
}

extern "C" int cco_relax_lbfgs_mixed(cco_problem* const* problems, void* stream, int batch,
                                     const double* s0, const cco_lbfgs_settings* cfg,
                                     int chunk_iters, cco_relax_out* out) {
  if (!problems) return fail(CCO_ERR_ARG, "null problem array");
  if (chunk_iters < 1) return fail(CCO_ERR_ARG, "chunk_iters must be positive");
  LaneSet L;
  if (make_laneset(problems, batch, 4, &L) != CCO_OK) return CCO_ERR_ARG;
  return relax_lbfgs_set(L, (cudaStream_t)stream, s0, cfg, out);
}
