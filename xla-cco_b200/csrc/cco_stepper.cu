// cco_stepper.cu - relaxations whose energy the caller evaluates.
//
// The reference's relax takes any AbstractEnergy (src/xla_cco/minimize/
// __init__.py:102-107, src/xla_cco/energy.py:115-137): the minimizers only
// call energy.value_and_grad. Here a stepper runs the same device state
// machines as cco_relax_descent / cco_relax_lbfgs (the same lane records and
// update kernels) but leaves each tick's evaluation to the caller: it hands
// out the probe positions of every lane, takes back the energies and
// gradients, and advances the lanes by one tick. Finished lanes are frozen
// exactly as in the fused path; the caller stops when no lane runs.
#include <cuda_runtime.h>

#include <vector>

#include "cco_host.cuh"
#include "cco_internal.cuh"
#include "cco_opt.cuh"

namespace cco {
int lbfgs_args(const cco_lbfgs_settings* cfg, LbArgs* A, RecordShape* shape);
}

using namespace cco;

struct cco_stepper {
  int device = 0;
  Method method = Method::Lbfgs;
  int B = 0, N = 0, d = 0, nd = 0, ld = 0;
  size_t rec_doubles = 0;
  size_t pf_off = 0, ps_off = 0, pg_off = 0;   // offsets inside a record
  std::vector<LaneRef> refs;
  LaneRef* d_refs = nullptr;
  double* records = nullptr;
  int* d_count = nullptr;
  int* h_count = nullptr;   // pinned
  DescentArgs ds{};
  LbArgs lb{};
  int64_t ticks = 0;
};

namespace {

__global__ void k_step_gather(const LaneRef* __restrict__ refs, int B, size_t ps_off, int nd,
                              double* __restrict__ out) {
  const int b = blockIdx.y;
  if (b >= B) return;
  const double* ps = refs[b].rec + ps_off;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < nd; e += gridDim.x * blockDim.x)
    out[(size_t)b * nd + e] = ps[e];
}

// The caller's evaluation of the probes into the records of RUNNING lanes
// (a frozen lane's record is never written again); gradient padding is zero.
__global__ void k_step_scatter(const LaneRef* __restrict__ refs, int B, size_t pf_off,
                               size_t pg_off, int nd, int ld, const double* __restrict__ f,
                               const double* __restrict__ g) {
  const int b = blockIdx.y;
  if (b >= B) return;
  double* rec = refs[b].rec;
  if (*rec_status(rec) != CCO_STATUS_RUNNING) return;
  double* pg = rec + pg_off;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < ld; e += gridDim.x * blockDim.x)
    pg[e] = e < nd ? g[(size_t)b * nd + e] : 0.0;
  if (blockIdx.x == 0 && threadIdx.x == 0) rec[pf_off] = f[b];
}

int grid_x(int nd) { return std::max(1, std::min(64, (nd + 255) / 256)); }

}  // namespace

extern "C" {

int cco_stepper_create(int device, void* stream, int method, const void* settings, int batch,
                       int n_particles, int d, const double* s0, cco_stepper** out) {
  if (!out) return fail(CCO_ERR_ARG, "out is null");
  *out = nullptr;
  if (!settings || !s0) return fail(CCO_ERR_ARG, "null settings or s0");
  if (method != 0 && method != 1) return fail(CCO_ERR_ARG, "method must be 0 (descent) or 1 (L-BFGS)");
  if (batch < 1 || n_particles < 1 || d < 1) return fail(CCO_ERR_ARG, "need batch, N, d >= 1");
  if (batch > 65535) return fail(CCO_ERR_ARG, "batch %d > 65535: split it", batch);
  int ndev = 0;
  if (cco_device_count(&ndev) != CCO_OK) return CCO_ERR_NODEVICE;
  if (device < 0 || device >= ndev) return fail(CCO_ERR_ARG, "device %d out of range", device);
  DeviceGuard guard(device);
  cudaStream_t st = (cudaStream_t)stream;
  auto* h = new cco_stepper();
  h->device = device;
  h->B = batch;
  h->N = n_particles;
  h->d = d;
  h->nd = n_particles * d;
  h->ld = pad4(h->nd);
  if (method == 0) {
    const auto* cfg = static_cast<const cco_descent_settings*>(settings);
    if (cfg->max_evals < 0) {
      delete h;
      return fail(CCO_ERR_ARG, "max_evals must be >= 0");
    }
    if (cfg->record_every > 0 && cfg->max_records > 0) {
      delete h;
      return fail(CCO_ERR_ARG, "trajectory recording is not available for caller-evaluated relaxations");
    }
    h->method = Method::Descent;
    DescentArgs& a = h->ds;
    a.step_init = cfg->step_init;
    a.step_min = cfg->step_min;
    a.shrink = cfg->shrink;
    a.grow = cfg->grow;
    a.rel_tol = cfg->rel_tol;
    a.energy_tol = cfg->energy_tol;
    a.max_iters = cfg->max_evals / 2;
    a.rec_every = 1;
    a.rec_cap = 0;
    h->rec_doubles = (ds_record_doubles(h->ld, 0, 0) + 31) & ~(size_t)31;
  } else {
    const auto* cfg = static_cast<const cco_lbfgs_settings*>(settings);
    if (cfg->n_rescales < 1 || cfg->n_rescales > CCO_MAX_RESCALES || cfg->memory < 1 ||
        cfg->memory > 256 || cfg->max_linesearch_steps < 1) {
      delete h;
      return fail(CCO_ERR_ARG, "invalid L-BFGS settings");
    }
    if (cfg->precision != 0) {
      delete h;
      return fail(CCO_ERR_ARG, "caller-evaluated relaxations are FP64 (precision 0)");
    }
    if (cfg->record_every > 0 && cfg->max_records > 0) {
      delete h;
      return fail(CCO_ERR_ARG, "trajectory recording is not available for caller-evaluated relaxations");
    }
    h->method = Method::Lbfgs;
    RecordShape shape;
    const int rc = lbfgs_args(cfg, &h->lb, &shape);
    if (rc != CCO_OK) {
      delete h;
      return rc;
    }
    h->rec_doubles = (lb_record_doubles(shape.m, shape.tri_len, h->ld, 0, 0) + 31) & ~(size_t)31;
    h->lb.nblkB = lb_nblk(h->ld);
    h->lb.nchA = lb_achunks(h->ld);
  }
  cudaError_t e = cudaMalloc(&h->records, h->rec_doubles * batch * sizeof(double));
  if (e == cudaSuccess) e = cudaMalloc(&h->d_refs, sizeof(LaneRef) * batch);
  if (e == cudaSuccess) e = cudaMalloc(&h->d_count, sizeof(int));
  if (e == cudaSuccess) e = cudaHostAlloc(&h->h_count, sizeof(int), cudaHostAllocDefault);
  if (e != cudaSuccess) {
    cco_stepper_destroy(h);
    return cuda_fail(e, "cco_stepper_create");
  }
  // offsets of the probe energy, probe positions and probe gradient in a record
  double* const base = h->records;
  if (h->method == Method::Descent) {
    const DsView v = ds_view(base, h->ld);
    h->pf_off = v.pf - base;
    h->ps_off = v.ps - base;
    h->pg_off = v.pg - base;
  } else {
    const LbView v = lb_view(base, h->lb.m, h->lb.tri_len, h->ld);
    h->pf_off = v.pf - base;
    h->ps_off = v.ps - base;
    h->pg_off = v.pg - base;
  }
  h->refs.resize(batch);
  for (int i = 0; i < batch; ++i) {
    LaneRef& r = h->refs[i];
    r.rec = h->records + (size_t)i * h->rec_doubles;
    r.nd = h->nd;
    r.ld = h->ld;
    r.soff = (int64_t)i * h->nd;
    r.toff = 0;
    r.idx = i;
    r.n = n_particles;
  }
  e = cudaMemcpyAsync(h->d_refs, h->refs.data(), sizeof(LaneRef) * batch, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    if (h->method == Method::Descent) {
      h->ds.B = batch;
      h->ds.lanes = h->d_refs;
      e = descent_init(h->ds, s0, st);
    } else {
      h->lb.B = batch;
      h->lb.lanes = h->d_refs;
      e = lbfgs_init(h->lb, s0, st);
    }
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);   // refs upload done before refs may change
  if (e != cudaSuccess) {
    cco_stepper_destroy(h);
    return cuda_fail(e, "cco_stepper_create");
  }
  *out = h;
  return CCO_OK;
}

int cco_stepper_probes(cco_stepper* h, void* stream, double* ps) {
  if (!h || !ps) return fail(CCO_ERR_ARG, "null argument");
  DeviceGuard guard(h->device);
  const dim3 grid(grid_x(h->nd), h->B);
  k_step_gather<<<grid, 256, 0, (cudaStream_t)stream>>>(h->d_refs, h->B, h->ps_off, h->nd, ps);
  CCO_CUDA(cudaGetLastError());
  return CCO_OK;
}

int cco_stepper_advance(cco_stepper* h, void* stream, const double* f, const double* g,
                        int64_t* n_running) {
  if (!h || !f || !g) return fail(CCO_ERR_ARG, "null argument");
  DeviceGuard guard(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  const dim3 grid(grid_x(h->ld), h->B);
  k_step_scatter<<<grid, 256, 0, st>>>(h->d_refs, h->B, h->pf_off, h->pg_off, h->nd, h->ld, f, g);
  CCO_CUDA(cudaGetLastError());
  if (h->method == Method::Descent) CCO_CUDA(descent_update(h->ds, st));
  else CCO_CUDA(lbfgs_update(h->lb, st));
  h->ticks += 1;
  if (n_running) {
    CCO_CUDA(count_running(h->d_refs, h->B, h->d_count, st));
    CCO_CUDA(cudaMemcpyAsync(h->h_count, h->d_count, sizeof(int), cudaMemcpyDeviceToHost, st));
    CCO_CUDA(cudaStreamSynchronize(st));
    *n_running = *h->h_count;
  }
  return CCO_OK;
}

int cco_stepper_finish(cco_stepper* h, void* stream, cco_relax_out* out) {
  if (!h || !out || !out->s || !out->energy || !out->grad_norm || !out->n_evals || !out->n_iters ||
      !out->status)
    return fail(CCO_ERR_ARG, "incomplete output struct");
  DeviceGuard guard(h->device);
  cudaStream_t st = (cudaStream_t)stream;
  if (h->method == Method::Descent)
    CCO_CUDA(descent_finalize(h->ds, out->s, out->energy, out->grad_norm, out->n_evals,
                              out->n_iters, out->status, out->latency_ns, st));
  else
    CCO_CUDA(lbfgs_finalize(h->lb, out->s, out->energy, out->grad_norm, out->n_evals,
                            out->n_iters, out->status, out->latency_ns, out->n_evals_fp32, st));
  out->ticks = h->ticks;
  out->launches = 0;
  out->branches = 0;
  out->graph_ticks = 0;
  return CCO_OK;
}

int cco_stepper_destroy(cco_stepper* h) {
  if (!h) return CCO_OK;
  DeviceGuard guard(h->device);
  if (h->records) cudaFree(h->records);   // cudaFree waits for the work that uses it
  if (h->d_refs) cudaFree(h->d_refs);
  if (h->d_count) cudaFree(h->d_count);
  if (h->h_count) cudaFreeHost(h->h_count);
  delete h;
  return CCO_OK;
}

}  // extern "C"
