/*
 * cco.h - C ABI of the B200-native collective-coordinate hot path.
 *
 * Plain pointers and sizes only. Every function returns an int status
 * (CCO_OK = 0); per-lane outcomes are written as the reference's status
 * codes 0..7 into caller-provided int64 arrays. Array arguments documented
 * "device" are CUDA device pointers on the problem's device; "host" are
 * ordinary host pointers. Streams are cudaStream_t passed as void*
 * (NULL = the legacy default stream).
 *
 * Reference interfaces replaced (paths inside sdawley1/xla-cco):
 *   cco_problem_create   <- make_stealthy_energy          src/xla_cco/energy.py:361-414
 *   cco_energy_grad      <- StealthyEnergy.value_grad_density / value_and_grad /
 *                           __call__ (trig path)         src/xla_cco/energy.py:186-225,301-324
 *                           and collective_density        src/xla_cco/energy.py:327-358
 *   cco_relax_descent    <- relax(energy, s0, DescentSettings, chunk_iters)
 *                                                         src/xla_cco/minimize/__init__.py:102-151
 *                                                         src/xla_cco/minimize/descent.py:121-209
 *   cco_relax_lbfgs      <- relax(energy, s0, LBFGSSettings, chunk_iters)
 *                                                         src/xla_cco/minimize/lbfgs.py:163-350
 *   cco_device_count     <- require_gpu                  src/xla_cco/_device.py:137-142
 *   cco_hessian          <- StealthyEnergy.hessian       src/xla_cco/energy.py:272-299
 * Each entry point is plain C so that an XLA FFI handler (or any other
 * foreign-function binding) can wrap it without C++ types.
 */
#ifndef CCO_H
#define CCO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CCO_ABI_VERSION 1

/* return codes */
#define CCO_OK 0
#define CCO_ERR_ARG 1        /* bad argument (Python: ValueError / TypeError)      */
#define CCO_ERR_OOM 2        /* device allocation failed                          */
#define CCO_ERR_ADMISSION 3  /* request refused by the HBM admission budget       */
#define CCO_ERR_DEVICE 4     /* CUDA error (Python: RuntimeError)                 */
#define CCO_ERR_TIMEOUT 5    /* a bounded wait ran out                            */
#define CCO_ERR_ROUNDS 6     /* relax did not finish within the round bound       */
#define CCO_ERR_NODEVICE 7   /* no CUDA device visible (Python: RuntimeError)     */

/* per-lane status codes (src/xla_cco/minimize/result.py:35-42) */
#define CCO_STATUS_RUNNING 0
#define CCO_STATUS_ENERGY_TOL 1
#define CCO_STATUS_STEP_FLOOR 2
#define CCO_STATUS_BUDGET 3
#define CCO_STATUS_STAGNATED 4
#define CCO_STATUS_LINESEARCH_FAIL 5
#define CCO_STATUS_GRAD_TOL 6
#define CCO_STATUS_DRIFT 7
#define CCO_STATUS_CANCELLED 8  /* serving pool only: the request was cancelled */

typedef struct cco_problem cco_problem;

/* Library / device queries. */
int cco_abi_version(void);
const char* cco_error_string(int code);
/* Message of the last failing call on this host thread ("" if none). */
const char* cco_last_error(void);
int cco_device_count(int* n_devices);

/*
 * A problem is one energy: the integer k-set (M rows of d int32, any order,
 * no all-zero row), per-row weights and the box volume, for N particles in
 * d = 1, 2 or 3 dimensions. It is uploaded once to `device` and reused by
 * every evaluation and relaxation. Outputs indexed by k use the caller's row
 * order. Host pointers.
 */
int cco_problem_create(int device, int d, int n_particles, int m,
                       const int32_t* n_vectors, const double* weights,
                       double volume, cco_problem** out);
int cco_problem_destroy(cco_problem* p);
/* Sizes of the device k-set layout (runs split into pass-1/pass-2 segments). */
int cco_problem_info(const cco_problem* p, int* d, int* n_particles, int* m,
                     int* n_seg1, int* n_seg2, int* table_rows);
/* Form of the FP64 density pass of a problem: *gemm_blocks > 0 when it runs
 * as a complex GEMM over (run group x last-axis window) blocks (d >= 2, dense
 * k-sets), 0 for the per-segment kernel. No reference counterpart. */
int cco_problem_pass1_form(const cco_problem* p, int* gemm_blocks);

/*
 * Energy, gradient and collective density of `batch` configurations.
 *   s      device [batch][N][d] fractional positions
 *   phi    device [batch]        Phi = (1/V) sum_k w_k |rho_k|^2
 *   grad   device [batch][N][d]  dPhi/ds (NULL: energy and density only)
 *   rho_re, rho_im device [batch][M] (NULL: not returned)
 * Deterministic: the same inputs give the same bits.
 */
int cco_energy_grad(cco_problem* p, void* stream, int batch, const double* s,
                    double* phi, double* grad, double* rho_re, double* rho_im);

/*
 * Closed-form Hessian d2 Phi / ds_ja ds_lb of `batch` configurations
 *   <- StealthyEnergy.hessian             src/xla_cco/energy.py:272-299
 * (the Jacobian of the ROS2 gradient flow, src/xla_cco/minimize/flow.py:367-398).
 *   s     device [batch][N][d] fractional positions
 *   hess  device [batch][N d][N d], row (j d + a), column (l d + b)
 * No (N, M) phase matrix is formed: the kernels build each k-chunk's phases
 * of a particle-tile pair in shared memory and exploit the symmetry. batch
 * <= 65535.
 */
int cco_hessian(cco_problem* p, void* stream, int batch, const double* s, double* hess);

/*
 * The mixed-precision evaluation that relaxations with precision = FP32 use
 * while a lane's energy is large (no reference counterpart; the reference is
 * FP64 only): phase tables seeded by FP64 sincospi and stored in FP32, FP32
 * phase recurrences, Kahan-compensated FP32 accumulation of each tile's
 * density, FP32 back-projection; the sum over tiles, rho, Phi and the final
 * gradient sums in FP64. Relative accuracy about 1e-6 of |rho| per term -
 * fine for descent far from the minimum, useless near Phi = 0, which is pure
 * cancellation. Same arguments as cco_energy_grad without the density.
 */
int cco_energy_grad_fp32(cco_problem* p, void* stream, int batch, const double* s,
                         double* phi, double* grad);

/*
 * cco_energy_grad without any allocation (no counterpart in the reference).
 *
 * For callers that must not allocate device memory during a call: code that
 * runs while a CUDA stream is being captured into a graph (cudaMalloc is
 * illegal there), code running under a custom or pre-reserved memory pool
 * that forbids outside allocations, and hard real-time loops that cannot
 * afford an allocator round trip. cco_energy_grad obtains its scratch (the
 * per-tile partial densities and the launch plan) from cudaMallocAsync on
 * every call; this variant carves it instead out of one fixed device array of
 * CCO_NOALLOC_SCRATCH_BYTES compiled into the library. Every GPU that loads
 * the library holds that array until the process exits.
 *
 * Same arguments and results as cco_energy_grad with rho_re = rho_im = NULL.
 * The problem itself is created beforehand (cco_problem_create allocates).
 * Limit: the scratch of one call, about batch * M * 16 * (2 + ceil(N / 64))
 * bytes plus the plan, must fit CCO_NOALLOC_SCRATCH_BYTES; a larger batch is
 * rejected with CCO_ERR_ARG and nothing is launched - split it into smaller
 * calls. The first call on each device resolves the array's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture. The resolved address is cached for the life of
 * the process: after cudaDeviceReset (or any teardown of the device's primary
 * context) it is stale, and this entry point must not be called again on that
 * device. All calls share the one array and nothing in it
 * needs to start at zero (every call writes all the scratch it reads), but
 * two calls that overlap on the GPU (different streams, or graph branches
 * without an ordering edge) race on it: order them.
 */
#define CCO_NOALLOC_SCRATCH_BYTES (16u << 20)
int cco_energy_grad_noalloc(cco_problem* p, void* stream, int batch, const double* s,
                            double* phi, double* grad);

/* Minimizer settings: same fields and meaning as the reference's settings. */
typedef struct {
  double step_init;    /* 1e-3  */
  double step_min;     /* 1e-15 */
  double shrink;       /* 0.5   */
  double grow;         /* 1.0   */
  double rel_tol;      /* 0.01  */
  int64_t max_evals;   /* 10000 */
  double energy_tol;   /* 0     */
  int64_t record_every;
  int64_t max_records;
} cco_descent_settings;

#define CCO_MAX_RESCALES 8
typedef struct {
  int64_t memory;                      /* 100 */
  int32_t n_rescales;                  /* 3   */
  int32_t precision;                   /* 0: FP64 throughout (the reference); 1: mixed -
                                          FP32 evaluations until Phi < 1e-6 N, then FP64
                                          (no reference counterpart) */
  double rescales[CCO_MAX_RESCALES];   /* 1e4, 1, 1e-2 */
  int64_t max_evals_per_pass;          /* 500000 */
  double energy_tol;                   /* 0 */
  double grad_tol;                     /* 0 */
  int64_t stagnation_patience;         /* 50 */
  int64_t max_linesearch_steps;        /* 30 */
  int64_t record_every;
  int64_t max_records;
} cco_lbfgs_settings;

/* Outputs of a relaxation: device arrays with a leading lane axis. */
typedef struct {
  double* s;            /* [B][N][d] final positions wrapped into [0, 1) */
  double* energy;       /* [B] */
  double* grad_norm;    /* [B] */
  int64_t* n_evals;     /* [B] reference counting (descent: 2 per iteration) */
  int64_t* n_iters;     /* [B] */
  int64_t* status;      /* [B] CCO_STATUS_* */
  /* trajectory (all NULL when recording is off; capacity max_records rows) */
  double* traj_s;       /* [B][max_records][N][d] wrapped */
  double* traj_energy;  /* [B][max_records] */
  double* traj_step;    /* [B][max_records] */
  int64_t* traj_iteration; /* [B][max_records] */
  int64_t* traj_count;  /* [B] */
  int64_t* latency_ns;  /* [B] optional: device time from the start of the call to the
                           lane's completion (%globaltimer), NULL to skip */
  int64_t* n_evals_fp32; /* [B] optional (L-BFGS): evaluations done in FP32 (precision = 1),
                           NULL to skip */
  int64_t ticks;        /* out: device ticks (one energy evaluation per running lane each) */
  int64_t launches;     /* out: kernel launches issued by the call */
  int32_t branches;     /* out: graph branches of the tick schedule used */
  int32_t graph_ticks;  /* out: ticks per captured graph of that schedule */
  int32_t overlap;      /* out: 1 if that schedule ran the branches half a tick apart with
                           the update kernels at high stream priority */
  int32_t reserved;     /* zero */
} cco_relax_out;

/*
 * Batched relaxation of `batch` configurations s0 (device [batch][N][d]).
 * Each lane runs its own state machine on the device; finished lanes are
 * frozen and skipped (on-device lane compaction). Results do not depend on
 * `chunk_iters`, which only sets how many device ticks run between host
 * completion checks. Returns CCO_ERR_ROUNDS if the reference's round bound
 * is exceeded.
 */
int cco_relax_descent(cco_problem* p, void* stream, int batch, const double* s0,
                      const cco_descent_settings* settings, int chunk_iters,
                      cco_relax_out* out);
int cco_relax_lbfgs(cco_problem* p, void* stream, int batch, const double* s0,
                    const cco_lbfgs_settings* settings, int chunk_iters,
                    cco_relax_out* out);

/*
 * Relaxations whose energy the caller evaluates  <- relax(energy, s0, settings)
 * with any AbstractEnergy          src/xla_cco/minimize/__init__.py:102-151,
 *                                  src/xla_cco/energy.py:115-137
 * The reference's minimizers only call energy.value_and_grad, so relax takes
 * any energy. A stepper runs the same device lanes as cco_relax_descent /
 * cco_relax_lbfgs (method 0 / 1, settings a cco_descent_settings or
 * cco_lbfgs_settings; FP64, no trajectory) and leaves every evaluation to the
 * caller:
 *   loop { cco_stepper_probes(h, st, ps)        ps: device [B][N][d] out, the
 *                                                positions to evaluate
 *          caller: f[B] = E(ps), g[B][N][d] = dE/ds at ps (device arrays)
 *          cco_stepper_advance(h, st, f, g, &n) one tick; n = lanes still running
 *   } until n == 0, then cco_stepper_finish(h, st, out) (the cco_relax_out
 * results, trajectory fields unused) and cco_stepper_destroy(h). s0: device
 * [B][N][d]. Lanes that have finished ignore further evaluations. batch <=
 * 65535.
 */
typedef struct cco_stepper cco_stepper;
int cco_stepper_create(int device, void* stream, int method, const void* settings, int batch,
                       int n_particles, int d, const double* s0, cco_stepper** out);
int cco_stepper_probes(cco_stepper* h, void* stream, double* ps);
int cco_stepper_advance(cco_stepper* h, void* stream, const double* f, const double* g,
                        int64_t* n_running);
int cco_stepper_finish(cco_stepper* h, void* stream, cco_relax_out* out);
int cco_stepper_destroy(cco_stepper* h);

/*
 * Mixed batches: lane i relaxes configuration i of problems[i], so one call
 * runs instances of different N, d and k-set side by side (the same
 * evaluation and minimizer launches serve every lane). All problems live on
 * one device. Positions are packed lane after lane without padding:
 *   s0, out->s      device, lane i at offset sum_{j<i} N_j d_j, N_i d_i doubles
 *   out->traj_s     device, lane i at offset max_records * sum_{j<i} N_j d_j
 * the per-lane scalars (energy, status, traj_energy rows, ...) keep their
 * [B] / [B][max_records] shapes. Each lane's result is bit-identical to the
 * same configuration relaxed by cco_relax_descent / cco_relax_lbfgs alone.
 * No reference counterpart: the reference relaxes one (energy, batch) pair
 * per call (src/xla_cco/minimize/__init__.py:102-151).
 */
int cco_relax_descent_mixed(cco_problem* const* problems, void* stream, int batch,
                            const double* s0, const cco_descent_settings* settings,
                            int chunk_iters, cco_relax_out* out);
int cco_relax_lbfgs_mixed(cco_problem* const* problems, void* stream, int batch,
                          const double* s0, const cco_lbfgs_settings* settings,
                          int chunk_iters, cco_relax_out* out);

/*
 * Gradient flow (adaptive Dormand-Prince 5(4)) of batch configurations,
 * lane i relaxing configuration i of problems[i] (repeat one problem for a
 * uniform batch). Replaces gradient_flow(energy, s0, basis, FlowSettings,
 * dt0) with method "dopri5" (src/xla_cco/minimize/flow.py:258-364,401-451),
 * vmapped over lanes. Same settings, stops, status precedence, clocks,
 * recording and evaluation count (6 per attempted step, 1 at the start).
 *   s0        device, packed as the mixed relaxations ([N_i][d_i] per lane)
 *   bases     host [batch][d_i][d_i] cell bases (rows = lattice vectors), packed
 *   dt0       host [batch] first step per lane (resume), or NULL for dt_init
 * Outputs (device): s (packed like s0, not wrapped), and per lane energy, t,
 * length, dt (next proposed step), n_steps, n_evals, status; with recording
 * traj_s ([max_records][N_i d_i] per lane, packed), traj_t, traj_length,
 * traj_energy ([batch][max_records]) and traj_count ([batch]).
 */
typedef struct {
  double rtol;          /* 1e-6  */
  double atol;          /* 1e-14 */
  double dt_init;       /* 1e-3  */
  double dt_min;        /* 1e-14 */
  double dt_max;        /* inf   */
  double t_max;         /* inf   */
  int64_t max_steps;    /* 200000 */
  double energy_tol;    /* 0 */
  double grad_tol;      /* 0 */
  int32_t arclength;    /* 0: parametrization "time", 1: "arclength" */
  int32_t pad_;
  int64_t record_every; /* 0 */
  int64_t max_records;  /* 0 */
} cco_flow_settings;

typedef struct {
  double* s;
  double* energy;
  double* t;
  double* length;
  double* dt;
  int64_t* n_steps;
  int64_t* n_evals;
  int64_t* status;
  double* traj_s;
  double* traj_t;
  double* traj_length;
  double* traj_energy;
  int64_t* traj_count;
  int64_t ticks;        /* out */
  int64_t launches;     /* out */
} cco_flow_out;

int cco_gradient_flow(cco_problem* const* problems, void* stream, int batch, const double* s0,
                      const double* bases, const double* dt0, const cco_flow_settings* settings,
                      cco_flow_out* out);

/*
 * Molecular-dynamics steps of batch lanes, lane i a configuration of
 * problems[i] in Cartesian coordinates r = s B (mass 1). Replaces repeated
 * verlet_step / andersen_reset / baoab_step (src/xla_cco/dynamics/
 * integrators.py:83-176) with the force F = -dPhi/ds B^-T of
 * value_grad_density(r B^-1) (dynamics/run.py:219-244); one force evaluation
 * per step, all steps on the device. Random draws (BAOAB noise, Andersen
 * coin, particle and velocity row) come from Philox4x32-10 keyed per lane and
 * counted by step, not from JAX's threefry streams.
 *   r0, v0   device, packed [N_i][d_i] per lane
 *   bases    host [batch][d_i][d_i] packed; keys host [batch][2] uint32
 *   acc0     host [batch] Andersen "count" accumulators, or NULL for 0
 * Outputs (device): r, v, f packed like r0, and per lane the energy Phi and
 * kinetic energy of the final state, the largest |E - E0| over the steps,
 * the Andersen reset count and accumulator, the next key, the status
 * (CCO_STATUS_BUDGET when the steps are done, CCO_STATUS_DRIFT if
 * drift_tol > 0 and |E - E0| exceeded it).
 */
typedef struct {
  double dt;
  int64_t n_steps;
  int32_t scheme;        /* 0: velocity Verlet, 1: BAOAB */
  int32_t andersen;      /* 0: off, 1: "count", 2: "bernoulli" (Verlet only) */
  double andersen_p;
  double gamma;          /* BAOAB friction */
  double temperature;
  double drift_tol;      /* 0: no drift stop */
} cco_md_settings;

typedef struct {
  double* r;
  double* v;
  double* f;             /* may be NULL */
  double* energy;
  double* kinetic;
  double* max_drift;
  int64_t* n_resets;
  double* reset_acc;
  uint32_t* keys;        /* [batch][2] */
  int64_t* status;
  int64_t ticks;         /* out */
  int64_t launches;      /* out */
} cco_md_out;

int cco_md_run(cco_problem* const* problems, void* stream, int batch, const double* r0,
               const double* v0, const double* bases, const uint32_t* keys, const double* acc0,
               const cco_md_settings* settings, cco_md_out* out);

/*
 * MD segments with observables  <- simulate / md_chunk / init_state
 *                                  src/xla_cco/dynamics/run.py:300-640
 * Advances `batch` lanes of one problem (one basis) by n_steps steps from
 * the batched state in `state` and writes the state back in place. Per step,
 * besides the integrator of cco_md_run: densities of the tracked waves (the
 * first n_constrained are the problem's rows `constrained_rows`, taken from
 * the force pass; the others are summed fresh on steps divisible by
 * wind_every), multiplied by exp(-i k . R_cm) unless the scheme is plain
 * Verlet; the winding update (phase_floor on |rho|^2 / N); running sums;
 * snapshots at record_steps; the rho trace every record_rho_every steps; the
 * drift guard of plain Verlet (|E - e0| <= drift_tol * d (N - 1) T / 2; inf:
 * none). Lanes whose status is not RUNNING are left as they are; a lane whose
 * rho_prev row is NaN gets that row recomputed first; a lane whose e0 is NaN
 * gets e0 = Phi + KE. n_steps = 0 only does those two. Status on return:
 * RUNNING or DRIFT.
 */
typedef struct {
  double dt, gamma, andersen_p, drift_tol, phase_floor;
  int64_t n_steps;
  int32_t scheme;            /* 0: velocity Verlet, 1: BAOAB */
  int32_t andersen;          /* Verlet only: 0 off, 1 "count", 2 "bernoulli" */
  int32_t wind_every;        /* >= 1 */
  int32_t n_record_steps;    /* <= 256 */
  const int64_t* record_steps;   /* host, strictly ascending, >= 1 */
  int32_t record_rho_every, max_rho_records;
} cco_md_segment_settings;

typedef struct {
  int32_t n_waves, n_constrained;
  const double* n_vectors;        /* host [w][d] reciprocal-basis coefficients */
  const double* kvec;             /* host [w][d] Cartesian wavevectors */
  const int32_t* constrained_rows;/* host [n_constrained] problem rows of the constrained waves */
} cco_md_waves;

/* Device arrays, [batch] leading; w waves, R = n_record_steps, Q = max_rho_records. */
typedef struct {
  double *r, *v, *f;                      /* [B][N][d] Cartesian */
  double *phi, *temperature, *time, *reset_acc, *e0, *max_drift;
  double *sum_kinetic, *sum_phi, *sum_phi2;
  uint32_t* keys;                         /* [B][2] */
  int64_t *step, *status, *n_sum;
  double* rho_prev;                       /* [B][w][2] */
  double *wind_abs, *wind_net, *sum_s;    /* [B][w] */
  int64_t* n_valid;                       /* [B][w] */
  int64_t *snap_step, *snap_count;        /* [B][R], [B] */
  double *snap_time, *snap_phi, *snap_kinetic;        /* [B][R] */
  double *snap_wind_abs, *snap_wind_net;  /* [B][R][w] */
  double* snap_rho;                       /* [B][R][w][2] */
  double* snap_r;                         /* [B][R][N][d] */
  double* trace_rho;                      /* [B][Q][w][2] */
  double* trace_time;                     /* [B][Q] */
  int64_t* trace_count;                   /* [B] */
} cco_md_state;

int cco_md_segment(cco_problem* p, void* stream, int batch, const double* basis,
                   const cco_md_segment_settings* settings, const cco_md_waves* waves,
                   cco_md_state* state, int64_t* ticks);

/*
 * Tick schedules (graph branches, ticks per graph) are tuned online on the
 * first relaxation of each shape class (minimizer, lane count and total
 * N M bucketed by powers of two, largest d) and cached for the process;
 * results never depend on the schedule. This forgets every cached schedule.
 * The environment variables CCO_BRANCHES, CCO_GRAPH_TICKS and CCO_OVERLAP
 * (0 or 1) force a schedule, CCO_AUTOTUNE=0 keeps the default (2 branches,
 * 16 ticks, no overlap). CCO_INFLIGHT (1..16, default 3) sets how many
 * graphs the driver keeps queued ahead of its completion checks.
 */
int cco_schedule_reset(void);

/*
 * Serving pool (no reference counterpart; the reference relaxes one batch
 * per call). A server owns one device and one L-BFGS setting. Requests - one
 * configuration of any problem on that device - are submitted from any host
 * thread and queue in arrival order. A driver thread admits them while the
 * lane records fit both max_lanes and the HBM budget (footprint per lane:
 * positions, gradients and search vectors 7 N d, history 2 m N d, the
 * density and pass-1 partials M (2 + ceil(N / 64)) complex, all FP64),
 * continuously: a request that arrives while others run joins the running
 * set at the next graph boundary, and a finished lane leaves it and frees
 * its memory. Every lane's result is bit-identical to the same
 * configuration relaxed alone by cco_relax_lbfgs with the same settings.
 * Problems must outlive the requests that use them.
 */
typedef struct cco_server cco_server;

typedef struct {
  int64_t max_lanes;        /* lanes on the device at once (0: 4096) */
  int64_t hbm_budget_bytes; /* admission budget for lane records (0: 150 GB), clamped to 90%
                               of the device memory free at creation */
  int32_t graph_ticks;      /* ticks per launched graph (0: 8) */
  int32_t branches;         /* graph branches (0: 2 when >= 64 lanes run, else 1) */
} cco_server_config;

typedef struct {
  double* s;                /* in: host [N][d] buffer for the final positions, or NULL */
  double energy, grad_norm;
  int64_t n_evals, n_iters, status;  /* status: CCO_STATUS_*, CANCELLED included */
  int64_t submit_ns, admit_ns, done_ns;  /* host steady clock (ns) */
  int64_t device_ns;        /* device time from the lane's first tick to its completion */
  int32_t error;            /* CCO_OK, or the code of a device failure that ended it */
  int32_t pad_;
  int64_t n_evals_fp32;     /* evaluations done in FP32 (precision = 1) */
} cco_request_result;

typedef struct {
  int64_t submitted, admitted, completed, cancelled, pending, running;
  int64_t bytes_in_use, peak_bytes, peak_lanes, budget_bytes;
  int64_t graphs, ticks, rebuilds;
} cco_server_stats;

int cco_server_create(int device, const cco_lbfgs_settings* settings,
                      const cco_server_config* config, cco_server** out);
/* Cancels what is still queued or running, stops the driver and frees all. */
int cco_server_destroy(cco_server* server);
/* Copies s0 (host [N][d]) and queues it. CCO_ERR_ADMISSION if this request
 * alone exceeds the budget; the driver's error code once it has failed. */
int cco_server_submit(cco_server* server, cco_problem* p, const double* s0, int64_t* ticket);
/* Waits up to timeout_ms (0: no wait, < 0: until done) for the request.
 * CCO_OK: done, `out` filled (out->s copied if non-NULL) and the ticket
 * released; CCO_ERR_TIMEOUT: not done yet; CCO_ERR_ARG: unknown ticket. */
int cco_server_poll(cco_server* server, int64_t ticket, int timeout_ms, cco_request_result* out);
/* Queued requests end at once, running ones at the next graph boundary,
 * both with status CCO_STATUS_CANCELLED. Finished ones are unaffected. */
int cco_server_cancel(cco_server* server, int64_t ticket);
int cco_server_get_stats(cco_server* server, cco_server_stats* out);

/*
 * Minimum-image pair statistics of a batch (the g2 and Hp inputs of the
 * ground-state driver), on the device.
 *   cco_pair_histogram   <- pair_distance_histogram   src/xla_cco/analysis/pairs.py:66-110
 *   cco_nearest_neighbor <- nearest_neighbor_distances src/xla_cco/analysis/pairs.py:41-63
 * s: device [batch][n][d] fractional positions wrapped to [0, 1); basis: host
 * [d][d], rows = lattice vectors. Distances use ds - round(ds) and the 3^d
 * image shifts (exact for reduced cells, as the reference). edges: host,
 * n_edges >= 2, finite, non-negative, strictly increasing; counts: device
 * int64 [n_edges - 1], overwritten with the counts of all pairs i < j summed
 * over the batch (np.histogram bins: left-closed, the last one closed).
 * out: device [batch][n] nearest-neighbour distances (a lone particle sees
 * its own images). batch <= 65535.
 */
int cco_pair_histogram(int device, void* stream, int batch, int n, int d, const double* s,
                       const double* basis, int n_edges, const double* edges, int64_t* counts);
int cco_nearest_neighbor(int device, void* stream, int batch, int n, int d, const double* s,
                         const double* basis, double* out);

#ifdef __cplusplus
}
#endif
#endif /* CCO_H */
