/*
 * cco_oracle.c - TEST INFRASTRUCTURE ONLY: CPU restatement of the reference
 * hot path, used as the parity checker and as the timed CPU baseline
 * ("port"). Never linked into or called by the product library.
 *
 * Follows (paths inside sdawley1/xla-cco):
 *   energy/gradient, trig path  src/xla_cco/energy.py:45-50,195-225,301-324
 *                               tests/oracle.py:38-98 (naive double loops)
 *   adaptive descent            src/xla_cco/minimize/descent.py:87-197
 *   L-BFGS schedule, statuses   src/xla_cco/minimize/lbfgs.py:163-329
 *   batched relax semantics     src/xla_cco/minimize/__init__.py:102-151
 * The L-BFGS direction and line search live in optax 0.2.8 (not vendored;
 * uv.lock pins it): restated from its published algorithm, the standard
 * L-BFGS two-loop recursion (Nocedal & Wright Alg. 7.4) with optax's
 * scale_by_lbfgs initial scaling, and a zoom line search (N&W Alg. 3.5/3.6)
 * with the Hager-Zhang approximate-Wolfe decrease test. Iterate-level parity
 * with optax is therefore unpinned; the energy, gradient and descent are
 * pinned against the reference's own golden data (tests/golden/).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define TWO_PI (2.0 * M_PI)

enum { ST_RUNNING = 0, ST_ENERGY_TOL = 1, ST_STEP_FLOOR = 2, ST_BUDGET = 3, ST_STAGNATED = 4,
       ST_LS_FAIL = 5, ST_GRAD_TOL = 6 };

/* Same layouts as include/cco.h's settings structs. */
typedef struct {
  double step_init, step_min, shrink, grow, rel_tol;
  int64_t max_evals;
  double energy_tol;
  int64_t record_every, max_records;
} od_settings;

typedef struct {
  int64_t memory;
  int32_t n_rescales, pad_;
  double rescales[8];
  int64_t max_evals_per_pass;
  double energy_tol, grad_tol;
  int64_t stagnation_patience, max_linesearch_steps, record_every, max_records;
} ol_settings;

typedef struct {
  int N, d, M;
  const double* n; /* (M, d) integer-valued */
  const double* w;
  double V;
} oproblem;

/* ------------------------------------------------------------------ energy */

/* Threads that one evaluation may use (oracle_relax_lanes sets it; 1 = the
 * plain serial loops). Rows and particles are split between the threads, and
 * every sum keeps its serial order, so the bits do not depend on it. */
static int g_inner_threads = 1;

/* Phi, dPhi/ds and rho of one configuration; grad/re/im may be NULL. */
double oracle_energy_grad(int N, int d, const double* s, int M, const double* n,
                          const double* w, double V, double* grad, double* re, double* im) {
  double* rr = (double*)malloc(sizeof(double) * 2 * (size_t)M);
  const int inner = g_inner_threads;
  (void)inner;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(inner) if (inner > 1)
#endif
  for (int k = 0; k < M; ++k) {
    double a = 0.0, b = 0.0;
    for (int j = 0; j < N; ++j) {
      double dot = 0.0;
      for (int c = 0; c < d; ++c) dot += n[(size_t)k * d + c] * s[(size_t)j * d + c];
      const double th = TWO_PI * dot;
      a += cos(th);
      b += sin(th);
    }
    rr[2 * k] = a;
    rr[2 * k + 1] = b;
  }
  double total = 0.0;
  for (int k = 0; k < M; ++k) {
    const double a = rr[2 * k], b = rr[2 * k + 1];
    total += w[k] * (a * a + b * b);
    if (re) re[k] = a;
    if (im) im[k] = b;
  }
  const double phi = total / V;
  if (grad) {
    const double pref = 2.0 * TWO_PI / V;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(inner) if (inner > 1)
#endif
    for (int j = 0; j < N; ++j) {
      double acc[3] = {0.0, 0.0, 0.0};
      for (int k = 0; k < M; ++k) {
        double dot = 0.0;
        for (int c = 0; c < d; ++c) dot += n[(size_t)k * d + c] * s[(size_t)j * d + c];
        const double th = TWO_PI * dot;
        const double coef = w[k] * (rr[2 * k + 1] * cos(th) - rr[2 * k] * sin(th));
        for (int c = 0; c < d; ++c) acc[c] += coef * n[(size_t)k * d + c];
      }
      for (int c = 0; c < d; ++c) grad[(size_t)j * d + c] = pref * acc[c];
    }
  }
  free(rr);
  return phi;
}

/* ------------------------------------------------------ accurate energy
 * A higher-accuracy restatement of the same sums, used only to measure the
 * device kernels' own error. The FP64 trig path above rounds the phase
 * argument 2 pi (n . s): for |n . s| ~ 10^3 that alone is ~1e-13 rad per
 * term. Here n . s is formed from error-free products (fma) and compensated
 * two-sums, its nearest integer removed exactly, and only the reduced
 * fraction r in [-1/2, 1/2] is scaled by 2 pi; the density, energy and
 * gradient sums are compensated (Neumaier). */
static void exact_phase(const double* nk, const double* sj, int d, double* c, double* s) {
  double hi = 0.0, lo = 0.0;
  for (int a = 0; a < d; ++a) {
    const double p = nk[a] * sj[a];
    const double e = fma(nk[a], sj[a], -p); /* p + e == n_a s_a exactly */
    const double t = hi + p;
    const double z = t - hi;
    lo += ((hi - (t - z)) + (p - z)) + e;
    hi = t;
  }
  const double r = (hi - nearbyint(hi)) + lo;
  *c = cos(TWO_PI * r);
  *s = sin(TWO_PI * r);
}

typedef struct { double s, c; } nsum;
static inline void nadd(nsum* a, double x) {
  const double t = a->s + x;
  if (fabs(a->s) >= fabs(x)) a->c += (a->s - t) + x; else a->c += (x - t) + a->s;
  a->s = t;
}

double oracle_energy_grad_accurate(int N, int d, const double* s, int M, const double* n,
                                   const double* w, double V, double* grad, double* re,
                                   double* im) {
  double* rr = (double*)malloc(sizeof(double) * 2 * (size_t)M);
  const int inner = g_inner_threads;
  (void)inner;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(inner) if (inner > 1)
#endif
  for (int k = 0; k < M; ++k) {
    nsum a = {0.0, 0.0}, b = {0.0, 0.0};
    for (int j = 0; j < N; ++j) {
      double c, sn;
      exact_phase(n + (size_t)k * d, s + (size_t)j * d, d, &c, &sn);
      nadd(&a, c);
      nadd(&b, sn);
    }
    rr[2 * k] = a.s + a.c;
    rr[2 * k + 1] = b.s + b.c;
  }
  nsum total = {0.0, 0.0};
  for (int k = 0; k < M; ++k) {
    const double a = rr[2 * k], b = rr[2 * k + 1];
    nadd(&total, w[k] * a * a);
    nadd(&total, w[k] * b * b);
    if (re) re[k] = a;
    if (im) im[k] = b;
  }
  const double phi = (total.s + total.c) / V;
  if (grad) {
    const double pref = 2.0 * TWO_PI / V;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(inner) if (inner > 1)
#endif
    for (int j = 0; j < N; ++j) {
      nsum acc[3] = {{0.0, 0.0}, {0.0, 0.0}, {0.0, 0.0}};
      for (int k = 0; k < M; ++k) {
        double c, sn;
        exact_phase(n + (size_t)k * d, s + (size_t)j * d, d, &c, &sn);
        const double coef = w[k] * (rr[2 * k + 1] * c - rr[2 * k] * sn);
        for (int a = 0; a < d; ++a) nadd(&acc[a], coef * n[(size_t)k * d + a]);
      }
      for (int a = 0; a < d; ++a) grad[(size_t)j * d + a] = pref * (acc[a].s + acc[a].c);
    }
  }
  free(rr);
  return phi;
}

/* Batched accurate evaluations, `threads` threads inside each one. */
void oracle_energy_grad_accurate_batch(int B, int N, int d, const double* s, int M,
                                       const double* n, const double* w, double V, double* phi,
                                       double* grad, double* re, double* im, int threads) {
  g_inner_threads = threads > 1 ? threads : 1;
  for (int b = 0; b < B; ++b) {
    const size_t off = (size_t)b * N * d;
    phi[b] = oracle_energy_grad_accurate(N, d, s + off, M, n, w, V, grad ? grad + off : NULL,
                                         re ? re + (size_t)b * M : NULL,
                                         im ? im + (size_t)b * M : NULL);
  }
  g_inner_threads = 1;
}

/* Batched energies/gradients, OpenMP over configurations. */
void oracle_energy_grad_batch(int B, int N, int d, const double* s, int M, const double* n,
                              const double* w, double V, double* phi, double* grad, int threads) {
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int b = 0; b < B; ++b) {
    const size_t off = (size_t)b * N * d;
    phi[b] = oracle_energy_grad(N, d, s + off, M, n, w, V, grad ? grad + off : NULL, NULL, NULL);
  }
}

static double vag(const oproblem* P, const double* s, double* g) {
  return oracle_energy_grad(P->N, P->d, s, P->M, P->n, P->w, P->V, g, NULL, NULL);
}

static double wrap01(double v) {
  const double x = v - floor(v);
  const double below = 0x1.fffffffffffffp-1;
  return x < below ? x : below;
}

static double dotv(const double* a, const double* b, size_t n) {
  double t = 0.0;
  for (size_t i = 0; i < n; ++i) t += a[i] * b[i];
  return t;
}

/* ------------------------------------------------------------------ descent */

static int descent_status(double f, const double* g, size_t nd, double step, int64_t it,
                          const od_settings* st) {
  int code = it >= st->max_evals / 2 ? ST_BUDGET : ST_RUNNING;
  if (step <= st->step_min) code = ST_STEP_FLOOR;
  int all0 = 1;
  for (size_t i = 0; i < nd; ++i) all0 &= g[i] == 0.0;
  if (all0) code = ST_GRAD_TOL;
  if (f < st->energy_tol) code = ST_ENERGY_TOL;
  return code;
}

static void record(int64_t every, int64_t cap, int64_t it, const double* s, size_t nd, double f,
                   double step, double* ts, double* te, double* tst, int64_t* tit,
                   int64_t* count) {
  if (!count || every <= 0 || cap <= 0) return;
  if (it % every != 0 || *count >= cap) return;
  const int64_t r = *count;
  for (size_t i = 0; i < nd; ++i) ts[(size_t)r * nd + i] = wrap01(s[i]);
  te[r] = f;
  tst[r] = step;
  tit[r] = it;
  *count = r + 1;
}

int oracle_descent(int N, int d, const double* s0, int M, const double* n, const double* w,
                   double V, const od_settings* st, double* s_out, double* f_out,
                   double* gn_out, int64_t* ne_out, int64_t* ni_out, int64_t* status_out,
                   double* ts, double* te, double* tst, int64_t* tit, int64_t* tcount) {
  const oproblem P = {N, d, M, n, w, V};
  const size_t nd = (size_t)N * d;
  double* s = (double*)malloc(sizeof(double) * nd);
  double* g = (double*)malloc(sizeof(double) * nd);
  double* xn = (double*)malloc(sizeof(double) * nd);
  double* g2 = (double*)malloc(sizeof(double) * nd);
  memcpy(s, s0, sizeof(double) * nd);
  double f = vag(&P, s, g);
  double step = st->step_init;
  int64_t it = 0, ne = 0;
  int status = descent_status(f, g, nd, step, it, st);
  if (tcount) *tcount = 0;
  record(st->record_every, st->max_records, 0, s, nd, f, step, ts, te, tst, tit, tcount);
  while (status == ST_RUNNING) {
    const double norm = sqrt(dotv(g, g, nd));
    for (size_t i = 0; i < nd; ++i) {
      const double gn = norm > 0.0 ? g[i] / norm : 0.0 * g[i];
      xn[i] = s[i] - gn * step;
    }
    const double f2 = vag(&P, xn, g2);
    const double df = f - f2;
    const double df2 = step * norm;
    const int reject = fabs(df - df2) / df2 > st->rel_tol;
    step = reject ? step * st->shrink : step * st->grow;
    if (!reject) {
      memcpy(s, xn, sizeof(double) * nd);
      memcpy(g, g2, sizeof(double) * nd);
      f = f2;
    }
    it += 1;
    ne += 2;
    status = descent_status(f, g, nd, step, it, st);
    record(st->record_every, st->max_records, it, s, nd, f, step, ts, te, tst, tit, tcount);
  }
  for (size_t i = 0; i < nd; ++i) s_out[i] = wrap01(s[i]);
  *f_out = f;
  *gn_out = sqrt(dotv(g, g, nd));
  *ne_out = ne;
  *ni_out = it;
  *status_out = status;
  free(s); free(g); free(xn); free(g2);
  return 0;
}

/* ------------------------------------------------------------------ L-BFGS */

#define C1 1e-4
#define C2 0.9
#define APPROX_EPS 1e-6

typedef struct { double a, f, d; } lspt;

static int ls_sufficient(double f0, double d0, double a, double f, double d) {
  if (!isfinite(f) || !isfinite(d)) return 0;
  const double armijo = f - (f0 + C1 * a * d0);
  const double approx = fmax(d - (2.0 * C1 - 1.0) * d0, f - f0 - APPROX_EPS * fabs(f0));
  return fmin(armijo, approx) <= 0.0;
}

/* cubic minimizer of the Hermite interpolant on [lo, hi], else bisection */
static double ls_interp(lspt lo, lspt hi) {
  const double dl = hi.a - lo.a;
  const double lb = fmin(lo.a, hi.a) + 0.1 * fabs(dl), ub = fmax(lo.a, hi.a) - 0.1 * fabs(dl);
  if (isfinite(hi.f) && isfinite(hi.d) && dl != 0.0) {
    const double d1 = lo.d + hi.d - 3.0 * (lo.f - hi.f) / (lo.a - hi.a);
    const double disc = d1 * d1 - lo.d * hi.d;
    if (disc >= 0.0 && isfinite(disc)) {
      const double d2 = copysign(sqrt(disc), dl);
      const double a = hi.a - dl * (hi.d + d2 - d1) / (hi.d - lo.d + 2.0 * d2);
      if (isfinite(a) && a >= lb && a <= ub) return a;
    }
  }
  return lo.a + 0.5 * dl;
}

typedef struct {
  const oproblem* P;
  double R;
  const double* x;
  const double* dir;
  double* xt;   /* scratch */
  double* st;   /* scratch: s at the probe */
  double* gs;   /* scratch: dPhi/ds at the probe */
} lsctx;

/* Evaluate phi(alpha) and phi'(alpha); gx receives dPhi/dx at the probe. */
static void ls_eval(lsctx* c, double a, double* f, double* dphi, double* gx) {
  const size_t nd = (size_t)c->P->N * c->P->d;
  for (size_t i = 0; i < nd; ++i) {
    c->xt[i] = c->x[i] + a * c->dir[i];
    c->st[i] = c->xt[i] / c->R;
  }
  *f = vag(c->P, c->st, c->gs);
  double t = 0.0;
  for (size_t i = 0; i < nd; ++i) {
    gx[i] = c->gs[i] / c->R;
    t += gx[i] * c->dir[i];
  }
  *dphi = t;
}

/* Returns 1 on success (alpha, f, g filled), 0 on failure. *steps = probes. */
static int line_search(lsctx* c, double f0, double d0, int64_t max_steps, double* a_out,
                       double* f_out, double* g_out, double* gprobe, int64_t* steps) {
  const size_t nd = (size_t)c->P->N * c->P->d;
  lspt prev = {0.0, f0, d0}, lo = prev, hi = prev;
  int have_lo = 0, zoom = 0;
  double a = 1.0;
  int64_t k = 0;
  while (k < max_steps) {
    double f, d;
    ls_eval(c, a, &f, &d, gprobe);
    ++k;
    const int suff = ls_sufficient(f0, d0, a, f, d);
    const int curv = fabs(d) <= C2 * fabs(d0);
    const lspt p = {a, f, d};
    if (!zoom) {
      if (!suff || (k > 1 && f >= prev.f)) {
        lo = prev; hi = p; zoom = 1;
      } else if (curv) {
        *a_out = a; *f_out = f; memcpy(g_out, gprobe, sizeof(double) * nd); *steps = k;
        return 1;
      } else if (d >= 0.0) {
        hi = prev; lo = p; have_lo = 1; memcpy(g_out, gprobe, sizeof(double) * nd); zoom = 1;
      } else {
        prev = p; lo = p; have_lo = 1; memcpy(g_out, gprobe, sizeof(double) * nd);
        a = 2.0 * a;
        continue;
      }
    } else {
      if (!suff || f >= lo.f) {
        hi = p;
      } else {
        if (curv) {
          *a_out = a; *f_out = f; memcpy(g_out, gprobe, sizeof(double) * nd); *steps = k;
          return 1;
        }
        if (d * (hi.a - lo.a) >= 0.0) hi = lo;
        lo = p; have_lo = 1; memcpy(g_out, gprobe, sizeof(double) * nd);
      }
    }
    a = ls_interp(lo, hi);
  }
  *steps = k;
  if (have_lo) {  /* best point with sufficient decrease (g_out already holds it) */
    *a_out = lo.a;
    *f_out = lo.f;
    return 1;
  }
  *a_out = a;
  return 0;
}

int oracle_lbfgs(int N, int d, const double* s0, int M, const double* n, const double* w,
                 double V, const ol_settings* st, double* s_out, double* f_out, double* gn_out,
                 int64_t* ne_out, int64_t* ni_out, int64_t* status_out, double* ts, double* te,
                 double* tst, int64_t* tit, int64_t* tcount) {
  const oproblem P = {N, d, M, n, w, V};
  const size_t nd = (size_t)N * d;
  const int m = (int)st->memory;
  double* x = calloc(nd, sizeof(double));
  double* s = calloc(nd, sizeof(double));
  double* g = calloc(nd, sizeof(double));
  double* q = calloc(nd, sizeof(double));
  double* dir = calloc(nd, sizeof(double));
  double* gn = calloc(nd, sizeof(double));
  double* gp = calloc(nd, sizeof(double));
  double* xt = calloc(nd, sizeof(double));
  double* stv = calloc(nd, sizeof(double));
  double* gs = calloc(nd, sizeof(double));
  double* S = calloc((size_t)m * nd, sizeof(double));
  double* Y = calloc((size_t)m * nd, sizeof(double));
  double* rho = calloc(m, sizeof(double));
  double* alpha = calloc(m, sizeof(double));
  double R = st->rescales[0];
  memcpy(s, s0, sizeof(double) * nd);
  double f = vag(&P, s, gs);
  for (size_t i = 0; i < nd; ++i) {
    x[i] = s[i] * R;
    g[i] = gs[i] / R;
  }
  int64_t ne = 1, it = 0, pass_evals = 0, stag = 0;
  int pass = 0, hk = 0, head = 0;
  double last_step = 0.0;
  int status = f < st->energy_tol ? ST_ENERGY_TOL : ST_RUNNING;
  if (tcount) *tcount = 0;
  record(st->record_every, st->max_records, 0, s, nd, f, 0.0, ts, te, tst, tit, tcount);
  lsctx c = {&P, R, x, dir, xt, stv, gs};
  while (status == ST_RUNNING) {
    /* direction: two-loop recursion (newest pair first) */
    memcpy(q, g, sizeof(double) * nd);
    for (int t = hk - 1; t >= 0; --t) {
      const int sl = (head - hk + t + m) % m;
      alpha[t] = rho[sl] * dotv(S + (size_t)sl * nd, q, nd);
      for (size_t i = 0; i < nd; ++i) q[i] -= alpha[t] * Y[(size_t)sl * nd + i];
    }
    double gamma;
    if (hk == 0) {
      gamma = fmin(1.0, 1.0 / sqrt(dotv(g, g, nd)));
    } else {
      const int sl = (head - 1 + m) % m;
      const double num = dotv(Y + (size_t)sl * nd, S + (size_t)sl * nd, nd);
      const double den = dotv(Y + (size_t)sl * nd, Y + (size_t)sl * nd, nd);
      gamma = den > 0.0 ? num / den : 1.0;
    }
    for (size_t i = 0; i < nd; ++i) q[i] *= gamma;
    for (int t = 0; t < hk; ++t) {
      const int sl = (head - hk + t + m) % m;
      const double beta = rho[sl] * dotv(Y + (size_t)sl * nd, q, nd);
      for (size_t i = 0; i < nd; ++i) q[i] += S[(size_t)sl * nd + i] * (alpha[t] - beta);
    }
    for (size_t i = 0; i < nd; ++i) dir[i] = -q[i];
    const double d0 = dotv(g, dir, nd);
    c.R = R;
    double a = 0.0, fn = f;
    int64_t steps = 0;
    const int ok = line_search(&c, f, d0, st->max_linesearch_steps, &a, &fn, gn, gp, &steps);
    const int fail = !ok || !isfinite(fn);
    const double f_old = f;
    if (!fail) {
      const int sl = head;
      for (size_t i = 0; i < nd; ++i) {
        const double xnew = x[i] + a * dir[i];
        S[(size_t)sl * nd + i] = xnew - x[i];
        Y[(size_t)sl * nd + i] = gn[i] - g[i];
        x[i] = xnew;
        s[i] = xnew / R;
        g[i] = gn[i];
      }
      const double ys = dotv(Y + (size_t)sl * nd, S + (size_t)sl * nd, nd);
      rho[sl] = ys == 0.0 ? 0.0 : 1.0 / ys;
      head = (head + 1) % m;
      hk = hk < m ? hk + 1 : m;
      f = fn;
      last_step = a;
    } else {
      last_step = a;
    }
    stag = f < f_old ? 0 : stag + 1;
    const int64_t ev = steps > 1 ? steps : 1;
    pass_evals += ev;
    ne += ev;
    it += 1;
    const double gnorm = sqrt(dotv(g, g, nd)) * R;
    int glob = gnorm < st->grad_tol ? ST_GRAD_TOL : ST_RUNNING;
    if (f < st->energy_tol) glob = ST_ENERGY_TOL;
    int local = pass_evals >= st->max_evals_per_pass ? ST_BUDGET : ST_RUNNING;
    if (stag >= st->stagnation_patience) local = ST_STAGNATED;
    if (fail) local = ST_LS_FAIL;
    const int last = pass >= st->n_rescales - 1;
    const int pass_end = local != ST_RUNNING && glob == ST_RUNNING;
    status = glob != ST_RUNNING ? glob : ST_RUNNING;
    if (pass_end && last) status = local;
    if (pass_end && !last) {
      const double rn = st->rescales[pass + 1];
      for (size_t i = 0; i < nd; ++i) {
        x[i] = s[i] * rn;
        g[i] = g[i] * R / rn;
      }
      R = rn;
      pass += 1;
      pass_evals = 0;
      stag = 0;
      hk = 0;
      head = 0;
    }
    record(st->record_every, st->max_records, it, s, nd, f, last_step, ts, te, tst, tit, tcount);
  }
  for (size_t i = 0; i < nd; ++i) s_out[i] = wrap01(s[i]);
  *f_out = f;
  *gn_out = sqrt(dotv(g, g, nd)) * R;
  *ne_out = ne;
  *ni_out = it;
  *status_out = status;
  free(x); free(s); free(g); free(q); free(dir); free(gn); free(gp); free(xt); free(stv);
  free(gs); free(S); free(Y); free(rho); free(alpha);
  return 0;
}

/* Batched relaxations (lanes are independent), OpenMP over lanes. method 0 =
 * descent (settings = od_settings), 1 = L-BFGS (ol_settings). */
void oracle_relax_batch(int method, int B, int N, int d, const double* s0, int M,
                        const double* n, const double* w, double V, const void* settings,
                        double* s_out, double* f_out, double* gn_out, int64_t* ne, int64_t* ni,
                        int64_t* status, int threads) {
  const size_t nd = (size_t)N * d;
#ifdef _OPENMP
  if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 1)
#endif
  for (int b = 0; b < B; ++b) {
    const size_t o = (size_t)b * nd;
    if (method == 0)
      oracle_descent(N, d, s0 + o, M, n, w, V, (const od_settings*)settings, s_out + o, f_out + b,
                     gn_out + b, ne + b, ni + b, status + b, NULL, NULL, NULL, NULL, NULL);
    else
      oracle_lbfgs(N, d, s0 + o, M, n, w, V, (const ol_settings*)settings, s_out + o, f_out + b,
                   gn_out + b, ne + b, ni + b, status + b, NULL, NULL, NULL, NULL, NULL);
  }
}

/* The same relaxations one lane after another, each evaluation spread over
 * `threads` threads (rows of the density pass, particles of the gradient
 * pass). Results are bit-identical to oracle_relax_batch; this form lets a
 * short sample of a batch use every host thread. */
void oracle_relax_lanes(int method, int B, int N, int d, const double* s0, int M,
                        const double* n, const double* w, double V, const void* settings,
                        double* s_out, double* f_out, double* gn_out, int64_t* ne, int64_t* ni,
                        int64_t* status, int threads) {
  const size_t nd = (size_t)N * d;
  g_inner_threads = threads > 1 ? threads : 1;
  for (int b = 0; b < B; ++b) {
    const size_t o = (size_t)b * nd;
    if (method == 0)
      oracle_descent(N, d, s0 + o, M, n, w, V, (const od_settings*)settings, s_out + o, f_out + b,
                     gn_out + b, ne + b, ni + b, status + b, NULL, NULL, NULL, NULL, NULL);
    else
      oracle_lbfgs(N, d, s0 + o, M, n, w, V, (const ol_settings*)settings, s_out + o, f_out + b,
                   gn_out + b, ne + b, ni + b, status + b, NULL, NULL, NULL, NULL, NULL);
  }
  g_inner_threads = 1;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
