/* ORACLE - test infrastructure only.
 *
 * Plain-C CPU restatement of the reference's Counter-V1 RNG and its
 * compressed, no-control, match-deletion JLA estimator.  It is the checker for
 * the device engine: only the tests, the smoke check and the CPU-baseline leg
 * of the benchmark load it.  The product never links or calls it.
 *
 * Restated reference functions (paths inside the reference project):
 *   rng            rust/crates/vckss-core/src/rng.rs:73-93, 130-305, 308-335
 *   full fit       rust/crates/vckss-core/src/operator.rs:269-343 (Schur RHS,
 *                  worker reconstruction), engine.rs:1107-1134
 *   plug-in        rust/crates/vckss-core/src/jla.rs:286-364
 *   leverage       rust/crates/vckss-core/src/engine.rs:1150-1228, 2562-2619
 *   adjustment     rust/crates/vckss-core/src/engine.rs:2269-2410
 *   target         rust/crates/vckss-core/src/engine.rs:2621-2879 (directions,
 *                  transpose, balance repair), 3003-3101 (contraction)
 *   mean / MCSE    rust/crates/vckss-core/src/engine.rs:3108-3200
 *   centering mean rust/crates/vckss-core/src/centering.rs:6-27
 *   generic (controls, match deletion, joint nuisance): control geometry
 *                  generic_jla.rs:4407-4537, deleted adjustment 6053-6196,
 *                  target correction 8554-8900, target draw
 *                  generic_jla/statistical_batches.rs:259-347
 * Linear solves use the firm Schur complement on the zero-sum quotient: a
 * dense grounded Cholesky factor when the firm count is small, otherwise
 * Jacobi-preconditioned CG to a tight tolerance.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ RNG */

static uint64_t splitmix64(uint64_t x) {
  x += 0x9e3779b97f4a7c15ull;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
  return x ^ (x >> 31);
}

void oracle_philox_block(uint64_t seed, uint64_t tag, uint64_t probe_block, uint64_t entity, uint64_t word,
                         uint64_t out[4]) {
  uint64_t c[4] = {entity, probe_block, word, tag};
  uint64_t k0 = splitmix64(seed), k1 = splitmix64(seed ^ 0xd1b54a32d192ed03ull);
  for (int round = 0; round < 10; ++round) {
    unsigned __int128 p0 = (unsigned __int128)0xd2b74407b1ce6e93ull * c[0];
    unsigned __int128 p1 = (unsigned __int128)0xca5a826395121157ull * c[2];
    uint64_t h0 = (uint64_t)(p0 >> 64), l0 = (uint64_t)p0, h1 = (uint64_t)(p1 >> 64), l1 = (uint64_t)p1;
    uint64_t n[4] = {h1 ^ c[1] ^ k0, l1, h0 ^ c[3] ^ k1, l0};
    memcpy(c, n, sizeof(c));
    if (round != 9) {
      k0 += 0x9e3779b97f4a7c15ull;
      k1 += 0xbb67ae8584caa73bull;
    }
  }
  memcpy(out, c, sizeof(c));
}

/* 2 * popcount(selected bits) - trials; returns 0 and sets *ok = 0 on a bad trial count */
int64_t oracle_rademacher_sum(uint64_t seed, uint64_t tag, uint64_t probe, uint64_t entity, uint64_t trials, int* ok) {
  if (trials == 0 || trials > (1ull << 53)) {
    if (ok) *ok = 0;
    return 0;
  }
  if (ok) *ok = 1;
  uint64_t full = trials / 64, rem = trials % 64, pos = 0, b[4];
  int lane = (int)(probe % 4);
  for (uint64_t w = 0; w < full; ++w) {
    oracle_philox_block(seed, tag, probe / 4, entity, w, b);
    pos += (uint64_t)__builtin_popcountll(b[lane]);
  }
  if (rem) {
    oracle_philox_block(seed, tag, probe / 4, entity, full, b);
    pos += (uint64_t)__builtin_popcountll(b[lane] & ((1ull << rem) - 1));
  }
  return 2 * (int64_t)pos - (int64_t)trials;
}

/* -------------------------------------------------------- compensated sums */

typedef struct {
  double sum, corr;
} Stable;

static void st_add(Stable* s, double v) {
  double t = s->sum + v;
  s->corr += (fabs(s->sum) >= fabs(v)) ? (s->sum - t) + v : (v - t) + s->sum;
  s->sum = t;
}
static double st_fin(const Stable* s) { return s->sum + s->corr; }

/* ---------------------------------------------------------------- problem */

typedef struct {
  uint64_t rows, workers, firms, cells, units, strata, physical_total;
  double target_total;
  const uint32_t *row_worker, *row_firm, *row_cell;
  const double *row_outcome, *row_target;
  const uint64_t* row_frequency;
  const uint32_t *cell_worker, *cell_firm;
  const double *cell_weight, *cell_outcome_sum, *cell_target_sum;
  const uint32_t* unit_cell;
  const uint64_t *unit_count, *unit_rank;
  const double* unit_outcome_sum;
  const uint32_t* stratum_cell;
  const double* stratum_per_copy;
  const uint64_t *stratum_count, *stratum_rank;
  uint64_t controls;
  const double* control_values; /* rows x controls, column-major */
  const uint64_t* group_ptr;
  const uint32_t* group_rows;
  const uint64_t* row_rank;        /* generic plans: semantic rank of every row */
  const uint64_t* row_copy_offset; /* not read: the oracle numbers copies itself */
  uint64_t deletion_mode;          /* 1 match, 2 observation */
} OracleProblem;

typedef struct {
  uint64_t seed;
  uint32_t probes;
  uint32_t centering; /* 0 none, 1 mean */
  double tolerance;   /* CG tolerance when the dense factor is not used */
  double rank_tolerance, block_tolerance;
  uint32_t dense_limit; /* use the dense factor when firms <= dense_limit */
  /* probe sharding (compressed estimator): probes [probe_begin, probe_end)
   * (end 0: all); phase 1 stops after the leverage moments and writes their
   * sums (units x 5) to shard_io; phase 2 reads the summed moments from
   * shard_io, writes the range's target draws and skips the components */
  uint32_t probe_begin, probe_end;
  int32_t phase;
  uint32_t reserved;
  double* shard_io;
} OracleOptions;

typedef struct {
  double plugin[4], correction[4], corrected[4], mcse[4];
  double* fitted_cell;          /* cells */
  double* projection_share;     /* units */
  double* residual_share;       /* units */
  double* finite_bias;          /* units */
  double* finite_variance;      /* units */
  double* residual_mass;        /* units */
  double* deleted_mass;         /* units */
  double* cell_correction_weight; /* cells */
  double* target_draws;         /* probes x 4 */
  uint64_t solves, cg_iterations;
  int error_code;
  char error[256];
} OracleResult;

typedef struct {
  const OracleProblem* p;
  double *wdiag, *fdiag;
  int dense;
  double* chol; /* (F-1)^2 lower factor of the grounded Schur complement */
  double tol;
  uint64_t iterations;
  double *t_sum, *t_r, *t_z, *t_p, *t_q;
} Solver;

static void schur_apply(const Solver* s, const double* x, double* y, double* wsum) {
  const OracleProblem* p = s->p;
  memset(wsum, 0, p->workers * sizeof(double));
  for (uint64_t c = 0; c < p->cells; ++c) wsum[p->cell_worker[c]] += p->cell_weight[c] * x[p->cell_firm[c]];
  for (uint64_t w = 0; w < p->workers; ++w) wsum[w] /= s->wdiag[w];
  for (uint64_t f = 0; f < p->firms; ++f) y[f] = s->fdiag[f] * x[f];
  for (uint64_t c = 0; c < p->cells; ++c) y[p->cell_firm[c]] -= p->cell_weight[c] * wsum[p->cell_worker[c]];
}

static void center(double* v, uint64_t n) {
  Stable s = {0, 0};
  for (uint64_t i = 0; i < n; ++i) st_add(&s, v[i]);
  double m = st_fin(&s) / (double)n;
  for (uint64_t i = 0; i < n; ++i) v[i] -= m;
}

static int solver_init(Solver* s, const OracleProblem* p, const OracleOptions* o) {
  memset(s, 0, sizeof(*s));
  s->p = p;
  s->tol = o->tolerance;
  s->wdiag = calloc(p->workers, sizeof(double));
  s->fdiag = calloc(p->firms, sizeof(double));
  s->t_sum = calloc(p->workers, sizeof(double));
  for (uint64_t c = 0; c < p->cells; ++c) {
    s->wdiag[p->cell_worker[c]] += p->cell_weight[c];
    s->fdiag[p->cell_firm[c]] += p->cell_weight[c];
  }
  uint64_t F = p->firms;
  s->dense = F <= o->dense_limit;
  if (s->dense) {
    uint64_t m = F - 1;
    double* A = calloc(m * m, sizeof(double));
    for (uint64_t f = 0; f < m; ++f) A[f * m + f] = s->fdiag[f];
    /* subtract sum_w a a^T / d_w over the worker's cells (cells of a worker are contiguous) */
    uint64_t c = 0;
    while (c < p->cells) {
      uint64_t e = c;
      while (e < p->cells && p->cell_worker[e] == p->cell_worker[c]) ++e;
      double d = s->wdiag[p->cell_worker[c]];
      for (uint64_t i = c; i < e; ++i)
        for (uint64_t j = c; j < e; ++j) {
          uint64_t fi = p->cell_firm[i], fj = p->cell_firm[j];
          if (fi < m && fj < m) A[fi * m + fj] -= p->cell_weight[i] * p->cell_weight[j] / d;
        }
      c = e;
    }
    for (uint64_t j = 0; j < m; ++j) {
      double dd = A[j * m + j];
      for (uint64_t k = 0; k < j; ++k) dd -= A[j * m + k] * A[j * m + k];
      if (!(dd > 0.0)) {
        free(A);
        return -1;
      }
      dd = sqrt(dd);
      A[j * m + j] = dd;
      for (uint64_t i = j + 1; i < m; ++i) {
        double v = A[i * m + j];
        for (uint64_t k = 0; k < j; ++k) v -= A[i * m + k] * A[j * m + k];
        A[i * m + j] = v / dd;
      }
    }
    s->chol = A;
  } else {
    s->t_r = calloc(F, sizeof(double));
    s->t_z = calloc(F, sizeof(double));
    s->t_p = calloc(F, sizeof(double));
    s->t_q = calloc(F, sizeof(double));
  }
  return 0;
}

static void solver_free(Solver* s) {
  free(s->wdiag);
  free(s->fdiag);
  free(s->t_sum);
  free(s->chol);
  free(s->t_r);
  free(s->t_z);
  free(s->t_p);
  free(s->t_q);
}

/* Solve the two-way normal equations for (worker_rhs, firm_rhs); firm solution centred. */
static int solve(Solver* s, const double* bw, const double* bf, double* alpha, double* psi) {
  const OracleProblem* p = s->p;
  uint64_t W = p->workers, F = p->firms;
  /* Schur RHS (operator.rs:269-304) */
  double* rhs = malloc(F * sizeof(double));
  memcpy(rhs, bf, F * sizeof(double));
  for (uint64_t c = 0; c < p->cells; ++c) {
    uint32_t w = p->cell_worker[c];
    rhs[p->cell_firm[c]] -= p->cell_weight[c] * (bw[w] / s->wdiag[w]);
  }
  center(rhs, F);
  if (s->dense) {
    uint64_t m = F - 1;
    const double* L = s->chol;
    for (uint64_t i = 0; i < m; ++i) {
      double v = rhs[i];
      for (uint64_t k = 0; k < i; ++k) v -= L[i * m + k] * psi[k];
      psi[i] = v / L[i * m + i];
    }
    for (uint64_t ii = m; ii-- > 0;) {
      double v = psi[ii];
      for (uint64_t k = ii + 1; k < m; ++k) v -= L[k * m + ii] * psi[k];
      psi[ii] = v / L[ii * m + ii];
    }
    psi[m] = 0.0;
  } else {
    double *r = s->t_r, *z = s->t_z, *pp = s->t_p, *q = s->t_q;
    double bn = 0;
    for (uint64_t f = 0; f < F; ++f) bn += rhs[f] * rhs[f];
    bn = sqrt(bn);
    memset(psi, 0, F * sizeof(double));
    if (bn > 0) {
      memcpy(r, rhs, F * sizeof(double));
      double rz = 0;
      for (uint64_t f = 0; f < F; ++f) {
        z[f] = r[f] / s->fdiag[f];
        rz += r[f] * z[f];
      }
      memcpy(pp, z, F * sizeof(double));
      for (int it = 0; it < 100000; ++it) {
        schur_apply(s, pp, q, s->t_sum);
        double pq = 0;
        for (uint64_t f = 0; f < F; ++f) pq += pp[f] * q[f];
        if (!(pq > 0)) break;
        double a = rz / pq, rr = 0, rz2 = 0;
        for (uint64_t f = 0; f < F; ++f) {
          psi[f] += a * pp[f];
          r[f] -= a * q[f];
          rr += r[f] * r[f];
        }
        s->iterations++;
        if (sqrt(rr) <= s->tol * bn) break;
        for (uint64_t f = 0; f < F; ++f) {
          z[f] = r[f] / s->fdiag[f];
          rz2 += r[f] * z[f];
        }
        double b = rz2 / rz;
        rz = rz2;
        for (uint64_t f = 0; f < F; ++f) pp[f] = z[f] + b * pp[f];
      }
    }
  }
  free(rhs);
  center(psi, F);
  /* worker reconstruction (operator.rs:311-343) */
  memcpy(alpha, bw, W * sizeof(double));
  for (uint64_t c = 0; c < p->cells; ++c) alpha[p->cell_worker[c]] -= p->cell_weight[c] * psi[p->cell_firm[c]];
  for (uint64_t w = 0; w < W; ++w) alpha[w] /= s->wdiag[w];
  return 0;
}

static int set_error(OracleResult* r, int code, const char* msg) {
  r->error_code = code;
  strncpy(r->error, msg, sizeof(r->error) - 1);
  return code;
}

#define TAG_LEVERAGE 0x4c45564552414745ull
#define TAG_TARGET 0x0054415247455401ull

int oracle_jla(const OracleProblem* p, const OracleOptions* o, OracleResult* res) {
  uint64_t W = p->workers, F = p->firms, C = p->cells, G = p->units, S = p->strata, P = o->probes;
  Solver s;
  res->error_code = 0;
  if (solver_init(&s, p, o)) return set_error(res, 82, "grounded Schur factor is not positive definite");
  double *bw = calloc(W, 8), *bf = calloc(F, 8), *alpha = calloc(W, 8), *psi = calloc(F, 8);
  double *alpha2 = calloc(W, 8), *psi2 = calloc(F, 8);
  /* ---- full fit */
  for (uint64_t c = 0; c < C; ++c) {
    bw[p->cell_worker[c]] += p->cell_outcome_sum[c];
    bf[p->cell_firm[c]] += p->cell_outcome_sum[c];
  }
  solve(&s, bw, bf, alpha, psi);
  res->solves++;
  for (uint64_t c = 0; c < C; ++c) res->fitted_cell[c] = alpha[p->cell_worker[c]] + psi[p->cell_firm[c]];
  {
    Stable wm = {0, 0}, fm = {0, 0};
    for (uint64_t r = 0; r < p->rows; ++r) {
      st_add(&wm, p->row_target[r] * alpha[p->row_worker[r]]);
      st_add(&fm, p->row_target[r] * psi[p->row_firm[r]]);
    }
    double mw = st_fin(&wm) / p->target_total, mf = st_fin(&fm) / p->target_total;
    Stable a = {0, 0}, b = {0, 0}, cv = {0, 0}, t = {0, 0};
    for (uint64_t r = 0; r < p->rows; ++r) {
      double x = alpha[p->row_worker[r]] - mw, y = psi[p->row_firm[r]] - mf, wt = p->row_target[r];
      st_add(&a, wt * x * x);
      st_add(&b, wt * y * y);
      st_add(&cv, wt * x * y);
      st_add(&t, wt * (x + y) * (x + y));
    }
    res->plugin[0] = st_fin(&a) / p->target_total;
    res->plugin[1] = st_fin(&b) / p->target_total;
    res->plugin[2] = st_fin(&cv) / p->target_total;
    res->plugin[3] = st_fin(&t) / p->target_total;
  }
  /* ---- leverage moments, one probe at a time (batch invariant) */
  Stable* mom = calloc(G * 5, sizeof(Stable));
  int64_t* atoms = calloc(G > S ? G : S, sizeof(int64_t));
  const uint64_t pb = o->probe_begin, pe = o->probe_end ? o->probe_end : P;
  if (o->phase == 2)
    for (uint64_t i = 0; i < G * 5; ++i) mom[i].sum = o->shard_io[i];
  for (uint64_t probe = pb; probe < (o->phase == 2 ? pb : pe); ++probe) {
    memset(bw, 0, W * 8);
    memset(bf, 0, F * 8);
    for (uint64_t g = 0; g < G; ++g) {
      int ok;
      atoms[g] = oracle_rademacher_sum(o->seed, TAG_LEVERAGE, probe, p->unit_rank[g], p->unit_count[g], &ok);
      if (!ok) return set_error(res, 70, "Rademacher trial count must lie in [1, 2^53]");
      uint32_t c = p->unit_cell[g];
      bw[p->cell_worker[c]] += (double)atoms[g];
      bf[p->cell_firm[c]] += (double)atoms[g];
    }
    solve(&s, bw, bf, alpha, psi);
    res->solves++;
    for (uint64_t g = 0; g < G; ++g) {
      uint32_t c = p->unit_cell[g];
      double rn = sqrt((double)p->unit_count[g]);
      double pr = rn * (alpha[p->cell_worker[c]] + psi[p->cell_firm[c]]);
      double m = (double)atoms[g] / rn - pr, p2 = pr * pr, m2 = m * m;
      st_add(&mom[g * 5 + 0], p2);
      st_add(&mom[g * 5 + 1], m2);
      st_add(&mom[g * 5 + 2], p2 * p2);
      st_add(&mom[g * 5 + 3], m2 * m2);
      st_add(&mom[g * 5 + 4], p2 * m2);
    }
  }
  if (o->phase == 1) {
    for (uint64_t i = 0; i < G * 5; ++i) o->shard_io[i] = st_fin(&mom[i]);
    free(mom);
    free(atoms);
    free(bw);
    free(bf);
    free(alpha);
    free(psi);
    free(alpha2);
    free(psi2);
    solver_free(&s);
    return 0;
  }
  /* ---- adjustment */
  double mean = 0.0;
  if (o->centering == 1) {
    double anchor = p->row_outcome[0];
    Stable sm = {0, 0};
    for (uint64_t r = 0; r < p->rows; ++r)
      st_add(&sm, (p->row_outcome[r] - anchor) * ((double)p->row_frequency[r] / (double)p->physical_total));
    mean = anchor + st_fin(&sm);
  }
  Stable* cw = calloc(C, sizeof(Stable));
  double Pd = (double)P;
  for (uint64_t g = 0; g < G; ++g) {
    double pf = st_fin(&mom[g * 5 + 0]), mf = st_fin(&mom[g * 5 + 1]);
    double tm = (pf + mf) / Pd;
    if (!(tm > o->block_tolerance)) return set_error(res, 74, "projection/residual mass failed");
    double proj = (pf / Pd) / tm, resid = (mf / Pd) / tm;
    double ps = st_fin(&mom[g * 5 + 2]) / Pd, ms = st_fin(&mom[g * 5 + 3]) / Pd, mx = st_fin(&mom[g * 5 + 4]) / Pd;
    double bias = (resid * ps - proj * ms + (resid - proj) * mx) / Pd;
    double var = (resid * resid * ps + proj * proj * ms - 2.0 * proj * resid * mx) / Pd;
    if (var < -100.0 * o->rank_tolerance) return set_error(res, 73, "finite-projection variance is negative");
    if (var < 0) var = 0;
    if (1.0 - proj <= o->block_tolerance) return set_error(res, 75, "match residual block is singular");
    double rec = 1.0 / resid;
    uint32_t c = p->unit_cell[g];
    double ro = p->unit_outcome_sum[g] - (double)p->unit_count[g] * res->fitted_cell[c];
    double mult = rec + bias * rec * rec - var * rec * rec * rec;
    double del = ro * mult;
    st_add(&cw[c], (p->unit_outcome_sum[g] - mean * (double)p->unit_count[g]) * del);
    res->projection_share[g] = proj;
    res->residual_share[g] = resid;
    res->finite_bias[g] = bias;
    res->finite_variance[g] = var;
    res->residual_mass[g] = ro;
    res->deleted_mass[g] = del;
  }
  for (uint64_t c = 0; c < C; ++c) res->cell_correction_weight[c] = st_fin(&cw[c]);
  /* ---- target draws */
  Stable* dir = calloc(C, sizeof(Stable));
  double* d = calloc(C, 8);
  double *sw = calloc(W, 8), *sf = calloc(F, 8), *zw = calloc(W, 8), *zf = calloc(F, 8);
  for (uint64_t probe = pb; probe < pe; ++probe) {
    memset(dir, 0, C * sizeof(Stable));
    for (uint64_t k = 0; k < S; ++k) {
      int ok;
      int64_t a = oracle_rademacher_sum(o->seed, TAG_TARGET, probe, p->stratum_rank[k], p->stratum_count[k], &ok);
      if (!ok) return set_error(res, 70, "Rademacher trial count must lie in [1, 2^53]");
      st_add(&dir[p->stratum_cell[k]], sqrt(p->stratum_per_copy[k] / p->target_total) * (double)a);
    }
    Stable tot = {0, 0}, ab = {0, 0};
    for (uint64_t c = 0; c < C; ++c) {
      d[c] = st_fin(&dir[c]);
      st_add(&tot, d[c]);
      st_add(&ab, fabs(d[c]));
    }
    double total = st_fin(&tot), refscale = st_fin(&ab) + fabs(total);
    for (uint64_t c = 0; c < C; ++c) d[c] -= p->cell_target_sum[c] / p->target_total * total;
    memset(sw, 0, W * 8);
    memset(sf, 0, F * 8);
    for (uint64_t c = 0; c < C; ++c) {
      sw[p->cell_worker[c]] += d[c];
      sf[p->cell_firm[c]] += d[c];
    }
    /* balance repair of the last entry */
    double* sides[2] = {sw, sf};
    uint64_t lens[2] = {W, F};
    for (int k = 0; k < 2; ++k) {
      Stable pre = {0, 0};
      for (uint64_t i = 0; i + 1 < lens[k]; ++i) st_add(&pre, sides[k][i]);
      double last = -st_fin(&pre), orig = sides[k][lens[k] - 1];
      if ((refscale == 0.0 && last != orig) || (refscale > 0.0 && fabs(last - orig) > 4096.0 * 2.220446049250313e-16 * refscale))
        return set_error(res, 77, "compatibility repair exceeded roundoff");
      sides[k][lens[k] - 1] = last;
    }
    memset(zw, 0, W * 8);
    memset(zf, 0, F * 8);
    solve(&s, sw, zf, alpha, psi);   /* worker side: (score_W, 0) */
    solve(&s, zw, sf, alpha2, psi2); /* firm side: (0, score_F) */
    res->solves += 2;
    Stable uu = {0, 0}, vv = {0, 0}, uv = {0, 0};
    for (uint64_t c = 0; c < C; ++c) {
      double u = alpha[p->cell_worker[c]] + psi[p->cell_firm[c]];
      double v = alpha2[p->cell_worker[c]] + psi2[p->cell_firm[c]];
      double wt = res->cell_correction_weight[c];
      st_add(&uu, wt * u * u);
      st_add(&vv, wt * v * v);
      st_add(&uv, wt * u * v);
    }
    double a = st_fin(&uu), b = st_fin(&vv), cv = st_fin(&uv);
    res->target_draws[probe * 4 + 0] = a;
    res->target_draws[probe * 4 + 1] = b;
    res->target_draws[probe * 4 + 2] = cv;
    res->target_draws[probe * 4 + 3] = a + b + 2.0 * cv;
  }
  /* ---- mean, corrected, MCSE */
  for (int k = 0; k < (o->phase == 2 ? 0 : 4); ++k) {
    Stable m = {0, 0};
    for (uint64_t q = 0; q < P; ++q) st_add(&m, res->target_draws[q * 4 + k]);
    res->correction[k] = st_fin(&m) / Pd;
    res->corrected[k] = res->plugin[k] - res->correction[k];
    Stable v = {0, 0};
    for (uint64_t q = 0; q < P; ++q) {
      double e = res->target_draws[q * 4 + k] - res->correction[k];
      st_add(&v, e * e);
    }
    res->mcse[k] = sqrt(st_fin(&v) / (Pd * (Pd - 1.0)));
  }
  res->cg_iterations = s.iterations;
  free(mom);
  free(atoms);
  free(cw);
  free(dir);
  free(d);
  free(sw);
  free(sf);
  free(zw);
  free(zf);
  free(bw);
  free(bf);
  free(alpha);
  free(psi);
  free(alpha2);
  free(psi2);
  solver_free(&s);
  return 0;
}

/* ------------------------------------------------------------ generic path */

static int dense_cholesky(double* a, int n) {
  for (int j = 0; j < n; ++j) {
    double d = a[j * n + j];
    for (int k = 0; k < j; ++k) d -= a[j * n + k] * a[j * n + k];
    if (!(d > 0.0)) return -1;
    d = sqrt(d);
    a[j * n + j] = d;
    for (int i = j + 1; i < n; ++i) {
      double v = a[i * n + j];
      for (int k = 0; k < j; ++k) v -= a[i * n + k] * a[j * n + k];
      a[i * n + j] = v / d;
    }
    for (int k = j + 1; k < n; ++k) a[j * n + k] = 0.0;
  }
  return 0;
}

static void dense_solve(const double* l, int n, double* b) {
  for (int i = 0; i < n; ++i) {
    double v = b[i];
    for (int k = 0; k < i; ++k) v -= l[i * n + k] * b[k];
    b[i] = v / l[i * n + i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double v = b[i];
    for (int k = i + 1; k < n; ++k) v -= l[k * n + i] * b[k];
    b[i] = v / l[i * n + i];
  }
}

/* Generic estimator: year controls through the FWL block, match deletion,
 * joint nuisance.  result->target_draws hold (worker, firm, covariance,
 * total) per probe; per-unit arrays are not filled. */
/* ---------------------------------------------- leave-observation-out */

static const uint64_t* g_rank_for_sort;
static int by_rank_then_row(const void* a, const void* b) {
  uint32_t x = *(const uint32_t*)a, y = *(const uint32_t*)b;
  if (g_rank_for_sort[x] != g_rank_for_sort[y]) return g_rank_for_sort[x] < g_rank_for_sort[y] ? -1 : 1;
  return x < y ? -1 : (x > y);
}

/* sign of copy `copy` of `entity`: bit copy % 64 of word copy / 64
 * (reference `rademacher_copy`, generic_jla.rs:10322-10329) */
static double copy_sign(uint64_t seed, uint64_t probe, uint64_t entity, uint64_t copy) {
  uint64_t b[4];
  oracle_philox_block(seed, TAG_LEVERAGE, probe / 4, entity, copy / 64, b);
  return ((b[probe % 4] >> (copy % 64)) & 1) ? 1.0 : -1.0;
}

/* Leverage probes with one sign per physical copy, the per-row and per-copy
 * moment sums, and the deleted residual of every row (reference
 * `observation_classes` generic_jla.rs:4158-4215,
 * `observation_and_match_leverage_moments` 5540-5881,
 * `observation_deleted_adjustment` 5893-6018, control leverage 4493-4523). */
static int observation_deleted(const OracleProblem* p, const OracleOptions* o, Solver* s, int q, const double* Rr,
                               const double* Si, const double* resid, double* deleted, OracleResult* res) {
  uint64_t W = p->workers, F = p->firms, R = p->rows, P = o->probes;
  double Pd = (double)P;
  /* classes: rows sorted by (rank, row); copies numbered through the class */
  uint32_t* order = malloc(R * sizeof(uint32_t));
  for (uint64_t r = 0; r < R; ++r) order[r] = (uint32_t)r;
  g_rank_for_sort = p->row_rank;
  qsort(order, R, sizeof(uint32_t), by_rank_then_row);
  uint64_t *off = calloc(R, 8), *phys = calloc(R + 1, 8);
  for (uint64_t i = 0, run = 0; i < R; ++i) {
    if (i > 0 && p->row_rank[order[i]] != p->row_rank[order[i - 1]]) run = 0;
    off[order[i]] = run;
    run += p->row_frequency[order[i]];
  }
  for (uint64_t r = 0; r < R; ++r) phys[r + 1] = phys[r] + p->row_frequency[r];
  uint64_t N = phys[R];
  Stable *p2 = calloc(R, sizeof(Stable)), *p4 = calloc(R, sizeof(Stable));
  Stable *c1 = calloc(N, sizeof(Stable)), *c3 = calloc(N, sizeof(Stable));
  double *bw = calloc(W, 8), *bf = calloc(F, 8), *al = calloc(W, 8), *ps = calloc(F, 8);
  for (uint64_t probe = 0; probe < P; ++probe) {
    memset(bw, 0, W * 8);
    memset(bf, 0, F * 8);
    for (uint64_t r = 0; r < R; ++r) {
      double a = 0.0;
      for (uint64_t i = 0; i < p->row_frequency[r]; ++i) a += copy_sign(o->seed, probe, p->row_rank[r], off[r] + i);
      bw[p->row_worker[r]] += a;
      bf[p->row_firm[r]] += a;
    }
    solve(s, bw, bf, al, ps);
    for (uint64_t r = 0; r < R; ++r) {
      double pr = al[p->row_worker[r]] + ps[p->row_firm[r]];
      st_add(&p2[r], pr * pr);
      st_add(&p4[r], pr * pr * pr * pr);
      for (uint64_t i = 0; i < p->row_frequency[r]; ++i) {
        double sg = copy_sign(o->seed, probe, p->row_rank[r], off[r] + i);
        st_add(&c1[phys[r] + i], sg * pr);
        st_add(&c3[phys[r] + i], sg * pr * pr * pr);
      }
    }
  }
  int code = 0;
  for (uint64_t r = 0; r < R && !code; ++r) {
    Stable lv = {0, 0};
    for (int i = 0; i < q; ++i)
      for (int j = 0; j < q; ++j) st_add(&lv, Rr[r * q + i] * Si[i * q + j] * Rr[r * q + j]);
    double lev = st_fin(&lv);
    if (!isfinite(lev) || lev < -100.0 * o->rank_tolerance) {
      code = set_error(res, 73, "analytic control leverage is negative or nonfinite");
      break;
    }
    lev = lev > 0.0 ? lev : 0.0;
    double pf = st_fin(&p2[r]), pq = st_fin(&p4[r]);
    Stable inv = {0, 0};
    for (uint64_t i = 0; i < p->row_frequency[r]; ++i) {
      double first = st_fin(&c1[phys[r] + i]), third = st_fin(&c3[phys[r] + i]);
      double mp = pf, mr = Pd + pf - 2.0 * first, m4p = pq;
      double m4r = Pd + 6.0 * pf + pq - 4.0 * first - 4.0 * third, mx = pf + pq - 2.0 * third;
      double total = (mp + mr) / Pd;
      if (!isfinite(total) || total <= o->block_tolerance) {
        code = set_error(res, 74, "projection and residual masses are not positive");
        break;
      }
      double proj = (mp / Pd) / total, rs = (mr / Pd) / total;
      double q4 = m4p / Pd, r4 = m4r / Pd, mix = mx / Pd;
      double bias = (rs * q4 - proj * r4 + (rs - proj) * mix) / Pd;
      double var = (rs * rs * q4 + proj * proj * r4 - 2.0 * proj * rs * mix) / Pd;
      if (var < -100.0 * o->rank_tolerance) {
        code = set_error(res, 73, "finite-projection variance is negative");
        break;
      }
      if (var < 0) var = 0;
      double tr = rs - lev;
      if (!isfinite(tr) || tr <= o->block_tolerance) {
        code = set_error(res, 75, "estimated residual leverage is nonpositive");
        break;
      }
      double rc = 1.0 / tr, v = rc + bias * rc * rc - var * rc * rc * rc;
      if (!isfinite(v) || v <= 0.0) {
        code = set_error(res, 76, "finite-projection observation inverse is nonpositive");
        break;
      }
      st_add(&inv, v);
    }
    deleted[r] = resid[r] * (st_fin(&inv) / (double)p->row_frequency[r]);
  }
  free(order);
  free(off);
  free(phys);
  free(p2);
  free(p4);
  free(c1);
  free(c3);
  free(bw);
  free(bf);
  free(al);
  free(ps);
  return code;
}

int oracle_jla_generic(const OracleProblem* p, const OracleOptions* o, OracleResult* res) {
  uint64_t W = p->workers, F = p->firms, C = p->cells, G = p->units, S = p->strata, P = o->probes, R = p->rows;
  int q = (int)p->controls;
  Solver s;
  res->error_code = 0;
  const int observation = p->deletion_mode == 2;
  if (observation ? !p->row_rank : (q < 1 || !p->group_ptr))
    return set_error(res, 11, "the generic oracle needs controls and match groups, or observation ranks");
  if (solver_init(&s, p, o)) return set_error(res, 82, "grounded Schur factor is not positive definite");
  double *bw = calloc(W, 8), *bf = calloc(F, 8), *alpha = calloc(W, 8), *psi = calloc(F, 8);
  double *alpha2 = calloc(W, 8), *psi2 = calloc(F, 8);
  double *aH = calloc(W * q, 8), *pH = calloc(F * q, 8), *Rr = calloc(R * q, 8);
  const double* Q = p->control_values;
  /* H = (X'WX)^+ X'WQ, one FE solve per control column */
  for (int k = 0; k < q; ++k) {
    memset(bw, 0, W * 8);
    memset(bf, 0, F * 8);
    for (uint64_t r = 0; r < R; ++r) {
      double v = (double)p->row_frequency[r] * Q[k * R + r];
      bw[p->row_worker[r]] += v;
      bf[p->row_firm[r]] += v;
    }
    solve(&s, bw, bf, alpha, psi);
    for (uint64_t w = 0; w < W; ++w) aH[w * q + k] = alpha[w];
    for (uint64_t f = 0; f < F; ++f) pH[f * q + k] = psi[f];
  }
  /* residualised controls, S = R'WR, S^{-1}, lower factor of S^{-1} */
  double Sm[64] = {0}, Si[64] = {0}, Lf[64];
  for (uint64_t r = 0; r < R; ++r) {
    double f = (double)p->row_frequency[r];
    for (int k = 0; k < q; ++k)
      Rr[r * q + k] = Q[k * R + r] - (aH[p->row_worker[r] * q + k] + pH[p->row_firm[r] * q + k]);
    for (int i = 0; i < q; ++i)
      for (int j = 0; j < q; ++j) Sm[i * q + j] += f * Rr[r * q + i] * Rr[r * q + j];
  }
  double Lc[64];
  memcpy(Lc, Sm, sizeof(Lc));
  if (dense_cholesky(Lc, q)) return set_error(res, 82, "residualised control information is singular");
  for (int c = 0; c < q; ++c) {
    double b[8] = {0};
    b[c] = 1.0;
    dense_solve(Lc, q, b);
    for (int i = 0; i < q; ++i) Si[i * q + c] = b[i];
  }
  memcpy(Lf, Si, sizeof(Lf));
  if (dense_cholesky(Lf, q)) return set_error(res, 76, "control inverse square root failed");
  /* joint fit */
  memset(bw, 0, W * 8);
  memset(bf, 0, F * 8);
  for (uint64_t c = 0; c < C; ++c) {
    bw[p->cell_worker[c]] += p->cell_outcome_sum[c];
    bf[p->cell_firm[c]] += p->cell_outcome_sum[c];
  }
  solve(&s, bw, bf, alpha, psi);
  double ry[8] = {0}, beta[8] = {0};
  for (uint64_t r = 0; r < R; ++r)
    for (int k = 0; k < q; ++k) ry[k] += (double)p->row_frequency[r] * Rr[r * q + k] * p->row_outcome[r];
  for (int k = 0; k < q; ++k)
    for (int l = 0; l < q; ++l) beta[k] += Si[k * q + l] * ry[l];
  for (uint64_t w = 0; w < W; ++w)
    for (int k = 0; k < q; ++k) alpha[w] -= aH[w * q + k] * beta[k];
  for (uint64_t f = 0; f < F; ++f)
    for (int k = 0; k < q; ++k) psi[f] -= pH[f * q + k] * beta[k];
  double* resid = calloc(R, 8);
  for (uint64_t r = 0; r < R; ++r) {
    double fit = alpha[p->row_worker[r]] + psi[p->row_firm[r]];
    for (int k = 0; k < q; ++k) fit += Q[k * R + r] * beta[k];
    resid[r] = p->row_outcome[r] - fit;
  }
  {
    /* plug-in over cells with cell target sums (generic_jla.rs:3735-3776) */
    Stable wm = {0, 0}, fm = {0, 0};
    for (uint64_t c = 0; c < C; ++c) {
      st_add(&wm, p->cell_target_sum[c] * alpha[p->cell_worker[c]]);
      st_add(&fm, p->cell_target_sum[c] * psi[p->cell_firm[c]]);
    }
    double mw = st_fin(&wm) / p->target_total, mf = st_fin(&fm) / p->target_total;
    Stable a = {0, 0}, b = {0, 0}, cv = {0, 0}, t = {0, 0};
    for (uint64_t c = 0; c < C; ++c) {
      double x = alpha[p->cell_worker[c]] - mw, y = psi[p->cell_firm[c]] - mf, wt = p->cell_target_sum[c];
      st_add(&a, wt * x * x);
      st_add(&b, wt * y * y);
      st_add(&cv, wt * x * y);
      st_add(&t, wt * (x + y) * (x + y));
    }
    res->plugin[0] = st_fin(&a) / p->target_total;
    res->plugin[1] = st_fin(&b) / p->target_total;
    res->plugin[2] = st_fin(&cv) / p->target_total;
    res->plugin[3] = st_fin(&t) / p->target_total;
  }
  double* deleted = calloc(R, 8);
  double Pd = (double)P;
  Stable* mom = NULL;
  if (observation) {
    int err = observation_deleted(p, o, &s, q, Rr, Si, resid, deleted, res);
    if (err) return err;
    goto target;
  }
  /* FE-only leverage moments */
  mom = calloc(G * 5, sizeof(Stable));
  for (uint64_t probe = 0; probe < P; ++probe) {
    memset(bw, 0, W * 8);
    memset(bf, 0, F * 8);
    int64_t* at = calloc(G, sizeof(int64_t));
    for (uint64_t g = 0; g < G; ++g) {
      int ok;
      at[g] = oracle_rademacher_sum(o->seed, TAG_LEVERAGE, probe, p->unit_rank[g], p->unit_count[g], &ok);
      uint32_t c = p->unit_cell[g];
      bw[p->cell_worker[c]] += (double)at[g];
      bf[p->cell_firm[c]] += (double)at[g];
    }
    solve(&s, bw, bf, alpha2, psi2);
    for (uint64_t g = 0; g < G; ++g) {
      uint32_t c = p->unit_cell[g];
      double rn = sqrt((double)p->unit_count[g]);
      double pr = rn * (alpha2[p->cell_worker[c]] + psi2[p->cell_firm[c]]);
      double m = (double)at[g] / rn - pr, p2 = pr * pr, m2 = m * m;
      st_add(&mom[g * 5 + 0], p2);
      st_add(&mom[g * 5 + 1], m2);
      st_add(&mom[g * 5 + 2], p2 * p2);
      st_add(&mom[g * 5 + 3], m2 * m2);
      st_add(&mom[g * 5 + 4], p2 * m2);
    }
    free(at);
  }
  /* deleted residuals per match group: (I - V V') X = [sqrt(f) e, common] */
  for (uint64_t g = 0; g < G; ++g) {
    double pf = st_fin(&mom[g * 5 + 0]), mf = st_fin(&mom[g * 5 + 1]);
    double tm = (pf + mf) / Pd;
    if (!(tm > o->block_tolerance)) return set_error(res, 74, "projection/residual mass failed");
    double proj = (pf / Pd) / tm, rs = (mf / Pd) / tm;
    double p4 = st_fin(&mom[g * 5 + 2]) / Pd, m4 = st_fin(&mom[g * 5 + 3]) / Pd, mx = st_fin(&mom[g * 5 + 4]) / Pd;
    double bias = (rs * p4 - proj * m4 + (rs - proj) * mx) / Pd;
    double var = (rs * rs * p4 + proj * proj * m4 - 2.0 * proj * rs * mx) / Pd;
    if (var < 0) var = 0;
    uint64_t b = p->group_ptr[g], e = p->group_ptr[g + 1];
    int width = (int)(e - b), rank = 1 + q;
    double* V = calloc((size_t)width * rank, 8);
    double* A = calloc((size_t)width * width, 8);
    double *x0 = calloc(width, 8), *x1 = calloc(width, 8), *cm = calloc(width, 8);
    double n = (double)p->unit_count[g];
    for (int l = 0; l < width; ++l) {
      uint32_t r = p->group_rows[b + l];
      double root = sqrt((double)p->row_frequency[r]);
      cm[l] = root / sqrt(n);
      V[l * rank] = sqrt(proj) * cm[l];
      for (int oo = 0; oo < q; ++oo) {
        double v = 0;
        for (int in = 0; in < q; ++in) v += Rr[r * q + in] * Lf[in * q + oo];
        V[l * rank + 1 + oo] = root * v;
      }
      x0[l] = root * resid[r];
      x1[l] = cm[l];
    }
    for (int i = 0; i < width; ++i)
      for (int j = 0; j < width; ++j) {
        double v = i == j ? 1.0 : 0.0;
        for (int k = 0; k < rank; ++k) v -= V[i * rank + k] * V[j * rank + k];
        A[i * width + j] = v;
      }
    if (dense_cholesky(A, width)) return set_error(res, 75, "a match residual block is singular");
    dense_solve(A, width, x0);
    dense_solve(A, width, x1);
    double ct = 0, ci = 0;
    for (int l = 0; l < width; ++l) {
      ct += cm[l] * x0[l];
      ci += cm[l] * x1[l];
    }
    for (int l = 0; l < width; ++l) deleted[p->group_rows[b + l]] = x0[l] + bias * x1[l] * ct - var * x1[l] * ci * ct;
    free(V);
    free(A);
    free(x0);
    free(x1);
    free(cm);
  }
target:;
  double mean = 0.0;
  if (o->centering == 1) {
    double anchor = p->row_outcome[0];
    Stable sm = {0, 0};
    for (uint64_t r = 0; r < R; ++r)
      st_add(&sm, (p->row_outcome[r] - anchor) * ((double)p->row_frequency[r] / (double)p->physical_total));
    mean = anchor + st_fin(&sm);
  }
  /* target draws on the full model */
  Stable* dir = calloc(C, sizeof(Stable));
  double *d = calloc(C, 8), *sw = calloc(W, 8), *sf = calloc(F, 8), *zw = calloc(W, 8), *zf = calloc(F, 8);
  for (uint64_t probe = 0; probe < P; ++probe) {
    memset(dir, 0, C * sizeof(Stable));
    for (uint64_t k = 0; k < S; ++k) {
      int ok;
      int64_t a = oracle_rademacher_sum(o->seed, TAG_TARGET, probe, p->stratum_rank[k], p->stratum_count[k], &ok);
      st_add(&dir[p->stratum_cell[k]], sqrt(p->stratum_per_copy[k] / p->target_total) * (double)a);
    }
    Stable tot = {0, 0};
    for (uint64_t c = 0; c < C; ++c) {
      d[c] = st_fin(&dir[c]);
      st_add(&tot, d[c]);
    }
    double total = st_fin(&tot);
    for (uint64_t c = 0; c < C; ++c) d[c] -= p->cell_target_sum[c] / p->target_total * total;
    memset(sw, 0, W * 8);
    memset(sf, 0, F * 8);
    for (uint64_t c = 0; c < C; ++c) {
      sw[p->cell_worker[c]] += d[c];
      sf[p->cell_firm[c]] += d[c];
    }
    Stable pre = {0, 0};
    for (uint64_t i = 0; i + 1 < W; ++i) st_add(&pre, sw[i]);
    sw[W - 1] = -st_fin(&pre);
    Stable pre2 = {0, 0};
    for (uint64_t i = 0; i + 1 < F; ++i) st_add(&pre2, sf[i]);
    sf[F - 1] = -st_fin(&pre2);
    memset(zw, 0, W * 8);
    memset(zf, 0, F * 8);
    solve(&s, sw, zf, alpha, psi);
    solve(&s, zw, sf, alpha2, psi2);
    double bW[8] = {0}, bF[8] = {0};
    for (uint64_t r = 0; r < R; ++r) {
      double fr = (double)p->row_frequency[r];
      double uw = alpha[p->row_worker[r]] + psi[p->row_firm[r]], uf = alpha2[p->row_worker[r]] + psi2[p->row_firm[r]];
      for (int k = 0; k < q; ++k) {
        bW[k] += fr * Q[k * R + r] * uw;
        bF[k] += fr * Q[k * R + r] * uf;
      }
    }
    double betaW[8] = {0}, betaF[8] = {0};
    for (int k = 0; k < q; ++k)
      for (int l = 0; l < q; ++l) {
        betaW[k] -= Si[k * q + l] * bW[l];
        betaF[k] -= Si[k * q + l] * bF[l];
      }
    Stable out[3] = {{0, 0}, {0, 0}, {0, 0}};
    if (observation) {
      /* f y d u^2 per row (reference `target_contraction`, generic_jla.rs:8926-8937) */
      for (uint64_t r = 0; r < R; ++r) {
        double fr = (double)p->row_frequency[r];
        double u[3];
        u[0] = alpha[p->row_worker[r]] + psi[p->row_firm[r]];
        u[1] = alpha2[p->row_worker[r]] + psi2[p->row_firm[r]];
        for (int k = 0; k < q; ++k) {
          u[0] += Rr[r * q + k] * betaW[k];
          u[1] += Rr[r * q + k] * betaF[k];
        }
        u[2] = u[0] + u[1];
        for (int t = 0; t < 3; ++t) st_add(&out[t], fr * (p->row_outcome[r] - mean) * deleted[r] * u[t] * u[t]);
      }
    }
    for (uint64_t g = 0; g < (observation ? 0 : G); ++g) {
      Stable first[3] = {{0, 0}, {0, 0}, {0, 0}}, second[3] = {{0, 0}, {0, 0}, {0, 0}};
      for (uint64_t i = p->group_ptr[g]; i < p->group_ptr[g + 1]; ++i) {
        uint32_t r = p->group_rows[i];
        double fr = (double)p->row_frequency[r];
        double u[3];
        u[0] = alpha[p->row_worker[r]] + psi[p->row_firm[r]];
        u[1] = alpha2[p->row_worker[r]] + psi2[p->row_firm[r]];
        for (int k = 0; k < q; ++k) {
          u[0] += Rr[r * q + k] * betaW[k];
          u[1] += Rr[r * q + k] * betaF[k];
        }
        u[2] = u[0] + u[1];
        for (int t = 0; t < 3; ++t) {
          st_add(&first[t], fr * (p->row_outcome[r] - mean) * u[t]);
          st_add(&second[t], sqrt(fr) * deleted[r] * u[t]);
        }
      }
      for (int t = 0; t < 3; ++t) st_add(&out[t], st_fin(&first[t]) * st_fin(&second[t]));
    }
    double ww = st_fin(&out[0]), ff = st_fin(&out[1]), tt = st_fin(&out[2]);
    res->target_draws[probe * 4 + 0] = ww;
    res->target_draws[probe * 4 + 1] = ff;
    res->target_draws[probe * 4 + 2] = 0.5 * (tt - ww - ff);
    res->target_draws[probe * 4 + 3] = tt;
  }
  for (int k = 0; k < 4; ++k) {
    Stable m = {0, 0};
    for (uint64_t pp = 0; pp < P; ++pp) st_add(&m, res->target_draws[pp * 4 + k]);
    res->correction[k] = st_fin(&m) / Pd;
    res->corrected[k] = res->plugin[k] - res->correction[k];
    Stable v = {0, 0};
    for (uint64_t pp = 0; pp < P; ++pp) {
      double e = res->target_draws[pp * 4 + k] - res->correction[k];
      st_add(&v, e * e);
    }
    res->mcse[k] = sqrt(st_fin(&v) / (Pd * (Pd - 1.0)));
  }
  res->cg_iterations = s.iterations;
  free(bw);
  free(bf);
  free(alpha);
  free(psi);
  free(alpha2);
  free(psi2);
  free(aH);
  free(pH);
  free(Rr);
  free(resid);
  free(mom);
  free(deleted);
  free(dir);
  free(d);
  free(sw);
  free(sf);
  free(zw);
  free(zf);
  solver_free(&s);
  return 0;
}
