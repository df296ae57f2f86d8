/* adjoint.c -- FP64 CPU restatement of the trajectory adjoint.  TEST
 * INFRASTRUCTURE ONLY (the checker of the CUDA adjoint; the product never
 * links it).
 *
 * The reference has no gradients, so this restatement is pinned by central
 * finite differences of its own FP64 forward (tests/test_adjoint.py), and the
 * forward itself follows the reference's force definitions:
 *   LJ with the linear force shift          lj.cpp:439-448
 *   Ewald real space (explicit cutoff)       electrostatic_ewald_r.cpp:196-198
 *   Ewald k space over the reference k-set   initialize.cpp:184-222,
 *                                            electrostatic_ewald_k.cpp:197-234
 *   self energy                              electrostatic_ewald_k/energy.cpp:31-50
 *   velocity Verlet ("type 2")               md_simulator.cpp:555-668
 * on one periodic cube under the minimum image (all cutoffs <= L/2).
 *
 * Loss J = (1/M) sum_{t=1..M} U(r_t), U = LJ + Ewald real + Ewald k + self.
 * Parameters: eps, sigma (symmetric T x T, the gradient of a shared
 * off-diagonal value goes to both entries), per-type charges.
 */
#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define A_PI 3.14159265358979323846
#define A_2PI 6.28318530717958647692
#define A_PIS_INV 0.56418958354775628695

struct orc_adj {
  int64_t n;
  double L, V;
  int nt;
  double mass[ORC_ADJ_TMAX], charge[ORC_ADJ_TMAX];
  double eps[ORC_ADJ_TMAX * ORC_ADJ_TMAX], sig[ORC_ADJ_TMAX * ORC_ADJ_TMAX];
  double rc_lj, alpha, rc_r, k_e, dt;
  int kmax;
  int64_t nk;
  int *kn; /* 3 per k */
  double *fk;
  int32_t *type;
  /* scratch */
  double complex *ex, *ey, *ez; /* per atom, m = -kmax..kmax */
  double complex *S, *Sa, *T, *Ta;
};

static double complex phase(const orc_adj *a, int64_t i, const int *kn) {
  const int K = a->kmax, W = 2 * K + 1;
  return a->ex[i * W + kn[0] + K] * a->ey[i * W + kn[1] + K] * a->ez[i * W + kn[2] + K];
}

orc_adj *orc_adj_create(int64_t n, double L, int nt, const double *mass, const double *charge, const double *eps,
                        const double *sigma, double rc_lj, double alpha, double rc_r, int kmax, double k_e, double dt,
                        const int32_t *type) {
  if (nt < 1 || nt > ORC_ADJ_TMAX || n < 2) return NULL;
  orc_adj *a = calloc(1, sizeof(orc_adj));
  a->n = n;
  a->L = L;
  a->V = L * L * L;
  a->nt = nt;
  for (int t = 0; t < nt; ++t) {
    a->mass[t] = mass[t];
    a->charge[t] = charge[t];
  }
  memcpy(a->eps, eps, sizeof(double) * nt * nt);
  memcpy(a->sig, sigma, sizeof(double) * nt * nt);
  a->rc_lj = rc_lj;
  a->alpha = alpha;
  a->rc_r = rc_r;
  a->kmax = kmax;
  a->k_e = k_e;
  a->dt = dt;
  a->type = malloc(sizeof(int32_t) * n);
  memcpy(a->type, type, sizeof(int32_t) * n);
  /* the reference's k-set: first (2k)^3 of the kx, ky, kz nesting, 0 skipped */
  const int64_t used = (int64_t)(2 * kmax) * (2 * kmax) * (2 * kmax);
  a->kn = malloc(sizeof(int) * 3 * (used ? used : 1));
  a->fk = malloc(sizeof(double) * (used ? used : 1));
  int64_t k = 0;
  for (int x = -kmax; x <= kmax && k < used; ++x)
    for (int y = -kmax; y <= kmax && k < used; ++y)
      for (int z = -kmax; z <= kmax && k < used; ++z) {
        if (!x && !y && !z) continue;
        a->kn[3 * k] = x;
        a->kn[3 * k + 1] = y;
        a->kn[3 * k + 2] = z;
        const double ksq = (A_2PI / L) * (A_2PI / L) * (double)(x * x + y * y + z * z);
        a->fk[k] = exp(-ksq / (4 * alpha * alpha)) / ksq;
        ++k;
      }
  a->nk = k;
  const int W = 2 * kmax + 1;
  a->ex = malloc(sizeof(double complex) * n * W);
  a->ey = malloc(sizeof(double complex) * n * W);
  a->ez = malloc(sizeof(double complex) * n * W);
  const size_t nkk = (size_t)(a->nk ? a->nk : 1);
  a->S = malloc(sizeof(double complex) * nkk);
  a->T = malloc(sizeof(double complex) * nkk);
  a->Sa = malloc(sizeof(double complex) * nkk * ORC_ADJ_TMAX);
  a->Ta = malloc(sizeof(double complex) * nkk * ORC_ADJ_TMAX);
  return a;
}

void orc_adj_destroy(orc_adj *a) {
  if (!a) return;
  free(a->kn);
  free(a->fk);
  free(a->type);
  free(a->ex);
  free(a->ey);
  free(a->ez);
  free(a->S);
  free(a->T);
  free(a->Sa);
  free(a->Ta);
  free(a);
}

void orc_adj_set_params(orc_adj *a, const double *eps, const double *sigma, const double *charge) {
  const int nt = a->nt;
  if (eps) memcpy(a->eps, eps, sizeof(double) * nt * nt);
  if (sigma) memcpy(a->sig, sigma, sizeof(double) * nt * nt);
  if (charge) memcpy(a->charge, charge, sizeof(double) * nt);
}

static void phase_tables(orc_adj *a, const double *pos) {
  const int K = a->kmax, W = 2 * K + 1;
  for (int64_t i = 0; i < a->n; ++i)
    for (int d = 0; d < 3; ++d) {
      double complex *t = d == 0 ? a->ex : (d == 1 ? a->ey : a->ez);
      for (int m = -K; m <= K; ++m) t[i * W + m + K] = cexp(I * (A_2PI / a->L) * m * pos[3 * i + d]);
    }
}

/* Per type pair: c (force coefficient, F_i += c d), c1 = (1/r) dc/dr, U, and
 * the parameter derivatives dc/deps, dc/dsig, dU/deps, dU/dsig (LJ) and the
 * same divided by q_i q_j for the Ewald real-space part (c_q, U_q). */
typedef struct {
  double c, c1, U;
  double dc_e, dc_s, dU_e, dU_s; /* LJ */
  double cq, c1q, Uq;            /* Ewald real space per unit q_i q_j */
} pair_terms;

static pair_terms pair_eval(const orc_adj *a, int ti, int tj, double r2) {
  pair_terms p;
  memset(&p, 0, sizeof(p));
  const int nt = a->nt;
  const double rc2 = a->rc_lj * a->rc_lj;
  const double e = a->eps[ti * nt + tj], sg = a->sig[ti * nt + tj];
  if (r2 <= rc2 && e != 0) {
    const double s2 = sg * sg / r2, s6 = s2 * s2 * s2, s12 = s6 * s6;
    const double c2 = sg * sg / rc2, c6 = c2 * c2 * c2, c12 = c6 * c6;
    const double ce = 4 * ((-12 * s12 + 6 * s6) / r2 + (12 * c12 - 6 * c6) / rc2); /* c / eps */
    const double Ue = 4 * (s12 - s6) - 4 * (c12 - c6) + 4 * (12 * c12 - 6 * c6) * (r2 - rc2) / (2 * rc2);
    p.c += e * ce;
    p.c1 += e * 4 * (168 * s12 - 48 * s6) / (r2 * r2);
    p.U += e * Ue;
    p.dc_e = ce;
    p.dU_e = Ue;
    p.dc_s = e * 4 * ((-144 * s12 + 36 * s6) / r2 + (144 * c12 - 36 * c6) / rc2) / sg;
    p.dU_s = e * (4 * (12 * s12 - 6 * s6) - 4 * (12 * c12 - 6 * c6) + (r2 - rc2) / (2 * rc2) * 4 * (144 * c12 - 36 * c6)) / sg;
  }
  if (r2 <= a->rc_r * a->rc_r && a->k_e != 0) {
    const double r = sqrt(r2), al = a->alpha, beta = 2 * al * A_PIS_INV;
    const double G = exp(-al * al * r2), ec = erfc(al * r);
    const double E1 = -beta * G / r - ec / r2;                            /* dE/dr, E = erfc(al r)/r */
    const double E2 = beta * G * (2 * al * al + 2 / r2) + 2 * ec / (r2 * r); /* d2E/dr2 */
    p.cq = a->k_e * E1 / r;
    p.c1q = a->k_e * (E2 - E1 / r) / r2;
    p.Uq = a->k_e * ec / r;
  }
  return p;
}

static void min_image(const orc_adj *a, const double *pi, const double *pj, double *d) {
  for (int k = 0; k < 3; ++k) {
    d[k] = pj[k] - pi[k];
    d[k] -= a->L * nearbyint(d[k] / a->L);
  }
}

static int sym(const orc_adj *a, int ti, int tj) { return ti * a->nt + tj; }

/* Forces F (not accelerations), energy terms {lj, ewald_r, ewald_k, self} and
 * dU/dtheta.  Any output may be NULL. */
void orc_adj_forces(orc_adj *a, const double *pos, double *force, double *energy, double *dU_eps, double *dU_sig,
                    double *dU_q) {
  const int64_t n = a->n;
  const int nt = a->nt;
  double elj = 0, eew = 0, ge[ORC_ADJ_TMAX * ORC_ADJ_TMAX] = {0}, gs[ORC_ADJ_TMAX * ORC_ADJ_TMAX] = {0},
         gq[ORC_ADJ_TMAX] = {0};
  if (force) memset(force, 0, sizeof(double) * 3 * n);
  for (int64_t i = 0; i < n; ++i) {
    const int ti = a->type[i];
    const double qi = a->charge[ti];
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const int tj = a->type[j];
      const double qj = a->charge[tj];
      double d[3];
      min_image(a, &pos[3 * i], &pos[3 * j], d);
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const pair_terms p = pair_eval(a, ti, tj, r2);
      const double c = p.c + qi * qj * p.cq;
      if (force)
        for (int k = 0; k < 3; ++k) force[3 * i + k] += c * d[k];
      /* energies: each ordered pair carries half */
      elj += 0.5 * p.U;
      eew += 0.5 * qi * qj * p.Uq;
      ge[sym(a, ti, tj)] += 0.5 * p.dU_e;
      gs[sym(a, ti, tj)] += 0.5 * p.dU_s;
      gq[ti] += 0.5 * qj * p.Uq;
      gq[tj] += 0.5 * qi * p.Uq;
    }
  }
  /* k space */
  phase_tables(a, pos);
  const double C = 4 * A_PI * a->k_e / a->V;
  double ek = 0;
  for (int64_t k = 0; k < a->nk; ++k) {
    double complex S = 0, Sa[ORC_ADJ_TMAX] = {0};
    for (int64_t i = 0; i < n; ++i) {
      const double complex e = phase(a, i, &a->kn[3 * k]);
      S += a->charge[a->type[i]] * e;
      Sa[a->type[i]] += e;
    }
    a->S[k] = S;
    ek += 0.5 * C * a->fk[k] * creal(S * conj(S));
    for (int t = 0; t < nt; ++t) gq[t] += C * a->fk[k] * creal(Sa[t] * conj(S));
  }
  if (force)
    for (int64_t i = 0; i < n; ++i) {
      const double qi = a->charge[a->type[i]];
      for (int64_t k = 0; k < a->nk; ++k) {
        const double im = cimag(phase(a, i, &a->kn[3 * k]) * conj(a->S[k]));
        for (int d = 0; d < 3; ++d) force[3 * i + d] += C * qi * a->fk[k] * (A_2PI / a->L) * a->kn[3 * k + d] * im;
      }
    }
  double q2 = 0;
  for (int64_t i = 0; i < n; ++i) q2 += a->charge[a->type[i]] * a->charge[a->type[i]];
  const double eself = a->nk ? -A_PIS_INV * a->alpha * a->k_e * q2 : 0.0;
  if (a->nk)
    for (int64_t i = 0; i < n; ++i) gq[a->type[i]] += -2 * A_PIS_INV * a->alpha * a->k_e * a->charge[a->type[i]];
  if (energy) {
    energy[0] = elj;
    energy[1] = eew;
    energy[2] = ek;
    energy[3] = eself;
  }
  /* a shared off-diagonal parameter gets both entries' derivative */
  for (int x = 0; x < nt; ++x)
    for (int y = 0; y < nt; ++y) {
      if (dU_eps) dU_eps[x * nt + y] = x == y ? ge[x * nt + y] : ge[x * nt + y] + ge[y * nt + x];
      if (dU_sig) dU_sig[x * nt + y] = x == y ? gs[x * nt + y] : gs[x * nt + y] + gs[y * nt + x];
    }
  if (dU_q) memcpy(dU_q, gq, sizeof(double) * nt);
}

/* Vector-Jacobian product of the forces at pos with cotangent u:
 * w = (dF/dr)^T u, and u . dF/dtheta for eps, sigma, charges. */
void orc_adj_force_vjp(orc_adj *a, const double *pos, const double *u, double *w, double *g_eps, double *g_sig,
                       double *g_q) {
  const int64_t n = a->n;
  const int nt = a->nt;
  double ge[ORC_ADJ_TMAX * ORC_ADJ_TMAX] = {0}, gs[ORC_ADJ_TMAX * ORC_ADJ_TMAX] = {0}, gq[ORC_ADJ_TMAX] = {0};
  memset(w, 0, sizeof(double) * 3 * n);
  for (int64_t i = 0; i < n; ++i) {
    const int ti = a->type[i];
    const double qi = a->charge[ti];
    const double *ui = &u[3 * i];
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const int tj = a->type[j];
      const double qj = a->charge[tj];
      double d[3];
      min_image(a, &pos[3 * i], &pos[3 * j], d);
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const pair_terms p = pair_eval(a, ti, tj, r2);
      const double c = p.c + qi * qj * p.cq, c1 = p.c1 + qi * qj * p.c1q;
      const double du[3] = {u[3 * j] - ui[0], u[3 * j + 1] - ui[1], u[3 * j + 2] - ui[2]};
      const double dd = d[0] * du[0] + d[1] * du[1] + d[2] * du[2];
      for (int k = 0; k < 3; ++k) w[3 * i + k] += c * du[k] + c1 * dd * d[k];
      const double ud = ui[0] * d[0] + ui[1] * d[1] + ui[2] * d[2];
      ge[sym(a, ti, tj)] += p.dc_e * ud;
      gs[sym(a, ti, tj)] += p.dc_s * ud;
      gq[ti] += qj * p.cq * ud;
      gq[tj] += qi * p.cq * ud;
    }
  }
  phase_tables(a, pos);
  const double C = 4 * A_PI * a->k_e / a->V, kf = A_2PI / a->L;
  for (int64_t k = 0; k < a->nk; ++k) {
    const int *kn = &a->kn[3 * k];
    double complex S = 0, T = 0, Sa[ORC_ADJ_TMAX] = {0}, Ta[ORC_ADJ_TMAX] = {0};
    for (int64_t i = 0; i < n; ++i) {
      const double complex e = phase(a, i, kn);
      const double q = a->charge[a->type[i]];
      const double ku = kf * (kn[0] * u[3 * i] + kn[1] * u[3 * i + 1] + kn[2] * u[3 * i + 2]);
      S += q * e;
      T += q * ku * e;
      Sa[a->type[i]] += e;
      Ta[a->type[i]] += ku * e;
    }
    a->S[k] = S;
    a->T[k] = T;
    for (int t = 0; t < nt; ++t) gq[t] += C * a->fk[k] * cimag(Ta[t] * conj(S) + T * conj(Sa[t]));
  }
  for (int64_t i = 0; i < n; ++i) {
    const double qi = a->charge[a->type[i]];
    for (int64_t k = 0; k < a->nk; ++k) {
      const int *kn = &a->kn[3 * k];
      const double complex e = phase(a, i, kn);
      const double ku = kf * (kn[0] * u[3 * i] + kn[1] * u[3 * i + 1] + kn[2] * u[3 * i + 2]);
      const double coef = C * qi * a->fk[k] * (ku * creal(e * conj(a->S[k])) - creal(a->T[k] * conj(e)));
      for (int d = 0; d < 3; ++d) w[3 * i + d] += coef * kf * kn[d];
    }
  }
  for (int x = 0; x < nt; ++x)
    for (int y = 0; y < nt; ++y) {
      if (g_eps) g_eps[x * nt + y] = x == y ? ge[x * nt + y] : ge[x * nt + y] + ge[y * nt + x];
      if (g_sig) g_sig[x * nt + y] = x == y ? gs[x * nt + y] : gs[x * nt + y] + gs[y * nt + x];
    }
  if (g_q) memcpy(g_q, gq, sizeof(double) * nt);
}

static double total(const double *e) { return e[0] + e[1] + e[2] + e[3]; }

/* J of M velocity-Verlet steps from (pos0, vel0); pos/vel outputs nullable. */
double orc_adj_loss(orc_adj *a, const double *pos0, const double *vel0, int64_t M, double *pos_out, double *vel_out) {
  const int64_t n = a->n;
  const double dt = a->dt;
  double *r = malloc(sizeof(double) * 3 * n), *v = malloc(sizeof(double) * 3 * n);
  double *F = malloc(sizeof(double) * 3 * n), *Fo = malloc(sizeof(double) * 3 * n);
  memcpy(r, pos0, sizeof(double) * 3 * n);
  memcpy(v, vel0, sizeof(double) * 3 * n);
  double e[4], J = 0;
  orc_adj_forces(a, r, F, NULL, NULL, NULL, NULL);
  for (int64_t t = 0; t < M; ++t) {
    for (int64_t i = 0; i < n; ++i) {
      const double mi = 1.0 / a->mass[a->type[i]];
      for (int d = 0; d < 3; ++d) r[3 * i + d] += v[3 * i + d] * dt + F[3 * i + d] * mi * 0.5 * dt * dt;
    }
    memcpy(Fo, F, sizeof(double) * 3 * n);
    orc_adj_forces(a, r, F, e, NULL, NULL, NULL);
    J += total(e);
    for (int64_t i = 0; i < n; ++i) {
      const double mi = 1.0 / a->mass[a->type[i]];
      for (int d = 0; d < 3; ++d) v[3 * i + d] += 0.5 * dt * (Fo[3 * i + d] + F[3 * i + d]) * mi;
    }
  }
  if (pos_out) memcpy(pos_out, r, sizeof(double) * 3 * n);
  if (vel_out) memcpy(vel_out, v, sizeof(double) * 3 * n);
  free(r);
  free(v);
  free(F);
  free(Fo);
  return M ? J / (double)M : 0.0;
}

/* dJ/d(pos0, vel0, eps, sigma, charge) by reverse-mode through the VV steps,
 * positions re-computed from checkpoints every K steps. */
double orc_adj_loss_grad(orc_adj *a, const double *pos0, const double *vel0, int64_t M, int64_t K, double *g_pos,
                         double *g_vel, double *g_eps, double *g_sig, double *g_q) {
  const int64_t n = a->n, n3 = 3 * n;
  const int nt = a->nt, ntt = nt * nt;
  const double dt = a->dt;
  if (K < 1) K = 1;
  const int64_t nseg = (M + K - 1) / K;
  double *ck_r = malloc(sizeof(double) * n3 * (nseg + 1)), *ck_v = malloc(sizeof(double) * n3 * (nseg + 1));
  double *segr = malloc(sizeof(double) * n3 * (K + 1)), *segF = malloc(sizeof(double) * n3 * (K + 1));
  double *r = malloc(sizeof(double) * n3), *v = malloc(sizeof(double) * n3), *F = malloc(sizeof(double) * n3),
         *Fo = malloc(sizeof(double) * n3);
  double *Gr = calloc(n3, sizeof(double)), *Gv = calloc(n3, sizeof(double)), *Ga = calloc(n3, sizeof(double));
  double *u = malloc(sizeof(double) * n3), *w = malloc(sizeof(double) * n3);
  double ge[ORC_ADJ_TMAX * ORC_ADJ_TMAX] = {0}, gs[ORC_ADJ_TMAX * ORC_ADJ_TMAX] = {0}, gq[ORC_ADJ_TMAX] = {0};
  double te[ORC_ADJ_TMAX * ORC_ADJ_TMAX], ts[ORC_ADJ_TMAX * ORC_ADJ_TMAX], tq[ORC_ADJ_TMAX], e[4];
  double J = 0;
  /* forward: loss, direct dU/dtheta, checkpoints (r, v) at t = s K */
  memcpy(r, pos0, sizeof(double) * n3);
  memcpy(v, vel0, sizeof(double) * n3);
  orc_adj_forces(a, r, F, NULL, NULL, NULL, NULL);
  for (int64_t t = 0; t < M; ++t) {
    if (t % K == 0) {
      memcpy(&ck_r[(t / K) * n3], r, sizeof(double) * n3);
      memcpy(&ck_v[(t / K) * n3], v, sizeof(double) * n3);
    }
    for (int64_t i = 0; i < n; ++i) {
      const double mi = 1.0 / a->mass[a->type[i]];
      for (int d = 0; d < 3; ++d) r[3 * i + d] += v[3 * i + d] * dt + F[3 * i + d] * mi * 0.5 * dt * dt;
    }
    memcpy(Fo, F, sizeof(double) * n3);
    orc_adj_forces(a, r, F, e, te, ts, tq);
    J += total(e);
    for (int x = 0; x < ntt; ++x) {
      ge[x] += te[x] / M;
      gs[x] += ts[x] / M;
    }
    for (int x = 0; x < nt; ++x) gq[x] += tq[x] / M;
    for (int64_t i = 0; i < n; ++i) {
      const double mi = 1.0 / a->mass[a->type[i]];
      for (int d = 0; d < 3; ++d) v[3 * i + d] += 0.5 * dt * (Fo[3 * i + d] + F[3 * i + d]) * mi;
    }
  }
  /* reverse, one segment at a time */
  for (int64_t s = nseg - 1; s >= 0; --s) {
    const int64_t t0 = s * K, t1 = (t0 + K < M) ? t0 + K : M;
    memcpy(r, &ck_r[s * n3], sizeof(double) * n3);
    memcpy(v, &ck_v[s * n3], sizeof(double) * n3);
    orc_adj_forces(a, r, F, NULL, NULL, NULL, NULL);
    memcpy(&segr[0], r, sizeof(double) * n3);
    memcpy(&segF[0], F, sizeof(double) * n3);
    for (int64_t t = t0; t < t1; ++t) {
      const int64_t q = t - t0 + 1;
      for (int64_t i = 0; i < n; ++i) {
        const double mi = 1.0 / a->mass[a->type[i]];
        for (int d = 0; d < 3; ++d) r[3 * i + d] += v[3 * i + d] * dt + F[3 * i + d] * mi * 0.5 * dt * dt;
      }
      memcpy(Fo, F, sizeof(double) * n3);
      orc_adj_forces(a, r, F, NULL, NULL, NULL, NULL);
      for (int64_t i = 0; i < n; ++i) {
        const double mi = 1.0 / a->mass[a->type[i]];
        for (int d = 0; d < 3; ++d) v[3 * i + d] += 0.5 * dt * (Fo[3 * i + d] + F[3 * i + d]) * mi;
      }
      memcpy(&segr[q * n3], r, sizeof(double) * n3);
      memcpy(&segF[q * n3], F, sizeof(double) * n3);
    }
    for (int64_t t = t1 - 1; t >= t0; --t) {
      const int64_t q = t - t0 + 1; /* r_{t+1} */
      for (int64_t x = 0; x < n3; ++x) {
        Gr[x] -= segF[q * n3 + x] / M; /* dU/dr = -F */
        Ga[x] += 0.5 * dt * Gv[x];
        u[x] = Ga[x] / a->mass[a->type[x / 3]];
      }
      orc_adj_force_vjp(a, &segr[q * n3], u, w, te, ts, tq);
      for (int x = 0; x < ntt; ++x) {
        ge[x] += te[x];
        gs[x] += ts[x];
      }
      for (int x = 0; x < nt; ++x) gq[x] += tq[x];
      for (int64_t x = 0; x < n3; ++x) {
        Gr[x] += w[x];
        const double gv = Gv[x];
        Gv[x] = gv + dt * Gr[x];
        Ga[x] = 0.5 * dt * gv + 0.5 * dt * dt * Gr[x];
      }
    }
  }
  /* a_0 = A(r_0) */
  for (int64_t x = 0; x < n3; ++x) u[x] = Ga[x] / a->mass[a->type[x / 3]];
  orc_adj_force_vjp(a, pos0, u, w, te, ts, tq);
  for (int x = 0; x < ntt; ++x) {
    ge[x] += te[x];
    gs[x] += ts[x];
  }
  for (int x = 0; x < nt; ++x) gq[x] += tq[x];
  for (int64_t x = 0; x < n3; ++x) Gr[x] += w[x];
  if (g_pos) memcpy(g_pos, Gr, sizeof(double) * n3);
  if (g_vel) memcpy(g_vel, Gv, sizeof(double) * n3);
  if (g_eps) memcpy(g_eps, ge, sizeof(double) * ntt);
  if (g_sig) memcpy(g_sig, gs, sizeof(double) * ntt);
  if (g_q) memcpy(g_q, gq, sizeof(double) * nt);
  free(ck_r);
  free(ck_v);
  free(segr);
  free(segF);
  free(r);
  free(v);
  free(F);
  free(Fo);
  free(Gr);
  free(Gv);
  free(Ga);
  free(u);
  free(w);
  return M ? J / (double)M : 0.0;
}
