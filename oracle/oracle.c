/* oracle.c -- CPU FP64 restatement of CAVIAR's per-timestep particle path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Nothing in
 * caviar_b200/ links or calls this file; only tests/, __graft_entry__.smoke
 * and bench.py's cpu_baseline leg load it (through oracle/oracle.py).
 *
 * It restates, loop for loop and in the same floating-point evaluation order,
 * the serial reference (CAVIAR, paths relative to its project root):
 *   - owned wrap            Domain::fix_position            src/caviar/objects/domain.cpp:418-468
 *   - ghost images          exchange_ghost_single_md_domain src/caviar/objects/atom_data/exchange_ghost_single_md_domain.cpp:26-218
 *   - cell bins             Neighborlist::init/binlist_index/update_cell_list/make_neigh_bin
 *                                                           src/caviar/objects/neighborlist.cpp:313-472,581-697
 *   - Verlet list           update_verlet_list_from_cell_list neighborlist.cpp:515-573
 *   - rebuild trigger       update_is_needed                neighborlist.cpp:91-139
 *   - LJ                    force_field::Lj::calculate_acceleration src/caviar/objects/force_field/lj.cpp:355-483
 *   - Ewald real space      Electrostatic_ewald_r::calculate_acceleration electrostatic_ewald_r.cpp:115-317
 *   - Ewald k space         make_k_vectors, S(k), force     electrostatic_ewald_k/initialize.cpp:31-222,
 *                                                           electrostatic_ewald_k.cpp:161-234
 *   - k-space / self energy electrostatic_ewald_k/energy.cpp:31-116, potential.cpp:47-130
 *   - velocity Verlet       Md_simulator::integrate_velocity_verlet src/caviar/objects/md_simulator.cpp:555-668
 *   - kinetic energy        Atom_data::kinetic_energy       src/caviar/objects/atom_data/kinetic_energy.cpp:30-154,413-456
 * Because the order of every sum is the reference's, accelerations agree with
 * the reference bit for bit (checked by tests/test_oracle_vs_reference.py).
 *
 * The restatement also supplies what the reference lacks: the LJ energy of
 * its linear force-shifted potential, the Ewald real-space energy of the
 * list pairs its forces use, and a displacement-only rebuild policy.
 *
 * Compile with -ffp-contract=off (oracle/Makefile) so that no multiply-add is
 * fused, like the reference's baseline x86-64 build.
 */
#include "oracle.h"

#include <complex.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* reference constants: include/caviar/utility/macro_constants.h:20-30 */
#define ORC_PI 3.14159265358979323846
#define ORC_2PI 6.28318530717958647692
#define ORC_4PI 12.56637061435917295384
#define ORC_PIS_INV 0.56418958354775628695

struct orc_sys {
  /* Domain (domain.cpp:206-266) */
  double lo[3], hi[3], L[3];
  int bc[3];
  /* Atom_data::atom_type_params */
  int nt;
  double *mass, *mass_inv, *charge;
  /* owned atoms; id == index */
  int64_t n;
  double *pos, *vel, *acc, *acc_old;
  int32_t *type, *mol;
  /* ghosts */
  int64_t ng, ng_cap;
  double *gpos;
  int64_t *gown;
  int8_t *gxv; /* x_val, y_val, z_val of exchange_ghost: image = pos - val*L */
  /* rebuild-check copies */
  double *pos_old, *gpos_old;
  int64_t ng_old;
  int have_old;
  /* Neighborlist */
  double cutoff, coef, gc, rl, rl_sq, thr_sq, cutoff_inv;
  int all_atom_test;
  int nb[3];
  int64_t nbins;
  int64_t *bin_start, *bin_items, *bin_fill;
  int64_t *nbr_start; /* neigh_bin in CSR */
  int64_t *nbr_items;
  /* Verlet list in CSR: entries j < n are owned, j >= n are ghost n+g */
  int64_t *nl_start;
  int64_t *nl_j;
  int64_t nl_cap;
  /* LJ */
  int lj_on;
  double lj_cut;
  double *eps, *sig, *cutl;
  int cutl_on, ignore_intra, jump_fix;
  double jump_tol;
  /* Ewald real space */
  int ewr_on;
  double ewr_alpha, ewr_ke, ewr_cut;
  double *lambda;
  /* Ewald k space */
  int ewk_on;
  double ewk_alpha, ewk_ke;
  int kmax[3];
  int64_t nk_used, nk_built;
  double *kvec, *fk;
  double complex *sk;
  double lx_inv, ly_inv, lz_inv, l_xyz_inv;
  /* integrator */
  double dt, k_b;
  int policy;
  /* scalars */
  double virial, e_lj, e_ewr, e_k, e_self;
  int64_t n_builds;
};

static void *xcalloc(size_t n, size_t sz) { return calloc(n ? n : 1, sz); }

orc_sys *orc_create(const double lo[3], const double hi[3], const int bc[3], int n_types,
                    const double *mass, const double *charge) {
  orc_sys *s = (orc_sys *)xcalloc(1, sizeof(orc_sys));
  for (int d = 0; d < 3; ++d) {
    s->lo[d] = lo[d];
    s->hi[d] = hi[d];
    s->L[d] = hi[d] - lo[d]; /* size_global = upper_global - lower_global (domain.cpp:470-477) */
    s->bc[d] = bc[d];
  }
  s->nt = n_types;
  s->mass = (double *)xcalloc((size_t)n_types, sizeof(double));
  s->mass_inv = (double *)xcalloc((size_t)n_types, sizeof(double));
  s->charge = (double *)xcalloc((size_t)n_types, sizeof(double));
  for (int t = 0; t < n_types; ++t) {
    s->mass[t] = mass[t];
    s->mass_inv[t] = (mass[t] == 0.0) ? 0.0 : 1.0 / mass[t]; /* atom_data.cpp:574-587 */
    s->charge[t] = charge ? charge[t] : 0.0;
  }
  s->coef = 1.12347; /* neighborlist.h:134 default */
  s->k_b = -1.0;
  return s;
}

static void free_lists(orc_sys *s) {
  free(s->bin_start); free(s->bin_items); free(s->bin_fill);
  free(s->nbr_start); free(s->nbr_items);
  s->bin_start = s->bin_items = s->bin_fill = s->nbr_start = s->nbr_items = NULL;
}

void orc_destroy(orc_sys *s) {
  if (!s) return;
  free(s->mass); free(s->mass_inv); free(s->charge);
  free(s->pos); free(s->vel); free(s->acc); free(s->acc_old);
  free(s->type); free(s->mol);
  free(s->gpos); free(s->gown); free(s->gxv);
  free(s->pos_old); free(s->gpos_old);
  free_lists(s);
  free(s->nl_start); free(s->nl_j);
  free(s->eps); free(s->sig); free(s->cutl); free(s->lambda);
  free(s->kvec); free(s->fk); free(s->sk);
  free(s);
}

int orc_set_atoms(orc_sys *s, int64_t n, const double *pos, const double *vel, const int32_t *type,
                  const int32_t *mol) {
  s->n = n;
  s->pos = (double *)realloc(s->pos, (size_t)(3 * n + 1) * sizeof(double));
  s->vel = (double *)realloc(s->vel, (size_t)(3 * n + 1) * sizeof(double));
  s->acc = (double *)realloc(s->acc, (size_t)(3 * n + 1) * sizeof(double));
  s->acc_old = (double *)realloc(s->acc_old, (size_t)(3 * n + 1) * sizeof(double));
  s->pos_old = (double *)realloc(s->pos_old, (size_t)(3 * n + 1) * sizeof(double));
  s->type = (int32_t *)realloc(s->type, (size_t)(n + 1) * sizeof(int32_t));
  s->mol = (int32_t *)realloc(s->mol, (size_t)(n + 1) * sizeof(int32_t));
  memcpy(s->pos, pos, (size_t)(3 * n) * sizeof(double));
  if (vel) memcpy(s->vel, vel, (size_t)(3 * n) * sizeof(double));
  else memset(s->vel, 0, (size_t)(3 * n) * sizeof(double));
  memset(s->acc, 0, (size_t)(3 * n) * sizeof(double));
  memset(s->acc_old, 0, (size_t)(3 * n) * sizeof(double));
  for (int64_t i = 0; i < n; ++i) {
    s->type[i] = type[i];
    s->mol[i] = mol ? mol[i] : -1;
    if (type[i] < 0 || type[i] >= s->nt) return -1;
  }
  s->have_old = 0;
  return 0;
}

void orc_set_neighborlist(orc_sys *s, double cutoff, double coef, double ghost_cutoff, int all_atom_test) {
  s->cutoff = cutoff;
  s->coef = coef;
  s->gc = ghost_cutoff;
  s->all_atom_test = all_atom_test;
}

static double *copy_tt(const orc_sys *s, const double *src) {
  if (!src) return NULL;
  double *d = (double *)xcalloc((size_t)(s->nt * s->nt), sizeof(double));
  memcpy(d, src, (size_t)(s->nt * s->nt) * sizeof(double));
  return d;
}

void orc_set_lj(orc_sys *s, double cutoff, const double *eps, const double *sigma, const double *cutoff_list,
                int ignore_intra, double jump_tol) {
  s->lj_on = 1;
  s->lj_cut = cutoff;
  free(s->eps); free(s->sig); free(s->cutl);
  s->eps = copy_tt(s, eps);
  s->sig = copy_tt(s, sigma);
  s->cutl = copy_tt(s, cutoff_list);
  s->cutl_on = cutoff_list != NULL;
  s->ignore_intra = ignore_intra;
  s->jump_fix = jump_tol > 0;
  s->jump_tol = jump_tol;
}

void orc_set_ewald_r(orc_sys *s, double alpha, double ke, const double *lambda, double cutoff) {
  s->ewr_on = 1;
  s->ewr_alpha = alpha;
  s->ewr_ke = ke;
  free(s->lambda);
  s->lambda = copy_tt(s, lambda);
  s->ewr_cut = cutoff;
}

/* make_k_vectors: electrostatic_ewald_k/initialize.cpp:184-222, with the box
 * lengths and inverses of initialize() :49-79. */
void orc_set_ewald_k(orc_sys *s, double alpha, int kx, int ky, int kz, double ke) {
  s->ewk_on = 1;
  s->ewk_alpha = alpha;
  s->ewk_ke = ke;
  s->kmax[0] = kx; s->kmax[1] = ky; s->kmax[2] = kz;
  const double lx = s->L[0], ly = s->L[1], lz = s->L[2];
  s->lx_inv = 1.0 / lx;
  s->ly_inv = 1.0 / ly;
  s->lz_inv = 1.0 / lz;
  s->l_xyz_inv = 1.0 / (lx * ly * lz);
  s->nk_used = (int64_t)(2 * kx) * (2 * ky) * (2 * kz);
  const int64_t cap = (int64_t)(2 * kx + 1) * (2 * ky + 1) * (2 * kz + 1);
  free(s->kvec); free(s->fk); free(s->sk);
  s->kvec = (double *)xcalloc((size_t)(3 * cap), sizeof(double));
  s->fk = (double *)xcalloc((size_t)cap, sizeof(double));
  s->sk = (double complex *)xcalloc((size_t)(s->nk_used > 0 ? s->nk_used : 1), sizeof(double complex));
  const double alpha_sq = alpha * alpha;
  const double four_alpha2_inv = 1.0 / (4.0 * alpha_sq);
  int64_t m = 0;
  for (int a = -kx; a <= kx; ++a)
    for (int b = -ky; b <= ky; ++b)
      for (int c = -kz; c <= kz; ++c) {
        const double k0 = ORC_2PI * a * s->lx_inv;
        const double k1 = ORC_2PI * b * s->ly_inv;
        const double k2 = ORC_2PI * c * s->lz_inv;
        const double ksq = k0 * k0 + k1 * k1 + k2 * k2;
        if (ksq == 0) continue;
        const double ksq_inv = 1.0 / ksq;
        s->kvec[3 * m] = k0;
        s->kvec[3 * m + 1] = k1;
        s->kvec[3 * m + 2] = k2;
        s->fk[m] = ksq_inv * exp(-ksq * four_alpha2_inv);
        ++m;
      }
  s->nk_built = m;
  if (s->nk_used > m) s->nk_used = m;
}

void orc_set_integrator(orc_sys *s, double dt, double k_b, int policy) {
  s->dt = dt;
  s->k_b = k_b;
  s->policy = policy;
}

/* ---------------------------------------------------------------- wrap */

/* Domain::fix_position (domain.cpp:418-468): one if/else-if per periodic axis. */
static int wrap_owned(orc_sys *s) {
  int any = 0;
  for (int64_t i = 0; i < s->n; ++i)
    for (int d = 0; d < 3; ++d) {
      if (s->bc[d] != 1) continue;
      double *p = &s->pos[3 * i + d];
      if (*p < s->lo[d]) {
        any = 1;
        *p += s->L[d];
      } else if (*p > s->hi[d]) {
        any = 1;
        *p -= s->L[d];
      }
    }
  return any;
}

/* -------------------------------------------------------------- ghosts */

static void push_ghost(orc_sys *s, int64_t owner, int xv, int yv, int zv) {
  if (s->ng == s->ng_cap) {
    s->ng_cap = s->ng_cap ? 2 * s->ng_cap : 1024;
    s->gpos = (double *)realloc(s->gpos, (size_t)(3 * s->ng_cap) * sizeof(double));
    s->gown = (int64_t *)realloc(s->gown, (size_t)s->ng_cap * sizeof(int64_t));
    s->gxv = (int8_t *)realloc(s->gxv, (size_t)(3 * s->ng_cap));
  }
  const double *p = &s->pos[3 * owner];
  const int64_t g = s->ng++;
  /* pos[i].x - x_val * x_width, only on the axes whose val is used */
  s->gpos[3 * g] = xv ? p[0] - xv * s->L[0] : p[0];
  s->gpos[3 * g + 1] = yv ? p[1] - yv * s->L[1] : p[1];
  s->gpos[3 * g + 2] = zv ? p[2] - zv * s->L[2] : p[2];
  s->gown[g] = owner;
  s->gxv[3 * g] = (int8_t)xv;
  s->gxv[3 * g + 1] = (int8_t)yv;
  s->gxv[3 * g + 2] = (int8_t)zv;
}

/* exchange_ghost_single_md_domain.cpp:26-218: for each owned atom in index
 * order, classify each axis (lower zone first, else upper zone), then emit
 * images in the order x, y, z, xy, xz, yz, xyz. */
static void make_ghosts(orc_sys *s) {
  s->ng = 0;
  const double llow[3] = {s->lo[0] + s->gc, s->lo[1] + s->gc, s->lo[2] + s->gc};
  const double lupp[3] = {s->hi[0] - s->gc, s->hi[1] - s->gc, s->hi[2] - s->gc};
  for (int64_t i = 0; i < s->n; ++i) {
    int v[3];
    for (int d = 0; d < 3; ++d) {
      const double x = s->pos[3 * i + d];
      v[d] = (x < llow[d]) ? -1 : ((x > lupp[d]) ? 1 : 0);
      v[d] *= s->bc[d];
    }
    if (v[0]) push_ghost(s, i, v[0], 0, 0);
    if (v[1]) push_ghost(s, i, 0, v[1], 0);
    if (v[2]) push_ghost(s, i, 0, 0, v[2]);
    if (v[0] && v[1]) push_ghost(s, i, v[0], v[1], 0);
    if (v[0] && v[2]) push_ghost(s, i, v[0], 0, v[2]);
    if (v[1] && v[2]) push_ghost(s, i, 0, v[1], v[2]);
    if (v[0] && v[1] && v[2]) push_ghost(s, i, v[0], v[1], v[2]);
  }
}

/* Ghost positions from their owners' current positions, ghost set unchanged
 * (used between rebuilds by the displacement policy only). */
static void refresh_ghosts(orc_sys *s) {
  for (int64_t g = 0; g < s->ng; ++g) {
    const double *p = &s->pos[3 * s->gown[g]];
    for (int d = 0; d < 3; ++d) {
      const int v = s->gxv[3 * g + d];
      s->gpos[3 * g + d] = v ? p[d] - v * s->L[d] : p[d];
    }
  }
}

/* ---------------------------------------------------------------- bins */

/* Neighborlist::init (neighborlist.cpp:313-406) and make_neigh_bin (:581-697).
 * The stencil of bin k is nbr_items[27k .. 27k + nbr_cnt[k]). */
static void init_bins(orc_sys *s) {
  s->rl = s->cutoff * s->coef;
  s->thr_sq = 0.25 * (s->rl - s->cutoff) * (s->rl - s->cutoff);
  s->cutoff_inv = 1.0 / s->rl;
  s->rl_sq = s->rl * s->rl;
  for (int d = 0; d < 3; ++d) s->nb[d] = (int)ceil(s->L[d] * s->cutoff_inv);
  free_lists(s);
  s->nbins = (int64_t)s->nb[0] * s->nb[1] * s->nb[2];
  s->bin_start = (int64_t *)xcalloc((size_t)(s->nbins + 1), sizeof(int64_t));
  s->bin_fill = (int64_t *)xcalloc((size_t)(s->nbins + 1), sizeof(int64_t));
  s->nbr_start = (int64_t *)xcalloc((size_t)(s->nbins + 1), sizeof(int64_t)); /* counts */
  s->nbr_items = (int64_t *)xcalloc((size_t)(27 * s->nbins), sizeof(int64_t));
  for (int ix = 0; ix < s->nb[0]; ++ix)
    for (int iy = 0; iy < s->nb[1]; ++iy)
      for (int iz = 0; iz < s->nb[2]; ++iz) {
        int mn[3] = {ix - 1, iy - 1, iz - 1}, mx[3] = {ix + 1, iy + 1, iz + 1};
        for (int d = 0; d < 3; ++d)
          if (s->bc[d] == 0) {
            if (mn[d] == -1) mn[d] = 0;
            if (mx[d] == s->nb[d]) mx[d] = s->nb[d] - 1;
          }
        const int64_t k = ix + (int64_t)s->nb[0] * iy + (int64_t)s->nb[0] * s->nb[1] * iz;
        int64_t *items = &s->nbr_items[27 * k];
        int64_t cnt = 0;
        for (int a = mn[0]; a <= mx[0]; ++a)
          for (int b = mn[1]; b <= mx[1]; ++b)
            for (int c = mn[2]; c <= mx[2]; ++c) {
              int v[3] = {a, b, c};
              for (int d = 0; d < 3; ++d) {
                if (v[d] == s->nb[d]) v[d] = 0;
                if (v[d] == -1) v[d] = s->nb[d] - 1;
              }
              const int64_t code = v[0] + (int64_t)s->nb[0] * v[1] + (int64_t)s->nb[0] * s->nb[1] * v[2];
              /* remove_duplicates keeps the first occurrence (neighborlist.cpp:31-40) */
              int dup = 0;
              for (int64_t q = 0; q < cnt; ++q)
                if (items[q] == code) dup = 1;
              if (!dup) items[cnt++] = code;
            }
        s->nbr_start[k] = cnt;
      }
}

/* Neighborlist::binlist_index (neighborlist.cpp:408-430): floor, then clamp. */
static int64_t bin_of(const orc_sys *s, const double *p) {
  int ind[3];
  for (int d = 0; d < 3; ++d) {
    ind[d] = (int)floor((p[d] - s->lo[d]) * s->cutoff_inv);
    if (ind[d] < 0) ind[d] = 0;
    if (ind[d] >= s->nb[d]) ind[d] = s->nb[d] - 1;
  }
  return ind[0] + (int64_t)s->nb[0] * ind[1] + (int64_t)s->nb[0] * s->nb[1] * ind[2];
}

/* update_cell_list (neighborlist.cpp:439-472): owned first in index order,
 * then ghosts as n+g; a stable counting sort keeps that insertion order. */
static void update_cell_list(orc_sys *s) {
  const int64_t tot = s->n + s->ng;
  free(s->bin_items);
  s->bin_items = (int64_t *)xcalloc((size_t)tot, sizeof(int64_t));
  int64_t *b = (int64_t *)xcalloc((size_t)tot, sizeof(int64_t));
  memset(s->bin_start, 0, (size_t)(s->nbins + 1) * sizeof(int64_t));
  for (int64_t i = 0; i < tot; ++i) {
    b[i] = bin_of(s, i < s->n ? &s->pos[3 * i] : &s->gpos[3 * (i - s->n)]);
    s->bin_start[b[i] + 1]++;
  }
  for (int64_t k = 0; k < s->nbins; ++k) s->bin_start[k + 1] += s->bin_start[k];
  memcpy(s->bin_fill, s->bin_start, (size_t)(s->nbins + 1) * sizeof(int64_t));
  for (int64_t i = 0; i < tot; ++i) s->bin_items[s->bin_fill[b[i]]++] = i;
  free(b);
}

static void nl_push(orc_sys *s, int64_t *len, int64_t j) {
  if (*len == s->nl_cap) {
    s->nl_cap = s->nl_cap ? 2 * s->nl_cap : 4096;
    s->nl_j = (int64_t *)realloc(s->nl_j, (size_t)s->nl_cap * sizeof(int64_t));
  }
  s->nl_j[(*len)++] = j;
}

/* update_verlet_list_from_cell_list (neighborlist.cpp:515-573), and
 * all_atom_test_function (:161-191) when all_atom_test is set. */
static void build_verlet(orc_sys *s) {
  const int64_t n = s->n;
  s->nl_start = (int64_t *)realloc(s->nl_start, (size_t)(n + 1) * sizeof(int64_t));
  int64_t len = 0;
  for (int64_t i = 0; i < n; ++i) {
    s->nl_start[i] = len;
    if (s->all_atom_test) {
      for (int64_t j = i + 1; j < n; ++j) nl_push(s, &len, j);
      for (int64_t g = 0; g < s->ng; ++g) nl_push(s, &len, g + n);
      continue;
    }
    const int64_t bi = bin_of(s, &s->pos[3 * i]);
    for (int64_t q = 0; q < s->nbr_start[bi]; ++q) {
      const int64_t bj = s->nbr_items[27 * bi + q];
      for (int64_t t = s->bin_start[bj]; t < s->bin_start[bj + 1]; ++t) {
        const int64_t j = s->bin_items[t];
        double dr[3] = {s->pos[3 * i], s->pos[3 * i + 1], s->pos[3 * i + 2]};
        const double *pj;
        if (j >= n) {
          pj = &s->gpos[3 * (j - n)];
        } else {
          if (j <= i) continue;
          pj = &s->pos[3 * j];
        }
        dr[0] -= pj[0];
        dr[1] -= pj[1];
        dr[2] -= pj[2];
        if (dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2] < s->rl_sq) nl_push(s, &len, j);
      }
    }
  }
  s->nl_start[n] = len;
  /* pos_old = pos; ghost_pos_old = pos_ghost (neighborlist.cpp:567-568) */
  memcpy(s->pos_old, s->pos, (size_t)(3 * n) * sizeof(double));
  s->gpos_old = (double *)realloc(s->gpos_old, (size_t)(3 * s->ng + 1) * sizeof(double));
  memcpy(s->gpos_old, s->gpos, (size_t)(3 * s->ng) * sizeof(double));
  s->ng_old = s->ng;
  s->have_old = 1;
  s->n_builds++;
}

/* update_is_needed (neighborlist.cpp:91-139) without the rebuild_test branch. */
static int update_is_needed(const orc_sys *s) {
  if (!s->have_old || s->ng != s->ng_old) return 1;
  for (int64_t i = 0; i < s->n; ++i) {
    const double dx = s->pos[3 * i] - s->pos_old[3 * i];
    const double dy = s->pos[3 * i + 1] - s->pos_old[3 * i + 1];
    const double dz = s->pos[3 * i + 2] - s->pos_old[3 * i + 2];
    if (dx * dx + dy * dy + dz * dz > s->thr_sq) return 1;
  }
  for (int64_t g = 0; g < s->ng; ++g) {
    const double dx = s->gpos[3 * g] - s->gpos_old[3 * g];
    const double dy = s->gpos[3 * g + 1] - s->gpos_old[3 * g + 1];
    const double dz = s->gpos[3 * g + 2] - s->gpos_old[3 * g + 2];
    if (dx * dx + dy * dy + dz * dz > s->thr_sq) return 1;
  }
  return 0;
}

/* setup's wrap + ghosts + Neighborlist::init + build(true) (md_simulator.cpp:524-531). */
int orc_build_list(orc_sys *s) {
  init_bins(s);
  wrap_owned(s);
  make_ghosts(s);
  update_cell_list(s);
  build_verlet(s);
  return 0;
}

/* -------------------------------------------------------------- forces */

static inline const double *pos_of(const orc_sys *s, int64_t j) {
  return j < s->n ? &s->pos[3 * j] : &s->gpos[3 * (j - s->n)];
}
static inline int64_t owner_of(const orc_sys *s, int64_t j) { return j < s->n ? j : s->gown[j - s->n]; }

/* Lj::calculate_acceleration (lj.cpp:355-483). */
static void lj_forces(orc_sys *s) {
  const double cutoff_sq = s->lj_cut * s->lj_cut;
  double c = cutoff_sq;
  double virial = 0;
  const int nt = s->nt;
  for (int64_t i = 0; i < s->n; ++i) {
    const double *pi = &s->pos[3 * i];
    const int ti = s->type[i];
    const double mass_inv_i = s->mass_inv[ti];
    const int64_t id_i = i;
    const int mol_i = s->mol[i];
    for (int64_t e = s->nl_start[i]; e < s->nl_start[i + 1]; ++e) {
      const int64_t j = s->nl_j[e];
      const int ghost = j >= s->n;
      const int64_t o = owner_of(s, j);
      const double *pj = pos_of(s, j);
      const int tj = s->type[o];
      const int64_t id_j = o;
      if (s->ignore_intra && mol_i == s->mol[o]) continue;
      const double dr[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
      double dr_sq = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
      if (s->cutl_on) c = s->cutl[ti * nt + tj] * s->cutl[ti * nt + tj];
      if (dr_sq > c) continue;
      if (s->jump_fix && dr_sq < s->jump_tol) dr_sq = s->jump_tol;
      const double eps_ij = s->eps[ti * nt + tj];
      if (eps_ij == 0) continue;
      const double sigma_ij = s->sig[ti * nt + tj];
      const double r_c_sq_inv = 1 / c;
      const double rho_c_sq_inv = sigma_ij * sigma_ij * r_c_sq_inv;
      const double rho_c_6_inv = rho_c_sq_inv * rho_c_sq_inv * rho_c_sq_inv;
      const double rho_c_12_inv = rho_c_6_inv * rho_c_6_inv;
      const double dr_sq_inv = 1 / dr_sq;
      const double rho_sq_inv = sigma_ij * sigma_ij * dr_sq_inv;
      const double rho_6_inv = rho_sq_inv * rho_sq_inv * rho_sq_inv;
      const double rho_12_inv = rho_6_inv * rho_6_inv;
      const double forceCoef =
          4 * eps_ij * (-12 * rho_12_inv * dr_sq_inv + 6 * rho_6_inv * dr_sq_inv + 12 * rho_c_12_inv * r_c_sq_inv -
                        6 * rho_c_6_inv * r_c_sq_inv);
      if (id_i < id_j) virial += -forceCoef * dr_sq;
      const double f[3] = {dr[0] * forceCoef, dr[1] * forceCoef, dr[2] * forceCoef};
      for (int d = 0; d < 3; ++d) s->acc[3 * i + d] += f[d] * mass_inv_i;
      if (!ghost) {
        const double mass_inv_j = s->mass_inv[tj];
        for (int d = 0; d < 3; ++d) s->acc[3 * j + d] -= f[d] * mass_inv_j;
      }
    }
  }
  s->virial += virial;
}

/* Electrostatic_ewald_r::calculate_acceleration (electrostatic_ewald_r.cpp:115-227).
 * With ewr_cut < 0 (the reference) every list pair is summed. */
static void ewald_r_forces(orc_sys *s) {
  const double alpha = s->ewr_alpha, alpha_sq = alpha * alpha, ke = s->ewr_ke;
  const double cut_sq = s->ewr_cut >= 0 ? s->ewr_cut * s->ewr_cut : -1.0;
  double virial = 0;
  const int nt = s->nt;
  for (int64_t i = 0; i < s->n; ++i) {
    const double *pi = &s->pos[3 * i];
    const int ti = s->type[i];
    const double charge_i = s->charge[ti];
    const double mass_inv_i = s->mass_inv[ti];
    const int64_t id_i = i;
    const int mol_i = s->mol[i];
    for (int64_t e = s->nl_start[i]; e < s->nl_start[i + 1]; ++e) {
      const int64_t j = s->nl_j[e];
      const int ghost = j >= s->n;
      const int64_t o = owner_of(s, j);
      const double *pj = pos_of(s, j);
      const int tj = s->type[o];
      const int64_t id_j = o;
      double lambda_coef = 1.0;
      if (s->lambda && mol_i == s->mol[o]) {
        if (s->lambda[ti * nt + tj] == 0.0) continue;
        lambda_coef *= s->lambda[ti * nt + tj];
      }
      const double r[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
      if (r[0] == 0 && r[1] == 0 && r[2] == 0) continue;
      const double charge_j = s->charge[tj];
      const double rsq = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
      if (cut_sq >= 0 && rsq > cut_sq) continue;
      const double rnorm = sqrt(rsq);
      const double erfc_arg = alpha * rnorm;
      const double sum_r_x = (2 * alpha * ORC_PIS_INV * exp(-alpha_sq * rsq) + erfc(erfc_arg) / rnorm) * (1.0 / rsq);
      const double forceCoef = -lambda_coef * ke * charge_i * charge_j * sum_r_x;
      if (id_i < id_j) virial += -forceCoef * rsq;
      const double f[3] = {r[0] * forceCoef, r[1] * forceCoef, r[2] * forceCoef};
      for (int d = 0; d < 3; ++d) s->acc[3 * i + d] += f[d] * mass_inv_i;
      if (!ghost) {
        const double mass_inv_j = s->mass_inv[tj];
        for (int d = 0; d < 3; ++d) s->acc[3 * j + d] -= f[d] * mass_inv_j;
      }
    }
  }
  s->virial += virial;
}

/* calculate_potential_k_coef_cmplx (initialize.cpp:117-146) and
 * Electrostatic_ewald_k::calculate_acceleration (electrostatic_ewald_k.cpp:161-234):
 * k outer, atoms inner, complex exponentials as in the reference. */
static void ewald_k_forces(orc_sys *s) {
  const int64_t nk = s->nk_used;
  for (int64_t k = 0; k < nk; ++k) {
    const double *kv = &s->kvec[3 * k];
    double complex rho = 0;
    for (int64_t j = 0; j < s->n; ++j) {
      const double *p = &s->pos[3 * j];
      const double q = s->charge[s->type[j]];
      const double kr = kv[0] * p[0] + kv[1] * p[1] + kv[2] * p[2];
      rho += q * cexp(I * kr);
    }
    s->sk[k] = rho;
  }
  for (int64_t k = 0; k < nk; ++k) {
    const double *kv = &s->kvec[3 * k];
    const double complex sum_j_c = conj(s->sk[k]);
    for (int64_t i = 0; i < s->n; ++i) {
      const double *p = &s->pos[3 * i];
      const int ti = s->type[i];
      const double charge_i = s->charge[ti];
      const double mass_inv_i = s->mass_inv[ti];
      const double kr = kv[0] * p[0] + kv[1] * p[1] + kv[2] * p[2];
      const double sum_j = cimag(sum_j_c * cexp(I * kr));
      const double c4 = ORC_4PI * s->fk[k];
      const double sum_k[3] = {kv[0] * c4 * sum_j, kv[1] * c4 * sum_j, kv[2] * c4 * sum_j};
      const double fc = s->ewk_ke * charge_i * s->l_xyz_inv;
      for (int d = 0; d < 3; ++d) s->acc[3 * i + d] += (sum_k[d] * fc) * mass_inv_i;
    }
  }
}

int orc_compute_forces(orc_sys *s) {
  memset(s->acc, 0, (size_t)(3 * s->n) * sizeof(double)); /* reset_owned_acceleration */
  s->virial = 0;                                           /* reset_virial */
  if (s->lj_on) lj_forces(s);
  if (s->ewr_on) ewald_r_forces(s);
  if (s->ewk_on) ewald_k_forces(s);
  return 0;
}

/* ------------------------------------------------------------ energies */

/* k_space_potential(r) (potential.cpp:96-129), k_space_energy (energy.cpp:61-107). */
static double k_space_energy(const orc_sys *s) {
  double energy_k = 0;
  for (int64_t j = 0; j < s->n; ++j) {
    const double *r = &s->pos[3 * j];
    double sum_k = 0;
    for (int64_t k = 0; k < s->nk_used; ++k) {
      const double *kv = &s->kvec[3 * k];
      double complex rho = s->sk[k];
      const double kr = kv[0] * r[0] + kv[1] * r[1] + kv[2] * r[2];
      rho *= cexp(-I * kr);
      sum_k += s->fk[k] * creal(rho);
    }
    const double pot = ORC_4PI * s->l_xyz_inv * sum_k * s->ewk_ke;
    energy_k += s->charge[s->type[j]] * pot;
  }
  return 0.5 * energy_k;
}

/* self_energy (energy.cpp:31-50). */
static double self_energy(const orc_sys *s) {
  double sum_j = 0;
  for (int64_t j = 0; j < s->n; ++j) {
    const double q = s->charge[s->type[j]];
    sum_j += q * q;
  }
  return -ORC_PIS_INV * s->ewk_alpha * sum_j * s->ewk_ke;
}

/* LJ pair energy consistent with lj.cpp:439-448's force:
 * U(r) = U_LJ(r) - U_LJ(rc) + g(rc) (r^2 - rc^2) / (2 rc^2), g(rc) = 4 eps (12 rho_c^12 - 6 rho_c^6);
 * Ewald real-space pair energy lambda k_e q_i q_j erfc(alpha r)/r over the
 * same list pairs as the force.  Each pair once (id_i < id_j), like the virial. */
static void pair_energies(orc_sys *s) {
  double elj = 0, eew = 0;
  const int nt = s->nt;
  for (int64_t i = 0; i < s->n; ++i) {
    const double *pi = &s->pos[3 * i];
    const int ti = s->type[i];
    for (int64_t e = s->nl_start[i]; e < s->nl_start[i + 1]; ++e) {
      const int64_t j = s->nl_j[e];
      const int64_t o = owner_of(s, j);
      if (!(i < o)) continue;
      const double *pj = pos_of(s, j);
      const int tj = s->type[o];
      const double dr[3] = {pj[0] - pi[0], pj[1] - pi[1], pj[2] - pi[2]};
      const double r2 = dr[0] * dr[0] + dr[1] * dr[1] + dr[2] * dr[2];
      if (s->lj_on && !(s->ignore_intra && s->mol[i] == s->mol[o])) {
        double c = s->lj_cut * s->lj_cut;
        if (s->cutl_on) c = s->cutl[ti * nt + tj] * s->cutl[ti * nt + tj];
        const double eps = s->eps[ti * nt + tj], sig = s->sig[ti * nt + tj];
        if (r2 <= c && eps != 0) {
          const double s2 = sig * sig / r2, s6 = s2 * s2 * s2;
          const double c2 = sig * sig / c, c6 = c2 * c2 * c2;
          const double g_rc = 4 * eps * (12 * c6 * c6 - 6 * c6);
          elj += 4 * eps * (s6 * s6 - s6) - 4 * eps * (c6 * c6 - c6) + g_rc * (r2 - c) / (2 * c);
        }
      }
      if (s->ewr_on && r2 > 0) {
        double lam = 1.0;
        if (s->lambda && s->mol[i] == s->mol[o]) lam = s->lambda[ti * nt + tj];
        if (s->ewr_cut < 0 || r2 <= s->ewr_cut * s->ewr_cut) {
          const double r = sqrt(r2);
          eew += lam * s->ewr_ke * s->charge[ti] * s->charge[tj] * erfc(s->ewr_alpha * r) / r;
        }
      }
    }
  }
  s->e_lj = elj;
  s->e_ewr = eew;
}

int orc_energy(orc_sys *s) {
  pair_energies(s);
  s->e_k = s->ewk_on ? k_space_energy(s) : 0.0;
  s->e_self = s->ewk_on ? self_energy(s) : 0.0;
  return 0;
}

/* kinetic_energy_mpi_domain (kinetic_energy.cpp:30-73), owned_velocity_cm (:413-456). */
static double kinetic_energy(const orc_sys *s) {
  const int bcsum = s->bc[0] + s->bc[1] + s->bc[2];
  const int n_r_df = (bcsum == 0) ? 6 : (bcsum == 3 ? 3 : 6 - bcsum);
  double vcm[3] = {0, 0, 0};
  if (n_r_df >= 1 && n_r_df <= 3) {
    double msum = 0;
    for (int64_t i = 0; i < s->n; ++i) {
      const double m = s->mass[s->type[i]];
      msum += m;
      for (int d = 0; d < 3; ++d) vcm[d] += s->vel[3 * i + d] * m;
    }
    for (int d = 0; d < 3; ++d) vcm[d] = vcm[d] / msum;
  }
  double e = 0;
  for (int64_t i = 0; i < s->n; ++i) {
    const double v[3] = {s->vel[3 * i] - vcm[0], s->vel[3 * i + 1] - vcm[1], s->vel[3 * i + 2] - vcm[2]};
    e += s->mass[s->type[i]] * (v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  }
  return e * 0.5;
}

/* ---------------------------------------------------------- integrator */

int orc_setup(orc_sys *s) {
  orc_build_list(s);
  return orc_compute_forces(s);
}

/* integrate_velocity_verlet (md_simulator.cpp:555-668) with re_calculate_acc
 * (:361-374) and boundary_condition (:487-502). */
int orc_step(orc_sys *s) {
  const double dt = s->dt;
  const int64_t n = s->n;
  for (int64_t i = 0; i < n; ++i) {
    double *a = &s->acc[3 * i];
    if (isnan(a[0]) || isnan(a[1]) || isnan(a[2])) return -1; /* md_simulator.cpp:584-590 */
    for (int d = 0; d < 3; ++d) {
      s->pos[3 * i + d] += s->vel[3 * i + d] * dt + a[d] * 0.5 * dt * dt;
      s->acc_old[3 * i + d] = a[d];
    }
  }
  if (s->policy == ORC_REBUILD_DISPLACEMENT) {
    int need = !s->have_old;
    for (int64_t i = 0; i < n && !need; ++i) {
      const double dx = s->pos[3 * i] - s->pos_old[3 * i];
      const double dy = s->pos[3 * i + 1] - s->pos_old[3 * i + 1];
      const double dz = s->pos[3 * i + 2] - s->pos_old[3 * i + 2];
      if (dx * dx + dy * dy + dz * dz > s->thr_sq) need = 1;
    }
    if (need) {
      wrap_owned(s);
      make_ghosts(s);
      update_cell_list(s);
      build_verlet(s);
    } else {
      refresh_ghosts(s);
    }
  } else {
    int flag = wrap_owned(s);
    make_ghosts(s);
    update_cell_list(s);
    if (s->policy == ORC_REBUILD_EVERY_STEP) flag = 1;
    if (!flag) flag = update_is_needed(s);
    if (flag) build_verlet(s);
  }
  orc_compute_forces(s);
  const double h = 0.5 * dt;
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) s->vel[3 * i + d] += (s->acc[3 * i + d] + s->acc_old[3 * i + d]) * h;
  return 0;
}

/* -------------------------------------------------------------- output */

typedef struct {
  int32_t v[5];
} orc_pair;

static int pair_cmp(const void *a, const void *b) {
  const int32_t *x = ((const orc_pair *)a)->v, *y = ((const orc_pair *)b)->v;
  for (int k = 0; k < 5; ++k)
    if (x[k] != y[k]) return x[k] < y[k] ? -1 : 1;
  return 0;
}

int64_t orc_pairs(orc_sys *s, int32_t *out) {
  const int64_t m = s->nl_start ? s->nl_start[s->n] : 0;
  orc_pair *p = (orc_pair *)xcalloc((size_t)m, sizeof(orc_pair));
  for (int64_t i = 0; i < s->n; ++i)
    for (int64_t e = s->nl_start[i]; e < s->nl_start[i + 1]; ++e) {
      const int64_t j = s->nl_j[e];
      int32_t a = (int32_t)i, b;
      int sh[3] = {0, 0, 0};
      if (j < s->n) {
        b = (int32_t)j;
      } else {
        const int64_t g = j - s->n;
        b = (int32_t)s->gown[g];
        for (int d = 0; d < 3; ++d) sh[d] = -s->gxv[3 * g + d];
      }
      int flip = a > b;
      if (a == b) flip = (sh[0] < -sh[0]) || (sh[0] == -sh[0] && (sh[1] < -sh[1] || (sh[1] == -sh[1] && sh[2] < -sh[2])));
      if (flip) {
        int32_t t = a; a = b; b = t;
        for (int d = 0; d < 3; ++d) sh[d] = -sh[d];
      }
      orc_pair *q = &p[e];
      q->v[0] = a; q->v[1] = b; q->v[2] = sh[0]; q->v[3] = sh[1]; q->v[4] = sh[2];
    }
  qsort(p, (size_t)m, sizeof(orc_pair), pair_cmp);
  int64_t u = 0;
  for (int64_t e = 0; e < m; ++e)
    if (u == 0 || pair_cmp(&p[u - 1], &p[e]) != 0) p[u++] = p[e];
  if (out) memcpy(out, p, (size_t)u * sizeof(orc_pair));
  free(p);
  return u;
}

int orc_get_state(const orc_sys *s, double *pos, double *vel, double *acc) {
  if (pos) memcpy(pos, s->pos, (size_t)(3 * s->n) * sizeof(double));
  if (vel) memcpy(vel, s->vel, (size_t)(3 * s->n) * sizeof(double));
  if (acc) memcpy(acc, s->acc, (size_t)(3 * s->n) * sizeof(double));
  return 0;
}

int64_t orc_n_kvec_used(const orc_sys *s) { return s->ewk_on ? s->nk_used : 0; }

int orc_get_sk(const orc_sys *s, double *out) {
  for (int64_t k = 0; k < s->nk_used; ++k) {
    out[2 * k] = creal(s->sk[k]);
    out[2 * k + 1] = cimag(s->sk[k]);
  }
  return 0;
}

int orc_get_scalars(orc_sys *s, double *out) {
  const int bcsum = s->bc[0] + s->bc[1] + s->bc[2];
  const int n_r_df = (bcsum == 0) ? 6 : (bcsum == 3 ? 3 : 6 - bcsum);
  out[0] = s->virial;
  out[1] = kinetic_energy(s);
  out[2] = s->e_lj;
  out[3] = s->e_ewr;
  out[4] = s->e_k;
  out[5] = s->e_self;
  out[6] = (double)s->n_builds;
  out[7] = (double)s->ng;
  out[8] = (double)(3 * s->n - n_r_df);
  return 0;
}

/* ------------------------------------------------------------- replicas */

/* Minimum-image all-pairs forces for one small periodic box.  The pair
 * formulas are the reference's (lj.cpp:439-448, electrostatic_ewald_r.cpp:196-198);
 * the k space is the reference's k-set and force (initialize.cpp:184-222,
 * electrostatic_ewald_k.cpp:197-234), with S(k) summed over all atoms. */
void orc_replica_forces(int64_t n, const double *pos, const int32_t *type, double L, int nt, const double *mass,
                        const double *charge, const double *eps, const double *sigma, double rc_lj, double alpha,
                        double rc_r, int kmax, double k_e, double *acc, double *energy) {
  double e_lj = 0, e_r = 0, e_k = 0, e_self = 0, vir = 0;
  const double rc2 = rc_lj * rc_lj, rr2 = rc_r * rc_r, alpha_sq = alpha * alpha;
  for (int64_t i = 0; i < 3 * n; ++i) acc[i] = 0;
  for (int64_t i = 0; i < n; ++i) {
    const int ti = type[i];
    double f[3] = {0, 0, 0};
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const int tj = type[j];
      double d[3];
      for (int a = 0; a < 3; ++a) {
        d[a] = pos[3 * j + a] - pos[3 * i + a];
        d[a] -= L * rint(d[a] / L);
      }
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      double c = 0;
      const double e = eps[ti * nt + tj], sg = sigma[ti * nt + tj];
      if (r2 <= rc2 && e != 0) {
        const double rcinv = 1 / rc2;
        const double c2 = sg * sg * rcinv, c6 = c2 * c2 * c2, c12 = c6 * c6;
        const double r2i = 1 / r2, s2 = sg * sg * r2i, s6 = s2 * s2 * s2, s12 = s6 * s6;
        c += 4 * e * (-12 * s12 * r2i + 6 * s6 * r2i + 12 * c12 * rcinv - 6 * c6 * rcinv);
        const double g = 4 * e * (12 * c12 - 6 * c6);
        e_lj += 0.5 * (4 * e * (s12 - s6) - 4 * e * (c12 - c6) + g * (r2 - rc2) / (2 * rc2));
      }
      const double qq = k_e * charge[ti] * charge[tj];
      if (qq != 0 && r2 <= rr2 && r2 > 0) {
        const double r = sqrt(r2);
        const double s = (2 * alpha * ORC_PIS_INV * exp(-alpha_sq * r2) + erfc(alpha * r) / r) / r2;
        c -= qq * s;
        e_r += 0.5 * qq * erfc(alpha * r) / r;
      }
      for (int a = 0; a < 3; ++a) f[a] += c * d[a];
      vir += -0.5 * c * r2;
    }
    const double mi = mass[ti] == 0 ? 0 : 1 / mass[ti];
    for (int a = 0; a < 3; ++a) acc[3 * i + a] = f[a] * mi;
  }
  if (kmax > 0) {
    const double two_pi = ORC_2PI, V = L * L * L;
    const double four_alpha2_inv = 1.0 / (4.0 * alpha_sq);
    const int64_t used = (int64_t)(2 * kmax) * (2 * kmax) * (2 * kmax);
    int64_t m = 0;
    for (int a = -kmax; a <= kmax && m < used; ++a)
      for (int b = -kmax; b <= kmax && m < used; ++b)
        for (int cz = -kmax; cz <= kmax && m < used; ++cz) {
          const double k0 = two_pi * a / L, k1 = two_pi * b / L, k2 = two_pi * cz / L;
          const double ksq = k0 * k0 + k1 * k1 + k2 * k2;
          if (ksq == 0) continue;
          ++m;
          const double fk = (1.0 / ksq) * exp(-ksq * four_alpha2_inv);
          double complex S = 0;
          for (int64_t j = 0; j < n; ++j) {
            const double kr = k0 * pos[3 * j] + k1 * pos[3 * j + 1] + k2 * pos[3 * j + 2];
            S += charge[type[j]] * cexp(I * kr);
          }
          e_k += (2 * ORC_PI / V) * k_e * fk * (creal(S) * creal(S) + cimag(S) * cimag(S));
          for (int64_t i = 0; i < n; ++i) {
            const int ti = type[i];
            const double kr = k0 * pos[3 * i] + k1 * pos[3 * i + 1] + k2 * pos[3 * i + 2];
            const double t = cimag(conj(S) * cexp(I * kr));
            const double coef = k_e * charge[ti] * (4 * ORC_PI / V) * fk * t;
            const double mi = mass[ti] == 0 ? 0 : 1 / mass[ti];
            acc[3 * i] += coef * k0 * mi;
            acc[3 * i + 1] += coef * k1 * mi;
            acc[3 * i + 2] += coef * k2 * mi;
          }
        }
    double q2 = 0;
    for (int64_t j = 0; j < n; ++j) q2 += charge[type[j]] * charge[type[j]];
    e_self = -ORC_PIS_INV * alpha * q2 * k_e;
  }
  if (energy) {
    energy[0] = e_lj;
    energy[1] = e_r;
    energy[2] = e_k;
    energy[3] = e_self;
    energy[4] = vir;
  }
}

void orc_replica_run(int64_t n, double *pos, double *vel, double *acc, const int32_t *type, double L, int nt,
                     const double *mass, const double *charge, const double *eps, const double *sigma, double rc_lj,
                     double alpha, double rc_r, int kmax, double k_e, double dt, int64_t nsteps) {
  orc_replica_forces(n, pos, type, L, nt, mass, charge, eps, sigma, rc_lj, alpha, rc_r, kmax, k_e, acc, NULL);
  for (int64_t s = 0; s < nsteps; ++s) {
    for (int64_t i = 0; i < 3 * n; ++i) {
      vel[i] += 0.5 * dt * acc[i];
      pos[i] += dt * vel[i];
      pos[i] -= L * floor(pos[i] / L);
    }
    orc_replica_forces(n, pos, type, L, nt, mass, charge, eps, sigma, rc_lj, alpha, rc_r, kmax, k_e, acc, NULL);
    for (int64_t i = 0; i < 3 * n; ++i) vel[i] += 0.5 * dt * acc[i];
  }
}
