/*
 * ndyn_oracle.c -- CPU oracle (TEST INFRASTRUCTURE, not product code).
 *
 * Plain-C restatement of the reference Fortran FP64 OpenMP path
 * (stewmasterj/Ndyn_OMP src/).  Every routine cites the reference lines it
 * follows.  It is compiled with -ffp-contract=off and without fast-math so
 * that its arithmetic is the literal operation sequence written in the
 * reference (d2 = x*x; d2 += y*y; d2 += z*z, FP32 table index, ...).
 * Used only by tests/ (parity checker) and by bench.py (timed CPU baseline).
 */
#include "ndyn_oracle.h"

#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define ORA_PI 3.141592653589793

struct ora_sys {
  int mode, nthreads;
  /* mostCommon, src/mods.f90:2-9 */
  int np;
  int *typ; /* 1-based type ids */
  double *pos, *vel, *acc, *force, *ftmp;
  double potential, kinetic, virial[6], e0;
  double box[3], box_build[3];
  /* interpot, src/mods.f90:51-77 */
  double rcut, rcut2, ptrmin;
  int ntypes, npairs, ptsize;
  int *pairmat; /* ntypes x ntypes column-major, values 1..npairs or 0 */
  int asympots; /* some Pairs line is one-sided ('asym'), src/read_input.f90:131-133 */
  int springpots; /* some pair is a 'spring', src/read_input.f90:136 */
  double *ipos, initbox[3]; /* initial positions and box of the spring strains */
  double *mass;
  double *ptdr2, *ptrc2, *pairparams /* 4 x npairs */, *ppair, *fpair,
      *qprod;
  char (*pairname)[9];
  /* control + listData */
  ora_control c;
  double skinsq;
  int ncell, mcell[3], neimax, nlist_updates;
  int *list, *head, *vnl;
  double *displist;
  /* hold groups, src/mods.f90 groupStuff: hold(np), bcDir/bcParm per group */
  int nhold, *hold, *bcdir;
  double *bcparm;
  int lists_ready;
  int err;
};

/* ------------------------------------------------------------------ */
static double ipow(double x, int n) {
  /* x**n for a small positive integer constant, by repeated squaring */
  double r = 1.0, b = x;
  int first = 1;
  while (n > 0) {
    if (n & 1) {
      r = first ? b : r * b;
      first = 0;
    }
    n >>= 1;
    if (n) b = b * b;
  }
  return r;
}

static int name_is(const char *name, const char *opt) {
  return strcmp(name, opt) == 0;
}

/* the Fortran 'select case (trim(typ))' buckets of pot/dpot */
enum { P_NONE, P_SINE, P_COSINE, P_SOFT, P_SPRING, P_MORSE, P_BUCK, P_LJ, P_JOHN };

static int pot_kind(const char *n) {
  if (name_is(n, "sine")) return P_SINE;
  if (name_is(n, "cosine")) return P_COSINE;
  if (name_is(n, "soft")) return P_SOFT;
  if (name_is(n, "spring")) return P_SPRING;
  if (name_is(n, "morse") || name_is(n, "Morse") || name_is(n, "morsec") ||
      name_is(n, "morseC") || name_is(n, "MorseC"))
    return P_MORSE;
  if (name_is(n, "Buck") || name_is(n, "BuckC") || name_is(n, "buck") ||
      name_is(n, "buckC") || name_is(n, "buckc"))
    return P_BUCK;
  if (name_is(n, "LJ") || name_is(n, "LJC")) return P_LJ;
  if (name_is(n, "John")) return P_JOHN;
  return P_NONE;
}

/* damped shifted Coulomb constants, src/potentials.f90:10,23-25 */
static const double DSF_ALPHA = 0.2;
static void dsf_consts(double rc, double *vcon, double *fcon) {
  double rc2 = rc * rc;
  *vcon = erfc(DSF_ALPHA * rc) / rc;
  *fcon = (erfc(DSF_ALPHA * rc) / rc2 +
           2. * DSF_ALPHA / sqrt(ORA_PI) * exp(-DSF_ALPHA * DSF_ALPHA * rc2) / rc);
}

/* pot(), src/potentials.f90:59-152 */
double ora_pot(const char *typ, double r, const double *parm, double qprd,
               double rcut) {
  double pot = 0.0, tmp, D, r0, rc, alfa, A, rho, C, eps, sig, B, vcon, fcon;
  dsf_consts(rcut, &vcon, &fcon);
  switch (pot_kind(typ)) {
  case P_SINE: pot = sin(r) * sin(r) - 1.0; break;
  case P_COSINE: pot = cos(r) * cos(r) - 1.0; break;
  case P_SOFT: pot = parm[1] * (1.0 + cos(ORA_PI * r / parm[2])); break;
  case P_SPRING:
    rc = parm[0]; D = parm[1]; C = parm[2];
    r0 = r / rc * C;
    pot = D * (r0 * r0 - C * C);
    break;
  case P_MORSE:
    rc = parm[0]; D = parm[1]; r0 = parm[3]; alfa = parm[2];
    tmp = r - r0;
    if (r0 <= 0.0) tmp = 0.0;
    pot = exp(-alfa * tmp);
    pot = D * (pot * pot - 2.0 * pot);
    if (name_is(typ, "MorseC") || name_is(typ, "morseC"))
      pot = pot + qprd * (erfc(DSF_ALPHA * r) / r - vcon + fcon * (r - rc));
    break;
  case P_BUCK:
    rc = parm[0]; A = parm[1]; rho = parm[2]; C = parm[3];
    pot = A * exp(-r / rho) - C / ipow(r, 6);
    if (rho <= 0.0) pot = A - C / ipow(r, 6);
    if (name_is(typ, "BuckC"))
      pot = pot + qprd * (erfc(DSF_ALPHA * r) / r - vcon + fcon * (r - rc));
    break;
  case P_LJ:
    rc = parm[0]; eps = parm[1]; sig = parm[2];
    tmp = sig / r;
    pot = 4. * eps * (ipow(tmp, 12) - ipow(tmp, 6));
    if (name_is(typ, "LJC"))
      pot = pot + qprd * (erfc(DSF_ALPHA * r) / r - vcon + fcon * (r - rc));
    break;
  case P_JOHN:
    eps = parm[1]; r0 = parm[2]; rc = parm[3];
    A = 2. * ipow(r0, 3) / ipow(rc - r0, 3);
    B = 3. * ipow(r0, 2) / ipow(rc - r0, 2);
    tmp = (r - rc) / r0;
    pot = (r < rc) ? -eps * (A * ipow(tmp, 3) + B * ipow(tmp, 2)) : 0.0;
    break;
  default: return NAN;
  }
  return pot;
}

/* dpot(), src/potentials.f90:154-247 */
double ora_dpot(const char *typ, double r, const double *parm, double qprd,
                double rcut) {
  double dpot = 0.0, tmp, D, r0, rc, alfa, A, rho, C, eps, sig, B, vcon, fcon;
  dsf_consts(rcut, &vcon, &fcon);
  switch (pot_kind(typ)) {
  case P_SINE: dpot = sin(2.0 * r); break;
  case P_COSINE: dpot = -sin(2.0 * r); break;
  case P_SOFT: /* parameters differ from pot() on purpose: reference lines 169-170 */
    dpot = ORA_PI * parm[0] * sin(ORA_PI * r / parm[1]) / parm[1];
    break;
  case P_SPRING:
    rc = parm[0]; D = parm[1]; C = parm[2];
    r0 = r / rc * C;
    dpot = -2.0 * D * r0;
    break;
  case P_MORSE:
    D = parm[1]; r0 = parm[3]; alfa = parm[2];
    tmp = r - r0;
    if (r0 <= 0.0) { tmp = 0.0; r0 = 1.0; }
    dpot = exp(-alfa * tmp);
    dpot = 2. * D * alfa * (dpot * dpot - dpot) / r;
    if (name_is(typ, "MorseC") || name_is(typ, "morseC"))
      dpot = dpot + qprd * (erfc(DSF_ALPHA * r) / (r * r) +
                            2. * DSF_ALPHA / sqrt(ORA_PI) *
                                exp(-(DSF_ALPHA * DSF_ALPHA) * (r * r)) / r -
                            fcon);
    break;
  case P_BUCK:
    A = parm[1]; rho = parm[2]; C = parm[3];
    dpot = A * exp(-r / rho) / rho - 6. * C / ipow(r, 7);
    if (rho <= 0.0) dpot = A - 6. * C / ipow(r, 7);
    if (name_is(typ, "BuckC"))
      dpot = dpot + qprd * (erfc(DSF_ALPHA * r) / (r * r) +
                            2. * DSF_ALPHA / sqrt(ORA_PI) *
                                exp(-(DSF_ALPHA * DSF_ALPHA) * (r * r)) / r -
                            fcon);
    break;
  case P_LJ:
    eps = parm[1]; sig = parm[2];
    tmp = sig / r;
    dpot = 24. * eps * (2. * ipow(tmp, 12) / r - ipow(tmp, 6) / r);
    if (name_is(typ, "LJC"))
      dpot = dpot + qprd * (erfc(DSF_ALPHA * r) / (r * r) +
                            2. * DSF_ALPHA / sqrt(ORA_PI) *
                                exp(-(DSF_ALPHA * DSF_ALPHA) * (r * r)) / r -
                            fcon);
    break;
  case P_JOHN:
    eps = parm[1]; r0 = parm[2]; rc = parm[3];
    A = 2. * ipow(r0, 3) / ipow(rc - r0, 3);
    B = 3. * ipow(r0, 2) / ipow(rc - r0, 2);
    tmp = (r - rc) / r0;
    dpot = (r < rc) ? eps / r0 * (3. * A * ipow(tmp, 2) + 2. * B * tmp) : 0.0;
    break;
  default: return NAN;
  }
  return dpot;
}

/* ------------------------------------------------------------------ */
ora_sys *ora_new(void) {
  ora_sys *s = (ora_sys *)calloc(1, sizeof(ora_sys));
  if (!s) return NULL;
  s->nthreads = omp_get_max_threads();
  s->mode = ORA_MODE_REF;
  s->rcut = ORA_PI / 2.0; /* src/read_input.f90:27 */
  s->ptsize = 1000;
  s->ptrmin = 0.25;
  ora_default_control(&s->c);
  return s;
}

static void free_lists(ora_sys *s) {
  free(s->list); free(s->head); free(s->vnl); free(s->displist); free(s->ftmp);
  s->list = s->head = s->vnl = NULL;
  s->displist = s->ftmp = NULL;
  s->lists_ready = 0;
}

static void free_holds(ora_sys *s) {
  free(s->hold); free(s->bcdir); free(s->bcparm);
  s->hold = NULL; s->bcdir = NULL; s->bcparm = NULL;
  s->nhold = 0;
}

/* Hold NAME ... / Disp NAME x y z, src/read_input.f90:177-190: hold[i] is the
 * group of atom i (0 = none); group g moves by du along the axes dir marks */
int ora_set_holds(ora_sys *s, const int *hold, int ngroups, const int *dir, const double *du) {
  free_holds(s);
  if (!hold || ngroups <= 0) return ORA_OK;
  s->hold = (int *)malloc(sizeof(int) * (size_t)s->np);
  s->bcdir = (int *)malloc(sizeof(int) * 3 * (size_t)ngroups);
  s->bcparm = (double *)malloc(sizeof(double) * 3 * (size_t)ngroups);
  for (int i = 0; i < s->np; ++i) {
    if (hold[i] < 0 || hold[i] > ngroups) { free_holds(s); return ORA_ERR_ARG; }
    s->hold[i] = hold[i];
  }
  for (int k = 0; k < 3 * ngroups; ++k) { s->bcdir[k] = dir[k] != 0; s->bcparm[k] = du[k]; }
  s->nhold = ngroups;
  return ORA_OK;
}

/* initPositionSet, src/nd.f90:1731-1762: the spring strains' reference
 * positions (NULL = the current ones) and box (NULL = the current one) */
int ora_init_positions(ora_sys *s, const double *ipos, const double *ibox) {
  if (!s->pos) return ORA_ERR_ARG;
  if (!s->ipos) s->ipos = (double *)malloc(sizeof(double) * 3 * (size_t)s->np);
  memcpy(s->ipos, ipos ? ipos : s->pos, sizeof(double) * 3 * (size_t)s->np);
  memcpy(s->initbox, ibox ? ibox : s->box, sizeof(double) * 3);
  return ORA_OK;
}

static void free_state(ora_sys *s) {
  free(s->typ); free(s->pos); free(s->vel); free(s->acc); free(s->force);
  s->typ = NULL;
  s->pos = s->vel = s->acc = s->force = NULL;
}

static void free_pairs(ora_sys *s) {
  free(s->pairmat); free(s->ptdr2); free(s->ptrc2); free(s->pairparams);
  free(s->ppair); free(s->fpair); free(s->pairname); free(s->qprod);
  s->pairmat = NULL;
  s->ptdr2 = s->ptrc2 = s->pairparams = s->ppair = s->fpair = s->qprod = NULL;
  s->pairname = NULL;
}

void ora_free(ora_sys *s) {
  if (!s) return;
  free_lists(s); free_state(s); free_pairs(s); free_holds(s); free(s->ipos); free(s->mass);
  free(s);
}

void ora_set_threads(ora_sys *s, int n) { s->nthreads = n > 0 ? n : 1; }
int ora_get_threads(const ora_sys *s) { return s->nthreads; }
void ora_set_mode(ora_sys *s, int mode) { s->mode = mode; }

void ora_default_control(ora_control *c) {
  /* src/read_input.f90:18-41 */
  memset(c, 0, sizeof(*c));
  c->dt = 0.0001;
  c->skin = -1.0;
  c->neimax = 0;
  c->renei = 1; c->renei_freq = 1;
  c->out_steps = 40;
  c->step = 0;
  c->ke_freq = 1; c->p_freq = 1; c->e_freq = 1;
}

int ora_set_control(ora_sys *s, const ora_control *c) {
  if (c->out_steps < 1 || c->renei_freq < 1 || c->ke_freq < 1 || c->p_freq < 1 ||
      c->e_freq < 1)
    return ORA_ERR_ARG;
  s->c = *c;
  return ORA_OK;
}
int ora_get_control(const ora_sys *s, ora_control *c) { *c = s->c; return ORA_OK; }

int ora_set_types(ora_sys *s, int ntypes, const double *mass) {
  if (ntypes < 1) return ORA_ERR_ARG;
  free(s->mass);
  s->mass = (double *)malloc(sizeof(double) * ntypes);
  memcpy(s->mass, mass, sizeof(double) * ntypes);
  s->ntypes = ntypes;
  return ORA_OK;
}

/* 'Pairs' directive (src/read_input.f90:136-172) then buildPairTables
 * (src/potentials.f90:2-56). */
int ora_set_pairs(ora_sys *s, int npairs, double ptrmin, int ptsize,
                  const int *p1, const int *p2, const int *sym,
                  const char *names, const double *params, const int *nparams,
                  const double *qprod) {
  if (s->ntypes < 1 || npairs < 1 || ptsize < 2) return ORA_ERR_ARG;
  free_pairs(s);
  s->npairs = npairs; s->ptrmin = ptrmin; s->ptsize = ptsize;
  s->pairmat = (int *)calloc((size_t)s->ntypes * s->ntypes, sizeof(int));
  s->pairparams = (double *)calloc(4 * (size_t)npairs, sizeof(double));
  s->ptdr2 = (double *)calloc(npairs, sizeof(double));
  s->ptrc2 = (double *)calloc(npairs, sizeof(double));
  s->qprod = (double *)calloc(npairs, sizeof(double));
  s->pairname = (char(*)[9])calloc(npairs, 9);
  for (int j = 0; j < npairs; ++j) s->pairparams[4 * j] = s->rcut; /* :156 */
  s->asympots = 0;
  s->springpots = 0;
  for (int j = 0; j < npairs; ++j) {
    if (!sym[j]) s->asympots = 1;
    int a = p1[j], b = p2[j];
    if (a < 1 || a > s->ntypes || b < 1 || b > s->ntypes) return ORA_ERR_ARG;
    s->pairmat[(a - 1) + (b - 1) * s->ntypes] = j + 1;
    if (sym[j]) s->pairmat[(b - 1) + (a - 1) * s->ntypes] = j + 1;
    memcpy(s->pairname[j], names + 8 * j, 8);
    s->pairname[j][8] = 0;
    for (int k = 7; k >= 0 && (s->pairname[j][k] == ' ' || s->pairname[j][k] == 0); --k)
      s->pairname[j][k] = 0;
    if (pot_kind(s->pairname[j]) == P_NONE) return ORA_ERR_POTENTIAL;
    if (pot_kind(s->pairname[j]) == P_SPRING) s->springpots = 1;
    for (int k = 0; k < nparams[j] && k < 4; ++k) s->pairparams[4 * j + k] = params[4 * j + k];
    s->qprod[j] = qprod ? qprod[j] : 0.0;
  }
  size_t ts = (size_t)(ptsize + 1) * npairs;
  s->ppair = (double *)malloc(sizeof(double) * ts);
  s->fpair = (double *)malloc(sizeof(double) * ts);
  for (int j = 0; j < npairs; ++j) {
    double rcut = s->pairparams[4 * j];
    s->ptrc2[j] = rcut * rcut;
    s->ptdr2[j] = (s->ptrc2[j] - ptrmin) / (ptsize - 1);
    for (int i = 1; i <= ptsize + 1; ++i) {
      double sv = ptrmin + (double)(i - 1) * s->ptdr2[j];
      double r = sqrt(sv);
      s->ppair[(size_t)(ptsize + 1) * j + (i - 1)] =
          ora_pot(s->pairname[j], r, &s->pairparams[4 * j], s->qprod[j], rcut);
      s->fpair[(size_t)(ptsize + 1) * j + (i - 1)] =
          r * ora_dpot(s->pairname[j], r, &s->pairparams[4 * j], s->qprod[j], rcut);
    }
  }
  double mx = s->pairparams[0];
  for (int j = 1; j < npairs; ++j)
    if (s->pairparams[4 * j] > mx) mx = s->pairparams[4 * j];
  s->rcut = mx; /* :36 */
  s->rcut2 = mx * mx;
  s->lists_ready = 0;
  return ORA_OK;
}

int ora_get_tables(const ora_sys *s, double *pp, double *fp, double *rc2, double *dr2) {
  size_t ts = (size_t)(s->ptsize + 1) * s->npairs;
  if (pp) memcpy(pp, s->ppair, ts * sizeof(double));
  if (fp) memcpy(fp, s->fpair, ts * sizeof(double));
  if (rc2) memcpy(rc2, s->ptrc2, s->npairs * sizeof(double));
  if (dr2) memcpy(dr2, s->ptdr2, s->npairs * sizeof(double));
  return ORA_OK;
}
int ora_get_pairmat(const ora_sys *s, int *pm) {
  memcpy(pm, s->pairmat, sizeof(int) * s->ntypes * s->ntypes);
  return ORA_OK;
}
double ora_get_rcut(const ora_sys *s) { return s->rcut; }

int ora_set_state(ora_sys *s, int np, const int *typ, const double *pos,
                  const double *vel, const double *acc, const double box[3]) {
  if (np < 1) return ORA_ERR_ARG;
  free_state(s);
  free_lists(s);
  free_holds(s); /* hold groups name atoms of the previous state */
  free(s->ipos);
  s->ipos = NULL;
  s->np = np;
  s->typ = (int *)malloc(sizeof(int) * np);
  s->pos = (double *)malloc(sizeof(double) * 3 * np);
  s->vel = (double *)calloc(3 * (size_t)np, sizeof(double));
  s->acc = (double *)calloc(3 * (size_t)np, sizeof(double));
  s->force = (double *)calloc(3 * (size_t)np, sizeof(double));
  memcpy(s->typ, typ, sizeof(int) * np);
  memcpy(s->pos, pos, sizeof(double) * 3 * np);
  if (vel) memcpy(s->vel, vel, sizeof(double) * 3 * np);
  if (acc) memcpy(s->acc, acc, sizeof(double) * 3 * np);
  for (int d = 0; d < 3; ++d) s->box[d] = box[d];
  return ORA_OK;
}

int ora_get_state(const ora_sys *s, double *pos, double *vel, double *acc, double *box) {
  size_t n = 3 * (size_t)s->np * sizeof(double);
  if (pos) memcpy(pos, s->pos, n);
  if (vel) memcpy(vel, s->vel, n);
  if (acc) memcpy(acc, s->acc, n);
  if (box) memcpy(box, s->box, 3 * sizeof(double));
  return ORA_OK;
}

int ora_get_forces(const ora_sys *s, double *force, double *pe, double *vir, double *ke) {
  if (force) memcpy(force, s->force, 3 * (size_t)s->np * sizeof(double));
  if (pe) *pe = s->potential;
  if (vir) memcpy(vir, s->virial, 6 * sizeof(double));
  if (ke) *ke = s->kinetic;
  return ORA_OK;
}
int ora_get_np(const ora_sys *s) { return s->np; }

/* ------------------------------------------------------------------ */
/* link cells and Verlet list                                          */

/* getJcellNP, src/nd.f90:1261-1306 (0-based vector, 0-based cell id) */
static const int STENCIL[14][3] = {
    {0, 0, 0},  {0, 0, 1},  {0, 1, 0},   {0, 1, -1}, {0, 1, 1},
    {1, 0, 0},  {1, 0, -1}, {1, 0, 1},   {1, 1, 0},  {1, 1, -1},
    {1, 1, 1},  {1, -1, 0}, {1, -1, -1}, {1, -1, 1}};

static int fold_cell(int t, int m) {
  /* tmp = real(t+1)/real(M+1)-0.5 ; t = t - M*nint(tmp)   (FP32) */
  volatile float tmp = (float)(t + 1) / (float)(m + 1);
  tmp = tmp - 0.5f;
  return t - m * (int)lroundf(tmp);
}

static int jcell(const ora_sys *s, const int ixyz[3], int k) {
  int t[3];
  for (int d = 0; d < 3; ++d) t[d] = fold_cell(ixyz[d] + STENCIL[k][d], s->mcell[d]);
  return t[0] + t[1] * s->mcell[0] + t[2] * s->mcell[0] * s->mcell[1];
}

static inline double pair_d2(const double *pi, const double *pj, const double *box,
                             double rij[3]) {
  double sr0 = pi[0] - pj[0], sr1 = pi[1] - pj[1], sr2 = pi[2] - pj[2];
  sr0 = sr0 - round(sr0);
  sr1 = sr1 - round(sr1);
  sr2 = sr2 - round(sr2);
  rij[0] = box[0] * sr0;
  rij[1] = box[1] * sr1;
  rij[2] = box[2] * sr2;
  double d2 = rij[0] * rij[0];
  d2 = d2 + rij[1] * rij[1];
  d2 = d2 + rij[2] * rij[2];
  return d2;
}

static inline int pm(const ora_sys *s, int ta, int tb) {
  return s->pairmat[(ta - 1) + (tb - 1) * s->ntypes];
}

/* add all pairs (i in ic, j in jc) into the lists of i; same==1 is the
 * first, same-cell loop of buildVerletList (i<j, PTrMin exclusion). */
static int add_cell_pairs(ora_sys *s, int ic, int jc, int same) {
  const int stride = s->neimax + 1;
  for (int i = s->head[ic]; i >= 0; i = s->list[i]) {
    int typi = s->typ[i];
    int *row = s->vnl + (size_t)stride * i;
    int nj;
    if (same) {
      memset(row, 0, sizeof(int) * s->neimax); /* VNL(1:NeiMax,i) = 0 */
      nj = 1;
    } else {
      nj = row[0];
    }
    const double *pi = s->pos + 3 * (size_t)i;
    for (int j = s->head[jc]; j >= 0; j = s->list[j]) {
      if (same && i >= j) continue;
      int a = pm(s, typi, s->typ[j]), b = pm(s, s->typ[j], typi);
      int mx = a > b ? a : b;
      if (mx <= 0) continue;
      double rij[3];
      double d2 = pair_d2(pi, s->pos + 3 * (size_t)j, s->box, rij);
      double rcuts2 = s->c.skin + s->pairparams[4 * (mx - 1)];
      if (same && d2 < s->ptrmin) continue;
      if (d2 > rcuts2 * rcuts2) continue;
      if (nj > s->neimax) return ORA_ERR_NEIMAX;
      row[nj] = j; /* VNL(nj+1,i) = j */
      nj = nj + 1;
    }
    row[0] = nj;
    s->displist[3 * (size_t)i] = s->displist[3 * (size_t)i + 1] =
        s->displist[3 * (size_t)i + 2] = 0.0;
  }
  return ORA_OK;
}

/* buildVerletList, src/nd.f90:1328-1446 */
static int build_verlet_list(ora_sys *s) {
  int all3 = s->mcell[0] >= 3 && s->mcell[1] >= 3 && s->mcell[2] >= 3;
  for (int ic = 0; ic < s->ncell; ++ic) {
    int rc = add_cell_pairs(s, ic, ic, 1);
    if (rc) return rc;
    int ixyz[3];
    /* getCellVector(ic, IXYZ, .false.) src/nd.f90:1307-1327 */
    ixyz[0] = ic % s->mcell[0];
    ixyz[2] = ic / (s->mcell[0] * s->mcell[1]);
    ixyz[1] = (ic % (s->mcell[0] * s->mcell[1])) / s->mcell[0];
    if (s->mode == ORA_MODE_REF || all3) {
      for (int k = 1; k < 14; ++k) {
        rc = add_cell_pairs(s, ic, jcell(s, ixyz, k), 0);
        if (rc) return rc;
      }
    } else {
      /* fixed mode with a cell count < 3: each distinct neighbouring cell
       * pair once (cells with a larger id than ic) */
      int seen[27], nseen = 0;
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            int t[3] = {ixyz[0] + dx, ixyz[1] + dy, ixyz[2] + dz};
            for (int d = 0; d < 3; ++d) t[d] = fold_cell(t[d], s->mcell[d]);
            int jc = t[0] + t[1] * s->mcell[0] + t[2] * s->mcell[0] * s->mcell[1];
            if (jc <= ic) continue;
            int dup = 0;
            for (int q = 0; q < nseen; ++q) dup |= (seen[q] == jc);
            if (dup) continue;
            seen[nseen++] = jc;
            rc = add_cell_pairs(s, ic, jc, 0);
            if (rc) return rc;
          }
    }
  }
  return ORA_OK;
}

/* buildCellList, src/nd.f90:1214-1260 */
int ora_build_cell_list(ora_sys *s) {
  for (int c = 0; c < s->ncell; ++c) s->head[c] = -1;
  for (int i = 0; i < s->np; ++i) s->list[i] = -1;
  for (int i = 0; i < s->np; ++i) {
    int ixyz[3];
    for (int d = 0; d < 3; ++d) {
      double p = s->pos[3 * (size_t)i + d];
      double sr = p - round(p);
      ixyz[d] = (int)((sr + 0.4999) * (double)s->mcell[d]);
      if (ixyz[d] < 0 || ixyz[d] >= s->mcell[d]) return ORA_ERR_OUT_OF_BOX;
    }
    int icell = ixyz[0] + ixyz[1] * s->mcell[0] + ixyz[2] * s->mcell[0] * s->mcell[1];
    s->list[i] = s->head[icell];
    s->head[icell] = i;
  }
  for (int d = 0; d < 3; ++d) s->box_build[d] = s->box[d];
  return build_verlet_list(s);
}

static int compute_mcell(ora_sys *s) {
  for (int d = 0; d < 3; ++d) s->mcell[d] = (int)(s->box[d] / (s->rcut + s->c.skin));
  if (s->mcell[0] < 2 || s->mcell[1] < 2 || s->mcell[2] < 2) return ORA_ERR_CELLS;
  s->ncell = s->mcell[0] * s->mcell[1] * s->mcell[2];
  return ORA_OK;
}

/* dynamics prologue, src/nd.f90:73-108 */
int ora_setup_lists(ora_sys *s) {
  if (!s->pos || !s->ppair) return ORA_ERR_ARG;
  if (s->c.skin < 0.0) s->c.skin = s->rcut * 0.2;
  if (s->springpots && !s->ipos) ora_init_positions(s, NULL, NULL); /* src/nd.f90:104 */
  int rc = compute_mcell(s);
  if (rc) return rc;
  if (s->c.neimax == 0) {
    /* NeiMax = int(4./3.*PI*((rcut+skin)*1.1)**3*np/(box1*box2*box3));
     * 4./3. and 1.1 are default (single precision) reals */
    double f43 = (double)(4.0f / 3.0f);
    double r = (s->rcut + s->c.skin) * (double)1.1f;
    s->c.neimax = (int)(f43 * ORA_PI * (r * r * r) * (double)s->np /
                        (s->box[0] * s->box[1] * s->box[2]));
  }
  s->neimax = s->c.neimax;
  free_lists(s);
  s->head = (int *)malloc(sizeof(int) * s->ncell);
  s->vnl = (int *)calloc((size_t)(s->neimax + 1) * s->np, sizeof(int));
  s->list = (int *)malloc(sizeof(int) * s->np);
  s->displist = (double *)calloc(3 * (size_t)s->np, sizeof(double));
  s->ftmp = (double *)malloc(sizeof(double) * 3 * (size_t)s->np * s->nthreads);
  if (!s->head || !s->vnl || !s->list || !s->displist || !s->ftmp) return ORA_ERR_NOMEM;
  s->nlist_updates = 0;
  s->skinsq = s->c.skin * s->c.skin;
  rc = ora_build_cell_list(s);
  if (rc) return rc;
  s->lists_ready = 1;
  return ORA_OK;
}

/* CheckListUpdate, src/nd.f90:1447-1499 */
int ora_check_list_update(ora_sys *s) {
  double t1 = 0.0, t2 = 0.0;
  const int fixed = s->mode == ORA_MODE_FIXED;
  for (int i = 0; i < s->np; ++i) {
    const double *dl = s->displist + 3 * (size_t)i;
    double disp = dl[0] * dl[0];
    disp = disp + dl[1] * dl[1];
    disp = disp + dl[2] * dl[2];
    if (disp >= t1) { t2 = t1; t1 = disp; }
    else if (disp >= t2) t2 = disp;
  }
  double disp = t1 + t2;
  int rebuild;
  if (!fixed) {
    rebuild = disp > s->skinsq;
  } else {
    /* Angstrom displacements: the two largest moves plus any box shrink
     * since the build must stay below the skin */
    double a1 = 0.0, a2 = 0.0;
    double bmax = s->box[0] > s->box[1] ? s->box[0] : s->box[1];
    bmax = bmax > s->box[2] ? bmax : s->box[2];
    for (int i = 0; i < s->np; ++i) {
      const double *dl = s->displist + 3 * (size_t)i;
      double x = dl[0] * s->box[0], y = dl[1] * s->box[1], z = dl[2] * s->box[2];
      double d = x * x + y * y + z * z;
      if (d >= a1) { a2 = a1; a1 = d; } else if (d >= a2) a2 = d;
    }
    (void)bmax;
    double shrink = 0.0;
    for (int d = 0; d < 3; ++d) {
      double f = 1.0 - s->box[d] / s->box_build[d];
      if (f > shrink) shrink = f;
    }
    rebuild = sqrt(a1) + sqrt(a2) + shrink * (s->rcut + s->c.skin) > s->c.skin;
  }
  if (rebuild) {
    if (disp > 1.0) return ORA_ERR_OUT_OF_BOX;
    s->nlist_updates++;
    if (fixed) {
      int old = s->ncell;
      int rc = compute_mcell(s);
      if (rc) return rc;
      if (s->ncell != old) {
        free(s->head);
        s->head = (int *)malloc(sizeof(int) * s->ncell);
      }
    }
    int rc = ora_build_cell_list(s);
    if (rc) return rc;
    return 1;
  }
  return 0;
}

/* ------------------------------------------------------------------ */
/* integrate1, src/nd.f90:984-1077: with hold groups (Nhold > 0) a held
 * atom's constrained components move by the group's displacement
 * (:1048-1074) */
void ora_integrate1(ora_sys *s) {
  const double li0 = 1.0 / s->box[0], li1 = 1.0 / s->box[1], li2 = 1.0 / s->box[2];
  const double dt = s->c.dt;
  double *pos = s->pos, *vel = s->vel, *acc = s->acc, *dl = s->displist;
  const int np = s->np;
#pragma omp parallel for num_threads(s->nthreads) schedule(static)
  for (int j = 0; j < np; ++j) {
    size_t o = 3 * (size_t)j;
    double du0 = li0 * (vel[o] * dt + 0.5 * acc[o] * dt * dt);
    double du1 = li1 * (vel[o + 1] * dt + 0.5 * acc[o + 1] * dt * dt);
    double du2 = li2 * (vel[o + 2] * dt + 0.5 * acc[o + 2] * dt * dt);
    if (s->nhold > 0) {
      int g = s->hold[j];
      if (g != 0) {
        const int *bd = s->bcdir + 3 * (g - 1);
        const double *bp = s->bcparm + 3 * (g - 1);
        if (bd[0]) du0 = bp[0];
        if (bd[1]) du1 = bp[1];
        if (bd[2]) du2 = bp[2];
      }
    }
    dl[o] = dl[o] + du0; dl[o + 1] = dl[o + 1] + du1; dl[o + 2] = dl[o + 2] + du2;
    pos[o] = pos[o] + du0; pos[o + 1] = pos[o + 1] + du1; pos[o + 2] = pos[o + 2] + du2;
  }
}

/* compute0, src/nd.f90:200-363: static atom split, per-thread force copies
 * (ftmp), Newton-3 scatter, then the hand reduction over thread copies. */
void ora_compute0(ora_sys *s, int cv, int cu) {
  const int T = s->nthreads, np = s->np, npairs = s->npairs;
  const int stride = s->neimax + 1, tsz = s->ptsize + 1;
  double *vtmp = (double *)calloc(6 * (size_t)T, sizeof(double));
  double *ptmp = (double *)calloc((size_t)T, sizeof(double));
  float *vdr2 = (float *)malloc(sizeof(float) * npairs);
  if (cv) for (int k = 0; k < 6; ++k) s->virial[k] = 0.0;
  if (cu) s->potential = 0.0;
  for (int p = 0; p < npairs; ++p) vdr2[p] = (float)(1.0 / s->ptdr2[p]);
  double *force = s->force, *ftmp = s->ftmp;
  const double *pos = s->pos, *box = s->box, *fp = s->fpair, *pp = s->ppair;
  const double *rc2 = s->ptrc2;
  const float ptrmin_unused = 0.0f;
  (void)ptrmin_unused;
  const double ptrmin = s->ptrmin;
  memset(force, 0, sizeof(double) * 3 * (size_t)np);
  memset(ftmp, 0, sizeof(double) * 3 * (size_t)np * T);
#pragma omp parallel num_threads(T)
  {
    int tid = omp_get_thread_num();
    int istart = (np / T) * tid;
    int iend = (np / T) * (tid + 1);
    if (iend < np && tid == T - 1) iend = np;
    double *ft = ftmp + 3 * (size_t)np * tid;
    double pt = 0.0, vt[6] = {0, 0, 0, 0, 0, 0};
    for (int i = istart; i < iend; ++i) {
      const double *pi = pos + 3 * (size_t)i;
      int typi = s->typ[i];
      const int *row = s->vnl + (size_t)stride * i;
      for (int jn = 1; jn < row[0]; ++jn) {
        int j = row[jn];
        int ptij = pm(s, typi, s->typ[j]);
        double rij[3];
        double d2 = pair_d2(pi, pos + 3 * (size_t)j, box, rij);
        if (d2 > rc2[ptij - 1]) continue;
        float rk = (float)(d2 - ptrmin) * vdr2[ptij - 1] + 1.0f;
        int k = (int)rk;
        if (k < 1) k = 1;
        double w = (double)rk - (double)k;
        const double *F = fp + (size_t)tsz * (ptij - 1) + (k - 1);
        double df = w * F[1] + (1.0 - w) * F[0];
        df = df / d2;
        ft[3 * (size_t)i] += rij[0] * df;
        ft[3 * (size_t)i + 1] += rij[1] * df;
        ft[3 * (size_t)i + 2] += rij[2] * df;
        ft[3 * (size_t)j] -= rij[0] * df;
        ft[3 * (size_t)j + 1] -= rij[1] * df;
        ft[3 * (size_t)j + 2] -= rij[2] * df;
        if (cu) {
          const double *P = pp + (size_t)tsz * (ptij - 1) + (k - 1);
          pt = pt + (w * P[1] + (1.0 - w) * P[0]);
        }
        if (cv) {
          vt[0] += rij[0] * rij[0] * df;
          vt[1] += rij[1] * rij[1] * df;
          vt[2] += rij[2] * rij[2] * df;
          vt[3] += rij[0] * rij[1] * df;
          vt[4] += rij[0] * rij[2] * df;
          vt[5] += rij[1] * rij[2] * df;
        }
      }
    }
    ptmp[tid] = pt;
    for (int k = 0; k < 6; ++k) vtmp[6 * tid + k] = vt[k];
#pragma omp barrier
    for (int t = 0; t < T; ++t) {
      const double *src = ftmp + 3 * (size_t)np * t;
      for (int i = istart; i < iend; ++i) {
        force[3 * (size_t)i] += src[3 * (size_t)i];
        force[3 * (size_t)i + 1] += src[3 * (size_t)i + 1];
        force[3 * (size_t)i + 2] += src[3 * (size_t)i + 2];
      }
    }
  }
  if (cv)
    for (int t = 0; t < T; ++t)
      for (int k = 0; k < 6; ++k) s->virial[k] += vtmp[6 * t + k];
  if (cu)
    for (int t = 0; t < T; ++t) s->potential += ptmp[t];
  free(vtmp); free(ptmp); free(vdr2);
}

/* compute1, src/nd.f90:364-530: the half-list loop of compute0 for a
 * PairMat with one-sided entries.  The table and cutoff are those of
 * max(PTij, PTji) (:447,462-472); i feels the pair only if PTji > 0
 * (:474-478), j only if PTij > 0 (:479-483); energy and virial count only
 * pairs with PTij == PTji (:485-498).  The reference leaves k unclamped here
 * (:467); a list entry closer than sqrt(PTrMin) would read outside the
 * table, and this restatement clamps k to 1 as compute0 does. */
void ora_compute1(ora_sys *s, int cv, int cu) {
  const int T = s->nthreads, np = s->np, npairs = s->npairs;
  const int stride = s->neimax + 1, tsz = s->ptsize + 1;
  double *vtmp = (double *)calloc(6 * (size_t)T, sizeof(double));
  double *ptmp = (double *)calloc((size_t)T, sizeof(double));
  float *vdr2 = (float *)malloc(sizeof(float) * npairs);
  if (cv) for (int k = 0; k < 6; ++k) s->virial[k] = 0.0;
  if (cu) s->potential = 0.0;
  for (int p = 0; p < npairs; ++p) vdr2[p] = (float)(1.0 / s->ptdr2[p]);
  double *force = s->force, *ftmp = s->ftmp;
  const double *pos = s->pos, *box = s->box, *fp = s->fpair, *pp = s->ppair;
  const double *rc2 = s->ptrc2;
  const double ptrmin = s->ptrmin;
  memset(force, 0, sizeof(double) * 3 * (size_t)np);
  memset(ftmp, 0, sizeof(double) * 3 * (size_t)np * T);
#pragma omp parallel num_threads(T)
  {
    int tid = omp_get_thread_num();
    int istart = (np / T) * tid;
    int iend = (np / T) * (tid + 1);
    if (iend < np && tid == T - 1) iend = np;
    double *ft = ftmp + 3 * (size_t)np * tid;
    double pt = 0.0, vt[6] = {0, 0, 0, 0, 0, 0};
    for (int i = istart; i < iend; ++i) {
      const double *pi = pos + 3 * (size_t)i;
      int typi = s->typ[i];
      const int *row = s->vnl + (size_t)stride * i;
      for (int jn = 1; jn < row[0]; ++jn) {
        int j = row[jn];
        int ptij = pm(s, typi, s->typ[j]), ptji = pm(s, s->typ[j], typi);
        int mx = ptij > ptji ? ptij : ptji;
        double rij[3];
        double d2 = pair_d2(pi, pos + 3 * (size_t)j, box, rij);
        if (d2 > rc2[mx - 1]) continue;
        float rk = (float)(d2 - ptrmin) * vdr2[mx - 1] + 1.0f;
        int k = (int)rk;
        if (k < 1) k = 1;
        double w = (double)rk - (double)k;
        const double *F = fp + (size_t)tsz * (mx - 1) + (k - 1);
        double df = w * F[1] + (1.0 - w) * F[0];
        df = df / d2;
        if (ptji > 0) {
          ft[3 * (size_t)i] += rij[0] * df;
          ft[3 * (size_t)i + 1] += rij[1] * df;
          ft[3 * (size_t)i + 2] += rij[2] * df;
        }
        if (ptij > 0) {
          ft[3 * (size_t)j] -= rij[0] * df;
          ft[3 * (size_t)j + 1] -= rij[1] * df;
          ft[3 * (size_t)j + 2] -= rij[2] * df;
        }
        if (cu && ptij == ptji) {
          const double *P = pp + (size_t)tsz * (mx - 1) + (k - 1);
          pt = pt + (w * P[1] + (1.0 - w) * P[0]);
        }
        if (cv && ptij == ptji) {
          vt[0] += rij[0] * rij[0] * df;
          vt[1] += rij[1] * rij[1] * df;
          vt[2] += rij[2] * rij[2] * df;
          vt[3] += rij[0] * rij[1] * df;
          vt[4] += rij[0] * rij[2] * df;
          vt[5] += rij[1] * rij[2] * df;
        }
      }
    }
    ptmp[tid] = pt;
    for (int k = 0; k < 6; ++k) vtmp[6 * tid + k] = vt[k];
#pragma omp barrier
    for (int t = 0; t < T; ++t) {
      const double *src = ftmp + 3 * (size_t)np * t;
      for (int i = istart; i < iend; ++i) {
        force[3 * (size_t)i] += src[3 * (size_t)i];
        force[3 * (size_t)i + 1] += src[3 * (size_t)i + 1];
        force[3 * (size_t)i + 2] += src[3 * (size_t)i + 2];
      }
    }
  }
  if (cv)
    for (int t = 0; t < T; ++t)
      for (int k = 0; k < 6; ++k) s->virial[k] += vtmp[6 * t + k];
  if (cu)
    for (int t = 0; t < T; ++t) s->potential += ptmp[t];
  free(vtmp); free(ptmp); free(vdr2);
}

/* compute2 (src/nd.f90:531-727) and compute3 (:728-933): compute0 and
 * compute1 with 'spring' pairs, which act through their strain against the
 * initial configuration (:627-660, :826-859): s = r/r0 - 1, no force while
 * s > PairParams(3); df = -PairParams(2)*s*Vol^2/r with Vol = PairParams(4),
 * energy PairParams(2)*s*Vol^2*s*r0/2; no cutoff test.  compute2 counts
 * every pair's energy and virial and pushes both atoms; compute3 applies
 * compute1's one-sided rules.  Table pairs as in compute0/compute1 (compute2
 * leaves k unclamped, :666; clamped to 1 here as compute0 does). */
static void compute_springs(ora_sys *s, int cv, int cu, int asym) {
  const int T = s->nthreads, np = s->np, npairs = s->npairs;
  const int stride = s->neimax + 1, tsz = s->ptsize + 1;
  double *vtmp = (double *)calloc(6 * (size_t)T, sizeof(double));
  double *ptmp = (double *)calloc((size_t)T, sizeof(double));
  float *vdr2 = (float *)malloc(sizeof(float) * npairs);
  if (cv) for (int k = 0; k < 6; ++k) s->virial[k] = 0.0;
  if (cu) s->potential = 0.0;
  for (int p = 0; p < npairs; ++p) vdr2[p] = (float)(1.0 / s->ptdr2[p]);
  double *force = s->force, *ftmp = s->ftmp;
  const double *pos = s->pos, *box = s->box, *fp = s->fpair, *pp = s->ppair;
  const double *rc2 = s->ptrc2, *ib = s->initbox, *ip = s->ipos;
  const double ptrmin = s->ptrmin;
  memset(force, 0, sizeof(double) * 3 * (size_t)np);
  memset(ftmp, 0, sizeof(double) * 3 * (size_t)np * T);
#pragma omp parallel num_threads(T)
  {
    int tid = omp_get_thread_num();
    int istart = (np / T) * tid;
    int iend = (np / T) * (tid + 1);
    if (iend < np && tid == T - 1) iend = np;
    double *ft = ftmp + 3 * (size_t)np * tid;
    double pt = 0.0, vt[6] = {0, 0, 0, 0, 0, 0};
    for (int i = istart; i < iend; ++i) {
      const double *pi = pos + 3 * (size_t)i;
      int typi = s->typ[i];
      const int *row = s->vnl + (size_t)stride * i;
      for (int jn = 1; jn < row[0]; ++jn) {
        int j = row[jn];
        int ptij = pm(s, typi, s->typ[j]), ptji = pm(s, s->typ[j], typi);
        int p = asym ? (ptij > ptji ? ptij : ptji) : ptij;
        int count = asym ? ptij == ptji : 1;
        double rij[3];
        double d2 = pair_d2(pi, pos + 3 * (size_t)j, box, rij);
        double df, dp = 0.0;
        if (pot_kind(s->pairname[p - 1]) == P_SPRING) {
          double sr[3], rij0[3];
          for (int d = 0; d < 3; ++d) {
            sr[d] = ip[3 * (size_t)i + d] - ip[3 * (size_t)j + d];
            sr[d] = sr[d] - round(sr[d]);
            rij0[d] = ib[d] * sr[d];
          }
          double d20 = rij0[0] * rij0[0];
          d20 = d20 + rij0[1] * rij0[1];
          d20 = d20 + rij0[2] * rij0[2];
          double r = sqrt(d2), r0 = sqrt(d20);
          double sij = r / r0 - 1.0;
          const double *prm = s->pairparams + 4 * (size_t)(p - 1);
          if (sij > prm[2]) continue;
          double vi = prm[3];
          df = prm[1] * sij * vi * vi;
          if (cu) dp = 0.5 * df * sij * r0;
          df = -df / r;
        } else {
          if (d2 > rc2[p - 1]) continue;
          float rk = (float)(d2 - ptrmin) * vdr2[p - 1] + 1.0f;
          int k = (int)rk;
          if (k < 1) k = 1;
          double w = (double)rk - (double)k;
          const double *F = fp + (size_t)tsz * (p - 1) + (k - 1);
          df = w * F[1] + (1.0 - w) * F[0];
          if (cu) {
            const double *P = pp + (size_t)tsz * (p - 1) + (k - 1);
            dp = w * P[1] + (1.0 - w) * P[0];
          }
          df = df / d2;
        }
        if (cu && count) pt = pt + dp;
        if (!asym || ptji > 0) {
          ft[3 * (size_t)i] += rij[0] * df;
          ft[3 * (size_t)i + 1] += rij[1] * df;
          ft[3 * (size_t)i + 2] += rij[2] * df;
        }
        if (!asym || ptij > 0) {
          ft[3 * (size_t)j] -= rij[0] * df;
          ft[3 * (size_t)j + 1] -= rij[1] * df;
          ft[3 * (size_t)j + 2] -= rij[2] * df;
        }
        if (cv && count) {
          vt[0] += rij[0] * rij[0] * df;
          vt[1] += rij[1] * rij[1] * df;
          vt[2] += rij[2] * rij[2] * df;
          vt[3] += rij[0] * rij[1] * df;
          vt[4] += rij[0] * rij[2] * df;
          vt[5] += rij[1] * rij[2] * df;
        }
      }
    }
    ptmp[tid] = pt;
    for (int k = 0; k < 6; ++k) vtmp[6 * tid + k] = vt[k];
#pragma omp barrier
    for (int t = 0; t < T; ++t) {
      const double *src = ftmp + 3 * (size_t)np * t;
      for (int i = istart; i < iend; ++i) {
        force[3 * (size_t)i] += src[3 * (size_t)i];
        force[3 * (size_t)i + 1] += src[3 * (size_t)i + 1];
        force[3 * (size_t)i + 2] += src[3 * (size_t)i + 2];
      }
    }
  }
  if (cv)
    for (int t = 0; t < T; ++t)
      for (int k = 0; k < 6; ++k) s->virial[k] += vtmp[6 * t + k];
  if (cu)
    for (int t = 0; t < T; ++t) s->potential += ptmp[t];
  free(vtmp); free(ptmp); free(vdr2);
}

void ora_compute2(ora_sys *s, int cv, int cu) { compute_springs(s, cv, cu, 0); }
void ora_compute3(ora_sys *s, int cv, int cu) { compute_springs(s, cv, cu, 1); }

/* the force routine dynamics calls, src/nd.f90:155-163 */
void ora_compute(ora_sys *s, int cv, int cu) {
  if (s->springpots) {
    if (!s->ipos) ora_init_positions(s, NULL, NULL);
    if (s->asympots) ora_compute3(s, cv, cu);
    else ora_compute2(s, cv, cu);
  } else if (s->asympots) {
    ora_compute1(s, cv, cu);
  } else {
    ora_compute0(s, cv, cu);
  }
}

/* integrate2, src/nd.f90:1081-1121 */
void ora_integrate2(ora_sys *s, int ck) {
  const int np = s->np, T = s->nthreads;
  const double dt = s->c.dt;
  double *vel = s->vel, *acc = s->acc;
  const double *force = s->force, *mass = s->mass;
  const int *typ = s->typ;
  double *kpart = (double *)calloc(T, sizeof(double));
#pragma omp parallel num_threads(T)
  {
    int tid = omp_get_thread_num();
    double kin = 0.0;
#pragma omp for schedule(static)
    for (int j = 0; j < np; ++j) {
      size_t o = 3 * (size_t)j;
      double rmass = 1.0 / mass[typ[j] - 1];
      vel[o] = vel[o] + 0.5 * dt * (force[o] * rmass + acc[o]);
      vel[o + 1] = vel[o + 1] + 0.5 * dt * (force[o + 1] * rmass + acc[o + 1]);
      vel[o + 2] = vel[o + 2] + 0.5 * dt * (force[o + 2] * rmass + acc[o + 2]);
      acc[o] = force[o] * rmass;
      acc[o + 1] = force[o + 1] * rmass;
      acc[o + 2] = force[o + 2] * rmass;
      if (ck) {
        double kt = vel[o] * vel[o];
        kt = kt + vel[o + 1] * vel[o + 1];
        kt = kt + vel[o + 2] * vel[o + 2];
        kt = kt * mass[typ[j] - 1];
        kin = kin + kt;
      }
    }
    kpart[tid] = kin;
  }
  double kinetic = 0.0;
  for (int t = 0; t < T; ++t) kinetic += kpart[t];
  if (ck) kinetic = kinetic * 0.5;
  s->kinetic = kinetic;
  free(kpart);
}

static void scale_vel(ora_sys *s, double lam) {
  const size_t n = 3 * (size_t)s->np;
  double *vel = s->vel;
#pragma omp parallel for num_threads(s->nthreads) schedule(static)
  for (size_t j = 0; j < n; ++j) vel[j] = vel[j] * lam;
}

/* mkIsoKE, src/nd.f90:1122-1158 */
void ora_mk_iso_ke(ora_sys *s) {
  double lam = 1.0 + s->c.dt / s->c.ke_parm * (s->c.ke_target * (double)s->np / s->kinetic - 1.0);
  lam = sqrt(lam);
  scale_vel(s, lam);
}

/* mkIsoE, src/nd.f90:1159-1182 */
void ora_mk_iso_e(ora_sys *s) {
  double lam = 1.0 - s->c.dt / s->c.e_parm * (s->e0 / (s->potential + s->kinetic) - 1.0);
  scale_vel(s, lam);
}

/* mkIsoP, src/nd.f90:1183-1213 (box rows updated in place, in order) */
void ora_mk_iso_p(ora_sys *s) {
  double *box = s->box, lam[6], press[6];
  double vol = box[0] * box[1] * box[2];
  for (int k = 0; k < 6; ++k) press[k] = s->virial[k] / vol;
  double f = s->c.dt / s->c.p_parm;
  lam[0] = 1.0 - f * (s->c.p_target[0] - press[0]);
  lam[1] = 1.0 - f * (s->c.p_target[1] - press[1]);
  lam[2] = 1.0 - f * (s->c.p_target[2] - press[2]);
  lam[3] = f * press[3];
  lam[4] = f * press[4];
  lam[5] = f * press[5];
  box[0] = box[0] * lam[0] + box[1] * lam[5] + box[2] * lam[4];
  box[1] = box[0] * lam[5] + box[1] * lam[1] + box[2] * lam[3];
  box[2] = box[0] * lam[4] + box[1] * lam[3] + box[2] * lam[2];
}

/* dynamics: prologue (lists) then the main loop */
int ora_run(ora_sys *s, int nsteps, double dt, ora_thermo_cb cb, void *user) {
  s->c.dt = dt;
  int rc = ora_setup_lists(s);
  if (rc) return rc;
  return ora_run_loop(s, nsteps, dt, cb, user);
}

/* dynamics main loop only, src/nd.f90:137-180 (the part the reference's
 * 'Elapsed time for main dynamics' measures, :129,186) */
int ora_run_loop(ora_sys *s, int nsteps, double dt, ora_thermo_cb cb, void *user) {
  int rc;
  s->c.dt = dt;
  if (!s->lists_ready) return ORA_ERR_ARG;
  ora_control *c = &s->c;
  for (int tt = 1; tt <= nsteps; ++tt) {
    c->step = c->step + 1;
    int step = c->step;
    int cv = 0, cu = 0, ck = 0;
    int out = (step % c->out_steps == 0) || tt == 1;
    if (out) cv = cu = ck = 1;
    if (c->isokinetic && step % c->ke_freq == 0) ck = 1;
    if (c->isobaric && step % c->p_freq == 0) cv = 1;
    if (c->isoenergetic && step % c->e_freq == 0) cu = ck = 1;
    if (c->renei && step % c->renei_freq == 0) {
      rc = ora_check_list_update(s);
      if (rc < 0) return rc;
    }
    ora_integrate1(s);
    ora_compute(s, cv, cu);
    ora_integrate2(s, ck);
    if (tt == 1) s->e0 = s->potential + s->kinetic;
    if (out && cb) {
      ora_thermo t;
      t.step = step;
      t.potential = s->potential;
      t.kinetic = s->kinetic;
      t.energy_error = (s->potential + s->kinetic - s->e0) / s->e0;
      t.pressure = (s->virial[0] + s->virial[1] + s->virial[2]) /
                   (s->box[0] * s->box[1] * s->box[2] * 3.0);
      t.volume = s->box[0] * s->box[1] * s->box[2];
      memcpy(t.virial, s->virial, sizeof(t.virial));
      memcpy(t.box, s->box, sizeof(t.box));
      cb(&t, user);
    }
    if (c->isokinetic && step % c->ke_freq == 0) ora_mk_iso_ke(s);
    if (c->isobaric && step % c->p_freq == 0) ora_mk_iso_p(s);
    if (c->isoenergetic && step % c->e_freq == 0) ora_mk_iso_e(s);
    if (c->box_load)
      for (int d = 0; d < 3; ++d) s->box[d] = s->box[d] + c->box_vel[d] * dt;
  }
  return ORA_OK;
}

/* ------------------------------------------------------------------ */
int ora_get_mcell(const ora_sys *s, int *m) { memcpy(m, s->mcell, sizeof(int) * 3); return ORA_OK; }

int ora_get_cells(const ora_sys *s, int *cell) {
  if (!s->lists_ready) return ORA_ERR_ARG;
  for (int c = 0; c < s->ncell; ++c)
    for (int i = s->head[c]; i >= 0; i = s->list[i]) cell[i] = c;
  return ORA_OK;
}

long ora_get_neighbors(const ora_sys *s, int *pairs, long cap) {
  if (!s->lists_ready) return -1;
  long n = 0;
  const int stride = s->neimax + 1;
  for (int i = 0; i < s->np; ++i) {
    const int *row = s->vnl + (size_t)stride * i;
    for (int jn = 1; jn < row[0]; ++jn) {
      int j = row[jn];
      if (pairs && n < cap) {
        pairs[2 * n] = i < j ? i : j;
        pairs[2 * n + 1] = i < j ? j : i;
      }
      ++n;
    }
  }
  return n;
}
int ora_get_list_updates(const ora_sys *s) { return s->nlist_updates; }
int ora_get_neimax(const ora_sys *s) { return s->neimax; }
double ora_get_skin(const ora_sys *s) { return s->c.skin; }

/* ------------------------------------------------------------------ */
/* normalVelocityDistribution, src/nd.f90:1500-1624: Kinderman-Monahan
 * ratio of uniforms in single precision; uniforms from SplitMix64. */
static uint64_t splitmix64(uint64_t *x) {
  uint64_t z = (*x += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static float uni(uint64_t *st) {
  return ((float)(splitmix64(st) >> 40) + 0.5f) * (1.0f / 16777216.0f);
}
static float normal_km(uint64_t *st) {
  const float s = 0.449871f, t = -0.386595f, a = 0.19600f, b = 0.25472f;
  const float r1 = 0.27597f, r2 = 0.27846f, half = 0.5f;
  float u, v, x, y, q;
  for (;;) {
    u = uni(st);
    v = uni(st);
    v = 1.7156f * (v - half);
    x = u - s;
    y = fabsf(v) - t;
    q = x * x + y * (a * y - b * x);
    if (q < r1) break;
    if (q > r2) continue;
    if (v * v < -4.0f * logf(u) * u * u) break;
  }
  return v / u;
}

void ora_velocity(ora_sys *s, float kt, unsigned long long seed) {
  uint64_t st = seed;
  double vt[3] = {0, 0, 0};
  for (int i = 0; i < s->np; ++i) {
    float nn[3];
    nn[0] = normal_km(&st);
    nn[1] = normal_km(&st);
    nn[2] = normal_km(&st);
    float coeff = sqrtf(2.0f * kt / (3.0f * (float)s->mass[s->typ[i] - 1]));
    for (int d = 0; d < 3; ++d) {
      s->vel[3 * (size_t)i + d] = (double)(nn[d] * coeff);
      vt[d] += s->vel[3 * (size_t)i + d];
    }
  }
  for (int d = 0; d < 3; ++d) vt[d] = vt[d] / (double)s->np;
  for (int i = 0; i < s->np; ++i)
    for (int d = 0; d < 3; ++d) s->vel[3 * (size_t)i + d] -= vt[d];
}

/* ------------------------------------------------------------------ */
/* Fortran G14.6 (used by write_thermo, src/read_input.f90:440) */
void ora_fmt_g14_6(double x, char *out) {
  char buf[64];
  if (x == 0.0) {
    snprintf(buf, sizeof buf, "%10.5f    ", x);
    if (signbit(x)) snprintf(buf, sizeof buf, "%10s    ", "-0.00000");
    memcpy(out, buf, 15);
    out[14] = 0;
    return;
  }
  if (!isfinite(x)) {
    snprintf(out, 15, "%14s", isnan(x) ? "NaN" : (x > 0 ? "Infinity" : "-Infinity"));
    return;
  }
  /* round to 6 significant digits and find the decimal exponent */
  snprintf(buf, sizeof buf, "%.5e", x);
  char *e = strchr(buf, 'e');
  int ex = atoi(e + 1) + 1; /* value = 0.dddddd x 10^ex */
  if (ex >= 0 && ex <= 6) {
    int dec = 6 - ex;
    if (dec > 0)
      snprintf(buf, sizeof buf, "%10.*f    ", dec, x);
    else
      snprintf(buf, sizeof buf, "%9.0f.    ", x); /* F10.0 keeps the point */
  } else {
    double m = fabs(x) / pow(10.0, ex);
    /* mantissa digits from the %e rendering to avoid double rounding */
    char dig[8];
    char tmp[64];
    snprintf(tmp, sizeof tmp, "%.5e", fabs(x));
    dig[0] = tmp[0];
    memcpy(dig + 1, tmp + 2, 5);
    dig[6] = 0;
    (void)m;
    if (ex >= -99 && ex <= 99)
      snprintf(buf, sizeof buf, "%s0.%sE%c%02d", x < 0 ? "-" : "", dig,
               ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    else
      snprintf(buf, sizeof buf, "%s0.%s%c%03d", x < 0 ? "-" : "", dig,
               ex < 0 ? '-' : '+', ex < 0 ? -ex : ex);
    char pad[64];
    snprintf(pad, sizeof pad, "%14s", buf);
    memcpy(buf, pad, 15);
  }
  memcpy(out, buf, 15);
  out[14] = 0;
}

void ora_fmt_thermo(const ora_thermo *t, char *out) {
  char a[15], b[15], c[15], d[15], e[15];
  ora_fmt_g14_6(t->potential, a);
  ora_fmt_g14_6(t->kinetic, b);
  ora_fmt_g14_6(t->energy_error, c);
  ora_fmt_g14_6(t->pressure, d);
  ora_fmt_g14_6(t->volume, e);
  snprintf(out, 96, " %8d %s %s %s %s %s", t->step, a, b, c, d, e);
}
