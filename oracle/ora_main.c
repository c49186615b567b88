/*
 * ora_main.c -- directive-script driver for the CPU oracle (TEST
 * INFRASTRUCTURE).  Reads an Ndyn directive script on stdin and runs it
 * through the oracle, printing write_thermo lines in the reference format.
 *
 * Restates the directive loop of src/read_input.f90:2-219 for the
 * directives on the timestep path; group/hold/spring/random-position
 * directives are reported as unsupported.  'Exec' is never executed.
 * Model readers restate read_model, src/read_input.f90:277-392.
 */
#include <ctype.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "ndyn_oracle.h"

#define MAXW 32
static int split(char *line, char *w[MAXW]) {
  int n = 0;
  char *p = line;
  while (*p && n < MAXW) {
    while (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n') ++p;
    if (!*p) break;
    w[n++] = p;
    while (*p && *p != ' ' && *p != '\t' && *p != '\r' && *p != '\n') ++p;
    if (*p) *p++ = 0;
  }
  return n;
}

static void strip_comment(char *line) {
  char *h = strchr(line, '#');
  if (h) *h = 0;
}

static int parse_logical(const char *v) {
  /* Fortran list-directed logical: optional '.', then T/t or F/f */
  if (*v == '.') ++v;
  return (*v == 'T' || *v == 't');
}

typedef struct {
  ora_sys *s;
  int ntypes;
  char tname[64][9];
  double mass[64], charge[64];
  int have_pairs;
  char model[256], model_type[16];
  unsigned long long seed;
  ora_control c;
  int threads;
} drv;

static int type_id(drv *d, const char *t) {
  for (int i = 0; i < d->ntypes; ++i)
    if (strcmp(t, d->tname[i]) == 0) return i + 1;
  return 0;
}

static void thermo_cb(const ora_thermo *t, void *user) {
  (void)user;
  char line[96];
  ora_fmt_thermo(t, line);
  printf("%s\n", line);
  fflush(stdout);
}

/* read_model for the 'dump' and 'xyz' formats */
static int read_model(drv *d, const double *boxset) {
  FILE *f = fopen(d->model, "r");
  if (!f) {
    fprintf(stderr, "read_model: ERROR: opening model file: %s\n", d->model);
    return -1;
  }
  char line[1024];
  int np = 0;
  double box[3] = {boxset[0], boxset[1], boxset[2]};
  int dump = strcmp(d->model_type, "dump") == 0 || strcmp(d->model_type, "trj") == 0;
  if (dump) {
    for (int k = 0; k < 3; ++k) fgets(line, sizeof line, f);
    fgets(line, sizeof line, f);
    np = atoi(line);
    fgets(line, sizeof line, f);
    for (int k = 0; k < 3; ++k) {
      float lm, lx;
      fgets(line, sizeof line, f);
      sscanf(line, "%f %f", &lm, &lx);
      box[k] = (double)(lx - lm); /* real(4) read, src/read_input.f90:334-336 */
    }
    fgets(line, sizeof line, f);
  } else {
    fgets(line, sizeof line, f);
    np = atoi(line);
    fgets(line, sizeof line, f);
  }
  int *typ = (int *)calloc(np, sizeof(int));
  double *pos = (double *)calloc(3 * (size_t)np, sizeof(double));
  for (int i = 0; i < np; ++i) {
    if (!fgets(line, sizeof line, f)) { fclose(f); return -1; }
    if (dump) {
      int id, ty;
      float x[3];
      sscanf(line, "%d %d %f %f %f", &id, &ty, &x[0], &x[1], &x[2]);
      typ[id - 1] = ty;
      for (int k = 0; k < 3; ++k) pos[3 * (size_t)(id - 1) + k] = (double)(x[k] - 0.5f);
    } else {
      char ct[64];
      double x[3];
      sscanf(line, "%63s %lf %lf %lf", ct, &x[0], &x[1], &x[2]);
      typ[i] = type_id(d, ct);
      if (!typ[i]) {
        fprintf(stderr, "ERROR: no atom type defined for atom %d\n", i + 1);
        fclose(f);
        return -1;
      }
      for (int k = 0; k < 3; ++k) pos[3 * (size_t)i + k] = x[k] / box[k];
    }
  }
  fclose(f);
  int rc = ora_set_state(d->s, np, typ, pos, NULL, NULL, box);
  free(typ);
  free(pos);
  printf("#  read_model: successfully read %8d model nodes.\n", np);
  return rc;
}

int main(int argc, char **argv) {
  drv d;
  memset(&d, 0, sizeof d);
  d.s = ora_new();
  d.seed = 123456789ULL;
  strcpy(d.model_type, "xyz");
  ora_default_control(&d.c);
  double boxset[3] = {10.0, 10.0, 10.0};
  int mode = ORA_MODE_REF;
  for (int a = 1; a < argc; ++a) {
    if (!strcmp(argv[a], "--fixed")) mode = ORA_MODE_FIXED;
    if (!strcmp(argv[a], "--threads") && a + 1 < argc) ora_set_threads(d.s, atoi(argv[++a]));
  }
  ora_set_mode(d.s, mode);
  char line[1024], raw[1024];
  int started = 0, ln = 0;
  while (fgets(raw, sizeof raw, stdin)) {
    char *w[MAXW];
    strcpy(line, raw);
    int wc0 = split(line, w);
    if (wc0 && !strcmp(w[0], "START")) { started = 1; break; }
  }
  if (!started) return 1;
  while (fgets(raw, sizeof raw, stdin)) {
    ++ln;
    strcpy(line, raw);
    strip_comment(line);
    char *w[MAXW];
    int wc = split(line, w);
    if (wc < 1) continue;
    const char *k = w[0];
#define ARG(n) (wc > (n) ? w[n] : "0")
    if (!strcmp(k, "help") || !strcmp(k, "WritePotentialTable")) {
    } else if (!strcmp(k, "BoxSize")) {
      for (int q = 0; q < 3; ++q) boxset[q] = atof(ARG(q + 1));
    } else if (!strcmp(k, "Model")) {
      snprintf(d.model, sizeof d.model, "%s", ARG(1));
      if (wc >= 3) snprintf(d.model_type, sizeof d.model_type, "%s", w[2]);
      if (read_model(&d, boxset)) return 2;
    } else if (!strcmp(k, "Seed")) {
      d.seed = strtoull(ARG(1), NULL, 10);
    } else if (!strcmp(k, "Velocity")) {
      ora_set_control(d.s, &d.c);
      ora_velocity(d.s, (float)atof(ARG(1)), d.seed);
    } else if (!strcmp(k, "ReNeibour") || !strcmp(k, "ReNeighbor")) {
      d.c.renei = parse_logical(ARG(1));
      if (wc >= 3) d.c.renei_freq = atoi(w[2]);
    } else if (!strcmp(k, "Skin")) {
      d.c.skin = atof(ARG(1));
    } else if (!strcmp(k, "NeiMax")) {
      d.c.neimax = atoi(ARG(1));
    } else if (!strcmp(k, "Types")) {
      d.ntypes = atoi(ARG(1));
      for (int i = 0; i < d.ntypes; ++i) {
        if (!fgets(raw, sizeof raw, stdin)) return 3;
        strcpy(line, raw);
        char *tw[MAXW];
        int n = split(line, tw);
        snprintf(d.tname[i], 9, "%s", n > 0 ? tw[0] : "");
        d.mass[i] = n > 1 ? atof(tw[1]) : 0.0;
        d.charge[i] = n > 2 ? atof(tw[2]) : 0.0;
      }
      ora_set_types(d.s, d.ntypes, d.mass);
    } else if (!strcmp(k, "Pairs")) {
      int np = atoi(ARG(1));
      double ptrmin = wc >= 3 ? atof(w[2]) : 0.25;
      int ptsize = wc >= 4 ? atoi(w[3]) : 1000;
      int *p1 = calloc(np, sizeof(int)), *p2 = calloc(np, sizeof(int));
      int *sym = calloc(np, sizeof(int)), *npar = calloc(np, sizeof(int));
      char *names = calloc(np, 8);
      double *par = calloc(4 * (size_t)np, sizeof(double)), *q = calloc(np, sizeof(double));
      for (int i = 0; i < np; ++i) {
        if (!fgets(raw, sizeof raw, stdin)) return 3;
        strcpy(line, raw);
        strip_comment(line);
        char *tw[MAXW];
        int n = split(line, tw);
        p1[i] = type_id(&d, n > 0 ? tw[0] : "");
        p2[i] = type_id(&d, n > 1 ? tw[1] : "");
        sym[i] = n > 2 && !strcmp(tw[2], "sym");
        if (n > 3) strncpy(names + 8 * i, tw[3], 8);
        npar[i] = n - 4 > 4 ? 4 : (n - 4 > 0 ? n - 4 : 0);
        for (int j = 0; j < npar[i]; ++j) par[4 * i + j] = atof(tw[4 + j]);
        if (p1[i] && p2[i]) q[i] = d.charge[p1[i] - 1] * d.charge[p2[i] - 1];
      }
      int rc = ora_set_pairs(d.s, np, ptrmin, ptsize, p1, p2, sym, names, par, npar, q);
      if (rc) { fprintf(stderr, "Pairs: error %d\n", rc); return 4; }
      printf("# Global maximum cutoff radius: %g\n", ora_get_rcut(d.s));
      free(p1); free(p2); free(sym); free(npar); free(names); free(par); free(q);
    } else if (!strcmp(k, "Isokinetic")) {
      d.c.isokinetic = 1;
      d.c.ke_target = atof(ARG(1));
      d.c.ke_parm = atof(ARG(2));
      if (wc >= 4) d.c.ke_freq = atoi(w[3]);
    } else if (!strcmp(k, "Anisokinetic")) {
      d.c.isokinetic = 0;
    } else if (!strcmp(k, "Isoenergetic")) {
      d.c.isoenergetic = 1;
      d.c.e_parm = atof(ARG(1));
      if (wc >= 3) d.c.e_freq = atoi(w[2]);
    } else if (!strcmp(k, "Anisoenergetic")) {
      d.c.isoenergetic = 0;
    } else if (!strcmp(k, "Isobaric")) {
      d.c.isobaric = 1;
      for (int q = 0; q < 3; ++q) d.c.p_target[q] = atof(ARG(q + 1));
      d.c.p_parm = atof(ARG(4));
      if (wc >= 6) d.c.p_freq = atoi(w[5]);
    } else if (!strcmp(k, "Anisobaric")) {
      d.c.isobaric = 0;
    } else if (!strcmp(k, "BoxVel")) {
      d.c.box_load = 1;
      for (int q = 0; q < 3; ++q) d.c.box_vel[q] = atof(ARG(q + 1));
    } else if (!strcmp(k, "StopBoxVel")) {
      d.c.box_load = 0;
    } else if (!strcmp(k, "Exec")) {
      printf("# Exec not executed by the oracle\n");
    } else if (!strcmp(k, "Print")) {
      printf("# %s", raw + 6);
    } else if (!strcmp(k, "OutFreq")) {
      d.c.out_steps = atoi(ARG(1));
    } else if (!strcmp(k, "StepNumber")) {
      d.c.step = atoi(ARG(1));
    } else if (!strcmp(k, "ConfOutFreq")) {
      /* configuration output is not part of the timestep path */
    } else if (!strcmp(k, "Run")) {
      int nsteps = atoi(ARG(1));
      if (wc >= 3) d.c.dt = atof(w[2]);
      ora_set_control(d.s, &d.c);
      printf("#  Step   Potential     Kinetic        EnergyError    pressure       volume\n");
      int rc = ora_run(d.s, nsteps, d.c.dt, thermo_cb, NULL);
      ora_get_control(d.s, &d.c);
      if (rc) {
        fprintf(stderr, "dynamics: error %d\n", rc);
        return 5;
      }
      printf("# Number of neighbour list updates:%8d\n", ora_get_list_updates(d.s));
      fflush(stdout);
    } else if (!strcmp(k, "END") || !strcmp(k, "DONE") || !strcmp(k, "end") ||
               !strcmp(k, "done")) {
      break;
    } else if (!strcmp(k, "EXIT") || !strcmp(k, "exit") || !strcmp(k, "quit") ||
               !strcmp(k, "abort")) {
      return 0;
    } else {
      fprintf(stderr, "#  read_input: unsupported directive: %s line:%4d\n", k, ln);
    }
  }
  ora_free(d.s);
  return 0;
}
