/*
 * ndyn_oracle.h -- CPU oracle for the Ndyn MD timestep path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C (C11 + OpenMP) restatement of
 * the reference Fortran FP64 path (stewmasterj/Ndyn_OMP, src/).  It is used
 *   - by tests/ as the parity checker for the CUDA library,
 *   - by bench.py as the timed CPU baseline ("port" of the reference's
 *     OpenMP path: static atom split, per-thread force copies, hand reduction).
 * The product (libndyn_gpu.so, the ndyn_gpu driver) never links or calls it.
 *
 * Parity pinning: the restatement is checked against the reference's own
 * committed run logs (examples/MorseTest/out:38, examples/testT/out:38-57,
 * examples/SineTest/out:38, examples/testCAF/OMP_4/out_omp1:38) by
 * tests/test_oracle_golden.py.  The reference itself cannot be compiled in
 * this image (no Fortran compiler), so those logs are the pin.
 *
 * Conventions: atoms are 0-based here (Fortran is 1-based); arrays keep the
 * Fortran column-major layouts, e.g. pos[3*i+c] == pos(c+1,i+1).  Pair ids
 * (PairMat values) stay 1-based with 0 meaning "no potential", as in
 * src/mods.f90:55.
 */
#ifndef NDYN_ORACLE_H
#define NDYN_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* quirk mode: ORA_MODE_REF reproduces the reference exactly (list rebuild
 * criterion mixing fractional and Angstrom units, duplicated pairs when a
 * cell count is < 3); ORA_MODE_FIXED compares Angstrom displacements and
 * visits each distinct neighbour cell once. */
enum { ORA_MODE_REF = 0, ORA_MODE_FIXED = 1 };

enum {
  ORA_OK = 0,
  ORA_ERR_ARG = -1,
  ORA_ERR_NEIMAX = -2,     /* 'too many neighbours in list' src/nd.f90:1378 */
  ORA_ERR_OUT_OF_BOX = -3, /* 'Particle outside of box' src/nd.f90:1494 */
  ORA_ERR_POTENTIAL = -4,  /* unknown potential name src/potentials.f90:148 */
  ORA_ERR_CELLS = -5,      /* fewer than 2 link cells in a direction */
  ORA_ERR_NOMEM = -6
};

typedef struct ora_sys ora_sys;

/* one thermo record, the values write_thermo prints (src/read_input.f90:433-446) */
typedef struct {
  int step;
  double potential, kinetic, energy_error, pressure, volume;
  double virial[6];
  double box[3];
} ora_thermo;

typedef void (*ora_thermo_cb)(const ora_thermo *t, void *user);

ora_sys *ora_new(void);
void ora_free(ora_sys *s);

/* number of OpenMP threads the static split uses (thread_num, src/nd.f90:37) */
void ora_set_threads(ora_sys *s, int nthreads);
int ora_get_threads(const ora_sys *s);
void ora_set_mode(ora_sys *s, int mode);

/* 'Types' directive, src/read_input.f90:124-134 */
int ora_set_types(ora_sys *s, int ntypes, const double *mass);

/* 'Pairs' directive + buildPairTables, src/read_input.f90:136-172,
 * src/potentials.f90:2-56.  names: npairs strings of 8 chars (padded or
 * NUL-terminated); params: 4*npairs (PairParams(1:4,j), trailing zeros for
 * absent parameters, PairParams(1,j) defaults to the current rcut);
 * p1/p2: 1-based type ids; sym: 1 for "sym". nparams[j] = number of
 * parameters given on the line (missing ones keep their defaults). */
int ora_set_pairs(ora_sys *s, int npairs, double ptrmin, int ptsize,
                  const int *p1, const int *p2, const int *sym,
                  const char *names, const double *params, const int *nparams,
                  const double *charge_prod);

/* read access to the tables: ppair/fpair are (ptsize+1)*npairs, column-major */
int ora_get_tables(const ora_sys *s, double *ppair, double *fpair,
                   double *rc2, double *dr2);
double ora_pot(const char *name, double r, const double *parm, double qprd,
               double rcut);
double ora_dpot(const char *name, double r, const double *parm, double qprd,
                double rcut);
int ora_get_pairmat(const ora_sys *s, int *pairmat);
double ora_get_rcut(const ora_sys *s);

/* model state; pos fractional, 3*np, vel/acc may be NULL (zero) */
int ora_set_state(ora_sys *s, int np, const int *typ, const double *pos,
                  const double *vel, const double *acc, const double box[3]);
int ora_get_state(const ora_sys *s, double *pos, double *vel, double *acc,
                  double *box);
int ora_get_forces(const ora_sys *s, double *force, double *potential,
                   double *virial, double *kinetic);
int ora_get_np(const ora_sys *s);

/* ensemble + list controls (src/read_input.f90:18-41 defaults) */
typedef struct {
  double dt;
  double skin;        /* < 0: 0.2*rcut at Run (src/nd.f90:77-79) */
  int neimax;         /* 0: estimate at Run (src/nd.f90:84-88) */
  int renei, renei_freq;
  int out_steps;
  int step;           /* global step counter (StepNumber) */
  int isokinetic, ke_freq; double ke_target, ke_parm;
  int isobaric, p_freq;    double p_target[3], p_parm;
  int isoenergetic, e_freq; double e_parm;
  int box_load;            double box_vel[3];
} ora_control;

void ora_default_control(ora_control *c);
int ora_set_control(ora_sys *s, const ora_control *c);
int ora_get_control(const ora_sys *s, ora_control *c);

/* per-routine entry points (the reference subroutines) */
int ora_setup_lists(ora_sys *s);       /* dynamics prologue src/nd.f90:73-108 */
int ora_build_cell_list(ora_sys *s);   /* src/nd.f90:1214-1260 (+Verlet) */
int ora_check_list_update(ora_sys *s); /* src/nd.f90:1447-1499; 1 if rebuilt */
void ora_integrate1(ora_sys *s);       /* src/nd.f90:984-1080 */
void ora_compute0(ora_sys *s, int cv, int cu); /* src/nd.f90:200-363 */
void ora_compute1(ora_sys *s, int cv, int cu); /* src/nd.f90:364-530 */
/* hold groups with displacement conditions, src/read_input.f90:177-190 */
int ora_set_holds(ora_sys *s, const int *hold, int ngroups, const int *dir, const double *du);
void ora_compute2(ora_sys *s, int cv, int cu); /* springs, src/nd.f90:531-727 */
void ora_compute3(ora_sys *s, int cv, int cu); /* springs + one-sided pairs, src/nd.f90:728-933 */
void ora_compute(ora_sys *s, int cv, int cu);  /* the dispatch of src/nd.f90:155-163 */
/* InitPos / initPositionSet, src/nd.f90:1731-1762 (NULL: the current state) */
int ora_init_positions(ora_sys *s, const double *ipos, const double *ibox);
void ora_integrate2(ora_sys *s, int ck);       /* src/nd.f90:1081-1121 */
void ora_mk_iso_ke(ora_sys *s);        /* src/nd.f90:1122-1158 */
void ora_mk_iso_e(ora_sys *s);         /* src/nd.f90:1159-1182 */
void ora_mk_iso_p(ora_sys *s);         /* src/nd.f90:1183-1213 */

/* the whole dynamics loop for nsteps steps (src/nd.f90:60-199) */
int ora_run(ora_sys *s, int nsteps, double dt, ora_thermo_cb cb, void *user);
/* the loop alone, after ora_setup_lists (what the reference times) */
int ora_run_loop(ora_sys *s, int nsteps, double dt, ora_thermo_cb cb, void *user);

/* list inspection: cell (0-based ICELL-1) of each atom; neighbour pairs
 * (i<j, 0-based, one entry per occurrence in the half list) */
int ora_get_mcell(const ora_sys *s, int *mcell);
int ora_get_cells(const ora_sys *s, int *cell);
long ora_get_neighbors(const ora_sys *s, int *pairs, long cap);
int ora_get_list_updates(const ora_sys *s);
int ora_get_neimax(const ora_sys *s);
double ora_get_skin(const ora_sys *s);

/* seeded Maxwell-Boltzmann velocities: the reference's ratio-of-uniforms
 * generator (src/nd.f90:1500-1624) driven by SplitMix64 instead of the
 * gfortran random_number stream (which cannot be reproduced here). */
void ora_velocity(ora_sys *s, float kt, unsigned long long seed);

/* Fortran G14.6 edit descriptor, for thermo lines identical to the reference */
void ora_fmt_g14_6(double x, char *out15);
void ora_fmt_thermo(const ora_thermo *t, char *out96);

#ifdef __cplusplus
}
#endif
#endif
