/*
 * ndyn_gpu.h -- C ABI of the B200 (sm_100a) Ndyn timestep library.
 *
 * Drop-in boundary for the MD timestep path of Ndyn (stewmasterj/Ndyn_OMP).
 * The reference has no FFI: its timestep routines are argument-less Fortran
 * subroutines working on module globals (src/mods.f90).  Each entry point
 * below replaces one of them and takes the module data explicitly, as plain
 * pointers and sizes in the reference's own layouts:
 *
 *   pos(3,np), vel(3,np), acc(3,np), force(3,np)  real(8), column-major
 *        (x,y,z of one atom contiguous); pos is fractional, in box units
 *   typ(np)                integer(4), 1-based type ids
 *   PairMat(ntypes,ntypes) integer(4), column-major, 1-based pair ids, 0=none
 *   PPairTable/FPairTable(PTsize+1,NPairs) real(8), column-major
 *   box(3), virial(6)      real(8)
 *
 * A context (ndg_ctx) owns the device copy of one or more independent
 * systems ("replicas"); system ids are small integers.  Every call returns
 * an int status: NDG_OK (0) or a negative NDG_ERR_* code, where the
 * reference would STOP.  Calls on one context are not thread-safe;
 * separate contexts are independent.  Host arrays are caller-owned and are
 * copied in or out during the call.
 *
 * Fortran binds these with ISO_C_BINDING interface blocks (bind(C,name=...),
 * value arguments for scalars, type(c_ptr) for the context).
 */
#ifndef NDYN_GPU_H
#define NDYN_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NDG_ABI_VERSION 1

/* status codes */
enum {
  NDG_OK = 0,
  NDG_ERR_ARG = -1,        /* bad argument or call order */
  NDG_ERR_NEIMAX = -2,     /* 'too many neighbours in list' src/nd.f90:1378,1421 */
  NDG_ERR_OUT_OF_BOX = -3, /* 'Particle outside of box' src/nd.f90:1494 */
  NDG_ERR_POTENTIAL = -4,  /* unknown potential name src/potentials.f90:148,244 */
  NDG_ERR_CELLS = -5,      /* fewer than 2 link cells in a direction
                              (box < 2*(rcut+skin): the single-anint minimum
                              image of src/nd.f90:283-288 is then invalid) */
  NDG_ERR_NOMEM = -6,      /* device allocation failed */
  NDG_ERR_CUDA = -7,       /* CUDA runtime error (see ndg_last_error) */
  NDG_ERR_BUDGET = -8,     /* request does not fit the HBM budget */
  NDG_ERR_NOT_FOUND = -9,  /* unknown system or request id */
  NDG_ERR_TIMEOUT = -10    /* bounded wait expired */
};

/* arithmetic of the pair loop */
enum {
  NDG_PREC_FP64 = 0,  /* the reference's FP64 path (FP32 table index only) */
  NDG_PREC_MIXED = 1  /* FP32 pair math on 32-bit fixed-point fractional
                         positions, 64-bit fixed-point force sums, FP64
                         integrator, reductions and box */
};

/* list semantics */
enum {
  NDG_QUIRK_REF = 0,   /* exactly the reference: list rebuild test compares
                          fractional displacements with skin^2 in A^2
                          (src/nd.f90:1488-1493), and the 14-cell half
                          stencil repeats pairs when a cell count is 2
                          (src/nd.f90:1268-1300) */
  NDG_QUIRK_FIXED = 1  /* rebuild when the two largest displacements (A)
                          plus any box shrink exceed the skin; each distinct
                          neighbour cell visited once */
};

typedef struct ndg_ctx ndg_ctx;

/* Run control; the values of module 'control' and 'listData'
 * (src/mods.f90:79-95) with the defaults of src/read_input.f90:18-41. */
typedef struct {
  double dt;            /* time step (Run [i] {r}) */
  double skin;          /* Skin; < 0 means 0.2*rcut at run start (src/nd.f90:77-79) */
  int neimax;           /* NeiMax; 0 = estimate (src/nd.f90:84-88) */
  int renei;            /* ReNeighbor T/F */
  int renei_freq;       /* check interval */
  int out_steps;        /* OutFreq */
  int step;             /* global step counter (StepNumber) */
  int isokinetic, ke_freq;
  double ke_target, ke_parm;
  int isobaric, p_freq;
  double p_target[3], p_parm;
  int isoenergetic, e_freq;
  double e_parm;
  int box_load;
  double box_vel[3];
  int quirk;            /* NDG_QUIRK_* */
} ndg_control;

/* One write_thermo record (src/read_input.f90:433-446), plus the raw
 * virial and box. */
typedef struct {
  int sys;
  int step;
  double potential, kinetic, energy_error, pressure, volume;
  double virial[6];
  double box[3];
} ndg_thermo;

typedef void (*ndg_thermo_cb)(const ndg_thermo *t, void *user);

/* ---- library ---------------------------------------------------------- */
int ndg_abi_version(void);
const char *ndg_error_string(int status);
/* last CUDA error text recorded on ctx (or globally when ctx is NULL) */
const char *ndg_last_error(const ndg_ctx *ctx);

/* Host restatement of buildPairTables + pot/dpot (src/potentials.f90:2-247)
 * for callers that do not tabulate themselves (the C++ driver).  names are
 * npairs blocks of 8 characters (blank- or NUL-padded), params 4*npairs
 * (PairParams(1:4,j), PairParams(1,j) = cutoff), qprod the charge products
 * (may be NULL).  Outputs: ppair/fpair (ptsize+1)*npairs, rc2/dr2 npairs. */
int ndg_build_pair_tables(int npairs, int ptsize, double ptrmin,
                          const char *names, const double *params,
                          const double *qprod, double *ppair, double *fpair,
                          double *rc2, double *dr2);

/* ---- context and systems --------------------------------------------- */
int ndg_create(ndg_ctx **ctx, int device, int precision);
int ndg_destroy(ndg_ctx *ctx);
int ndg_set_precision(ndg_ctx *ctx, int precision);

/* Add a system: the interpot module (src/mods.f90:51-77) for it plus its
 * atoms.  rcpair = PairParams(1,1:npairs).  Tables are copied.  Returns the
 * new id in *sys.  vel/acc may be NULL (zero, as read_model leaves them,
 * src/read_input.f90:354-355). */
int ndg_add_system(ndg_ctx *ctx, int np, int ntypes, int npairs, int ptsize,
                   double ptrmin, const double *mass, const int *pairmat,
                   const double *rcpair, const double *ppair,
                   const double *fpair, const int *typ, const double *pos,
                   const double *vel, const double *acc, const double *box,
                   int *sys);
int ndg_remove_system(ndg_ctx *ctx, int sys);
int ndg_num_systems(const ndg_ctx *ctx);

/* replace (load) or read (get) positions/velocities/accelerations/box of a
 * system; vel/acc/box may be NULL (load: zero velocities/accelerations, box
 * kept).  sys = -1 moves every live system at once: the arrays hold the
 * systems one after another in ascending id order (3*np doubles each, in
 * the reference's layout) and box holds 3 doubles per system.  That form
 * copies each array in one transfer, straight from or into the caller's
 * buffers (page-locked ones move by DMA), and waits once for all systems. */
int ndg_load_state(ndg_ctx *ctx, int sys, const double *pos, const double *vel,
                   const double *acc, const double *box);
int ndg_get_state(ndg_ctx *ctx, int sys, double *pos, double *vel, double *acc,
                  double *box);
int ndg_set_control(ndg_ctx *ctx, int sys, const ndg_control *c);
int ndg_get_control(ndg_ctx *ctx, int sys, ndg_control *c);
/* Hold groups with displacement conditions, integrate1's Nhold branch
 * (src/nd.f90:1048-1077; the Hold and Disp directives fill hold(np),
 * bcDir and bcParm, src/read_input.f90:177-190).  hold[i] is the group
 * (1..ngroups, 0 = none) of atom i in input order; where
 * dir[3*(g-1)+d] != 0, an atom of group g moves by du[3*(g-1)+d]
 * (fractional units) along axis d every step instead of by its velocity.
 * hold == NULL or ngroups == 0 removes the system's holds. */
int ndg_set_holds(ndg_ctx *ctx, int sys, const int *hold, int ngroups, const int *dir,
                  const double *du);
/* Spring pairs (compute2/compute3, src/nd.f90:531-933): where spring[k] != 0
 * pair k+1 is a 'spring' line with PairParams params[4k..4k+3] = rc, D0, sc,
 * Vol (src/read_input.f90:136, :271).  Such a pair acts through its strain
 * against the initial positions, s = r/r0 - 1, with force -D0*s*Vol^2 along
 * the pair and energy D0*s^2*Vol^2*r0/2, and not at all while s > sc.
 * spring == NULL removes them.  Until ndg_set_initial_positions is called,
 * the first run's prologue takes the positions it starts from
 * (src/nd.f90:104). */
int ndg_set_springs(ndg_ctx *ctx, int sys, const int *spring, const double *params);
/* InitPos (initPositionSet, src/nd.f90:1731-1762): the initial positions
 * (3 x np fractional, input order) and box of the spring strains; NULL takes
 * the system's current positions or box. */
int ndg_set_initial_positions(ndg_ctx *ctx, int sys, const double *ipos, const double *ibox);
void ndg_default_control(ndg_control *c);

/* ---- the reference routines, one call each (all systems of ctx) -------- */
/* dynamics prologue src/nd.f90:73-108: skin default, link-cell counts,
 * neighbour capacity, cell list + Verlet list build */
int ndg_setup_lists(ndg_ctx *ctx);
/* buildCellList + buildVerletList, src/nd.f90:1214-1446 */
int ndg_build_cell_list(ndg_ctx *ctx);
/* CheckListUpdate, src/nd.f90:1447-1499; *rebuilt (may be NULL) gets the
 * number of systems whose lists were rebuilt */
int ndg_check_list_update(ndg_ctx *ctx, int *rebuilt);
/* integrate1, src/nd.f90:984-1047 */
int ndg_integrate1(ndg_ctx *ctx);
/* compute0(CV,CU), src/nd.f90:200-363 */
int ndg_compute(ndg_ctx *ctx, int cv, int cu);
/* integrate2(CK), src/nd.f90:1081-1121 */
int ndg_integrate2(ndg_ctx *ctx, int ck);
/* mkIsoKE / mkIsoE / mkIsoP, src/nd.f90:1122-1213, on system sys */
int ndg_mk_iso_ke(ndg_ctx *ctx, int sys);
int ndg_mk_iso_e(ndg_ctx *ctx, int sys);
int ndg_mk_iso_p(ndg_ctx *ctx, int sys);

/* force(3,np), potential, virial(6), kinetic of the last compute/integrate */
int ndg_get_forces(ndg_ctx *ctx, int sys, double *force, double *potential,
                   double *virial, double *kinetic);

/* ---- the dynamics loop ------------------------------------------------- */
/* The time-step loop of dynamics (src/nd.f90:137-180) for nsteps steps on
 * every system, fused on the device (CUDA graphs of fixed step blocks).
 * Lists are rebuilt at the start (as dynamics does).  cb (may be NULL)
 * receives every write_thermo record in step order. */
int ndg_run(ndg_ctx *ctx, int nsteps, ndg_thermo_cb cb, void *user);
/* Continues the last run by nsteps more steps, without the prologue list
 * build: the step count within the run, e0 and the list decision carry on,
 * so ndg_run(n) followed by ndg_run_continue(m) gives the same states and
 * write_thermo records as ndg_run(n + m).  A caller that writes the model
 * every ConfOutFreq steps (write_model, src/nd.f90:172) runs the steps in
 * such pieces and reads the state in between. */
int ndg_run_continue(ndg_ctx *ctx, int nsteps, ndg_thermo_cb cb, void *user);
/* thermo scalars of the last completed step of a system */
int ndg_get_thermo(ndg_ctx *ctx, int sys, ndg_thermo *t);
/* number of list rebuilds since the run started (NlistUpdates) */
int ndg_get_list_updates(ndg_ctx *ctx, int sys, int *n);

/* ---- inspection (tests) ------------------------------------------------ */
/* link-cell counts MCELL(3) */
int ndg_get_mcell(ndg_ctx *ctx, int sys, int *mcell);
/* 0-based cell id (ICELL-1) of each atom, in the caller's atom order */
int ndg_get_cells(ndg_ctx *ctx, int sys, int *cell);
/* neighbour pairs (i<j, 0-based, caller's atom order): one entry per
 * occurrence of the unordered pair in the reference's half list.  With
 * pairs == NULL returns the count in *npairs. */
int ndg_get_neighbors(ndg_ctx *ctx, int sys, int *pairs, long long cap,
                      long long *npairs);
/* total entries of the system's full neighbour list (each pair counted
 * from both atoms), the length the pair loop of compute0 walks */
int ndg_get_neighbor_count(ndg_ctx *ctx, int sys, long long *entries);

/* ---- compute0 without device allocation ------------------------------- */
/* No counterpart in the reference (which allocates nothing on a GPU).
 *
 * The same forces, potential energy and virial as ndg_compute (compute0,
 * FP64) for one system, for callers that cannot allocate device memory:
 * host applications that hand all of a GPU's memory to their own pool (a
 * framework's caching allocator, a Fortran code that sizes everything at
 * start-up) and only lend out buffers, so that a cudaMalloc of ours would
 * fail or fragment their pool; and loops that must not stall on
 * cudaMalloc/cudaFree, which can synchronise the whole device.
 *
 * The caller owns every buffer: pos_d (3*np, fractional, reference layout),
 * typ_d (np), the tables fpair_d/ppair_d ((ptsize+1)*npairs, column-major)
 * and the output force_d (3*np) are device pointers; pairmat (ntypes^2,
 * column-major), rcpair (npairs) and box (3) are host arrays; skin and quirk
 * select the link-cell grid as ndg_setup_lists does (skin >= 0,
 * rcut + skin > 0).  Every typ_d entry must lie in 1..ntypes: an atom of
 * another type is left out of the sums and the call returns NDG_ERR_ARG.
 * potential and virial (6) are written on the host: the call waits for its
 * stream (cudaStreamSynchronize) and returns when they are.  stream is a
 * cudaStream_t (NULL: the legacy default stream).
 *
 * Scratch lives in one static device array of about 0.8 MB that every GPU
 * loading the library keeps until the process exits.  Limits: 32768 atoms,
 * 32768 link cells, 8 types, 36 pairs; larger inputs return NDG_ERR_ARG
 * with a message on stderr.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress).  The call waits for its
 * stream, so it cannot be recorded into a CUDA graph by stream capture.
 * All calls share the array: calls that overlap on the GPU (other streams
 * or threads) corrupt each other; order them. */
int ndg_compute0_static(int np, int ntypes, int npairs, int ptsize, double ptrmin,
                        const int *pairmat, const double *rcpair, double skin,
                        int quirk, const double *box, const double *fpair_d,
                        const double *ppair_d, const double *pos_d,
                        const int *typ_d, double *force_d, double *potential,
                        double *virial, void *stream);

/* ---- tuning ------------------------------------------------------------ */
/* threads per atom in the pair kernel (1,2,4,8; 0 = choose from the atom
 * count and mean neighbour count) and steps per CUDA-graph block */
int ndg_set_tuning(ndg_ctx *ctx, int threads_per_atom, int graph_steps);
int ndg_get_tuning(ndg_ctx *ctx, int *threads_per_atom, int *graph_steps);
/* neighbour gathers in flight per thread in the mixed one-thread-per-atom
 * pair loop: 4 (more resident warps) or 8 (more latency hidden) */
int ndg_set_gather_depth(ndg_ctx *ctx, int depth);
int ndg_get_gather_depth(ndg_ctx *ctx, int *depth);
/* Atoms to threads by list length: in a dynamics step, systems whose mean
 * full-list length (entries per atom at their last list build) is at least
 * `rows` run in pair launches of their own with `tpa_long` threads per atom
 * (1,2,4,8); the others with the context's threads per atom.  rows = 0: one
 * class (the default).  Mixed-precision forces do not depend on the split;
 * FP64 ones change in the last bits (the summation order of an atom's
 * neighbours follows its threads).  Standalone compute0 is not split.  No
 * counterpart in the reference (its OpenMP loop splits atoms evenly,
 * src/nd.f90:269-271). */
int ndg_set_list_split(ndg_ctx *ctx, int rows, int tpa_long);
int ndg_get_list_split(ndg_ctx *ctx, int *rows, int *tpa_long);
/* time candidate launch shapes (threads per atom; gather depth for one
 * thread per atom in mixed precision) on the current systems for a few
 * steps and keep the fastest; then, where the systems' mean list lengths
 * differ by 1.5x or more, the long-list class (ndg_set_list_split: the
 * threshold at the geometric middle of the shortest and longest, 2 or 4
 * threads per atom) is kept if a trial runs faster (state is restored
 * afterwards) */
int ndg_autotune(ndg_ctx *ctx, int steps_per_trial);
/* The rebuild-interval autotuner: choose each fixed-semantics system's list
 * skin (so its rebuild interval).  A trial of `steps` steps from freshly
 * built lists measures the pair kernel's cost per list row, the rebuild
 * cost per rebuilt tile and each system's rebuild count; a model proposes a
 * skin in [0.5, 2] x the current one per system, and a second trial with
 * the proposed skins must run at least 2% faster than the first, or every
 * skin stays.  Both trials are undone (state restored); the fixed systems'
 * lists are rebuilt (with the new skins, where kept), and the skins read
 * back through ndg_get_control.  Forces do not depend on the skin in the
 * fixed semantics; systems in the reference semantics keep theirs.
 * *changed (may be NULL) = systems whose skin changed.  No counterpart in the
 * reference (its Skin is an input, src/read_input.f90:95; its default
 * 0.2*rcut, src/nd.f90:77-79). */
int ndg_autotune_skin(ndg_ctx *ctx, int steps, int *changed);
/* device bytes the context holds, and the bytes one more system of np
 * atoms with ntypes/npairs/ptsize would need */
int ndg_device_bytes(const ndg_ctx *ctx, long long *bytes);
long long ndg_system_bytes(int np, int ntypes, int npairs, int ptsize,
                           double density, double rlist, int precision);

/* the CUDA stream every kernel of ctx is launched on (cudaStream_t) */
int ndg_get_stream(ndg_ctx *ctx, void **stream);
/* Continue the run for nsteps with eager launches and a CUDA event pair
 * around every kernel group; the mean duration per launch is then read with
 * ndg_get_kernel_times (integrate1, pair loop, list-rebuild group). */
int ndg_profile_run(ndg_ctx *ctx, int nsteps);
int ndg_get_kernel_times(ndg_ctx *ctx, double *integrate_ms, double *pair_ms,
                         double *rebuild_ms, int *launches);

/* ---- serving loop: continuous batching of MD runs ----------------------
 * No counterpart in the reference (one run per process).  A server owns a
 * context and keeps every admitted run's state on the device until the run
 * completes.  Requests queue on submit; each ndg_server_step admits queued
 * requests in submission order while their estimated device bytes
 * (ndg_system_bytes) fit the HBM budget (a request that does not fit waits,
 * later smaller ones may pass it), builds the new runs' lists, and advances
 * every resident run by one block of block_steps steps in one graph launch.
 * A run's trajectory does not depend on the runs it shares the device with:
 * in mixed precision it is the same bits as the run alone.  Not thread-safe
 * per server. */
typedef struct ndg_server ndg_server;

typedef struct ndg_request {
  int np, ntypes, npairs, ptsize; /* as ndg_add_system */
  double ptrmin;
  const double *mass;
  const int *pairmat;
  const double *rcpair, *ppair, *fpair;
  const int *typ;
  const double *pos, *vel; /* vel may be NULL (zero) */
  const double *box;
  ndg_control control; /* dt, skin, ensembles, OutSteps, quirk, ... */
  int nsteps;          /* steps of the run (one Run directive) */
  /* spring pairs as ndg_set_springs takes them, or NULL: none (the run's
   * prologue takes the positions it starts from as the initial ones) */
  const int *spring;
  const double *pair_params;
} ndg_request;

typedef struct ndg_server_stats {
  int queued, resident, completed, failed;
  long long bytes_in_use, budget;
  double atom_steps; /* atom-steps advanced so far */
  /* host wall seconds spent so far in admission (adding systems), run
   * prologues (list builds), blocks (graph launch to completion, including
   * graph captures) and retiring runs (state copies) */
  double t_admit, t_setup, t_block, t_retire;
  int graph_captures; /* step-block graphs captured by the context */
  int blocks;         /* blocks run */
} ndg_server_stats;

int ndg_server_create(ndg_server **srv, int device, int precision, long long hbm_budget_bytes,
                      int block_steps);
int ndg_server_destroy(ndg_server *srv);
/* copy the request's arrays and queue it; *ticket identifies it */
int ndg_server_submit(ndg_server *srv, const ndg_request *req, long long *ticket);
/* admit what fits, then one block for every resident run; *completed =
 * runs that finished in this call (their results wait for ndg_server_result) */
int ndg_server_step(ndg_server *srv, int *completed);
/* tickets finished (or failed) since the last poll, up to cap */
int ndg_server_poll(ndg_server *srv, long long *tickets, int cap, int *n);
/* status of a ticket: 0 queued, 1 resident, 2 done, a negative NDG_ERR_*
 * if the run failed */
int ndg_server_status(ndg_server *srv, long long ticket, int *status);
/* copy a finished run's final state (caller's atom order) and up to cap
 * write_thermo rows, then forget the request */
int ndg_server_result(ndg_server *srv, long long ticket, double *pos, double *vel, double *acc,
                      double *box, ndg_thermo *rows, int cap, int *nrows);
int ndg_server_stats_get(ndg_server *srv, ndg_server_stats *st);
/* the server's context (stream, tuning, kernel timings) */
int ndg_server_context(ndg_server *srv, ndg_ctx **ctx);
/* The admission rule alone (host only): walk the queue in order and admit
 * each request whose bytes fit what remains of the budget; admit[k] = 1 for
 * admitted ones.  Returns the number admitted. */
int ndg_admit_plan(const long long *bytes, int n, long long budget, long long in_use, int *admit);

#ifdef __cplusplus
}
#endif
#endif /* NDYN_GPU_H */
