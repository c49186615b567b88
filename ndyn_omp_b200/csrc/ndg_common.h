// ndg_common.h -- device data layout and the host/device-shared arithmetic of
// the Ndyn timestep library.
//
// Layout in HBM (one context = a batch of independent systems):
//   * every system owns a contiguous atom range [atom_off, atom_off+npad),
//     npad = n rounded up to ATOM_ALIGN, so a block of any atom-parallel
//     kernel never straddles two systems; padding slots have gid = -1.
//   * pos   double4 per atom: fractional x,y,z (unwrapped, as the reference
//           keeps them) and w = (type | sys<<16) stored as an integer bit
//           pattern, so a neighbour gather brings the type along.
//   * pfx   int4 per atom (mixed precision only): x,y,z as 32-bit fixed-point
//           fractions of the box (2^32 = one box length; integer wrap-around
//           is the periodic minimum image), w as in pos.
//   * vel, acc, disp, force: (3,np) FP64, the reference's own layout.
//   * nbr   full neighbour list, blocked SoA per system: tiles of 128 atoms,
//           entry k of atom t of a tile at word k*128 + t of the tile's
//           block (nbr_off + (local_i/128)*maxnb*128), k < maxnb; nnb[i] =
//           count.  Packed lists (SysParam::nb16) hold 16-bit offsets from
//           the system's first atom, entries 2w and 2w+1 in the low and high
//           half of word w*128 + t.  A tile's list is one contiguous region,
//           so the pair kernel streams it with dense DRAM access.
//   * atoms are kept sorted by link cell (cell-major, original id inside a
//     cell); gid[i] maps back to the caller's order.
#pragma once
#include <cstdint>

#ifdef __CUDACC__
#define NDG_HD __host__ __device__ __forceinline__
#else
#define NDG_HD inline
#endif

namespace ndg {

constexpr int ATOM_ALIGN = 256;   // padding unit of a system's atom range
constexpr int BLOCK = 256;        // threads of the atom-parallel kernels
constexpr int MAX_STENCIL = 27;   // neighbour-cell entries incl. repeats
constexpr int MAX_TYPES = 64;
constexpr double FX_ONE = 4294967296.0;  // 2^32: one box length in pfx units
constexpr double FORCE_FX = 4294967296.0; // 2^32 fixed-point units per eV/A

// per-step work flags (SysState::flags)
enum : int {
  F_CV = 1,        // virial this step (calcVirial)
  F_CU = 2,        // potential energy (calcPot)
  F_CK = 4,        // kinetic energy (calcKE)
  F_OUT = 8,       // write_thermo this step
  F_ACTIVE = 16,   // system has steps left in the current run
  F_KE_SCALE = 32, // mkIsoKE after this step
  F_P_SCALE = 64,  // mkIsoP after this step
  F_E_SCALE = 128, // mkIsoE after this step
  F_FIRST = 256,   // first step of a run (tt == 1): e0 is set
  F_DONE = 512     // the pair kernel finished this step (set with the next
                   // step's flags, cleared by the next integrate1)
};

// Entry (ti, tj) of the pair kernel's gather matrix: the table of the force
// on an atom of type ti from one of type tj, max(PairMat(ti,tj),
// PairMat(tj,ti)), when PairMat(tj,ti) > 0 and else 0, with PT_ASYM set
// where the two directions differ (compute1, src/nd.f90:447,474-498: such
// pairs add no energy and no virial).  Symmetric matrices gather PairMat.
constexpr int PT_ASYM = 1 << 16, PT_MASK = PT_ASYM - 1;
NDG_HD int gather_entry(const int *pm, int nt, int ti, int tj) {
  const int ij = pm[(ti - 1) + (tj - 1) * nt], ji = pm[(tj - 1) + (ti - 1) * nt];
  if (ji <= 0) return 0;
  return (ij > ji ? ij : ji) | (ij != ji ? PT_ASYM : 0);
}

// error bits (SysState::err)
enum : int { E_NEIMAX = 1, E_OUT_OF_BOX = 2, E_CELLS = 4 };

// Read-only per-system parameters (changed only between runs).
struct SysParam {
  int atom_off, n, npad;
  int cell_off, ncell_cap;       // cells reserved for this system
  int mcell0[3];                 // link cells at run start
  long long nbr_off;
  int maxnb;
  int nb16;                      // list entries packed as 16-bit offsets from atom_off,
                                 // two per 32-bit word (list_entry, ndg_kernels.cu)
  int neimax_stop;               // reference semantics: NeiMax, the longest half list
                                 // an atom may have (else 'too many neighbours'); 0 = none
  int tab_off;                   // table entry of pair 1, entry 1
  int pair_off, type_off, pm_off;
  int ntypes, npairs, ptsize;
  int quirk;
  double ptrmin;
  double dt, skin, skinsq, rlist; // rlist = rcut + skin
  int renei, renei_freq, out_steps;
  int isokinetic, ke_freq, isobaric, p_freq, isoenergetic, e_freq, box_load;
  double ke_target, ke_parm, p_target[3], p_parm, e_parm, box_vel[3];
  int nhold, bc_off;             // hold groups, their first entry in DevCtx::bcd
  int nspring;                   // spring pairs (their DevCtx::spr entries are set)
  double ibox[3];                // box of the initial positions (spring strains)
};

// Mutable per-system state, resident on the device for the whole run.
struct SysState {
  double box[3];
  double box_build[3];   // box at the last list build
  double li[3];          // 1/box used by integrate1
  double potential, kinetic, virial[6], e0;
  double lam_ke, lam_e;  // velocity scales pending from mkIsoKE / mkIsoE
  double dtop[2];        // two largest displacement measures (list check)
  int mcell[3], ncell;
  int step, tt, steps_left;
  int flags;
  int pend;              // bit0: lam_ke pending, bit1: lam_e pending
  int rebuild;           // rebuild lists before the next integrate1
  int nlist_updates;
  int nstencil;                  // neighbour-cell stencil of the current grid:
  int stencil[MAX_STENCIL];      // (dx+1) | (dy+1)<<4 | (dz+1)<<8 | center<<12
  int err;
  unsigned int ticket;   // last-block election of the pair kernel
  unsigned int ticket_i; // last-block election of integrate2 (standalone)
  int run_left;          // steps of the current run not yet given to a block
  int start;             // how the next block begins: START_* (0 = continue)
  unsigned long long rows;  // rows of the last list build summed over the tiles
};

// SysState::start: a block continues the run, or starts a new one (tt = 1)
// with its lists just built (no list check on its first step) or without
enum : int { START_CONTINUE = 0, START_BUILT = 1, START_NEW = 2 };

// Device copy of one write_thermo record; layout equals ndg_thermo.
struct ThermoRec {
  int sys, step;
  double potential, kinetic, energy_error, pressure, volume;
  double virial[6];
  double box[3];
};

// ---- shared arithmetic (identical bits on host and device) -------------

NDG_HD int step_flags(const SysParam &p, int step, int tt) {
  int f = 0;
  const bool out = (step % p.out_steps == 0) || tt == 1;
  if (out) f |= F_CV | F_CU | F_CK | F_OUT;
  if (p.isokinetic && step % p.ke_freq == 0) f |= F_CK | F_KE_SCALE;
  if (p.isobaric && step % p.p_freq == 0) f |= F_CV | F_P_SCALE;
  if (p.isoenergetic && step % p.e_freq == 0) f |= F_CU | F_CK | F_E_SCALE;
  if (tt == 1) f |= F_FIRST;
  return f;
}

// mkIsoKE, src/nd.f90:1135-1136
NDG_HD double lam_iso_ke(const SysParam &p, double kinetic, int n) {
  double lam = 1.0 + p.dt / p.ke_parm * (p.ke_target * (double)n / kinetic - 1.0);
  return sqrt(lam);
}

// mkIsoE, src/nd.f90:1168
NDG_HD double lam_iso_e(const SysParam &p, double e0, double potential, double kinetic) {
  return 1.0 - p.dt / p.e_parm * (e0 / (potential + kinetic) - 1.0);
}

// mkIsoP, src/nd.f90:1192-1210: rows updated in place, in order
NDG_HD void iso_p_box(const SysParam &p, const double *virial, double *box) {
  double vol = box[0] * box[1] * box[2];
  double press[6], lam[6];
  for (int k = 0; k < 6; ++k) press[k] = virial[k] / vol;
  const double f = p.dt / p.p_parm;
  lam[0] = 1.0 - f * (p.p_target[0] - press[0]);
  lam[1] = 1.0 - f * (p.p_target[1] - press[1]);
  lam[2] = 1.0 - f * (p.p_target[2] - press[2]);
  lam[3] = f * press[3];
  lam[4] = f * press[4];
  lam[5] = f * press[5];
  box[0] = box[0] * lam[0] + box[1] * lam[5] + box[2] * lam[4];
  box[1] = box[0] * lam[5] + box[1] * lam[1] + box[2] * lam[3];
  box[2] = box[0] * lam[4] + box[1] * lam[3] + box[2] * lam[2];
}

// write_thermo, src/read_input.f90:440-443
NDG_HD void make_thermo(ThermoRec &t, int sys, int step, double pe, double ke, double e0,
                        const double *vir, const double *box) {
  t.sys = sys;
  t.step = step;
  t.potential = pe;
  t.kinetic = ke;
  t.energy_error = (pe + ke - e0) / e0;
  t.pressure = (vir[0] + vir[1] + vir[2]) / (box[0] * box[1] * box[2] * 3.0);
  t.volume = box[0] * box[1] * box[2];
  for (int k = 0; k < 6; ++k) t.virial[k] = vir[k];
  for (int k = 0; k < 3; ++k) t.box[k] = box[k];
}

// List rebuild test of CheckListUpdate, src/nd.f90:1486-1497.  t1,t2 are
// the two largest per-atom measures: squared fractional displacements in
// the reference semantics, squared Angstrom displacements in the fixed one.
// Returns 1 = rebuild, 0 = keep, -1 = particle outside of box.
NDG_HD int list_check(const SysParam &p, const SysState &s, double t1, double t2) {
  if (p.quirk == 0) {
    double disp = t1 + t2;
    if (disp > p.skinsq) return disp > 1.0 ? -1 : 1;
    return 0;
  }
  double shrink = 0.0;
  for (int d = 0; d < 3; ++d) {
    double f = 1.0 - s.box[d] / s.box_build[d];
    if (f > shrink) shrink = f;
  }
  double moved = sqrt(t1) + sqrt(t2) + shrink * p.rlist;
  if (!(moved == moved)) return -1;  // NaN positions
  return moved > p.skin ? 1 : 0;
}

NDG_HD int pack_tw(int type, int sys) { return (type & 0xffff) | (sys << 16); }
NDG_HD int tw_type(int w) { return w & 0xffff; }
NDG_HD int tw_sys(int w) { return (int)((unsigned)w >> 16); }

}  // namespace ndg
