// ndg_kernels.h -- kernel launch interface of the Ndyn timestep library.
#pragma once
#include <cuda_runtime.h>

#include "ndg_common.h"

namespace ndg {

// Work plan of the two pair launches of a dynamics step (made by integrate1): launch L
// (0 without energy/virial, 1 with) lists its systems in id order with the
// exclusive prefix of their cost, and names for each of its blocks the
// entry that holds the block's first unit of cost.
struct PlanEnt {
  long long cum;  // cost of the launch's earlier systems
  int sys, cpt;   // system, cost of one of its tiles
};
// A dynamics step's pair launches: (energy/virial or not) x (list-length
// class: 1 for systems whose mean list length reaches DevCtx::rows_split,
// which run with DevCtx::tpa_long threads per atom); launch L = ev + 2 cls.
constexpr int PLAN_NL = 4;
struct PlanHdr {
  long long tot[PLAN_NL];  // total cost of each launch
  int m[PLAN_NL];          // systems of each launch
};
constexpr int PLAN_GMAX = 8192;  // largest pair-kernel grid the plan covers

// Everything a kernel needs, passed by value (pointers into the arenas).
struct DevCtx {
  const SysParam *P;
  SysState *S;
  const int *chunk_sys;  // per ATOM_ALIGN-atom chunk: system id or -1
  const int *cell_sys;   // per global cell: system id or -1
  int nchunks, ncells, nsys_cap;
  int stab_smem;  // shared-memory bytes of the staged pair tables, 0 = read from global
  int stab_lean;  // the same without the energy table (kernel without energy/virial)
  int gather;   // mixed pair loop: neighbour gathers in flight (4 or 8)
  int any_spring;  // some system holds spring pairs: the pair kernels' spring variant
  int any_neimax;  // some system checks the reference's NeiMax after its list builds
  double4 *pos;
  int4 *pfx;
  double *vel, *acc, *disp, *force;
  int *gid;
  const int *hold;     // per atom, by input index: hold group (0 = none)
  const double4 *bcd;  // per hold group: displacement per step (x, y, z), w = axis mask
  const double4 *ipos; // per atom, by input index: initial position (spring strains)
  const double4 *spr;  // per pair: spring D0, sc, Vol, w = 1 for a spring pair
  int *nbr;  // blocked neighbour list (128-atom tiles), atom slots
  int *nnb;
  int *tile_rows;  // per tile: rows of its list in use (L2 prefetch size)
  int *atom_cell, *atom_slot, *cell_count, *cell_start;
  int *perm, *tmp_src, *tmp_key;
  double4 *s_pos;
  double *s_vel, *s_acc;
  int *s_gid, *s_cell;
  int *cxyz;  // per atom slot: link cell grid coordinates, x | y << 11 | z << 22 (rebuild scratch)
  const int *pairmat;  // PairMat per system (the list build)
  const int *pairg;    // gather matrix per system (the pair kernel)
  const double *mass, *rc2, *rlist2;
  const float *vdr2, *rc2f;
  const double *tabF, *tabP;
  const float2 *tabF2, *tabP2;
  double *red;   // pair-kernel block partials, 8 per block
  double *itop;  // integrate1 chunk partials, 2 per chunk
  double *ired;  // integrate2 (standalone) chunk partials
  ThermoRec *ring;
  int *ring_count;  // [0] records written, [1] error bits of any system,
                    // [2] largest tile candidate count, [3] systems on rb_list
  int *rb_list;     // systems whose lists the next rebuild group rebuilds
  PlanEnt *plan;    // 2 x nsys_cap entries
  int *plan_kb;     // PLAN_NL x PLAN_GMAX block starts
  int rows_split;   // list-length class threshold (mean entries per atom; 0: one class)
  int tpa_long;     // threads per atom of the long-list class
  PlanHdr *plan_hdr;
  int ring_cap;
};

// launchers (stream-ordered; safe to capture in a CUDA graph)
// a dynamics step's integrate1 (standalone 0) also plans the step's pair
// launches for tpa threads per atom
void launch_integrate1(const DevCtx &c, cudaStream_t st, int standalone, int mixed, int tpa = 1);
// next_h: conditional-node handle of the next step's rebuild group (0 when
// not launched inside a captured step block)
void launch_pair(const DevCtx &c, cudaStream_t st, int tpa, int mixed, int fuse, int host_flags,
                 unsigned long long next_h = 0);
void launch_decide(const DevCtx &c, cudaStream_t st, unsigned long long h);
void launch_integrate2(const DevCtx &c, cudaStream_t st, int ck);
void launch_rebuild(const DevCtx &c, cudaStream_t st, int counting, int mixed);
void launch_arm(const DevCtx &c, cudaStream_t st, int nsys_cap, int sys, int nsteps, int start);
void launch_begin_block(const DevCtx &c, cudaStream_t st, int nsys_cap, int K);
void launch_flush(const DevCtx &c, cudaStream_t st, int nsys_cap, int sys, int chunk0 = 0,
                  int nch = 0);
void launch_check(const DevCtx &c, cudaStream_t st, int nsys_cap);
void launch_scale_vel(const DevCtx &c, cudaStream_t st, int sys, double lam);
void launch_refresh_pfx(const DevCtx &c, cudaStream_t st);
// every system's state in one pass: xoff[s] = system s's first atom in the
// caller's concatenated (3,total) arrays, -1 to skip it; the staging blocks
// xp/xv/xa (device, that layout) may be null where an array is not moved
void launch_load_all(const DevCtx &c, cudaStream_t st, const long long *xoff, const double *xp,
                     const double *xv, const double *xa);
void launch_store_all(const DevCtx &c, cudaStream_t st, const long long *xoff, double *xp,
                      double *xv, double *xa);

// bytes of shared memory a system's tables need in the staged layout of the
// pair kernel: pair matrix, per-pair cutoffs/scales, then the F and P tables
NDG_HD int stab_bytes(int ntypes, int npairs, int ptsize) {
  int b = (ntypes * ntypes * 4 + 15) / 16 * 16;
  b += npairs * 8;  // rc2 (double)
  b = (b + 15) / 16 * 16;
  b += npairs * 16;  // packed float4 per pair
  b += npairs * (ptsize + 1) * 16;  // F and P: a double each, or a float2 each
  return b;
}

// the staged layout without the P table
NDG_HD int stab_bytes_lean(int ntypes, int npairs, int ptsize) {
  return stab_bytes(ntypes, npairs, ptsize) - npairs * (ptsize + 1) * 8;
}

// stencil of neighbour cells for a link-cell grid (shared host/device)
NDG_HD int make_stencil(const int *mcell, int quirk, int *out) {
  // the 13 forward offsets of getJcellNP cases 2..14, src/nd.f90:1270-1282
  const int fwd[13][3] = {{0, 0, 1}, {0, 1, 0},  {0, 1, -1},  {0, 1, 1},  {1, 0, 0},
                          {1, 0, -1}, {1, 0, 1}, {1, 1, 0},   {1, 1, -1}, {1, 1, 1},
                          {1, -1, 0}, {1, -1, -1}, {1, -1, 1}};
  int n = 0;
  out[n++] = (1) | (1 << 4) | (1 << 8) | (1 << 12);  // the cell itself
  if (mcell[0] >= 3 && mcell[1] >= 3 && mcell[2] >= 3) {
    // three or more cells per axis: the 26 neighbours are distinct cells,
    // and each is one forward offset of the half stencil or the negative of
    // one (multiplicity 1 in either semantics); the order of the loop below
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx)
          if (dx || dy || dz) out[n++] = (dx + 1) | ((dy + 1) << 4) | ((dz + 1) << 8);
    return n;
  }
  int seen[27][3];
  int nseen = 0;
  for (int dz = -1; dz <= 1; ++dz)
    for (int dy = -1; dy <= 1; ++dy)
      for (int dx = -1; dx <= 1; ++dx) {
        if (!dx && !dy && !dz) continue;
        const int o[3] = {dx, dy, dz};
        int f[3];
        for (int d = 0; d < 3; ++d) f[d] = ((o[d] % mcell[d]) + mcell[d]) % mcell[d];
        if (!f[0] && !f[1] && !f[2]) continue;  // folds onto itself (1 cell)
        bool dup = false;
        for (int q = 0; q < nseen; ++q)
          dup |= seen[q][0] == f[0] && seen[q][1] == f[1] && seen[q][2] == f[2];
        if (dup) continue;
        seen[nseen][0] = f[0];
        seen[nseen][1] = f[1];
        seen[nseen][2] = f[2];
        ++nseen;
        int mult = 1;
        if (quirk == 0) {
          // times the reference's half stencil reaches this cell from either
          // side: forward offsets equal to +f or to -f modulo the cell count
          mult = 0;
          for (int k = 0; k < 13; ++k) {
            bool pos = true, neg = true;
            for (int d = 0; d < 3; ++d) {
              int t = ((fwd[k][d] % mcell[d]) + mcell[d]) % mcell[d];
              pos &= t == f[d];
              neg &= t == (mcell[d] - f[d]) % mcell[d];
            }
            mult += pos + neg;
          }
        }
        for (int m = 0; m < mult && n < MAX_STENCIL; ++m)
          out[n++] = (dx + 1) | ((dy + 1) << 4) | ((dz + 1) << 8);
      }
  return n;
}

}  // namespace ndg
