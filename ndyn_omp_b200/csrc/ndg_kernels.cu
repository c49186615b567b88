// ndg_kernels.cu -- sm_100a kernels of the Ndyn MD timestep path.
//
// Compiled with --fmad=false: every FP64 expression that restates the
// reference keeps its literal operation order (the neighbour list and the
// link-cell assignment are compared bit for bit with the reference's
// arithmetic).  The mixed-precision pair kernel asks for FMAs explicitly.
//
// Kernels of one MD step (src/nd.f90:137-178), all systems in one launch:
//   [rebuild]  k_bin -> k_scan -> k_scatter -> k_order -> k_permute ->
//              k_copyback -> k_build_atoms | k_build_cells
//              [-> k_neimax]                (only systems whose check fired)
//   k_integrate1                           (integrate1 + pending mkIso* scales;
//                                           one more block plans the pair
//                                           launches' shares of the systems)
//   k_pair<TPA,MIXED,FUSE>                 (compute0 + integrate2, and in the
//                                           last block of each system:
//                                           reductions, write_thermo,
//                                           mkIsoKE/P/E, BoxVel, next step's
//                                           CheckListUpdate decision)
#include <cstdio>

#include <algorithm>
#include <climits>
#include <type_traits>

#include "ndg_kernels.h"

namespace ndg {

constexpr int TILE = 128;  // atoms per tile of the neighbour list and the pair kernel

__device__ __forceinline__ int tw_of(double w) { return (int)__double_as_longlong(w); }

// Entry k of an atom's neighbour list; col points at the atom's column of
// its tile's list block (block start + the atom's index in the tile).  A
// plain list holds atom slots, one per 32-bit word, entry k in word k*TILE;
// a packed list (SysParam::nb16: mixed precision, systems under 65,536
// atoms) holds 16-bit offsets from the system's first atom, entry k in half
// k&1 of word (k>>1)*TILE, so one 32-bit load brings two entries.
__device__ __forceinline__ int list_entry(const int *col, int nb16, int atom_off, int k) {
  if (nb16)
    return atom_off + (int)__ldg((const unsigned short *)(col + (k >> 1) * TILE) + (k & 1));
  return __ldg(col + k * TILE);
}

__device__ __forceinline__ void list_store(int *col, int nb16, int atom_off, int k, int j) {
  if (nb16) ((unsigned short *)(col + (k >> 1) * TILE))[k & 1] = (unsigned short)(j - atom_off);
  else col[k * TILE] = j;
}

// 32-bit words a tile's list of `rows` rows occupies
__device__ __forceinline__ int list_words(int rows, int nb16) {
  return nb16 ? (rows + 1) >> 1 : rows;
}

// An atom's list has landed: its tile's rows (the tile's longest list,
// capped at maxnb; the pair kernel's L2 prefetch size) and the system's sum
// of them (the work plan's list-length measure) follow it.  atomicMax
// returns the tile's previous maximum, so the increments added to the sum
// add up to the final maximum of every tile, whatever the order.
__device__ __forceinline__ void note_rows(const DevCtx &c, SysState *S, int i, int r) {
  const int old = atomicMax(c.tile_rows + i / TILE, r);
  if (r > old) atomicAdd(&S->rows, (unsigned long long)(r - old));
}

// record an error on the system and in the context-wide error word
__device__ __forceinline__ void set_err(const DevCtx &c, SysState *S, int bits) {
  atomicOr(&S->err, bits);
  atomicOr(c.ring_count + 1, bits);
}

__device__ __forceinline__ int fx32(double x) {
  // fractional coordinate -> 32-bit fixed point, wrapping modulo one box
  long long q = __double2ll_rn(x * FX_ONE);
  return (int)(unsigned int)(unsigned long long)q;
}

// two largest of {a1,a2,b1,b2} given a1>=a2, b1>=b2
__device__ __forceinline__ void top2_merge(double &a1, double &a2, double b1, double b2) {
  double r1 = fmax(a1, b1);
  double r2 = fmax(fmin(a1, b1), fmax(a2, b2));
  a1 = r1;
  a2 = r2;
}

__device__ __forceinline__ void warp_top2(double &t1, double &t2) {
  for (int o = 16; o > 0; o >>= 1) {
    double b1 = __shfl_down_sync(0xffffffffu, t1, o);
    double b2 = __shfl_down_sync(0xffffffffu, t2, o);
    top2_merge(t1, t2, b1, b2);
  }
}

template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double *sm /*NV*32*/) {
  // deterministic tree: shuffle-down inside warps, then warp 0 over warps
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int k = 0; k < NV; ++k)
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < NV; ++k) sm[k * 32 + warp] = v[k];
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int k = 0; k < NV; ++k) {
      double x = lane < nw ? sm[k * 32 + lane] : 0.0;
      for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
      v[k] = x;
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Work plan of a dynamics step's two pair launches (g0 and g1 blocks), made
// by one extra block of the step's integrate1 (the flags and lists are set
// by then).  An active system's tile costs the mean row count of its last
// list build plus TILE_OVH (the per-tile integration and reduction work);
// every block of a launch takes the tiles whose first cost unit falls in
// its equal share of the launch's total, so systems with long lists, short
// lists or the other launch's flags leave no block idle and no block steps
// over tiles.
constexpr int TILE_OVH = 16;

// NL launches: 2 (energy/virial or not) with one list-length class, 4 with two
template <int NL>
__device__ void plan_block(const DevCtx &c, const int *g /*NL grids*/) {
  __shared__ long long w_cost[NL][32];
  __shared__ int w_cnt[NL][32];
  __shared__ long long carry_cost[NL];
  __shared__ int carry_cnt[NL];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x < NL) {
    carry_cost[threadIdx.x] = 0;
    carry_cnt[threadIdx.x] = 0;
  }
  __syncthreads();
  for (int base = 0; base < c.nsys_cap; base += blockDim.x) {
    const int s = base + threadIdx.x;
    int L = -1, cpt = 0;
    long long cost = 0;
    if (s < c.nsys_cap) {
      const SysParam *P = c.P + s;
      const SysState *S = c.S + s;
      const int f = S->flags;  // F_DONE of the last step is being cleared
      if (P->n > 0 && (f & F_ACTIVE)) {
        const long long nt = P->npad / TILE;
        const int rows = (int)((S->rows + nt / 2) / nt);  // mean list rows of a tile
        // atoms to threads by list length: the long-list class runs with
        // more threads per atom
        const int cls = (NL > 2 && rows >= c.rows_split) ? 1 : 0;
        L = ((f & (F_CU | F_CV)) ? 1 : 0) + 2 * cls;
        cpt = rows + TILE_OVH;
        cost = nt * cpt;
      }
    }
    // block-wide inclusive scans of (systems, cost) of every launch
    int n[NL];
    long long q[NL];
#pragma unroll
    for (int l = 0; l < NL; ++l) {
      n[l] = L == l;
      q[l] = L == l ? cost : 0;
    }
    for (int o = 1; o < 32; o <<= 1) {
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        const int y = __shfl_up_sync(0xffffffffu, n[l], o);
        const long long z = __shfl_up_sync(0xffffffffu, q[l], o);
        if (lane >= o) {
          n[l] += y;
          q[l] += z;
        }
      }
    }
    if (lane == 31) {
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        w_cnt[l][warp] = n[l];
        w_cost[l][warp] = q[l];
      }
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
      for (int l = 0; l < NL; ++l) {
        int a = lane < nw ? w_cnt[l][lane] : 0;
        long long b = lane < nw ? w_cost[l][lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, a, o);
          const long long z = __shfl_up_sync(0xffffffffu, b, o);
          if (lane >= o) {
            a += y;
            b += z;
          }
        }
        w_cnt[l][lane] = a;
        w_cost[l][lane] = b;
      }
    }
    __syncthreads();
    if (L >= 0) {
      int nl = 0;
      long long ql = 0;
#pragma unroll
      for (int l = 0; l < NL; ++l)
        if (l == L) {
          nl = n[l];
          ql = q[l];
        }
      const int k = carry_cnt[L] + (warp ? w_cnt[L][warp - 1] : 0) + nl - 1;
      const long long cum = carry_cost[L] + (warp ? w_cost[L][warp - 1] : 0) + ql - cost;
      c.plan[(size_t)L * c.nsys_cap + k] = PlanEnt{cum, s, cpt};
    }
    __syncthreads();
    if (threadIdx.x < NL) {
      carry_cnt[threadIdx.x] += w_cnt[threadIdx.x][nw - 1];
      carry_cost[threadIdx.x] += w_cost[threadIdx.x][nw - 1];
    }
    __syncthreads();
  }
  // block b of launch L starts in the entry whose cost range holds
  // lo_b = floor(b * tot / G): the blocks with cum * G <= b * tot < end * G
  for (int L = 0; L < NL; ++L) {
    const int m = carry_cnt[L], G = g[L];
    const long long tot = carry_cost[L];
    const PlanEnt *pl = c.plan + (size_t)L * c.nsys_cap;
    for (int k = threadIdx.x; k < m; k += blockDim.x) {
      const long long cum = pl[k].cum, end = k + 1 < m ? pl[k + 1].cum : tot;
      const long long b0 = (cum * G + tot - 1) / tot, b1 = (end * G + tot - 1) / tot;
      for (long long b = b0; b < b1 && b < G; ++b) c.plan_kb[L * PLAN_GMAX + b] = k;
    }
  }
  if (threadIdx.x < NL) {
    c.plan_hdr->tot[threadIdx.x] = carry_cost[threadIdx.x];
    c.plan_hdr->m[threadIdx.x] = carry_cnt[threadIdx.x];
  }
}

// integrate1, src/nd.f90:1027-1077 (both Nhold branches); applies velocity
// scales left pending by the previous step's mkIsoKE/mkIsoE first
// (src/nd.f90:1145-1155,1173-1180).
// Emits each chunk's two largest displacement measures for the next
// CheckListUpdate.  A dynamics step's launch has one more block (its first),
// which plans the step's pair launches.
// (six blocks per SM: the streaming body's registers; the planning block's
// scans may spill, one block of the launch)
__global__ __launch_bounds__(BLOCK, 6) void k_integrate1(DevCtx c, int standalone, int mixed,
                                                        int4 grids) {
  // a dynamics step's launch has one block more, its first, so that the
  // plan's serial scan runs beside the integration rather than after it
  const int lead = (!standalone && (int)gridDim.x > c.nchunks) ? 1 : 0;
  if (lead && blockIdx.x == 0) {
    const int g[PLAN_NL] = {grids.x, grids.y, grids.z, grids.w};
    if (c.rows_split > 0) plan_block<4>(c, g);
    else plan_block<2>(c, g);
    return;
  }
  const int chunk = blockIdx.x - lead;
  const int sys = c.chunk_sys[chunk];
  double t1 = 0.0, t2 = 0.0;
  if (sys >= 0) {
    const SysParam *__restrict__ P = c.P + sys;
    const SysState *S = c.S + sys;
    if (standalone || (S->flags & F_ACTIVE)) {
      const int i = chunk * ATOM_ALIGN + threadIdx.x;
      const int local = i - P->atom_off;
      if (local < P->n) {
        const double dt = P->dt;
        const double li0 = S->li[0], li1 = S->li[1], li2 = S->li[2];
        double *v = c.vel + 3 * (size_t)i;
        double *a = c.acc + 3 * (size_t)i;
        double *dl = c.disp + 3 * (size_t)i;
        double v0 = v[0], v1 = v[1], v2 = v[2];
        const int pend = standalone ? 0 : S->pend;
        if (pend) {
          if (pend & 1) { const double l = S->lam_ke; v0 = v0 * l; v1 = v1 * l; v2 = v2 * l; }
          if (pend & 2) { const double l = S->lam_e; v0 = v0 * l; v1 = v1 * l; v2 = v2 * l; }
          v[0] = v0; v[1] = v1; v[2] = v2;
        }
        const double a0 = a[0], a1 = a[1], a2 = a[2];
        double du0 = li0 * (v0 * dt + 0.5 * a0 * dt * dt);
        double du1 = li1 * (v1 * dt + 0.5 * a1 * dt * dt);
        double du2 = li2 * (v2 * dt + 0.5 * a2 * dt * dt);
        if (P->nhold > 0) {
          // displacement conditions of the atom's hold group replace the
          // constrained components (src/nd.f90:1058-1066)
          const int hg = c.hold[P->atom_off + c.gid[i]];
          if (hg > 0) {
            const double4 b = c.bcd[P->bc_off + hg - 1];
            const int m = (int)b.w;
            if (m & 1) du0 = b.x;
            if (m & 2) du1 = b.y;
            if (m & 4) du2 = b.z;
          }
        }
        const double d0 = dl[0] + du0, d1 = dl[1] + du1, d2 = dl[2] + du2;
        dl[0] = d0; dl[1] = d1; dl[2] = d2;
        double4 p = c.pos[i];
        p.x = p.x + du0;
        p.y = p.y + du1;
        p.z = p.z + du2;
        c.pos[i] = p;
        if (mixed) c.pfx[i] = make_int4(fx32(p.x), fx32(p.y), fx32(p.z), tw_of(p.w));
        if (P->quirk == 0) {
          double m = d0 * d0;
          m = m + d1 * d1;
          m = m + d2 * d2;
          t1 = m;
        } else {
          const double x = d0 * S->box[0], y = d1 * S->box[1], z = d2 * S->box[2];
          t1 = x * x + y * y + z * z;
        }
      }
    }
  }
  // this step's rebuild group is done with the rebuild list
  if (!standalone && chunk == 0 && threadIdx.x == 0) c.ring_count[3] = 0;
  // a new step: the system's pair kernel has not run yet (only the block of
  // the system's first chunk writes; the others read flag bits this leaves)
  if (!standalone && sys >= 0 && threadIdx.x == 0 && chunk == c.P[sys].atom_off / ATOM_ALIGN)
    c.S[sys].flags &= ~F_DONE;
  warp_top2(t1, t2);
  __shared__ double s1[BLOCK / 32], s2[BLOCK / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { s1[warp] = t1; s2[warp] = t2; }
  __syncthreads();
  if (warp == 0) {
    t1 = lane < BLOCK / 32 ? s1[lane] : 0.0;
    t2 = lane < BLOCK / 32 ? s2[lane] : 0.0;
    warp_top2(t1, t2);
    if (lane == 0) {
      c.itop[2 * chunk] = t1;
      c.itop[2 * chunk + 1] = t2;
    }
  }
}

// ---------------------------------------------------------------------------
// End-of-step epilogue for one system, run by the last block of the pair
// kernel to finish (dynamics, src/nd.f90:164-178 and the next step's head
// :138-151).
// The next step's list decision for a system (dynamics, src/nd.f90:138-151):
// CheckListUpdate every ReNeiFreq steps on the two largest displacement
// measures; in fixed semantics a rebuild also resizes the cell grid to stay
// at least rcut+skin wide.  A rebuilding system goes on the rebuild list
// and, inside a captured step block, switches on the next step's rebuild
// node.
__device__ void decide_rebuild(const DevCtx &c, int sys, const SysParam *P, SysState *S,
                               double t1, double t2, unsigned long long next_h) {
  int rb = 0;
  if (P->renei && S->step % P->renei_freq == 0) {
    rb = list_check(*P, *S, t1, t2);
    if (rb < 0) {
      set_err(c, S, E_OUT_OF_BOX);
      rb = 0;
    }
  }
  if (rb && P->quirk != 0) {
    int nc = 1;
    for (int d = 0; d < 3; ++d) {
      const int m = (int)(S->box[d] / P->rlist);
      S->mcell[d] = m < P->mcell0[d] ? m : P->mcell0[d];
      if (S->mcell[d] < 2) set_err(c, S, E_CELLS);
      nc *= S->mcell[d];
    }
    S->ncell = nc;
  }
  S->rebuild = rb;
  if (rb) c.rb_list[atomicAdd(c.ring_count + 3, 1)] = sys;
  if (rb && next_h) cudaGraphSetConditional((cudaGraphConditionalHandle)next_h, 1u);
}

// The tiles' partials are summed in an order that depends only on the tile
// index (the first FIN threads, whatever the block size): FP64 values by a
// fixed tree in `fs` (shared, NR rows of FIN doubles: the 7 energy/virial
// rows and the kinetic row in FP64, the kinetic row alone when mixed), the
// mixed path's fixed-point energy and virial exactly.
constexpr int FIN = 128;

template <bool MIXED>
__device__ void finalize_system(const DevCtx &c, int sys, int blk0, int nblk, int flags,
                                int fuse, unsigned long long next_h, double (*fs)[FIN]) {
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  constexpr int NR = MIXED ? 1 : 8, KR = NR - 1;
  __shared__ unsigned long long fq[7];
  const bool ev = flags & (F_CU | F_CV);
  if (threadIdx.x < 7) fq[threadIdx.x] = 0ull;
  __syncthreads();
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (threadIdx.x < FIN) {
    long long q[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < nblk; b += FIN) {
      const double *r = c.red + 8 * (size_t)(blk0 + b);
      if (ev) {
#pragma unroll
        for (int k = 0; k < 7; ++k) {
          if (MIXED) q[k] += __double_as_longlong(__ldcg(r + k));
          else v[k] += __ldcg(r + k);
        }
      }
      v[7] += __ldcg(r + 7);
    }
    if (!MIXED)
#pragma unroll
      for (int k = 0; k < 7; ++k) fs[k][threadIdx.x] = v[k];
    fs[KR][threadIdx.x] = v[7];
    if (MIXED && ev) {
#pragma unroll
      for (int k = 0; k < 7; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) q[k] += __shfl_xor_sync(0xffffffffu, q[k], o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&fq[k], (unsigned long long)q[k]);
      }
    }
  }
  __syncthreads();
#pragma unroll 1
  for (int sft = FIN / 2; sft > 0; sft >>= 1) {
    if ((int)threadIdx.x < sft)
      for (int k = 0; k < NR; ++k) fs[k][threadIdx.x] += fs[k][threadIdx.x + sft];
    __syncthreads();
  }
  if (!MIXED)
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = fs[k][0];
  v[7] = fs[KR][0];
  if (MIXED && ev)
#pragma unroll
    for (int k = 0; k < 7; ++k) v[k] = (double)(long long)fq[k] * (1.0 / FORCE_FX);
  // two largest displacement measures of this system (integrate1 partials)
  double t1 = 0.0, t2 = 0.0;
  if (fuse) {
    const int ch0 = P->atom_off / ATOM_ALIGN, nch = P->npad / ATOM_ALIGN;
    for (int q = threadIdx.x; q < nch; q += blockDim.x)
      top2_merge(t1, t2, __ldcg(c.itop + 2 * (ch0 + q)), __ldcg(c.itop + 2 * (ch0 + q) + 1));
    warp_top2(t1, t2);
    __shared__ double s1[32], s2[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) { s1[warp] = t1; s2[warp] = t2; }
    __syncthreads();
    if (warp == 0) {
      t1 = lane < (int)(blockDim.x >> 5) ? s1[lane] : 0.0;
      t2 = lane < (int)(blockDim.x >> 5) ? s2[lane] : 0.0;
      warp_top2(t1, t2);
    }
  }
  if (threadIdx.x != 0) return;
  // the pair loop visits each pair from both atoms: halve PE and virial
  if (flags & F_CU) S->potential = 0.5 * v[0];
  if (flags & F_CV)
    for (int k = 0; k < 6; ++k) S->virial[k] = 0.5 * v[1 + k];
  if (!fuse) return;
  S->kinetic = (flags & F_CK) ? v[7] * 0.5 : 0.0;  // integrate2, src/nd.f90:1119
  if (flags & F_FIRST) S->e0 = S->potential + S->kinetic;
  if (flags & F_OUT) {
    const int idx = atomicAdd(c.ring_count, 1);
    if (idx < c.ring_cap)
      make_thermo(c.ring[idx], sys, S->step, S->potential, S->kinetic, S->e0, S->virial, S->box);
  }
  int pend = 0;
  if (flags & F_KE_SCALE) {
    S->lam_ke = lam_iso_ke(*P, S->kinetic, P->n);
    pend |= 1;
  }
  if (flags & F_P_SCALE) iso_p_box(*P, S->virial, S->box);
  if (flags & F_E_SCALE) {
    S->lam_e = lam_iso_e(*P, S->e0, S->potential, S->kinetic);
    pend |= 2;
  }
  if (P->box_load)
    for (int d = 0; d < 3; ++d) S->box[d] = S->box[d] + P->box_vel[d] * P->dt;
  for (int d = 0; d < 3; ++d) S->li[d] = 1.0 / S->box[d];
  S->pend = pend;
  S->dtop[0] = t1;
  S->dtop[1] = t2;
  S->steps_left -= 1;
  if (S->steps_left > 0) {
    S->step += 1;
    S->tt += 1;
    // F_DONE keeps the step's second pair kernel (the other energy/virial
    // variant) from taking this system again under the next step's flags
    S->flags = step_flags(*P, S->step, S->tt) | F_ACTIVE | F_DONE;
    decide_rebuild(c, sys, P, S, t1, t2, next_h);
  } else {
    S->flags = 0;
    S->rebuild = 0;
  }
}

// ---------------------------------------------------------------------------
// integrate2(CK) on its own (src/nd.f90:1081-1121), reading force(3,np).
__global__ __launch_bounds__(BLOCK) void k_integrate2(DevCtx c, int ck) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0) return;
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  if (P->n == 0) return;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  double ke = 0.0;
  if (i - P->atom_off < P->n) {
    const int t = tw_type(tw_of(c.pos[i].w));
    const double m = c.mass[P->type_off + t - 1];
    const double rmass = 1.0 / m, dt = P->dt;
    double *v = c.vel + 3 * (size_t)i;
    double *a = c.acc + 3 * (size_t)i;
    const double *f = c.force + 3 * (size_t)i;
    for (int d = 0; d < 3; ++d) v[d] = v[d] + 0.5 * dt * (f[d] * rmass + a[d]);
    for (int d = 0; d < 3; ++d) a[d] = f[d] * rmass;
    if (ck) {
      double kt = v[0] * v[0];
      kt = kt + v[1] * v[1];
      kt = kt + v[2] * v[2];
      ke = kt * m;
    }
  }
  __shared__ double sm[32];
  double r[1] = {ke};
  block_sum<1>(r, sm);
  __shared__ int last;
  if (threadIdx.x == 0) {
    c.ired[chunk] = r[0];
    __threadfence();
    const unsigned t = atomicAdd(&S->ticket_i, 1u);
    last = (t == (unsigned)(P->npad / ATOM_ALIGN) - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    const int ch0 = P->atom_off / ATOM_ALIGN, nch = P->npad / ATOM_ALIGN;
    double v[1] = {0.0};
    for (int q = threadIdx.x; q < nch; q += blockDim.x) v[0] += __ldcg(c.ired + ch0 + q);
    block_sum<1>(v, sm);
    if (threadIdx.x == 0) {
      S->kinetic = ck ? v[0] * 0.5 : 0.0;
      S->ticket_i = 0;
    }
  }
}

// ---------------------------------------------------------------------------
// run bookkeeping
// give every system (sys < 0) or one system a run of nsteps starting as
// `start` (START_*)
__global__ void k_arm(DevCtx c, int nsys_cap, int sys, int nsteps, int start) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys_cap || (sys >= 0 && s != sys) || c.P[s].n == 0) return;
  c.S[s].run_left = nsteps;
  c.S[s].start = start;
}

// Head of a block of up to K steps: each system with steps left in its run
// takes min(K, left) of them.  A new run starts at tt = 1 (write_thermo and
// e0 on its first step, src/nd.f90:139-148,167); a continued run takes the
// step the previous block's last epilogue left off, with the same list
// decision (dynamics, src/nd.f90:138-151).
__global__ void k_begin_block(DevCtx c, int nsys_cap, int K) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys_cap) return;
  const SysParam &P = c.P[s];
  SysState &S = c.S[s];
  S.ticket = 0;
  S.ticket_i = 0;
  if (P.n == 0 || S.run_left <= 0) {
    S.flags = 0;
    S.steps_left = 0;
    S.rebuild = 0;
    return;
  }
  const int k = S.run_left < K ? S.run_left : K;
  S.run_left -= k;
  S.steps_left = k;
  const int start = S.start;
  S.start = START_CONTINUE;
  S.tt = start == START_CONTINUE ? S.tt + 1 : 1;
  S.step = S.step + 1;
  S.flags = step_flags(P, S.step, S.tt) | F_ACTIVE;
  for (int d = 0; d < 3; ++d) S.li[d] = 1.0 / S.box[d];
  if (start == START_BUILT) S.rebuild = 0;
  else decide_rebuild(c, s, &P, &S, S.dtop[0], S.dtop[1], 0ull);
}

// apply pending mkIsoKE/mkIsoE velocity scales at the end of a run
__global__ __launch_bounds__(BLOCK) void k_flush(DevCtx c, int only, int chunk0) {
  const int chunk = chunk0 + blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0 || (only >= 0 && sys != only)) return;
  const SysParam *__restrict__ P = c.P + sys;
  const SysState *S = c.S + sys;
  const int pend = S->pend;
  if (!pend) return;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  double *v = c.vel + 3 * (size_t)i;
  for (int d = 0; d < 3; ++d) {
    double x = v[d];
    if (pend & 1) x = x * S->lam_ke;
    if (pend & 2) x = x * S->lam_e;
    v[d] = x;
  }
}

__global__ void k_clear_pend(DevCtx c, int nsys_cap, int sys) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys_cap && (sys < 0 || s == sys)) c.S[s].pend = 0;
}

__global__ __launch_bounds__(BLOCK) void k_scale_vel(DevCtx c, int sys, double lam) {
  const int chunk = blockIdx.x;
  if (c.chunk_sys[chunk] != sys) return;
  const SysParam *__restrict__ P = c.P + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  double *v = c.vel + 3 * (size_t)i;
  v[0] = v[0] * lam;
  v[1] = v[1] * lam;
  v[2] = v[2] * lam;
}

__global__ __launch_bounds__(BLOCK) void k_refresh_pfx(DevCtx c) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0) return;
  const SysParam *__restrict__ P = c.P + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  const double4 p = c.pos[i];
  c.pfx[i] = make_int4(fx32(p.x), fx32(p.y), fx32(p.z), tw_of(p.w));
}

// CheckListUpdate called on its own (src/nd.f90:1447-1499): one block per
// system reduces the integrate1 displacement partials.
__global__ void k_check(DevCtx c, int nsys_cap) {
  const int s = blockIdx.x;
  if (s >= nsys_cap) return;
  const SysParam *__restrict__ P = c.P + s;
  SysState *S = c.S + s;
  if (P->n == 0) return;
  double t1 = 0.0, t2 = 0.0;
  const int ch0 = P->atom_off / ATOM_ALIGN, nch = P->npad / ATOM_ALIGN;
  for (int q = threadIdx.x; q < nch; q += blockDim.x)
    top2_merge(t1, t2, c.itop[2 * (ch0 + q)], c.itop[2 * (ch0 + q) + 1]);
  warp_top2(t1, t2);
  __shared__ double s1[32], s2[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) { s1[warp] = t1; s2[warp] = t2; }
  __syncthreads();
  if (threadIdx.x >= 32) return;
  t1 = lane < (int)(blockDim.x >> 5) ? s1[lane] : 0.0;
  t2 = lane < (int)(blockDim.x >> 5) ? s2[lane] : 0.0;
  warp_top2(t1, t2);
  if (lane != 0) return;
  S->dtop[0] = t1;
  S->dtop[1] = t2;
  int rb = list_check(*P, *S, t1, t2);
  if (rb < 0) {
    set_err(c, S, E_OUT_OF_BOX);
    rb = 0;
  }
  if (rb && P->quirk != 0) {
    int nc = 1;
    for (int d = 0; d < 3; ++d) {
      int m = (int)(S->box[d] / P->rlist);
      S->mcell[d] = m < P->mcell0[d] ? m : P->mcell0[d];
      if (S->mcell[d] < 2) set_err(c, S, E_CELLS);
      nc *= S->mcell[d];
    }
    S->ncell = nc;
  }
  S->rebuild = rb;
  if (rb) c.rb_list[atomicAdd(c.ring_count + 3, 1)] = s;
}

// ---------------------------------------------------------------------------
// List rebuild: buildCellList + buildVerletList (src/nd.f90:1214-1446).
//
// Only the systems on the rebuild list are touched.  The per-system epilogue
// (or k_check / k_begin_run) appends a system when its CheckListUpdate
// fires, and the setup paths list every system.  Each rebuild kernel runs a
// small persistent grid: the listed systems' units (256-atom chunks,
// 128-atom tiles, groups of cells) form one sequence dealt round-robin to
// the blocks, so a step in which a few of many replicas rebuild costs a few
// replicas' worth of work.  k_integrate1 empties the list afterwards.

constexpr int LIST_STAGE = 256;  // listed systems whose ranges a block stages at once

template <class Range, class Body>
__device__ __forceinline__ void for_listed(const DevCtx &c, Range range, Body body) {
  // the listed systems' unit ranges, loaded in parallel into shared memory
  __shared__ int l_sys[LIST_STAGE], l_first[LIST_STAGE], l_cnt[LIST_STAGE];
  const int n = c.ring_count[3];
  const int G = gridDim.x, b = blockIdx.x;
  long long base = 0;
  for (int k0 = 0; k0 < n; k0 += LIST_STAGE) {
    const int m = min(LIST_STAGE, n - k0);
    __syncthreads();  // the previous group's entries are no longer read
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
      const int sys = c.rb_list[k0 + t];
      int first = 0, cnt = 0;
      range(sys, first, cnt);
      l_sys[t] = sys;
      l_first[t] = first;
      l_cnt[t] = cnt;
    }
    __syncthreads();
    for (int k = 0; k < m; ++k) {
      const int sys = l_sys[k], first = l_first[k], cnt = l_cnt[k];
      for (int q = (int)(((long long)b - base % G + G) % G); q < cnt; q += G) body(sys, first + q);
      base += cnt;
    }
  }
}

__device__ __forceinline__ void chunk_range(const DevCtx &c, int sys, int &first, int &cnt) {
  first = c.P[sys].atom_off / ATOM_ALIGN;
  cnt = c.P[sys].npad / ATOM_ALIGN;
}

// link cell of each atom, src/nd.f90:1237-1248, counted with warp-aggregated
// atomics (lanes with the same cell elect one atomicAdd)
__device__ void bin_chunk(const DevCtx &c, int sys, int chunk) {
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  const int local = i - P->atom_off;
  int cell = -1;
  if (local < P->n) {
    const double4 p = c.pos[i];
    const double q[3] = {p.x, p.y, p.z};
    int ix[3];
    bool bad = false;
    for (int d = 0; d < 3; ++d) {
      const double sr = q[d] - round(q[d]);
      const double t = (sr + 0.4999) * (double)S->mcell[d];
      ix[d] = (int)t;
      bad |= !(t == t) || ix[d] < 0 || ix[d] >= S->mcell[d];
    }
    if (bad) {
      // keep the atom counted (in cell 0) so the permutation stays complete;
      // the run stops with 'Particle outside of box' after this step
      set_err(c, S, E_OUT_OF_BOX);
      cell = 0;
    } else {
      cell = ix[0] + ix[1] * S->mcell[0] + ix[2] * S->mcell[0] * S->mcell[1];
    }
    c.atom_cell[i] = cell;
  }
  const unsigned grp = __match_any_sync(0xffffffffu, cell);
  const int lane = threadIdx.x & 31;
  const int leader = __ffs(grp) - 1;
  const int rank = __popc(grp & ((1u << lane) - 1u));
  int base = 0;
  if (cell >= 0 && lane == leader) base = atomicAdd(c.cell_count + P->cell_off + cell, __popc(grp));
  base = __shfl_sync(0xffffffffu, base, leader);
  if (local < P->n) c.atom_slot[i] = cell >= 0 ? base + rank : 0;
}

__global__ __launch_bounds__(BLOCK) void k_bin(DevCtx c) {
  if (blockIdx.x == 0 && threadIdx.x == 0) c.ring_count[2] = 0;  // k_scan counts the cells
  for_listed(c, [&](int s, int &f, int &n) { chunk_range(c, s, f, n); },
             [&](int s, int u) { bin_chunk(c, s, u); });
}

// exclusive scan of one system's cell counts (a whole block)
__device__ void scan_system(const DevCtx &c, int s, int counting) {
  const SysParam *__restrict__ P = c.P + s;
  SysState *S = c.S + s;
  __shared__ int wsum[32];
  __shared__ int carry;
  if (threadIdx.x == 0) {
    carry = 0;
    S->rows = 0;  // the build that follows sums its tiles' rows
  }
  __syncthreads();
  const int ncell = S->ncell;
  int *cnt = c.cell_count + P->cell_off;
  int *start = c.cell_start + P->cell_off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int base = 0; base < ncell; base += blockDim.x) {
    const int idx = base + threadIdx.x;
    const int x = idx < ncell ? cnt[idx] : 0;
    int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
      int w = lane < (int)(blockDim.x >> 5) ? wsum[lane] : 0;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      wsum[lane] = w;
    }
    __syncthreads();
    const int wpre = warp ? wsum[warp - 1] : 0;
    if (idx < ncell) {
      start[idx] = carry + wpre + incl - x;
      cnt[idx] = 0;
    }
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += wpre + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    start[ncell] = carry;
    S->nstencil = make_stencil(S->mcell, P->quirk, S->stencil);
    for (int d = 0; d < 3; ++d) S->box_build[d] = S->box[d];
    if (counting) S->nlist_updates += 1;  // NlistUpdates, src/nd.f90:1495
    atomicAdd(c.ring_count + 2, ncell);  // the build chooses its form by the cells listed
  }
}

// exclusive scan of the cell counts, one listed system at a time per block
__global__ __launch_bounds__(1024) void k_scan(DevCtx c, int counting) {
  const int nl = c.ring_count[3];
  for (int k = blockIdx.x; k < nl; k += gridDim.x) {
    scan_system(c, c.rb_list[k], counting);
    __syncthreads();  // carry and wsum are reused by the next system
  }
}

__device__ void scatter_chunk(const DevCtx &c, int sys, int chunk) {
  const SysParam *__restrict__ P = c.P + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  const int dest = c.cell_start[P->cell_off + c.atom_cell[i]] + c.atom_slot[i];
  c.tmp_src[P->atom_off + dest] = i;
  c.tmp_key[P->atom_off + dest] = c.gid[i];
}

__global__ __launch_bounds__(BLOCK) void k_scatter(DevCtx c) {
  for_listed(c, [&](int s, int &f, int &n) { chunk_range(c, s, f, n); },
             [&](int s, int u) { scatter_chunk(c, s, u); });
}

// order the atoms of each cell by original id (one warp per cell) so the
// layout, and the neighbour order, do not depend on atomic timing
__device__ void order_cell(const DevCtx &c, int sys, int cl) {
  const SysParam *__restrict__ P = c.P + sys;
  if (cl >= c.S[sys].ncell) return;
  const int s0 = c.cell_start[P->cell_off + cl], s1 = c.cell_start[P->cell_off + cl + 1];
  const int *key = c.tmp_key + P->atom_off + s0;
  const int *src = c.tmp_src + P->atom_off + s0;
  const int m = s1 - s0;
  for (int e = threadIdx.x & 31; e < m; e += 32) {
    const int k = key[e];
    int rank = 0;
    for (int q = 0; q < m; ++q) rank += key[q] < k;
    c.perm[P->atom_off + s0 + rank] = src[e];
  }
}

__global__ __launch_bounds__(BLOCK) void k_order(DevCtx c) {
  constexpr int W = BLOCK / 32;
  for_listed(c,
             [&](int s, int &f, int &n) {
               f = 0;
               n = (c.S[s].ncell + W - 1) / W;
             },
             [&](int s, int u) { order_cell(c, s, u * W + (threadIdx.x >> 5)); });
}

__device__ void permute_chunk(const DevCtx &c, int sys, int chunk) {
  const SysParam *__restrict__ P = c.P + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  int s = c.perm[i];
  if (s < P->atom_off || s >= P->atom_off + P->n) {
    set_err(c, c.S + sys, E_OUT_OF_BOX);
    s = i;
  }
  c.s_pos[i] = c.pos[s];
  for (int d = 0; d < 3; ++d) {
    c.s_vel[3 * (size_t)i + d] = c.vel[3 * (size_t)s + d];
    c.s_acc[3 * (size_t)i + d] = c.acc[3 * (size_t)s + d];
  }
  c.s_gid[i] = c.gid[s];
  c.s_cell[i] = c.atom_cell[s];
}

__global__ __launch_bounds__(BLOCK) void k_permute(DevCtx c) {
  for_listed(c, [&](int s, int &f, int &n) { chunk_range(c, s, f, n); },
             [&](int s, int u) { permute_chunk(c, s, u); });
}

__device__ void copyback_chunk(const DevCtx &c, int sys, int chunk, int mixed) {
  const SysParam *__restrict__ P = c.P + sys;
  if (threadIdx.x == 0) {
    c.itop[2 * chunk] = 0.0;  // dispList was reset: the displacement measure is 0
    c.itop[2 * chunk + 1] = 0.0;
  }
  if (threadIdx.x < ATOM_ALIGN / TILE) c.tile_rows[chunk * (ATOM_ALIGN / TILE) + threadIdx.x] = 0;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  const double4 p = c.s_pos[i];
  c.pos[i] = p;
  // the fixed-point positions the list build (and the mixed pair loop) read
  c.pfx[i] = make_int4(fx32(p.x), fx32(p.y), fx32(p.z), tw_of(p.w));
  (void)mixed;
  for (int d = 0; d < 3; ++d) {
    c.vel[3 * (size_t)i + d] = c.s_vel[3 * (size_t)i + d];
    c.acc[3 * (size_t)i + d] = c.s_acc[3 * (size_t)i + d];
    c.disp[3 * (size_t)i + d] = 0.0;  // src/nd.f90:1384,1427
  }
  c.gid[i] = c.s_gid[i];
  const int cl = c.s_cell[i];
  c.atom_cell[i] = cl;
  // the cell's grid coordinates, once per atom here rather than by every
  // stencil lane of the list build (grids above 2047 x 2047 x 1023 cells
  // leave them to the build)
  const SysState *S = c.S + sys;
  const int M0 = S->mcell[0], M1 = S->mcell[1];
  c.cxyz[i] = (cl % M0) | (((cl / M0) % M1) << 11) | ((cl / (M0 * M1)) << 22);
}

__global__ __launch_bounds__(BLOCK) void k_copyback(DevCtx c, int mixed) {
  for_listed(c, [&](int s, int &f, int &n) { chunk_range(c, s, f, n); },
             [&](int s, int u) { copyback_chunk(c, s, u, mixed); });
}

// Neighbour build (buildVerletList, src/nd.f90:1328-1446).  An FP32
// distance on the 32-bit fixed-point positions decides every candidate
// farther than a 1e-5 relative margin from the list radius (and from PTrMin
// in the atom's own cell); candidates inside the margin take the
// reference's exact FP64 test, so membership is bit-identical to the
// reference's.  Every atom's list holds its hits in stencil order, then
// cell order.  Two forms share this test: a warp per atom (k_build_atoms,
// rebuilds of few atoms: a step's few replicas) and a warp per link cell
// (k_build_cells, many cells: a prologue, a large system); the number of
// listed cells, counted by k_scan, picks one on the device.
constexpr float NB_MARGIN = 1e-5f;
constexpr int CELL_BUILD_MIN = 16384;  // listed cells from which the cell form builds

// exclusive prefix sum of one int per thread over the whole block, in
// thread order (wsum: one int per warp of shared scratch)
__device__ __forceinline__ int block_excl_scan(int v, int *wsum) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int incl = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += y;
  }
  __syncthreads();  // wsum free for reuse
  if (lane == 31) wsum[warp] = incl;
  __syncthreads();
  int before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  return before + incl - v;
}

// ---------------------------------------------------------------------------
// Neighbour build by link cell (buildVerletList, src/nd.f90:1328-1446): one
// warp per cell of a listed system, one lane per atom of the cell (32 at a
// time).  The candidates of the cell's stencil entries pass the warp one
// after another, in stencil order and, within a cell, in cell order; every
// lane tests each against its own atom and appends the hits to its own
// column of the blocked list.  Each list thus has the order of the
// reference's cell walk (stencil entry, then cell order), and the candidate
// test is the shared one above: FP32 on the fixed-point positions outside a
// 1e-5 band around the list radius and PTrMin, the reference's FP64 test
// inside it.  A candidate costs the warp one broadcast load and one test
// for all 32 atoms of the cell at once.
constexpr int CB_THREADS = 256;

__device__ __forceinline__ int wrap_step(int x, int d, int M) {
  const int y = x + d;  // d in {-1, 0, 1}, x in [0, M)
  return y < 0 ? y + M : (y >= M ? y - M : y);
}

template <bool B>
struct BoolTag {
  static constexpr bool value = B;
};

// Stencil entries whose candidate ranges follow one another in memory (an
// entry's first candidate right after the previous entry's last: the cells
// of one row of the stencil, or a left-out or empty range between them)
// pass as one range: the same candidates in the same order, in fuller
// batches of 32.  The own cell, the one entry that tests PTrMin, stays a
// range of its own.  Lane e < ne holds entry e; bit e of the result marks
// the first entry of a range, which runs to the entry before the next mark.
__device__ __forceinline__ unsigned range_heads(int q0, int q1, int center, int lane, int ne) {
  const int pq1 = __shfl_up_sync(0xffffffffu, q1, 1);
  const int pcen = __shfl_up_sync(0xffffffffu, center, 1);
  return __ballot_sync(0xffffffffu, lane < ne && (lane == 0 || center || pcen || q0 != pq1));
}

__device__ __forceinline__ void build_cell(const DevCtx &c, int sys, int cell, int lane) {
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  const int *cst = c.cell_start + P->cell_off;
  const int o0 = cst[cell], o1 = cst[cell + 1];
  if (o0 >= o1) return;
  const int M0 = S->mcell[0], M1 = S->mcell[1], M2 = S->mcell[2];
  const int ne = S->nstencil;
  // lane e < ne holds stencil entry e: its cell's candidate range and
  // whether it is the own cell
  int e_q0 = 0, e_q1 = 0, e_center = 0;
  if (lane < ne) {
    const int cx = cell % M0, cy = (cell / M0) % M1, cz = cell / (M0 * M1);
    const int st = S->stencil[lane];
    const int nc = wrap_step(cx, (st & 15) - 1, M0) +
                   (wrap_step(cy, ((st >> 4) & 15) - 1, M1) +
                    wrap_step(cz, ((st >> 8) & 15) - 1, M2) * M1) * M0;
    e_q0 = cst[nc];
    e_q1 = cst[nc + 1];
    e_center = (st >> 12) & 1;
  }
  const unsigned heads = range_heads(e_q0, e_q1, e_center, lane, ne);
  const int aoff = P->atom_off, nt = P->ntypes, maxnb = P->maxnb, nb16 = P->nb16;
  const int *pm = c.pairmat + P->pm_off;
  const double *rl2 = c.rlist2 + P->pair_off;
  const float sb0 = (float)(S->box[0] * (1.0 / FX_ONE)), sb1 = (float)(S->box[1] * (1.0 / FX_ONE)),
              sb2 = (float)(S->box[2] * (1.0 / FX_ONE));
  const float ptrlo = (float)P->ptrmin * (1.f - NB_MARGIN),
              ptrhi = (float)P->ptrmin * (1.f + NB_MARGIN);
  const bool one = nt == 1 && P->npairs == 1 && pm[0] == 1;
  const float rf1 = (float)rl2[0];
  const float2 band1 = make_float2(rf1 * (1.f - NB_MARGIN), rf1 * (1.f + NB_MARGIN));
  // a candidate farther than the list radius from the box of the warp's own
  // atoms cannot be a neighbour of any of them; the box is kept as offsets
  // from the first own atom, whose wrap-around differences are minimum
  // images on grids of five or more cells per axis
  const bool prune = M0 >= 5 && M1 >= 5 && M2 >= 5;
  const float rlbox = (float)(P->rlist * P->rlist) * (1.f + 4.f * NB_MARGIN);
  for (int g0 = o0; g0 < o1; g0 += 32) {
    const int li = g0 + lane;  // the lane's own atom (local slot)
    const bool own = li < o1;
    const int i = aoff + (own ? li : o0);
    const int4 pi = c.pfx[i];
    const int ti = tw_type(pi.w);
    const int ax = __shfl_sync(0xffffffffu, pi.x, 0), ay = __shfl_sync(0xffffffffu, pi.y, 0),
              az = __shfl_sync(0xffffffffu, pi.z, 0);
    const int ox = (int)((unsigned)pi.x - (unsigned)ax), oy = (int)((unsigned)pi.y - (unsigned)ay),
              oz = (int)((unsigned)pi.z - (unsigned)az);
    const int lx = __reduce_min_sync(0xffffffffu, own ? ox : INT_MAX),
              hx = __reduce_max_sync(0xffffffffu, own ? ox : INT_MIN),
              ly = __reduce_min_sync(0xffffffffu, own ? oy : INT_MAX),
              hy = __reduce_max_sync(0xffffffffu, own ? oy : INT_MIN),
              lz = __reduce_min_sync(0xffffffffu, own ? oz : INT_MAX),
              hz = __reduce_max_sync(0xffffffffu, own ? oz : INT_MIN);
    int *col = c.nbr + P->nbr_off + (long long)(li / TILE) * maxnb * TILE + (li % TILE);
    int cnt = 0;
    // one pass of 32 candidates [qb, qb + 32) of a range ending at q1; only
    // the own cell (CEN) tests PTrMin and holds the own atoms, and a system
    // of one type and one pair (ONE) takes no pair-matrix lookup
    auto pass = [&](auto cen, auto onet, int qb, int q1) {
      constexpr bool CEN = decltype(cen)::value, ONE = decltype(onet)::value;
      // 32 candidates at once, one per lane; the lanes test their own
      // candidate against the own atoms' box, then the kept ones pass
      // the warp in cell order
      const int qq = qb + lane;
      const bool have = qq < q1;
      const int4 pc = c.pfx[aoff + (have ? qq : qb)];
      bool keep = have;
      if (prune && keep) {
        const int dx = (int)((unsigned)pc.x - (unsigned)ax), dy = (int)((unsigned)pc.y - (unsigned)ay),
                  dz = (int)((unsigned)pc.z - (unsigned)az);
        const float gx = dx < lx ? (float)lx - (float)dx : (dx > hx ? (float)dx - (float)hx : 0.f);
        const float gy = dy < ly ? (float)ly - (float)dy : (dy > hy ? (float)dy - (float)hy : 0.f);
        const float gz = dz < lz ? (float)lz - (float)dz : (dz > hz ? (float)dz - (float)hz : 0.f);
        const float d2b = (gx * sb0) * (gx * sb0) + (gy * sb1) * (gy * sb1) + (gz * sb2) * (gz * sb2);
        keep = d2b <= rlbox;
      }
      unsigned m = __ballot_sync(0xffffffffu, keep);
      while (m) {
        const int k = __ffs(m) - 1;
        m &= m - 1;
        const int4 pj = make_int4(__shfl_sync(0xffffffffu, pc.x, k), __shfl_sync(0xffffffffu, pc.y, k),
                                  __shfl_sync(0xffffffffu, pc.z, k), __shfl_sync(0xffffffffu, pc.w, k));
        const int j = aoff + qb + k;
        int mx = 1;
        if (!ONE) {
          const int tj = tw_type(pj.w);
          const int a = pm[(ti - 1) + (tj - 1) * nt], b = pm[(tj - 1) + (ti - 1) * nt];
          mx = a > b ? a : b;
        }
        const float r0 = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * sb0;
        const float r1 = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * sb1;
        const float r2 = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * sb2;
        const float d2f = r0 * r0 + r1 * r1 + r2 * r2;
        const bool live = own && (!CEN || j != i) && (ONE || mx > 0);
        float2 band = band1;
        if (!ONE && live) {
          const float rf = (float)rl2[mx - 1];
          band = make_float2(rf * (1.f - NB_MARGIN), rf * (1.f + NB_MARGIN));
        }
        // outside both margins FP32 decides; inside either, FP64 does
        bool hit = live && d2f < band.x && !(CEN && d2f < ptrhi);
        const bool unsure = live && ((d2f >= band.x && d2f <= band.y) ||
                                     (CEN && d2f >= ptrlo && d2f <= ptrhi));
        if (unsure) {
          // the reference's FP64 test (src/nd.f90:1362-1377, 1419-1420),
          // its operands read again on this rare path
          const double4 pid = c.pos[i], pjd = c.pos[j];
          double s0 = pid.x - pjd.x, s1 = pid.y - pjd.y, s2 = pid.z - pjd.z;
          s0 = s0 - round(s0);
          s1 = s1 - round(s1);
          s2 = s2 - round(s2);
          const double x0 = S->box[0] * s0, x1 = S->box[1] * s1, x2 = S->box[2] * s2;
          double d2 = x0 * x0;
          d2 = d2 + x1 * x1;
          d2 = d2 + x2 * x2;
          hit = !(CEN && d2 < P->ptrmin) && !(d2 > rl2[mx - 1]);
        }
        if (hit) {
          if (cnt < maxnb) list_store(col, nb16, aoff, cnt, j);
          ++cnt;
        }
      }
    };
    auto ranges = [&](auto onet) {
      for (unsigned hd = heads; hd;) {
        const int e = __ffs(hd) - 1;
        hd &= hd - 1;
        const int last = hd ? __ffs(hd) - 2 : ne - 1;
        const bool center = __shfl_sync(0xffffffffu, e_center, e) != 0;
        const int q0 = __shfl_sync(0xffffffffu, e_q0, e), q1 = __shfl_sync(0xffffffffu, e_q1, last);
        if (center)
          for (int qb = q0; qb < q1; qb += 32) pass(BoolTag<true>{}, onet, qb, q1);
        else
          for (int qb = q0; qb < q1; qb += 32) pass(BoolTag<false>{}, onet, qb, q1);
      }
    };
    if (one)
      ranges(BoolTag<true>{});
    else
      ranges(BoolTag<false>{});
    if (own) {
      c.nnb[aoff + li] = cnt;
      if (cnt > maxnb) set_err(c, S, E_NEIMAX);
      note_rows(c, S, aoff + li, min(cnt, maxnb));
    }
  }
}

// Neighbour build by atom, for rebuilds of few atoms (a step's rebuilds of
// a few replicas): one warp per own atom, 32 candidates of a stencil cell at
// a time (one coalesced load of their fixed-point positions, a lane each),
// hits compacted with __ballot_sync/__popc into the atom's column in
// stencil order, then cell order, the order of the other two forms.  No
// shared staging and no barriers, so every warp of the grid works on its
// own atom; the test is theirs (FP32 outside the 1e-5 band, the
// reference's FP64 test inside it).
__device__ __forceinline__ void build_atom(const DevCtx &c, int sys, int local, int lane) {
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  const int aoff = P->atom_off, i = aoff + local;
  const int *cst = c.cell_start + P->cell_off;
  const int ne = S->nstencil;
  const int4 pi = c.pfx[i];
  int e_q0 = 0, e_q1 = 0, e_center = 0;  // lane e < ne: stencil entry e
  if (lane < ne) {
    const int M[3] = {S->mcell[0], S->mcell[1], S->mcell[2]};
    int cv[3];
    if (M[0] < 2048 && M[1] < 2048 && M[2] < 1024) {
      const int w = c.cxyz[i];
      cv[0] = w & 2047;
      cv[1] = (w >> 11) & 2047;
      cv[2] = (unsigned)w >> 22;
    } else {
      const int cl = c.atom_cell[i];
      cv[0] = cl % M[0];
      cv[1] = (cl / M[0]) % M[1];
      cv[2] = cl / (M[0] * M[1]);
    }
    const int st = S->stencil[lane];
    int nv[3];
    for (int d = 0; d < 3; ++d) nv[d] = wrap_step(cv[d], ((st >> (4 * d)) & 15) - 1, M[d]);
    const int nc = nv[0] + (nv[1] + nv[2] * M[1]) * M[0];
    e_q0 = cst[nc];
    e_q1 = cst[nc + 1];
    e_center = (st >> 12) & 1;
    // A stencil cell no part of which lies within the list radius of this
    // atom holds none of its neighbours: its range is left out.  Cell n
    // of an axis holds the fractional coordinates sr (sr = x - anint(x))
    // with int((sr + 0.4999) M) = n (src/nd.f90:1243-1245), an interval
    // widened here by 2e-4 of the box; the distance to it is taken on the
    // periodic axis (from the interval's middle, minimum image).  A
    // prefilter only, so FP32 serves: its rounding is ~1e-7 of the box,
    // far inside the widening.
    const int pq[3] = {pi.x, pi.y, pi.z};
    float d2min = 0.f;
    for (int d = 0; d < 3; ++d) {
      const float im = __fdividef(1.0f, (float)M[d]);
      const float lo = (nv[d] == 0 ? -0.5f : (float)nv[d] * im - 0.4999f) - 2e-4f;
      const float hi = (float)(nv[d] + 1) * im - 0.4999f + 2e-4f;
      const float q = (float)pq[d] * (1.0f / 4294967296.0f);
      float dm = q - 0.5f * (lo + hi);
      dm = dm - rintf(dm);
      const float gap = fmaxf(fabsf(dm) - 0.5f * (hi - lo), 0.f) * (float)S->box[d];
      d2min = __fmaf_rn(gap, gap, d2min);
    }
    if (d2min > (float)(P->rlist * P->rlist) * (1.f + 1e-5f)) e_q1 = e_q0;
  }
  const unsigned heads = range_heads(e_q0, e_q1, e_center, lane, ne);
  const int nt = P->ntypes, maxnb = P->maxnb, nb16 = P->nb16;
  const int *pm = c.pairmat + P->pm_off;
  const double *rl2 = c.rlist2 + P->pair_off;
  const float sb0 = (float)(S->box[0] * (1.0 / FX_ONE)), sb1 = (float)(S->box[1] * (1.0 / FX_ONE)),
              sb2 = (float)(S->box[2] * (1.0 / FX_ONE));
  const float ptrlo = (float)P->ptrmin * (1.f - NB_MARGIN),
              ptrhi = (float)P->ptrmin * (1.f + NB_MARGIN);
  const bool one = nt == 1 && P->npairs == 1 && pm[0] == 1;
  const float rf1 = (float)rl2[0];
  const float2 band1 = make_float2(rf1 * (1.f - NB_MARGIN), rf1 * (1.f + NB_MARGIN));
  const int ti = tw_type(pi.w);
  int *col = c.nbr + P->nbr_off + (long long)(local / TILE) * maxnb * TILE + (local % TILE);
  const unsigned below = (1u << lane) - 1u;
  int cnt = 0;
  // one pass of 32 candidates [qb, qb + 32) of a range ending at q1; only
  // the own cell (CEN) tests PTrMin and holds the atom itself (the other
  // entries are other cells), and a system of one type and one pair (ONE)
  // takes no pair-matrix lookup; NB16: the list's 16-bit entries
  auto pass = [&](auto cen, auto onet, auto nbt, int qb, int q1) {
    constexpr bool CEN = decltype(cen)::value, ONE = decltype(onet)::value, NB16 = decltype(nbt)::value;
    const int qq = qb + lane;
    const int j = aoff + qq;
    const bool have = qq < q1;
    const int4 pj = c.pfx[have ? j : i];
    int mx = 1;
    if (!ONE) {
      const int tj = tw_type(pj.w);
      const int a = pm[(ti - 1) + (tj - 1) * nt], b = pm[(tj - 1) + (ti - 1) * nt];
      mx = a > b ? a : b;
    }
    const float r0 = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * sb0;
    const float r1 = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * sb1;
    const float r2 = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * sb2;
    // (FMAs: the FP32 rounding stays far inside the 1e-5 band)
    const float d2f = __fmaf_rn(r0, r0, __fmaf_rn(r1, r1, __fmul_rn(r2, r2)));
    const bool live = have && (!CEN || j != i) && (ONE || mx > 0);
    float2 band = band1;
    if (!ONE && live) {
      const float rf = (float)rl2[mx - 1];
      band = make_float2(rf * (1.f - NB_MARGIN), rf * (1.f + NB_MARGIN));
    }
    // outside both margins FP32 decides; inside either, FP64 does
    bool hit = live && d2f < band.x && !(CEN && d2f < ptrhi);
    const bool unsure = live && ((d2f >= band.x && d2f <= band.y) ||
                                 (CEN && d2f >= ptrlo && d2f <= ptrhi));
    if (__any_sync(0xffffffffu, unsure) && unsure) {
      // the reference's FP64 test (src/nd.f90:1362-1377, 1419-1420)
      const double4 pid = c.pos[i], pjd = c.pos[j];
      double s0 = pid.x - pjd.x, s1 = pid.y - pjd.y, s2 = pid.z - pjd.z;
      s0 = s0 - round(s0);
      s1 = s1 - round(s1);
      s2 = s2 - round(s2);
      const double x0 = S->box[0] * s0, x1 = S->box[1] * s1, x2 = S->box[2] * s2;
      double d2 = x0 * x0;
      d2 = d2 + x1 * x1;
      d2 = d2 + x2 * x2;
      hit = !(CEN && d2 < P->ptrmin) && !(d2 > rl2[mx - 1]);
    }
    const unsigned bal = __ballot_sync(0xffffffffu, hit);
    if (hit) {
      const int k = cnt + __popc(bal & below);
      if (k < maxnb) list_store(col, NB16, aoff, k, j);
    }
    cnt += __popc(bal);
  };
  auto ranges = [&](auto onet, auto nbt) {
    for (unsigned hd = heads; hd;) {
      const int e = __ffs(hd) - 1;
      hd &= hd - 1;
      const int last = hd ? __ffs(hd) - 2 : ne - 1;
      const bool center = __shfl_sync(0xffffffffu, e_center, e) != 0;
      const int q0 = __shfl_sync(0xffffffffu, e_q0, e), q1 = __shfl_sync(0xffffffffu, e_q1, last);
      if (center)
        for (int qb = q0; qb < q1; qb += 32) pass(BoolTag<true>{}, onet, nbt, qb, q1);
      else
        for (int qb = q0; qb < q1; qb += 32) pass(BoolTag<false>{}, onet, nbt, qb, q1);
    }
  };
  if (one) {
    if (nb16)
      ranges(BoolTag<true>{}, BoolTag<true>{});
    else
      ranges(BoolTag<true>{}, BoolTag<false>{});
  } else {
    if (nb16)
      ranges(BoolTag<false>{}, BoolTag<true>{});
    else
      ranges(BoolTag<false>{}, BoolTag<false>{});
  }
  if (lane == 0) {
    c.nnb[i] = cnt;
    if (cnt > maxnb) set_err(c, S, E_NEIMAX);
    note_rows(c, S, i, min(cnt, maxnb));
  }
}

// the listed systems' atoms, dealt round-robin to every warp of the grid
__global__ __launch_bounds__(CB_THREADS, 4) void k_build_atoms(DevCtx c) {
  __shared__ int l_sys[LIST_STAGE], l_pre[LIST_STAGE + 1];
  __shared__ int wsum[CB_THREADS / 32];
  if (c.ring_count[2] >= CELL_BUILD_MIN) return;  // many cells: the cell form builds
  const int n = c.ring_count[3];
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (CB_THREADS / 32);
  const int gw = blockIdx.x * (CB_THREADS / 32) + (threadIdx.x >> 5);
  for (int k0 = 0; k0 < n; k0 += LIST_STAGE) {
    const int m = min(LIST_STAGE, n - k0);
    __syncthreads();  // the previous group's entries are no longer read
    int cnt = 0;
    if ((int)threadIdx.x < m) {
      const int s = c.rb_list[k0 + threadIdx.x];
      l_sys[threadIdx.x] = s;
      cnt = c.P[s].n;
    }
    const int pre = block_excl_scan(cnt, wsum);
    if ((int)threadIdx.x < m) l_pre[threadIdx.x] = pre;
    if ((int)threadIdx.x == m - 1) l_pre[m] = pre + cnt;
    __syncthreads();
    const int total = l_pre[m];
    for (int u = gw; u < total; u += nw) {
      int lo = 0, hi = m - 1;  // the listed system whose atoms hold unit u
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (l_pre[mid] <= u) lo = mid;
        else hi = mid - 1;
      }
      build_atom(c, l_sys[lo], u - l_pre[lo], lane);
    }
  }
}

// the listed systems' cells, dealt round-robin to every warp of the grid
__global__ __launch_bounds__(CB_THREADS, 4) void k_build_cells(DevCtx c) {
  __shared__ int l_sys[LIST_STAGE], l_pre[LIST_STAGE + 1];
  __shared__ int wsum[CB_THREADS / 32];
  static_assert(CB_THREADS == LIST_STAGE, "one listed system per thread when staging");
  if (c.ring_count[2] < CELL_BUILD_MIN) return;  // few cells: the atom form builds
  const int n = c.ring_count[3];
  const int lane = threadIdx.x & 31;
  const int nw = gridDim.x * (CB_THREADS / 32);
  const int gw = blockIdx.x * (CB_THREADS / 32) + (threadIdx.x >> 5);
  for (int k0 = 0; k0 < n; k0 += LIST_STAGE) {
    const int m = min(LIST_STAGE, n - k0);
    __syncthreads();  // the previous group's entries are no longer read
    int cnt = 0;
    if ((int)threadIdx.x < m) {
      const int s = c.rb_list[k0 + threadIdx.x];
      l_sys[threadIdx.x] = s;
      cnt = c.S[s].ncell;
    }
    const int pre = block_excl_scan(cnt, wsum);
    if ((int)threadIdx.x < m) l_pre[threadIdx.x] = pre;
    if ((int)threadIdx.x == m - 1) l_pre[m] = pre + cnt;
    __syncthreads();
    const int total = l_pre[m];
    for (int u = gw; u < total; u += nw) {
      int lo = 0, hi = m - 1;  // the listed system whose cells hold unit u
      while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (l_pre[mid] <= u) lo = mid;
        else hi = mid - 1;
      }
      build_cell(c, l_sys[lo], u - l_pre[lo], lane);
    }
  }
}

// ---------------------------------------------------------------------------
// Pair loop: compute0 (src/nd.f90:273-333) over the full neighbour list,
// TPA threads per atom, and with FUSE the integrate2 update
// (src/nd.f90:1094-1116) of each atom as soon as its force is complete.
//
// One CTA (TILE*TPA threads) works on one 128-atom tile at a time; CTAs are
// persistent and own contiguous tile ranges.  The tile's list rows are one
// contiguous region, bulk-prefetched into L2 one tile ahead; neighbour
// positions are gathered from global memory (the atoms are sorted by link
// cell, so a tile's neighbours are a compact set that stays in L1/L2); the
// pair matrix, cutoffs and interpolation tables of the system are staged in
// shared memory once per system change.
constexpr int UNR_D = 2;  // FP64: pairs in flight per thread

// Mixed precision: a pair whose FP32 squared distance lies within NEAR_CUT
// (relative) of the squared cutoff takes compute0's FP64 cutoff test, so
// the two precisions sum the same set of pairs (the tabulated force at the
// cutoff is not zero).  The FP32 distance from 32-bit fixed-point
// positions is within 1e-6 relative of the FP64 one for boxes up to
// 1e3 cutoffs wide, so 1e-5 leaves a tenfold margin.
constexpr float NEAR_CUT = 1e-5f;

struct TabView {
  const int *pm;
  const double *rc2;
  const float *rc2f, *vdr2;
  const float4 *pp;         // staged: per pair {rc2f(1-NEAR_CUT), rc2f(1+NEAR_CUT), vdr2, rc2f}
  const double *tF, *tP;    // FP64 tables
  const float2 *tF2, *tP2;  // FP32 (k, k+1) pairs
};

// Staged layout (stab_bytes_lean): pair matrix | rc2 (double) | packed
// per-pair float4 | F table.  The P table stays in global memory (L1-cached):
// only output steps read it, and leaving it out keeps the energy/virial
// kernel (every step of a barostat) at the lean kernel's residency.
template <bool MIXED, bool EV>
__device__ void stage_tables(const DevCtx &c, const SysParam *P, unsigned char *sm, TabView &tv) {
  const int nt = P->ntypes, np = P->npairs, T = P->ptsize + 1;
  int *pm = (int *)sm;
  int off = (nt * nt * 4 + 15) / 16 * 16;
  double *rc2 = (double *)(sm + off);
  off = (off + np * 8 + 15) / 16 * 16;
  float4 *pp = (float4 *)(sm + off);
  off += np * 16;
  for (int k = threadIdx.x; k < nt * nt; k += blockDim.x) pm[k] = c.pairg[P->pm_off + k];
  for (int k = threadIdx.x; k < np; k += blockDim.x) {
    rc2[k] = c.rc2[P->pair_off + k];
    const float r = c.rc2f[P->pair_off + k];
    pp[k] = make_float4(r * (1.f - NEAR_CUT), r * (1.f + NEAR_CUT), c.vdr2[P->pair_off + k], r);
  }
  tv.pm = pm;
  tv.rc2 = rc2;
  tv.pp = pp;
  tv.rc2f = c.rc2f + P->pair_off;
  tv.vdr2 = c.vdr2 + P->pair_off;
  if (MIXED) {
    float2 *dF = (float2 *)(sm + off);
    const float2 *sF = c.tabF2 + P->tab_off;
    for (int k = threadIdx.x; k < np * T; k += blockDim.x) dF[k] = sF[k];
    tv.tF2 = dF;
    tv.tP2 = c.tabP2 + P->tab_off;
  } else {
    double *dF = (double *)(sm + off);
    const double *sF = c.tabF + P->tab_off;
    for (int k = threadIdx.x; k < np * T; k += blockDim.x) dF[k] = sF[k];
    tv.tF = dF;
    tv.tP = c.tabP + P->tab_off;
  }
}

__device__ __forceinline__ void global_tables(const DevCtx &c, const SysParam *P, TabView &tv) {
  tv.pm = c.pairg + P->pm_off;
  tv.rc2 = c.rc2 + P->pair_off;
  tv.rc2f = c.rc2f + P->pair_off;
  tv.vdr2 = c.vdr2 + P->pair_off;
  tv.pp = nullptr;
  tv.tF = c.tabF + P->tab_off;
  tv.tP = c.tabP + P->tab_off;
  tv.tF2 = c.tabF2 + P->tab_off;
  tv.tP2 = c.tabP2 + P->tab_off;
}

// L2 eviction priority for streams read once per step (the neighbour list
// rows): their lines go first, so the gathered positions, which every tile
// re-reads, keep their place in L2
__device__ __forceinline__ unsigned long long l2_evict_first() {
  unsigned long long p;
  asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}

__device__ __forceinline__ int ld_stream(const int *a, unsigned long long pol) {
  int v;
  asm("ld.global.nc.L1::no_allocate.L2::cache_hint.b32 %0, [%1], %2;"
      : "=r"(v)
      : "l"(a), "l"(pol));
  return v;
}

// per-pair cutoff band and table scale of the mixed loop
template <bool STAB>
__device__ __forceinline__ float4 pair_params(const TabView &tv, int p1) {
  if (STAB) return tv.pp[p1];
  const float r = tv.rc2f[p1];
  return make_float4(r * (1.f - NEAR_CUT), r * (1.f + NEAR_CUT), tv.vdr2[p1], r);
}

// A spring pair (compute2/compute3, src/nd.f90:627-660, 826-859): strain
// s = r/r0 - 1 of the pair against its initial separation (initial
// positions ipos, box ibox, minimum image by one anint); no force while
// s > sc; else df = -D0*s*Vol^2/r along rij and energy D0*s^2*Vol^2*r0/2.
// Returns false where the pair is broken.
__device__ __forceinline__ bool spring_df(const DevCtx &c, const SysParam *P, int gi, int gj,
                                          double d2, const double4 &sp, double &df, double &dp) {
  const double4 a = c.ipos[P->atom_off + gi], b = c.ipos[P->atom_off + gj];
  double s0 = a.x - b.x, s1 = a.y - b.y, s2 = a.z - b.z;
  s0 = s0 - round(s0);
  s1 = s1 - round(s1);
  s2 = s2 - round(s2);
  const double x0 = P->ibox[0] * s0, x1 = P->ibox[1] * s1, x2 = P->ibox[2] * s2;
  double d20 = x0 * x0;
  d20 = d20 + x1 * x1;
  d20 = d20 + x2 * x2;
  const double r = sqrt(d2), r0 = sqrt(d20);
  const double sij = r / r0 - 1.0;
  if (sij > sp.y) return false;
  const double f = sp.x * sij * sp.z * sp.z;
  dp = 0.5 * f * sij * r0;
  df = -f / r;
  return true;
}

// One atom's spring pairs, its share of the list entries (k = la, la+tpa,
// ...), in FP64: force, energy (cu) and virial (cv) of the pairs with
// PTij = PTji.  Mixed precision takes each pair's terms in 64-bit fixed
// point (q), so the totals do not depend on the launch shape; FP64 sums
// them in list order (d).
struct SpringSum {
  long long q[10];  // fx, fy, fz, pe, virial xx yy zz xy xz yz
  double d[10];
};

template <bool MIXED>
__device__ __noinline__ SpringSum spring_pass(const DevCtx &c, const SysParam *P, const SysState *S,
                                              const int *pm, int i, int ti, int ntypes,
                                              const int *nb, int cnt, int la, int tpa, bool cu,
                                              bool cv) {
  SpringSum o;
  for (int k = 0; k < 10; ++k) {
    o.q[k] = 0;
    o.d[k] = 0.0;
  }
  const double4 pid = c.pos[i];
  const double b0 = S->box[0], b1 = S->box[1], b2 = S->box[2];
  const int gi = c.gid[i];
  for (int k = la; k < cnt; k += tpa) {
    const int j = list_entry(nb, P->nb16, P->atom_off, k);
    const double4 pjd = c.pos[j];
    const int pg = pm[(ti - 1) + (tw_type(tw_of(pjd.w)) - 1) * ntypes];
    const int pt = pg & PT_MASK;
    if (pt == 0) continue;
    const double4 sp = c.spr[P->pair_off + pt - 1];
    if (sp.w == 0.0) continue;
    double s0 = pid.x - pjd.x, s1 = pid.y - pjd.y, s2 = pid.z - pjd.z;
    s0 = s0 - round(s0);
    s1 = s1 - round(s1);
    s2 = s2 - round(s2);
    const double x[3] = {b0 * s0, b1 * s1, b2 * s2};
    double dd = x[0] * x[0];
    dd = dd + x[1] * x[1];
    dd = dd + x[2] * x[2];
    double df, dp;
    if (!spring_df(c, P, gi, c.gid[j], dd, sp, df, dp)) continue;
    const bool sym = pg < PT_ASYM;
    double t[10] = {x[0] * df, x[1] * df, x[2] * df, (cu && sym) ? dp : 0.0, 0, 0, 0, 0, 0, 0};
    if (cv && sym) {
      t[4] = x[0] * x[0] * df;
      t[5] = x[1] * x[1] * df;
      t[6] = x[2] * x[2] * df;
      t[7] = x[0] * x[1] * df;
      t[8] = x[0] * x[2] * df;
      t[9] = x[1] * x[2] * df;
    }
    for (int q = 0; q < 10; ++q) {
      if (MIXED) o.q[q] += __double2ll_rn(t[q] * FORCE_FX);
      else o.d[q] = o.d[q] + t[q];
    }
  }
  return o;
}

// STAB: tables staged in shared memory (else read from global memory).
// EV: the kernel of steps that need the potential energy or the virial
// (calcPot / calcVirial); the kernel of the other steps carries no energy
// or virial state, so its pair loop holds fewer registers.  Per tile, a
// system with one type and one pair potential takes the loop with the pair
// parameters in registers, others look them up per pair.
//
// Mixed precision: each thread sums whole chunks of CHUNK consecutive list
// entries in FP32 (in list order; a full chunk of a one-potential system
// in the lean kernel as its even entries' sum plus its odd entries' sum, two
// entries per f32x2 instruction), and adds every chunk's sum to 64-bit
// fixed-point totals (the force in registers; with EV, the potential energy
// and virial in per-thread shared-memory slots).  Chunks are dealt to the
// TPA threads of an atom round-robin, so every launch shape forms the same
// chunks and the integer totals, which do not depend on the order of
// addition, are the same bits for any TPA, grid or batch composition.
// Packed FP32 pairs (sm_100's f32x2 add/sub/mul/fma: two FP32 operations in
// one instruction, each rounded as its scalar form): the mixed loop's
// full-chunk path evaluates two list entries per instruction.
typedef unsigned long long f32x2;
__device__ __forceinline__ f32x2 pk2(float a, float b) {
  f32x2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
  return r;
}
__device__ __forceinline__ void upk2(f32x2 v, float &a, float &b) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ f32x2 add2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 sub2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 mul2(f32x2 a, f32x2 b) {
  f32x2 r;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
  return r;
}
__device__ __forceinline__ f32x2 fma2(f32x2 a, f32x2 b, f32x2 c) {
  f32x2 r;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

constexpr int CHUNK = 8;   // mixed: list entries per FP32 partial sum
// mixed: neighbour gathers in flight per thread, 4 or 8 (a tuning choice:
// 8 hides more latency when the gathers miss L2, 4 keeps more warps resident)

// resident 128-thread CTAs per SM each variant is compiled for (register
// budget 65536 / (128 * n)): the mixed lean loop fits 72 registers (80 with
// eight gathers in flight), its energy/virial form about 100, the FP64 ones
// 100 and 128
template <bool MIXED, bool EV, int GATHER>
constexpr int pair_ctas() {
  return MIXED ? (EV ? 5 : (GATHER > 4 ? 6 : 7)) : (EV ? 4 : 5);
}

// SPRING: the variant for contexts that hold spring pairs (one thread per
// atom, gather depth 4); the others carry no spring code at all.
template <int TPA, bool MIXED, bool FUSE, bool STAB, bool EV, int GATHER, bool SPRING = false>
__global__ __launch_bounds__(TILE * TPA, (pair_ctas<MIXED, EV, GATHER>() * 128 / (TILE * TPA)) > 0
                                             ? pair_ctas<MIXED, EV, GATHER>() * 128 / (TILE * TPA)
                                             : 1) void k_pair(DevCtx c, int host_flags, int ntiles,
                                                     unsigned long long next_h, int cls) {
  constexpr int NT = TILE * TPA;
  extern __shared__ __align__(16) unsigned char dsm[];
  // mixed EV: 7 fixed-point slots (energy, virial) per thread, after the tables
  unsigned long long *evq = (unsigned long long *)(dsm + (STAB ? c.stab_lean : 0));
  const int G = gridDim.x;
  // the block's tiles: in a dynamics step its equal share of the planned
  // cost of this launch's systems (runs of consecutive tiles, usually of
  // one or two systems), in standalone compute0 an even split of all tiles
  // (only tcur, tend and the plan entry kk stay live across tiles; the
  // block's cost range is worked out again where a system starts)
  const int L = (EV ? 1 : 0) + 2 * cls;  // this launch's plan
  int tcur = 0, tend = 0, kk = -1;
  if (FUSE) {
    const long long tot = c.plan_hdr->tot[L];
    if ((long long)blockIdx.x * tot / G < (long long)(blockIdx.x + 1) * tot / G)
      kk = c.plan_kb[L * PLAN_GMAX + blockIdx.x];
  } else {
    tcur = (int)((long long)blockIdx.x * ntiles / G);
    tend = (int)((long long)(blockIdx.x + 1) * ntiles / G);
  }
  int loaded = -1;
  TabView tv;
  __shared__ int last;
  constexpr int NR = MIXED ? 1 : 8, KR = NR - 1;  // rows: FP64 energy/virial 0-6, kinetic KR
  __shared__ double s_red[NR][TILE];          // per-atom values, reduced by atom index
  __shared__ unsigned long long s_q[7];       // mixed: tile's fixed-point PE and virial
  if (threadIdx.x < 7) s_q[threadIdx.x] = 0ull;
  if (MIXED && EV)
    for (int k = 0; k < 7; ++k) evq[k * NT + threadIdx.x] = 0ull;
  __syncthreads();

  for (;;) {
    if (tcur >= tend) {
      // next system of the plan: its tiles whose first cost unit lies in
      // [lo, hi), tile j starting at cum + j * cpt
      if (!FUSE || kk < 0 || kk >= c.plan_hdr->m[L]) break;
      const long long tot = c.plan_hdr->tot[L];
      const long long lo = (long long)blockIdx.x * tot / G;
      const long long hi = (long long)(blockIdx.x + 1) * tot / G;
      const PlanEnt e = c.plan[(size_t)L * c.nsys_cap + kk++];
      if (e.cum >= hi) break;
      const SysParam *Pe = c.P + e.sys;
      const long long nt = Pe->npad / TILE;
      const long long j0 = lo > e.cum ? (lo - e.cum + e.cpt - 1) / e.cpt : 0;
      const long long j1 = min(nt, (hi - e.cum + e.cpt - 1) / e.cpt);
      tcur = Pe->atom_off / TILE + (int)j0;
      tend = Pe->atom_off / TILE + (int)j1;
      continue;
    }
    const int tile = tcur++;
    const int a0 = tile * TILE;
    const int sys = c.chunk_sys[a0 / ATOM_ALIGN];
    if (sys < 0) continue;
    const SysParam *__restrict__ P = c.P + sys;
    SysState *S = c.S + sys;
    const int flags = FUSE ? S->flags : host_flags;
    if (FUSE && (flags & (F_ACTIVE | F_DONE)) != F_ACTIVE) continue;
    if (FUSE && (((flags & (F_CU | F_CV)) != 0) != EV)) continue;  // the other kernel's tile
    if (!FUSE && P->n == 0) continue;
    if (sys != loaded) {
      if (STAB) {
        __syncthreads();  // no thread still reads the previous system's tables
        stage_tables<MIXED, EV>(c, P, dsm, tv);
        __syncthreads();  // tables complete before the first pair
      } else {
        global_tables(c, P, tv);
      }
      loaded = sys;
    }
    // prefetch the next tile's neighbour list (one contiguous region of
    // rows x TILE ints) into L2 while this tile computes
    if (threadIdx.x == 0 && tcur < tend) {
      const int nt_ = tcur;
      const int ns = c.chunk_sys[nt_ * TILE / ATOM_ALIGN];
      if (ns >= 0) {
        const SysParam *Pn = c.P + ns;
        const int rows = list_words(min(c.tile_rows[nt_], Pn->maxnb), Pn->nb16);
        const int *src = c.nbr + Pn->nbr_off + (long long)((nt_ * TILE - Pn->atom_off) / TILE) *
                                                   Pn->maxnb * TILE;
        if (rows > 0) {
          asm volatile("cp.async.bulk.prefetch.L2.global.L2::cache_hint [%0], %1, %2;" ::"l"(
                           __cvta_generic_to_global(src)),
                       "r"(rows * TILE * 4), "l"(l2_evict_first())
                       : "memory");
        }
      }
    }
    const int g = threadIdx.x / TPA, la = threadIdx.x % TPA;
    const int i = a0 + g;
    const int local = i - P->atom_off;
    const bool valid = local < P->n;
    const bool cu = EV && (flags & F_CU), cv = EV && (flags & F_CV);
    const int ntypes = P->ntypes, T = P->ptsize + 1, ptsize = P->ptsize;
    const bool one = ntypes == 1 && P->npairs == 1 && tv.pm[0] == 1;

    double pe = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};  // FP64 path
    double fx = 0.0, fy = 0.0, fz = 0.0;
    long long qx = 0, qy = 0, qz = 0;  // mixed: 64-bit fixed-point force
    int ti = 1;
    if (valid) {
      // blocked list: row k of this tile is TILE contiguous ints
      const int *__restrict__ nb =
          c.nbr + P->nbr_off + (long long)(local / TILE) * P->maxnb * TILE + g;
      int cnt = c.nnb[i];
      cnt = cnt < P->maxnb ? cnt : P->maxnb;
      const int nb16 = P->nb16, aoff = P->atom_off;
      if (!MIXED) {
        const double4 pi = c.pos[i];
        ti = tw_type(tw_of(pi.w));
        const int *pmr = tv.pm + (ti - 1);
        const double b0 = S->box[0], b1 = S->box[1], b2 = S->box[2];
        const double ptrmin = P->ptrmin;
        auto loop = [&](auto one_t) {
          constexpr bool ONE = decltype(one_t)::value;
          for (int k0 = la; k0 < cnt; k0 += UNR_D * TPA) {
            int qq[UNR_D];
            double4 pj[UNR_D];
#pragma unroll
            for (int q = 0; q < UNR_D; ++q) {
              const int k = k0 + q * TPA;
              qq[q] = k < cnt ? list_entry(nb, nb16, aoff, k) : -1;
            }
#pragma unroll
            for (int q = 0; q < UNR_D; ++q) pj[q] = c.pos[qq[q] >= 0 ? qq[q] : i];
#pragma unroll
            for (int q = 0; q < UNR_D; ++q) {
              const int pg = ONE ? 1 : pmr[(tw_type(tw_of(pj[q].w)) - 1) * ntypes];
              const int pt = pg & PT_MASK;
              const bool sym = ONE || pg < PT_ASYM;  // energy and virial count
              const int p1 = ONE ? 0 : (pt > 0 ? pt - 1 : 0);
              double s0 = pi.x - pj[q].x, s1 = pi.y - pj[q].y, s2 = pi.z - pj[q].z;
              s0 = s0 - round(s0);
              s1 = s1 - round(s1);
              s2 = s2 - round(s2);
              const double r0 = b0 * s0, r1 = b1 * s1, r2 = b2 * s2;
              double d2 = r0 * r0;
              d2 = d2 + r1 * r1;
              d2 = d2 + r2 * r2;
              const bool ok = qq[q] >= 0 && pt > 0 && !(d2 > tv.rc2[p1]);
              const float rk = (float)(d2 - ptrmin) * tv.vdr2[p1] + 1.0f;
              int kk = (int)rk;
              kk = kk < 1 ? 1 : (kk > ptsize ? ptsize : kk);
              const double w = (double)rk - (double)kk;
              const int base = p1 * T + kk - 1;
              const double fk1 = tv.tF[base + 1], fk = tv.tF[base];
              double df = w * fk1 + (1.0 - w) * fk;
              df = ok ? df / d2 : 0.0;
              fx = fx + r0 * df;
              fy = fy + r1 * df;
              fz = fz + r2 * df;
              if (cu && ok && sym) pe = pe + (w * tv.tP[base + 1] + (1.0 - w) * tv.tP[base]);
              if (cv && sym) {
                vir[0] = vir[0] + r0 * r0 * df;
                vir[1] = vir[1] + r1 * r1 * df;
                vir[2] = vir[2] + r2 * r2 * df;
                vir[3] = vir[3] + r0 * r1 * df;
                vir[4] = vir[4] + r0 * r2 * df;
                vir[5] = vir[5] + r1 * r2 * df;
              }
            }
          }
        };
        if (one) loop(std::true_type{});
        else loop(std::false_type{});
      } else {
        const int4 pi = c.pfx[i];
        ti = tw_type(pi.w);
        const int *pmr = tv.pm + (ti - 1);
        const float sb0 = (float)(S->box[0] * (1.0 / FX_ONE));
        const float sb1 = (float)(S->box[1] * (1.0 / FX_ONE));
        const float sb2 = (float)(S->box[2] * (1.0 / FX_ONE));
        const float ptrmin = (float)P->ptrmin;
        const int nch = (cnt + CHUNK - 1) / CHUNK;
        const unsigned long long lpol = l2_evict_first();
        auto loop = [&](auto one_t) {
          constexpr bool ONE = decltype(one_t)::value;
          const float4 pp1 = ONE ? pair_params<STAB>(tv, 0) : make_float4(0.f, 0.f, 0.f, 0.f);
          for (int m = la; m < nch; m += TPA) {
            const int kb = m * CHUNK;
            float ax = 0.f, ay = 0.f, az = 0.f, ape = 0.f;
            float av0 = 0.f, av1 = 0.f, av2 = 0.f, av3 = 0.f, av4 = 0.f, av5 = 0.f;
            unsigned nm = 0;  // entries of this chunk within FP32 rounding of the cutoff
            if (ONE && !EV && kb + CHUNK <= cnt) {
              // a full chunk of a one-potential system: no per-entry masks,
              // entries 2q and 2q+1 side by side in f32x2 operations, the
              // chunk's sum as the sum of its even and its odd entries
              const int4 *__restrict__ pb = nb16 ? c.pfx + aoff : c.pfx;
              int jj[CHUNK];
              if (nb16) {
#pragma unroll
                for (int q = 0; q < CHUNK; q += 2) {
                  const int w = ld_stream(nb + ((kb + q) >> 1) * TILE, lpol);
                  jj[q] = w & 0xffff;
                  jj[q + 1] = (int)((unsigned)w >> 16);
                }
              } else {
#pragma unroll
                for (int q = 0; q < CHUNK; ++q) jj[q] = ld_stream(nb + (kb + q) * TILE, lpol);
              }
              const f32x2 SB0 = pk2(sb0, sb0), SB1 = pk2(sb1, sb1), SB2 = pk2(sb2, sb2);
              const f32x2 NPT = pk2(-ptrmin, -ptrmin), VDR = pk2(pp1.z, pp1.z),
                          ONE2 = pk2(1.0f, 1.0f);
              f32x2 AX = 0ull, AY = 0ull, AZ = 0ull;
#pragma unroll
              for (int h = 0; h < CHUNK; h += GATHER) {
                int4 pj[GATHER];
#pragma unroll
                for (int q = 0; q < GATHER; ++q) pj[q] = pb[jj[h + q]];
#pragma unroll
                for (int q = 0; q < GATHER; q += 2) {
                  const int4 pa = pj[q], pc = pj[q + 1];
                  // minimum image by 32-bit wrap-around of the fixed-point difference
                  const f32x2 R0 = mul2(pk2((float)(int)((unsigned)pi.x - (unsigned)pa.x),
                                            (float)(int)((unsigned)pi.x - (unsigned)pc.x)), SB0);
                  const f32x2 R1 = mul2(pk2((float)(int)((unsigned)pi.y - (unsigned)pa.y),
                                            (float)(int)((unsigned)pi.y - (unsigned)pc.y)), SB1);
                  const f32x2 R2 = mul2(pk2((float)(int)((unsigned)pi.z - (unsigned)pa.z),
                                            (float)(int)((unsigned)pi.z - (unsigned)pc.z)), SB2);
                  const f32x2 D2 = fma2(R0, R0, fma2(R1, R1, mul2(R2, R2)));
                  float da, dc;
                  upk2(D2, da, dc);
                  const bool oka = da <= pp1.x, okc = dc <= pp1.x;
                  nm |= (!oka && da <= pp1.y ? 1u << (h + q) : 0u) |
                        (!okc && dc <= pp1.y ? 2u << (h + q) : 0u);
                  const f32x2 RK = fma2(add2(D2, NPT), VDR, ONE2);
                  float rka, rkc;
                  upk2(RK, rka, rkc);
                  int ka = (int)rka, kc = (int)rkc;
                  ka = ka < 1 ? 1 : (ka > ptsize ? ptsize : ka);
                  kc = kc < 1 ? 1 : (kc > ptsize ? ptsize : kc);
                  const f32x2 W = sub2(RK, pk2((float)ka, (float)kc));
                  const float2 Fa = tv.tF2[ka - 1], Fc = tv.tF2[kc - 1];
                  const f32x2 FX = pk2(Fa.x, Fc.x);
                  const f32x2 NUM = fma2(W, sub2(pk2(Fa.y, Fc.y), FX), FX);
                  float na, nc;
                  upk2(mul2(NUM, pk2(rcp_approx(da), rcp_approx(dc))), na, nc);
                  const f32x2 DF = pk2(oka ? na : 0.f, okc ? nc : 0.f);
                  AX = fma2(R0, DF, AX);
                  AY = fma2(R1, DF, AY);
                  AZ = fma2(R2, DF, AZ);
                }
              }
              float e0, e1;
              upk2(AX, e0, e1);
              ax = e0 + e1;
              upk2(AY, e0, e1);
              ay = e0 + e1;
              upk2(AZ, e0, e1);
              az = e0 + e1;
            } else {
              int qq[CHUNK];
              if (nb16) {
                // two 16-bit entries per word (CHUNK and kb are even)
#pragma unroll
                for (int q = 0; q < CHUNK; q += 2) {
                  const int w = kb + q < cnt ? ld_stream(nb + ((kb + q) >> 1) * TILE, lpol) : 0;
                  qq[q] = kb + q < cnt ? aoff + (w & 0xffff) : -1;
                  qq[q + 1] = kb + q + 1 < cnt ? aoff + (int)((unsigned)w >> 16) : -1;
                }
              } else {
#pragma unroll
                for (int q = 0; q < CHUNK; ++q)
                  qq[q] = kb + q < cnt ? ld_stream(nb + (kb + q) * TILE, lpol) : -1;
              }
#pragma unroll
              for (int h = 0; h < CHUNK; h += GATHER) {
                int4 pj[GATHER];
#pragma unroll
                for (int q = 0; q < GATHER; ++q) pj[q] = c.pfx[qq[h + q] >= 0 ? qq[h + q] : i];
#pragma unroll
                for (int q = 0; q < GATHER; ++q) {
                  const int pg = ONE ? 1 : pmr[(tw_type(pj[q].w) - 1) * ntypes];
                  const int pt = pg & PT_MASK;
                  const bool sym = ONE || pg < PT_ASYM;  // energy and virial count
                  const int p1 = ONE ? 0 : (pt > 0 ? pt - 1 : 0);
                  const float4 prm = ONE ? pp1 : pair_params<STAB>(tv, p1);
                  // minimum image by 32-bit wrap-around of the fixed-point difference
                  const float r0 = (float)(int)((unsigned)pi.x - (unsigned)pj[q].x) * sb0;
                  const float r1 = (float)(int)((unsigned)pi.y - (unsigned)pj[q].y) * sb1;
                  const float r2 = (float)(int)((unsigned)pi.z - (unsigned)pj[q].z) * sb2;
                  const float d2 = __fmaf_rn(r0, r0, __fmaf_rn(r1, r1, __fmul_rn(r2, r2)));
                  const bool live = qq[h + q] >= 0 && pt > 0;
                  const bool ok = live && d2 <= prm.x;
                  nm |= (live && d2 > prm.x && d2 <= prm.y) ? (1u << (h + q)) : 0u;
                  // branch-free: every lane evaluates the pair, excluded ones add 0
                  const float rk = __fmaf_rn(d2 - ptrmin, prm.z, 1.0f);
                  int kk = (int)rk;
                  kk = kk < 1 ? 1 : (kk > ptsize ? ptsize : kk);
                  const float w = rk - (float)kk;
                  const int base = p1 * T + kk - 1;
                  const float2 F = tv.tF2[base];
                  const float df = ok ? __fdividef(__fmaf_rn(w, F.y - F.x, F.x), d2) : 0.f;
                  ax = __fmaf_rn(r0, df, ax);
                  ay = __fmaf_rn(r1, df, ay);
                  az = __fmaf_rn(r2, df, az);
                  if (cu && ok && sym) {
                    const float2 Pp = tv.tP2[base];
                    ape += __fmaf_rn(w, Pp.y - Pp.x, Pp.x);
                  }
                  if (cv) {
                    const float dv = sym ? df : 0.f;
                    const float r0d = r0 * dv, r1d = r1 * dv;
                    av0 = __fmaf_rn(r0d, r0, av0);
                    av1 = __fmaf_rn(r1d, r1, av1);
                    av2 = __fmaf_rn(r2 * dv, r2, av2);
                    av3 = __fmaf_rn(r0d, r1, av3);
                    av4 = __fmaf_rn(r0d, r2, av4);
                    av5 = __fmaf_rn(r1d, r2, av5);
                  }
                }
              }
            }
            if (nm) {
              // the chunk's entries near the cutoff: compute0's FP64 test
              // decides (src/nd.f90:283-296), then the same FP32 evaluation
              const double4 pid = c.pos[i];
              const double b0 = S->box[0], b1 = S->box[1], b2 = S->box[2];
#pragma unroll 1
              while (nm) {
                const int q = __ffs(nm) - 1;
                nm &= nm - 1;
                const int j = list_entry(nb, nb16, aoff, kb + q);
                const int4 pj = c.pfx[j];
                const int pg = ONE ? 1 : pmr[(tw_type(pj.w) - 1) * ntypes];
                const bool sym = ONE || pg < PT_ASYM;
                const int p1 = (pg & PT_MASK) - 1;
                const double4 pjd = c.pos[j];
                double s0 = pid.x - pjd.x, s1 = pid.y - pjd.y, s2 = pid.z - pjd.z;
                s0 = s0 - round(s0);
                s1 = s1 - round(s1);
                s2 = s2 - round(s2);
                const double x0 = b0 * s0, x1 = b1 * s1, x2 = b2 * s2;
                double dd = x0 * x0;
                dd = dd + x1 * x1;
                dd = dd + x2 * x2;
                if (dd > tv.rc2[p1]) continue;
                const float4 prm = ONE ? pp1 : pair_params<STAB>(tv, p1);
                const float r0 = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * sb0;
                const float r1 = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * sb1;
                const float r2 = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * sb2;
                const float d2 = __fmaf_rn(r0, r0, __fmaf_rn(r1, r1, __fmul_rn(r2, r2)));
                const float rk = __fmaf_rn(d2 - ptrmin, prm.z, 1.0f);
                int kk = (int)rk;
                kk = kk < 1 ? 1 : (kk > ptsize ? ptsize : kk);
                const float w = rk - (float)kk;
                const int base = p1 * T + kk - 1;
                const float2 F = tv.tF2[base];
                const float df = __fdividef(__fmaf_rn(w, F.y - F.x, F.x), d2);
                ax = __fmaf_rn(r0, df, ax);
                ay = __fmaf_rn(r1, df, ay);
                az = __fmaf_rn(r2, df, az);
                if (cu && sym) {
                  const float2 Pp = tv.tP2[base];
                  ape += __fmaf_rn(w, Pp.y - Pp.x, Pp.x);
                }
                if (cv && sym) {
                  const float r0d = r0 * df, r1d = r1 * df;
                  av0 = __fmaf_rn(r0d, r0, av0);
                  av1 = __fmaf_rn(r1d, r1, av1);
                  av2 = __fmaf_rn(r2 * df, r2, av2);
                  av3 = __fmaf_rn(r0d, r1, av3);
                  av4 = __fmaf_rn(r0d, r2, av4);
                  av5 = __fmaf_rn(r1d, r2, av5);
                }
              }
            }
            qx += __float2ll_rn(ax * (float)FORCE_FX);
            qy += __float2ll_rn(ay * (float)FORCE_FX);
            qz += __float2ll_rn(az * (float)FORCE_FX);
            if (EV) {
              unsigned long long *q = evq + threadIdx.x;
              q[0] += (unsigned long long)__float2ll_rn(ape * (float)FORCE_FX);
              q[NT] += (unsigned long long)__float2ll_rn(av0 * (float)FORCE_FX);
              q[2 * NT] += (unsigned long long)__float2ll_rn(av1 * (float)FORCE_FX);
              q[3 * NT] += (unsigned long long)__float2ll_rn(av2 * (float)FORCE_FX);
              q[4 * NT] += (unsigned long long)__float2ll_rn(av3 * (float)FORCE_FX);
              q[5 * NT] += (unsigned long long)__float2ll_rn(av4 * (float)FORCE_FX);
              q[6 * NT] += (unsigned long long)__float2ll_rn(av5 * (float)FORCE_FX);
            }
          }
        };
        if (one) loop(std::true_type{});
        else loop(std::false_type{});
      }
      if (SPRING && P->nspring > 0) {
        // spring pairs (compute2/compute3), left out of the loops above by
        // their cutoff word (-1), out of line so that they cost the other
        // systems nothing
        const SpringSum sp = spring_pass<MIXED>(c, P, S, tv.pm, i, ti, ntypes, nb, cnt, la, TPA,
                                                cu, cv);
        if (MIXED) {
          qx += sp.q[0];
          qy += sp.q[1];
          qz += sp.q[2];
          if (EV)
            for (int k = 0; k < 7; ++k) evq[k * NT + threadIdx.x] += (unsigned long long)sp.q[3 + k];
        } else {
          fx = fx + sp.d[0];
          fy = fy + sp.d[1];
          fz = fz + sp.d[2];
          pe = pe + sp.d[3];
          for (int k = 0; k < 6; ++k) vir[k] = vir[k] + sp.d[4 + k];
        }
      }
    }
    if (!MIXED) {
      // combine the TPA partial forces of an atom (fixed tree: deterministic)
#pragma unroll
      for (int o = TPA / 2; o > 0; o >>= 1) {
        fx += __shfl_xor_sync(0xffffffffu, fx, o);
        fy += __shfl_xor_sync(0xffffffffu, fy, o);
        fz += __shfl_xor_sync(0xffffffffu, fz, o);
        if (EV) {
          pe += __shfl_xor_sync(0xffffffffu, pe, o);
#pragma unroll
          for (int k = 0; k < 6; ++k) vir[k] += __shfl_xor_sync(0xffffffffu, vir[k], o);
        }
      }
    } else {
      // fixed-point sums are exact, so any combination order gives one result
#pragma unroll
      for (int o = TPA / 2; o > 0; o >>= 1) {
        qx += __shfl_xor_sync(0xffffffffu, qx, o);
        qy += __shfl_xor_sync(0xffffffffu, qy, o);
        qz += __shfl_xor_sync(0xffffffffu, qz, o);
      }
      fx = (double)qx * (1.0 / FORCE_FX);
      fy = (double)qy * (1.0 / FORCE_FX);
      fz = (double)qz * (1.0 / FORCE_FX);
    }
    double ke = 0.0;
    if (valid && la == 0) {
      if (FUSE) {
        const double m = c.mass[P->type_off + ti - 1];
        const double rmass = 1.0 / m;
        const double dt = P->dt;
        double *v = c.vel + 3 * (size_t)i;
        double *a = c.acc + 3 * (size_t)i;
        // velocities and accelerations stream through once per step
        const double v0 = __ldcs(v) + 0.5 * dt * (fx * rmass + __ldcs(a));
        const double v1 = __ldcs(v + 1) + 0.5 * dt * (fy * rmass + __ldcs(a + 1));
        const double v2 = __ldcs(v + 2) + 0.5 * dt * (fz * rmass + __ldcs(a + 2));
        __stcs(v, v0);
        __stcs(v + 1, v1);
        __stcs(v + 2, v2);
        __stcs(a, fx * rmass);
        __stcs(a + 1, fy * rmass);
        __stcs(a + 2, fz * rmass);
        if (flags & F_CK) {
          double kt = v0 * v0;
          kt = kt + v1 * v1;
          kt = kt + v2 * v2;
          ke = kt * m;
        }
      } else {
        double *f = c.force + 3 * (size_t)i;
        f[0] = fx; f[1] = fy; f[2] = fz;
      }
    }
    // per-tile partial sums (only what the step needs), reduced in an order
    // fixed by the atom index, then the last tile of the system runs the
    // end-of-step epilogue
    const bool ck = FUSE && (flags & F_CK);
    if (EV && MIXED) {
      // exact integer sums: the thread's slots, a warp butterfly, then one
      // shared atomic per warp; the slots start the next tile at zero
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        long long v = (long long)evq[k * NT + threadIdx.x];
        evq[k * NT + threadIdx.x] = 0ull;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&s_q[k], (unsigned long long)v);
      }
    }
    if (la == 0) {
      if (EV && !MIXED) {
        s_red[0][g] = pe;
#pragma unroll
        for (int k = 0; k < 6; ++k) s_red[(1 + k) % NR][g] = vir[k];
      }
      if (ck) s_red[KR][g] = ke;
    }
    // one warp sums the rows: lane l adds atoms l, l+32, l+64, l+96, then a
    // butterfly over the lanes, a tree fixed by the atom index (the same bits
    // for any threads-per-atom); one barrier before it, one after
    const int r0 = (EV && !MIXED) ? 0 : KR, r1 = ck ? NR : KR;
    if (EV || ck) __syncthreads();
    if (threadIdx.x < 32) {
      double *red = c.red + 8 * (size_t)tile;
      const int lane = threadIdx.x;
#pragma unroll 1
      for (int r = r0; r < r1; ++r) {
        double v = s_red[r][lane];
#pragma unroll
        for (int q = 1; q < TILE / 32; ++q) v += s_red[r][lane + 32 * q];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) red[r == KR ? 7 : r] = v;
      }
      if (lane == 0) {
        if (EV && MIXED) {
#pragma unroll
          for (int k = 0; k < 7; ++k) {
            red[k] = __longlong_as_double((long long)s_q[k]);  // bits of the integer sum
            s_q[k] = 0ull;
          }
        }
        if (!ck) red[7] = 0.0;
        __threadfence();
        const unsigned nblk = (unsigned)(P->npad / TILE);
        const unsigned t = atomicAdd(&S->ticket, 1u);
        last = (t == nblk - 1);
      }
    }
    __syncthreads();
    if (last) {
      __threadfence();
      finalize_system<MIXED>(c, sys, P->atom_off / TILE, P->npad / TILE, flags, FUSE, next_h,
                             s_red);
      if (threadIdx.x == 0) S->ticket = 0;
      __syncthreads();  // finalize's shared values are read before the next tile writes
    }
  }
}

// ---------------------------------------------------------------------------
// Bulk state transfer of every system at once (ndg_load_state and
// ndg_get_state with sys = -1).  The caller's arrays hold the systems one
// after another in id order, unpadded, each in the reference's (3,np) input
// order; xoff[s] is system s's first atom there (-1: not transferred).  The
// device staging blocks xp, xv, xa have the same (3,total) layout.

// the type word of every atom by input index (tw[atom_off + gid]), read
// before a load replaces the layout
__global__ __launch_bounds__(BLOCK) void k_type_words(DevCtx c, int *tw) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  const int sys = c.chunk_sys[i / ATOM_ALIGN];
  if (sys < 0) return;
  const SysParam &P = c.P[sys];
  if (i - P.atom_off >= P.n) return;
  const int g = c.gid[i];
  if (g < 0 || g >= P.n) return;
  tw[P.atom_off + g] = tw_of(c.pos[i].w);
}

// load: slot atom_off + l takes input atom l (identity order, as a
// per-system load leaves it); the lists are rebuilt before the next step
__global__ __launch_bounds__(BLOCK) void k_load_all(DevCtx c, const long long *xoff, const int *tw,
                                                    const double *xp, const double *xv,
                                                    const double *xa) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  const int sys = c.chunk_sys[i / ATOM_ALIGN];
  if (sys < 0) return;
  const SysParam &P = c.P[sys];
  const int l = i - P.atom_off;
  const long long o = xoff[sys];
  if (l >= P.n || o < 0) return;
  const size_t src = 3 * (size_t)(o + l), dst = 3 * (size_t)i;
  const long long w = (long long)(unsigned)tw[i];
  c.pos[i] = make_double4(xp[src], xp[src + 1], xp[src + 2], __longlong_as_double(w));
  c.gid[i] = l;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    c.vel[dst + d] = xv ? xv[src + d] : 0.0;
    c.acc[dst + d] = xa ? xa[src + d] : 0.0;
    c.disp[dst + d] = 0.0;
  }
}

// store: the atom of slot i (input index gid[i]) goes to its place in the
// caller's layout
__global__ __launch_bounds__(BLOCK) void k_store_all(DevCtx c, const long long *xoff, double *xp,
                                                     double *xv, double *xa) {
  const int i = blockIdx.x * BLOCK + threadIdx.x;
  const int sys = c.chunk_sys[i / ATOM_ALIGN];
  if (sys < 0) return;
  const SysParam &P = c.P[sys];
  const long long o = xoff[sys];
  if (i - P.atom_off >= P.n || o < 0) return;
  const int g = c.gid[i];
  if (g < 0 || g >= P.n) return;
  const size_t dst = 3 * (size_t)(o + g), src = 3 * (size_t)i;
  const double4 p = c.pos[i];
  if (xp) {
    xp[dst] = p.x;
    xp[dst + 1] = p.y;
    xp[dst + 2] = p.z;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    if (xv) xv[dst + d] = c.vel[src + d];
    if (xa) xa[dst + d] = c.acc[src + d];
  }
}

void launch_load_all(const DevCtx &c, cudaStream_t st, const long long *xoff, const double *xp,
                     const double *xv, const double *xa) {
  // type words go through tmp_key (rebuild scratch; the lists are rebuilt
  // after a load anyway)
  k_type_words<<<c.nchunks * (ATOM_ALIGN / BLOCK), BLOCK, 0, st>>>(c, c.tmp_key);
  k_load_all<<<c.nchunks * (ATOM_ALIGN / BLOCK), BLOCK, 0, st>>>(c, xoff, c.tmp_key, xp, xv, xa);
}

void launch_store_all(const DevCtx &c, cudaStream_t st, const long long *xoff, double *xp,
                      double *xv, double *xa) {
  k_store_all<<<c.nchunks * (ATOM_ALIGN / BLOCK), BLOCK, 0, st>>>(c, xoff, xp, xv, xa);
}

// ---------------------------------------------------------------------------
// launchers
static void pair_grids(const DevCtx &c, int tpa, int mixed, int *g);

void launch_integrate1(const DevCtx &c, cudaStream_t st, int standalone, int mixed, int tpa) {
  if (standalone || !c.plan_hdr) {
    k_integrate1<<<c.nchunks, BLOCK, 0, st>>>(c, standalone, mixed, make_int4(0, 0, 0, 0));
    return;
  }
  int g[PLAN_NL] = {0, 0, 0, 0};
  pair_grids(c, tpa, mixed, g);
  k_integrate1<<<c.nchunks + 1, BLOCK, 0, st>>>(c, 0, mixed, make_int4(g[0], g[1], g[2], g[3]));
}

static int sm_count() {
  static int n = 0;
  if (!n) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (n < 1) n = 148;
  }
  return n;
}

// grid of a pair-kernel variant (one wave of resident blocks); with launch
// set, also launches it
template <int TPA, bool MIXED, bool FUSE, bool STAB, bool EV, int GATHER, bool SPRING = false>
static int pair_launch(const DevCtx &c, cudaStream_t st, int hf, unsigned long long nh,
                       bool launch, int cls) {
  auto kern = k_pair<TPA, MIXED, FUSE, STAB, EV, GATHER, SPRING>;
  const int smem = (STAB ? c.stab_lean : 0) + ((MIXED && EV) ? 7 * 8 * TILE * TPA : 0);
  static int cfg_smem = -1, occ = 0;
  if (smem != cfg_smem) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, TILE * TPA, smem);
    if (occ < 1) occ = 1;
    // Registers bound the residency; the shared-memory carve-out need only
    // hold that many blocks, and the rest of the SM's 256 KB stays L1 for
    // the neighbour gathers (left alone, the carve-out is sized for the
    // blocks shared memory alone would admit).
    cudaFuncAttributes fa;
    int dev = 0, smmax = 0;
    cudaGetDevice(&dev);
    if (cudaFuncGetAttributes(&fa, kern) == cudaSuccess &&
        cudaDeviceGetAttribute(&smmax, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) ==
            cudaSuccess &&
        smmax > 0) {
      const long long need = (long long)occ * (smem + (long long)fa.sharedSizeBytes + 1024);
      const int pct = (int)std::min<long long>(100, (need * 100 + smmax - 1) / smmax);
      cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
    }
    cfg_smem = smem;
  }
  const int nsm = sm_count();
  const int ntiles = c.nchunks * (ATOM_ALIGN / TILE);
  const int grid = std::min(std::min(ntiles, nsm * occ), PLAN_GMAX);
  if (launch) kern<<<grid, TILE * TPA, smem, st>>>(c, hf, ntiles, nh, cls);
  return grid;
}

// the deeper gather only for the mixed one-thread-per-atom loop
template <int TPA, bool MIXED, bool FUSE, bool STAB, bool EV>
static int pair_go(const DevCtx &c, cudaStream_t st, int hf, unsigned long long nh, bool launch,
                   int cls) {
  if constexpr (TPA == 1) {
    if (c.any_spring)
      return pair_launch<1, MIXED, FUSE, STAB, EV, 4, true>(c, st, hf, nh, launch, cls);
  }
  if (MIXED && TPA == 1 && c.gather > 4)
    return pair_launch<TPA, MIXED, FUSE, STAB, EV, 8>(c, st, hf, nh, launch, cls);
  return pair_launch<TPA, MIXED, FUSE, STAB, EV, 4>(c, st, hf, nh, launch, cls);
}

// FUSE (a dynamics step, after the integrate1 that planned it): the kernel
// without energy/virial takes the class's systems whose step needs neither,
// the EV kernel the others.  Standalone compute0: the host flags choose.
// With g set, only the class's two dynamics grids are worked out.
template <int TPA, bool MIXED, bool FUSE, bool STAB>
static void pair_ev(const DevCtx &c, cudaStream_t st, int hf, unsigned long long nh, int *g,
                    int cls) {
  if (g) {
    g[2 * cls] = pair_go<TPA, MIXED, FUSE, STAB, false>(c, st, hf, nh, false, cls);
    g[2 * cls + 1] = pair_go<TPA, MIXED, FUSE, STAB, true>(c, st, hf, nh, false, cls);
  } else if (FUSE) {
    if (!c.plan_hdr) return;  // no system was ever added
    pair_go<TPA, MIXED, FUSE, STAB, false>(c, st, hf, nh, true, cls);
    pair_go<TPA, MIXED, FUSE, STAB, true>(c, st, hf, nh, true, cls);
  } else if (hf & (F_CU | F_CV)) {
    pair_go<TPA, MIXED, FUSE, STAB, true>(c, st, hf, nh, true, 0);
  } else {
    pair_go<TPA, MIXED, FUSE, STAB, false>(c, st, hf, nh, true, 0);
  }
}

template <int TPA, bool MIXED, bool FUSE>
static void pair_mode(const DevCtx &c, cudaStream_t st, int hf, unsigned long long nh, int *g,
                      int cls) {
  if (c.stab_smem <= 0) pair_ev<TPA, MIXED, FUSE, false>(c, st, hf, nh, g, cls);
  else pair_ev<TPA, MIXED, FUSE, true>(c, st, hf, nh, g, cls);
}

template <int TPA>
static void pair_tpa(const DevCtx &c, cudaStream_t st, int mixed, int fuse, int hf,
                     unsigned long long nh, int *g, int cls) {
  if (mixed) {
    if (fuse) pair_mode<TPA, true, true>(c, st, hf, nh, g, cls);
    else pair_mode<TPA, true, false>(c, st, hf, nh, g, cls);
  } else {
    if (fuse) pair_mode<TPA, false, true>(c, st, hf, nh, g, cls);
    else pair_mode<TPA, false, false>(c, st, hf, nh, g, cls);
  }
}

static void pair_class(const DevCtx &c, cudaStream_t st, int tpa, int mixed, int fuse, int hf,
                       unsigned long long next_h, int *g, int cls) {
  if (c.any_spring) tpa = 1;  // the spring variant is built for one thread per atom
  switch (tpa) {
    case 1: pair_tpa<1>(c, st, mixed, fuse, hf, next_h, g, cls); break;
    case 2: pair_tpa<2>(c, st, mixed, fuse, hf, next_h, g, cls); break;
    case 4: pair_tpa<4>(c, st, mixed, fuse, hf, next_h, g, cls); break;
    default: pair_tpa<8>(c, st, mixed, fuse, hf, next_h, g, cls); break;
  }
}

// A dynamics step launches each list-length class (the long-list class
// only while a threshold is set: DevCtx::rows_split, DevCtx::tpa_long);
// standalone compute0 one launch over all tiles.
static void pair_dispatch(const DevCtx &c, cudaStream_t st, int tpa, int mixed, int fuse, int hf,
                          unsigned long long next_h, int *g) {
  pair_class(c, st, tpa, mixed, fuse, hf, next_h, g, 0);
  if (fuse && c.rows_split > 0) pair_class(c, st, c.tpa_long, mixed, fuse, hf, next_h, g, 1);
}

void launch_pair(const DevCtx &c, cudaStream_t st, int tpa, int mixed, int fuse, int hf,
                 unsigned long long next_h) {
  pair_dispatch(c, st, tpa, mixed, fuse, hf, next_h, nullptr);
}

// the grids of a dynamics step's pair launches
static void pair_grids(const DevCtx &c, int tpa, int mixed, int *g) {
  pair_dispatch(c, 0, tpa, mixed, 1, 0, 0ull, g);
}

__global__ void k_decide(DevCtx c, unsigned long long h) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int s = threadIdx.x; s < c.nsys_cap; s += blockDim.x)
    if (c.P[s].n > 0 && (c.S[s].flags & F_ACTIVE) && c.S[s].rebuild) any = 1;
  __syncthreads();
  if (threadIdx.x == 0) cudaGraphSetConditional((cudaGraphConditionalHandle)h, any ? 1u : 0u);
}

void launch_decide(const DevCtx &c, cudaStream_t st, unsigned long long h) {
  k_decide<<<1, 256, 0, st>>>(c, h);
}

void launch_integrate2(const DevCtx &c, cudaStream_t st, int ck) {
  k_integrate2<<<c.nchunks, BLOCK, 0, st>>>(c, ck);
}


// The reference's NeiMax check (buildVerletList, src/nd.f90:1378,1421: STOP
// 'too many neighbours in list'), for systems in the reference semantics:
// each atom's half list as the reference builds it, the atoms of its own
// cell with a larger index (input order, :1358) plus those of the 13
// forward cells of getJcellNP (:1268-1300, folded periodically, so a grid
// of two cells visits a cell more than once), counted with the reference's
// FP64 test (:1362-1377, 1405-1420), must not exceed NeiMax.  The lists the
// pair kernels use are the full ones the build makes; this pass only counts.
__device__ void neimax_chunk(const DevCtx &c, int sys, int chunk) {
  const SysParam *__restrict__ P = c.P + sys;
  if (P->neimax_stop <= 0) return;
  SysState *S = c.S + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  // the forward offsets of getJcellNP cases 2..14
  const int fwd[13][3] = {{0, 0, 1}, {0, 1, 0},  {0, 1, -1},  {0, 1, 1},  {1, 0, 0},
                          {1, 0, -1}, {1, 0, 1}, {1, 1, 0},   {1, 1, -1}, {1, 1, 1},
                          {1, -1, 0}, {1, -1, -1}, {1, -1, 1}};
  const int M0 = S->mcell[0], M1 = S->mcell[1], M2 = S->mcell[2];
  const int cl = c.atom_cell[i];
  const int cx = cl % M0, cy = (cl / M0) % M1, cz = cl / (M0 * M1);
  const int *cst = c.cell_start + P->cell_off;
  const int *pm = c.pairmat + P->pm_off;
  const int nt = P->ntypes, gi = c.gid[i];
  const double4 pi = c.pos[i];
  const int ti = tw_type(tw_of(pi.w));
  const double b0 = S->box[0], b1 = S->box[1], b2 = S->box[2], ptrmin = P->ptrmin;
  int count = 0;
  for (int k = -1; k < 13; ++k) {
    const bool same = k < 0;
    int nc = cl;
    if (!same) {
      const int nx = (cx + fwd[k][0] + M0) % M0, ny = (cy + fwd[k][1] + M1) % M1,
                nz = (cz + fwd[k][2] + M2) % M2;
      nc = nx + ny * M0 + nz * M0 * M1;
    }
    for (int q = cst[nc]; q < cst[nc + 1]; ++q) {
      const int j = P->atom_off + q;
      if (same && c.gid[j] <= gi) continue;
      const double4 pj = c.pos[j];
      const int tj = tw_type(tw_of(pj.w));
      const int a = pm[(ti - 1) + (tj - 1) * nt], b = pm[(tj - 1) + (ti - 1) * nt];
      const int mx = a > b ? a : b;
      if (mx <= 0) continue;
      double s0 = pi.x - pj.x, s1 = pi.y - pj.y, s2 = pi.z - pj.z;
      s0 = s0 - round(s0);
      s1 = s1 - round(s1);
      s2 = s2 - round(s2);
      const double x0 = b0 * s0, x1 = b1 * s1, x2 = b2 * s2;
      double d2 = x0 * x0;
      d2 = d2 + x1 * x1;
      d2 = d2 + x2 * x2;
      if (same && d2 < ptrmin) continue;
      if (d2 > c.rlist2[P->pair_off + mx - 1]) continue;
      ++count;
    }
  }
  if (count > P->neimax_stop) set_err(c, S, E_NEIMAX);
}

__global__ __launch_bounds__(BLOCK) void k_neimax(DevCtx c) {
  for_listed(c, [&](int s, int &f, int &n) { chunk_range(c, s, f, n); },
             [&](int s, int u) { neimax_chunk(c, s, u); });
}

// the rebuild group over the systems on the rebuild list; `counting` adds
// the rebuild to each system's NlistUpdates (not for the setup builds)
void launch_rebuild(const DevCtx &c, cudaStream_t st, int counting, int mixed) {
  const int nsm = sm_count();
  const int gchunk = std::min(c.nchunks, nsm * 4);
  const int gcell = std::min((c.ncells + BLOCK / 32 - 1) / (BLOCK / 32), nsm * 4);
  k_bin<<<gchunk, BLOCK, 0, st>>>(c);
  k_scan<<<std::min(c.nsys_cap, nsm), 1024, 0, st>>>(c, counting);
  k_scatter<<<gchunk, BLOCK, 0, st>>>(c);
  k_order<<<gcell, BLOCK, 0, st>>>(c);
  k_permute<<<gchunk, BLOCK, 0, st>>>(c);
  k_copyback<<<gchunk, BLOCK, 0, st>>>(c, mixed);
  // the two forms of the list build; each returns at once unless the
  // number of listed cells (counted by k_scan) selects it
  static int gab = 0;
  if (!gab) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_build_atoms, CB_THREADS, 0);
    gab = nsm * (occ > 0 ? occ : 1);
  }
  k_build_atoms<<<gab, CB_THREADS, 0, st>>>(c);
  static int gcb = 0;
  if (!gcb) {
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_build_cells, CB_THREADS, 0);
    gcb = nsm * (occ > 0 ? occ : 1);
  }
  k_build_cells<<<gcb, CB_THREADS, 0, st>>>(c);
  if (c.any_neimax) k_neimax<<<gchunk, BLOCK, 0, st>>>(c);
}

void launch_arm(const DevCtx &c, cudaStream_t st, int nsys_cap, int sys, int nsteps, int start) {
  k_arm<<<(nsys_cap + 127) / 128, 128, 0, st>>>(c, nsys_cap, sys, nsteps, start);
}

void launch_begin_block(const DevCtx &c, cudaStream_t st, int nsys_cap, int K) {
  k_begin_block<<<(nsys_cap + 127) / 128, 128, 0, st>>>(c, nsys_cap, K);
}

// apply and clear the pending velocity scales of every system (sys < 0) or one
// sys >= 0: only that system's chunks [chunk0, chunk0 + nch) are launched
void launch_flush(const DevCtx &c, cudaStream_t st, int nsys_cap, int sys, int chunk0, int nch) {
  if (sys >= 0 && nch > 0) k_flush<<<nch, BLOCK, 0, st>>>(c, sys, chunk0);
  else if (sys < 0) k_flush<<<c.nchunks, BLOCK, 0, st>>>(c, -1, 0);
  k_clear_pend<<<(nsys_cap + 127) / 128, 128, 0, st>>>(c, nsys_cap, sys);
}

void launch_check(const DevCtx &c, cudaStream_t st, int nsys_cap) {
  k_check<<<nsys_cap, 256, 0, st>>>(c, nsys_cap);
}

void launch_scale_vel(const DevCtx &c, cudaStream_t st, int sys, double lam) {
  k_scale_vel<<<c.nchunks, BLOCK, 0, st>>>(c, sys, lam);
}

void launch_refresh_pfx(const DevCtx &c, cudaStream_t st) {
  k_refresh_pfx<<<c.nchunks, BLOCK, 0, st>>>(c);
}

}  // namespace ndg
