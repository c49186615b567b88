// ndg_context.cu -- host side of the Ndyn timestep library: contexts,
// systems, device arenas, the C ABI of include/ndyn_gpu.h and the
// graph-block dynamics loop.
//
// Device memory is organised as arenas with stable offsets: a system keeps
// its atom range, cell range and neighbour-list range until it is removed,
// so adding or retiring systems (replicas, served requests) never moves the
// state of the others and never changes a captured graph's arguments unless
// an arena has to grow.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/ndyn_gpu.h"
#include "ndg_common.h"
#include "ndg_internal.h"
#include "ndg_kernels.h"

using namespace ndg;

namespace {

thread_local std::string g_last_error;

struct Range {
  long long off = -1, len = 0;
};

// first-fit allocator over an index space that grows on demand
struct Arena {
  std::vector<std::pair<long long, long long>> used;  // sorted (off, len)
  long long cap = 0;
  long long find(long long len) const {
    long long at = 0;
    for (auto &u : used) {
      if (u.first - at >= len) return at;
      at = std::max(at, u.first + u.second);
    }
    return cap - at >= len ? at : -1;
  }
  long long end_used() const {
    long long e = 0;
    for (auto &u : used) e = std::max(e, u.first + u.second);
    return e;
  }
  void take(long long off, long long len) {
    used.emplace_back(off, len);
    std::sort(used.begin(), used.end());
  }
  void give(long long off) {
    for (size_t k = 0; k < used.size(); ++k)
      if (used[k].first == off) {
        used.erase(used.begin() + k);
        return;
      }
  }
};

struct HostSys {
  bool alive = false;
  int n = 0, ntypes = 0, npairs = 0, ptsize = 0;
  double ptrmin = 0.25;
  std::vector<double> mass, rcpair, ppair, fpair;
  std::vector<float2> tF2, tP2;  // FP32 (k, k+1) pairs of fpair and ppair
  std::vector<double4> bc;       // hold groups: displacement per step, w = axis mask
  std::vector<double4> spr;      // per pair: spring D0, sc, Vol, w = 1 (empty: no springs)
  bool ipos_set = false;         // initial positions of the spring strains uploaded
  double ibox[3] = {0, 0, 0};
  std::vector<int> pairmat;
  ndg_control ctl{};
  Range atoms, cells, nbr;  // atoms/cells in elements, nbr in ints
  int maxnb = 0, ncell_cap = 0;
  int mcell0[3] = {0, 0, 0};
  double rcut = 0.0;
  bool lists_valid = false;
  SysParam prm{};
};

// Test hook (host-side fault injection): NDG_TEST_ALLOC_LIMIT=<bytes> in the
// environment makes every device allocation above that size fail as if the
// device were full, so the growth fallbacks run without filling a GPU.
size_t alloc_limit() {
  static const size_t lim = [] {
    const char *e = getenv("NDG_TEST_ALLOC_LIMIT");
    return e ? (size_t)strtoull(e, nullptr, 10) : (size_t)0;
  }();
  return lim;
}

template <class T>
T *dalloc(size_t n) {
  void *p = nullptr;
  if (n == 0) n = 1;
  if (alloc_limit() && n * sizeof(T) > alloc_limit()) return nullptr;
  if (cudaMalloc(&p, n * sizeof(T)) != cudaSuccess) {
    // the caller reports NDG_ERR_NOMEM; the failed call must not stay the
    // runtime's last error for the next launch's check to pick up
    cudaGetLastError();
    return nullptr;
  }
  return (T *)p;
}

}  // namespace

struct ndg_ctx {
  int device = 0, precision = NDG_PREC_FP64;
  cudaStream_t st = nullptr;
  cudaStream_t st2 = nullptr;  // captures the conditional rebuild bodies
  std::string last_err;
  std::vector<HostSys> sys;
  // arenas
  Arena atoms, cells, nbrs;  // atoms in chunks, cells in cells, nbrs in ints
  int nsys_cap = 0;
  size_t cap_pm = 0, cap_pg = 0, cap_bc = 0, cap_spr = 0, cap_mass = 0, cap_rc2 = 0, cap_rlist2 = 0, cap_vdr2 = 0, cap_rc2f = 0,
         cap_tabF = 0, cap_tabP = 0, cap_tabF2 = 0, cap_tabP2 = 0;
  // device buffers
  SysParam *dP = nullptr;
  SysState *dS = nullptr;
  int *chunk_sys = nullptr, *cell_sys = nullptr;
  double4 *pos = nullptr, *s_pos = nullptr;
  int4 *pfx = nullptr;
  double *vel = nullptr, *acc = nullptr, *disp = nullptr, *force = nullptr;
  double *s_vel = nullptr, *s_acc = nullptr;
  int *gid = nullptr, *s_gid = nullptr, *s_cell = nullptr, *nnb = nullptr;
  int *hold = nullptr;     // per atom slot, by input index: hold group
  double4 *ipos = nullptr; // per atom slot, by input index: initial position
  double4 *sprd = nullptr; // spring parameters per pair of all systems
  double4 *bcd = nullptr;  // hold groups of all systems
  int *atom_cell = nullptr, *atom_slot = nullptr, *perm = nullptr, *tmp_src = nullptr,
      *tmp_key = nullptr;
  int *cxyz = nullptr;  // per atom slot: its link cell's grid coordinates (rebuild scratch)
  int *cell_count = nullptr, *cell_start = nullptr;
  int *nbr = nullptr;
  int *tile_rows = nullptr;
  char *pin = nullptr;  // pinned host staging of atom copies (reused)
  size_t pin_cap = 0;
  int *pin_words = nullptr;  // pinned copy of the status words (ring_count[0..1])
  long long *xoff = nullptr;  // bulk state transfer: each system's first atom in the
  size_t cap_xoff = 0;        // caller's concatenated arrays (-1: not a live system)
  int *rb_list = nullptr;  // systems listed for a list rebuild
  PlanEnt *plan = nullptr;  // pair-launch work plan (integrate1's extra block)
  int *plan_kb = nullptr;
  PlanHdr *plan_hdr = nullptr;
  double *red = nullptr, *itop = nullptr, *ired = nullptr;
  int *pairmat = nullptr, *pairg = nullptr;
  double *mass = nullptr, *rc2 = nullptr, *rlist2 = nullptr;
  float *vdr2 = nullptr, *rc2f = nullptr;
  double *tabF = nullptr, *tabP = nullptr;
  float2 *tabF2 = nullptr, *tabP2 = nullptr;
  ThermoRec *ring = nullptr;
  int *ring_count = nullptr;
  int ring_cap = 0;
  std::vector<int> chunk_sys_h, cell_sys_h;
  bool params_dirty = true;
  // tuning and graphs
  int tpa = 0, graph_steps = 100;
  int gather = 4;  // mixed pair loop gather depth (4 or 8)
  // atoms to threads by list length: systems whose mean full-list length
  // reaches rows_split run with tpa_long threads per atom (0: one class)
  int rows_split = 0, tpa_long = 2;
  int any_spring = 0;  // some system holds spring pairs
  int any_neimax = 0;  // some system checks the reference's NeiMax at list builds
  int stab_smem = 0;  // staged-table bytes of the pair kernel (0: tables from global)
  int stab_lean = 0;  // the same without the energy table
  std::map<int, cudaGraphExec_t> graphs;
  int captures = 0;  // graphs captured (a changed arena or layout drops them)
  // per-kernel timing of the last profiled block
  double t_int = 0, t_pair = 0, t_reb = 0;
  int t_launches = 0;
  ~ndg_ctx();
};

// ---------------------------------------------------------------------------
namespace {

int cuda_fail(ndg_ctx *c, cudaError_t e, const char *what) {
  std::string m = std::string(what) + ": " + cudaGetErrorString(e);
  if (c) c->last_err = m;
  g_last_error = m;
  return NDG_ERR_CUDA;
}

#define CK(ctx, call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return cuda_fail(ctx, _e, #call); \
  } while (0)

void drop_graphs(ndg_ctx *c) {
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
  c->graphs.clear();
}

template <class T>
void dfree(T *&p) {
  if (p) cudaFree(p);
  p = nullptr;
}

DevCtx devctx(ndg_ctx *c) {
  DevCtx d{};
  d.P = c->dP;
  d.S = c->dS;
  d.chunk_sys = c->chunk_sys;
  d.cell_sys = c->cell_sys;
  d.nchunks = (int)c->atoms.cap;
  d.ncells = (int)c->cells.cap;
  d.nsys_cap = c->nsys_cap;
  d.pos = c->pos;
  d.pfx = c->pfx;
  d.vel = c->vel;
  d.acc = c->acc;
  d.disp = c->disp;
  d.force = c->force;
  d.gid = c->gid;
  d.hold = c->hold;
  d.ipos = c->ipos;
  d.spr = c->sprd;
  d.bcd = c->bcd;
  d.nbr = c->nbr;
  d.tile_rows = c->tile_rows;
  d.gather = c->gather;
  d.any_spring = c->any_spring;
  d.any_neimax = c->any_neimax;
  d.nnb = c->nnb;
  d.atom_cell = c->atom_cell;
  d.cxyz = c->cxyz;
  d.atom_slot = c->atom_slot;
  d.cell_count = c->cell_count;
  d.cell_start = c->cell_start;
  d.perm = c->perm;
  d.tmp_src = c->tmp_src;
  d.tmp_key = c->tmp_key;
  d.s_pos = c->s_pos;
  d.s_vel = c->s_vel;
  d.s_acc = c->s_acc;
  d.s_gid = c->s_gid;
  d.s_cell = c->s_cell;
  d.pairmat = c->pairmat;
  d.pairg = c->pairg;
  d.mass = c->mass;
  d.rc2 = c->rc2;
  d.rlist2 = c->rlist2;
  d.vdr2 = c->vdr2;
  d.rc2f = c->rc2f;
  d.tabF = c->tabF;
  d.tabP = c->tabP;
  d.tabF2 = c->tabF2;
  d.tabP2 = c->tabP2;
  d.red = c->red;
  d.itop = c->itop;
  d.ired = c->ired;
  d.ring = c->ring;
  d.ring_count = c->ring_count;
  d.rb_list = c->rb_list;
  d.plan = c->plan;
  d.plan_kb = c->plan_kb;
  d.plan_hdr = c->plan_hdr;
  // the spring variant is built for one thread per atom: one class
  d.rows_split = c->any_spring ? 0 : c->rows_split;
  d.tpa_long = c->tpa_long;
  d.ring_cap = c->ring_cap;
  d.stab_smem = c->stab_smem;
  d.stab_lean = c->stab_lean;
  return d;
}

// grow a device buffer, keeping its first `keep` elements
template <class T>
int grow(ndg_ctx *c, T *&p, size_t keep, size_t n) {
  T *q = dalloc<T>(n);
  if (!q) return NDG_ERR_NOMEM;
  if (p && keep) {
    cudaError_t e = cudaMemcpy(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice);
    if (e != cudaSuccess) {
      cudaFree(q);
      return cuda_fail(c, e, "grow");
    }
  }
  dfree(p);
  p = q;
  return NDG_OK;
}

int grow_atoms(ndg_ctx *c, long long new_chunks) {
  const size_t old = (size_t)c->atoms.cap * ATOM_ALIGN, n = (size_t)new_chunks * ATOM_ALIGN;
  int rc = 0;
  rc |= grow(c, c->pos, old, n);
  rc |= grow(c, c->pfx, old, n);
  rc |= grow(c, c->vel, 3 * old, 3 * n);
  rc |= grow(c, c->acc, 3 * old, 3 * n);
  rc |= grow(c, c->disp, 3 * old, 3 * n);
  rc |= grow(c, c->force, 3 * old, 3 * n);
  rc |= grow(c, c->gid, old, n);
  rc |= grow(c, c->hold, old, n);
  rc |= grow(c, c->ipos, old, n);
  rc |= grow(c, c->nnb, old, n);
  rc |= grow(c, c->atom_cell, old, n);
  rc |= grow(c, c->atom_slot, 0, n);
  rc |= grow(c, c->perm, 0, n);
  rc |= grow(c, c->tmp_src, 0, n);
  rc |= grow(c, c->tmp_key, 0, n);
  rc |= grow(c, c->s_pos, 0, n);
  rc |= grow(c, c->s_vel, 0, 3 * n);
  rc |= grow(c, c->s_acc, 0, 3 * n);
  rc |= grow(c, c->s_gid, 0, n);
  rc |= grow(c, c->s_cell, 0, n);
  rc |= grow(c, c->cxyz, 0, n);
  rc |= grow(c, c->itop, 2 * (size_t)c->atoms.cap, 2 * (size_t)new_chunks);
  rc |= grow(c, c->ired, 0, (size_t)new_chunks);
  rc |= grow(c, c->red, 0, 8 * 32 * (size_t)new_chunks);
  rc |= grow(c, c->chunk_sys, (size_t)c->atoms.cap, (size_t)new_chunks);
  {
    const size_t t_old = 2 * (size_t)c->atoms.cap, t_new = 2 * (size_t)new_chunks;
    rc |= grow(c, c->tile_rows, t_old, t_new);
    if (!rc) cudaMemset(c->tile_rows + t_old, 0, (t_new - t_old) * sizeof(int));
  }
  // arrays reallocated before a failure have moved too: no captured graph
  // may keep their old addresses
  drop_graphs(c);
  if (rc) return NDG_ERR_NOMEM;
  c->chunk_sys_h.resize(new_chunks, -1);
  cudaMemcpy(c->chunk_sys + c->atoms.cap, c->chunk_sys_h.data() + c->atoms.cap,
             (new_chunks - c->atoms.cap) * sizeof(int), cudaMemcpyHostToDevice);
  c->atoms.cap = new_chunks;
  return NDG_OK;
}

int grow_cells(ndg_ctx *c, long long n) {
  int rc = 0;
  rc |= grow(c, c->cell_count, (size_t)c->cells.cap, (size_t)n);
  rc |= grow(c, c->cell_start, (size_t)c->cells.cap, (size_t)n);
  rc |= grow(c, c->cell_sys, (size_t)c->cells.cap, (size_t)n);
  drop_graphs(c);  // arrays reallocated before a failure have moved too
  if (rc) return NDG_ERR_NOMEM;
  cudaMemset(c->cell_count + c->cells.cap, 0, (n - c->cells.cap) * sizeof(int));
  c->cell_sys_h.resize(n, -1);
  cudaMemcpy(c->cell_sys + c->cells.cap, c->cell_sys_h.data() + c->cells.cap,
             (n - c->cells.cap) * sizeof(int), cudaMemcpyHostToDevice);
  c->cells.cap = n;
  return NDG_OK;
}

int grow_nbr(ndg_ctx *c, long long n) {
  if (grow(c, c->nbr, (size_t)c->nbrs.cap, (size_t)n)) {
    drop_graphs(c);
    return NDG_ERR_NOMEM;
  }
  c->nbrs.cap = n;
  drop_graphs(c);
  return NDG_OK;
}

int grow_sys(ndg_ctx *c, int n) {
  int rc = 0;
  rc |= grow(c, c->dP, (size_t)c->nsys_cap, (size_t)n);
  rc |= grow(c, c->dS, (size_t)c->nsys_cap, (size_t)n);
  rc |= grow(c, c->rb_list, 0, (size_t)n);
  rc |= grow(c, c->plan, 0, (size_t)PLAN_NL * n);
  if (!c->plan_kb) rc |= grow(c, c->plan_kb, 0, (size_t)PLAN_NL * PLAN_GMAX);
  if (!c->plan_hdr) rc |= grow(c, c->plan_hdr, 0, 1);
  if (rc) return NDG_ERR_NOMEM;
  drop_graphs(c);
  std::vector<SysParam> z(n - c->nsys_cap);
  std::vector<SysState> zs(n - c->nsys_cap);
  memset(z.data(), 0, z.size() * sizeof(SysParam));
  memset(zs.data(), 0, zs.size() * sizeof(SysState));
  cudaMemcpy(c->dP + c->nsys_cap, z.data(), z.size() * sizeof(SysParam), cudaMemcpyHostToDevice);
  cudaMemcpy(c->dS + c->nsys_cap, zs.data(), zs.size() * sizeof(SysState),
             cudaMemcpyHostToDevice);
  c->nsys_cap = n;
  // thermo ring: graph_steps records per system
  const int need = std::max(256, c->graph_steps * n);
  if (need > c->ring_cap) {
    dfree(c->ring);
    c->ring = dalloc<ThermoRec>(need);
    if (!c->ring) return NDG_ERR_NOMEM;
    c->ring_cap = need;
  }
  drop_graphs(c);
  return NDG_OK;
}

// grow an arena of capacity cap to hold need: 2x, else 1.5x, 1.25x, the
// exact need, the first that the device can allocate
template <class F>
int grow_ladder(long long need, long long cap, F grow_to) {
  static const double steps[] = {2.0, 1.5, 1.25};
  for (double f : steps) {
    const long long want = (long long)(f * (double)cap);
    if (want <= need) break;
    const int rc = grow_to(want);
    if (rc != NDG_ERR_NOMEM) return rc;
  }
  return grow_to(need);
}

// Allocate `len` units in an arena, growing the device buffers if needed.
long long arena_take(ndg_ctx *c, Arena &a, long long len, int which) {
  long long off = a.find(len);
  if (off < 0) {
    // each growth copies and re-captures: double, or where the doubled
    // arena does not fit the device, the largest of 1.5x, 1.25x and the
    // exact need that does (headroom keeps later admissions from growing
    // again, each a copy of the whole arena)
    const long long need = a.end_used() + len;
    const int rc = grow_ladder(need, a.cap, [&](long long want) {
      return which == 0 ? grow_atoms(c, want) : which == 1 ? grow_cells(c, want) : grow_nbr(c, want);
    });
    if (rc) return -1;
    off = a.find(len);
    if (off < 0) return -1;
  }
  a.take(off, len);
  return off;
}

// copy a host vector to a device array, reallocating (with headroom) when
// it no longer fits; a reallocation invalidates captured graphs
template <class T>
int upload_vec(ndg_ctx *c, T *&dst, size_t &cap, const std::vector<T> &v) {
  if (!dst || v.size() > cap) {
    dfree(dst);
    cap = std::max<size_t>(v.size() * 2, 64);
    dst = dalloc<T>(cap);
    if (!dst) return NDG_ERR_NOMEM;
    drop_graphs(c);
  }
  if (!v.empty() && cudaMemcpy(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice))
    return NDG_ERR_CUDA;
  return NDG_OK;
}

// the rebuild group runs the NeiMax check while some system needs it
void note_neimax(ndg_ctx *c) {
  int any = 0;
  for (auto &h : c->sys)
    if (h.alive && h.prm.neimax_stop > 0) any = 1;
  if (any != c->any_neimax) {
    c->any_neimax = any;
    drop_graphs(c);
  }
}

// small per-pair/per-type arrays: rebuilt for all systems on any change
int upload_params(ndg_ctx *c) {
  std::vector<int> pm, pg;
  std::vector<double4> bc, spr;
  std::vector<double> mass, rc2, rlist2, tabF, tabP;
  std::vector<float> vdr2, rc2f;
  std::vector<float2> tF2, tP2;
  std::vector<SysParam> prm(c->nsys_cap);
  memset(prm.data(), 0, prm.size() * sizeof(SysParam));
  size_t ntab = 0;
  for (auto &h : c->sys)
    if (h.alive) ntab += h.fpair.size();
  tabF.reserve(ntab);
  tabP.reserve(ntab);
  tF2.reserve(ntab);
  tP2.reserve(ntab);
  for (size_t s = 0; s < c->sys.size(); ++s) {
    HostSys &h = c->sys[s];
    if (!h.alive) continue;
    SysParam &p = h.prm;
    p.tab_off = (int)tabF.size();
    p.pair_off = (int)rc2.size();
    p.type_off = (int)mass.size();
    p.pm_off = (int)pm.size();
    pm.insert(pm.end(), h.pairmat.begin(), h.pairmat.end());
    p.bc_off = (int)bc.size();
    p.nhold = (int)h.bc.size();
    bc.insert(bc.end(), h.bc.begin(), h.bc.end());
    p.nspring = 0;
    for (auto &q : h.spr) p.nspring += q.w != 0.0;
    for (int d = 0; d < 3; ++d) p.ibox[d] = h.ibox[d];
    for (int b = 1; b <= h.ntypes; ++b)
      for (int a = 1; a <= h.ntypes; ++a) pg.push_back(gather_entry(h.pairmat.data(), h.ntypes, a, b));
    mass.insert(mass.end(), h.mass.begin(), h.mass.end());
    const double skin = h.ctl.skin < 0 ? 0.2 * h.rcut : h.ctl.skin;
    for (int j = 0; j < h.npairs; ++j) {
      const double r = h.rcpair[j];
      const double prc2 = r * r;
      const double pdr2 = (prc2 - h.ptrmin) / (h.ptsize - 1);
      // a spring pair has no cutoff test: cutoff words of -1 keep it out of
      // the kernels' table loops, and their spring pass applies the strain rule
      const bool spring = !h.spr.empty() && h.spr[j].w != 0.0;
      rc2.push_back(spring ? -1.0 : prc2);
      rc2f.push_back(spring ? -1.0f : (float)prc2);
      spr.push_back(h.spr.empty() ? make_double4(0, 0, 0, 0) : h.spr[j]);
      vdr2.push_back((float)(1.0 / pdr2));  // vPTdr2 = real(1.d0/PTdr2), src/nd.f90:254
      const double rl = skin + r;            // rcuts2 = skin + PairParams(1,.), :1375
      rlist2.push_back(rl * rl);
    }
    tabF.insert(tabF.end(), h.fpair.begin(), h.fpair.end());
    tabP.insert(tabP.end(), h.ppair.begin(), h.ppair.end());
    tF2.insert(tF2.end(), h.tF2.begin(), h.tF2.end());
    tP2.insert(tP2.end(), h.tP2.begin(), h.tP2.end());
    prm[s] = p;
  }
  // contexts with spring pairs run the pair kernels' spring variant
  int anys = 0;
  for (auto &h : c->sys)
    if (h.alive && !h.spr.empty()) anys = 1;
  if (anys != c->any_spring) {
    c->any_spring = anys;
    drop_graphs(c);
  }
  note_neimax(c);
  // stage the tables in shared memory when every system's fit (B200 allows
  // 227 KB per block; keep room for two resident blocks per SM)
  int stab = 0, lean = 0;
  for (auto &h : c->sys)
    if (h.alive) {
      stab = std::max(stab, stab_bytes(h.ntypes, h.npairs, h.ptsize));
      lean = std::max(lean, stab_bytes_lean(h.ntypes, h.npairs, h.ptsize));
    }
  if (stab > 100 * 1024) stab = lean = 0;
  // a high-water mark while systems come and go (a change re-captures the
  // step graphs), unless staging is off or no system is left
  bool any = false;
  for (auto &h : c->sys) any |= h.alive;
  if (stab > 0 && c->stab_smem > 0 && any) {
    stab = std::max(stab, c->stab_smem);
    lean = std::max(lean, c->stab_lean);
  }
  if (stab != c->stab_smem || lean != c->stab_lean) {
    c->stab_smem = stab;
    c->stab_lean = lean;
    drop_graphs(c);
  }
  int rc = 0;
  rc |= upload_vec(c, c->pairmat, c->cap_pm, pm);
  rc |= upload_vec(c, c->pairg, c->cap_pg, pg);
  rc |= upload_vec(c, c->bcd, c->cap_bc, bc);
  rc |= upload_vec(c, c->sprd, c->cap_spr, spr);
  rc |= upload_vec(c, c->mass, c->cap_mass, mass);
  rc |= upload_vec(c, c->rc2, c->cap_rc2, rc2);
  rc |= upload_vec(c, c->rlist2, c->cap_rlist2, rlist2);
  rc |= upload_vec(c, c->vdr2, c->cap_vdr2, vdr2);
  rc |= upload_vec(c, c->rc2f, c->cap_rc2f, rc2f);
  rc |= upload_vec(c, c->tabF, c->cap_tabF, tabF);
  rc |= upload_vec(c, c->tabP, c->cap_tabP, tabP);
  rc |= upload_vec(c, c->tabF2, c->cap_tabF2, tF2);
  rc |= upload_vec(c, c->tabP2, c->cap_tabP2, tP2);
  if (rc) return NDG_ERR_NOMEM;
  CK(c, cudaMemcpy(c->dP, prm.data(), prm.size() * sizeof(SysParam), cudaMemcpyHostToDevice));
  c->params_dirty = false;
  return NDG_OK;
}

// upload the per-pair/per-type arrays once before the next launch that
// needs them, so that adding many systems stays linear in their number
int ensure_params(ndg_ctx *c) { return c->params_dirty ? upload_params(c) : NDG_OK; }

// the per-system records alone, when only ranges, grids or list capacities
// changed (their table offsets are those of the last full upload)
int upload_sysparams(ndg_ctx *c) {
  note_neimax(c);
  std::vector<SysParam> prm(c->nsys_cap);
  memset(prm.data(), 0, prm.size() * sizeof(SysParam));
  for (size_t s = 0; s < c->sys.size(); ++s)
    if (c->sys[s].alive) prm[s] = c->sys[s].prm;
  CK(c, cudaMemcpy(c->dP, prm.data(), prm.size() * sizeof(SysParam), cudaMemcpyHostToDevice));
  return NDG_OK;
}

void fill_control_params(HostSys &h) {
  SysParam &p = h.prm;
  const ndg_control &q = h.ctl;
  p.dt = q.dt;
  p.skin = q.skin < 0 ? 0.2 * h.rcut : q.skin;
  p.skinsq = p.skin * p.skin;
  p.rlist = h.rcut + p.skin;
  p.renei = q.renei;
  p.renei_freq = q.renei_freq;
  p.out_steps = q.out_steps;
  p.isokinetic = q.isokinetic;
  p.ke_freq = q.ke_freq;
  p.ke_target = q.ke_target;
  p.ke_parm = q.ke_parm;
  p.isobaric = q.isobaric;
  p.p_freq = q.p_freq;
  for (int d = 0; d < 3; ++d) p.p_target[d] = q.p_target[d];
  p.p_parm = q.p_parm;
  p.isoenergetic = q.isoenergetic;
  p.e_freq = q.e_freq;
  p.e_parm = q.e_parm;
  p.box_load = q.box_load;
  for (int d = 0; d < 3; ++d) p.box_vel[d] = q.box_vel[d];
  p.quirk = q.quirk;
  p.ptrmin = h.ptrmin;
  p.ntypes = h.ntypes;
  p.npairs = h.npairs;
  p.ptsize = h.ptsize;
}

bool valid_sys(ndg_ctx *c, int s) {
  return c && s >= 0 && s < (int)c->sys.size() && c->sys[s].alive;
}

int get_state_dev(ndg_ctx *c, int s, SysState &S) {
  CK(c, cudaMemcpy(&S, c->dS + s, sizeof(SysState), cudaMemcpyDeviceToHost));
  return NDG_OK;
}
int put_state_dev(ndg_ctx *c, int s, const SysState &S) {
  CK(c, cudaMemcpy(c->dS + s, &S, sizeof(SysState), cudaMemcpyHostToDevice));
  return NDG_OK;
}

// upload atoms in caller order (identity permutation)
// pinned host memory of at least `bytes` for the atom copies, or nullptr
char *pinned(ndg_ctx *c, size_t bytes) {
  if (bytes <= c->pin_cap) return c->pin;
  if (c->pin) cudaFreeHost(c->pin);
  c->pin = nullptr;
  const size_t want = std::max(bytes, c->pin_cap + c->pin_cap / 2);
  c->pin_cap = 0;
  if (cudaHostAlloc((void **)&c->pin, want, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    c->pin = nullptr;
    return nullptr;
  }
  c->pin_cap = want;
  return c->pin;
}

int upload_atoms(ndg_ctx *c, int s, const int *typ, const double *pos, const double *vel,
                 const double *acc) {
  HostSys &h = c->sys[s];
  const int n = h.n;
  const size_t off = (size_t)h.atoms.off * ATOM_ALIGN;
  // staged in pinned memory: positions (with type words) | slots | velocities
  // | accelerations, then copied in one stream-ordered batch
  const size_t bp = (size_t)n * sizeof(double4), bg = ((size_t)n * sizeof(int) + 15) / 16 * 16;
  const size_t b3 = 3 * (size_t)n * sizeof(double);
  const size_t total = bp + bg + (vel ? b3 : 0) + (acc ? b3 : 0);
  std::vector<char> pageable;
  char *buf = pinned(c, total);
  if (!buf) {
    pageable.resize(total);
    buf = pageable.data();
  }
  double4 *p4 = (double4 *)buf;
  int *g = (int *)(buf + bp);
  double *vs = (double *)(buf + bp + bg), *as = vs + (vel ? 3 * (size_t)n : 0);
  std::vector<int> tw(n);
  if (typ) {
    for (int i = 0; i < n; ++i) tw[i] = pack_tw(typ[i], s);
  } else {
    // keep the types already on the device (they are in pos.w, device
    // order), read through the same staging
    CK(c, cudaMemcpyAsync(p4, c->pos + off, bp, cudaMemcpyDeviceToHost, c->st));
    CK(c, cudaMemcpyAsync(g, c->gid + off, n * sizeof(int), cudaMemcpyDeviceToHost, c->st));
    CK(c, cudaStreamSynchronize(c->st));
    for (int i = 0; i < n; ++i) {
      long long w;
      memcpy(&w, &p4[i].w, 8);
      tw[g[i]] = (int)w;
    }
  }
  for (int i = 0; i < n; ++i) {
    const long long w = (long long)(unsigned)tw[i];
    double wd;
    memcpy(&wd, &w, 8);
    p4[i] = make_double4(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], wd);
    g[i] = i;
  }
  if (vel) memcpy(vs, vel, b3);
  if (acc) memcpy(as, acc, b3);
  cudaStream_t st = c->st;
  CK(c, cudaMemcpyAsync(c->pos + off, p4, bp, cudaMemcpyHostToDevice, st));
  CK(c, cudaMemcpyAsync(c->gid + off, g, n * sizeof(int), cudaMemcpyHostToDevice, st));
  if (vel) CK(c, cudaMemcpyAsync(c->vel + 3 * off, vs, b3, cudaMemcpyHostToDevice, st));
  else CK(c, cudaMemsetAsync(c->vel + 3 * off, 0, b3, st));
  if (acc) CK(c, cudaMemcpyAsync(c->acc + 3 * off, as, b3, cudaMemcpyHostToDevice, st));
  else CK(c, cudaMemsetAsync(c->acc + 3 * off, 0, b3, st));
  CK(c, cudaMemsetAsync(c->disp + 3 * off, 0, b3, st));
  CK(c, cudaStreamSynchronize(st));  // the staging buffer is reused
  h.lists_valid = false;
  return NDG_OK;
}

std::vector<int> live_systems(ndg_ctx *c) {
  std::vector<int> ids;
  for (size_t s = 0; s < c->sys.size(); ++s)
    if (c->sys[s].alive) ids.push_back((int)s);
  return ids;
}

// put the given systems on the rebuild list
int list_systems(ndg_ctx *c, const std::vector<int> &ids) {
  const int n = (int)ids.size();
  if (n) CK(c, cudaMemcpy(c->rb_list, ids.data(), n * sizeof(int), cudaMemcpyHostToDevice));
  CK(c, cudaMemcpy(c->ring_count + 3, &n, sizeof(int), cudaMemcpyHostToDevice));
  return NDG_OK;
}

int list_all_systems(ndg_ctx *c) { return list_systems(c, live_systems(c)); }

// dynamics prologue, src/nd.f90:73-108, for the given systems: skin default,
// MCELL, neighbour capacity; then one rebuild of their lists (the other
// systems are left as they are)
// initPositionSet (src/nd.f90:1731-1762): the spring strains' reference
// positions (input order; nullptr = the current ones) and box (nullptr =
// the current one)
int init_positions(ndg_ctx *c, int s, const double *ipos, const double *ibox) {
  HostSys &h = c->sys[s];
  std::vector<double> cur;
  if (!ipos) {
    cur.resize(3 * (size_t)h.n);
    int rc = ndg_get_state(c, s, cur.data(), nullptr, nullptr, nullptr);
    if (rc) return rc;
    ipos = cur.data();
  }
  std::vector<double4> p4(h.n);
  for (int i = 0; i < h.n; ++i)
    p4[i] = make_double4(ipos[3 * i], ipos[3 * i + 1], ipos[3 * i + 2], 0.0);
  CK(c, cudaMemcpy(c->ipos + (size_t)h.atoms.off * ATOM_ALIGN, p4.data(),
                   h.n * sizeof(double4), cudaMemcpyHostToDevice));
  if (ibox) {
    for (int d = 0; d < 3; ++d) h.ibox[d] = ibox[d];
  } else {
    SysState S;
    int rc = get_state_dev(c, s, S);
    if (rc) return rc;
    for (int d = 0; d < 3; ++d) h.ibox[d] = S.box[d];
  }
  h.ipos_set = true;
  c->params_dirty = true;
  return NDG_OK;
}

int setup_lists(ndg_ctx *c, const std::vector<int> &which) {
  // every system's state record read and written once (not one round trip
  // per system), and the cell owners uploaded once
  std::vector<SysState> Sall(c->nsys_cap);
  CK(c, cudaMemcpy(Sall.data(), c->dS, Sall.size() * sizeof(SysState), cudaMemcpyDeviceToHost));
  bool cells_moved = false;
  for (int s : which) {
    HostSys &h = c->sys[s];
    if (!h.alive) continue;
    if (!h.spr.empty() && !h.ipos_set) {
      // the dynamics prologue takes the current positions (src/nd.f90:104)
      int rc = init_positions(c, s, nullptr, nullptr);
      if (rc) return rc;
    }
    if (h.ctl.skin < 0) h.ctl.skin = 0.2 * h.rcut;  // persists, as in the reference
    fill_control_params(h);
    SysState &S = Sall[s];
    int rc = 0;
    int nc = 1;
    for (int d = 0; d < 3; ++d) {
      h.mcell0[d] = (int)(S.box[d] / (h.rcut + h.prm.skin));
      if (h.mcell0[d] < 2) return NDG_ERR_CELLS;
      nc *= h.mcell0[d];
      h.prm.mcell0[d] = h.mcell0[d];
      S.mcell[d] = h.mcell0[d];
    }
    S.ncell = nc;
    // neighbour capacity of the full list: sphere of radius 1.1*(rcut+skin)
    // at the mean density (the reference's NeiMax estimate counts the same
    // sphere, src/nd.f90:84-88), doubled where the reference stencil repeats
    // pairs (a cell count of 2 in ref semantics)
    const double vol = S.box[0] * S.box[1] * S.box[2];
    if (h.ctl.quirk == NDG_QUIRK_REF && h.ctl.neimax == 0) {
      // NeiMax = int(4./3.*PI*((rcut+skin)*1.1)**3*np/(box(1)*box(2)*box(3))),
      // src/nd.f90:84-88, with 4./3. and 1.1 default (single precision) reals;
      // the value persists, as the reference's module variable does
      const double f43 = (double)(4.0f / 3.0f), rr = (h.rcut + h.prm.skin) * (double)1.1f;
      h.ctl.neimax = (int)(f43 * 3.141592653589793 * (rr * rr * rr) * (double)h.n / vol);
    }
    // the reference semantics stop where a half list outgrows NeiMax
    // (k_neimax); the fixed semantics size the lists and only stop where
    // the device capacity itself runs out
    h.prm.neimax_stop = h.ctl.quirk == NDG_QUIRK_REF ? std::max(h.ctl.neimax, 0) : 0;
    const double r = (h.rcut + h.prm.skin) * 1.1;
    double est = 4.0 / 3.0 * 3.141592653589793 * r * r * r * h.n / vol;
    if (h.ctl.quirk == NDG_QUIRK_REF &&
        (h.mcell0[0] == 2 || h.mcell0[1] == 2 || h.mcell0[2] == 2))
      est *= 2.0;
    int maxnb = (int)(est * 1.2) + 16;
    if (h.ctl.neimax > 0) maxnb = std::max(maxnb, 2 * h.ctl.neimax);
    maxnb = std::min((maxnb + 7) / 8 * 8, std::max(h.n - 1, 8) * (h.ctl.quirk == 0 ? 2 : 1) + 8);
    // list capacity: a tile's lists up to 512 entries each are assembled in
    // shared memory, longer ones by the build's direct path
    maxnb = std::min(maxnb, 4096);
    const long long npad = (long long)h.atoms.len * ATOM_ALIGN;
    if (maxnb > h.maxnb) {
      if (h.nbr.off >= 0) c->nbrs.give(h.nbr.off);
      const long long off = arena_take(c, c->nbrs, (long long)maxnb * npad, 2);
      if (off < 0) return NDG_ERR_NOMEM;
      h.nbr.off = off;
      h.nbr.len = (long long)maxnb * npad;
      h.maxnb = maxnb;
    }
    if (nc + 1 > h.ncell_cap) {
      if (h.cells.off >= 0) {
        c->cells.give(h.cells.off);
        for (long long q = h.cells.off; q < h.cells.off + h.cells.len; ++q) c->cell_sys_h[q] = -1;
      }
      const long long off = arena_take(c, c->cells, nc + 1, 1);
      if (off < 0) return NDG_ERR_NOMEM;
      h.cells.off = off;
      h.cells.len = nc + 1;
      h.ncell_cap = nc + 1;
      for (long long q = off; q < off + nc; ++q) c->cell_sys_h[q] = (int)s;
      cells_moved = true;
    }
    h.prm.atom_off = (int)(h.atoms.off * ATOM_ALIGN);
    h.prm.n = h.n;
    h.prm.npad = (int)npad;
    h.prm.cell_off = (int)h.cells.off;
    h.prm.ncell_cap = h.ncell_cap;
    h.prm.nbr_off = h.nbr.off;
    h.prm.maxnb = h.maxnb;
    // mixed precision lists of systems under 65,536 atom slots are packed as
    // 16-bit offsets, two per word: half the list bytes to write and stream
    h.prm.nb16 = (c->precision == NDG_PREC_MIXED && npad <= 65536) ? 1 : 0;
    S.nlist_updates = 0;
    S.rebuild = 0;
    S.err = 0;
    S.pend = 0;
    for (int d = 0; d < 3; ++d) S.box_build[d] = S.box[d];
  }
  if (cells_moved)
    CK(c, cudaMemcpy(c->cell_sys, c->cell_sys_h.data(), c->cells.cap * sizeof(int),
                     cudaMemcpyHostToDevice));
  CK(c, cudaMemcpy(c->dS, Sall.data(), Sall.size() * sizeof(SysState), cudaMemcpyHostToDevice));
  // the prologue changes only the systems' ranges and grids: the tables go
  // up again only when something else changed them
  int rc = c->params_dirty ? upload_params(c) : upload_sysparams(c);
  if (rc) return rc;
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  rc = list_systems(c, which);
  if (rc) return rc;
  DevCtx d = devctx(c);
  launch_rebuild(d, c->st, 0, c->precision == NDG_PREC_MIXED);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  CK(c, cudaMemset(c->ring_count + 3, 0, sizeof(int)));
  int words[4];
  CK(c, cudaMemcpy(words, c->ring_count, sizeof(words), cudaMemcpyDeviceToHost));
  if (words[1]) {
    if (words[1] & E_NEIMAX) return NDG_ERR_NEIMAX;
    if (words[1] & E_OUT_OF_BOX) return NDG_ERR_OUT_OF_BOX;
    return NDG_ERR_CELLS;
  }
  for (int s : which)
    if (c->sys[s].alive) c->sys[s].lists_valid = true;
  return NDG_OK;
}

int setup_lists(ndg_ctx *c) { return setup_lists(c, live_systems(c)); }

int choose_tpa(ndg_ctx *c) {
  if (c->tpa > 0) return c->tpa;
  long long atoms = 0;
  double nb = 0.0;
  for (auto &h : c->sys)
    if (h.alive) {
      atoms += h.n;
      nb += (double)h.n * std::max(h.maxnb / 1.5, 8.0);
    }
  if (!atoms) return 1;
  nb /= atoms;
  // more threads per atom only while there are too few atoms to fill the
  // 148 SMs: with enough atoms one thread per atom gathers best
  (void)nb;
  int t = 1;
  while (t < 8 && (double)atoms * t < 148.0 * 1024.0) t *= 2;
  return t;
}

void enqueue_steps(ndg_ctx *c, int nsteps) {
  DevCtx d = devctx(c);
  const int mixed = c->precision == NDG_PREC_MIXED;
  const int tpa = choose_tpa(c);
  for (int k = 0; k < nsteps; ++k) {
    launch_rebuild(d, c->st, 1, mixed);
    launch_integrate1(d, c->st, 0, mixed, tpa);
    launch_pair(d, c->st, tpa, mixed, 1, 0);
  }
}

int check_words(ndg_ctx *c, int *count) {
  // read through pinned memory: a copy into pageable memory goes through
  // the driver's staging and wakes the host late
  int local[2];
  int *words = c->pin_words ? c->pin_words : local;
  CK(c, cudaMemcpyAsync(words, c->ring_count, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->st));
  CK(c, cudaStreamSynchronize(c->st));
  *count = words[0];
  if (words[1] & E_NEIMAX) return NDG_ERR_NEIMAX;
  if (words[1] & E_OUT_OF_BOX) return NDG_ERR_OUT_OF_BOX;
  if (words[1] & E_CELLS) return NDG_ERR_CELLS;
  return NDG_OK;
}

int drain_ring(ndg_ctx *c, int count, ndg_thermo_cb cb, void *user) {
  if (count <= 0) return NDG_OK;
  const int n = std::min(count, c->ring_cap);
  std::vector<ThermoRec> r(n);
  CK(c, cudaMemcpy(r.data(), c->ring, n * sizeof(ThermoRec), cudaMemcpyDeviceToHost));
  CK(c, cudaMemset(c->ring_count, 0, sizeof(int)));
  std::stable_sort(r.begin(), r.end(), [](const ThermoRec &a, const ThermoRec &b) {
    return a.step != b.step ? a.step < b.step : a.sys < b.sys;
  });
  if (cb)
    for (auto &t : r) cb(reinterpret_cast<const ndg_thermo *>(&t), user);
  return NDG_OK;
}

// Capture a block of g steps as one graph.  Each step's list-rebuild group
// sits in a conditional IF node whose handle the previous step's pair
// kernel sets when a system's CheckListUpdate fires (the first step's is
// seeded by k_decide), so steps without a rebuild launch no rebuild kernel.
int capture_block(ndg_ctx *c, int g, cudaGraphExec_t *out) {
  DevCtx d = devctx(c);
  const int mixed = c->precision == NDG_PREC_MIXED;
  const int tpa = choose_tpa(c);
  if (!c->st2) CK(c, cudaStreamCreate(&c->st2));
  cudaGraph_t graph;
  CK(c, cudaGraphCreate(&graph, 0));
  std::vector<cudaGraphConditionalHandle> h(g);
  for (int k = 0; k < g; ++k)
    CK(c, cudaGraphConditionalHandleCreate(&h[k], graph, 0, cudaGraphCondAssignDefault));
  CK(c, cudaStreamBeginCaptureToGraph(c->st, graph, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal));
  launch_decide(d, c->st, h[0]);
  for (int k = 0; k < g; ++k) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg;
    const cudaGraphNode_t *deps = nullptr;
    size_t ndeps = 0;
    CK(c, cudaStreamGetCaptureInfo(c->st, &cs, nullptr, &cg, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h[k];
    cp.conditional.type = cudaGraphCondTypeIf;
    cp.conditional.size = 1;
    cudaGraphNode_t cn;
    CK(c, cudaGraphAddNode(&cn, cg, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    CK(c, cudaStreamUpdateCaptureDependencies(c->st, &cn, 1, cudaStreamSetCaptureDependencies));
    CK(c, cudaStreamBeginCaptureToGraph(c->st2, body, nullptr, nullptr, 0,
                                        cudaStreamCaptureModeThreadLocal));
    launch_rebuild(d, c->st2, 1, mixed);
    cudaGraph_t body_out;
    CK(c, cudaStreamEndCapture(c->st2, &body_out));
    launch_integrate1(d, c->st, 0, mixed, tpa);
    launch_pair(d, c->st, tpa, mixed, 1, 0, k + 1 < g ? (unsigned long long)h[k + 1] : 0ull);
  }
  cudaGraph_t done;
  CK(c, cudaStreamEndCapture(c->st, &done));
  cudaError_t e = cudaGraphInstantiate(out, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return cuda_fail(c, e, "cudaGraphInstantiate");
  return NDG_OK;
}

// Run nsteps as blocks of up to graph_steps: each block's head gives every
// armed system its share of the block (k_begin_block), then the block runs
// as one captured graph (or as eager launches when graph_steps is 1).
int run_blocks(ndg_ctx *c, int nsteps, ndg_thermo_cb cb, void *user, bool flush_end = false) {
  int left = nsteps;
  while (left > 0) {
    const int g = std::min(left, std::max(c->graph_steps, 1));
    {
      DevCtx d = devctx(c);
      launch_begin_block(d, c->st, c->nsys_cap, g);
    }
    cudaGraphExec_t exec = nullptr;
    auto it = c->graphs.find(g);
    if (it != c->graphs.end()) {
      exec = it->second;
    } else if (c->graph_steps > 1) {
      int rc = capture_block(c, g, &exec);
      if (rc) return rc;
      c->graphs[g] = exec;
      c->captures += 1;
    }
    if (exec) {
      CK(c, cudaGraphLaunch(exec, c->st));
    } else {
      enqueue_steps(c, g);
      CK(c, cudaGetLastError());
    }
    if (flush_end && left == g) {
      // the run's last block: its pending velocity scales are applied in
      // the same stream batch, so one host wait covers both
      DevCtx d = devctx(c);
      launch_flush(d, c->st, c->nsys_cap, -1);
    }
    int count = 0;
    int rc = check_words(c, &count);
    if (rc) return rc;
    rc = drain_ring(c, count, cb, user);
    if (rc) return rc;
    left -= g;
  }
  return NDG_OK;
}

int flush_pending(ndg_ctx *c, int sys = -1) {
  DevCtx d = devctx(c);
  if (sys >= 0) {
    // the system's own chunks only (a context may hold thousands of systems)
    const HostSys &h = c->sys[sys];
    launch_flush(d, c->st, c->nsys_cap, sys, (int)h.atoms.off, (int)h.atoms.len);
  } else {
    launch_flush(d, c->st, c->nsys_cap, -1);
  }
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  return NDG_OK;
}

int status_from_words(ndg_ctx *c) {
  int count;
  return check_words(c, &count);
}

}  // namespace

ndg_ctx::~ndg_ctx() {
  drop_graphs(this);
  void *ptrs[] = {dP, dS, chunk_sys, cell_sys, pos, s_pos, pfx, vel, acc, disp, force, s_vel,
                  s_acc, gid, s_gid, s_cell, cxyz, nnb, hold, bcd, ipos, sprd, atom_cell, atom_slot, perm, tmp_src, tmp_key,
                  cell_count, cell_start, rb_list, plan, plan_kb, plan_hdr, nbr, tile_rows, red, itop, ired, pairmat, pairg, mass, rc2, rlist2,
                  vdr2, rc2f, tabF, tabP, tabF2, tabP2, ring, ring_count};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  if (pin) cudaFreeHost(pin);
  if (pin_words) cudaFreeHost(pin_words);
  if (xoff) cudaFree(xoff);
  if (st) cudaStreamDestroy(st);
  if (st2) cudaStreamDestroy(st2);
}

// ---------------------------------------------------------------------------
namespace ndg_internal {

int setup_systems(ndg_ctx *c, const std::vector<int> &ids) {
  if (!c) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  return setup_lists(c, ids);
}

int arm_built(ndg_ctx *c, int sys, int nsteps) {
  if (!valid_sys(c, sys)) return NDG_ERR_ARG;
  DevCtx d = devctx(c);
  launch_arm(d, c->st, c->nsys_cap, sys, nsteps, START_BUILT);
  CK(c, cudaGetLastError());
  return NDG_OK;
}

int run_block(ndg_ctx *c, int K, ndg_thermo_cb cb, void *user) {
  if (!c || K < 1) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = ensure_params(c);
  if (rc) return rc;
  CK(c, cudaMemset(c->ring_count, 0, 2 * sizeof(int)));
  return run_blocks(c, K, cb, user);
}

int flush_system(ndg_ctx *c, int sys) {
  if (!valid_sys(c, sys)) return NDG_ERR_ARG;
  return flush_pending(c, sys);
}

int graph_captures(ndg_ctx *c) { return c ? c->captures : 0; }

int reserve_atoms(ndg_ctx *c, long long atoms) {
  if (!c || atoms < 0) return NDG_ERR_ARG;
  // every system's range is padded to whole chunks
  const long long need = c->atoms.end_used() + (atoms + ATOM_ALIGN - 1) / ATOM_ALIGN;
  if (need <= c->atoms.cap) return NDG_OK;
  cudaSetDevice(c->device);
  return grow_ladder(need, c->atoms.cap, [&](long long want) { return grow_atoms(c, want); });
}

int take_system_error(ndg_ctx *c, int sys, int *err) {
  if (!valid_sys(c, sys) || !err) return NDG_ERR_ARG;
  SysState S;
  int rc = get_state_dev(c, sys, S);
  if (rc) return rc;
  *err = S.err;
  if (S.err) {
    S.err = 0;
    rc = put_state_dev(c, sys, S);
  }
  return rc;
}

}  // namespace ndg_internal

// ===========================================================================
// C ABI
extern "C" {

int ndg_abi_version(void) { return NDG_ABI_VERSION; }

const char *ndg_error_string(int s) {
  switch (s) {
    case NDG_OK: return "ok";
    case NDG_ERR_ARG: return "invalid argument or call order";
    case NDG_ERR_NEIMAX: return "too many neighbours in list";
    case NDG_ERR_OUT_OF_BOX: return "Particle outside of box";
    case NDG_ERR_POTENTIAL: return "no potential available for potential type";
    case NDG_ERR_CELLS: return "fewer than 2 link cells in a direction (box < 2*(rcut+skin))";
    case NDG_ERR_NOMEM: return "device memory exhausted";
    case NDG_ERR_CUDA: return "CUDA runtime error";
    case NDG_ERR_BUDGET: return "request exceeds the HBM budget";
    case NDG_ERR_NOT_FOUND: return "unknown system or request";
    case NDG_ERR_TIMEOUT: return "bounded wait expired";
    default: return "unknown status";
  }
}

const char *ndg_last_error(const ndg_ctx *c) {
  return c ? c->last_err.c_str() : g_last_error.c_str();
}

void ndg_default_control(ndg_control *q) {
  memset(q, 0, sizeof(*q));
  q->dt = 0.0001;  // src/read_input.f90:19-41
  q->skin = -1.0;
  q->neimax = 0;
  q->renei = 1;
  q->renei_freq = 1;
  q->out_steps = 40;
  q->step = 0;
  q->ke_freq = q->p_freq = q->e_freq = 1;
  q->quirk = NDG_QUIRK_REF;
}

int ndg_create(ndg_ctx **out, int device, int precision) {
  if (!out || (precision != NDG_PREC_FP64 && precision != NDG_PREC_MIXED)) return NDG_ERR_ARG;
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess || ndev == 0) return cuda_fail(nullptr, e ? e : cudaErrorNoDevice, "device");
  if (device < 0 || device >= ndev) return NDG_ERR_ARG;
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaSetDevice");
  ndg_ctx *c = new ndg_ctx();
  c->device = device;
  c->precision = precision;
  // a blocking stream: the host paths' plain cudaMemcpy/cudaMemset (legacy
  // default stream) are ordered with the kernels launched on it
  if (cudaStreamCreate(&c->st) != cudaSuccess) {
    delete c;
    return NDG_ERR_CUDA;
  }
  c->ring_count = dalloc<int>(4);  // records, error bits, max tile candidates
  if (!c->ring_count) {
    delete c;
    return NDG_ERR_NOMEM;
  }
  cudaMemset(c->ring_count, 0, 4 * sizeof(int));
  if (cudaHostAlloc((void **)&c->pin_words, 4 * sizeof(int), cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    c->pin_words = nullptr;  // check_words falls back to a pageable copy
  }
  int rc = grow_sys(c, 4);
  if (!rc) rc = grow_atoms(c, 16);
  if (!rc) rc = grow_cells(c, 1024);
  if (!rc) rc = grow_nbr(c, 1 << 16);
  if (rc) {
    delete c;
    return rc;
  }
  *out = c;
  return NDG_OK;
}

int ndg_destroy(ndg_ctx *c) {
  if (!c) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  delete c;
  return NDG_OK;
}

int ndg_set_precision(ndg_ctx *c, int precision) {
  if (!c || (precision != NDG_PREC_FP64 && precision != NDG_PREC_MIXED)) return NDG_ERR_ARG;
  if (precision != c->precision) {
    c->precision = precision;
    drop_graphs(c);
    if (precision == NDG_PREC_MIXED) {
      int e = ensure_params(c);
      if (e) return e;
      DevCtx d = devctx(c);
      launch_refresh_pfx(d, c->st);
      CK(c, cudaStreamSynchronize(c->st));
    }
  }
  return NDG_OK;
}

int ndg_add_system(ndg_ctx *c, int np, int ntypes, int npairs, int ptsize, double ptrmin,
                   const double *mass, const int *pairmat, const double *rcpair,
                   const double *ppair, const double *fpair, const int *typ, const double *pos,
                   const double *vel, const double *acc, const double *box, int *sys_out) {
  if (!c || np < 1 || ntypes < 1 || ntypes > MAX_TYPES || npairs < 1 || ptsize < 2 || !mass ||
      !pairmat || !rcpair || !ppair || !fpair || !typ || !pos || !box)
    return NDG_ERR_ARG;
  for (int i = 0; i < np; ++i)
    if (typ[i] < 1 || typ[i] > ntypes) return NDG_ERR_ARG;
  for (int k = 0; k < ntypes * ntypes; ++k)
    if (pairmat[k] < 0 || pairmat[k] > npairs) return NDG_ERR_ARG;
  // a PairMat with one-sided ('asym') entries selects compute1's rules
  // (src/nd.f90:155-163): the kernels read it through the gather matrix
  cudaSetDevice(c->device);
  int s = -1;
  for (size_t k = 0; k < c->sys.size(); ++k)
    if (!c->sys[k].alive) {
      s = (int)k;
      break;
    }
  if (s < 0) {
    s = (int)c->sys.size();
    c->sys.emplace_back();
  }
  if (s >= 65535) return NDG_ERR_ARG;
  if (s >= c->nsys_cap) {
    int rc = grow_sys(c, std::max(s + 1, c->nsys_cap * 2));
    if (rc) return rc;
  }
  HostSys &h = c->sys[s];
  h = HostSys();
  h.alive = true;
  h.n = np;
  h.ntypes = ntypes;
  h.npairs = npairs;
  h.ptsize = ptsize;
  h.ptrmin = ptrmin;
  h.mass.assign(mass, mass + ntypes);
  h.pairmat.assign(pairmat, pairmat + ntypes * ntypes);
  h.rcpair.assign(rcpair, rcpair + npairs);
  h.ppair.assign(ppair, ppair + (size_t)(ptsize + 1) * npairs);
  h.fpair.assign(fpair, fpair + (size_t)(ptsize + 1) * npairs);
  {
    // the mixed kernel's tables: entry k holds values k and k+1 in FP32
    const int T = ptsize + 1;
    h.tF2.resize((size_t)T * npairs);
    h.tP2.resize((size_t)T * npairs);
    for (int j = 0; j < npairs; ++j)
      for (int k = 0; k < T; ++k) {
        const size_t a = (size_t)j * T + k, b = k + 1 < T ? a + 1 : a;
        h.tF2[a] = make_float2((float)h.fpair[a], (float)h.fpair[b]);
        h.tP2[a] = make_float2((float)h.ppair[a], (float)h.ppair[b]);
      }
  }
  h.rcut = *std::max_element(rcpair, rcpair + npairs);  // src/potentials.f90:36
  ndg_default_control(&h.ctl);
  const long long nch = (np + ATOM_ALIGN - 1) / ATOM_ALIGN;
  const long long off = arena_take(c, c->atoms, nch, 0);
  if (off < 0) {
    h.alive = false;
    return NDG_ERR_NOMEM;
  }
  h.atoms.off = off;
  h.atoms.len = nch;
  for (long long q = off; q < off + nch; ++q) c->chunk_sys_h[q] = s;
  CK(c, cudaMemcpy(c->chunk_sys + off, c->chunk_sys_h.data() + off, nch * sizeof(int),
                   cudaMemcpyHostToDevice));
  // padding slots: gid -1, zero state
  const size_t a0 = (size_t)off * ATOM_ALIGN, na = (size_t)nch * ATOM_ALIGN;
  CK(c, cudaMemset(c->gid + a0, 0xff, na * sizeof(int)));
  CK(c, cudaMemset(c->pos + a0, 0, na * sizeof(double4)));
  CK(c, cudaMemset(c->nnb + a0, 0, na * sizeof(int)));
  h.prm = SysParam();
  fill_control_params(h);
  h.prm.atom_off = (int)a0;
  h.prm.n = np;
  h.prm.npad = (int)na;
  SysState S;
  memset(&S, 0, sizeof(S));
  for (int d = 0; d < 3; ++d) {
    S.box[d] = box[d];
    S.box_build[d] = box[d];
    S.li[d] = 1.0 / box[d];
  }
  S.lam_ke = S.lam_e = 1.0;
  int rc = put_state_dev(c, s, S);
  if (rc) return rc;
  rc = upload_atoms(c, s, typ, pos, vel, acc);
  if (rc) return rc;
  // per-pair/per-type arrays are uploaded once before the next launch; the
  // fixed-point positions are written by the list build every run starts with
  c->params_dirty = true;
  if (sys_out) *sys_out = s;
  return NDG_OK;
}

int ndg_remove_system(ndg_ctx *c, int s) {
  if (!valid_sys(c, s)) return NDG_ERR_NOT_FOUND;
  HostSys &h = c->sys[s];
  for (long long q = h.atoms.off; q < h.atoms.off + h.atoms.len; ++q) c->chunk_sys_h[q] = -1;
  CK(c, cudaMemcpy(c->chunk_sys + h.atoms.off, c->chunk_sys_h.data() + h.atoms.off,
                   h.atoms.len * sizeof(int), cudaMemcpyHostToDevice));
  c->atoms.give(h.atoms.off);
  if (h.cells.off >= 0) {
    for (long long q = h.cells.off; q < h.cells.off + h.cells.len; ++q) c->cell_sys_h[q] = -1;
    CK(c, cudaMemcpy(c->cell_sys + h.cells.off, c->cell_sys_h.data() + h.cells.off,
                     h.cells.len * sizeof(int), cudaMemcpyHostToDevice));
    c->cells.give(h.cells.off);
  }
  if (h.nbr.off >= 0) c->nbrs.give(h.nbr.off);
  h = HostSys();
  SysState S;
  memset(&S, 0, sizeof(S));
  int rc = put_state_dev(c, s, S);
  if (rc) return rc;
  // no kernel sees the system from here on; the other systems' parameters
  // are packed again once, before the next launch that needs them
  SysParam z;
  memset(&z, 0, sizeof(z));
  CK(c, cudaMemcpy(c->dP + s, &z, sizeof(z), cudaMemcpyHostToDevice));
  c->params_dirty = true;
  return NDG_OK;
}

int ndg_num_systems(const ndg_ctx *c) {
  if (!c) return 0;
  int n = 0;
  for (auto &h : c->sys) n += h.alive;
  return n;
}

int ndg_set_holds(ndg_ctx *c, int s, const int *hold, int ngroups, const int *dir,
                  const double *du) {
  if (!valid_sys(c, s) || ngroups < 0 || (hold && ngroups > 0 && (!dir || !du)))
    return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  HostSys &h = c->sys[s];
  c->params_dirty = true;
  if (!hold || ngroups == 0) {
    h.bc.clear();
    return NDG_OK;
  }
  for (int i = 0; i < h.n; ++i)
    if (hold[i] < 0 || hold[i] > ngroups) return NDG_ERR_ARG;
  // the groups are read through the atoms' input index (gid), which the
  // list builds' reordering keeps
  CK(c, cudaMemcpy(c->hold + (size_t)h.atoms.off * ATOM_ALIGN, hold, h.n * sizeof(int),
                   cudaMemcpyHostToDevice));
  h.bc.resize(ngroups);
  for (int g = 0; g < ngroups; ++g) {
    const int m = (dir[3 * g] ? 1 : 0) | (dir[3 * g + 1] ? 2 : 0) | (dir[3 * g + 2] ? 4 : 0);
    h.bc[g] = make_double4(du[3 * g], du[3 * g + 1], du[3 * g + 2], (double)m);
  }
  return NDG_OK;
}

int ndg_set_springs(ndg_ctx *c, int s, const int *spring, const double *params) {
  if (!valid_sys(c, s) || (spring && !params)) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  HostSys &h = c->sys[s];
  c->params_dirty = true;
  h.spr.clear();
  if (!spring) return NDG_OK;
  bool any = false;
  for (int k = 0; k < h.npairs; ++k) any |= spring[k] != 0;
  if (!any) return NDG_OK;
  h.spr.resize(h.npairs);
  for (int k = 0; k < h.npairs; ++k) {
    const double *q = params + 4 * k;  // PairParams(1:4, k): rc, D0, sc, Vol
    h.spr[k] = spring[k] ? make_double4(q[1], q[2], q[3], 1.0) : make_double4(0, 0, 0, 0);
  }
  return NDG_OK;
}

int ndg_set_initial_positions(ndg_ctx *c, int s, const double *ipos, const double *ibox) {
  if (!valid_sys(c, s)) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  return init_positions(c, s, ipos, ibox);
}

// ---------------------------------------------------------------------------
// Bulk state transfer (sys = -1): every live system at once, the caller's
// arrays holding them one after another in ascending id order.  The host
// data moves in one copy per array (straight from the caller's buffers, so
// pinned ones go by DMA) through the rebuild's scratch arrays, and one
// kernel puts each atom in place; the boxes move with one copy of the state
// records.  One host wait per call, however many systems.

// each live system's first atom in the concatenated arrays, on the device;
// *total = all atoms, *nlive = live systems
static int xfer_offsets(ndg_ctx *c, long long *total, int *nlive) {
  std::vector<long long> xo(std::max(c->nsys_cap, 1), -1);
  long long t = 0;
  int m = 0;
  for (size_t s = 0; s < c->sys.size(); ++s)
    if (c->sys[s].alive) {
      xo[s] = t;
      t += c->sys[s].n;
      ++m;
    }
  if (!c->xoff || c->cap_xoff < xo.size()) {
    if (c->xoff) cudaFree(c->xoff);
    c->xoff = dalloc<long long>(xo.size());
    c->cap_xoff = c->xoff ? xo.size() : 0;
    if (!c->xoff) return NDG_ERR_NOMEM;
  }
  CK(c, cudaMemcpyAsync(c->xoff, xo.data(), xo.size() * sizeof(long long),
                        cudaMemcpyHostToDevice, c->st));
  CK(c, cudaStreamSynchronize(c->st));  // xo is a local
  *total = t;
  *nlive = m;
  return NDG_OK;
}

static int load_all(ndg_ctx *c, const double *pos, const double *vel, const double *acc,
                    const double *box) {
  int rc = ensure_params(c);
  if (rc) return rc;
  long long t = 0;
  int m = 0;
  rc = xfer_offsets(c, &t, &m);
  if (rc || m == 0) return rc;
  const size_t b3 = 3 * (size_t)t * sizeof(double);
  cudaStream_t st = c->st;
  double *xp = (double *)c->s_pos, *xv = vel ? c->s_vel : nullptr, *xa = acc ? c->s_acc : nullptr;
  CK(c, cudaMemcpyAsync(xp, pos, b3, cudaMemcpyHostToDevice, st));
  if (vel) CK(c, cudaMemcpyAsync(xv, vel, b3, cudaMemcpyHostToDevice, st));
  if (acc) CK(c, cudaMemcpyAsync(xa, acc, b3, cudaMemcpyHostToDevice, st));
  DevCtx d = devctx(c);
  launch_load_all(d, st, c->xoff, xp, xv, xa);
  CK(c, cudaGetLastError());
  if (box) {
    std::vector<SysState> S(c->nsys_cap);
    CK(c, cudaMemcpyAsync(S.data(), c->dS, S.size() * sizeof(SysState), cudaMemcpyDeviceToHost,
                          st));
    CK(c, cudaStreamSynchronize(st));
    int k = 0;
    for (size_t s = 0; s < c->sys.size(); ++s)
      if (c->sys[s].alive) {
        for (int q = 0; q < 3; ++q) {
          S[s].box[q] = box[3 * k + q];
          S[s].li[q] = 1.0 / box[3 * k + q];
        }
        ++k;
      }
    CK(c, cudaMemcpyAsync(c->dS, S.data(), S.size() * sizeof(SysState), cudaMemcpyHostToDevice,
                          st));
    CK(c, cudaStreamSynchronize(st));  // S is a local
  }
  if (c->precision == NDG_PREC_MIXED) launch_refresh_pfx(d, st);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(st));
  for (auto &h : c->sys)
    if (h.alive) h.lists_valid = false;
  return NDG_OK;
}

static int get_all(ndg_ctx *c, double *pos, double *vel, double *acc, double *box) {
  int rc = ensure_params(c);
  if (rc) return rc;
  long long t = 0;
  int m = 0;
  rc = xfer_offsets(c, &t, &m);
  if (rc || m == 0) return rc;
  const size_t b3 = 3 * (size_t)t * sizeof(double);
  cudaStream_t st = c->st;
  double *xp = pos ? (double *)c->s_pos : nullptr, *xv = vel ? c->s_vel : nullptr,
         *xa = acc ? c->s_acc : nullptr;
  DevCtx d = devctx(c);
  launch_store_all(d, st, c->xoff, xp, xv, xa);
  CK(c, cudaGetLastError());
  if (pos) CK(c, cudaMemcpyAsync(pos, xp, b3, cudaMemcpyDeviceToHost, st));
  if (vel) CK(c, cudaMemcpyAsync(vel, xv, b3, cudaMemcpyDeviceToHost, st));
  if (acc) CK(c, cudaMemcpyAsync(acc, xa, b3, cudaMemcpyDeviceToHost, st));
  std::vector<SysState> S(box ? c->nsys_cap : 0);
  if (box)
    CK(c, cudaMemcpyAsync(S.data(), c->dS, S.size() * sizeof(SysState), cudaMemcpyDeviceToHost,
                          st));
  CK(c, cudaStreamSynchronize(st));
  if (box) {
    int k = 0;
    for (size_t s = 0; s < c->sys.size(); ++s)
      if (c->sys[s].alive) {
        for (int q = 0; q < 3; ++q) box[3 * k + q] = S[s].box[q];
        ++k;
      }
  }
  return NDG_OK;
}

int ndg_load_state(ndg_ctx *c, int s, const double *pos, const double *vel, const double *acc,
                   const double *box) {
  if (c && s == -1 && pos) {
    cudaSetDevice(c->device);
    return load_all(c, pos, vel, acc, box);
  }
  if (!valid_sys(c, s) || !pos) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = ensure_params(c);
  if (rc) return rc;
  rc = upload_atoms(c, s, nullptr, pos, vel, acc);
  if (rc) return rc;
  if (box) {
    SysState S;
    rc = get_state_dev(c, s, S);
    if (rc) return rc;
    for (int d = 0; d < 3; ++d) {
      S.box[d] = box[d];
      S.li[d] = 1.0 / box[d];
    }
    rc = put_state_dev(c, s, S);
    if (rc) return rc;
  }
  if (c->precision == NDG_PREC_MIXED) {
    DevCtx d = devctx(c);
    launch_refresh_pfx(d, c->st);
    CK(c, cudaStreamSynchronize(c->st));
  }
  return NDG_OK;
}

int ndg_get_state(ndg_ctx *c, int s, double *pos, double *vel, double *acc, double *box) {
  if (c && s == -1) {
    cudaSetDevice(c->device);
    return get_all(c, pos, vel, acc, box);
  }
  if (!valid_sys(c, s)) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  HostSys &h = c->sys[s];
  const int n = h.n;
  const size_t off = (size_t)h.atoms.off * ATOM_ALIGN;
  // one stream-ordered batch of copies into pinned staging: slots |
  // positions | velocities | accelerations, then scattered to input order
  const size_t bg = ((size_t)n * sizeof(int) + 15) / 16 * 16, bp = (size_t)n * sizeof(double4);
  const size_t b3 = 3 * (size_t)n * sizeof(double);
  const size_t total = bg + (pos ? bp : 0) + (vel ? b3 : 0) + (acc ? b3 : 0);
  std::vector<char> pageable;
  char *buf = pinned(c, total);
  if (!buf) {
    pageable.resize(total);
    buf = pageable.data();
  }
  int *g = (int *)buf;
  double4 *p = (double4 *)(buf + bg);
  double *vt = (double *)(buf + bg + (pos ? bp : 0)), *at = vt + (vel ? 3 * (size_t)n : 0);
  cudaStream_t st = c->st;
  CK(c, cudaMemcpyAsync(g, c->gid + off, n * sizeof(int), cudaMemcpyDeviceToHost, st));
  if (pos) CK(c, cudaMemcpyAsync(p, c->pos + off, bp, cudaMemcpyDeviceToHost, st));
  if (vel) CK(c, cudaMemcpyAsync(vt, c->vel + 3 * off, b3, cudaMemcpyDeviceToHost, st));
  if (acc) CK(c, cudaMemcpyAsync(at, c->acc + 3 * off, b3, cudaMemcpyDeviceToHost, st));
  CK(c, cudaStreamSynchronize(st));
  if (pos)
    for (int i = 0; i < n; ++i) {
      pos[3 * g[i]] = p[i].x;
      pos[3 * g[i] + 1] = p[i].y;
      pos[3 * g[i] + 2] = p[i].z;
    }
  if (vel)
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) vel[3 * g[i] + d] = vt[3 * i + d];
  if (acc)
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) acc[3 * g[i] + d] = at[3 * i + d];
  if (box) {
    SysState S;
    int rc = get_state_dev(c, s, S);
    if (rc) return rc;
    for (int d = 0; d < 3; ++d) box[d] = S.box[d];
  }
  return NDG_OK;
}

int ndg_set_control(ndg_ctx *c, int s, const ndg_control *q) {
  if (!valid_sys(c, s) || !q) return NDG_ERR_ARG;
  if (q->out_steps < 1 || q->renei_freq < 1 || q->ke_freq < 1 || q->p_freq < 1 ||
      q->e_freq < 1 || (q->quirk != NDG_QUIRK_REF && q->quirk != NDG_QUIRK_FIXED))
    return NDG_ERR_ARG;
  HostSys &h = c->sys[s];
  h.ctl = *q;
  fill_control_params(h);
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  S.step = q->step;
  rc = put_state_dev(c, s, S);
  if (rc) return rc;
  c->params_dirty = true;
  return NDG_OK;
}

int ndg_get_control(ndg_ctx *c, int s, ndg_control *q) {
  if (!valid_sys(c, s) || !q) return NDG_ERR_ARG;
  *q = c->sys[s].ctl;
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  q->step = S.step;
  return NDG_OK;
}

int ndg_setup_lists(ndg_ctx *c) {
  if (!c) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  return setup_lists(c);
}

int ndg_build_cell_list(ndg_ctx *c) {
  if (!c) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  for (auto &h : c->sys)
    if (h.alive && h.maxnb == 0) return setup_lists(c);
  DevCtx d = devctx(c);
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  int rc = list_all_systems(c);
  if (rc) return rc;
  launch_rebuild(d, c->st, 0, c->precision == NDG_PREC_MIXED);
  CK(c, cudaGetLastError());
  rc = status_from_words(c);
  CK(c, cudaMemset(c->ring_count + 3, 0, sizeof(int)));
  if (!rc)
    for (auto &h : c->sys)
      if (h.alive) h.lists_valid = true;
  return rc;
}

static bool lists_ready(ndg_ctx *c) {
  for (auto &h : c->sys)
    if (h.alive && !h.lists_valid) return false;
  return true;
}

int ndg_check_list_update(ndg_ctx *c, int *rebuilt) {
  if (!c || !lists_ready(c)) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  DevCtx d = devctx(c);
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  launch_check(d, c->st, c->nsys_cap);  // lists the systems to rebuild
  launch_rebuild(d, c->st, 1, c->precision == NDG_PREC_MIXED);
  CK(c, cudaGetLastError());
  int rc = status_from_words(c);
  CK(c, cudaMemset(c->ring_count + 3, 0, sizeof(int)));
  if (rc) return rc;
  if (rebuilt) {
    std::vector<SysState> S(c->nsys_cap);
    CK(c, cudaMemcpy(S.data(), c->dS, S.size() * sizeof(SysState), cudaMemcpyDeviceToHost));
    int n = 0;
    for (size_t s = 0; s < c->sys.size(); ++s) n += c->sys[s].alive && S[s].rebuild;
    *rebuilt = n;
  }
  return NDG_OK;
}

int ndg_integrate1(ndg_ctx *c) {
  if (!c) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  std::vector<SysState> S(c->nsys_cap);
  CK(c, cudaMemcpy(S.data(), c->dS, S.size() * sizeof(SysState), cudaMemcpyDeviceToHost));
  for (auto &x : S)
    for (int d = 0; d < 3; ++d) x.li[d] = 1.0 / x.box[d];  // li = 1/box, src/nd.f90:1023-1025
  CK(c, cudaMemcpy(c->dS, S.data(), S.size() * sizeof(SysState), cudaMemcpyHostToDevice));
  DevCtx d = devctx(c);
  launch_integrate1(d, c->st, 1, c->precision == NDG_PREC_MIXED);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  return NDG_OK;
}

int ndg_compute(ndg_ctx *c, int cv, int cu) {
  if (!c || !lists_ready(c)) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  DevCtx d = devctx(c);
  const int flags = (cv ? F_CV : 0) | (cu ? F_CU : 0);
  launch_pair(d, c->st, choose_tpa(c), c->precision == NDG_PREC_MIXED, 0, flags);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  return NDG_OK;
}

int ndg_integrate2(ndg_ctx *c, int ck) {
  if (!c) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  DevCtx d = devctx(c);
  launch_integrate2(d, c->st, ck);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  return NDG_OK;
}

int ndg_mk_iso_ke(ndg_ctx *c, int s) {
  if (!valid_sys(c, s)) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  const double lam = lam_iso_ke(c->sys[s].prm, S.kinetic, c->sys[s].n);
  DevCtx d = devctx(c);
  launch_scale_vel(d, c->st, s, lam);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  return NDG_OK;
}

int ndg_mk_iso_e(ndg_ctx *c, int s) {
  if (!valid_sys(c, s)) return NDG_ERR_ARG;
  {
    int e = ensure_params(c);
    if (e) return e;
  }
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  const double lam = lam_iso_e(c->sys[s].prm, S.e0, S.potential, S.kinetic);
  DevCtx d = devctx(c);
  launch_scale_vel(d, c->st, s, lam);
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  return NDG_OK;
}

int ndg_mk_iso_p(ndg_ctx *c, int s) {
  if (!valid_sys(c, s)) return NDG_ERR_ARG;
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  iso_p_box(c->sys[s].prm, S.virial, S.box);
  for (int d = 0; d < 3; ++d) S.li[d] = 1.0 / S.box[d];
  return put_state_dev(c, s, S);
}

int ndg_get_forces(ndg_ctx *c, int s, double *force, double *potential, double *virial,
                   double *kinetic) {
  if (!valid_sys(c, s)) return NDG_ERR_ARG;
  CK(c, cudaStreamSynchronize(c->st));
  HostSys &h = c->sys[s];
  const int n = h.n;
  const size_t off = (size_t)h.atoms.off * ATOM_ALIGN;
  if (force) {
    std::vector<int> g(n);
    std::vector<double> f(3 * (size_t)n);
    CK(c, cudaMemcpy(g.data(), c->gid + off, n * sizeof(int), cudaMemcpyDeviceToHost));
    CK(c, cudaMemcpy(f.data(), c->force + 3 * off, 3 * n * sizeof(double),
                     cudaMemcpyDeviceToHost));
    for (int i = 0; i < n; ++i)
      for (int d = 0; d < 3; ++d) force[3 * g[i] + d] = f[3 * i + d];
  }
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  if (potential) *potential = S.potential;
  if (virial)
    for (int k = 0; k < 6; ++k) virial[k] = S.virial[k];
  if (kinetic) *kinetic = S.kinetic;
  return NDG_OK;
}

static int run_impl(ndg_ctx *c, int nsteps, ndg_thermo_cb cb, void *user, int cont) {
  if (!c || nsteps < 0) return NDG_ERR_ARG;
  if (nsteps == 0) return NDG_OK;
  cudaSetDevice(c->device);
  int rc;
  if (!cont || !lists_ready(c)) {
    rc = setup_lists(c);
    if (rc) return rc;
    cont = 0;
  }
  // controls may have changed between runs; the parameters go up again only
  // when some system's did (an upload re-packs every system's tables, about
  // 10 ms for 512 systems, which a short run would otherwise pay each time)
  for (auto &h : c->sys)
    if (h.alive) {
      const SysParam before = h.prm;
      fill_control_params(h);
      if (memcmp(&before, &h.prm, sizeof(SysParam)) != 0) c->params_dirty = true;
    }
  rc = ensure_params(c);
  if (rc) return rc;
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  DevCtx d = devctx(c);
  // a continued run carries on from the last step (its counter tt, e0 and
  // list decision), as if the two calls were one Run
  launch_arm(d, c->st, c->nsys_cap, -1, nsteps, cont ? START_CONTINUE : START_BUILT);
  CK(c, cudaGetLastError());
  rc = run_blocks(c, nsteps, cb, user, true);
  if (rc) flush_pending(c);  // a failed block left the last flush unlaunched
  return rc;
}

int ndg_run(ndg_ctx *c, int nsteps, ndg_thermo_cb cb, void *user) {
  return run_impl(c, nsteps, cb, user, 0);
}

int ndg_run_continue(ndg_ctx *c, int nsteps, ndg_thermo_cb cb, void *user) {
  return run_impl(c, nsteps, cb, user, 1);
}

int ndg_get_thermo(ndg_ctx *c, int s, ndg_thermo *t) {
  if (!valid_sys(c, s) || !t) return NDG_ERR_ARG;
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  ThermoRec r;
  make_thermo(r, s, S.step, S.potential, S.kinetic, S.e0, S.virial, S.box);
  memcpy(t, &r, sizeof(r));
  return NDG_OK;
}

int ndg_get_list_updates(ndg_ctx *c, int s, int *n) {
  if (!valid_sys(c, s) || !n) return NDG_ERR_ARG;
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  *n = S.nlist_updates;
  return NDG_OK;
}

int ndg_get_mcell(ndg_ctx *c, int s, int *m) {
  if (!valid_sys(c, s) || !m) return NDG_ERR_ARG;
  SysState S;
  int rc = get_state_dev(c, s, S);
  if (rc) return rc;
  for (int d = 0; d < 3; ++d) m[d] = S.mcell[d];
  return NDG_OK;
}

int ndg_get_cells(ndg_ctx *c, int s, int *cell) {
  if (!valid_sys(c, s) || !cell || !c->sys[s].lists_valid) return NDG_ERR_ARG;
  HostSys &h = c->sys[s];
  const int n = h.n;
  const size_t off = (size_t)h.atoms.off * ATOM_ALIGN;
  std::vector<int> g(n), a(n);
  CK(c, cudaStreamSynchronize(c->st));
  CK(c, cudaMemcpy(g.data(), c->gid + off, n * sizeof(int), cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(a.data(), c->atom_cell + off, n * sizeof(int), cudaMemcpyDeviceToHost));
  for (int i = 0; i < n; ++i) cell[g[i]] = a[i];
  return NDG_OK;
}

int ndg_get_neighbors(ndg_ctx *c, int s, int *pairs, long long cap, long long *npairs) {
  if (!valid_sys(c, s) || !c->sys[s].lists_valid) return NDG_ERR_ARG;
  HostSys &h = c->sys[s];
  const int n = h.n;
  const size_t off = (size_t)h.atoms.off * ATOM_ALIGN;
  const long long npad = h.atoms.len * ATOM_ALIGN;
  CK(c, cudaStreamSynchronize(c->st));
  std::vector<int> g(n), cnt(n);
  std::vector<int> nb((size_t)h.maxnb * npad);
  CK(c, cudaMemcpy(g.data(), c->gid + off, n * sizeof(int), cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(cnt.data(), c->nnb + off, n * sizeof(int), cudaMemcpyDeviceToHost));
  CK(c, cudaMemcpy(nb.data(), c->nbr + h.nbr.off, nb.size() * sizeof(int),
                   cudaMemcpyDeviceToHost));
  long long m = 0;
  const bool nb16 = h.prm.nb16 != 0;
  for (int i = 0; i < n; ++i) {
    const int k1 = std::min(cnt[i], h.maxnb);
    const size_t col = (size_t)(i / 128) * h.maxnb * 128 + (i % 128);
    for (int k = 0; k < k1; ++k) {
      int j;
      if (nb16) {
        // entry k: half k&1 of word (k>>1)*128 of the column, an offset from
        // the system's first atom (little-endian: the low half comes first)
        unsigned short e[2];
        memcpy(e, &nb[col + (size_t)(k >> 1) * 128], sizeof(e));
        j = e[k & 1];
      } else {
        j = nb[col + (size_t)k * 128] - (int)off;
      }
      const int gi = g[i], gj = g[j];
      if (gi < gj) {
        if (pairs && m < cap) {
          pairs[2 * m] = gi;
          pairs[2 * m + 1] = gj;
        }
        ++m;
      }
    }
  }
  if (npairs) *npairs = m;
  return NDG_OK;
}

int ndg_get_neighbor_count(ndg_ctx *c, int s, long long *entries) {
  if (!valid_sys(c, s) || !entries || !c->sys[s].lists_valid) return NDG_ERR_ARG;
  HostSys &h = c->sys[s];
  const size_t off = (size_t)h.atoms.off * ATOM_ALIGN;
  std::vector<int> cnt(h.n);
  CK(c, cudaStreamSynchronize(c->st));
  CK(c, cudaMemcpy(cnt.data(), c->nnb + off, h.n * sizeof(int), cudaMemcpyDeviceToHost));
  long long m = 0;
  for (int x : cnt) m += std::min(x, h.maxnb);
  *entries = m;
  return NDG_OK;
}

int ndg_set_tuning(ndg_ctx *c, int tpa, int graph_steps) {
  if (!c) return NDG_ERR_ARG;
  if (tpa != 0 && tpa != 1 && tpa != 2 && tpa != 4 && tpa != 8)
    return NDG_ERR_ARG;
  if (graph_steps < 1) return NDG_ERR_ARG;
  if (tpa != c->tpa || graph_steps != c->graph_steps) drop_graphs(c);
  c->tpa = tpa;
  if (graph_steps != c->graph_steps) {
    c->graph_steps = graph_steps;
    const int need = std::max(256, graph_steps * c->nsys_cap);
    if (need > c->ring_cap) {
      dfree(c->ring);
      c->ring = dalloc<ThermoRec>(need);
      if (!c->ring) return NDG_ERR_NOMEM;
      c->ring_cap = need;
    }
  }
  return NDG_OK;
}

int ndg_set_gather_depth(ndg_ctx *c, int depth) {
  if (!c || (depth != 4 && depth != 8)) return NDG_ERR_ARG;
  if (depth != c->gather) drop_graphs(c);
  c->gather = depth;
  return NDG_OK;
}

int ndg_get_gather_depth(ndg_ctx *c, int *depth) {
  if (!c || !depth) return NDG_ERR_ARG;
  *depth = c->gather;
  return NDG_OK;
}

int ndg_set_list_split(ndg_ctx *c, int rows, int tpa_long) {
  if (!c || rows < 0 || (tpa_long != 1 && tpa_long != 2 && tpa_long != 4 && tpa_long != 8))
    return NDG_ERR_ARG;
  if (rows != c->rows_split || tpa_long != c->tpa_long) drop_graphs(c);
  c->rows_split = rows;
  c->tpa_long = tpa_long;
  return NDG_OK;
}

int ndg_get_list_split(ndg_ctx *c, int *rows, int *tpa_long) {
  if (!c) return NDG_ERR_ARG;
  if (rows) *rows = c->rows_split;
  if (tpa_long) *tpa_long = c->tpa_long;
  return NDG_OK;
}

int ndg_get_tuning(ndg_ctx *c, int *tpa, int *graph_steps) {
  if (!c) return NDG_ERR_ARG;
  if (tpa) *tpa = choose_tpa(c);
  if (graph_steps) *graph_steps = c->graph_steps;
  return NDG_OK;
}

int ndg_device_bytes(const ndg_ctx *c, long long *bytes) {
  if (!c || !bytes) return NDG_ERR_ARG;
  const long long A = c->atoms.cap * ATOM_ALIGN;
  long long b = A * (2 * 32 + 16 + 4 * 24 + 2 * 24 + 4 * 10) + c->cells.cap * 12 +
                c->nbrs.cap * 4 + (long long)c->nsys_cap * (sizeof(SysParam) + sizeof(SysState)) +
                (long long)c->ring_cap * sizeof(ThermoRec);
  *bytes = b;
  return NDG_OK;
}

long long ndg_system_bytes(int np, int ntypes, int npairs, int ptsize, double density,
                           double rlist, int precision) {
  (void)ntypes;
  (void)precision;
  const long long npad = ((long long)np + ATOM_ALIGN - 1) / ATOM_ALIGN * ATOM_ALIGN;
  const double r = rlist * 1.1;
  const long long maxnb =
      (long long)(4.0 / 3.0 * 3.141592653589793 * r * r * r * density * 1.2 * 2.0) + 24;
  const long long per_atom = 2 * 32 + 16 + 4 * 24 + 2 * 24 + 4 * 11;
  const long long ncell = (long long)(np / std::max(density * rlist * rlist * rlist, 1e-9)) + 8;
  return npad * per_atom + npad * maxnb * 4 + ncell * 12 +
         (long long)npairs * (ptsize + 1) * 32;
}

// Autotuner: every mutable device array is snapshotted, each candidate
// launch shape (threads per atom) runs `steps` real graph steps on the
// current systems, timed with CUDA events on the library's stream, the state
// is restored after each trial, and the fastest shape is kept.
namespace {
// A device copy of every mutable array of a context (positions, lists,
// state records, ...), so that trial steps can be undone.
struct Snapshot {
  struct Buf {
    void *p;
    size_t bytes;
  };
  ndg_ctx *c;
  std::vector<Buf> bufs;
  char *snap = nullptr;
  explicit Snapshot(ndg_ctx *ctx) : c(ctx) {
    const size_t A = (size_t)c->atoms.cap * ATOM_ALIGN, T = 2 * (size_t)c->atoms.cap;
    bufs = {{c->pos, A * sizeof(double4)},       {c->pfx, A * sizeof(int4)},
            {c->vel, 3 * A * sizeof(double)},    {c->acc, 3 * A * sizeof(double)},
            {c->disp, 3 * A * sizeof(double)},   {c->gid, A * sizeof(int)},
            {c->nnb, A * sizeof(int)},           {c->atom_cell, A * sizeof(int)},
            {c->itop, 2 * (size_t)c->atoms.cap * sizeof(double)},
            {c->tile_rows, T * sizeof(int)},
            {c->cell_start, (size_t)c->cells.cap * sizeof(int)},
            {c->nbr, (size_t)c->nbrs.cap * sizeof(int)},
            {c->dS, (size_t)c->nsys_cap * sizeof(SysState)}};
    size_t total = 0;
    for (auto &b : bufs) total += b.bytes;
    snap = dalloc<char>(total);
  }
  ~Snapshot() {
    if (snap) cudaFree(snap);
  }
  bool ok() const { return snap != nullptr; }
  cudaError_t copy(bool save) {
    size_t off = 0;
    for (auto &b : bufs) {
      cudaError_t e = save ? cudaMemcpyAsync(snap + off, b.p, b.bytes, cudaMemcpyDeviceToDevice, c->st)
                           : cudaMemcpyAsync(b.p, snap + off, b.bytes, cudaMemcpyDeviceToDevice, c->st);
      if (e != cudaSuccess) return e;
      off += b.bytes;
    }
    return cudaStreamSynchronize(c->st);
  }
};
}  // namespace

int ndg_autotune(ndg_ctx *c, int steps) {
  if (!c || steps < 1) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = NDG_OK;
  if (!lists_ready(c)) {
    rc = setup_lists(c);
    if (rc) return rc;
  }
  rc = ensure_params(c);
  if (rc) return rc;
  Snapshot sn(c);
  if (!sn.ok()) return NDG_ERR_NOMEM;
  auto copy = [&](bool save) { return sn.copy(save); };
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int keep_tpa = c->tpa, keep_gather = c->gather;
  const int keep_split = c->rows_split, keep_long = c->tpa_long;
  c->rows_split = 0;  // the launch shapes are timed as one class
  int best = 0, best_g = 4;
  float best_ms = 0.f;
  cudaError_t ce = copy(true);
  // launch shapes: threads per atom, and for one thread per atom in mixed
  // precision the gather depth
  const int cand[5][2] = {{1, 4}, {1, 8}, {2, 4}, {4, 4}, {8, 4}};
  const int ncand = c->precision == NDG_PREC_MIXED ? 5 : 4;
  for (int k = 0, kk = 0; kk < ncand && ce == cudaSuccess && rc == NDG_OK; ++k) {
    if (c->precision != NDG_PREC_MIXED && cand[k][1] != 4) continue;
    ++kk;
    c->tpa = cand[k][0];
    c->gather = cand[k][1];
    drop_graphs(c);
    CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
    DevCtx d = devctx(c);
    launch_arm(d, c->st, c->nsys_cap, -1, 2 * steps, START_NEW);
    rc = run_blocks(c, steps, nullptr, nullptr);  // warm: capture + first launch
    if (rc) break;
    cudaEventRecord(e0, c->st);
    rc = run_blocks(c, steps, nullptr, nullptr);
    cudaEventRecord(e1, c->st);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (!rc && (best == 0 || ms < best_ms)) {
      best = cand[k][0];
      best_g = cand[k][1];
      best_ms = ms;
    }
    ce = copy(false);
  }
  c->tpa = best ? best : keep_tpa;
  c->gather = best ? best_g : keep_gather;
  // atoms to threads by list length: where the systems' mean list lengths
  // (rows of a tile at their last build) spread by 1.5x or more, a class of
  // the long-list systems with 2 or 4 times the threads per atom, kept if
  // its trial beats the best single shape
  if (best && ce == cudaSuccess && rc == NDG_OK && !c->any_spring) {
    std::vector<SysState> S(c->nsys_cap);
    ce = cudaMemcpy(S.data(), c->dS, S.size() * sizeof(SysState), cudaMemcpyDeviceToHost);
    double rmin = 1e30, rmax = 0.0;
    for (size_t s = 0; s < c->sys.size() && ce == cudaSuccess; ++s) {
      const HostSys &h = c->sys[s];
      if (!h.alive || h.n == 0) continue;
      const double nt = (double)h.prm.npad / 128.0;
      const double r = (double)S[s].rows / nt;
      rmin = std::min(rmin, r);
      rmax = std::max(rmax, r);
    }
    if (ce == cudaSuccess && rmax > 0.0 && rmax >= 1.5 * rmin) {
      const int split = (int)std::ceil(std::sqrt(rmin * rmax));
      int best_long = 0;
      for (int mul = 2; mul <= 4 && c->tpa * mul <= 8 && rc == NDG_OK && ce == cudaSuccess;
           mul *= 2) {
        c->rows_split = split;
        c->tpa_long = c->tpa * mul;
        drop_graphs(c);
        CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
        DevCtx d = devctx(c);
        launch_arm(d, c->st, c->nsys_cap, -1, 2 * steps, START_NEW);
        rc = run_blocks(c, steps, nullptr, nullptr);
        if (rc) break;
        cudaEventRecord(e0, c->st);
        rc = run_blocks(c, steps, nullptr, nullptr);
        cudaEventRecord(e1, c->st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (!rc && ms < best_ms) {
          best_ms = ms;
          best_long = c->tpa_long;
        }
        ce = copy(false);
      }
      c->rows_split = best_long ? split : 0;
      c->tpa_long = best_long ? best_long : keep_long;
    }
  } else if (!best) {
    c->rows_split = keep_split;
    c->tpa_long = keep_long;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  drop_graphs(c);
  if (ce != cudaSuccess) return cuda_fail(c, ce, "autotune snapshot");
  return rc;
}

// The rebuild-interval autotuner: a list skin per system (fixed semantics).
//
// A larger skin makes every list longer, and the pair kernel's work per step
// grows with the list (as (rcut+skin)^3); a smaller one makes the fixed
// rebuild test (the two largest displacements since the last build against
// the skin) fire sooner.  From lists built afresh, a trial of `steps` eager
// steps measures the two costs on this batch: the pair kernel's time per
// unit of the work plan's tile cost (rows + 16 per tile), the rebuild
// group's time per rebuilt tile, and each system's rebuild count.  With the
// rebuild interval taken as proportional to the skin (displacements grow
// about linearly over the few tens of steps between builds), each system
// gets the skin of the grid f * skin, f in [0.5, 2], with the lowest
// modelled cost per step, if that beats its current skin by 2%.  A second
// trial from the same state with the new skins' lists must then run at
// least 2% faster than the first, or every skin goes back: the model only
// proposes, the clock decides.  Forces do not depend on the skin in these
// semantics (every pair within the cutoff is in the list at every step).
// The trials are undone.  Systems in the reference semantics keep their
// skin: their rebuild test is the reference's, and their list contents
// depend on it.
namespace {
// one trial from the current state, undone afterwards: the mean time per
// step of the step's kernels, and the state records after the trial
int skin_trial(ndg_ctx *c, int steps, double *ms, std::vector<SysState> &after) {
  Snapshot sn(c);
  if (!sn.ok()) return NDG_ERR_NOMEM;
  cudaError_t ce = sn.copy(true);
  if (ce != cudaSuccess) return cuda_fail(c, ce, "autotune_skin snapshot");
  int rc = ndg_profile_run(c, steps);
  if (rc == NDG_OK) {
    *ms = c->t_int + c->t_pair + c->t_reb;
    CK(c, cudaMemcpy(after.data(), c->dS, after.size() * sizeof(SysState),
                     cudaMemcpyDeviceToHost));
  }
  ce = sn.copy(false);
  if (ce != cudaSuccess) return cuda_fail(c, ce, "autotune_skin restore");
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  return rc;
}
}  // namespace

int ndg_autotune_skin(ndg_ctx *c, int steps, int *changed) {
  if (changed) *changed = 0;
  if (!c || steps < 4) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  std::vector<int> fixed;
  for (size_t s = 0; s < c->sys.size(); ++s)
    if (c->sys[s].alive && c->sys[s].ctl.quirk == NDG_QUIRK_FIXED) fixed.push_back((int)s);
  if (fixed.empty()) return NDG_OK;
  int rc = lists_ready(c) ? ensure_params(c) : setup_lists(c);
  if (rc) return rc;
  rc = setup_lists(c, fixed);  // fresh lists: both trials start alike
  if (rc) return rc;
  std::vector<SysState> S0(c->nsys_cap), S1(c->nsys_cap), S2(c->nsys_cap);
  CK(c, cudaMemcpy(S0.data(), c->dS, S0.size() * sizeof(SysState), cudaMemcpyDeviceToHost));
  double msA = 0.0, msB = 0.0;
  rc = skin_trial(c, steps, &msA, S1);
  if (rc) return rc;
  const double t_pair = c->t_pair * steps, t_reb = c->t_reb * steps;  // ms over the trial
  double units = 0.0, rebuilt_tiles = 0.0;
  for (int s : fixed) {
    const double tiles = (double)c->sys[s].prm.npad / 128.0;
    units += tiles * 16.0 + (double)S0[s].rows;
    rebuilt_tiles += tiles * (double)(S1[s].nlist_updates - S0[s].nlist_updates);
  }
  if (units <= 0.0 || rebuilt_tiles <= 0.0 || t_pair <= 0.0 || t_reb <= 0.0)
    return NDG_OK;  // nothing rebuilt in the trial: no measure of a rebuild's cost
  const double alpha = t_pair / steps / units;  // ms per tile-cost unit per step
  const double beta = t_reb / rebuilt_tiles;    // ms per rebuilt tile
  static const double grid[] = {0.5, 0.625, 0.75, 0.875, 1.0, 1.25, 1.5, 1.75, 2.0};
  std::vector<int> ids;
  std::vector<double> old_skin;
  for (int s : fixed) {
    HostSys &h = c->sys[s];
    const double skin0 = h.prm.skin, rl0 = h.rcut + skin0;
    if (!(skin0 > 0.0)) continue;
    const double tiles = (double)h.prm.npad / 128.0;
    const double rows = (double)S0[s].rows / tiles;  // mean list rows of a tile
    const int nup = std::max(S1[s].nlist_updates - S0[s].nlist_updates, 1);
    const double bmin = std::min(S0[s].box[0], std::min(S0[s].box[1], S0[s].box[2]));
    auto cost = [&](double skin) {
      const double g = (h.rcut + skin) / rl0;
      return alpha * tiles * (rows * g * g * g + 16.0) +
             beta * tiles * ((double)nup / steps) * (skin0 / skin);
    };
    const double c0 = cost(skin0);
    double best = skin0, bc = c0;
    for (double f : grid) {
      const double skin = f * skin0;
      if ((int)(bmin / (h.rcut + skin)) < 3) continue;  // keep three link cells per axis
      const double cf = cost(skin);
      if (cf < bc) {
        bc = cf;
        best = skin;
      }
    }
    if (best != skin0 && bc < 0.98 * c0) {
      ids.push_back(s);
      old_skin.push_back(h.ctl.skin);
      h.ctl.skin = best;
      fill_control_params(h);
    }
  }
  if (ids.empty()) return NDG_OK;
  c->params_dirty = true;
  rc = setup_lists(c, ids);  // the proposed skins' lists
  if (!rc) rc = skin_trial(c, steps, &msB, S2);
  if (rc || !(msB < 0.98 * msA)) {
    // the clock does not confirm the model: every skin goes back
    for (size_t k = 0; k < ids.size(); ++k) {
      HostSys &h = c->sys[ids[k]];
      h.ctl.skin = old_skin[k];
      fill_control_params(h);
    }
    c->params_dirty = true;
    const int rr = setup_lists(c, ids);
    return rc ? rc : rr;
  }
  if (changed) *changed = (int)ids.size();
  return NDG_OK;
}

int ndg_get_stream(ndg_ctx *c, void **stream) {
  if (!c || !stream) return NDG_ERR_ARG;
  *stream = (void *)c->st;
  return NDG_OK;
}

int ndg_profile_run(ndg_ctx *c, int nsteps) {
  if (!c || nsteps < 1 || !lists_ready(c)) return NDG_ERR_ARG;
  cudaSetDevice(c->device);
  int rc = ensure_params(c);
  if (rc) return rc;
  CK(c, cudaMemset(c->ring_count, 0, 4 * sizeof(int)));
  DevCtx d = devctx(c);
  const int mixed = c->precision == NDG_PREC_MIXED;
  const int tpa = choose_tpa(c);
  // the steps continue the last run (no first-step energy output), as the
  // step blocks of a run do
  launch_arm(d, c->st, c->nsys_cap, -1, nsteps, START_CONTINUE);
  launch_begin_block(d, c->st, c->nsys_cap, nsteps);
  std::vector<cudaEvent_t> ev(4 * (size_t)nsteps);
  for (auto &e : ev) CK(c, cudaEventCreate(&e));
  for (int k = 0; k < nsteps; ++k) {
    CK(c, cudaEventRecord(ev[4 * k], c->st));
    launch_rebuild(d, c->st, 1, mixed);
    CK(c, cudaEventRecord(ev[4 * k + 1], c->st));
    launch_integrate1(d, c->st, 0, mixed, tpa);
    CK(c, cudaEventRecord(ev[4 * k + 2], c->st));
    launch_pair(d, c->st, tpa, mixed, 1, 0);
    CK(c, cudaEventRecord(ev[4 * k + 3], c->st));
  }
  CK(c, cudaGetLastError());
  CK(c, cudaStreamSynchronize(c->st));
  double tr = 0, ti = 0, tp = 0;
  for (int k = 0; k < nsteps; ++k) {
    float a, b, e;
    cudaEventElapsedTime(&a, ev[4 * k], ev[4 * k + 1]);
    cudaEventElapsedTime(&b, ev[4 * k + 1], ev[4 * k + 2]);
    cudaEventElapsedTime(&e, ev[4 * k + 2], ev[4 * k + 3]);
    tr += a;
    ti += b;
    tp += e;
  }
  for (auto &e : ev) cudaEventDestroy(e);
  c->t_reb = tr / nsteps;
  c->t_int = ti / nsteps;
  c->t_pair = tp / nsteps;
  c->t_launches = 9 * nsteps;
  int count = 0;
  rc = check_words(c, &count);
  if (!rc) rc = drain_ring(c, count, nullptr, nullptr);
  int rf = flush_pending(c);
  return rc ? rc : rf;
}

int ndg_get_kernel_times(ndg_ctx *c, double *ti, double *tp, double *tr, int *launches) {
  if (!c) return NDG_ERR_ARG;
  if (ti) *ti = c->t_int;
  if (tp) *tp = c->t_pair;
  if (tr) *tr = c->t_reb;
  if (launches) *launches = c->t_launches;
  return NDG_OK;
}

}  // extern "C"
