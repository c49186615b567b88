// ndg_static.cu -- compute0 without any device allocation.
//
// ndg_compute0_static() evaluates the reference's compute0 (forces, potential
// energy, virial; src/nd.f90:200-363) for one system in FP64, with the same
// pair arithmetic as the context path (ndg_compute), but it allocates
// nothing: every scratch array it needs (link-cell counts and offsets, the
// cell-sorted atom order, per-block partial sums, the per-pair constants)
// lives in the file-scope array g_static_scratch below, which the CUDA
// driver reserves on every GPU that loads the library's device code and
// keeps until the process exits.  The caller passes its own device buffers
// for the inputs and the force output.  The call waits for its stream and
// returns the potential energy and virial on the host.
//
// Limits: STATIC_MAX_ATOMS atoms, STATIC_MAX_CELLS link cells,
// STATIC_MAX_TYPES types, STATIC_MAX_PAIRS pair potentials.
//
// All calls share the one array: two calls that run concurrently on the GPU
// (different streams, different host threads) overwrite each other's
// scratch.  Calls must be ordered, e.g. issued on one stream.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/ndyn_gpu.h"
#include "ndg_common.h"
#include "ndg_kernels.h"

namespace ndg {
namespace {

constexpr int STATIC_MAX_ATOMS = 32768;
constexpr int STATIC_MAX_CELLS = 32768;
constexpr int STATIC_MAX_TYPES = 8;
constexpr int STATIC_MAX_PAIRS = 36;
constexpr int SB = 128;  // threads per block of the force kernel
constexpr int STATIC_MAX_BLOCKS = (STATIC_MAX_ATOMS + SB - 1) / SB;

// per-call constants, copied in by the host before the kernels run
struct StaticParams {
  int np, ntypes, npairs, ptsize, ncell, nstencil, quirk;
  int mcell[3];
  int pairmat[STATIC_MAX_TYPES * STATIC_MAX_TYPES];  // gather matrix (gather_entry)
  int stencil[MAX_STENCIL];
  double ptrmin;
  double box[3];
  double rc2[STATIC_MAX_PAIRS];
  float vdr2[STATIC_MAX_PAIRS];
};

// what the host reads back after the kernels
struct StaticOut {
  double result[7];  // potential, virial(6)
  int bad_type;      // set when some typ[i] lies outside 1..ntypes
  int pad;
};

struct StaticScratch {
  StaticParams prm;
  int cell_count[STATIC_MAX_CELLS];
  int cell_start[STATIC_MAX_CELLS + 1];
  int cellof[STATIC_MAX_ATOMS];
  int slot[STATIC_MAX_ATOMS];
  int unsorted[STATIC_MAX_ATOMS];
  int order[STATIC_MAX_ATOMS];
  double partial[STATIC_MAX_BLOCKS * 7];
  StaticOut out;
};

// The scratch.  In host code this name is only a stand-in for the symbol,
// not a device address; the host obtains the address with
// cudaGetSymbolAddress (once per device) and passes it to the kernels.
static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

// link cell of each atom (src/nd.f90:1237-1248) and its slot in the cell
__global__ void ks_bin(StaticScratch *s, const double *pos, const int *typ) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const StaticParams &p = s->prm;
  if (i >= p.np) return;
  const int t = typ[i];
  if (t < 1 || t > p.ntypes) s->out.bad_type = 1;  // the force kernel skips the atom
  int ix[3];
  for (int d = 0; d < 3; ++d) {
    const double q = pos[3 * (size_t)i + d];
    const double sr = q - round(q);
    int v = (int)((sr + 0.4999) * (double)p.mcell[d]);
    ix[d] = v < 0 ? 0 : (v >= p.mcell[d] ? p.mcell[d] - 1 : v);
  }
  const int c = ix[0] + ix[1] * p.mcell[0] + ix[2] * p.mcell[0] * p.mcell[1];
  s->cellof[i] = c;
  s->slot[i] = atomicAdd(&s->cell_count[c], 1);
}

__global__ void ks_scan(StaticScratch *s) {
  // one block: exclusive scan of the cell counts
  __shared__ int wsum[32];
  __shared__ int carry;
  const int n = s->prm.ncell;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int base = 0; base < n; base += blockDim.x) {
    const int idx = base + threadIdx.x;
    const int x = idx < n ? s->cell_count[idx] : 0;
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
    if (idx < n) s->cell_start[idx] = carry + wpre + incl - x;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) carry += wpre + incl;
    __syncthreads();
  }
  if (threadIdx.x == 0) s->cell_start[n] = carry;
}

__global__ void ks_scatter(StaticScratch *s) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s->prm.np) return;
  s->unsorted[s->cell_start[s->cellof[i]] + s->slot[i]] = i;
}

// atoms of a cell in ascending index order (deterministic sums)
__global__ void ks_order(StaticScratch *s) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (c >= s->prm.ncell) return;
  const int s0 = s->cell_start[c], m = s->cell_start[c + 1] - s0;
  for (int e = threadIdx.x & 31; e < m; e += 32) {
    const int k = s->unsorted[s0 + e];
    int rank = 0;
    for (int q = 0; q < m; ++q) rank += s->unsorted[s0 + q] < k;
    s->order[s0 + rank] = k;
  }
}

// compute0 over the stencil cells of each atom: the pairs the Verlet list
// would hold (src/nd.f90:1356-1426) that lie within the potential cutoff,
// with compute0's arithmetic (src/nd.f90:283-330)
__global__ __launch_bounds__(SB) void ks_force(StaticScratch *s, const double *pos,
                                               const int *typ, const double *tabF,
                                               const double *tabP, double *force) {
  const StaticParams &p = s->prm;
  const int i = blockIdx.x * SB + threadIdx.x;
  double fx = 0, fy = 0, fz = 0, pe = 0, vir[6] = {0, 0, 0, 0, 0, 0};
  if (i < p.np && typ[i] >= 1 && typ[i] <= p.ntypes) {
    const double xi = pos[3 * (size_t)i], yi = pos[3 * (size_t)i + 1], zi = pos[3 * (size_t)i + 2];
    const int ti = typ[i];
    const int cl = s->cellof[i];
    const int M0 = p.mcell[0], M1 = p.mcell[1], M2 = p.mcell[2];
    const int cx = cl % M0, cy = (cl / M0) % M1, cz = cl / (M0 * M1);
    const int T = p.ptsize + 1;
    for (int e = 0; e < p.nstencil; ++e) {
      const int st = p.stencil[e];
      const bool center = (st >> 12) & 1;
      const int nx = (cx + (st & 15) - 1 + M0) % M0;
      const int ny = (cy + ((st >> 4) & 15) - 1 + M1) % M1;
      const int nz = (cz + ((st >> 8) & 15) - 1 + M2) % M2;
      const int nc = nx + ny * M0 + nz * M0 * M1;
      for (int q = s->cell_start[nc]; q < s->cell_start[nc + 1]; ++q) {
        const int j = s->order[q];
        if (j == i) continue;
        const int tj = typ[j];
        if (tj < 1 || tj > p.ntypes) continue;
        const int pg = p.pairmat[(ti - 1) + (tj - 1) * p.ntypes];  // gather matrix
        const int pt = pg & PT_MASK;
        if (pt <= 0) continue;
        const double ev = pg < PT_ASYM ? 1.0 : 0.0;  // one-sided pairs: force only
        double s0 = xi - pos[3 * (size_t)j], s1 = yi - pos[3 * (size_t)j + 1],
               s2 = zi - pos[3 * (size_t)j + 2];
        s0 = s0 - round(s0);
        s1 = s1 - round(s1);
        s2 = s2 - round(s2);
        const double r0 = p.box[0] * s0, r1 = p.box[1] * s1, r2 = p.box[2] * s2;
        double d2 = r0 * r0;
        d2 = d2 + r1 * r1;
        d2 = d2 + r2 * r2;
        if (center && d2 < p.ptrmin) continue;
        if (d2 > p.rc2[pt - 1]) continue;
        const float rk = (float)(d2 - p.ptrmin) * p.vdr2[pt - 1] + 1.0f;
        int kk = (int)rk;
        if (kk < 1) kk = 1;
        const double w = (double)rk - (double)kk;
        const int base = (pt - 1) * T + kk - 1;
        double df = w * tabF[base + 1] + (1.0 - w) * tabF[base];
        df = df / d2;
        fx = fx + r0 * df;
        fy = fy + r1 * df;
        fz = fz + r2 * df;
        if (ev != 0.0) {
          pe = pe + (w * tabP[base + 1] + (1.0 - w) * tabP[base]);
          vir[0] = vir[0] + r0 * r0 * df;
          vir[1] = vir[1] + r1 * r1 * df;
          vir[2] = vir[2] + r2 * r2 * df;
          vir[3] = vir[3] + r0 * r1 * df;
          vir[4] = vir[4] + r0 * r2 * df;
          vir[5] = vir[5] + r1 * r2 * df;
        }
      }
    }
  }
  if (i < p.np) {
    force[3 * (size_t)i] = fx;
    force[3 * (size_t)i + 1] = fy;
    force[3 * (size_t)i + 2] = fz;
  }
  // block partials in a fixed order
  __shared__ double sm[7][SB];
  sm[0][threadIdx.x] = pe;
  for (int k = 0; k < 6; ++k) sm[1 + k][threadIdx.x] = vir[k];
  __syncthreads();
  for (int h = SB / 2; h > 0; h >>= 1) {
    if (threadIdx.x < h)
      for (int k = 0; k < 7; ++k) sm[k][threadIdx.x] += sm[k][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < 7; ++k) s->partial[7 * blockIdx.x + k] = sm[k][0];
}

__global__ void ks_reduce(StaticScratch *s, int nblk) {
  // one warp: partial sums over blocks in a fixed order, then halve (each
  // pair was visited from both atoms)
  for (int k = threadIdx.x; k < 7; k += blockDim.x) {
    double a = 0.0;
    for (int b = 0; b < nblk; ++b) a += s->partial[7 * b + k];
    s->out.result[k] = 0.5 * a;
  }
}

std::mutex g_mu;
StaticScratch *g_addr[128];  // device address of the scratch, per device
bool g_ready[128];

}  // namespace
}  // namespace ndg

using namespace ndg;

extern "C" int ndg_compute0_static(int np, int ntypes, int npairs, int ptsize, double ptrmin,
                                   const int *pairmat, const double *rcpair, double skin,
                                   int quirk, const double *box, const double *fpair_d,
                                   const double *ppair_d, const double *pos_d, const int *typ_d,
                                   double *force_d, double *potential, double *virial,
                                   void *stream) {
  if (np < 1 || ntypes < 1 || npairs < 1 || ptsize < 2 || !pairmat || !rcpair || !box ||
      !fpair_d || !ppair_d || !pos_d || !typ_d || !force_d || (quirk != 0 && quirk != 1))
    return NDG_ERR_ARG;
  if (np > STATIC_MAX_ATOMS || ntypes > STATIC_MAX_TYPES || npairs > STATIC_MAX_PAIRS) {
    std::fprintf(stderr,
                 "ndg_compute0_static: %d atoms, %d types, %d pairs exceed the static scratch "
                 "limits (%d atoms, %d types, %d pairs)\n",
                 np, ntypes, npairs, STATIC_MAX_ATOMS, STATIC_MAX_TYPES, STATIC_MAX_PAIRS);
    return NDG_ERR_ARG;
  }
  cudaStream_t st = (cudaStream_t)stream;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 128) return NDG_ERR_CUDA;
  StaticScratch *s = nullptr;
  {
    // set-up once per device, with that device current: the device address
    // of the scratch array (a host-side use of the symbol name itself would
    // not be a device address)
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_ready[dev]) {
      void *ptr = nullptr;
      if (cudaGetSymbolAddress(&ptr, g_static_scratch) != cudaSuccess || !ptr) {
        std::fprintf(stderr, "ndg_compute0_static: cudaGetSymbolAddress failed on device %d\n",
                     dev);
        return NDG_ERR_CUDA;
      }
      g_addr[dev] = (StaticScratch *)ptr;
      g_ready[dev] = true;
    }
    s = g_addr[dev];
  }
  // per-call constants (host -> device scratch)
  StaticParams p;
  std::memset(&p, 0, sizeof(p));
  p.np = np;
  p.ntypes = ntypes;
  p.npairs = npairs;
  p.ptsize = ptsize;
  p.quirk = quirk;
  p.ptrmin = ptrmin;
  double rcut = rcpair[0];
  for (int j = 1; j < npairs; ++j) rcut = rcpair[j] > rcut ? rcpair[j] : rcut;
  // the cell grid: MCELL = int(box/(rcut+skin)), src/nd.f90:80-83, worked
  // out in double and bounded before any cast, so no size can wrap
  const double rl = rcut + skin;
  if (!(skin >= 0.0) || !(rl > 0.0) || !std::isfinite(rl)) return NDG_ERR_ARG;
  long long ncell = 1;
  for (int d = 0; d < 3; ++d) {
    if (!(box[d] > 0.0) || !std::isfinite(box[d])) return NDG_ERR_ARG;
    const double m = std::floor(box[d] / rl);
    if (m < 2.0) return NDG_ERR_CELLS;
    if (m > (double)STATIC_MAX_CELLS) {
      std::fprintf(stderr, "ndg_compute0_static: %.0f link cells along axis %d exceed the static "
                   "limit of %d\n", m, d + 1, STATIC_MAX_CELLS);
      return NDG_ERR_ARG;
    }
    p.box[d] = box[d];
    p.mcell[d] = (int)m;
    ncell *= p.mcell[d];
  }
  if (ncell > STATIC_MAX_CELLS) {
    std::fprintf(stderr, "ndg_compute0_static: %lld link cells exceed the static limit of %d\n",
                 ncell, STATIC_MAX_CELLS);
    return NDG_ERR_ARG;
  }
  p.ncell = (int)ncell;
  for (int k = 0; k < ntypes * ntypes; ++k)
    if (pairmat[k] < 0 || pairmat[k] > npairs) return NDG_ERR_ARG;
  for (int b = 1; b <= ntypes; ++b)
    for (int a = 1; a <= ntypes; ++a)
      p.pairmat[(a - 1) + (b - 1) * ntypes] = gather_entry(pairmat, ntypes, a, b);
  for (int j = 0; j < npairs; ++j) {
    p.rc2[j] = rcpair[j] * rcpair[j];
    p.vdr2[j] = (float)(1.0 / ((p.rc2[j] - ptrmin) / (ptsize - 1)));
  }
  p.nstencil = make_stencil(p.mcell, quirk, p.stencil);
  cudaError_t e = cudaMemcpyAsync(&s->prm, &p, sizeof(p), cudaMemcpyHostToDevice, st);
  // the cell counts accumulate with atomics and the type check only ever
  // sets its flag: both must start at zero, and the array still holds the
  // previous call's values
  if (e == cudaSuccess) e = cudaMemsetAsync(s->cell_count, 0, (size_t)ncell * sizeof(int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(&s->out.bad_type, 0, sizeof(int), st);
  if (e != cudaSuccess) return NDG_ERR_CUDA;
  const int nb = (np + SB - 1) / SB;
  ks_bin<<<nb, SB, 0, st>>>(s, pos_d, typ_d);
  ks_scan<<<1, 1024, 0, st>>>(s);
  ks_scatter<<<nb, SB, 0, st>>>(s);
  ks_order<<<(p.ncell + 7) / 8, 256, 0, st>>>(s);
  ks_force<<<nb, SB, 0, st>>>(s, pos_d, typ_d, fpair_d, ppair_d, force_d);
  ks_reduce<<<1, 32, 0, st>>>(s, nb);
  StaticOut res;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(&res, &s->out, sizeof(res), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return NDG_ERR_CUDA;
  if (res.bad_type) {
    std::fprintf(stderr, "ndg_compute0_static: an atom type lies outside 1..%d\n", ntypes);
    return NDG_ERR_ARG;
  }
  if (potential) *potential = res.result[0];
  if (virial)
    for (int k = 0; k < 6; ++k) virial[k] = res.result[1 + k];
  return NDG_OK;
}
