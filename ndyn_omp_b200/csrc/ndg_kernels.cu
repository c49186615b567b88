// ndg_kernels.cu -- sm_100a kernels of the Ndyn MD timestep path.
//
// Compiled with --fmad=false: every FP64 expression that restates the
// reference keeps its literal operation order (the neighbour list and the
// link-cell assignment are compared bit for bit with the reference's
// arithmetic).  The mixed-precision pair kernel asks for FMAs explicitly.
//
// Kernels of one MD step (src/nd.f90:137-178), all systems in one launch:
//   [rebuild]  k_bin -> k_scan -> k_scatter -> k_order -> k_permute ->
//              k_copyback -> k_build        (only systems whose check fired)
//   k_integrate1                           (integrate1 + pending mkIso* scales)
//   k_pair<TPA,MIXED,FUSE>                 (compute0 + integrate2, and in the
//                                           last block of each system:
//                                           reductions, write_thermo,
//                                           mkIsoKE/P/E, BoxVel, next step's
//                                           CheckListUpdate decision)
#include <cstdio>

#include "ndg_kernels.h"

namespace ndg {

__device__ __forceinline__ int tw_of(double w) { return (int)__double_as_longlong(w); }

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
// integrate1, src/nd.f90:1027-1046; applies velocity scales left pending by
// the previous step's mkIsoKE/mkIsoE first (src/nd.f90:1145-1155,1173-1180).
// Emits each chunk's two largest displacement measures for the next
// CheckListUpdate.
__global__ __launch_bounds__(BLOCK) void k_integrate1(DevCtx c, int standalone, int mixed) {
  const int chunk = blockIdx.x;
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
        const double du0 = li0 * (v0 * dt + 0.5 * a0 * dt * dt);
        const double du1 = li1 * (v1 * dt + 0.5 * a1 * dt * dt);
        const double du2 = li2 * (v2 * dt + 0.5 * a2 * dt * dt);
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
__device__ void finalize_system(const DevCtx &c, int sys, int blk0, int nblk, int flags,
                                int fuse) {
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  __shared__ double sm[8 * 32];
  double v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
    const double *r = c.red + 8 * (size_t)(blk0 + b);
#pragma unroll
    for (int k = 0; k < 8; ++k) v[k] += __ldcg(r + k);
  }
  block_sum<8>(v, sm);
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
    S->flags = step_flags(*P, S->step, S->tt) | F_ACTIVE;
    int rb = 0;
    if (P->renei && S->step % P->renei_freq == 0) {
      rb = list_check(*P, *S, t1, t2);
      if (rb < 0) {
        set_err(c, S, E_OUT_OF_BOX);
        rb = 0;
      }
    }
    if (rb && P->quirk != 0) {
      // fixed semantics: cells must stay at least rcut+skin wide
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
  } else {
    S->flags = 0;
    S->rebuild = 0;
  }
}

// ---------------------------------------------------------------------------
// Pair loop: compute0 (src/nd.f90:273-333) over the full neighbour list,
// TPA threads per atom, and with FUSE the integrate2 update
// (src/nd.f90:1094-1116) of the atom as soon as its force is complete.
template <int TPA, bool MIXED, bool FUSE>
__global__ __launch_bounds__(BLOCK) void k_pair(DevCtx c, int host_flags) {
  constexpr int APB = BLOCK / TPA;
  const int a0 = blockIdx.x * APB;
  const int sys = c.chunk_sys[a0 / ATOM_ALIGN];
  if (sys < 0) return;
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  const int flags = FUSE ? S->flags : host_flags;
  if (FUSE && !(flags & F_ACTIVE)) return;
  if (!FUSE && P->n == 0) return;

  const int g = threadIdx.x / TPA, la = threadIdx.x % TPA;
  const int i = a0 + g;
  const int local = i - P->atom_off;
  const bool valid = local < P->n;
  const bool cu = flags & F_CU, cv = flags & F_CV;

  double pe = 0.0, vir[6] = {0, 0, 0, 0, 0, 0};
  double fx = 0.0, fy = 0.0, fz = 0.0;
  long long qx = 0, qy = 0, qz = 0;  // mixed: 64-bit fixed-point force
  int ti = 1;
  if (valid) {
    const int ntypes = P->ntypes, ptsize1 = P->ptsize + 1;
    const int *__restrict__ pm = c.pairmat + P->pm_off;
    const int *__restrict__ nb = c.nbr + P->nbr_off + local;
    const long long stride = P->npad;
    int cnt = c.nnb[i];
    cnt = cnt < P->maxnb ? cnt : P->maxnb;
    if (!MIXED) {
      const double4 pi = c.pos[i];
      ti = tw_type(tw_of(pi.w));
      const double b0 = S->box[0], b1 = S->box[1], b2 = S->box[2];
      const double ptrmin = P->ptrmin;
      const double *__restrict__ rc2 = c.rc2 + P->pair_off;
      const float *__restrict__ vdr2 = c.vdr2 + P->pair_off;
      const double *__restrict__ tF = c.tabF + P->tab_off;
      const double *__restrict__ tP = c.tabP + P->tab_off;
      for (int k = la; k < cnt; k += TPA) {
        const int j = __ldg(nb + k * stride);
        const double4 pj = c.pos[j];
        const int tj = tw_type(tw_of(pj.w));
        const int pt = __ldg(pm + (ti - 1) + (tj - 1) * ntypes);
        if (pt <= 0) continue;
        double s0 = pi.x - pj.x, s1 = pi.y - pj.y, s2 = pi.z - pj.z;
        s0 = s0 - round(s0);
        s1 = s1 - round(s1);
        s2 = s2 - round(s2);
        const double r0 = b0 * s0, r1 = b1 * s1, r2 = b2 * s2;
        double d2 = r0 * r0;
        d2 = d2 + r1 * r1;
        d2 = d2 + r2 * r2;
        if (d2 > __ldg(rc2 + pt - 1)) continue;
        const float rk = (float)(d2 - ptrmin) * __ldg(vdr2 + pt - 1) + 1.0f;
        int kk = (int)rk;
        if (kk < 1) kk = 1;
        const double w = (double)rk - (double)kk;
        const int base = (pt - 1) * ptsize1 + kk - 1;
        double df = w * __ldg(tF + base + 1) + (1.0 - w) * __ldg(tF + base);
        df = df / d2;
        fx = fx + r0 * df;
        fy = fy + r1 * df;
        fz = fz + r2 * df;
        if (cu) pe = pe + (w * __ldg(tP + base + 1) + (1.0 - w) * __ldg(tP + base));
        if (cv) {
          vir[0] = vir[0] + r0 * r0 * df;
          vir[1] = vir[1] + r1 * r1 * df;
          vir[2] = vir[2] + r2 * r2 * df;
          vir[3] = vir[3] + r0 * r1 * df;
          vir[4] = vir[4] + r0 * r2 * df;
          vir[5] = vir[5] + r1 * r2 * df;
        }
      }
    } else {
      const int4 pi = c.pfx[i];
      ti = tw_type(pi.w);
      const float sb0 = (float)(S->box[0] * (1.0 / FX_ONE));
      const float sb1 = (float)(S->box[1] * (1.0 / FX_ONE));
      const float sb2 = (float)(S->box[2] * (1.0 / FX_ONE));
      const float ptrmin = (float)P->ptrmin;
      const float *__restrict__ rc2 = c.rc2f + P->pair_off;
      const float *__restrict__ vdr2 = c.vdr2 + P->pair_off;
      const float2 *__restrict__ tF = c.tabF2 + P->tab_off;
      const float2 *__restrict__ tP = c.tabP2 + P->tab_off;
      float ax = 0.f, ay = 0.f, az = 0.f, ape = 0.f;
      float av0 = 0.f, av1 = 0.f, av2 = 0.f, av3 = 0.f, av4 = 0.f, av5 = 0.f;
      int nacc = 0;
      for (int k = la; k < cnt; k += TPA) {
        const int j = __ldg(nb + k * stride);
        const int4 pj = c.pfx[j];
        const int tj = tw_type(pj.w);
        const int pt = __ldg(pm + (ti - 1) + (tj - 1) * ntypes);
        if (pt <= 0) continue;
        const float r0 = (float)(int)((unsigned)pi.x - (unsigned)pj.x) * sb0;
        const float r1 = (float)(int)((unsigned)pi.y - (unsigned)pj.y) * sb1;
        const float r2 = (float)(int)((unsigned)pi.z - (unsigned)pj.z) * sb2;
        const float d2 = __fmaf_rn(r0, r0, __fmaf_rn(r1, r1, __fmul_rn(r2, r2)));
        if (d2 > __ldg(rc2 + pt - 1)) continue;
        const float rk = __fmaf_rn(d2 - ptrmin, __ldg(vdr2 + pt - 1), 1.0f);
        int kk = (int)rk;
        if (kk < 1) kk = 1;
        const float w = rk - (float)kk;
        const int base = (pt - 1) * (P->ptsize + 1) + kk - 1;
        const float2 F = __ldg(tF + base);
        const float df = __fdividef(__fmaf_rn(w, F.y - F.x, F.x), d2);
        ax = __fmaf_rn(r0, df, ax);
        ay = __fmaf_rn(r1, df, ay);
        az = __fmaf_rn(r2, df, az);
        if (cu) {
          const float2 Pp = __ldg(tP + base);
          ape += __fmaf_rn(w, Pp.y - Pp.x, Pp.x);
        }
        if (cv) {
          const float r0d = r0 * df, r1d = r1 * df;
          av0 = __fmaf_rn(r0d, r0, av0);
          av1 = __fmaf_rn(r1d, r1, av1);
          av2 = __fmaf_rn(r2 * df, r2, av2);
          av3 = __fmaf_rn(r0d, r1, av3);
          av4 = __fmaf_rn(r0d, r2, av4);
          av5 = __fmaf_rn(r1d, r2, av5);
        }
        if (++nacc == 8) {
          // flush the FP32 partial sums into the 64-bit fixed-point totals
          qx += __float2ll_rn(ax * (float)FORCE_FX);
          qy += __float2ll_rn(ay * (float)FORCE_FX);
          qz += __float2ll_rn(az * (float)FORCE_FX);
          ax = ay = az = 0.f;
          nacc = 0;
        }
      }
      qx += __float2ll_rn(ax * (float)FORCE_FX);
      qy += __float2ll_rn(ay * (float)FORCE_FX);
      qz += __float2ll_rn(az * (float)FORCE_FX);
      pe = (double)ape;
      vir[0] = av0; vir[1] = av1; vir[2] = av2; vir[3] = av3; vir[4] = av4; vir[5] = av5;
    }
  }
  if (!MIXED) {
    // combine the TPA partial forces of an atom (fixed tree: deterministic)
#pragma unroll
    for (int o = TPA / 2; o > 0; o >>= 1) {
      fx += __shfl_xor_sync(0xffffffffu, fx, o);
      fy += __shfl_xor_sync(0xffffffffu, fy, o);
      fz += __shfl_xor_sync(0xffffffffu, fz, o);
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
      const double rmass = 1.0 / c.mass[P->type_off + ti - 1];
      const double dt = P->dt;
      double *v = c.vel + 3 * (size_t)i;
      double *a = c.acc + 3 * (size_t)i;
      const double v0 = v[0] + 0.5 * dt * (fx * rmass + a[0]);
      const double v1 = v[1] + 0.5 * dt * (fy * rmass + a[1]);
      const double v2 = v[2] + 0.5 * dt * (fz * rmass + a[2]);
      v[0] = v0; v[1] = v1; v[2] = v2;
      a[0] = fx * rmass; a[1] = fy * rmass; a[2] = fz * rmass;
      if (flags & F_CK) {
        double kt = v0 * v0;
        kt = kt + v1 * v1;
        kt = kt + v2 * v2;
        ke = kt * c.mass[P->type_off + ti - 1];
      }
    } else {
      double *f = c.force + 3 * (size_t)i;
      f[0] = fx; f[1] = fy; f[2] = fz;
    }
  }
  __shared__ double sm[8 * 32];
  double red[8] = {pe, vir[0], vir[1], vir[2], vir[3], vir[4], vir[5], ke};
  block_sum<8>(red, sm);
  __shared__ int last;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < 8; ++k) c.red[8 * (size_t)blockIdx.x + k] = red[k];
    __threadfence();
    const unsigned nblk = (unsigned)(P->npad / APB);
    const unsigned t = atomicAdd(&S->ticket, 1u);
    last = (t == nblk - 1);
  }
  __syncthreads();
  if (last) {
    __threadfence();
    finalize_system(c, sys, P->atom_off / APB, P->npad / APB, flags, FUSE);
    if (threadIdx.x == 0) S->ticket = 0;
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
__global__ void k_begin_run(DevCtx c, int nsys_cap, int nsteps, int cont) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= nsys_cap) return;
  const SysParam &P = c.P[s];
  SysState &S = c.S[s];
  if (P.n == 0) {
    S.flags = 0;
    return;
  }
  S.steps_left = nsteps;
  S.tt = 1;
  S.step = S.step + 1;
  S.flags = step_flags(P, S.step, 1) | F_ACTIVE;
  for (int d = 0; d < 3; ++d) S.li[d] = 1.0 / S.box[d];
  int rb = 0;
  if (cont && P.renei && S.step % P.renei_freq == 0) {
    rb = list_check(P, S, S.dtop[0], S.dtop[1]);
    if (rb < 0) {
      set_err(c, &S, E_OUT_OF_BOX);
      rb = 0;
    }
  }
  S.rebuild = rb;
  S.ticket = 0;
  S.ticket_i = 0;
}

// apply pending mkIsoKE/mkIsoE velocity scales at the end of a run
__global__ __launch_bounds__(BLOCK) void k_flush(DevCtx c) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0) return;
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

__global__ void k_clear_pend(DevCtx c, int nsys_cap) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s < nsys_cap) c.S[s].pend = 0;
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
}

// ---------------------------------------------------------------------------
// List rebuild: buildCellList + buildVerletList (src/nd.f90:1214-1446).

__device__ __forceinline__ bool rebuilding(const DevCtx &c, int sys, int force_all) {
  return force_all || c.S[sys].rebuild;
}

// link cell of each atom, src/nd.f90:1237-1248, counted with warp-aggregated
// atomics (lanes with the same cell elect one atomicAdd)
__global__ __launch_bounds__(BLOCK) void k_bin(DevCtx c, int force_all) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0 || !rebuilding(c, sys, force_all)) return;
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

// exclusive scan of the cell counts of one system (one block per system)
__global__ __launch_bounds__(1024) void k_scan(DevCtx c, int nsys_cap, int force_all) {
  const int s = blockIdx.x;
  if (s >= nsys_cap) return;
  const SysParam *__restrict__ P = c.P + s;
  SysState *S = c.S + s;
  if (P->n == 0 || !(force_all || S->rebuild)) return;
  __shared__ int wsum[32];
  __shared__ int carry;
  if (threadIdx.x == 0) carry = 0;
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
    for (int d = 0; d < 3; ++d) S->box_build[d] = S->box[d];
    if (!force_all) S->nlist_updates += 1;
  }
}

__global__ __launch_bounds__(BLOCK) void k_scatter(DevCtx c, int force_all) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0 || !rebuilding(c, sys, force_all)) return;
  const SysParam *__restrict__ P = c.P + sys;
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  const int dest = c.cell_start[P->cell_off + c.atom_cell[i]] + c.atom_slot[i];
  c.tmp_src[P->atom_off + dest] = i;
  c.tmp_key[P->atom_off + dest] = c.gid[i];
}

// order the atoms of each cell by original id (one warp per cell) so the
// layout, and the neighbour order, do not depend on atomic timing
__global__ __launch_bounds__(BLOCK) void k_order(DevCtx c, int force_all) {
  const int gc = blockIdx.x * (BLOCK / 32) + (threadIdx.x >> 5);
  if (gc >= c.ncells) return;
  const int sys = c.cell_sys[gc];
  if (sys < 0 || !rebuilding(c, sys, force_all)) return;
  const SysParam *__restrict__ P = c.P + sys;
  const int cl = gc - P->cell_off;
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

__global__ __launch_bounds__(BLOCK) void k_permute(DevCtx c, int force_all) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0 || !rebuilding(c, sys, force_all)) return;
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

__global__ __launch_bounds__(BLOCK) void k_copyback(DevCtx c, int force_all, int mixed) {
  const int chunk = blockIdx.x;
  const int sys = c.chunk_sys[chunk];
  if (sys < 0 || !rebuilding(c, sys, force_all)) return;
  const SysParam *__restrict__ P = c.P + sys;
  if (threadIdx.x == 0) {
    c.itop[2 * chunk] = 0.0;  // dispList was reset: the displacement measure is 0
    c.itop[2 * chunk + 1] = 0.0;
  }
  const int i = chunk * ATOM_ALIGN + threadIdx.x;
  if (i - P->atom_off >= P->n) return;
  const double4 p = c.s_pos[i];
  c.pos[i] = p;
  if (mixed) c.pfx[i] = make_int4(fx32(p.x), fx32(p.y), fx32(p.z), tw_of(p.w));
  for (int d = 0; d < 3; ++d) {
    c.vel[3 * (size_t)i + d] = c.s_vel[3 * (size_t)i + d];
    c.acc[3 * (size_t)i + d] = c.s_acc[3 * (size_t)i + d];
    c.disp[3 * (size_t)i + d] = 0.0;  // src/nd.f90:1384,1427
  }
  c.gid[i] = c.s_gid[i];
  c.atom_cell[i] = c.s_cell[i];
}

// Neighbour build: one CTA per link cell stages the atoms of its stencil
// cells in shared memory; a warp takes one atom i of the cell, tests 32
// candidates per pass and compacts the hits with __ballot_sync/__popc into
// the padded SoA list.  Criteria of buildVerletList (src/nd.f90:1356-1383
// for the cell itself, :1403-1426 for the neighbour cells).
constexpr int NB_THREADS = 128;
constexpr int NB_CAP = 768;    // candidates staged per pass
constexpr int NB_IBATCH = 128; // own atoms per pass

__global__ __launch_bounds__(NB_THREADS) void k_build(DevCtx c, int force_all) {
  const int gc = blockIdx.x;
  const int sys = c.cell_sys[gc];
  if (sys < 0 || !rebuilding(c, sys, force_all)) return;
  const SysParam *__restrict__ P = c.P + sys;
  SysState *S = c.S + sys;
  const int cl = gc - P->cell_off;
  const int M0 = S->mcell[0], M1 = S->mcell[1], M2 = S->mcell[2];
  if (cl >= S->ncell) return;

  __shared__ double4 cpos[NB_CAP];
  __shared__ int cj[NB_CAP];
  __shared__ int ent_start[MAX_STENCIL + 1], ent_cell[MAX_STENCIL], ent_center[MAX_STENCIL];
  __shared__ int ncnt[NB_IBATCH];
  __shared__ int nent;

  const int *cst = c.cell_start + P->cell_off;
  if (threadIdx.x == 0) {
    int st[MAX_STENCIL];
    const int m[3] = {M0, M1, M2};
    const int ne = make_stencil(m, P->quirk, st);
    const int cx = cl % M0, cy = (cl / M0) % M1, cz = cl / (M0 * M1);
    int tot = 0;
    for (int e = 0; e < ne; ++e) {
      const int dx = (st[e] & 15) - 1, dy = ((st[e] >> 4) & 15) - 1, dz = ((st[e] >> 8) & 15) - 1;
      const int nx = (cx + dx + M0) % M0, ny = (cy + dy + M1) % M1, nz = (cz + dz + M2) % M2;
      const int nc = nx + ny * M0 + nz * M0 * M1;
      ent_cell[e] = nc;
      ent_center[e] = (st[e] >> 12) & 1;
      ent_start[e] = tot;
      tot += cst[nc + 1] - cst[nc];
    }
    ent_start[ne] = tot;
    nent = ne;
  }
  __syncthreads();
  const int ne = nent;
  const int ncand = ent_start[ne];
  const int own0 = cst[cl], own1 = cst[cl + 1];
  const double b0 = S->box[0], b1 = S->box[1], b2 = S->box[2];
  const double ptrmin = P->ptrmin;
  const int ntypes = P->ntypes;
  const int *__restrict__ pm = c.pairmat + P->pm_off;
  const double *__restrict__ rl2 = c.rlist2 + P->pair_off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const long long stride = P->npad;
  const int maxnb = P->maxnb;

  for (int ib = own0; ib < own1; ib += NB_IBATCH) {
    const int ie = min(ib + NB_IBATCH, own1);
    for (int t = threadIdx.x; t < NB_IBATCH; t += NB_THREADS) ncnt[t] = 0;
    for (int q0 = 0; q0 < ncand; q0 += NB_CAP) {
      const int q1 = min(q0 + NB_CAP, ncand);
      __syncthreads();
      for (int q = q0 + threadIdx.x; q < q1; q += NB_THREADS) {
        int e = 0;
        while (ent_start[e + 1] <= q) ++e;
        const int j = P->atom_off + cst[ent_cell[e]] + (q - ent_start[e]);
        cpos[q - q0] = c.pos[j];
        cj[q - q0] = j | (ent_center[e] << 31);
      }
      __syncthreads();
      for (int il = ib + warp; il < ie; il += NB_THREADS / 32) {
        const int i = P->atom_off + il;
        const double4 pi = c.pos[i];
        const int ti = tw_type(tw_of(pi.w));
        int cnt = ncnt[il - ib];
        for (int qb = 0; qb < q1 - q0; qb += 32) {
          const int q = qb + lane;
          bool hit = false;
          int j = 0;
          if (q < q1 - q0) {
            const int raw = cj[q];
            j = raw & 0x7fffffff;
            const bool center = raw < 0;
            const double4 pj = cpos[q];
            const int tj = tw_type(tw_of(pj.w));
            const int a = __ldg(pm + (ti - 1) + (tj - 1) * ntypes);
            const int b = __ldg(pm + (tj - 1) + (ti - 1) * ntypes);
            const int mx = a > b ? a : b;
            if (j != i && mx > 0) {
              double s0 = pi.x - pj.x, s1 = pi.y - pj.y, s2 = pi.z - pj.z;
              s0 = s0 - round(s0);
              s1 = s1 - round(s1);
              s2 = s2 - round(s2);
              const double r0 = b0 * s0, r1 = b1 * s1, r2 = b2 * s2;
              double d2 = r0 * r0;
              d2 = d2 + r1 * r1;
              d2 = d2 + r2 * r2;
              hit = !(center && d2 < ptrmin) && !(d2 > __ldg(rl2 + mx - 1));
            }
          }
          const unsigned bal = __ballot_sync(0xffffffffu, hit);
          if (hit) {
            const int k = cnt + __popc(bal & ((1u << lane) - 1u));
            if (k < maxnb) c.nbr[P->nbr_off + (long long)k * stride + il] = j;
          }
          cnt += __popc(bal);
        }
        if (lane == 0) ncnt[il - ib] = cnt;
      }
    }
    __syncthreads();
    for (int il = ib + threadIdx.x; il < ie; il += NB_THREADS) {
      const int cnt = ncnt[il - ib];
      c.nnb[P->atom_off + il] = cnt;
      if (cnt > maxnb) set_err(c, S, E_NEIMAX);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// launchers
void launch_integrate1(const DevCtx &c, cudaStream_t st, int standalone, int mixed) {
  k_integrate1<<<c.nchunks, BLOCK, 0, st>>>(c, standalone, mixed);
}

template <int TPA>
static void pair_tpa(const DevCtx &c, cudaStream_t st, int mixed, int fuse, int hf) {
  const int grid = c.nchunks * TPA;
  if (mixed) {
    if (fuse) k_pair<TPA, true, true><<<grid, BLOCK, 0, st>>>(c, hf);
    else k_pair<TPA, true, false><<<grid, BLOCK, 0, st>>>(c, hf);
  } else {
    if (fuse) k_pair<TPA, false, true><<<grid, BLOCK, 0, st>>>(c, hf);
    else k_pair<TPA, false, false><<<grid, BLOCK, 0, st>>>(c, hf);
  }
}

void launch_pair(const DevCtx &c, cudaStream_t st, int tpa, int mixed, int fuse, int hf) {
  switch (tpa) {
    case 1: pair_tpa<1>(c, st, mixed, fuse, hf); break;
    case 2: pair_tpa<2>(c, st, mixed, fuse, hf); break;
    case 4: pair_tpa<4>(c, st, mixed, fuse, hf); break;
    case 8: pair_tpa<8>(c, st, mixed, fuse, hf); break;
    case 16: pair_tpa<16>(c, st, mixed, fuse, hf); break;
    default: pair_tpa<32>(c, st, mixed, fuse, hf); break;
  }
}

void launch_integrate2(const DevCtx &c, cudaStream_t st, int ck) {
  k_integrate2<<<c.nchunks, BLOCK, 0, st>>>(c, ck);
}

void launch_rebuild(const DevCtx &c, cudaStream_t st, int force_all, int mixed) {
  k_bin<<<c.nchunks, BLOCK, 0, st>>>(c, force_all);
  k_scan<<<c.nsys_cap, 1024, 0, st>>>(c, c.nsys_cap, force_all);
  k_scatter<<<c.nchunks, BLOCK, 0, st>>>(c, force_all);
  k_order<<<(c.ncells + BLOCK / 32 - 1) / (BLOCK / 32), BLOCK, 0, st>>>(c, force_all);
  k_permute<<<c.nchunks, BLOCK, 0, st>>>(c, force_all);
  k_copyback<<<c.nchunks, BLOCK, 0, st>>>(c, force_all, mixed);
  k_build<<<c.ncells, NB_THREADS, 0, st>>>(c, force_all);
}

void launch_begin_run(const DevCtx &c, cudaStream_t st, int nsys_cap, int nsteps, int cont) {
  (void)nsys_cap;
  k_begin_run<<<(nsys_cap + 127) / 128, 128, 0, st>>>(c, nsys_cap, nsteps, cont);
}

void launch_flush(const DevCtx &c, cudaStream_t st, int nsys_cap) {
  k_flush<<<c.nchunks, BLOCK, 0, st>>>(c);
  k_clear_pend<<<(nsys_cap + 127) / 128, 128, 0, st>>>(c, nsys_cap);
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
