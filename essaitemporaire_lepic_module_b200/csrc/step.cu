// Fused FP64 timestep kernels of the device-resident step loop.
//
// k_push_deposit_f64 does, for one species and in one pass over the particle
// stream, what Src/part_expmover.f90 does in two routines: the trilinear
// gather + Boris push + loss test of part_mover (lines 55-272) and the CIC
// deposition of the new position of charge_deposition (lines 591-656).  The
// new state is written in place (96 B per particle: one read and one write of
// x,y,z,vx,vy,vz).  The eight node weights of the particles of a warp that
// deposit into the same cell are grouped by a bitonic sort of the warp's
// deposit cells, summed by a warp-segmented reduction and added by one lane:
// a warp issues 8 global FP64 atomics per distinct cell instead of 8 per
// particle (particles are kept cell-sorted, so a warp holds few cells).  A
// shared-memory tile was measured slower: its block barriers stall the memory
// stream.  kq (1 or 2) is applied to the summed weight, which is exact.
//
// Lost and dead particles leave holes (flag_dead = 2) that k_fill_* close by
// moving alive particles from the tail into them: the work is proportional to
// the number of holes, not to N.  The order of the particles changes; the
// periodic sort restores cell order.  (The drop-in part_mover_ keeps the
// reference's in-order compaction.)
#include <cstring>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int FB = 256;

struct FusedConst {
  double h0, h1, h2, dt, k1, Nm, mass, kdep;
  double Bx, By, Bz;
  int boris, flag_nmn, flag_pbc, ngrid;
  double ymax, zmax;
};

__device__ __forceinline__ unsigned lanemask_le() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// run id of each lane: runs are maximal groups of consecutive lanes with the
// same key
__device__ __forceinline__ int run_id(long long key, bool &head) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  long long prev = __shfl_up_sync(full, key, 1);
  head = (lane == 0) || (prev != key);
  unsigned heads = __ballot_sync(full, head);
  return __popc(heads & lanemask_le());
}

// BMAP: B from the map m (else the uniform c.Bx, c.By, c.Bz)
template <bool BMAP>
__global__ void __launch_bounds__(FB) k_push_deposit_f64(
    Dims d, FusedConst c, BMapF64 m, Dielectric die, const double *__restrict__ Ei, const int *__restrict__ bcnd,
    const unsigned char *__restrict__ cw, double *__restrict__ p, long long cap,
    const int *__restrict__ count, signed char *__restrict__ flag, const double *__restrict__ kq,
    double *__restrict__ np, int *__restrict__ holes, int *__restrict__ nholes,
    double *__restrict__ acc, int *__restrict__ err) {
  const unsigned full = 0xffffffffu;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int N = *count;
  long long q = -1;  // deposit base node of this lane, -1: nothing to deposit
  double w0 = 0, w1 = 0, w2 = 0, w3 = 0, w4 = 0, w5 = 0, w6 = 0, w7 = 0;
  bool hole = false;
  if (i < N) {
    double xp = p[i], yp = p[cap + i], zp = p[2 * cap + i];
    double vx = p[3 * cap + i], vy = p[4 * cap + i], vz = p[5 * cap + i];
    const signed char fl = flag[i];
    if (fl == 1) {
      // killed in a collision: removed here (Src/part_expmover.f90:70-84)
      atomicAdd(&acc[1], -(0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz)));
      hole = true;
    } else if (!(xp >= 0.0 && yp >= 0.0 && zp >= 0.0 && xp < (d.n1 + 1) * c.h0 &&
                 yp < (d.n2 + 1) * c.h1 && zp < (d.n3 + 1) * c.h2)) {
      raise_err(err, LEPIC_ERR_CELL, (int)i);
      hole = true;
    } else {
      // ---- gather + push (same expression order as the drop-in kernel)
      int ix = (int)(xp / c.h0) + 1, iy = (int)(yp / c.h1) + 1, iz = (int)(zp / c.h2) + 1;
      double px = (ix * c.h0 - xp) / c.h0;
      double py = (iy * c.h1 - yp) / c.h1;
      double pz = (iz * c.h2 - zp) / c.h2;
      const double k0 = px * py * pz, ka = (1.0 - px) * py * pz, kb = (1.0 - px) * (1.0 - py) * pz,
                   kc = px * (1.0 - py) * pz, kd = px * py * (1.0 - pz),
                   ke = (1.0 - px) * py * (1.0 - pz), kf = (1.0 - px) * (1.0 - py) * (1.0 - pz),
                   kg = px * (1.0 - py) * (1.0 - pz);
      const long long sy = d.N1, sz = d.N1 * d.N2;
      const long long g0 = d.g(ix, iy, iz);
      const double *e0 = Ei + 3 * g0, *e1 = Ei + 3 * (g0 + 1), *e2 = Ei + 3 * (g0 + 1 + sy),
                   *e3 = Ei + 3 * (g0 + sy), *e4 = Ei + 3 * (g0 + sz), *e5 = Ei + 3 * (g0 + 1 + sz),
                   *e6 = Ei + 3 * (g0 + 1 + sy + sz), *e7 = Ei + 3 * (g0 + sy + sz);
      double E[3];
#pragma unroll
      for (int a = 0; a < 3; ++a)
        E[a] = k0 * __ldg(e0 + a) + ka * __ldg(e1 + a) + kb * __ldg(e2 + a) + kc * __ldg(e3 + a) +
               kd * __ldg(e4 + a) + ke * __ldg(e5 + a) + kf * __ldg(e6 + a) + kg * __ldg(e7 + a);
      const double k1 = c.k1;
      double Bx = c.Bx, By = c.By, Bz = c.Bz;
      bool boris = c.boris;
      if (BMAP && boris) {
        const double kE[8] = {k0, ka, kb, kc, kd, ke, kf, kg};
        boris = bmap_gather_f64(m, xp, yp, zp, ix, iy, iz, kE, Bx, By, Bz);
      }
      if (boris) {
        double B_tot = sqrt(Bx * Bx + By * By + Bz * Bz);
        double kk = k1 * (2.0 / (1.0 + (k1 * B_tot) * (k1 * B_tot)));
        double v1x = vx + k1 * E[0], v1y = vy + k1 * E[1], v1z = vz + k1 * E[2];
        double v3x = v1x + k1 * (v1y * Bz - v1z * By);
        double v3y = v1y + k1 * (v1z * Bx - v1x * Bz);
        double v3z = v1z + k1 * (v1x * By - v1y * Bx);
        double v2x = v1x + kk * (v3y * Bz - v3z * By);
        double v2y = v1y + kk * (v3z * Bx - v3x * Bz);
        double v2z = v1z + kk * (v3x * By - v3y * Bx);
        vx = v2x + k1 * E[0];
        vy = v2y + k1 * E[1];
        vz = v2z + k1 * E[2];
      } else {
        vx = vx + 2.0 * k1 * E[0];
        vy = vy + 2.0 * k1 * E[1];
        vz = vz + 2.0 * k1 * E[2];
      }
      xp = xp + c.dt * vx;
      yp = yp + c.dt * vy;
      zp = zp + c.dt * vz;
      int jx = (int)floor(xp / c.h0) + 1, jy = (int)floor(yp / c.h1) + 1, jz = (int)floor(zp / c.h2) + 1;
      jx = jx < 0 ? 0 : (jx > d.n1 + 1 ? d.n1 + 1 : jx);
      jy = jy < 0 ? 0 : (jy > d.n2 + 1 ? d.n2 + 1 : jy);
      jz = jz < 0 ? 0 : (jz > d.n3 + 1 ? d.n3 + 1 : jz);
      if (cw[d.c(jx, jy, jz)]) {
        // lost at a wall (Src/part_expmover.f90:275-433)
        double Eki = 0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz);
        int igrid = bcnd[d.g(jx, jy, jz)];
        atomicAdd(&acc[0], Eki);
        if (igrid >= 0 && igrid <= c.ngrid) {
          atomicAdd(&acc[2 + 2 * igrid], 1.0);
          atomicAdd(&acc[3 + 2 * igrid], Eki);
          dielectric_charge(die, d, igrid, xp, yp, zp, jx, jy, jz, c.h0, c.h1, c.h2, c.flag_pbc, c.zmax);
        }
        hole = true;
      } else {
        if (c.flag_nmn == 1 && xp <= 0.0) {
          xp = -xp;
          vx = -vx;
        }
        if (c.flag_pbc == 1) {
          if (yp >= c.ymax) yp = yp - c.ymax;
          if (yp <= 0.0) yp = c.ymax + yp;
          if (zp >= c.zmax) zp = zp - c.zmax;
          if (zp <= 0.0) zp = c.zmax + zp;
        }
        p[i] = xp;
        p[cap + i] = yp;
        p[2 * cap + i] = zp;
        p[3 * cap + i] = vx;
        p[4 * cap + i] = vy;
        p[5 * cap + i] = vz;
        // ---- CIC weights of the new position (charge_deposition order)
        int dx = (int)(xp / c.h0) + 1, dy = (int)(yp / c.h1) + 1, dz = (int)(zp / c.h2) + 1;
        double qx = (dx * c.h0 - xp) / c.h0;
        double qy = (dy * c.h1 - yp) / c.h1;
        double qz = (dz * c.h2 - zp) / c.h2;
        const double k = c.kdep;
        w0 = k * qx * qy * qz;
        w1 = k * (1.0 - qx) * qy * qz;
        w2 = k * (1.0 - qx) * (1.0 - qy) * qz;
        w3 = k * qx * (1.0 - qy) * qz;
        w4 = k * qx * qy * (1.0 - qz);
        w5 = k * (1.0 - qx) * qy * (1.0 - qz);
        w6 = k * (1.0 - qx) * (1.0 - qy) * (1.0 - qz);
        w7 = k * qx * (1.0 - qy) * (1.0 - qz);
        q = d.g(dx, dy, dz);
      }
    }
    if (hole) flag[i] = 2;
  }
  // ---- hole list (warp-aggregated append)
  const int lane = threadIdx.x & 31;
  const unsigned hm = __ballot_sync(full, hole);
  if (hm) {
    const int leader = __ffs(hm) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(nholes, __popc(hm));
    base = __shfl_sync(full, base, leader);
    if (hole) holes[base + __popc(hm & lanemask_lt())] = (int)i;
  }
  // ---- group equal deposit cells: bitonic sort of (node, lane) across the
  // warp, each lane then takes the weights of its sorted source lane, so all
  // lanes depositing into one cell form one run of consecutive lanes
  long long sk = (q < 0) ? (long long)0x7fffffffffffffffLL : q;
  int sl = lane;
#pragma unroll
  for (int k = 2; k <= 32; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      const long long ok = __shfl_xor_sync(full, sk, j);
      const int ol = __shfl_xor_sync(full, sl, j);
      const bool up = ((lane & k) == 0);
      const bool lower = ((lane & j) == 0);
      const bool mine_first = (sk < ok) || (sk == ok && sl < ol);
      const bool keep = (lower == up) ? mine_first : !mine_first;
      if (!keep) {
        sk = ok;
        sl = ol;
      }
    }
  }
  w0 = __shfl_sync(full, w0, sl);
  w1 = __shfl_sync(full, w1, sl);
  w2 = __shfl_sync(full, w2, sl);
  w3 = __shfl_sync(full, w3, sl);
  w4 = __shfl_sync(full, w4, sl);
  w5 = __shfl_sync(full, w5, sl);
  w6 = __shfl_sync(full, w6, sl);
  w7 = __shfl_sync(full, w7, sl);
  q = (sk == (long long)0x7fffffffffffffffLL) ? -1 : sk;
  // ---- warp-segmented sum of the weights over runs of equal base node
  bool head;
  const int rid = run_id(q, head);
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int orid = __shfl_down_sync(full, rid, off);
    const bool same = (lane + off < 32) && (orid == rid);
    double t;
    t = __shfl_down_sync(full, w0, off); if (same) w0 += t;
    t = __shfl_down_sync(full, w1, off); if (same) w1 += t;
    t = __shfl_down_sync(full, w2, off); if (same) w2 += t;
    t = __shfl_down_sync(full, w3, off); if (same) w3 += t;
    t = __shfl_down_sync(full, w4, off); if (same) w4 += t;
    t = __shfl_down_sync(full, w5, off); if (same) w5 += t;
    t = __shfl_down_sync(full, w6, off); if (same) w6 += t;
    t = __shfl_down_sync(full, w7, off); if (same) w7 += t;
  }
  if (head && q >= 0) {
    const long long sy = d.N1, sz = d.N1 * d.N2;
    atomicAdd(&np[q], __ldg(&kq[q]) * w0);
    atomicAdd(&np[q + 1], __ldg(&kq[q + 1]) * w1);
    atomicAdd(&np[q + 1 + sy], __ldg(&kq[q + 1 + sy]) * w2);
    atomicAdd(&np[q + sy], __ldg(&kq[q + sy]) * w3);
    atomicAdd(&np[q + sz], __ldg(&kq[q + sz]) * w4);
    atomicAdd(&np[q + 1 + sz], __ldg(&kq[q + 1 + sz]) * w5);
    atomicAdd(&np[q + 1 + sy + sz], __ldg(&kq[q + 1 + sy + sz]) * w6);
    atomicAdd(&np[q + sy + sz], __ldg(&kq[q + sy + sz]) * w7);
  }
}

// Hole filling.  side[0] = number of holes L, side[1] = alive tail count,
// side[2] = holes below N - L, side[3] = N - L.
__global__ void k_fill_lists(const int *__restrict__ count, const int *__restrict__ holes,
                             const signed char *__restrict__ flag, int *side, int *tailA, int *holeH) {
  const int N = *count, L = side[0], Np = N - L;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < L; t += stride) {
    const int tail = Np + (int)t;
    if (flag[tail] != 2) tailA[atomicAdd(&side[1], 1)] = tail;
    const int h = holes[t];
    if (h < Np) holeH[atomicAdd(&side[2], 1)] = h;
  }
}

__global__ void k_fill_move(double *__restrict__ p, long long cap, const int *__restrict__ count,
                            signed char *__restrict__ flag, const int *side, const int *__restrict__ tailA,
                            const int *__restrict__ holeH) {
  const int N = *count, L = side[0], Np = N - L, na = side[1];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < na; t += stride) {
    const long long src = tailA[t], dst = holeH[t];
#pragma unroll
    for (int a = 0; a < 6; ++a) p[a * cap + dst] = p[a * cap + src];
    flag[dst] = 0;
  }
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < L; t += stride)
    flag[Np + t] = 0;
}

__global__ void k_fill_count(int *count, const int *side) { *count = *count - side[0]; }

}  // namespace

int launch_push_deposit(const lepic_grid_t &g, const double *Ei, lepic_species_f64_t &sp, int ptype,
                        int ngrid, const lepic_phys_t &P, double *np, double *acc_dev, int n_hint,
                        cudaStream_t s) {
  Dims d(g.n);
  const int p = ptype - 1;
  FusedConst c;
  memset(&c, 0, sizeof(c));
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  c.dt = P.dt;
  c.k1 = P.dt * P.charge[p] / (2.0 * P.mass[p]);
  c.Nm = P.Nm[p];
  c.mass = P.mass[p];
  c.kdep = P.Nm[p] / (g.h[0] * g.h[1] * g.h[2]);
  c.Bx = P.Bconst[0];
  c.By = P.Bconst[1];
  c.Bz = P.Bconst[2];
  c.boris = (P.flag_B == 1) ? 1 : 0;
  if (P.flag_B_pos == 1 && P.charge[p] > 0.0) c.boris = 0;
  c.flag_nmn = P.flag_nmn;
  c.flag_pbc = P.flag_pbc;
  c.ymax = P.ymax;
  c.zmax = P.zmax;
  c.ngrid = ngrid;
  if (!sp.flag_dead) return LEPIC_ERR_ARG;
  BMapF64 m;
  if (int rc = bmap_from_phys(P, g.n, m)) return rc;
  const Dielectric die = dielectric_from_phys(P, g.n, ptype);
  const size_t cap = (size_t)sp.cap;
  char nm[32];
  snprintf(nm, sizeof nm, "work_list%d", p);
  int *holes = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "fused_tail%d", p);
  int *tailA = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "fused_hh%d", p);
  int *holeH = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "fused_side%d", p);
  int *side = (int *)scratch(nm, sizeof(int) * 4);
  if (!holes || !tailA || !holeH || !side) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(side, 0, sizeof(int) * 4, s));
  const int nthreads = n_hint > 0 ? n_hint : sp.cap;
  int t0 = timer_start("push_deposit_f64", s);
  if (m.B)
    k_push_deposit_f64<true><<<grid_for(nthreads, FB), FB, 0, s>>>(d, c, m, die, Ei, g.bcnd, g.cell_wall, sp.p,
                                                                   sp.cap, sp.count, sp.flag_dead, g.kq, np,
                                                                   holes, side, acc_dev, ctx().d_err);
  else
    k_push_deposit_f64<false><<<grid_for(nthreads, FB), FB, 0, s>>>(d, c, m, die, Ei, g.bcnd, g.cell_wall, sp.p,
                                                                    sp.cap, sp.count, sp.flag_dead, g.kq, np,
                                                                    holes, side, acc_dev, ctx().d_err);
  timer_stop(t0, s);
  LEPIC_CUDA(cudaGetLastError());
  int t1 = timer_start("fill_holes", s);
  const int fb = ctx().sms * 2;
  k_fill_lists<<<fb, 256, 0, s>>>(sp.count, holes, sp.flag_dead, side, tailA, holeH);
  k_fill_move<<<fb, 256, 0, s>>>(sp.p, sp.cap, sp.count, sp.flag_dead, side, tailA, holeH);
  k_fill_count<<<1, 1, 0, s>>>(sp.count, side);
  timer_stop(t1, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

}  // namespace lepic

extern "C" int lepic_dev_push_deposit(const lepic_grid_t *g, const double *Ei, lepic_species_f64_t *s,
                                      int ptype, int ngrid, const lepic_phys_t *P, double *np,
                                      double *acc, int n_hint, void *stream) {
  if (!g || !s || !P || ptype < 1 || !acc) return LEPIC_ERR_ARG;
  return lepic::launch_push_deposit(*g, Ei, *s, ptype, ngrid, *P, np, acc, n_hint, (cudaStream_t)stream);
}
