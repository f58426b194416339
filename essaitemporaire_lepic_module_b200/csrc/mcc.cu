// Null-collision Monte Carlo against neutral targets (Src/collisions.f90).
//
// The reference draws Nc = N * nu_max * ns_coll * dt incident particles with
// replacement from a serial ran2 stream and tests each against
// sum_r nu_r / nu_max.  Here every particle draws its own Bernoulli trial
// with probability Pmax = nu_max * ns_coll * dt from a Philox4x32-10 counter
// keyed by (seed, call, species, particle, sub-stream): the expected number
// of collisions of each process, nu_r * ns_coll * dt per particle, is the
// same, and no two threads ever touch the same particle.  The physics of a
// selected collision follows Src/collisions.f90:437-998 step for step:
// Maxwellian neutral target (load_gauss form), relative energy in the
// centre-of-mass frame, linear interpolation of sigma on the merged energy
// grid, elastic / excitation scattering, ionization with equal-momentum
// byproducts on equally spaced angles rotated by `scatter`, and charge
// exchange by velocity swap.  Ionization products are appended at the end of
// their species' arrays (warp-aggregated atomic slot reservation).
#include <vector>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int MB = 256;
constexpr int MAXR = 8;   // reactions per incident species
constexpr int MAXBY = 4;  // byproducts per reaction

struct MCCConst {
  int ptype, nr;
  double Pmax, nu_max, qe, pi;
  double m_p;                   // |mass| of incident
  int ind[MAXR];                // 1-based reaction index
  int tt[MAXR];                 // target species (1-based)
  int rt[MAXR], n_by[MAXR], n_re[MAXR];
  int by[MAXR][MAXBY];
  int re[MAXR][2];
  double Eth[MAXR], np_t[MAXR];
  double mass[LEPIC_NPART];     // signed masses
  double vt0[LEPIC_NPART];
  int npt, npt_mx;
  unsigned int k0, k1, c2, c3;  // Philox key and counter words
  // region counters of Src/collisions.f90:1005-1013 (drop-in path only)
  int n_rg, ncol_mx, n1, n2;
  int ixl[LEPIC_NM_RG], ixr[LEPIC_NM_RG], iyl, iyr, izl, izr;
  double w_rg[LEPIC_NM_RG];     // 1 / np_tot_rg(ptype, i_rg)
  double h0, h1, h2;
};

// Src/collisions.f90:1022-1050
__device__ __forceinline__ void scatter(double &vx1, double &vy1, double &vz1, double vx, double vy,
                                        double vz, double costheta, double phi) {
  double sintheta = sqrt(fmax(1.0 - costheta * costheta, 0.0));
  double sinphi, cosphi;
  sincos(phi, &sinphi, &cosphi);
  double v = sqrt(vx * vx + vy * vy + vz * vz);
  if (v == 0.0) return;
  if (fabs(vy) > fabs(vz)) {
    double vv = sqrt(vx * vx + vy * vy);
    vx1 = vx * costheta + (vy * v * sinphi + vx * vz * cosphi) / vv * sintheta;
    vy1 = vy * costheta + (-vx * v * sinphi + vy * vz * cosphi) / vv * sintheta;
    vz1 = vz * costheta - vv * cosphi * sintheta;
  } else {
    double vv = sqrt(vx * vx + vz * vz);
    vx1 = vx * costheta + (vz * v * sinphi - vy * vx * cosphi) / vv * sintheta;
    vy1 = vy * costheta + vv * cosphi * sintheta;
    vz1 = vz * costheta - (vx * v * sinphi + vy * vz * cosphi) / vv * sintheta;
  }
}

// sigma(Ekr) on the merged grid: the unique interval Er[j-1] < E <= Er[j]
// (Src/collisions.f90:485-521); 0 when E <= Er[0].
__device__ __forceinline__ double sigma_at(const double *__restrict__ Er, const double *__restrict__ sig,
                                           int npt, double E, int &found) {
  found = 0;
  if (!(E > Er[0]) || E > Er[npt - 1]) return 0.0;
  int lo = 0, hi = npt - 1;  // Er[lo] < E <= Er[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (E > Er[mid]) lo = mid;
    else hi = mid;
  }
  found = 1;
  double EL = Er[lo], ER = Er[hi], sL = sig[lo], sR = sig[hi];
  return sL + (E - EL) * (sR - sL) / (ER - EL);
}

struct SpPtrs {
  double *p[LEPIC_NPART];
  int *count[LEPIC_NPART];
  int cap[LEPIC_NPART];
};

__global__ void __launch_bounds__(MB) k_mcc(MCCConst c, SpPtrs S, const double *__restrict__ Er,
                                            const double *__restrict__ sig, signed char *flag_dead,
                                            int *add, unsigned long long *counts, double *cnt_col,
                                            int *err) {
  const int P = c.ptype - 1;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int N = *S.count[P];
  int sel = -1;
  if (i < N) {
    U4 ctr = {(uint32_t)i, 0u, c.c2, c.c3};
    U4 r0 = philox4x32_10(ctr, c.k0, c.k1);
    if (u01(r0.x) < c.Pmax) {
      const long long cap = S.cap[P];
      double *pp = S.p[P];
      double vx0 = pp[3 * cap + i], vy0 = pp[4 * cap + i], vz0 = pp[5 * cap + i];
      ctr.y = 1u;
      U4 r1 = philox4x32_10(ctr, c.k0, c.k1);
      // one Maxwellian target per target species (Src/collisions.f90:437-449)
      double vr_t = 0, Ekr_t = 0, mu_t = 0, vxc = 0, vyc = 0, vzc = 0, tvx = 0, tvy = 0, tvz = 0;
      int cur_tt = -1;
      double nu[MAXR];
      double sum_nu = 0.0;
      for (int r = 0; r < c.nr; ++r) {
        int tt = c.tt[r];
        if (tt != cur_tt) {
          double vt = c.vt0[tt - 1];
          double vp = vt * sqrt(-log(u01(r1.x)));
          double s1, c1;
          sincos(2.0 * c.pi * u01(r1.y), &s1, &c1);
          tvx = vp * c1;
          tvy = vp * s1;
          double vp2 = vt * sqrt(-log(u01(r1.z)));
          tvz = vp2 * cos(2.0 * c.pi * u01(r1.w));
          double mt = fabs(c.mass[tt - 1]);
          mu_t = c.m_p * mt / (c.m_p + mt);
          vr_t = sqrt((vx0 - tvx) * (vx0 - tvx) + (vy0 - tvy) * (vy0 - tvy) + (vz0 - tvz) * (vz0 - tvz));
          Ekr_t = (0.5 * mu_t * (vr_t * vr_t)) / c.qe;
          double sm = c.m_p + mt;
          vxc = (c.m_p * vx0 + mt * tvx) / sm;
          vyc = (c.m_p * vy0 + mt * tvy) / sm;
          vzc = (c.m_p * vz0 + mt * tvz) / sm;
          if (Ekr_t > Er[c.npt - 1]) raise_err(err, LEPIC_ERR_EKR_TABLE, (int)i);
          cur_tt = tt;
        }
        int found;
        double sp = sigma_at(Er, sig + (long long)c.npt_mx * (c.ind[r] - 1), c.npt, Ekr_t, found);
        nu[r] = found ? c.np_t[r] * sp * vr_t / c.nu_max : 0.0;
        sum_nu += nu[r];
      }
      double u = u01(r0.y);
      if (u <= sum_nu) {
        double s = 0.0;
        for (int r = 0; r < c.nr; ++r) {
          s += nu[r];
          if (u <= s) {
            sel = r;
            break;
          }
        }
      }
      if (sel >= 0) {
        const int rt = c.rt[sel];
        if (rt == 4) {
          // charge exchange: the incident takes the target's velocity
          pp[3 * cap + i] = tvx;
          pp[4 * cap + i] = tvy;
          pp[5 * cap + i] = tvz;
        } else {
          double Ee = 0.5 * mu_t * (vr_t * vr_t) - c.Eth[sel] * c.qe;
          if (Ee < 0.0) {
            raise_err(err, LEPIC_ERR_NEG_ENERGY, (int)i);
            Ee = 0.0;
          }
          const int nby = c.n_by[sel];
          double sum_mass = 0.0;
          for (int a = 0; a < nby; ++a) sum_mass = sum_mass + 1.0 / fabs(c.mass[c.by[sel][a] - 1]);
          double th_add = 2.0 * c.pi / (double)nby;
          double cos_th = 1.0 - 2.0 * u01(r0.z);
          double th = acos(cos_th);
          double phi = 2.0 * c.pi * u01(r0.w);
          double sin_ph, cos_ph;
          sincos(phi, &sin_ph, &cos_ph);
          ctr.y = 2u;
          U4 r2 = philox4x32_10(ctr, c.k0, c.k1);
          double cos_th_s = 1.0 - 2.0 * u01(r2.x);
          double phi_s = 2.0 * c.pi * u01(r2.y);
          double xp = pp[i], yp = pp[cap + i], zp = pp[2 * cap + i];
          bool incident_reused = false;
          for (int a = 0; a < nby; ++a) {
            double sth, cth;
            sincos(th, &sth, &cth);
            th = th + th_add;
            double ex = cth, ey = sth * sin_ph, ez = sth * cos_ph;
            double ex1 = 0, ey1 = 0, ez1 = 0;
            scatter(ex1, ey1, ez1, ex, ey, ez, cos_th_s, phi_s);
            int bt = c.by[sel][a];
            if (c.mass[bt - 1] <= 0) continue;
            double mb = fabs(c.mass[bt - 1]);
            double vp = sqrt(2.0 * (Ee / sum_mass) / (mb * mb));
            double nvx = vxc + vp * ex1, nvy = vyc + vp * ey1, nvz = vzc + vp * ez1;
            bool reuse = (a == 0 && bt == c.ptype) || ((rt == 1 || rt == 3) && bt == c.ptype);
            if (reuse) {
              pp[3 * cap + i] = nvx;
              pp[4 * cap + i] = nvy;
              pp[5 * cap + i] = nvz;
              incident_reused = true;
            } else {
              const int B = bt - 1;
              int slot = atomicAdd(&add[B], 1);
              long long j = (long long)*S.count[B] + slot;
              if (j >= S.cap[B]) {
                raise_err(err, LEPIC_ERR_CAPACITY, B);
              } else {
                const long long cb = S.cap[B];
                double *qb = S.p[B];
                qb[j] = xp;
                qb[cb + j] = yp;
                qb[2 * cb + j] = zp;
                qb[3 * cb + j] = nvx;
                qb[4 * cb + j] = nvy;
                qb[5 * cb + j] = nvz;
              }
            }
          }
          if (!incident_reused && flag_dead) flag_dead[i] = 1;
        }
        if (cnt_col) {
          int ix = (int)(pp[i] / c.h0) + 1, iy = (int)(pp[cap + i] / c.h1) + 1,
              iz = (int)(pp[2 * cap + i] / c.h2) + 1;
          for (int g = 0; g < c.n_rg; ++g) {
            if (ix >= c.ixl[g] && ix <= c.ixr[g] && iy >= c.iyl && iy <= c.iyr && iz >= c.izl &&
                iz <= c.izr) {
              atomicAdd(&cnt_col[(c.ind[sel] - 1) + (long long)c.ncol_mx * g], c.w_rg[g]);
              break;
            }
          }
        }
      }
    }
  }
  // warp-aggregated collision counters
  const unsigned mask = __ballot_sync(0xffffffffu, sel >= 0);
  if (mask) {
    for (int r = 0; r < c.nr; ++r) {
      unsigned m = __ballot_sync(0xffffffffu, sel == r);
      if ((threadIdx.x & 31) == 0 && m) atomicAdd(&counts[c.ind[r] - 1], (unsigned long long)__popc(m));
    }
  }
}

__global__ void k_mcc_finalize(int *count0, int *count1, int *count2, const int *add, int ntype) {
  int *cs[3] = {count0, count1, count2};
  for (int p = 0; p < ntype && p < 3; ++p)
    if (cs[p]) *cs[p] += add[p];
}

}  // namespace

int launch_collisions(const lepic_grid_t &g, lepic_species_f64_t *sp, int ntype,
                      const lepic_tables_t &T, const lepic_phys_t &P, unsigned long long seed,
                      unsigned long long call_index, double *nu_max, long long *counts,
                      cudaStream_t s, const RegionCount *rg) {
  if (ntype > 3) return LEPIC_ERR_UNSUPPORTED;
  auto CI = [&](int icol, int info) { return T.col_info_h[(icol - 1) + (long long)T.ncol * (info - 1)]; };
  int *add = (int *)scratch("mcc_add", sizeof(int) * LEPIC_NPART);
  unsigned long long *cnt = (unsigned long long *)scratch("mcc_cnt", sizeof(unsigned long long) * 64);
  if (!add || !cnt || T.ncol > 64) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(add, 0, sizeof(int) * LEPIC_NPART, s));
  LEPIC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 64, s));
  SpPtrs S;
  memset(&S, 0, sizeof(S));
  for (int p = 0; p < ntype; ++p) {
    S.p[p] = sp[p].p;
    S.count[p] = sp[p].count;
    S.cap[p] = sp[p].cap;
  }
  std::vector<double> Eth(T.ncol > 0 ? T.ncol : 1, 0.0);
  if (T.ncol > 0)
    LEPIC_CUDA(cudaMemcpyAsync(Eth.data(), T.sig_Eth, sizeof(double) * T.ncol, cudaMemcpyDeviceToHost, s));
  std::vector<int> Nh(ntype, 0);
  for (int p = 0; p < ntype; ++p) {
    LEPIC_CUDA(cudaMemcpyAsync(&Nh[p], sp[p].count, sizeof(int), cudaMemcpyDeviceToHost, s));
  }
  LEPIC_CUDA(cudaStreamSynchronize(s));
  for (int p = 1; p <= ntype; ++p) {
    nu_max[p - 1] = 0.0;
    int pn = T.p_ncol[p - 1];
    if (pn == 0 || P.mass[p - 1] <= 0) continue;
    if (pn > MAXR) return LEPIC_ERR_UNSUPPORTED;
    MCCConst c;
    memset(&c, 0, sizeof(c));
    c.ptype = p;
    c.nr = pn;
    c.qe = P.qe;
    c.pi = P.pi;
    c.m_p = fabs(P.mass[p - 1]);
    for (int q = 0; q < LEPIC_NPART; ++q) {
      c.mass[q] = P.mass[q];
      c.vt0[q] = P.vt0[q];
    }
    double num = 0.0;
    for (int r = 0; r < pn; ++r) {
      int ind = T.sig_list[(p - 1) + LEPIC_NPART * r];
      int n_re = CI(ind, 1), n_by = CI(ind, 2);
      if (n_by > MAXBY || n_re > 2) return LEPIC_ERR_UNSUPPORTED;
      int tt = CI(ind, 2 + n_re);
      if (P.charge[tt - 1] != 0.0) return LEPIC_ERR_UNSUPPORTED;  // DSMC targets
      c.ind[r] = ind;
      c.tt[r] = tt;
      c.n_re[r] = n_re;
      c.n_by[r] = n_by;
      for (int a = 0; a < n_re; ++a) c.re[r][a] = CI(ind, 3 + a);
      for (int a = 0; a < n_by; ++a) c.by[r][a] = CI(ind, 3 + n_re + a);
      c.rt[r] = CI(ind, 3 + n_re + n_by);
      c.Eth[r] = Eth[ind - 1];
      c.np_t[r] = P.np_mx[tt - 1];
      num = num + P.np_mx[tt - 1] * T.sigv_mx[(p - 1) + LEPIC_NPART * (ind - 1)];
    }
    nu_max[p - 1] = num < P.nu_uplim[p - 1] ? num : P.nu_uplim[p - 1];
    double Pmax = nu_max[p - 1] * (double)(float)P.ns_coll * P.dt;
    if (Pmax > 1.0) return LEPIC_ERR_PMAX;
    if (Nh[p - 1] == 0 || nu_max[p - 1] <= 0.0) continue;
    c.Pmax = Pmax;
    c.nu_max = nu_max[p - 1];
    c.npt = T.npt;
    c.npt_mx = T.npt_mx;
    c.k0 = (unsigned)(seed & 0xffffffffu);
    c.k1 = (unsigned)(seed >> 32);
    c.c2 = (unsigned)(call_index & 0xffffffffu);
    c.c3 = (unsigned)((call_index >> 32) << 8) | (unsigned)p;
    c.h0 = g.h[0];
    c.h1 = g.h[1];
    c.h2 = g.h[2];
    double *cc = nullptr;
    if (rg && rg->cnt_col_dev) {
      c.n_rg = rg->n_rg;
      c.ncol_mx = rg->ncol_mx;
      for (int q = 0; q < LEPIC_NM_RG; ++q) {
        c.ixl[q] = rg->ixl[q];
        c.ixr[q] = rg->ixr[q];
        c.w_rg[q] = rg->w[p - 1][q];
      }
      c.iyl = rg->iyl;
      c.iyr = rg->iyr;
      c.izl = rg->izl;
      c.izr = rg->izr;
      cc = rg->cnt_col_dev;
    }
    int tm = timer_start("mcc_f64", s);
    k_mcc<<<grid_for(Nh[p - 1], MB), MB, 0, s>>>(c, S, T.sig_Er, T.sig, sp[p - 1].flag_dead, add, cnt,
                                                  cc, ctx().d_err);
    timer_stop(tm, s);
    LEPIC_CUDA(cudaGetLastError());
  }
  k_mcc_finalize<<<1, 1, 0, s>>>(sp[0].count, ntype > 1 ? sp[1].count : nullptr,
                                 ntype > 2 ? sp[2].count : nullptr, add, ntype);
  LEPIC_CUDA(cudaGetLastError());
  unsigned long long hc[64];
  LEPIC_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
  int rc = check_err(s);
  if (counts)
    for (int q = 0; q < T.ncol; ++q) counts[q] += (long long)hc[q];
  return rc;
}

}  // namespace lepic
