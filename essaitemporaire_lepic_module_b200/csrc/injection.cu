// Particle injection (Src/part_injection.f90): electron-ion pairs at a fixed
// current or replacing the ions lost to the walls, an electron beam, or
// electron emission off a cathode.
//
// The reference draws every injection event from one serial ran2 stream.
// Here one thread handles one event with Philox4x32-10 draws keyed by the
// seed, counter (event, try, call): the position (uniform in the injection
// box, or the cosine / flat-top profile of opt_inj < 0; a disk of radius
// min(dx, dy)/2 for the beam and the cathode; redrawn while the cell has only
// wall nodes, at most MAX_TRIES times), then for every species a Bernoulli
// trial with probability ni0 and a velocity (Maxwellian of vt0; the shifted
// Maxwellian flux of the beam; the half-Maxwellian flux of the cathode, the
// position spread over the distance travelled in ns_inj dt).  The particles
// are appended behind each species' count.  P_loss(4) gains their kinetic
// energy (and for the beam Nm q phi at the particle).  For the step loop,
// whose push and deposition run fused before the injection, the kernel also
// deposits the new particles (CIC with kq, the weights of
// Src/part_expmover.f90:591-656); the drop-in leaves that to
// charge_deposition like the reference.
#include <cstring>
#include <vector>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int IB = 128;
constexpr int MAX_TRIES = 64;

struct InjC {
  int opt, ntype, n_cath, tag_beam, pbc, pbcz, dir0, mixed;
  double xl, xr, yl, yr, zl, zr, xm, ym, zm, dx, dy, dz, Rb, zmax, pi;
  double vb, vt_e, fmax, ns_dt;
  double zg[2];
  double ni0[LEPIC_NPART], vt0[LEPIC_NPART], Nm[LEPIC_NPART], mass[LEPIC_NPART], charge[LEPIC_NPART],
      kdep[LEPIC_NPART];
  double h0, h1, h2;
  Dims d;
  uint32_t k0, k1, call;
};

// the particle arrays of both layouts
struct InjDst {
  double *p64[LEPIC_NPART];
  int *cell[LEPIC_NPART];
  float *p32[LEPIC_NPART];
  int *count[LEPIC_NPART];
  long long cap[LEPIC_NPART];
  double *np[LEPIC_NPART];      // density grids to deposit into, or nullptr
};

__device__ __forceinline__ double uni(const U4 &r, int k) { return u01((&r.x)[k]); }

// the load_gauss pair (Src/load_part.f90:268-291)
__device__ __forceinline__ void gauss2(double vt, double u1, double u2, double pi, double &a, double &b) {
  const double vp = vt * sqrt(-log(u1));
  double s, c;
  sincos(2.0 * pi * u2, &s, &c);
  a = vp * c;
  b = vp * s;
}

__global__ void __launch_bounds__(IB) k_inject(InjC c, InjDst D, long long nev, const unsigned char *__restrict__ cw,
                                               const double *__restrict__ kq, const double *__restrict__ phi,
                                               int *add, double *acc, int *err) {
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (e >= nev) return;
  const int beam = (c.opt == 3 || c.opt == -3 || c.opt == 4 || c.opt == -4);
  double x = 0, y = 0, z = 0;
  bool ok = false;
  for (int t = 0; t < MAX_TRIES && !ok; ++t) {
    const U4 r = philox4x32_10({(uint32_t)e, (uint32_t)(e >> 32), (uint32_t)t, c.call}, c.k0, c.k1);
    const double u1 = uni(r, 0), u2 = uni(r, 1), u3 = uni(r, 2);
    if (c.opt > 0) {
      x = -u1 * c.dx + c.xr;
      y = -u2 * c.dy + c.yr;
      z = -u3 * c.dz + c.zr;
    } else {
      // cosine profile S0 cos(pi (x-xm)/dx) ... (Src/part_injection.f90:80-95)
      x = c.xm + (c.dx / c.pi) * asin(2.0 * u1 - 1.0);
      y = (c.pbc == 0 || c.pbcz == 1) ? c.ym + (c.dy / c.pi) * asin(2.0 * u2 - 1.0) : -u2 * c.dy + c.yr;
      z = c.pbc == 0 ? c.zm + (c.zmax / c.pi) * asin(2.0 * u3 - 1.0) : -u3 * c.dz + c.zr;
    }
    if (beam && (x - c.xm) * (x - c.xm) + (y - c.ym) * (y - c.ym) > c.Rb * c.Rb) continue;
    const int ix = (int)floor(x / c.h0) + 1, iy = (int)floor(y / c.h1) + 1, iz = (int)floor(z / c.h2) + 1;
    if (ix < 0 || ix > c.d.n1 + 1 || iy < 0 || iy > c.d.n2 + 1 || iz < 0 || iz > c.d.n3 + 1) continue;
    if (cw[c.d.c(ix, iy, iz)]) continue;   // only wall nodes (Src/part_injection.f90:104-108)
    ok = true;
  }
  if (!ok) {
    raise_err(err, LEPIC_ERR_ARG, (int)e);
    return;
  }
  for (int p = 0; p < c.ntype; ++p) {
    if (beam && (c.tag_beam == 0 ? p >= 1 : p != c.tag_beam - 1)) continue;
    const U4 r = philox4x32_10({(uint32_t)e, (uint32_t)(e >> 32), 0x100u + (uint32_t)p, c.call}, c.k0, c.k1);
    if (uni(r, 0) > c.ni0[p]) continue;   // Src/part_injection.f90:142-143
    double vx, vy, vz, zp = z;
    if (beam) {
      // the emissive plane: with two cathodes the events alternate
      const int ng = (c.n_cath == 2 && (c.opt == 4 || c.opt == -4)) ? (int)(e & 1) : (c.dir0 < 0 ? 1 : 0);
      const int dir = (c.n_cath == 2 && (c.opt == 4 || c.opt == -4)) ? (ng == 0 ? 1 : -1) : c.dir0;
      bool in = false;
      vx = vy = vz = 0.0;
      for (int t = 0; t < MAX_TRIES && !in; ++t) {
        const U4 q = philox4x32_10({(uint32_t)e, (uint32_t)(e >> 32), 0x200u + (uint32_t)t, c.call}, c.k0, c.k1);
        if (c.opt == 3 || c.opt == -3) {
          // shifted Maxwellian flux by acceptance / rejection (Src/part_injection.f90:247-293)
          const double vt = c.vt0[p];
          const double vm = fmax(0.0, c.vb - 4.0 * vt), vp = c.vb + 4.0 * vt;
          const double v = vm + uni(q, 0) * (vp - vm);
          const double f = v * exp(-(v - c.vb) * (v - c.vb) / (vt * vt));
          if (uni(q, 1) > f / c.fmax) continue;
          vz = v;
          const U4 g = philox4x32_10({(uint32_t)e, (uint32_t)(e >> 32), 0x300u + (uint32_t)t, c.call}, c.k0, c.k1);
          gauss2(vt, uni(g, 0), uni(g, 1), c.pi, vx, vy);
          zp = c.zg[ng] + vz * (uni(g, 2) * c.ns_dt);
        } else {
          // half-Maxwellian flux off the cathode (Src/part_injection.f90:177-185)
          vz = (double)dir * c.vb * sqrt(-log(uni(q, 0)));
          gauss2(c.vb, uni(q, 1), uni(q, 2), c.pi, vx, vy);
          zp = c.zg[ng] + vz * (uni(q, 3) * c.ns_dt);
        }
        in = !(zp < 0.0 || zp > c.zmax);
      }
      if (!in) continue;
    } else {
      const U4 g = philox4x32_10({(uint32_t)e, (uint32_t)(e >> 32), 0x400u + (uint32_t)p, c.call}, c.k0, c.k1);
      double tmp;
      gauss2(c.vt0[p], uni(g, 0), uni(g, 1), c.pi, vx, vy);
      gauss2(c.vt0[p], uni(g, 2), uni(g, 3), c.pi, vz, tmp);
    }
    const int slot = atomicAdd(&add[p], 1);
    const long long j = (long long)*D.count[p] + slot;
    if (j >= D.cap[p]) {
      raise_err(err, LEPIC_ERR_CAPACITY, p);
      continue;
    }
    const int ix = (int)floor(x / c.h0) + 1, iy = (int)floor(y / c.h1) + 1, iz = (int)floor(zp / c.h2) + 1;
    if (!c.mixed) {
      double *q = D.p64[p];
      const long long cp = D.cap[p];
      q[j] = x;
      q[cp + j] = y;
      q[2 * cp + j] = zp;
      q[3 * cp + j] = vx;
      q[4 * cp + j] = vy;
      q[5 * cp + j] = vz;
    } else {
      float *q = D.p32[p];
      const long long cp = D.cap[p];
      int jx = (int)(x / c.h0) + 1, jy = (int)(y / c.h1) + 1, jz = (int)(zp / c.h2) + 1;
      jx = jx < 1 ? 1 : (jx > c.d.n1 ? c.d.n1 : jx);
      jy = jy < 1 ? 1 : (jy > c.d.n2 ? c.d.n2 : jy);
      jz = jz < 1 ? 1 : (jz > c.d.n3 ? c.d.n3 : jz);
      D.cell[p][j] = (jx - 1) | (jy - 1) << LEPIC_CELL_BITS | (jz - 1) << (2 * LEPIC_CELL_BITS);
      q[j] = fminf(fmaxf((float)(x / c.h0 - (jx - 1)), 0.f), 0.99999994f);
      q[cp + j] = fminf(fmaxf((float)(y / c.h1 - (jy - 1)), 0.f), 0.99999994f);
      q[2 * cp + j] = fminf(fmaxf((float)(zp / c.h2 - (jz - 1)), 0.f), 0.99999994f);
      q[3 * cp + j] = (float)vx;
      q[4 * cp + j] = (float)vy;
      q[5 * cp + j] = (float)vz;
    }
    // injected power P_loss(4) (Src/part_injection.f90:219-245)
    double Ek = 0.5 * c.Nm[p] * c.mass[p] * (vx * vx + vy * vy + vz * vz);
    const int kx = (int)(x / c.h0) + 1, ky = (int)(y / c.h1) + 1, kz = (int)(zp / c.h2) + 1;
    const double px = (kx * c.h0 - x) / c.h0, py = (ky * c.h1 - y) / c.h1, pz = (kz * c.h2 - zp) / c.h2;
    const double w[8] = {px * py * pz,
                         (1.0 - px) * py * pz,
                         (1.0 - px) * (1.0 - py) * pz,
                         px * (1.0 - py) * pz,
                         px * py * (1.0 - pz),
                         (1.0 - px) * py * (1.0 - pz),
                         (1.0 - px) * (1.0 - py) * (1.0 - pz),
                         px * (1.0 - py) * (1.0 - pz)};
    const long long sy = c.d.N1, sz = c.d.N1 * c.d.N2, g0 = c.d.g(kx, ky, kz);
    const long long o[8] = {0, 1, 1 + sy, sy, sz, 1 + sz, 1 + sy + sz, sy + sz};
    if ((c.opt == 3 || c.opt == -3) && phi) {
      double ph = 0.0;
      for (int a = 0; a < 8; ++a) ph += w[a] * phi[g0 + o[a]];
      Ek += c.Nm[p] * c.charge[p] * ph;
    }
    atomicAdd(&acc[p], Ek);
    (void)ix;
    (void)iy;
    (void)iz;
    if (D.np[p])
      for (int a = 0; a < 8; ++a) atomicAdd(&D.np[p][g0 + o[a]], kq[g0 + o[a]] * (c.kdep[p] * w[a]));
  }
}

struct InjCounts {
  int *count[LEPIC_NPART];
  long long cap[LEPIC_NPART];
};

__global__ void k_inject_finalize(InjCounts C, const int *add, int ntype) {
  for (int p = 0; p < ntype; ++p) {
    const long long v = (long long)*C.count[p] + add[p];
    *C.count[p] = (int)(v < C.cap[p] ? v : C.cap[p]);
  }
}

}  // namespace

// n_events < 0: the events of the current, I_inj ns_inj dt / (qe Nm(1)),
// rounded stochastically (Src/part_injection.f90:58-65) with a Philox draw
int launch_inject(const lepic_grid_t &g, lepic_species_f64_t *e64, lepic_species_mixed_t *m, int ntype,
                  const lepic_phys_t &P, const lepic_inject_t &I, long long n_events, unsigned long long seed,
                  unsigned long long call, double *const *np, const double *phi, double *P_loss4,
                  long long *injected, cudaStream_t s) {
  if (ntype < 1 || ntype > LEPIC_NPART || !g.cell_wall) return LEPIC_ERR_ARG;
  if (n_events < 0) {
    const double dN = I.I_inj * I.ns_inj * P.dt / (P.qe * P.Nm[0]);
    n_events = (long long)dN;
    const U4 r = philox4x32_10({(uint32_t)call, (uint32_t)(call >> 32), 0x494E4Au, 0u},
                               (uint32_t)(seed & 0xffffffffu), (uint32_t)(seed >> 32));
    if (u01(r.x) <= dN - (double)n_events) n_events += 1;
  }
  InjC c;
  memset(&c, 0, sizeof(c));
  c.opt = I.opt_inj;
  c.ntype = ntype;
  c.n_cath = I.n_cath;
  c.tag_beam = I.tag_beam;
  c.pbc = P.flag_pbc;
  c.pbcz = I.flag_pbcz;
  c.dir0 = I.dir_sec < 0 ? -1 : 1;
  c.mixed = m ? 1 : 0;
  c.xl = I.xl;
  c.xr = I.xr;
  c.yl = I.yl;
  c.yr = I.yr;
  c.zl = I.zl;
  c.zr = I.zr;
  c.xm = (I.xl + I.xr) / 2.0;
  c.dx = I.xr - I.xl;
  c.ym = (I.yl + I.yr) / 2.0;
  c.dy = I.yr - I.yl;
  c.zm = (I.zl + I.zr) / 2.0;
  c.dz = I.zr - I.zl;
  c.Rb = (c.dx < c.dy ? c.dx : c.dy) / 2.0;
  c.zmax = P.zmax;
  c.pi = P.pi;
  c.zg[0] = I.zg_sec[0];
  c.zg[1] = I.zg_sec[1];
  c.ns_dt = (double)I.ns_inj * P.dt;
  c.vt_e = P.vt0[0];
  if (I.opt_inj == 3 || I.opt_inj == -3 || I.opt_inj == 4 || I.opt_inj == -4) {
    // Src/part_injection.f90:47-53
    c.vb = sqrt(2.0 * P.qe * I.THm / fabs(P.mass[0]));
    const double vmax = (c.vb + sqrt(c.vb * c.vb + 2.0 * c.vt_e * c.vt_e)) / 2.0;
    c.fmax = vmax * exp(-(vmax - c.vb) * (vmax - c.vb) / (c.vt_e * c.vt_e));
  }
  for (int p = 0; p < LEPIC_NPART; ++p) {
    c.ni0[p] = I.ni0[p];
    c.vt0[p] = P.vt0[p];
    c.Nm[p] = P.Nm[p];
    c.mass[p] = P.mass[p];
    c.charge[p] = P.charge[p];
    c.kdep[p] = P.Nm[p] / (g.h[0] * g.h[1] * g.h[2]);
  }
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  c.d = Dims(g.n);
  c.k0 = (uint32_t)(seed & 0xffffffffu);
  c.k1 = (uint32_t)(seed >> 32);
  c.call = (uint32_t)call;
  InjDst D;
  memset(&D, 0, sizeof(D));
  InjCounts fc;
  memset(&fc, 0, sizeof(fc));
  for (int p = 0; p < ntype; ++p) {
    if (m) {
      D.cell[p] = m[p].cell;
      D.p32[p] = m[p].p;
      D.count[p] = m[p].count;
      D.cap[p] = m[p].cap;
    } else {
      D.p64[p] = e64[p].p;
      D.count[p] = e64[p].count;
      D.cap[p] = e64[p].cap;
    }
    D.np[p] = np ? np[p] : nullptr;
    fc.count[p] = D.count[p];
    fc.cap[p] = D.cap[p];
  }
  int *add = (int *)scratch("inj_add", sizeof(int) * LEPIC_NPART);
  double *acc = (double *)scratch("inj_acc", sizeof(double) * LEPIC_NPART);
  if (!add || !acc) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(add, 0, sizeof(int) * LEPIC_NPART, s));
  LEPIC_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * LEPIC_NPART, s));
  int t = timer_start(m ? "inject_mixed" : "inject_f64", s);
  if (n_events > 0)
    k_inject<<<grid_for(n_events, IB), IB, 0, s>>>(c, D, n_events, g.cell_wall, g.kq, phi, add, acc, ctx().d_err);
  k_inject_finalize<<<1, 1, 0, s>>>(fc, add, ntype);
  timer_stop(t, s);
  LEPIC_CUDA(cudaGetLastError());
  int ha[LEPIC_NPART];
  double hacc[LEPIC_NPART];
  LEPIC_CUDA(cudaMemcpyAsync(ha, add, sizeof(ha), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(hacc, acc, sizeof(hacc), cudaMemcpyDeviceToHost, s));
  const int rc = check_err(s);
  for (int p = 0; p < ntype; ++p) {
    if (P_loss4) P_loss4[p] += hacc[p];
    if (injected) injected[p] += ha[p];
  }
  return rc;
}

}  // namespace lepic

extern "C" {

int lepic_dev_inject(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype, const lepic_phys_t *P,
                     const lepic_inject_t *I, long long n_events, unsigned long long seed, unsigned long long call,
                     double *const *np, const double *phi, double *P_loss4, long long *injected, void *stream) {
  if (!g || !sp || !P || !I) return LEPIC_ERR_ARG;
  return lepic::launch_inject(*g, sp, nullptr, ntype, *P, *I, n_events, seed, call, np, phi, P_loss4, injected,
                              (cudaStream_t)stream);
}

int lepic_dev_inject_mixed(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype, const lepic_phys_t *P,
                           const lepic_inject_t *I, long long n_events, unsigned long long seed,
                           unsigned long long call, double *const *np, const double *phi, double *P_loss4,
                           long long *injected, void *stream) {
  if (!g || !sp || !P || !I) return LEPIC_ERR_ARG;
  return lepic::launch_inject(*g, nullptr, sp, ntype, *P, *I, n_events, seed, call, np, phi, P_loss4, injected,
                              (cudaStream_t)stream);
}

}  // extern "C"
