// Internal declarations of the sm_100a PIC-MCC library.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/lepic_gpu.h"

namespace lepic {

// Node-grid indexing of the reference arrays g(0:n1+2,0:n2+2,0:n3+2)
// (column-major) and rhs arrays b(0:n1+1,0:n2+1,0:n3+1).
struct Dims {
  int n1, n2, n3;
  long long N1, N2, N3;
  __host__ __device__ Dims() : n1(0), n2(0), n3(0), N1(3), N2(3), N3(3) {}
  __host__ __device__ Dims(int a, int b, int c) : n1(a), n2(b), n3(c), N1(a + 3), N2(b + 3), N3(c + 3) {}
  __host__ __device__ explicit Dims(const int *n) : Dims(n[0], n[1], n[2]) {}
  __host__ __device__ long long g(int ix, int iy, int iz) const { return ix + N1 * (iy + N2 * (long long)iz); }
  __host__ __device__ long long cnt() const { return N1 * N2 * N3; }
  __host__ __device__ long long r(int ix, int iy, int iz) const {
    return ix + (N1 - 1) * (iy + (N2 - 1) * (long long)iz);
  }
  __host__ __device__ long long rcnt() const { return (N1 - 1) * (N2 - 1) * (N3 - 1); }
  // cells with ix in 0..n1+1 (the clamped range of the loss test)
  __host__ __device__ long long c(int ix, int iy, int iz) const {
    return ix + (N1 - 1) * (iy + (N2 - 1) * (long long)iz);
  }
};

// Device error word: [0] = first status code, [1] = detail (index / value).
__device__ __forceinline__ void raise_err(int *err, int code, int info) {
  if (atomicCAS(err, 0, code) == 0) err[1] = info;
}

// Per-device library context: error word, SM count, cached scratch.
struct Ctx {
  int device = -1;
  int sms = 0;
  int *d_err = nullptr;       // device int[2]
  int *h_err = nullptr;       // pinned host int[2]
  cudaDeviceProp prop{};
};
Ctx &ctx();                                     // context of the current device
void *scratch(const char *name, size_t bytes);  // cached device buffer (grows)
int check_err(cudaStream_t s);                  // sync, read + clear device error word
int timer_start(const char *name, cudaStream_t s);  // -1 when timing is off
void timer_stop(int id, cudaStream_t s);
int cuda_status(cudaError_t e, const char *what);

inline int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > 2147483647LL) g = 2147483647LL;
  return (int)g;
}

// ---------------------------------------------------------------- Philox
// Philox4x32-10 counter-based generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11): ten rounds of the
// 32x32->64 multiply-xor round function with the published multipliers and
// Weyl key increments.
struct U4 { uint32_t x, y, z, w; };
__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    uint64_t p0 = (uint64_t)M0 * c.x, p1 = (uint64_t)M1 * c.z;
    uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}
// uniform in (0,1) from 32 random bits
__host__ __device__ __forceinline__ double u01(uint32_t v) { return ((double)v + 0.5) * 2.3283064365386963e-10; }

// ------------------------------------------------------------ B-field map
// The push's B-field map (Src/part_expmover.f90:148-203):
// Bi(4, 0:nB1+2, 0:nB2+2, 0:nB3+2), component fastest, Bi(4,...) = |B|.
struct BMapF64 {
  const double *B;        // nullptr: uniform field
  int own;                // 1: own grid (flag_gridB = 1): index and weights from h_B
  int nb1, nb2, nb3;      // n_B
  long long N1, N2;       // nB1 + 3, nB2 + 3
  double h0, h1, h2;      // h_B
};

// validated map of P for a push on the node grid n; LEPIC_OK also when P has
// no map (m.B = nullptr)
inline int bmap_from_phys(const lepic_phys_t &P, const int n[3], BMapF64 &m) {
  m = BMapF64{};
  if (P.flag_B != 1 || !P.Bmap) return LEPIC_OK;
  if (P.n_B[0] < 2 || P.n_B[1] < 1 || P.n_B[2] < 1) return LEPIC_ERR_ARG;
  m.B = P.Bmap;
  m.nb1 = P.n_B[0];
  m.nb2 = P.n_B[1];
  m.nb3 = P.n_B[2];
  m.N1 = m.nb1 + 3;
  m.N2 = m.nb2 + 3;
  m.own = (m.nb1 != n[0] || m.nb2 != n[1] || m.nb3 != n[2]) ? 1 : 0;
  m.h0 = P.h_B[0];
  m.h1 = P.h_B[1];
  m.h2 = P.h_B[2];
  if (m.own && !(m.h0 > 0.0 && m.h1 > 0.0 && m.h2 > 0.0)) return LEPIC_ERR_ARG;
  return LEPIC_OK;
}

// B at a particle at (xp, yp, zp) whose E gather used cell (ix, iy, iz) and
// weights k[0..7], in the reference's expression order (FP64 files are built
// without FMA contraction, so this reproduces the oracle bit for bit).
// Returns false when |B| at the left map node is not above 1e-5 T: the
// particle then takes the leapfrog step.  On its own grid the map index is
// clamped to 0..nB+1, which only changes particles outside the box.
__device__ __forceinline__ bool bmap_gather_f64(const BMapF64 &m, double xp, double yp, double zp, int ix,
                                                int iy, int iz, const double (&kE)[8], double &Bx, double &By,
                                                double &Bz) {
  double k[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) k[a] = kE[a];
  if (m.own) {
    ix = (int)(xp / m.h0) + 1;
    iy = (int)(yp / m.h1) + 1;
    iz = (int)(zp / m.h2) + 1;
    ix = ix < 0 ? 0 : (ix > m.nb1 + 1 ? m.nb1 + 1 : ix);
    iy = iy < 0 ? 0 : (iy > m.nb2 + 1 ? m.nb2 + 1 : iy);
    iz = iz < 0 ? 0 : (iz > m.nb3 + 1 ? m.nb3 + 1 : iz);
  }
  const long long q = ix + m.N1 * (iy + m.N2 * (long long)iz);
  if (!(__ldg(m.B + 4 * q + 3) > 1.e-5)) return false;
  if (m.own) {
    const double px = (ix * m.h0 - xp) / m.h0;
    const double py = (iy * m.h1 - yp) / m.h1;
    const double pz = (iz * m.h2 - zp) / m.h2;
    k[0] = px * py * pz;
    k[1] = (1.0 - px) * py * pz;
    k[2] = (1.0 - px) * (1.0 - py) * pz;
    k[3] = px * (1.0 - py) * pz;
    k[4] = px * py * (1.0 - pz);
    k[5] = (1.0 - px) * py * (1.0 - pz);
    k[6] = (1.0 - px) * (1.0 - py) * (1.0 - pz);
    k[7] = px * (1.0 - py) * (1.0 - pz);
  }
  const long long sy = m.N1, sz = m.N1 * m.N2;
  const long long o[8] = {0, 1, 1 + sy, sy, sz, 1 + sz, 1 + sy + sz, sy + sz};
  double B[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double s = k[0] * __ldg(m.B + 4 * (q + o[0]) + a);
#pragma unroll
    for (int c = 1; c < 8; ++c) s = s + k[c] * __ldg(m.B + 4 * (q + o[c]) + a);
    B[a] = s;
  }
  Bx = B[0];
  By = B[1];
  Bz = B[2];
  return true;
}

// Dielectric walls (Src/part_expmover.f90:302-348): the charge of a particle
// lost on a wall whose type dtype(igrid) is 2 (Y = const plane) or 3, 4
// (X = const planes #1, #2) is spread bilinearly on that plane's node sums.
struct Dielectric {
  const int *dtype;   // device dtype(0:ngrid), nullptr: no dielectric walls
  double *qxz;        // sum_q_xz(0:n1+2, 0:n3+2) of the species pushed
  double *qyz;        // sum_q_yz(2, 0:n2+2, 0:n3+2) of the species pushed
  double k3;          // Nm charge
};

// The walls of P (device API) for species ptype; die.dtype stays nullptr
// when P has none.
inline Dielectric dielectric_from_phys(const lepic_phys_t &P, const int n[3], int ptype) {
  Dielectric die{};
  if (P.dtype && P.sum_q_xz && P.sum_q_yz) {
    const int p = ptype - 1;
    die.dtype = P.dtype;
    die.qxz = P.sum_q_xz + (size_t)p * (n[0] + 3) * (n[2] + 3);
    die.qyz = P.sum_q_yz + (size_t)p * 2 * (n[1] + 3) * (n[2] + 3);
    die.k3 = P.Nm[p] * P.charge[p];
  }
  return die;
}

// A particle lost at the new position (xp, yp, zp) in cell (ix, iy, iz)
// (clamped to 0..n+1) on wall label igrid: its charge on the wall's plane
// sums when the wall is a dielectric.  pbc: periodic planes along z (the
// position wraps first).
__device__ __forceinline__ void dielectric_charge(const Dielectric &die, const Dims &d, int igrid, double xp,
                                                  double yp, double zp, int ix, int iy, int iz, double h0,
                                                  double h1, double h2, int pbc, double zmax) {
  const int dt = die.dtype ? die.dtype[igrid] : 0;
  if (dt <= 1) return;
  double zq = zp;
  int iq = iz;
  if (pbc == 1) {
    if (zq >= zmax) {
      zq = zq - zmax;
      iq = (int)floor(zq / h2) + 1;
    }
    if (zq <= 0.0) {
      zq = zmax + zq;
      iq = (int)floor(zq / h2) + 1;
    }
  }
  iq = iq < 0 ? 0 : (iq > d.n3 + 1 ? d.n3 + 1 : iq);
  const double pz = (iq * h2 - zq) / h2;
  if (dt == 2) {
    const double px = (ix * h0 - xp) / h0;
    double *q = die.qxz;
    const long long NX = d.N1;
    atomicAdd(&q[ix + NX * iq], die.k3 * px * pz);
    atomicAdd(&q[ix + 1 + NX * iq], die.k3 * (1.0 - px) * pz);
    atomicAdd(&q[ix + 1 + NX * (iq + 1)], die.k3 * (1.0 - px) * (1.0 - pz));
    atomicAdd(&q[ix + NX * (iq + 1)], die.k3 * px * (1.0 - pz));
  } else if (dt == 3 || dt == 4) {
    const double py = (iy * h1 - yp) / h1;
    double *q = die.qyz + (dt - 3);
    const long long NY = d.N2;
    atomicAdd(&q[2 * (iy + NY * iq)], die.k3 * py * pz);
    atomicAdd(&q[2 * (iy + 1 + NY * iq)], die.k3 * (1.0 - py) * pz);
    atomicAdd(&q[2 * (iy + 1 + NY * (iq + 1))], die.k3 * (1.0 - py) * (1.0 - pz));
    atomicAdd(&q[2 * (iy + NY * (iq + 1))], die.k3 * py * (1.0 - pz));
  }
}

// ------------------------------------------------------------ launchers
// fields.cu
// Src/main.f90:859-949 for one rank: the dielectric walls' potential update
// from the summed surface charges of every species, then the sums cleared
int launch_dielectric_phi(const Dims &d, double *phi, const int *bcnd, const lepic_phys_t &P, int ngrid,
                          double Ca, cudaStream_t s);
int launch_calc_rho(const Dims &d, double *np, double *rhs, const int *bcnd, int ntype,
                    const lepic_phys_t &P, cudaStream_t s);
int launch_dens_red(const Dims &d, const double *np, double *np_red, const int *bcnd, int ntype,
                    double *np_mx_host, cudaStream_t s);
int launch_efield(const Dims &d, const double h[3], const double *phi, double *Ei, const int *bcnd,
                  cudaStream_t s);
int launch_cell_wall(const Dims &d, const int *bcnd, unsigned char *cw, cudaStream_t s);
// mg.cu
// pbc: periodic planes in y and z (bcnd 0); nmn: Neumann plane at x = 0 (bcnd -2)
int launch_pdesolver(const Dims &d, const double h[3], double *u, const double *b, const int *bcnd,
                     int ncycl, double eps, double omega, int ng, double eps0, int *k, double *ktot,
                     double *res, cudaStream_t s, int pbc = 0, int nmn = 0);
// particles.cu
// The drop-in mover's negative-ion bookkeeping (species tag_neg: flag_cex in
// slot order in cex, compacted into cex_out; device counters cnt_cex[3],
// cnt_dead, beam_div[4] accumulated) and secondary emission (gam_sec > 0, a
// positive species: electrons appended to species e1, *ploss4 accumulated,
// Philox key key0/key1/call).  Src/part_expmover.f90:76, 278-301, 353-470.
struct MoverExtras {
  int tag_neg, tag_neu, num_grd;
  const int *cex;
  int *cex_out;
  int *cnt_cex;
  double *cnt_dead;
  double *beam_div;
  double gam_sec, THm, zg_sec[2];
  int igrid_sec;
  lepic_species_f64_t *e1;
  double *ploss4;
  uint32_t key0, key1, call;
};
// dtype_dev (device dtype(0:ngrid)) with qxz_dev / qyz_dev (device planes of
// the species pushed): the charge of particles lost on dielectric walls
// (without them, the walls of P, if any)
int launch_part_mover(const lepic_grid_t &g, const double *Ei, lepic_species_f64_t &sp, int ptype,
                      int ntype, int ngrid, const lepic_phys_t &P, double *p_mac, double *P_loss,
                      cudaStream_t s, const int *dtype_dev = nullptr, double *qxz_dev = nullptr,
                      double *qyz_dev = nullptr, const MoverExtras *ex = nullptr);
int launch_deposit(const lepic_grid_t &g, const lepic_species_f64_t &sp, int ptype,
                   const lepic_phys_t &P, double *np, cudaStream_t s);
int launch_sort(const lepic_grid_t &g, lepic_species_f64_t &sp, int *Plist, int pl_max,
                cudaStream_t s);
int launch_load_uniform(const lepic_grid_t &g, lepic_species_f64_t *sp, int ntype, long long n,
                        const lepic_phys_t &P, unsigned long long seed, cudaStream_t s);
int exclusive_scan_i32(const int *in, int *out, long long n, cudaStream_t s);
// mcc.cu
// Region counters of the drop-in path (Src/collisions.f90:1005-1013):
// cnt_col(c, 1, i_rg) += 1/np_tot_rg(ptype, i_rg) for the first region that
// contains the incident particle's cell.
// The same path's per-collision bookkeeping (Src/collisions.f90:862-869,
// 894-902, 982-990): ploss3_dev (device double[LEPIC_NPART]) += the kinetic
// energy change of every particle a collision sets, P_loss(3, btype);
// sour_xy_dev / sour_xz_dev (device int planes (0:n1+2, 0:n2+2, ntype) /
// (0:n1+2, 0:n3+2, ntype)) += 1 per particle created in the incident's cell
// when its iz is iz_pl / its iy is iy_pl.  nullptr: not kept.
struct RegionCount {
  double *cnt_col_dev;          // device (ncol_mx, n_rg) slice for iproc = 1
  int n_rg, ncol_mx;
  int ixl[LEPIC_NM_RG], ixr[LEPIC_NM_RG], iyl, iyr, izl, izr;
  double w[LEPIC_NPART][LEPIC_NM_RG];
  double *ploss3_dev;
  int *sour_xy_dev, *sour_xz_dev;
  int iz_pl, iy_pl;
};
// tg: charged-target (DSMC) inputs and outputs, nullptr when the tables have none
int launch_collisions(const lepic_grid_t &g, lepic_species_f64_t *sp, int ntype,
                      const lepic_tables_t &T, const lepic_phys_t &P, unsigned long long seed,
                      unsigned long long call_index, double *nu_max, long long *counts,
                      cudaStream_t s, const RegionCount *rg = nullptr, lepic_targets_t *tg = nullptr);
int launch_collisions_mixed(const lepic_grid_t &g, lepic_species_mixed_t *sp, int ntype,
                            const lepic_tables_t &T, const lepic_phys_t &P, unsigned long long seed,
                            unsigned long long call_index, double *nu_max, long long *counts,
                            cudaStream_t s, lepic_targets_t *tg = nullptr);
// mixed.cu
int launch_push_deposit_mixed(const lepic_grid_t &g, const float *E32, lepic_species_mixed_t &sp,
                              int ptype, int ngrid, const lepic_phys_t &P, double *np, double *acc,
                              int n_hint, cudaStream_t s);
int launch_sort_mixed(const lepic_grid_t &g, lepic_species_mixed_t &sp, int n_hint, cudaStream_t s);
// mgmixed.cu
int launch_pdesolver_mixed(const Dims &d, const double h[3], double *u, const double *b, const int *bcnd,
                           double eps, double omega, int ng, double eps0, int max_refine, int nu_fine_pre,
                           int nu_fine_post, int nu_pre, int nu_post, int coarse_sweeps, int *iters,
                           double *res_out, cudaStream_t s);

// heating.cu (e or m: the electrons in one of the two layouts)
int launch_eheating(const lepic_grid_t &g, lepic_species_f64_t *e, lepic_species_mixed_t *m, const lepic_phys_t &P,
                    const lepic_heat_t &H, double vt, const double *stats, unsigned long long seed,
                    unsigned long long call, double *acc, cudaStream_t s);
int launch_heat_stats(const lepic_grid_t &g, const lepic_species_f64_t *e, const lepic_species_mixed_t *m,
                      const lepic_phys_t &P, const lepic_heat_t &H, double *stats, cudaStream_t s);

// injection.cu (e64 or m: the species in one of the two layouts)
int launch_inject(const lepic_grid_t &g, lepic_species_f64_t *e64, lepic_species_mixed_t *m, int ntype,
                  const lepic_phys_t &P, const lepic_inject_t &I, long long n_events, unsigned long long seed,
                  unsigned long long call, double *const *np, const double *phi, double *P_loss4,
                  long long *injected, cudaStream_t s);

// residency.cu: device mirrors of the drop-ins' host arrays
bool residency_on();
// device pointer for host range [h, h + bytes) inside its mirror (created and
// filled from the host on first use); `write` marks the mirror device-newer
void *mirror_array(const void *h, size_t bytes, bool write, cudaStream_t s, int *rc);
unsigned long long mirror_generation(const void *h);  // changes on every host reload
int mirror_to_host(const void *h, size_t bytes, cudaStream_t s);
// particle slice vxp(6, 1:nmax) with np_h particles on the host side
int mirror_species(double *vxp_h, int np_h, int nmax, signed char *fd_h, cudaStream_t s,
                   lepic_species_f64_t *out);
int mirror_species_done(double *vxp_h, const lepic_species_f64_t &sp, bool wrote, bool fd_wrote,
                        int *np_out, cudaStream_t s);
// counted host<->device copies of the drop-in layer
int mirror_h2d(void *d, const void *h, size_t bytes, cudaStream_t s);
int mirror_d2h(void *h, const void *d, size_t bytes, cudaStream_t s);
int aos_to_soa(const double *aos, double *soa, long long first, long long n, long long cap, cudaStream_t s);
int soa_to_aos(const double *soa, double *aos, long long n, long long cap, cudaStream_t s);

// Integer CIC weights of the mixed-precision deposit (the step loop's tiled
// push and the FP32 collisional window): 2^QBITS units per particle.
constexpr int QBITS = 20;                  // 2^20 weight units per particle
constexpr double QI = 1.0 / 1048576.0;

// x rounded to the nearest integer for 0 <= x <= 2^22, by the FP32 addition
// of 1.5 * 2^23 (whose unit in the last place is 1) and integer arithmetic
// (weights are at most 2^QBITS <= 2^22)
__device__ __forceinline__ int round_q(float x) { return __float_as_int(x + 12582912.f) - 0x4B400000; }

// integer CIC weights of offsets (gx, gy, gz) in units of 2^-20 summing to
// exactly 2^20 (node order of Src/part_expmover.f90:591-656: (0,0,0),
// (1,0,0), (1,1,0), (0,1,0), then the same at z+1): seven rounded, the
// eighth the remainder.  The remainder may be a few units below zero for a
// particle next to the opposite corner (the seven rounding errors are at
// most 0.5 units each), and no weight is above 2^20.
constexpr int QNEG = 5;                    // a weight is above -QNEG units
__device__ __forceinline__ void qweights(float gx, float gy, float gz, int w[8]) {
  const float S = (float)(1 << QBITS);
  const float qx = 1.f - gx, qy = 1.f - gy, qz = 1.f - gz;
  const float a = qy * qz * S, b = gy * qz * S, e = qy * gz * S, f = gy * gz * S;
  w[0] = round_q(qx * a);
  w[1] = round_q(gx * a);
  w[2] = round_q(gx * b);
  w[3] = round_q(qx * b);
  w[4] = round_q(qx * e);
  w[5] = round_q(gx * e);
  w[6] = round_q(gx * f);
  w[7] = (1 << QBITS) - (w[0] + w[1] + w[2] + w[3] + w[4] + w[5] + w[6]);
}

// A node's 32-bit sum over a window of at most n particles lies in
// [-QNEG n, 2^20 n]; read back modulo 2^32 (the two ends must stay apart:
// qsum_window_ok)
constexpr bool qsum_window_ok(long long n) { return n * ((1LL << QBITS) + 2 * QNEG) < (1LL << 32); }
__device__ __forceinline__ double qsum_value(unsigned v, long long n) {
  return v <= (unsigned)(n * ((1LL << QBITS) + QNEG)) ? (double)v : (double)v - 4294967296.0;
}

__device__ __forceinline__ unsigned run_lanemask_le() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

// Sum of v over each run of consecutive lanes with the same key: afterwards
// the first lane of a run (head) holds the run's totals.  Lanes with key -1
// contribute zeros.  All 32 lanes must call this.  Particles sorted by cell
// give a warp few runs, so the atomics that follow are one per run instead
// of one per particle (lanes adding to one shared word are serialised).
template <int NV, class T = double>
__device__ __forceinline__ bool warp_run_sum(long long key, T (&v)[NV]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long prev = __shfl_up_sync(full, key, 1);
  const bool head = (lane == 0) || prev != key;
  const unsigned heads = __ballot_sync(full, head);
  const int rid = __popc(heads & run_lanemask_le());
  const unsigned above = heads & ~(0xffffffffu >> (31 - lane));
  const int len = head ? ((above ? __ffs(above) - 1 : 32) - lane) : 0;
  const int maxlen = (int)__reduce_max_sync(full, (unsigned)len);
  for (int o = 1; o < maxlen; o <<= 1) {
    const int orid = __shfl_down_sync(full, rid, o);
    const bool same = (lane + o < 32) && orid == rid;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      const T t = __shfl_down_sync(full, v[c], o);
      if (same) v[c] += t;
    }
  }
  return head && key >= 0;
}

// ------------------------------------------------ async copies and mbarriers
__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ unsigned long long gtime() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ bool mbar_try(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}

// a float4 from shared memory at 32-bit shared address a (a box staged
// before a barrier and not written afterwards)
__device__ __forceinline__ float4 lds4(uint32_t a) {
  float4 v;
  asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];" : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w) : "r"(a));
  return v;
}

// per-thread asynchronous copies global -> shared (16 bytes: both 16-byte
// aligned; 4 bytes: both 4-byte aligned), completed by cp.async.wait_group
__device__ __forceinline__ void cp_async16(void *dst, const void *src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(dst)), "l"(src) : "memory");
}

// wait for phase `parity` of the mbarrier, at most limit_ns of %globaltimer
__device__ inline bool mbar_wait_ns(uint32_t bar, uint32_t parity, unsigned long long limit_ns) {
  if (mbar_try(bar, parity)) return true;
  const unsigned long long t0 = gtime();
  while (!mbar_try(bar, parity))
    if (gtime() - t0 > limit_ns) return false;
  return true;
}

// the library's waits on copies: at most one second
__device__ inline bool mbar_wait(uint32_t bar, uint32_t parity) { return mbar_wait_ns(bar, parity, 1000000000ull); }

}  // namespace lepic


#define LEPIC_CUDA(call)                                                 \
  do {                                                                   \
    cudaError_t e__ = (call);                                            \
    if (e__ != cudaSuccess) return ::lepic::cuda_status(e__, #call);     \
  } while (0)
