// Maxwellian electron heating (Src/part_expmover.f90:484-568, eheating) and
// the heating-region statistics that set its temperature
// (Src/part_expmover.f90:658-681 in charge_deposition, Src/main.f90:1206-1227).
//
// Every electron whose cell index ix lies in [ixl_pow, ixr_pow] (and, with
// flag_circxh, inside or outside the circle of radius R_ahp about the box
// axis) is heated with probability nudt: it gets a new Maxwellian velocity of
// thermal speed vt (the load_gauss form vp = vt sqrt(-ln u1), angle 2 pi u2,
// the third component from a second pair).  The reference draws these from
// one serial ran2 stream; here each electron draws from Philox4x32-10 keyed by
// the seed with the counter (particle index, call), so the electrons are
// independent and the heated fraction and the heated velocity distribution
// are those of the reference.  P_loss(2) gains 0.5 Nm m (v^2 - v_old^2).
//
// With Pabs > 0 the temperature is self-consistent: Te = 2/3 (sum Ek +
// Pabs / nu_h) / (Nm qe Nh) over the electrons of the region, computed on the
// device from the statistics kernel's sums, so no host round trip is needed.
#include <cstring>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int HB = 256;

struct HeatC {
  int ixl, ixr, circ, ahp;
  double R2, nudt, ymax, zmax, h0, h1, h2;
  double vt;                 // thermal speed when no statistics are given
  double Nm, mass, qe, Pabs, nu_h;
  uint32_t k0, k1, call;
};

__device__ __forceinline__ bool in_region(const HeatC &c, int ix, double y, double z) {
  if (ix < c.ixl || ix > c.ixr) return false;
  if (c.circ == 1) {
    const double r2 = (y - c.ymax / 2.0) * (y - c.ymax / 2.0) + (z - c.zmax / 2.0) * (z - c.zmax / 2.0);
    if (c.ahp == 0 ? r2 > c.R2 : r2 < c.R2) return false;
  }
  return true;
}

// vt of this call: Src/main.f90:1224-1226 from the statistics stats[0] =
// sum Ek, stats[1] = Nh when given, else c.vt
__device__ __forceinline__ double heat_vt(const HeatC &c, const double *stats) {
  if (!stats || !(c.Pabs > 0.0) || stats[1] < 1.0) return c.vt;
  const double Te = (2.0 / 3.0) * (stats[0] + c.Pabs / c.nu_h) / (c.Nm * c.qe * stats[1]);
  return sqrt(2.0 * c.qe * Te / fabs(c.mass));
}

// a new Maxwellian velocity or false (not heated this call)
__device__ __forceinline__ bool heat_draw(const HeatC &c, long long i, double vt, double &vx, double &vy,
                                          double &vz) {
  const U4 r = philox4x32_10({(uint32_t)i, (uint32_t)(i >> 32), c.call, 0x48454154u}, c.k0, c.k1);
  if (!(u01(r.x) <= c.nudt)) return false;
  const U4 q = philox4x32_10({(uint32_t)i, (uint32_t)(i >> 32), c.call, 0x48454155u}, c.k0, c.k1);
  double s1, c1, s2, c2;
  sincos(2.0 * 3.141592653589793 * u01(q.y), &s1, &c1);
  sincos(2.0 * 3.141592653589793 * u01(q.w), &s2, &c2);
  const double vp = vt * sqrt(-log(u01(q.x)));
  const double vq = vt * sqrt(-log(u01(q.z)));
  vx = vp * c1;
  vy = vp * s1;
  vz = vq * c2;
  return true;
}

// block sums of (dE, heated) into acc[0..1]
__device__ __forceinline__ void add_block(double a, double b, double *acc) {
  __shared__ double sa[HB / 32], sb[HB / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xffffffffu, a, o);
    b += __shfl_xor_sync(0xffffffffu, b, o);
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  if (lane == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double ta = 0.0, tb = 0.0;
    for (int k = 0; k < HB / 32; ++k) {
      ta += sa[k];
      tb += sb[k];
    }
    if (ta != 0.0 || tb != 0.0) {
      atomicAdd(&acc[0], ta);
      atomicAdd(&acc[1], tb);
    }
  }
}

__global__ void __launch_bounds__(HB) k_eheating_f64(HeatC c, double *__restrict__ p, long long cap,
                                                     const int *__restrict__ count, const double *stats,
                                                     double *acc) {
  const long long N = *count;
  const double vt = heat_vt(c, stats);
  double dE = 0.0, nh = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const double x = p[i];
    if (!in_region(c, (int)(x / c.h0) + 1, p[cap + i], p[2 * cap + i])) continue;
    double vx, vy, vz;
    if (!heat_draw(c, i, vt, vx, vy, vz)) continue;
    const double ox = p[3 * cap + i], oy = p[4 * cap + i], oz = p[5 * cap + i];
    p[3 * cap + i] = vx;
    p[4 * cap + i] = vy;
    p[5 * cap + i] = vz;
    dE += 0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz - (ox * ox + oy * oy + oz * oz));
    nh += 1.0;
  }
  add_block(dE, nh, acc);
  if (blockIdx.x == 0 && threadIdx.x == 0) acc[2] = vt;
}

__global__ void __launch_bounds__(HB) k_eheating_mixed(HeatC c, const int *__restrict__ cell, float *__restrict__ p,
                                                       long long cap, const int *__restrict__ count,
                                                       const double *stats, double *acc) {
  const long long N = *count;
  const double vt = heat_vt(c, stats);
  double dE = 0.0, nh = 0.0;
  constexpr int CB = LEPIC_CELL_BITS, CM = LEPIC_CELL_MAX - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int cc = cell[i];
    const int ix = (cc & CM) + 1, iy = ((cc >> CB) & CM) + 1, iz = (cc >> (2 * CB)) + 1;
    const double y = ((double)(iy - 1) + p[cap + i]) * c.h1, z = ((double)(iz - 1) + p[2 * cap + i]) * c.h2;
    if (!in_region(c, ix, y, z)) continue;
    double vx, vy, vz;
    if (!heat_draw(c, i, vt, vx, vy, vz)) continue;
    const double ox = p[3 * cap + i], oy = p[4 * cap + i], oz = p[5 * cap + i];
    p[3 * cap + i] = (float)vx;
    p[4 * cap + i] = (float)vy;
    p[5 * cap + i] = (float)vz;
    const double nx = (float)vx, ny = (float)vy, nz = (float)vz;
    dE += 0.5 * c.Nm * c.mass * (nx * nx + ny * ny + nz * nz - (ox * ox + oy * oy + oz * oz));
    nh += 1.0;
  }
  add_block(dE, nh, acc);
  if (blockIdx.x == 0 && threadIdx.x == 0) acc[2] = vt;
}

// sum Ek and Nh of the electrons in the region into stats[0..1]
__global__ void __launch_bounds__(HB) k_heat_stats_f64(HeatC c, const double *__restrict__ p, long long cap,
                                                       const int *__restrict__ count, double *stats) {
  const long long N = *count;
  double s = 0.0, n = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    if (!in_region(c, (int)(p[i] / c.h0) + 1, p[cap + i], p[2 * cap + i])) continue;
    const double vx = p[3 * cap + i], vy = p[4 * cap + i], vz = p[5 * cap + i];
    s += 0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz);
    n += 1.0;
  }
  add_block(s, n, stats);
}

__global__ void __launch_bounds__(HB) k_heat_stats_mixed(HeatC c, const int *__restrict__ cell,
                                                         const float *__restrict__ p, long long cap,
                                                         const int *__restrict__ count, double *stats) {
  const long long N = *count;
  double s = 0.0, n = 0.0;
  constexpr int CB = LEPIC_CELL_BITS, CM = LEPIC_CELL_MAX - 1;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
    const int cc = cell[i];
    const int ix = (cc & CM) + 1, iy = ((cc >> CB) & CM) + 1, iz = (cc >> (2 * CB)) + 1;
    const double y = ((double)(iy - 1) + p[cap + i]) * c.h1, z = ((double)(iz - 1) + p[2 * cap + i]) * c.h2;
    if (!in_region(c, ix, y, z)) continue;
    const double vx = p[3 * cap + i], vy = p[4 * cap + i], vz = p[5 * cap + i];
    s += 0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz);
    n += 1.0;
  }
  add_block(s, n, stats);
}

HeatC make_heat(const lepic_grid_t &g, const lepic_phys_t &P, const lepic_heat_t &H, double vt,
                unsigned long long seed, unsigned long long call) {
  HeatC c;
  memset(&c, 0, sizeof(c));
  c.ixl = H.ixl_pow;
  c.ixr = H.ixr_pow;
  c.circ = H.flag_circxh;
  c.ahp = H.flag_ahp;
  c.R2 = H.R_ahp * H.R_ahp;
  c.nudt = H.nudt;
  c.ymax = P.ymax;
  c.zmax = P.zmax;
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  c.vt = vt;
  c.Nm = P.Nm[0];
  c.mass = P.mass[0];
  c.qe = P.qe;
  c.Pabs = H.Pabs;
  c.nu_h = H.nu_h;
  c.k0 = (uint32_t)(seed & 0xffffffffu);
  c.k1 = (uint32_t)(seed >> 32);
  c.call = (uint32_t)call;
  return c;
}

int heat_grid(long long cap) {
  long long b = (cap + HB - 1) / HB;
  const long long mx = (long long)ctx().sms * 8;
  if (b > mx) b = mx;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace

int launch_eheating(const lepic_grid_t &g, lepic_species_f64_t *e, lepic_species_mixed_t *m, const lepic_phys_t &P,
                    const lepic_heat_t &H, double vt, const double *stats, unsigned long long seed,
                    unsigned long long call, double *acc, cudaStream_t s) {
  const HeatC c = make_heat(g, P, H, vt, seed, call);
  int t = timer_start(e ? "eheating_f64" : "eheating_mixed", s);
  if (e)
    k_eheating_f64<<<heat_grid(e->cap), HB, 0, s>>>(c, e->p, e->cap, e->count, stats, acc);
  else
    k_eheating_mixed<<<heat_grid(m->cap), HB, 0, s>>>(c, m->cell, m->p, m->cap, m->count, stats, acc);
  timer_stop(t, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int launch_heat_stats(const lepic_grid_t &g, const lepic_species_f64_t *e, const lepic_species_mixed_t *m,
                      const lepic_phys_t &P, const lepic_heat_t &H, double *stats, cudaStream_t s) {
  const HeatC c = make_heat(g, P, H, 0.0, 0, 0);
  int t = timer_start(e ? "heat_stats_f64" : "heat_stats_mixed", s);
  if (e)
    k_heat_stats_f64<<<heat_grid(e->cap), HB, 0, s>>>(c, e->p, e->cap, e->count, stats);
  else
    k_heat_stats_mixed<<<heat_grid(m->cap), HB, 0, s>>>(c, m->cell, m->p, m->cap, m->count, stats);
  timer_stop(t, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

}  // namespace lepic

using lepic::Dims;

extern "C" {

int lepic_dev_eheating(const lepic_grid_t *g, lepic_species_f64_t *e, const lepic_phys_t *P,
                       const lepic_heat_t *H, double vt, const double *stats, unsigned long long seed,
                       unsigned long long call, double *acc, void *stream) {
  if (!g || !e || !P || !H || !acc || !(H->nudt >= 0.0)) return LEPIC_ERR_ARG;
  return lepic::launch_eheating(*g, e, nullptr, *P, *H, vt, stats, seed, call, acc, (cudaStream_t)stream);
}

int lepic_dev_eheating_mixed(const lepic_grid_t *g, lepic_species_mixed_t *e, const lepic_phys_t *P,
                             const lepic_heat_t *H, double vt, const double *stats, unsigned long long seed,
                             unsigned long long call, double *acc, void *stream) {
  if (!g || !e || !P || !H || !acc || !(H->nudt >= 0.0)) return LEPIC_ERR_ARG;
  return lepic::launch_eheating(*g, nullptr, e, *P, *H, vt, stats, seed, call, acc, (cudaStream_t)stream);
}

int lepic_dev_heat_stats(const lepic_grid_t *g, const lepic_species_f64_t *e, const lepic_phys_t *P,
                         const lepic_heat_t *H, double *stats, void *stream) {
  if (!g || !e || !P || !H || !stats) return LEPIC_ERR_ARG;
  return lepic::launch_heat_stats(*g, e, nullptr, *P, *H, stats, (cudaStream_t)stream);
}

int lepic_dev_heat_stats_mixed(const lepic_grid_t *g, const lepic_species_mixed_t *e, const lepic_phys_t *P,
                               const lepic_heat_t *H, double *stats, void *stream) {
  if (!g || !e || !P || !H || !stats) return LEPIC_ERR_ARG;
  return lepic::launch_heat_stats(*g, nullptr, e, *P, *H, stats, (cudaStream_t)stream);
}

}  // extern "C"
