// Discrete adjoint of the collisionless FP64 timestep over a K-step window
// (no counterpart in the reference; the forward operations it transposes are
// Src/part_expmover.f90:89-246 (gather, Boris, leapfrog),
// Src/part_expmover.f90:591-656 (CIC deposition), Src/calc_rho.f90:73-90
// (rhs = -sum q np), Src/pdesolver.f90 (A phi = rhs on plasma nodes with the
// wall potentials as Dirichlet values) and Src/Efield.f90 (E = -grad phi
// with wall extrapolation)).
//
// Inside the window particles keep their slots: a particle that reaches a
// wall is marked not alive and is neither pushed nor deposited again (wall
// losses are events; the adjoint does not differentiate through them).
//
// Step n maps (x^n, v^{n-1/2}) to (x^{n+1}, v^{n+1/2}):
//   np^n = deposit(x^n), rhs^n = -q np^n, A phi^n = rhs^n (walls at V),
//   E^n = G phi^n, v^{n+1/2} = Boris(v^{n-1/2}, gather(E^n, x^n), B),
//   x^{n+1} = x^n + dt v^{n+1/2}.
// Its adjoint, given (lx, lv) of the outputs:
//   lv += dt lx;  Boris^T gives lv^{n-1/2}, the adjoint of the gathered
//   field lEp and the B_z derivative;  lE^n = gather^T(lEp) (the deposit
//   pattern);  lphi = G^T lE^n;  A mu = lphi on plasma nodes (A is symmetric:
//   the same multigrid solves it);  dJ/dV_label += lphi(walls of the label)
//   - sum of the stencil couplings of mu into those walls;  lnp = -q mu;
//   lx += deposit^T(lnp) (the gather pattern with weight gradients) plus
//   the gather-weight gradient of the field term.
#include <cstring>

#include <type_traits>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int AB = 256;
constexpr int MAX_LABEL = 16;

struct WinConst {
  double h0, h1, h2, dt, k1, kk, Bx, By, Bz, kdep, q, mass;
  double dkk;       // d kk / d Bz
  double Nm;        // macroparticle weight
  int boris;
};

// left-node weight factors of coordinate x in cell ix (Src/part_expmover.f90:89-99)
struct Cic {
  long long g0;
  double px, py, pz;
};

__device__ __forceinline__ bool cic(const Dims &d, const WinConst &c, double xp, double yp, double zp, Cic &w) {
  if (!(xp >= 0.0 && yp >= 0.0 && zp >= 0.0)) return false;
  const int ix = (int)(xp / c.h0) + 1, iy = (int)(yp / c.h1) + 1, iz = (int)(zp / c.h2) + 1;
  if (ix > d.n1 || iy > d.n2 || iz > d.n3) return false;
  w.px = (ix * c.h0 - xp) / c.h0;
  w.py = (iy * c.h1 - yp) / c.h1;
  w.pz = (iz * c.h2 - zp) / c.h2;
  w.g0 = d.g(ix, iy, iz);
  return true;
}

// the 8 nodes in the order of Src/part_expmover.f90:100-108: (0,0,0),
// (1,0,0), (1,1,0), (0,1,0), (0,0,1), (1,0,1), (1,1,1), (0,1,1)
__device__ __forceinline__ int ox(int c) { return (c == 1 || c == 2 || c == 5 || c == 6) ? 1 : 0; }
__device__ __forceinline__ int oy(int c) { return (c == 2 || c == 3 || c == 6 || c == 7) ? 1 : 0; }
__device__ __forceinline__ int oz(int c) { return c >= 4 ? 1 : 0; }

__device__ __forceinline__ long long node(const Dims &d, const Cic &w, int c) {
  return w.g0 + ox(c) + d.N1 * (oy(c) + d.N2 * (long long)oz(c));
}
__device__ __forceinline__ double weight(const Cic &w, int c) {
  return (ox(c) ? 1.0 - w.px : w.px) * (oy(c) ? 1.0 - w.py : w.py) * (oz(c) ? 1.0 - w.pz : w.pz);
}
// d weight / d (x, y, z)
__device__ __forceinline__ void dweight(const WinConst &k, const Cic &w, int c, double &gx, double &gy, double &gz) {
  const double fx = ox(c) ? 1.0 - w.px : w.px, fy = oy(c) ? 1.0 - w.py : w.py, fz = oz(c) ? 1.0 - w.pz : w.pz;
  const double sx = ox(c) ? 1.0 / k.h0 : -1.0 / k.h0, sy = oy(c) ? 1.0 / k.h1 : -1.0 / k.h1,
               sz = oz(c) ? 1.0 / k.h2 : -1.0 / k.h2;
  gx = sx * fy * fz;
  gy = fx * sy * fz;
  gz = fx * fy * sz;
}

// warp_run_sum (the shared header): the window's particles are sorted by
// cell, so a warp holds few runs and adds one word per run.

// Reduce-scatter of NV <= 32 values over the 32 lanes (a butterfly in which
// each lane sends the half of its values it does not keep): afterwards lane L
// < NV holds the warp's total of value L.  31 shuffles for 24 values instead
// of 24 per halving step.
template <int NV>
__device__ __forceinline__ float warp_transpose_sum(const float (&v)[NV]) {
  static_assert(NV <= 32, "one value per lane at most");
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  float a[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) a[q] = q < NV ? v[q] : 0.f;
#pragma unroll
  for (int m = 32; m > 1; m >>= 1) {
    const int h = m >> 1;          // values kept; lane bit h selects the upper half
    const bool up = (lane & h) != 0;
#pragma unroll
    for (int q = 0; q < h; ++q) {
      if (q >= NV) continue;   // padding in both halves on every lane (lane 0's indices are 0..m-1)
      const float send = up ? a[q] : a[q + h];
      const float keep = up ? a[q + h] : a[q];
      a[q] = keep + __shfl_xor_sync(full, send, h);
    }
  }
  return a[0];
}

// The warp's per-key sums of v scattered through add(key, slot, q, total) for
// every key >= 0 and value q: one call per key and value.  slot is the
// caller's per-lane handle of its key's cell (equal on lanes of equal key).
// For more than 16 values a warp with one or two keys (particles sorted by
// cell: ions, electrons soon after the sort) sums by warp_transpose_sum, the
// totals landing on NV lanes that add at once (24 values: 5 % faster push
// adjoint; 8 values: the run sums are cheaper), and a warp with more keys
// sorts them first; otherwise warp_run_sum, one lane per run adding.  All 32
// lanes must call this; lanes with key -1 contribute nothing.
template <int NV, class F>
__device__ __forceinline__ void warp_scatter_sum(long long key, int slot, float (&v)[NV], F add) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned act = __ballot_sync(full, key >= 0);
  if (!act) return;
  const int l0 = __ffs(act) - 1, l1 = 31 - __clz(act);
  const long long k0 = __shfl_sync(full, key, l0), k1 = __shfl_sync(full, key, l1);
  const int s0 = __shfl_sync(full, slot, l0), s1 = __shfl_sync(full, slot, l1);
  if (NV > 16 && __all_sync(full, key < 0 || key == k0 || key == k1)) {
#pragma unroll 1
    for (int t = 0; t < (k1 == k0 ? 1 : 2); ++t) {
      const long long kt = t ? k1 : k0;
      float m[NV];
#pragma unroll
      for (int q = 0; q < NV; ++q) m[q] = key == kt ? v[q] : 0.f;
      const float tot = warp_transpose_sum<NV>(m);
      if (lane < NV) add(kt, t ? s1 : s0, lane, tot);
    }
    return;
  }
  if (NV > 16) {
    // more cells: a bitonic sort of (key, lane) makes each cell one run
    // before the run sums (7 % faster push adjoint than the unsorted runs,
    // in which one cell can recur and its head lanes contend)
    long long sk = key < 0 ? (long long)0x7fffffffffffffffLL : key;
    int sl = lane;
#pragma unroll
    for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
      for (int jj = kk >> 1; jj > 0; jj >>= 1) {
        const long long ok = __shfl_xor_sync(full, sk, jj);
        const int ol = __shfl_xor_sync(full, sl, jj);
        const bool up = (lane & kk) == 0, lower = (lane & jj) == 0;
        const bool mine_first = sk < ok || (sk == ok && sl < ol);
        if ((lower == up) ? !mine_first : mine_first) {
          sk = ok;
          sl = ol;
        }
      }
    }
#pragma unroll
    for (int c = 0; c < NV; ++c) v[c] = __shfl_sync(full, v[c], sl);
    const int sslot = __shfl_sync(full, slot, sl);
    const long long skey = sk == (long long)0x7fffffffffffffffLL ? -1 : sk;
    if (warp_run_sum<NV, float>(skey, v)) {
#pragma unroll
      for (int q = 0; q < NV; ++q) add(skey, sslot, q, v[q]);
    }
    return;
  }
  if (warp_run_sum<NV, float>(key, v)) {
#pragma unroll
    for (int q = 0; q < NV; ++q) add(key, slot, q, v[q]);
  }
}

__device__ __forceinline__ void cross(double ax, double ay, double az, double bx, double by, double bz, double &rx,
                                      double &ry, double &rz) {
  rx = ay * bz - az * by;
  ry = az * bx - ax * bz;
  rz = ax * by - ay * bx;
}

// forward push of the window (no compaction): alive particles only
__global__ void __launch_bounds__(AB) k_win_push(Dims d, WinConst c, const double *__restrict__ Ei,
                                                 const unsigned char *__restrict__ cw, double *__restrict__ p,
                                                 long long cap, int n, signed char *__restrict__ alive) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || !alive[i]) return;
  double xp = p[i], yp = p[cap + i], zp = p[2 * cap + i];
  double vx = p[3 * cap + i], vy = p[4 * cap + i], vz = p[5 * cap + i];
  Cic w;
  if (!cic(d, c, xp, yp, zp, w)) {
    alive[i] = 0;
    return;
  }
  double E[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double wq = weight(w, q);
    const double *e = Ei + 3 * node(d, w, q);
    E[0] += wq * e[0];
    E[1] += wq * e[1];
    E[2] += wq * e[2];
  }
  if (c.boris) {
    const double v1x = vx + c.k1 * E[0], v1y = vy + c.k1 * E[1], v1z = vz + c.k1 * E[2];
    double tx, ty, tz;
    cross(v1x, v1y, v1z, c.Bx, c.By, c.Bz, tx, ty, tz);
    const double v3x = v1x + c.k1 * tx, v3y = v1y + c.k1 * ty, v3z = v1z + c.k1 * tz;
    cross(v3x, v3y, v3z, c.Bx, c.By, c.Bz, tx, ty, tz);
    vx = v1x + c.kk * tx + c.k1 * E[0];
    vy = v1y + c.kk * ty + c.k1 * E[1];
    vz = v1z + c.kk * tz + c.k1 * E[2];
  } else {
    vx = vx + 2.0 * c.k1 * E[0];
    vy = vy + 2.0 * c.k1 * E[1];
    vz = vz + 2.0 * c.k1 * E[2];
  }
  xp = xp + c.dt * vx;
  yp = yp + c.dt * vy;
  zp = zp + c.dt * vz;
  int jx = (int)floor(xp / c.h0) + 1, jy = (int)floor(yp / c.h1) + 1, jz = (int)floor(zp / c.h2) + 1;
  jx = jx < 0 ? 0 : (jx > d.n1 + 1 ? d.n1 + 1 : jx);
  jy = jy < 0 ? 0 : (jy > d.n2 + 1 ? d.n2 + 1 : jy);
  jz = jz < 0 ? 0 : (jz > d.n3 + 1 ? d.n3 + 1 : jz);
  p[i] = xp;
  p[cap + i] = yp;
  p[2 * cap + i] = zp;
  p[3 * cap + i] = vx;
  p[4 * cap + i] = vy;
  p[5 * cap + i] = vz;
  if (cw[d.c(jx, jy, jz)]) alive[i] = 0;  // lost at a wall (Src/part_expmover.f90:258-262)
}

// CIC deposition of the alive particles (kq applied per node)
__global__ void __launch_bounds__(AB) k_win_deposit(Dims d, WinConst c, const double *__restrict__ p,
                                                    long long cap, int n, const signed char *__restrict__ alive,
                                                    const double *__restrict__ kq, double *__restrict__ np,
                                                    int *err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  Cic w;
  long long key = -1;
  double v[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = 0.0;
  if (i < n && alive[i]) {
    if (cic(d, c, p[i], p[cap + i], p[2 * cap + i], w)) {
      key = w.g0;
#pragma unroll
      for (int q = 0; q < 8; ++q) v[q] = weight(w, q);
    } else {
      raise_err(err, LEPIC_ERR_CELL, (int)i);
    }
  }
  if (warp_run_sum<8>(key, v)) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long g = node(d, w, q);
      atomicAdd(&np[g], kq[g] * (c.kdep * v[q]));
    }
  }
}

// Adjoint of the push of step n for the particles alive before it.  In: the
// state before the push (x^n, v^{n-1/2}), E^n, the output adjoints (lx, lv)
// and whether the particle survived the push.  Out: lv <- lv^{n-1/2},
// lx <- lx^{n+1} + the gather-weight gradient, lE += gather^T, dBz.
__global__ void __launch_bounds__(AB) k_adj_push(Dims d, WinConst c, const double *__restrict__ Ei,
                                                 const double *__restrict__ p, long long cap, int n,
                                                 const signed char *__restrict__ alive_before,
                                                 const signed char *__restrict__ alive_after,
                                                 double *__restrict__ lam, long long lcap, double *__restrict__ lE,
                                                 double *dBz) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double gB = 0.0;
  long long key = -1;
  Cic g0;
  double sc[24];
#pragma unroll
  for (int q = 0; q < 24; ++q) sc[q] = 0.0;
  if (i < n && alive_before[i]) {
    double lx = lam[i], ly = lam[lcap + i], lz = lam[2 * lcap + i];
    double lvx = lam[3 * lcap + i], lvy = lam[4 * lcap + i], lvz = lam[5 * lcap + i];
    if (!alive_after[i]) lx = ly = lz = lvx = lvy = lvz = 0.0;  // lost: nothing downstream
    const double xp = p[i], yp = p[cap + i], zp = p[2 * cap + i];
    const double vx = p[3 * cap + i], vy = p[4 * cap + i], vz = p[5 * cap + i];
    Cic w;
    cic(d, c, xp, yp, zp, w);
    double E[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const double wq = weight(w, q);
      const double *e = Ei + 3 * node(d, w, q);
      E[0] += wq * e[0];
      E[1] += wq * e[1];
      E[2] += wq * e[2];
    }
    // x^{n+1} = x^n + dt v^{n+1/2}
    lvx += c.dt * lx;
    lvy += c.dt * ly;
    lvz += c.dt * lz;
    double lEx, lEy, lEz, ux, uy, uz;
    if (c.boris) {
      const double v1x = vx + c.k1 * E[0], v1y = vy + c.k1 * E[1], v1z = vz + c.k1 * E[2];
      double tx, ty, tz;
      cross(v1x, v1y, v1z, c.Bx, c.By, c.Bz, tx, ty, tz);
      const double v3x = v1x + c.k1 * tx, v3y = v1y + c.k1 * ty, v3z = v1z + c.k1 * tz;
      // B_z derivative: v2 = v1 + kk (v3 x B), v3 = v1 + k1 (v1 x B)
      double ax, ay, az, bx, by, bz, ex, ey, ez;
      cross(v3x, v3y, v3z, c.Bx, c.By, c.Bz, ax, ay, az);  // v3 x B
      cross(v1x, v1y, v1z, 0.0, 0.0, 1.0, bx, by, bz);     // v1 x e_z = d(v3)/dBz / k1
      double cx, cy, cz;
      cross(c.k1 * bx, c.k1 * by, c.k1 * bz, c.Bx, c.By, c.Bz, cx, cy, cz);
      cross(v3x, v3y, v3z, 0.0, 0.0, 1.0, ex, ey, ez);
      const double dvx = c.dkk * ax + c.kk * (cx + ex), dvy = c.dkk * ay + c.kk * (cy + ey),
                   dvz = c.dkk * az + c.kk * (cz + ez);
      gB = lvx * dvx + lvy * dvy + lvz * dvz;
      // v+ = v2 + k1 E, v2 = v1 + kk (v3 x B), v3 = v1 + k1 (v1 x B), v1 = v + k1 E
      lEx = c.k1 * lvx;
      lEy = c.k1 * lvy;
      lEz = c.k1 * lvz;
      double l3x, l3y, l3z;
      cross(c.Bx, c.By, c.Bz, lvx, lvy, lvz, l3x, l3y, l3z);
      l3x *= c.kk;
      l3y *= c.kk;
      l3z *= c.kk;
      double t3x, t3y, t3z;
      cross(c.Bx, c.By, c.Bz, l3x, l3y, l3z, t3x, t3y, t3z);
      ux = lvx + l3x + c.k1 * t3x;
      uy = lvy + l3y + c.k1 * t3y;
      uz = lvz + l3z + c.k1 * t3z;
      lEx += c.k1 * ux;
      lEy += c.k1 * uy;
      lEz += c.k1 * uz;
    } else {
      ux = lvx;
      uy = lvy;
      uz = lvz;
      lEx = 2.0 * c.k1 * lvx;
      lEy = 2.0 * c.k1 * lvy;
      lEz = 2.0 * c.k1 * lvz;
    }
    // the weight gradient of the gather into lx; gather^T below
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long g = node(d, w, q);
      const double wq = weight(w, q);
      sc[3 * q + 0] = wq * lEx;
      sc[3 * q + 1] = wq * lEy;
      sc[3 * q + 2] = wq * lEz;
      double gx, gy, gz;
      dweight(c, w, q, gx, gy, gz);
      const double s = Ei[3 * g] * lEx + Ei[3 * g + 1] * lEy + Ei[3 * g + 2] * lEz;
      lx += gx * s;
      ly += gy * s;
      lz += gz * s;
    }
    key = w.g0;
    g0 = w;
    lam[i] = lx;
    lam[lcap + i] = ly;
    lam[2 * lcap + i] = lz;
    lam[3 * lcap + i] = ux;
    lam[4 * lcap + i] = uy;
    lam[5 * lcap + i] = uz;
  }
  // gather^T: lE at the 8 nodes, summed over the runs of the warp
  if (warp_run_sum<24>(key, sc)) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long g = node(d, g0, q);
      atomicAdd(&lE[3 * g + 0], sc[3 * q + 0]);
      atomicAdd(&lE[3 * g + 1], sc[3 * q + 1]);
      atomicAdd(&lE[3 * g + 2], sc[3 * q + 2]);
    }
  }
  // block sum of the B_z derivative
  for (int o = 16; o > 0; o >>= 1) gB += __shfl_xor_sync(0xffffffffu, gB, o);
  __shared__ double sh[AB / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = gB;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < AB / 32; ++k) s += sh[k];
    atomicAdd(dBz, s);
  }
}

// lx += deposit^T(lnp): kdep sum_c kq lnp(node_c) grad w_c (alive at x^n)
__global__ void __launch_bounds__(AB) k_adj_deposit(Dims d, WinConst c, const double *__restrict__ p, long long cap,
                                                    int n, const signed char *__restrict__ alive,
                                                    const double *__restrict__ kq, const double *__restrict__ lnp,
                                                    double *__restrict__ lam, long long lcap) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n || !alive[i]) return;
  Cic w;
  if (!cic(d, c, p[i], p[cap + i], p[2 * cap + i], w)) return;
  double lx = 0.0, ly = 0.0, lz = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const long long g = node(d, w, q);
    const double s = c.kdep * kq[g] * lnp[g];
    double gx, gy, gz;
    dweight(c, w, q, gx, gy, gz);
    lx += gx * s;
    ly += gy * s;
    lz += gz * s;
  }
  lam[i] += lx;
  lam[lcap + i] += ly;
  lam[2 * lcap + i] += lz;
}

// E = G phi transposed, pass 1: the wall nodes (bcnd >= 1) of the forward
// boundary pass (k_efield_boundary, Dirichlet walls): the last matching
// extrapolation branch writes E there; its extrapolated component moves to
// the E of the two nodes it reads (when the second one is not a wall, whose
// value the forward takes as given), its central components to phi.
__global__ void k_adj_efield_walls(Dims d, double hx, double hy, double hz, const int *__restrict__ bcnd,
                                   double *__restrict__ lE, double *__restrict__ lphi) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nx = d.n1 + 1, ny = d.n2 + 1, nz = d.n3 + 1;
  if (t >= nx * ny * nz) return;
  const int ix = 1 + (int)(t % nx), iy = 1 + (int)((t / nx) % ny), iz = 1 + (int)(t / (nx * ny));
  const long long q = d.g(ix, iy, iz);
  if (bcnd[q] < 1) return;
  const long long sy = d.N1, sz = d.N1 * d.N2;
  const bool xp2 = ix + 2 <= d.n1 + 2, xm2 = ix - 2 >= 0;
  const bool yp2 = iy + 2 <= d.n2 + 2, ym2 = iy - 2 >= 0;
  const bool zp2 = iz + 2 <= d.n3 + 2, zm2 = iz - 2 >= 0;
  // the forward's branches in order; the last one that matches wins
  int axis = -1;
  long long step = 0;
  if (bcnd[q + 1] <= 0 && xp2) { axis = 0; step = 1; }
  if (bcnd[q - 1] <= 0 && xm2) { axis = 0; step = -1; }
  if (bcnd[q + sy] <= 0 && yp2) { axis = 1; step = sy; }
  if (bcnd[q - sy] <= 0 && ym2) { axis = 1; step = -sy; }
  if (bcnd[q + sz] <= 0 && zp2) { axis = 2; step = sz; }
  if (bcnd[q - sz] <= 0 && zm2) { axis = 2; step = -sz; }
  if (axis < 0) return;  // keeps its value: constant in phi
  const double hh[3] = {hx, hy, hz};
  const long long st[3] = {1, sy, sz};
  for (int a = 0; a < 3; ++a) {
    const double l = lE[3 * q + a];
    if (l == 0.0) continue;
    if (a == axis) {
      atomicAdd(&lE[3 * (q + step) + a], 2.0 * l);
      if (bcnd[q + 2 * step] <= 0) atomicAdd(&lE[3 * (q + 2 * step) + a], -l);
    } else {
      atomicAdd(&lphi[q + st[a]], -l / (2.0 * hh[a]));
      atomicAdd(&lphi[q - st[a]], l / (2.0 * hh[a]));
    }
  }
}

// pass 2: the plasma nodes' central differences (k_efield_interior)
__global__ void k_adj_efield_plasma(Dims d, double hx, double hy, double hz, const int *__restrict__ bcnd,
                                    const double *__restrict__ lE, double *__restrict__ lphi) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long nx = d.n1 + 1, ny = d.n2 + 1, nz = d.n3 + 1;
  if (t >= nx * ny * nz) return;
  const int ix = 1 + (int)(t % nx), iy = 1 + (int)((t / nx) % ny), iz = 1 + (int)(t / (nx * ny));
  const long long q = d.g(ix, iy, iz);
  if (bcnd[q] > 0) return;
  const long long sy = d.N1, sz = d.N1 * d.N2;
  const double lx = lE[3 * q], ly = lE[3 * q + 1], lz = lE[3 * q + 2];
  if (lx != 0.0) {
    atomicAdd(&lphi[q + 1], -lx / (2.0 * hx));
    atomicAdd(&lphi[q - 1], lx / (2.0 * hx));
  }
  if (ly != 0.0) {
    atomicAdd(&lphi[q + sy], -ly / (2.0 * hy));
    atomicAdd(&lphi[q - sy], ly / (2.0 * hy));
  }
  if (lz != 0.0) {
    atomicAdd(&lphi[q + sz], -lz / (2.0 * hz));
    atomicAdd(&lphi[q - sz], lz / (2.0 * hz));
  }
}

// the right-hand side of the adjoint solve: lphi on plasma nodes, in the
// (n+2)^3 layout of the Poisson right-hand side
__global__ void k_adj_rhs(Dims d, const int *__restrict__ bcnd, const double *__restrict__ lphi,
                          double *__restrict__ b) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long R1 = d.N1 - 1, R2 = d.N2 - 1;
  if (t >= d.rcnt()) return;
  const int ix = (int)(t % R1), iy = (int)((t / R1) % R2), iz = (int)(t / (R1 * R2));
  double v = 0.0;
  if (ix >= 1 && iy >= 1 && iz >= 1) {
    const long long q = d.g(ix, iy, iz);
    if (bcnd[q] <= 0) v = lphi[q];
  }
  b[t] = v;
}

// dJ/dV_label: lphi on the label's nodes minus the couplings a mu_p of the
// plasma nodes p next to them; lnp = -q mu for the deposit adjoint
__global__ void __launch_bounds__(AB) k_adj_walls(Dims d, double aw, double an, double at, double q_s,
                                                  const int *__restrict__ bcnd, const double *__restrict__ lphi,
                                                  const double *__restrict__ mu, double *__restrict__ lnp,
                                                  double *__restrict__ dV, int nlabel) {
  __shared__ double sv[MAX_LABEL];
  if (threadIdx.x < MAX_LABEL) sv[threadIdx.x] = 0.0;
  __syncthreads();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t < d.cnt()) {
    const int b = bcnd[t];
    if (b >= 1 && b <= nlabel && lphi[t] != 0.0) atomicAdd(&sv[b - 1], lphi[t]);
    lnp[t] = -q_s * mu[t];
    if (b == -1) {
      const long long sy = d.N1, sz = d.N1 * d.N2;
      const long long nb[6] = {t - 1, t + 1, t - sy, t + sy, t - sz, t + sz};
      const double a[6] = {aw, aw, an, an, at, at};
      const double m = mu[t];
      for (int k = 0; k < 6; ++k) {
        const int bb = bcnd[nb[k]];
        if (bb >= 1 && bb <= nlabel) atomicAdd(&sv[bb - 1], -a[k] * m);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < nlabel && threadIdx.x < MAX_LABEL && sv[threadIdx.x] != 0.0)
    atomicAdd(&dV[threadIdx.x], sv[threadIdx.x]);
}

WinConst win_const(const lepic_grid_t &g, const lepic_phys_t &P, int ptype) {
  const int p = ptype - 1;
  WinConst c;
  memset(&c, 0, sizeof(c));
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  c.dt = P.dt;
  c.k1 = P.dt * P.charge[p] / (2.0 * P.mass[p]);
  c.Bx = P.Bconst[0];
  c.By = P.Bconst[1];
  c.Bz = P.Bconst[2];
  const double B2 = c.Bx * c.Bx + c.By * c.By + c.Bz * c.Bz;
  const double den = 1.0 + c.k1 * c.k1 * B2;
  c.kk = 2.0 * c.k1 / den;
  c.dkk = -4.0 * c.k1 * c.k1 * c.k1 * c.Bz / (den * den);
  c.boris = (P.flag_B == 1) ? 1 : 0;
  if (P.flag_B_pos == 1 && P.charge[p] > 0.0) c.boris = 0;
  c.kdep = P.Nm[p] / (g.h[0] * g.h[1] * g.h[2]);
  c.q = P.charge[p];
  c.mass = P.mass[p];
  c.Nm = P.Nm[p];
  return c;
}

// ============================================================ collisional window
// The differentiable window of the collisional step in the mixed layout
// (lepic_win_species_t): particles keep their slots, positions are a packed
// cell and offsets in [0,1), real type R = float (the mixed form) or double
// (its FP64 reference).  Step n maps (x^n, v^{n-1/2}) to (x^{n+1}, v^{n+1/2}):
// deposit x^n, field solve, E^n, collisions of step n (v^{n-1/2} -> v+),
// push.  The backward pass runs the steps in reverse without checkpoints:
// the push is reversed exactly up to rounding (x^n = x^{n+1} - dt v^{n+1/2},
// then the inverse Boris rotation with E^n gathered at x^n), a collision is
// undone from its record (the incident's velocity before it), a particle a
// wall took kept its state from before that push, and a particle a collision
// created does not exist before its step.  Only the fields phi^n of every
// step are kept.
constexpr int WALIVE = 0x7fff;
__device__ __forceinline__ int born_of(int b) { return (short)(b & 0xffff); }
__device__ __forceinline__ int lost_of(int b) { return b >> 16; }

template <class R>
struct WinS {
  int *cell;
  R *p;
  R *lam;
  int *bl;
  long long cap;
};

template <class R>
WinS<R> win_view(const lepic_win_species_t &w) {
  WinS<R> v;
  v.cell = w.cell;
  v.p = (R *)w.p;
  v.lam = (R *)w.lam;
  v.bl = w.bl;
  v.cap = w.cap;
  return v;
}

// cell (1-based) and offsets of a packed window particle
__device__ __forceinline__ void unpack_cell(int cc, int &ix, int &iy, int &iz) {
  ix = (cc & (LEPIC_CELL_MAX - 1)) + 1;
  iy = ((cc >> LEPIC_CELL_BITS) & (LEPIC_CELL_MAX - 1)) + 1;
  iz = (cc >> (2 * LEPIC_CELL_BITS)) + 1;
}
__device__ __forceinline__ int pack_cell(int ix, int iy, int iz) {
  return (ix - 1) | ((iy - 1) << LEPIC_CELL_BITS) | ((iz - 1) << (2 * LEPIC_CELL_BITS));
}

// the eight left-node weights (the order of Src/part_expmover.f90:100-108)
// of offsets (fx, fy, fz): the left-node factor is 1 - f
template <class R>
__device__ __forceinline__ void weights8(R fx, R fy, R fz, R (&w)[8]) {
  const R px = R(1) - fx, py = R(1) - fy, pz = R(1) - fz;
  w[0] = px * py * pz;
  w[1] = (R(1) - px) * py * pz;
  w[2] = (R(1) - px) * (R(1) - py) * pz;
  w[3] = px * (R(1) - py) * pz;
  w[4] = px * py * (R(1) - pz);
  w[5] = (R(1) - px) * py * (R(1) - pz);
  w[6] = (R(1) - px) * (R(1) - py) * (R(1) - pz);
  w[7] = px * (R(1) - py) * (R(1) - pz);
}

// E at node g: FP32 (Ex, Ey, Ez, 0) per node for the mixed form, FP64 (3 per
// node) for its reference
template <class R>
__device__ __forceinline__ void node_E(const void *E, long long g, R &ex, R &ey, R &ez);
template <>
__device__ __forceinline__ void node_E<float>(const void *E, long long g, float &ex, float &ey, float &ez) {
  const float4 e = reinterpret_cast<const float4 *>(E)[g];
  ex = e.x;
  ey = e.y;
  ez = e.z;
}
template <>
__device__ __forceinline__ void node_E<double>(const void *E, long long g, double &ex, double &ey, double &ez) {
  const double *e = reinterpret_cast<const double *>(E) + 3 * g;
  ex = e[0];
  ey = e[1];
  ez = e[2];
}

template <class R>
__device__ __forceinline__ void gather_E(const Dims &d, const void *E, long long g0, const R (&w)[8], R &Ex, R &Ey,
                                         R &Ez) {
  Ex = Ey = Ez = R(0);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    R ex, ey, ez;
    node_E<R>(E, g0 + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q)), ex, ey, ez);
    Ex += w[q] * ex;
    Ey += w[q] * ey;
    Ez += w[q] * ez;
  }
}

// the Boris rotation (Src/part_expmover.f90:214-240) and its inverse
template <class R>
__device__ __forceinline__ void boris(const WinConst &c, R Ex, R Ey, R Ez, R &vx, R &vy, R &vz) {
  const R k1 = (R)c.k1;
  if (c.boris) {
    const R Bx = (R)c.Bx, By = (R)c.By, Bz = (R)c.Bz, kk = (R)c.kk;
    const R v1x = vx + k1 * Ex, v1y = vy + k1 * Ey, v1z = vz + k1 * Ez;
    const R v3x = v1x + k1 * (v1y * Bz - v1z * By), v3y = v1y + k1 * (v1z * Bx - v1x * Bz),
            v3z = v1z + k1 * (v1x * By - v1y * Bx);
    vx = v1x + kk * (v3y * Bz - v3z * By) + k1 * Ex;
    vy = v1y + kk * (v3z * Bx - v3x * Bz) + k1 * Ey;
    vz = v1z + kk * (v3x * By - v3y * Bx) + k1 * Ez;
  } else {
    vx = vx + R(2) * k1 * Ex;
    vy = vy + R(2) * k1 * Ey;
    vz = vz + R(2) * k1 * Ez;
  }
}
template <class R>
__device__ __forceinline__ void boris_inverse(const WinConst &c, R Ex, R Ey, R Ez, R &vx, R &vy, R &vz) {
  const R k1 = (R)c.k1;
  if (c.boris) {
    const R Bx = (R)c.Bx, By = (R)c.By, Bz = (R)c.Bz, kk = (R)c.kk;
    const R v2x = vx - k1 * Ex, v2y = vy - k1 * Ey, v2z = vz - k1 * Ez;
    const R v3x = v2x - k1 * (v2y * Bz - v2z * By), v3y = v2y - k1 * (v2z * Bx - v2x * Bz),
            v3z = v2z - k1 * (v2x * By - v2y * Bx);
    vx = v2x - kk * (v3y * Bz - v3z * By) - k1 * Ex;
    vy = v2y - kk * (v3z * Bx - v3x * Bz) - k1 * Ey;
    vz = v2z - kk * (v3x * By - v3y * Bx) - k1 * Ez;
  } else {
    vx = vx - R(2) * k1 * Ex;
    vy = vy - R(2) * k1 * Ey;
    vz = vz - R(2) * k1 * Ez;
  }
}

// offset f moved by s cells of (possibly negative) displacement df: the
// new offset in [0,1) and the cell shift
template <class R>
__device__ __forceinline__ int move_offset(R &f, R df) {
  f = f + df;
  int sh = 0;
  if (!(f >= R(0) && f < R(1))) {
    sh = (int)floor((double)f);
    f = f - (R)sh;
    if (f >= R(1)) {
      f = R(0);
      sh += 1;
    }
    if (f < R(0)) f = R(0);
  }
  return sh;
}

// block-reduced FP64 atomic add
__device__ __forceinline__ void block_add(double v, double *dst) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __shared__ double sh[AB / 32];
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < AB / 32; ++k) s += sh[k];
    if (s != 0.0) atomicAdd(dst, s);
  }
}

// The window's particles of one tile of the sort that ordered them (slots
// tile_off[t] .. tile_off[t+1]) are scattered by one block into a box of
// nodes in shared memory: the tile's 8^3 cells and WH halo cells on each
// side, FP32 sums flushed into the FP64 grid after every WFLUSH particles and
// at the end.  A particle whose cell left the box (it drifted more than WH
// cells from its tile during the window) adds into the FP64 grid directly,
// and slots past the last tile (appended since that sort, collision
// products) are scattered by the untiled kernels.  Any slot order gives the
// same sums; the order only decides how many land in the box.
constexpr int WTC = LEPIC_TILE_CELLS;
constexpr int WH = 2;                       // halo cells
constexpr int WB = WTC + 2 * WH + 1;        // box nodes per axis
constexpr int WBN = WB * WB * WB;
constexpr int WFLUSH = 8 * AB;              // particles between flushes

struct WinTiles {
  const int *off;     // tile_off[0..ntiles] of the sort
  int ntx, nty;       // tiles per axis
};

WinTiles win_tiles(const lepic_grid_t &g, const lepic_win_species_t &w) {
  WinTiles T;
  T.off = w.tile_off;
  T.ntx = (g.n[0] + WTC - 1) / WTC;
  T.nty = (g.n[1] + WTC - 1) / WTC;
  return T;
}

// box origin (grid node of box node 0) of tile t
__device__ __forceinline__ void tile_box(const WinTiles &T, int t, int &bx, int &by, int &bz) {
  const int tx = t % T.ntx, ty = (t / T.ntx) % T.nty, tz = t / (T.ntx * T.nty);
  bx = tx * WTC + 1 - WH;
  by = ty * WTC + 1 - WH;
  bz = tz * WTC + 1 - WH;
}

// box-local base node of cell (ix, iy, iz), or -1 when the cell's 8 nodes
// are not all in the box
__device__ __forceinline__ int box_base(int ix, int iy, int iz, int bx, int by, int bz) {
  const int lx = ix - bx, ly = iy - by, lz = iz - bz;
  if ((unsigned)lx >= (unsigned)(WB - 1) || (unsigned)ly >= (unsigned)(WB - 1) || (unsigned)lz >= (unsigned)(WB - 1))
    return -1;
  return lx + WB * (ly + WB * lz);
}

__device__ __forceinline__ int box_off(int q) { return ox(q) + WB * (oy(q) + WB * oz(q)); }

// the deposit weights of slot i at step `step` (created before it, not lost
// before its push): true with the cell and the 8 weights
template <class R>
__device__ __forceinline__ bool cw_dep_one(const WinS<R> &S, long long i, int step, int &ix, int &iy, int &iz,
                                           R (&w)[8]) {
  const int b = S.bl[i];
  if (!(born_of(b) < step && lost_of(b) >= step)) return false;
  unpack_cell(S.cell[i], ix, iy, iz);
  weights8<R>(S.p[i], S.p[S.cap + i], S.p[2 * S.cap + i], w);
  return true;
}

// deposit of the slots first.. into np, kq applied
template <class R>
__global__ void __launch_bounds__(AB) k_cw_deposit(Dims d, WinConst c, WinS<R> S, const int *__restrict__ count,
                                                   long long first, int step, const double *__restrict__ kq,
                                                   double *__restrict__ np) {
  const long long i = first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long key = -1;
  double v[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) v[q] = 0.0;
  if (i < *count) {
    int ix, iy, iz;
    R w[8];
    if (cw_dep_one<R>(S, i, step, ix, iy, iz, w)) {
      key = d.g(ix, iy, iz);
      if constexpr (std::is_same<R, float>::value) {
        // the FP32 window deposits the integer weights of the mixed step
        int qw[8];
        qweights(S.p[i], S.p[S.cap + i], S.p[2 * S.cap + i], qw);
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = (double)qw[q] * QI;
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = (double)w[q];
      }
    }
  }
  if (warp_run_sum<8>(key, v)) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long g = key + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
      atomicAdd(&np[g], kq[g] * (c.kdep * v[q]));
    }
  }
}

// the box's non-zero node sums (NC components per node) into the FP64 grid
// dst (NC values per node, scaled by kdep kq[node] when kq is given), then
// cleared
template <int NC>
__device__ void flush_box(const Dims &d, float *box, int bx, int by, int bz, const double *__restrict__ kq,
                          double kdep, double *__restrict__ dst) {
  for (int e = threadIdx.x; e < WBN; e += blockDim.x) {
    float v[NC];
    bool any = false;
#pragma unroll
    for (int a = 0; a < NC; ++a) {
      v[a] = box[NC * e + a];
      any = any || v[a] != 0.f;
    }
    if (!any) continue;
    const int lx = e % WB, ly = (e / WB) % WB, lz = e / (WB * WB);
    const int gx = bx + lx, gy = by + ly, gz = bz + lz;
    // only nodes of cells 1..n receive weights: the box part outside the grid stays 0
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2) {
      const long long g = d.g(gx, gy, gz);
      const double k = kq ? kq[g] * kdep : 1.0;
#pragma unroll
      for (int a = 0; a < NC; ++a)
        if (v[a] != 0.f) atomicAdd(&dst[NC * g + a], k * (double)v[a]);
    }
#pragma unroll
    for (int a = 0; a < NC; ++a) box[NC * e + a] = 0.f;
  }
}

// the box's non-zero integer weight sums (units of 2^-QBITS, exact modulo
// 2^32: a node's sum over WFLUSH particles lies in [-5, 2^20 + 5] x WFLUSH)
// into the FP64 grid, kdep kq applied, then cleared
__device__ void flush_qbox(const Dims &d, unsigned *box, int bx, int by, int bz, const double *__restrict__ kq,
                           double kdep, double *__restrict__ np) {
  for (int e = threadIdx.x; e < WBN; e += blockDim.x) {
    const unsigned v = box[e];
    if (!v) continue;
    const int gx = bx + e % WB, gy = by + (e / WB) % WB, gz = bz + e / (WB * WB);
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2) {
      const long long g = d.g(gx, gy, gz);
      atomicAdd(&np[g], kq[g] * (kdep * (qsum_value(v, WFLUSH) * QI)));
    }
    box[e] = 0u;
  }
}
static_assert(qsum_window_ok(WFLUSH), "node sums of a flush window are read back modulo 2^32");

// the FP32 window's deposit, one block per tile: the integer weights of the
// mixed step (2^20 units per particle), summed exactly in a 32-bit node box
__global__ void __launch_bounds__(AB) k_cw_deposit_tiles(Dims d, WinConst c, WinS<float> S, const int *__restrict__ count,
                                                         WinTiles T, int step, const double *__restrict__ kq,
                                                         double *__restrict__ np) {
  __shared__ unsigned s_box[WBN];
  int bx, by, bz;
  tile_box(T, blockIdx.x, bx, by, bz);
  for (int e = threadIdx.x; e < WBN; e += AB) s_box[e] = 0u;
  __syncthreads();
  const long long N = *count;
  const long long lo = T.off[blockIdx.x];
  long long hi = T.off[blockIdx.x + 1];
  if (hi > N) hi = N;
  int chunks = 0;
  for (long long base = lo; base < hi; base += AB) {
    // every lane takes part in the run sums (base is uniform over the block)
    const long long i = base + threadIdx.x;
    int ix = 0, iy = 0, iz = 0;
    int w[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long key = -1;
    float wf[8];
    if (i < hi && cw_dep_one<float>(S, i, step, ix, iy, iz, wf)) {
      key = d.g(ix, iy, iz);
      qweights(S.p[i], S.p[S.cap + i], S.p[2 * S.cap + i], w);
    }
    // the lanes of one cell (consecutive in the sort's order) are summed
    // first, so a cell's particles do not contend for the same shared words
    if (warp_run_sum<8, int>(key, w)) {
      const int b0 = box_base(ix, iy, iz, bx, by, bz);
      if (b0 >= 0) {
#pragma unroll
        for (int q = 0; q < 8; ++q) atomicAdd(&s_box[b0 + box_off(q)], (unsigned)w[q]);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const long long g = key + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
          atomicAdd(&np[g], kq[g] * (c.kdep * ((double)w[q] * QI)));
        }
      }
    }
    if (++chunks == WFLUSH / AB && base + AB < hi) {
      chunks = 0;
      __syncthreads();
      flush_qbox(d, s_box, bx, by, bz, kq, c.kdep, np);
      __syncthreads();
    }
  }
  __syncthreads();
  flush_qbox(d, s_box, bx, by, bz, kq, c.kdep, np);
}

// E gathers of a cell's 8 nodes in the order of gather_E: from the FP32 /
// FP64 node array, or (FP32 window, one block per tile) from the tile's node
// box in shared memory when the cell lies in it
struct EGlobal {
  Dims d;
  const void *E;
  template <class R>
  __device__ __forceinline__ void operator()(int ix, int iy, int iz, const R (&w)[8], R &Ex, R &Ey, R &Ez) const {
    gather_E<R>(d, E, d.g(ix, iy, iz), w, Ex, Ey, Ez);
  }
};

struct ETile {
  Dims d;
  const void *E;
  const float4 *box;
  int bx, by, bz;
  __device__ __forceinline__ void operator()(int ix, int iy, int iz, const float (&w)[8], float &Ex, float &Ey,
                                             float &Ez) const {
    const int b0 = box_base(ix, iy, iz, bx, by, bz);
    if (b0 < 0) {
      gather_E<float>(d, E, d.g(ix, iy, iz), w, Ex, Ey, Ez);
      return;
    }
    Ex = Ey = Ez = 0.f;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 e = box[b0 + box_off(q)];
      Ex += w[q] * e.x;
      Ey += w[q] * e.y;
      Ez += w[q] * e.z;
    }
  }
};

// E (one float4 per node) of tile t's node box into shared memory
__device__ void stage_E_box(const Dims &d, const float4 *__restrict__ E, int bx, int by, int bz, float4 *box) {
  for (int e = threadIdx.x; e < WBN; e += blockDim.x) {
    const int gx = bx + e % WB, gy = by + (e / WB) % WB, gz = bz + e / (WB * WB);
    const bool in = gx >= 0 && gy >= 0 && gz >= 0 && gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2;
    box[e] = in ? E[d.g(gx, gy, gz)] : make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// the stored state of slot i (history word, cell, offsets, velocities),
// read in one go so that a thread can have two slots' loads in flight
template <class R>
struct PSt {
  int b, cell;
  R f[3], v[3];
};
template <class R>
__device__ __forceinline__ void pst_load(const WinS<R> &S, long long i, PSt<R> &s) {
  const long long cap = S.cap;
  s.b = S.bl[i];
  s.cell = S.cell[i];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    s.f[a] = S.p[a * cap + i];
    s.v[a] = S.p[(3 + a) * cap + i];
  }
}

// push of step `step`; a particle whose new cell is a wall cell (or outside
// the grid) is lost at this step and keeps its state from before the push;
// wl += the kinetic energy (J) the lost macroparticle carries
template <class R, class G>
__device__ __forceinline__ void cw_push_one(const Dims &d, const WinConst &c, const unsigned char *__restrict__ cw,
                                            const WinS<R> &S, long long i, const PSt<R> &st, int step,
                                            const G &gather, double &wl) {
  const int b = st.b;
  if (!(born_of(b) <= step && lost_of(b) >= step)) return;
  int ix, iy, iz;
  unpack_cell(st.cell, ix, iy, iz);
  const long long cap = S.cap;
  R fx = st.f[0], fy = st.f[1], fz = st.f[2];
  R vx = st.v[0], vy = st.v[1], vz = st.v[2];
  R w[8];
  weights8<R>(fx, fy, fz, w);
  R Ex, Ey, Ez;
  gather(ix, iy, iz, w, Ex, Ey, Ez);
  boris<R>(c, Ex, Ey, Ez, vx, vy, vz);
  const int ax = ix + move_offset<R>(fx, vx * (R)(c.dt / c.h0));
  const int ay = iy + move_offset<R>(fy, vy * (R)(c.dt / c.h1));
  const int az = iz + move_offset<R>(fz, vz * (R)(c.dt / c.h2));
  const int cx = ax < 0 ? 0 : (ax > d.n1 + 1 ? d.n1 + 1 : ax);
  const int cy = ay < 0 ? 0 : (ay > d.n2 + 1 ? d.n2 + 1 : ay);
  const int cz = az < 0 ? 0 : (az > d.n3 + 1 ? d.n3 + 1 : az);
  const bool lost = ax < 1 || ay < 1 || az < 1 || ax > d.n1 || ay > d.n2 || az > d.n3 || cw[d.c(cx, cy, cz)];
  if (lost) {
    S.bl[i] = (b & 0xffff) | (step << 16);
    wl += 0.5 * c.Nm * c.mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
  } else {
    S.cell[i] = pack_cell(ax, ay, az);
    S.p[i] = fx;
    S.p[cap + i] = fy;
    S.p[2 * cap + i] = fz;
    S.p[3 * cap + i] = vx;
    S.p[4 * cap + i] = vy;
    S.p[5 * cap + i] = vz;
  }
}

// slots first..; wall_acc += the kinetic energy carried to the walls
template <class R>
__global__ void __launch_bounds__(AB) k_cw_push(Dims d, WinConst c, const void *__restrict__ E,
                                                const unsigned char *__restrict__ cw, WinS<R> S,
                                                const int *__restrict__ count, long long first, int step,
                                                double *wall_acc) {
  const long long i = first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double wl = 0.0;
  if (i < *count) {
    PSt<R> st;
    pst_load<R>(S, i, st);
    cw_push_one<R>(d, c, cw, S, i, st, step, EGlobal{d, E}, wl);
  }
  block_add(wl, wall_acc);
}

// the FP32 window's push, one block per tile, E of the tile's box staged.
// (A variant that also deposited the kept particles for the next step, in a
// node box beside E, was 4 % slower than this push and k_cw_deposit_tiles.)
__global__ void __launch_bounds__(AB, 3) k_cw_push_tiles(Dims d, WinConst c, const float4 *__restrict__ E,
                                                      const unsigned char *__restrict__ cw, WinS<float> S,
                                                      const int *__restrict__ count, WinTiles T, int step,
                                                      double *wall_acc) {
  __shared__ float4 s_E[WBN];
  int bx, by, bz;
  tile_box(T, blockIdx.x, bx, by, bz);
  stage_E_box(d, E, bx, by, bz, s_E);
  __syncthreads();
  const ETile G{d, E, s_E, bx, by, bz};
  const long long N = *count;
  const long long lo = T.off[blockIdx.x];
  long long hi = T.off[blockIdx.x + 1];
  if (hi > N) hi = N;
  double wl = 0.0;
  // two slots per pass, both loaded before either is pushed
  for (long long i = lo + threadIdx.x; i < hi; i += 2 * AB) {
    const long long j = i + AB;
    PSt<float> s0, s1;
    pst_load<float>(S, i, s0);
    if (j < hi) pst_load<float>(S, j, s1);
    cw_push_one<float>(d, c, cw, S, i, s0, step, G, wl);
    if (j < hi) cw_push_one<float>(d, c, cw, S, j, s1, step, G, wl);
  }
  block_add(wl, wall_acc);
}

// the push of step `step` undone for the particles it kept: x^n from
// x^{n+1} and v^{n+1/2}, then v+ by the inverse rotation with E^n at x^n
// on a state in registers: true when the push of `step` was undone (st
// updated in place)
template <class R, class G>
__device__ __forceinline__ bool cw_reverse_core(const Dims &d, const WinConst &c, PSt<R> &st, int step,
                                                const G &gather) {
  const int b = st.b;
  if (!(born_of(b) <= step && lost_of(b) > step)) return false;
  int ix, iy, iz;
  unpack_cell(st.cell, ix, iy, iz);
  R fx = st.f[0], fy = st.f[1], fz = st.f[2];
  R vx = st.v[0], vy = st.v[1], vz = st.v[2];
  ix += move_offset<R>(fx, -vx * (R)(c.dt / c.h0));
  iy += move_offset<R>(fy, -vy * (R)(c.dt / c.h1));
  iz += move_offset<R>(fz, -vz * (R)(c.dt / c.h2));
  ix = ix < 1 ? 1 : (ix > d.n1 ? d.n1 : ix);
  iy = iy < 1 ? 1 : (iy > d.n2 ? d.n2 : iy);
  iz = iz < 1 ? 1 : (iz > d.n3 ? d.n3 : iz);
  R w[8];
  weights8<R>(fx, fy, fz, w);
  R Ex, Ey, Ez;
  gather(ix, iy, iz, w, Ex, Ey, Ez);
  boris_inverse<R>(c, Ex, Ey, Ez, vx, vy, vz);
  st.cell = pack_cell(ix, iy, iz);
  st.f[0] = fx;
  st.f[1] = fy;
  st.f[2] = fz;
  st.v[0] = vx;
  st.v[1] = vy;
  st.v[2] = vz;
  return true;
}

template <class R>
__device__ __forceinline__ void pst_store(const WinS<R> &S, long long i, const PSt<R> &st) {
  const long long cap = S.cap;
  S.cell[i] = st.cell;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    S.p[a * cap + i] = st.f[a];
    S.p[(3 + a) * cap + i] = st.v[a];
  }
}

template <class R, class G>
__device__ __forceinline__ void cw_reverse_one(const Dims &d, const WinConst &c, const WinS<R> &S, long long i,
                                               const PSt<R> &st0, int step, const G &gather) {
  PSt<R> st = st0;
  if (cw_reverse_core<R>(d, c, st, step, gather)) pst_store<R>(S, i, st);
}

template <class R>
__global__ void __launch_bounds__(AB) k_cw_reverse(Dims d, WinConst c, const void *__restrict__ E, WinS<R> S,
                                                   const int *__restrict__ count, long long first, int step) {
  const long long i = first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < *count) {
    PSt<R> st;
    pst_load<R>(S, i, st);
    cw_reverse_one<R>(d, c, S, i, st, step, EGlobal{d, E});
  }
}

__global__ void __launch_bounds__(AB, 3) k_cw_reverse_tiles(Dims d, WinConst c, const float4 *__restrict__ E,
                                                         WinS<float> S, const int *__restrict__ count, WinTiles T,
                                                         int step) {
  __shared__ float4 s_E[WBN];
  int bx, by, bz;
  tile_box(T, blockIdx.x, bx, by, bz);
  stage_E_box(d, E, bx, by, bz, s_E);
  __syncthreads();
  const ETile G{d, E, s_E, bx, by, bz};
  const long long N = *count;
  const long long lo = T.off[blockIdx.x];
  long long hi = T.off[blockIdx.x + 1];
  if (hi > N) hi = N;
  for (long long i = lo + threadIdx.x; i < hi; i += 2 * AB) {
    const long long j = i + AB;
    PSt<float> s0, s1;
    pst_load<float>(S, i, s0);
    if (j < hi) pst_load<float>(S, j, s1);
    cw_reverse_one<float>(d, c, S, i, s0, step, G);
    if (j < hi) cw_reverse_one<float>(d, c, S, j, s1, step, G);
  }
}

// adjoint of the push of step `step` at the state (x^n, v+) for the
// particles it moved: lam (dJ/dx^{n+1}, dJ/dv^{n+1/2}) -> (the push's part of
// dJ/dx^n, dJ/dv+), lE += gather^T, dBz.  A particle lost at this step has no
// later use except the wall-flux observable: wflux Nm m v^{n+1/2}.
// Per slot: true when slot i was pushed at `step`, with its cell, its 24
// contributions to lE (node q, component a at 3 q + a) and gB += its dJ/dB_z.
// On a state and adjoint held in registers: st the particle at (x^n, v+),
// lam in: (dJ/dx^{n+1}, dJ/dv^{n+1/2}), out: the push's part of dJ/dx^n and
// dJ/dv+ (a particle lost at this step starts from zero, or from wflux).
template <class R, class N>
__device__ __forceinline__ bool cw_adj_push_core(const WinConst &c, const N &nodes, const PSt<R> &st, int step,
                                                 double wflux, R (&lam)[6], int &ix, int &iy, int &iz,
                                                 R (&sc)[24], double &gB) {
  const int b = st.b;
  if (!(born_of(b) <= step && lost_of(b) >= step)) return false;
  unpack_cell(st.cell, ix, iy, iz);
  const R fx = st.f[0], fy = st.f[1], fz = st.f[2];
  const R vx = st.v[0], vy = st.v[1], vz = st.v[2];
  R w[8];
  weights8<R>(fx, fy, fz, w);
  // E at the cell's 8 nodes, read once for the gather and its weight gradient
  R en[8][3];
  nodes(ix, iy, iz, en);
  R Ex = R(0), Ey = R(0), Ez = R(0);   // the order of gather_E
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    Ex += w[q] * en[q][0];
    Ey += w[q] * en[q][1];
    Ez += w[q] * en[q][2];
  }
  R lx, ly, lz, lvx, lvy, lvz;
  if (lost_of(b) == step) {
    lx = ly = lz = R(0);
    lvx = lvy = lvz = R(0);
    if (wflux != 0.0) {
      R ux = vx, uy = vy, uz = vz;
      boris<R>(c, Ex, Ey, Ez, ux, uy, uz);
      const R k = (R)(wflux * c.Nm * c.mass);
      lvx = k * ux;
      lvy = k * uy;
      lvz = k * uz;
    }
  } else {
    lx = lam[0];
    ly = lam[1];
    lz = lam[2];
    lvx = lam[3];
    lvy = lam[4];
    lvz = lam[5];
  }
  // x^{n+1} = x^n + dt v^{n+1/2}
  const R dt = (R)c.dt, k1 = (R)c.k1, kk = (R)c.kk;
  lvx += dt * lx;
  lvy += dt * ly;
  lvz += dt * lz;
  R lEx, lEy, lEz, ux, uy, uz;
  if (c.boris) {
    const R Bx = (R)c.Bx, By = (R)c.By, Bz = (R)c.Bz;
    const R v1x = vx + k1 * Ex, v1y = vy + k1 * Ey, v1z = vz + k1 * Ez;
    const R v3x = v1x + k1 * (v1y * Bz - v1z * By), v3y = v1y + k1 * (v1z * Bx - v1x * Bz),
            v3z = v1z + k1 * (v1x * By - v1y * Bx);
    // d v^{n+1/2} / d Bz: v2 = v1 + kk (v3 x B), v3 = v1 + k1 (v1 x B)
    const R ax = v3y * Bz - v3z * By, ay = v3z * Bx - v3x * Bz, az = v3x * By - v3y * Bx;   // v3 x B
    const R bx = v1y, by = -v1x;                                                            // v1 x e_z
    const R cx = k1 * (by * Bz), cy = k1 * (-bx * Bz), cz = k1 * (bx * By - by * Bx);     // (k1 v1 x e_z) x B
    const R ex = v3y, ey = -v3x;                                                            // v3 x e_z
    const R dkk = (R)c.dkk;
    gB += (double)(lvx * (dkk * ax + kk * (cx + ex)) + lvy * (dkk * ay + kk * (cy + ey)) + lvz * (dkk * az + kk * cz));
    lEx = k1 * lvx;
    lEy = k1 * lvy;
    lEz = k1 * lvz;
    // l3 = kk (B x lv), u = lv + l3 + k1 (B x l3)
    const R l3x = kk * (By * lvz - Bz * lvy), l3y = kk * (Bz * lvx - Bx * lvz), l3z = kk * (Bx * lvy - By * lvx);
    ux = lvx + l3x + k1 * (By * l3z - Bz * l3y);
    uy = lvy + l3y + k1 * (Bz * l3x - Bx * l3z);
    uz = lvz + l3z + k1 * (Bx * l3y - By * l3x);
    lEx += k1 * ux;
    lEy += k1 * uy;
    lEz += k1 * uz;
  } else {
    ux = lvx;
    uy = lvy;
    uz = lvz;
    lEx = R(2) * k1 * lvx;
    lEy = R(2) * k1 * lvy;
    lEz = R(2) * k1 * lvz;
  }
  // gather^T and the weight gradient of the gather into lx
  const R px = R(1) - fx, py = R(1) - fy, pz = R(1) - fz;
  const R hx = (R)(1.0 / c.h0), hy = (R)(1.0 / c.h1), hz = (R)(1.0 / c.h2);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    sc[3 * q + 0] = w[q] * lEx;
    sc[3 * q + 1] = w[q] * lEy;
    sc[3 * q + 2] = w[q] * lEz;
    const R ax_ = ox(q) ? R(1) - px : px, ay_ = oy(q) ? R(1) - py : py, az_ = oz(q) ? R(1) - pz : pz;
    const R sx = ox(q) ? hx : -hx, sy = oy(q) ? hy : -hy, sz = oz(q) ? hz : -hz;
    const R s = en[q][0] * lEx + en[q][1] * lEy + en[q][2] * lEz;
    lx += sx * ay_ * az_ * s;
    ly += ax_ * sy * az_ * s;
    lz += ax_ * ay_ * sz * s;
  }
  lam[0] = lx;
  lam[1] = ly;
  lam[2] = lz;
  lam[3] = ux;
  lam[4] = uy;
  lam[5] = uz;
  return true;
}

// the same on slot i of the window's stores
template <class R, class N>
__device__ __forceinline__ bool cw_adj_push_one(const WinConst &c, const N &nodes, const WinS<R> &S, long long i,
                                                int step, double wflux, int &ix, int &iy, int &iz, R (&sc)[24],
                                                double &gB) {
  PSt<R> st;
  pst_load<R>(S, i, st);
  if (!(born_of(st.b) <= step && lost_of(st.b) >= step)) return false;
  const long long cap = S.cap;
  R lam[6];
#pragma unroll
  for (int a = 0; a < 6; ++a) lam[a] = S.lam[a * cap + i];
  cw_adj_push_core<R>(c, nodes, st, step, wflux, lam, ix, iy, iz, sc, gB);
#pragma unroll
  for (int a = 0; a < 6; ++a) S.lam[a * cap + i] = lam[a];
  return true;
}

// E at the 8 nodes of a cell: from the node array, or from the tile's node
// box in shared memory when the cell lies in it
struct ENodesGlobal {
  Dims d;
  const void *E;
  template <class R>
  __device__ __forceinline__ void operator()(int ix, int iy, int iz, R (&en)[8][3]) const {
    const long long g0 = d.g(ix, iy, iz);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      node_E<R>(E, g0 + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q)), en[q][0], en[q][1], en[q][2]);
  }
};

struct ENodesTile {
  Dims d;
  const void *E;
  const float4 *box;
  int bx, by, bz;
  __device__ __forceinline__ void operator()(int ix, int iy, int iz, float (&en)[8][3]) const {
    const int b0 = box_base(ix, iy, iz, bx, by, bz);
    if (b0 < 0) {
      ENodesGlobal{d, E}(ix, iy, iz, en);
      return;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const float4 e = box[b0 + box_off(q)];
      en[q][0] = e.x;
      en[q][1] = e.y;
      en[q][2] = e.z;
    }
  }
};

// slots first..: warp run sums and FP64 atomics into lE
template <class R>
__global__ void __launch_bounds__(AB) k_cw_adj_push(Dims d, WinConst c, const void *__restrict__ E, WinS<R> S,
                                                    const int *__restrict__ count, long long first, int step,
                                                    double wflux, double *__restrict__ lE, double *dBz) {
  const long long i = first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double gB = 0.0;
  long long key = -1;
  double sc[24];
#pragma unroll
  for (int q = 0; q < 24; ++q) sc[q] = 0.0;
  if (i < *count) {
    int ix, iy, iz;
    R r[24];
    if (cw_adj_push_one<R>(c, ENodesGlobal{d, E}, S, i, step, wflux, ix, iy, iz, r, gB)) {
      key = d.g(ix, iy, iz);
#pragma unroll
      for (int q = 0; q < 24; ++q) sc[q] = (double)r[q];
    }
  }
  if (warp_run_sum<24>(key, sc)) {
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long g = key + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
      atomicAdd(&lE[3 * g + 0], sc[3 * q + 0]);
      atomicAdd(&lE[3 * g + 1], sc[3 * q + 1]);
      atomicAdd(&lE[3 * g + 2], sc[3 * q + 2]);
    }
  }
  block_add(gB, dBz);
}

// the FP32 window's push adjoint, one block per tile: E of the tile's node
// box staged, lE summed in the box (FP32, flushed into FP64 after every
// WFLUSH particles); dynamic shared memory CW_ADJ_SMEM
constexpr int CW_ADJ_SMEM = WBN * (16 + 12);
__global__ void __launch_bounds__(AB, 3) k_cw_adj_push_tiles(Dims d, WinConst c, const float4 *__restrict__ E,
                                                          WinS<float> S, const int *__restrict__ count, WinTiles T,
                                                          int step, double wflux, double *__restrict__ lE,
                                                          double *dBz) {
  extern __shared__ __align__(16) unsigned char s_dyn[];
  float4 *s_E = reinterpret_cast<float4 *>(s_dyn);
  float *s_box = reinterpret_cast<float *>(s_dyn + 16 * WBN);
  int bx, by, bz;
  tile_box(T, blockIdx.x, bx, by, bz);
  stage_E_box(d, E, bx, by, bz, s_E);
  for (int e = threadIdx.x; e < 3 * WBN; e += AB) s_box[e] = 0.f;
  __syncthreads();
  const ENodesTile nodes{d, E, s_E, bx, by, bz};
  const long long N = *count;
  const long long lo = T.off[blockIdx.x];
  long long hi = T.off[blockIdx.x + 1];
  if (hi > N) hi = N;
  double gB = 0.0;
  int chunks = 0;
  for (long long base = lo; base < hi; base += AB) {
    // every lane takes part in the run sums (base is uniform over the block)
    const long long i = base + threadIdx.x;
    int ix = 0, iy = 0, iz = 0;
    float r[24];
    long long key = -1;
    int b0 = -1;
    if (i < hi && cw_adj_push_one<float>(c, nodes, S, i, step, wflux, ix, iy, iz, r, gB)) {
      key = d.g(ix, iy, iz);
      b0 = box_base(ix, iy, iz, bx, by, bz);
    } else {
#pragma unroll
      for (int q = 0; q < 24; ++q) r[q] = 0.f;
    }
    // value v = 3 q + a: component a of node q of the cell
    warp_scatter_sum<24>(key, b0, r, [&](long long k, int b, int v, float val) {
      const int q = v / 3, a = v - 3 * q;
      if (b >= 0) {
        atomicAdd(&s_box[3 * (b + box_off(q)) + a], val);
      } else {
        const long long g = k + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
        atomicAdd(&lE[3 * g + a], (double)val);
      }
    });
    if (++chunks == WFLUSH / AB && base + AB < hi) {
      chunks = 0;
      __syncthreads();
      flush_box<3>(d, s_box, bx, by, bz, nullptr, 1.0, lE);
      __syncthreads();
    }
  }
  __syncthreads();
  flush_box<3>(d, s_box, bx, by, bz, nullptr, 1.0, lE);
  block_add(gB, dBz);
}

// lx += deposit^T of the adjoint potential mu for the particles deposited at
// `step`: the deposit adds kq kdep w to np, rhs = -q np, so
// dJ/dx += -q kdep sum_c kq mu grad w_c
// the deposit adjoint of a particle at offsets (fx, fy, fz) given the
// weights m_q = -q kdep kq mu at its cell's 8 nodes (M(q) returns them):
// (lx, ly, lz) += -q kdep sum kq mu grad w
template <class M>
__device__ __forceinline__ void cw_adj_dep_core(const WinConst &c, double fx, double fy, double fz, M m, double &lx,
                                                double &ly, double &lz) {
  const double px = 1.0 - fx, py = 1.0 - fy, pz = 1.0 - fz;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double s = m(q);
    const double ax = ox(q) ? 1.0 - px : px, ay = oy(q) ? 1.0 - py : py, az = oz(q) ? 1.0 - pz : pz;
    const double sx = ox(q) ? 1.0 / c.h0 : -1.0 / c.h0, sy = oy(q) ? 1.0 / c.h1 : -1.0 / c.h1,
                 sz = oz(q) ? 1.0 / c.h2 : -1.0 / c.h2;
    lx += sx * ay * az * s;
    ly += ax * sy * az * s;
    lz += ax * ay * sz * s;
  }
}

// the deposit adjoint of slot i at `step` given the weights m_q = -q kdep kq
// mu at its cell's 8 nodes (M(q) returns them)
template <class R, class M>
__device__ __forceinline__ void cw_adj_dep_one(const WinConst &c, const WinS<R> &S, long long i, M m) {
  const long long cap = S.cap;
  const double fx = S.p[i], fy = S.p[cap + i], fz = S.p[2 * cap + i];
  const double px = 1.0 - fx, py = 1.0 - fy, pz = 1.0 - fz;
  double lx = 0.0, ly = 0.0, lz = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const double s = m(q);
    const double ax = ox(q) ? 1.0 - px : px, ay = oy(q) ? 1.0 - py : py, az = oz(q) ? 1.0 - pz : pz;
    const double sx = ox(q) ? 1.0 / c.h0 : -1.0 / c.h0, sy = oy(q) ? 1.0 / c.h1 : -1.0 / c.h1,
                 sz = oz(q) ? 1.0 / c.h2 : -1.0 / c.h2;
    lx += sx * ay * az * s;
    ly += ax * sy * az * s;
    lz += ax * ay * sz * s;
  }
  S.lam[i] += (R)lx;
  S.lam[cap + i] += (R)ly;
  S.lam[2 * cap + i] += (R)lz;
}

template <class R>
__global__ void __launch_bounds__(AB) k_cw_adj_deposit(Dims d, WinConst c, WinS<R> S, const int *__restrict__ count,
                                                       long long first, int step, const double *__restrict__ kq,
                                                       const double *__restrict__ mu) {
  const long long i = first + blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= *count) return;
  const int b = S.bl[i];
  if (!(born_of(b) < step && lost_of(b) >= step)) return;
  int ix, iy, iz;
  unpack_cell(S.cell[i], ix, iy, iz);
  const long long g0 = d.g(ix, iy, iz);
  cw_adj_dep_one<R>(c, S, i, [&](int q) {
    const long long g = g0 + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
    return -c.q * c.kdep * kq[g] * mu[g];
  });
}

// the FP32 window's deposit adjoint, one block per tile: -q kdep kq mu of
// the tile's node box read into shared memory once
__global__ void __launch_bounds__(AB) k_cw_adj_deposit_tiles(Dims d, WinConst c, WinS<float> S,
                                                             const int *__restrict__ count, WinTiles T, int step,
                                                             const double *__restrict__ kq,
                                                             const double *__restrict__ mu) {
  __shared__ double s_m[WBN];
  int bx, by, bz;
  tile_box(T, blockIdx.x, bx, by, bz);
  for (int e = threadIdx.x; e < WBN; e += AB) {
    const int gx = bx + e % WB, gy = by + (e / WB) % WB, gz = bz + e / (WB * WB);
    double m = 0.0;
    if (gx >= 0 && gy >= 0 && gz >= 0 && gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2) {
      const long long g = d.g(gx, gy, gz);
      m = -c.q * c.kdep * kq[g] * mu[g];
    }
    s_m[e] = m;
  }
  __syncthreads();
  const long long N = *count;
  const long long lo = T.off[blockIdx.x];
  long long hi = T.off[blockIdx.x + 1];
  if (hi > N) hi = N;
  // two slots per pass: both slots' history words and cells read first
  for (long long i0 = lo + threadIdx.x; i0 < hi; i0 += 2 * AB) {
    int bb[2], cc[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const long long i = i0 + u * AB;
      bb[u] = i < hi ? S.bl[i] : -1;
      cc[u] = i < hi ? S.cell[i] : 0;
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const long long i = i0 + u * AB;
      if (i >= hi || !(born_of(bb[u]) < step && lost_of(bb[u]) >= step)) continue;
      int ix, iy, iz;
      unpack_cell(cc[u], ix, iy, iz);
      const int b0 = box_base(ix, iy, iz, bx, by, bz);
      if (b0 >= 0) {
        cw_adj_dep_one<float>(c, S, i, [&](int q) { return s_m[b0 + box_off(q)]; });
      } else {
        const long long g0 = d.g(ix, iy, iz);
        cw_adj_dep_one<float>(c, S, i, [&](int q) {
          const long long g = g0 + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
          return -c.q * c.kdep * kq[g] * mu[g];
        });
      }
    }
  }
}

// One backward step of the FP32 window fused per particle, one block per
// tile: the deposit adjoint of step + 1 at x^{step+1} (mu of that step's
// adjoint solve, none when mu is null), the push of `step` undone, and the
// adjoint of that push (lE scattered through the node box as
// k_cw_adj_push_tiles does).  The particle's state and adjoint are read and
// written once instead of by three kernels; a thread's next slot (history
// word, cell, 6 planes, 6 adjoint planes) is copied into shared memory by
// cp.async while it works on the current one.  Dynamic shared memory
// CW_BACK_SMEM: E (float4), -q kdep kq mu (double) and lE (3 floats) of the
// tile's node box, then the staging slots (14 words per thread).
constexpr int CW_BACK_PF = 14;
constexpr int CW_BACK_SMEM = WBN * (16 + 8 + 12) + CW_BACK_PF * 4 * AB;
__global__ void __launch_bounds__(AB, 2) k_cw_back_tiles(Dims d, WinConst c, const float4 *__restrict__ E,
                                                         WinS<float> S, const int *__restrict__ count, WinTiles T,
                                                         int step, const double *__restrict__ kq,
                                                         const double *__restrict__ mu, double wflux,
                                                         double *__restrict__ lE, double *dBz) {
  extern __shared__ __align__(16) unsigned char s_dyn[];
  float4 *s_E = reinterpret_cast<float4 *>(s_dyn);
  double *s_m = reinterpret_cast<double *>(s_dyn + 16 * WBN);
  float *s_box = reinterpret_cast<float *>(s_dyn + 24 * WBN);
  unsigned *s_pf = reinterpret_cast<unsigned *>(s_dyn + 36 * WBN);   // [CW_BACK_PF][AB]
  const long long N = *count;
  const long long lo = T.off[blockIdx.x];
  long long hi = T.off[blockIdx.x + 1];
  if (hi > N) hi = N;
  const long long cap = S.cap;
  // the copies of slot i into this thread's staging words
  auto fetch = [&](long long i) {
    if (i < hi) {
      unsigned *w = s_pf + threadIdx.x;
      cp_async4(w, S.bl + i);
      cp_async4(w + AB, S.cell + i);
#pragma unroll
      for (int a = 0; a < 6; ++a) {
        cp_async4(w + (2 + a) * AB, S.p + a * cap + i);
        cp_async4(w + (8 + a) * AB, S.lam + a * cap + i);
      }
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  fetch(lo + threadIdx.x);
  int bx, by, bz;
  tile_box(T, blockIdx.x, bx, by, bz);
  stage_E_box(d, E, bx, by, bz, s_E);
  for (int e = threadIdx.x; e < WBN; e += AB) {
    const int gx = bx + e % WB, gy = by + (e / WB) % WB, gz = bz + e / (WB * WB);
    double m = 0.0;
    if (mu && gx >= 0 && gy >= 0 && gz >= 0 && gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2) {
      const long long g = d.g(gx, gy, gz);
      m = -c.q * c.kdep * kq[g] * mu[g];
    }
    s_m[e] = m;
  }
  for (int e = threadIdx.x; e < 3 * WBN; e += AB) s_box[e] = 0.f;
  __syncthreads();
  const ETile G{d, E, s_E, bx, by, bz};
  const ENodesTile nodes{d, E, s_E, bx, by, bz};
  double gB = 0.0;
  int chunks = 0;
  for (long long base = lo; base < hi; base += AB) {
    // every lane takes part in the scatter sums (base is uniform over the block)
    const long long i = base + threadIdx.x;
    int ix = 0, iy = 0, iz = 0;
    float r[24];
    long long key = -1;
    int b0 = -1;
#pragma unroll
    for (int q = 0; q < 24; ++q) r[q] = 0.f;
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    PSt<float> st;
    float lam[6];
    if (i < hi) {
      const unsigned *w = s_pf + threadIdx.x;
      st.b = (int)w[0];
      st.cell = (int)w[AB];
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        st.f[a] = __uint_as_float(w[(2 + a) * AB]);
        st.v[a] = __uint_as_float(w[(5 + a) * AB]);
      }
#pragma unroll
      for (int a = 0; a < 6; ++a) lam[a] = __uint_as_float(w[(8 + a) * AB]);
    }
    fetch(i + AB);
    if (i < hi) {
      bool lam_changed = false;
      // the deposit adjoint of step + 1, at the position before the undo
      if (mu && born_of(st.b) < step + 1 && lost_of(st.b) >= step + 1) {
        int jx, jy, jz;
        unpack_cell(st.cell, jx, jy, jz);
        double lx = 0.0, ly = 0.0, lz = 0.0;
        const int bm = box_base(jx, jy, jz, bx, by, bz);
        if (bm >= 0) {
          cw_adj_dep_core(c, st.f[0], st.f[1], st.f[2], [&](int q) { return s_m[bm + box_off(q)]; }, lx, ly, lz);
        } else {
          const long long g0 = d.g(jx, jy, jz);
          cw_adj_dep_core(c, st.f[0], st.f[1], st.f[2], [&](int q) {
            const long long g = g0 + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
            return -c.q * c.kdep * kq[g] * mu[g];
          }, lx, ly, lz);
        }
        lam[0] += (float)lx;
        lam[1] += (float)ly;
        lam[2] += (float)lz;
        lam_changed = true;
      }
      if (cw_reverse_core<float>(d, c, st, step, G)) pst_store<float>(S, i, st);
      if (cw_adj_push_core<float>(c, nodes, st, step, wflux, lam, ix, iy, iz, r, gB)) {
        key = d.g(ix, iy, iz);
        b0 = box_base(ix, iy, iz, bx, by, bz);
        lam_changed = true;
      }
      if (lam_changed)
#pragma unroll
        for (int a = 0; a < 6; ++a) S.lam[a * cap + i] = lam[a];
    }
    warp_scatter_sum<24>(key, b0, r, [&](long long k, int b, int v, float val) {
      const int q = v / 3, a = v - 3 * q;
      if (b >= 0) {
        atomicAdd(&s_box[3 * (b + box_off(q)) + a], val);
      } else {
        const long long g = k + ox(q) + d.N1 * (oy(q) + d.N2 * (long long)oz(q));
        atomicAdd(&lE[3 * g + a], (double)val);
      }
    });
    if (++chunks == WFLUSH / AB && base + AB < hi) {
      chunks = 0;
      __syncthreads();
      flush_box<3>(d, s_box, bx, by, bz, nullptr, 1.0, lE);
      __syncthreads();
    }
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
  __syncthreads();
  flush_box<3>(d, s_box, bx, by, bz, nullptr, 1.0, lE);
  block_add(gB, dBz);
}

// every species of the window, for the collision kernels
template <class R>
struct CwSet {
  WinS<R> S[LEPIC_NPART];
  int *count[LEPIC_NPART];
  double mass[LEPIC_NPART];
};

// the recorded collisions of one step applied again (a later forward pass:
// finite differences, the FP64 reference): each byproduct from the
// incident's current velocity, the recorded target and directions; the
// incident's velocity before is written back into the record
template <class R>
__global__ void __launch_bounds__(AB) k_cw_replay(lepic_win_event_t *ev, int ne, CwSet<R> set, double qe) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  lepic_win_event_t &e = ev[k];
  const WinS<R> A = set.S[e.P];
  const long long i = e.i, ca = A.cap;
  const double vx = A.p[3 * ca + i], vy = A.p[4 * ca + i], vz = A.p[5 * ca + i];
  e.vold[0] = vx;
  e.vold[1] = vy;
  e.vold[2] = vz;
  const double mp = fabs(set.mass[e.P]), mt = e.m_t, M = mp + mt, mu = mp * mt / M;
  const double rx = vx - e.tv[0], ry = vy - e.tv[1], rz = vz - e.tv[2];
  const double vcx = (mp * vx + mt * e.tv[0]) / M, vcy = (mp * vy + mt * e.tv[1]) / M,
               vcz = (mp * vz + mt * e.tv[2]) / M;
  double Ee = 0.5 * mu * (rx * rx + ry * ry + rz * rz) - e.Eth * qe;
  if (Ee < 0.0) Ee = 0.0;
  for (int a = 0; a < e.nby && a < 4; ++a) {
    const int B = e.by[a];
    if (B < 0) continue;
    double nx, ny, nz;
    if (e.rt == 4) {
      if (B != e.P) continue;
      nx = e.tv[0];
      ny = e.tv[1];
      nz = e.tv[2];
    } else {
      const double mb = fabs(set.mass[B]);
      const double vp = sqrt(2.0 * (Ee / e.sum_mass) / (mb * mb));
      nx = vcx + vp * e.e1[a][0];
      ny = vcy + vp * e.e1[a][1];
      nz = vcz + vp * e.e1[a][2];
    }
    const WinS<R> Bs = set.S[B];
    long long j = e.slot[a];
    if (j < 0) {
      j = i;
    } else {
      const long long cb = Bs.cap;
      Bs.cell[j] = A.cell[i];
      Bs.p[j] = A.p[i];
      Bs.p[cb + j] = A.p[ca + i];
      Bs.p[2 * cb + j] = A.p[2 * ca + i];
      Bs.bl[j] = (e.step & 0xffff) | (WALIVE << 16);
      atomicMax(set.count[B], (int)j + 1);
    }
    const long long cb = Bs.cap;
    Bs.p[3 * cb + j] = (R)nx;
    Bs.p[4 * cb + j] = (R)ny;
    Bs.p[5 * cb + j] = (R)nz;
  }
}

// adjoint of the recorded collisions of one step, then the collisions undone
// (the incident's velocity before them back in its slot): the byproducts'
// dJ/dv through v_b = v_cm + vp_b e1_b (v_cm = (m_p v + m_t v_t)/(m_p + m_t),
// vp_b from the centre-of-mass energy of v - v_t), the products' dJ/dx onto
// the incident's position (they were created there), charge exchange
// (v = v_t) passing nothing back
template <class R>
__global__ void __launch_bounds__(AB) k_cw_adj_collide(const lepic_win_event_t *ev, int ne, CwSet<R> set,
                                                       double qe) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= ne) return;
  const lepic_win_event_t &e = ev[k];
  const WinS<R> A = set.S[e.P];
  const long long i = e.i, ca = A.cap;
  const double vx = e.vold[0], vy = e.vold[1], vz = e.vold[2];
  const double mp = fabs(set.mass[e.P]), mt = e.m_t, M = mp + mt, mu = mp * mt / M;
  const double rx = vx - e.tv[0], ry = vy - e.tv[1], rz = vz - e.tv[2];
  double Ee = 0.5 * mu * (rx * rx + ry * ry + rz * rz) - e.Eth * qe;
  const bool pos = Ee > 0.0;
  if (!pos) Ee = 0.0;
  double gx = 0.0, gy = 0.0, gz = 0.0;   // dJ/dv before
  double px = 0.0, py = 0.0, pz = 0.0;   // dJ/dx from the products
  for (int a = 0; a < e.nby && a < 4; ++a) {
    const int B = e.by[a];
    if (B < 0) continue;
    if (e.rt == 4 && B != e.P) continue;
    const WinS<R> Bs = set.S[B];
    const long long j = e.slot[a] < 0 ? i : e.slot[a], cb = Bs.cap;
    const double lx = Bs.lam[3 * cb + j], ly = Bs.lam[4 * cb + j], lz = Bs.lam[5 * cb + j];
    if (e.slot[a] >= 0) {
      px += Bs.lam[j];
      py += Bs.lam[cb + j];
      pz += Bs.lam[2 * cb + j];
      for (int q = 0; q < 6; ++q) Bs.lam[q * cb + j] = R(0);
    }
    if (e.rt == 4) continue;
    const double mb = fabs(set.mass[B]);
    const double vp = sqrt(2.0 * (Ee / e.sum_mass) / (mb * mb));
    gx += (mp / M) * lx;
    gy += (mp / M) * ly;
    gz += (mp / M) * lz;
    if (pos && vp > 0.0) {
      const double el = e.e1[a][0] * lx + e.e1[a][1] * ly + e.e1[a][2] * lz;
      const double s = el * mu / (vp * e.sum_mass * mb * mb);
      gx += s * rx;
      gy += s * ry;
      gz += s * rz;
    }
  }
  A.lam[i] += (R)px;
  A.lam[ca + i] += (R)py;
  A.lam[2 * ca + i] += (R)pz;
  A.lam[3 * ca + i] = (R)gx;
  A.lam[4 * ca + i] = (R)gy;
  A.lam[5 * ca + i] = (R)gz;
  A.p[3 * ca + i] = (R)vx;
  A.p[4 * ca + i] = (R)vy;
  A.p[5 * ca + i] = (R)vz;
}

}  // namespace

}  // namespace lepic

using lepic::Dims;

extern "C" {

int lepic_dev_win_push(const lepic_grid_t *g, const double *Ei, double *p, int cap, int n, signed char *alive,
                       int ptype, const lepic_phys_t *P, void *stream) {
  if (!g || !Ei || !p || !alive || !P || ptype < 1 || n < 0 || n > cap) return LEPIC_ERR_ARG;
  // the window differentiates a uniform B (dJ/dBz): no B-field map
  if (P->flag_pbc || P->flag_nmn || (P->flag_B == 1 && P->Bmap)) return LEPIC_ERR_UNSUPPORTED;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return LEPIC_OK;
  int tm = lepic::timer_start("win_push_f64", s);
  lepic::k_win_push<<<lepic::grid_for(n, lepic::AB), lepic::AB, 0, s>>>(d, lepic::win_const(*g, *P, ptype), Ei,
                                                                          g->cell_wall, p, cap, n, alive);
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_win_deposit(const lepic_grid_t *g, const double *p, int cap, int n, const signed char *alive,
                          int ptype, const lepic_phys_t *P, double *np, void *stream) {
  if (!g || !p || !alive || !P || !np || ptype < 1 || n < 0 || n > cap) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return LEPIC_OK;
  int tm = lepic::timer_start("win_deposit_f64", s);
  lepic::k_win_deposit<<<lepic::grid_for(n, lepic::AB), lepic::AB, 0, s>>>(
      d, lepic::win_const(*g, *P, ptype), p, cap, n, alive, g->kq, np, lepic::ctx().d_err);
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return lepic::check_err(s);
}

int lepic_dev_adj_push(const lepic_grid_t *g, const double *Ei, const double *p, int cap, int n,
                       const signed char *alive_before, const signed char *alive_after, double *lam, int lcap,
                       int ptype, const lepic_phys_t *P, double *lE, double *dBz, void *stream) {
  if (!g || !Ei || !p || !alive_before || !alive_after || !lam || !P || !lE || !dBz || ptype < 1 || n < 0 ||
      n > cap || n > lcap)
    return LEPIC_ERR_ARG;
  if (P->flag_B == 1 && P->Bmap) return LEPIC_ERR_UNSUPPORTED;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return LEPIC_OK;
  int tm = lepic::timer_start("adj_push_f64", s);
  lepic::k_adj_push<<<lepic::grid_for(n, lepic::AB), lepic::AB, 0, s>>>(
      d, lepic::win_const(*g, *P, ptype), Ei, p, cap, n, alive_before, alive_after, lam, lcap, lE, dBz);
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_adj_deposit(const lepic_grid_t *g, const double *p, int cap, int n, const signed char *alive,
                          const double *lnp, double *lam, int lcap, int ptype, const lepic_phys_t *P,
                          void *stream) {
  if (!g || !p || !alive || !lnp || !lam || !P || ptype < 1 || n < 0 || n > cap || n > lcap) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  if (n == 0) return LEPIC_OK;
  int tm = lepic::timer_start("adj_deposit_f64", s);
  lepic::k_adj_deposit<<<lepic::grid_for(n, lepic::AB), lepic::AB, 0, s>>>(d, lepic::win_const(*g, *P, ptype), p,
                                                                             cap, n, alive, g->kq, lnp, lam, lcap);
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_adj_efield(const lepic_grid_t *g, double *lE, double *lphi, void *stream) {
  if (!g || !lE || !lphi) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const long long nn = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 + 1);
  LEPIC_CUDA(cudaMemsetAsync(lphi, 0, sizeof(double) * d.cnt(), s));
  lepic::k_adj_efield_walls<<<lepic::grid_for(nn, 256), 256, 0, s>>>(d, g->h[0], g->h[1], g->h[2], g->bcnd, lE,
                                                                      lphi);
  lepic::k_adj_efield_plasma<<<lepic::grid_for(nn, 256), 256, 0, s>>>(d, g->h[0], g->h[1], g->h[2], g->bcnd, lE,
                                                                       lphi);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_adj_rhs(const lepic_grid_t *g, const double *lphi, double *b, void *stream) {
  if (!g || !lphi || !b) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  lepic::k_adj_rhs<<<lepic::grid_for(d.rcnt(), 256), 256, 0, s>>>(d, g->bcnd, lphi, b);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_deposit(const lepic_grid_t *g, const lepic_win_species_t *ws, int ptype, const lepic_phys_t *P,
                         int step, double *np, void *stream) {
  if (!g || !ws || !P || !np || ptype < 1 || ptype > LEPIC_NPART) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const lepic::WinConst c = lepic::win_const(*g, *P, ptype);
  int tm = lepic::timer_start("cw_deposit", s);
  if (ws->fp64) {
    lepic::k_cw_deposit<double><<<lepic::grid_for(ws->cap, lepic::AB), lepic::AB, 0, s>>>(
        d, c, lepic::win_view<double>(*ws), ws->count, 0, step, g->kq, np);
  } else {
    long long first = 0;
    if (ws->tile_off) {
      const lepic::WinTiles T = lepic::win_tiles(*g, *ws);
      lepic::k_cw_deposit_tiles<<<LEPIC_TILES(g->n), lepic::AB, 0, s>>>(d, c, lepic::win_view<float>(*ws), ws->count,
                                                                         T, step, g->kq, np);
      first = ws->tile_end;
    }
    lepic::k_cw_deposit<float><<<lepic::grid_for(ws->cap - first, lepic::AB), lepic::AB, 0, s>>>(
        d, c, lepic::win_view<float>(*ws), ws->count, first, step, g->kq, np);
  }
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_push(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                      const lepic_phys_t *P, int step, double *wall_acc, void *stream) {
  if (!g || !E || !ws || !P || !wall_acc || ptype < 1 || ptype > LEPIC_NPART || !g->cell_wall) return LEPIC_ERR_ARG;
  if (P->flag_pbc || P->flag_nmn || (P->flag_B == 1 && P->Bmap)) return LEPIC_ERR_UNSUPPORTED;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const lepic::WinConst c = lepic::win_const(*g, *P, ptype);
  int tm = lepic::timer_start("cw_push", s);
  if (ws->fp64) {
    lepic::k_cw_push<double><<<lepic::grid_for(ws->cap, lepic::AB), lepic::AB, 0, s>>>(
        d, c, E, g->cell_wall, lepic::win_view<double>(*ws), ws->count, 0, step, wall_acc);
  } else {
    long long first = 0;
    if (ws->tile_off) {
      const lepic::WinTiles T = lepic::win_tiles(*g, *ws);
      lepic::k_cw_push_tiles<<<LEPIC_TILES(g->n), lepic::AB, 0, s>>>(
          d, c, (const float4 *)E, g->cell_wall, lepic::win_view<float>(*ws), ws->count, T, step, wall_acc);
      first = ws->tile_end;
    }
    lepic::k_cw_push<float><<<lepic::grid_for(ws->cap - first, lepic::AB), lepic::AB, 0, s>>>(
        d, c, E, g->cell_wall, lepic::win_view<float>(*ws), ws->count, first, step, wall_acc);
  }
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_reverse(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                         const lepic_phys_t *P, int step, void *stream) {
  if (!g || !E || !ws || !P || ptype < 1 || ptype > LEPIC_NPART) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const lepic::WinConst c = lepic::win_const(*g, *P, ptype);
  int tm = lepic::timer_start("cw_reverse", s);
  if (ws->fp64) {
    lepic::k_cw_reverse<double><<<lepic::grid_for(ws->cap, lepic::AB), lepic::AB, 0, s>>>(
        d, c, E, lepic::win_view<double>(*ws), ws->count, 0, step);
  } else {
    long long first = 0;
    if (ws->tile_off) {
      const lepic::WinTiles T = lepic::win_tiles(*g, *ws);
      lepic::k_cw_reverse_tiles<<<LEPIC_TILES(g->n), lepic::AB, 0, s>>>(d, c, (const float4 *)E,
                                                                         lepic::win_view<float>(*ws), ws->count, T,
                                                                         step);
      first = ws->tile_end;
    }
    lepic::k_cw_reverse<float><<<lepic::grid_for(ws->cap - first, lepic::AB), lepic::AB, 0, s>>>(
        d, c, E, lepic::win_view<float>(*ws), ws->count, first, step);
  }
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_adj_push(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                          const lepic_phys_t *P, int step, double wflux, double *lE, double *dBz, void *stream) {
  if (!g || !E || !ws || !P || !lE || !dBz || ptype < 1 || ptype > LEPIC_NPART) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const lepic::WinConst c = lepic::win_const(*g, *P, ptype);
  int tm = lepic::timer_start("cw_adj_push", s);
  if (ws->fp64) {
    lepic::k_cw_adj_push<double><<<lepic::grid_for(ws->cap, lepic::AB), lepic::AB, 0, s>>>(
        d, c, E, lepic::win_view<double>(*ws), ws->count, 0, step, wflux, lE, dBz);
  } else {
    long long first = 0;
    if (ws->tile_off) {
      const lepic::WinTiles T = lepic::win_tiles(*g, *ws);
      cudaFuncSetAttribute(lepic::k_cw_adj_push_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           lepic::CW_ADJ_SMEM);
      lepic::k_cw_adj_push_tiles<<<LEPIC_TILES(g->n), lepic::AB, lepic::CW_ADJ_SMEM, s>>>(
          d, c, (const float4 *)E, lepic::win_view<float>(*ws), ws->count, T, step, wflux, lE, dBz);
      first = ws->tile_end;
    }
    lepic::k_cw_adj_push<float><<<lepic::grid_for(ws->cap - first, lepic::AB), lepic::AB, 0, s>>>(
        d, c, E, lepic::win_view<float>(*ws), ws->count, first, step, wflux, lE, dBz);
  }
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_back(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype, const lepic_phys_t *P,
                      int step, const double *mu, double wflux, double *lE, double *dBz, void *stream) {
  if (!g || !E || !ws || !P || !lE || !dBz || ptype < 1 || ptype > LEPIC_NPART) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const lepic::WinConst c = lepic::win_const(*g, *P, ptype);
  int tm = lepic::timer_start("cw_back", s);
  if (ws->fp64) {
    const lepic::WinS<double> S = lepic::win_view<double>(*ws);
    const int gb = lepic::grid_for(ws->cap, lepic::AB);
    if (mu) lepic::k_cw_adj_deposit<double><<<gb, lepic::AB, 0, s>>>(d, c, S, ws->count, 0, step + 1, g->kq, mu);
    lepic::k_cw_reverse<double><<<gb, lepic::AB, 0, s>>>(d, c, E, S, ws->count, 0, step);
    lepic::k_cw_adj_push<double><<<gb, lepic::AB, 0, s>>>(d, c, E, S, ws->count, 0, step, wflux, lE, dBz);
  } else {
    const lepic::WinS<float> S = lepic::win_view<float>(*ws);
    long long first = 0;
    if (ws->tile_off) {
      const lepic::WinTiles T = lepic::win_tiles(*g, *ws);
      cudaFuncSetAttribute(lepic::k_cw_back_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, lepic::CW_BACK_SMEM);
      lepic::k_cw_back_tiles<<<LEPIC_TILES(g->n), lepic::AB, lepic::CW_BACK_SMEM, s>>>(
          d, c, (const float4 *)E, S, ws->count, T, step, g->kq, mu, wflux, lE, dBz);
      first = ws->tile_end;
    }
    const int gb = lepic::grid_for(ws->cap - first, lepic::AB);
    if (mu) lepic::k_cw_adj_deposit<float><<<gb, lepic::AB, 0, s>>>(d, c, S, ws->count, first, step + 1, g->kq, mu);
    lepic::k_cw_reverse<float><<<gb, lepic::AB, 0, s>>>(d, c, E, S, ws->count, first, step);
    lepic::k_cw_adj_push<float><<<gb, lepic::AB, 0, s>>>(d, c, E, S, ws->count, first, step, wflux, lE, dBz);
  }
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_adj_deposit(const lepic_grid_t *g, lepic_win_species_t *ws, int ptype, const lepic_phys_t *P,
                             int step, const double *mu, void *stream) {
  if (!g || !ws || !P || !mu || ptype < 1 || ptype > LEPIC_NPART) return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const lepic::WinConst c = lepic::win_const(*g, *P, ptype);
  int tm = lepic::timer_start("cw_adj_deposit", s);
  if (ws->fp64) {
    lepic::k_cw_adj_deposit<double><<<lepic::grid_for(ws->cap, lepic::AB), lepic::AB, 0, s>>>(
        d, c, lepic::win_view<double>(*ws), ws->count, 0, step, g->kq, mu);
  } else {
    long long first = 0;
    if (ws->tile_off) {
      const lepic::WinTiles T = lepic::win_tiles(*g, *ws);
      lepic::k_cw_adj_deposit_tiles<<<LEPIC_TILES(g->n), lepic::AB, 0, s>>>(d, c, lepic::win_view<float>(*ws),
                                                                             ws->count, T, step, g->kq, mu);
      first = ws->tile_end;
    }
    lepic::k_cw_adj_deposit<float><<<lepic::grid_for(ws->cap - first, lepic::AB), lepic::AB, 0, s>>>(
        d, c, lepic::win_view<float>(*ws), ws->count, first, step, g->kq, mu);
  }
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

extern "C++" {
template <class R>
static lepic::CwSet<R> cw_set(lepic_win_species_t *ws, int ntype, const lepic_phys_t &P) {
  lepic::CwSet<R> set;
  memset(&set, 0, sizeof(set));
  for (int p = 0; p < ntype; ++p) {
    set.S[p] = lepic::win_view<R>(ws[p]);
    set.count[p] = ws[p].count;
  }
  for (int p = 0; p < LEPIC_NPART; ++p) set.mass[p] = P.mass[p];
  return set;
}

static bool cw_uniform(const lepic_win_species_t *ws, int ntype) {
  for (int p = 1; p < ntype; ++p)
    if (ws[p].fp64 != ws[0].fp64) return false;
  return true;
}
}  // extern "C++"

int lepic_dev_cw_replay(const lepic_grid_t *g, lepic_win_species_t *ws, int ntype, const lepic_phys_t *P,
                        lepic_win_event_t *events, int ne, void *stream) {
  if (!g || !ws || !P || ntype < 1 || ntype > LEPIC_NPART || ne < 0 || (ne > 0 && !events) ||
      !cw_uniform(ws, ntype))
    return LEPIC_ERR_ARG;
  if (ne == 0) return LEPIC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  if (ws[0].fp64)
    lepic::k_cw_replay<double><<<lepic::grid_for(ne, lepic::AB), lepic::AB, 0, s>>>(
        events, ne, cw_set<double>(ws, ntype, *P), P->qe);
  else
    lepic::k_cw_replay<float><<<lepic::grid_for(ne, lepic::AB), lepic::AB, 0, s>>>(
        events, ne, cw_set<float>(ws, ntype, *P), P->qe);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_cw_adj_collide(const lepic_grid_t *g, lepic_win_species_t *ws, int ntype, const lepic_phys_t *P,
                             const lepic_win_event_t *events, int ne, void *stream) {
  if (!g || !ws || !P || ntype < 1 || ntype > LEPIC_NPART || ne < 0 || (ne > 0 && !events) ||
      !cw_uniform(ws, ntype))
    return LEPIC_ERR_ARG;
  if (ne == 0) return LEPIC_OK;
  cudaStream_t s = (cudaStream_t)stream;
  int tm = lepic::timer_start("cw_adj_collide", s);
  if (ws[0].fp64)
    lepic::k_cw_adj_collide<double><<<lepic::grid_for(ne, lepic::AB), lepic::AB, 0, s>>>(
        events, ne, cw_set<double>(ws, ntype, *P), P->qe);
  else
    lepic::k_cw_adj_collide<float><<<lepic::grid_for(ne, lepic::AB), lepic::AB, 0, s>>>(
        events, ne, cw_set<float>(ws, ntype, *P), P->qe);
  lepic::timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_adj_walls(const lepic_grid_t *g, const lepic_phys_t *P, int ptype, const double *lphi,
                        const double *mu, double *lnp, double *dV, int nlabel, void *stream) {
  if (!g || !P || !lphi || !mu || !lnp || !dV || ptype < 1 || nlabel < 0 || nlabel > lepic::MAX_LABEL)
    return LEPIC_ERR_ARG;
  const Dims d(g->n);
  cudaStream_t s = (cudaStream_t)stream;
  const double aw = P->eps0 / (g->h[0] * g->h[0]), an = P->eps0 / (g->h[1] * g->h[1]),
               at = P->eps0 / (g->h[2] * g->h[2]);
  lepic::k_adj_walls<<<lepic::grid_for(d.cnt(), lepic::AB), lepic::AB, 0, s>>>(
      d, aw, an, at, P->charge[ptype - 1], g->bcnd, lphi, mu, lnp, dV, nlabel);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

}  // extern "C"
