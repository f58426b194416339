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

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int AB = 256;
constexpr int MAX_LABEL = 16;

struct WinConst {
  double h0, h1, h2, dt, k1, kk, Bx, By, Bz, kdep, q, mass;
  double dkk;       // d kk / d Bz
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

__device__ __forceinline__ unsigned lanemask_le() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

// Sum of v over each run of consecutive lanes with the same key: afterwards
// the first lane of a run (head) holds the run's totals.  Lanes with key -1
// contribute zeros.  All 32 lanes must call this.  The window's particles are
// sorted by cell, so a warp holds few runs and the atomics that follow are
// one per run instead of one per particle.
template <int NV>
__device__ __forceinline__ bool warp_run_sum(long long key, double (&v)[NV]) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long prev = __shfl_up_sync(full, key, 1);
  const bool head = (lane == 0) || prev != key;
  const unsigned heads = __ballot_sync(full, head);
  const int rid = __popc(heads & lanemask_le());
  const unsigned above = heads & ~(0xffffffffu >> (31 - lane));
  const int len = head ? ((above ? __ffs(above) - 1 : 32) - lane) : 0;
  const int maxlen = (int)__reduce_max_sync(full, (unsigned)len);
  for (int o = 1; o < maxlen; o <<= 1) {
    const int orid = __shfl_down_sync(full, rid, o);
    const bool same = (lane + o < 32) && orid == rid;
#pragma unroll
    for (int c = 0; c < NV; ++c) {
      const double t = __shfl_down_sync(full, v[c], o);
      if (same) v[c] += t;
    }
  }
  return head && key >= 0;
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
  return c;
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
