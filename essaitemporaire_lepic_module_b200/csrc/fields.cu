// Grid kernels: rho reduction (Src/calc_rho.f90), density reduction
// (dens_red), E = -grad(phi) (Src/Efield.f90) and the per-cell wall mask of
// the particle loss test (Src/part_expmover.f90:250-272).
//
// Compiled with --fmad=false: every expression is evaluated in the order the
// Fortran writes it, so node values match the strict-IEEE CPU oracle bit for
// bit.  Grids are the reference's column-major node arrays; HBM traffic is
// one coalesced pass over each array (x fastest, one thread per node).
#include "lepic_internal.cuh"

namespace lepic {

// Periodic stitching of np, y planes then z planes (Src/calc_rho.f90:29-68).
__global__ void k_rho_pbc_y(Dims d, double *np, const int *bcnd, int ntype) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long nx = d.n1 + 1, nz = d.n3 + 1;
  if (t >= nx * nz * ntype) return;
  int ix = 1 + (int)(t % nx);
  int iz = 1 + (int)((t / nx) % nz);
  int p = (int)(t / (nx * nz));
  double *g = np + (long long)p * d.cnt();
  const int n2 = d.n2;
  if (bcnd[d.g(ix, 1, iz)] == 0) {
    g[d.g(ix, 1, iz)] = 0.5 * (g[d.g(ix, 1, iz)] + g[d.g(ix, n2 + 1, iz)]);
    g[d.g(ix, 0, iz)] = g[d.g(ix, n2, iz)];
  }
  if (bcnd[d.g(ix, n2 + 1, iz)] == 0) {
    g[d.g(ix, n2 + 2, iz)] = g[d.g(ix, 2, iz)];
    g[d.g(ix, n2 + 1, iz)] = g[d.g(ix, 1, iz)];
  }
}

__global__ void k_rho_pbc_z(Dims d, double *np, const int *bcnd, int ntype) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long nx = d.n1 + 1, ny = d.n2 + 1;
  if (t >= nx * ny * ntype) return;
  int ix = 1 + (int)(t % nx);
  int iy = 1 + (int)((t / nx) % ny);
  int p = (int)(t / (nx * ny));
  double *g = np + (long long)p * d.cnt();
  const int n3 = d.n3;
  if (bcnd[d.g(ix, iy, 1)] == 0) {
    g[d.g(ix, iy, 1)] = 0.5 * (g[d.g(ix, iy, 1)] + g[d.g(ix, iy, n3 + 1)]);
    g[d.g(ix, iy, 0)] = g[d.g(ix, iy, n3)];
  }
  if (bcnd[d.g(ix, iy, n3 + 1)] == 0) {
    g[d.g(ix, iy, n3 + 2)] = g[d.g(ix, iy, 2)];
    g[d.g(ix, iy, n3 + 1)] = g[d.g(ix, iy, 1)];
  }
}

struct Charges {
  double q[LEPIC_NPART];
};

// rhs = -sum_p charge(p) np_p over nodes 1..n+1, zero elsewhere
// (Src/calc_rho.f90:73-90).
__global__ void k_calc_rho(Dims d, const double *np, double *rhs, int ntype, Charges Q) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long R1 = d.N1 - 1, R2 = d.N2 - 1;
  if (t >= d.rcnt()) return;
  int ix = (int)(t % R1);
  int iy = (int)((t / R1) % R2);
  int iz = (int)(t / (R1 * R2));
  double acc = 0.0;
  if (ix >= 1 && iy >= 1 && iz >= 1) {
    long long q = d.g(ix, iy, iz);
    for (int p = 0; p < ntype; ++p) acc = acc - Q.q[p] * np[(long long)p * d.cnt() + q];
  }
  rhs[t] = acc;
}

int launch_calc_rho(const Dims &d, double *np, double *rhs, const int *bcnd, int ntype,
                    const lepic_phys_t &P, cudaStream_t s) {
  if (P.flag_pbc == 1) {
    long long n1 = (long long)(d.n1 + 1) * (d.n3 + 1) * ntype;
    k_rho_pbc_y<<<grid_for(n1, 256), 256, 0, s>>>(d, np, bcnd, ntype);
    long long n2 = (long long)(d.n1 + 1) * (d.n2 + 1) * ntype;
    k_rho_pbc_z<<<grid_for(n2, 256), 256, 0, s>>>(d, np, bcnd, ntype);
  }
  Charges Q;
  for (int p = 0; p < LEPIC_NPART; ++p) Q.q[p] = P.charge[p];
  int tm = timer_start("calc_rho_f64", s);
  k_calc_rho<<<grid_for(d.rcnt(), 256), 256, 0, s>>>(d, np, rhs, ntype, Q);
  timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

// np_red = np over nodes 1..n+1 (one thread slice) and the per-species max
// over plasma nodes (Src/calc_rho.f90:116-186).  Max of non-negative doubles
// is taken on their bit patterns, which order like the values.
__global__ void k_dens_red(Dims d, const double *np, double *np_red, const int *bcnd, int ntype,
                           unsigned long long *mx) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= d.cnt() * ntype) return;
  int p = (int)(t / d.cnt());
  long long q = t % d.cnt();
  int ix = (int)(q % d.N1), iy = (int)((q / d.N1) % d.N2), iz = (int)(q / (d.N1 * d.N2));
  double v = 0.0;
  if (ix >= 1 && ix <= d.n1 + 1 && iy >= 1 && iy <= d.n2 + 1 && iz >= 1 && iz <= d.n3 + 1) {
    v = 0.0 + np[t];
    if (bcnd[q] == -1 && v > 0.0) atomicMax(&mx[p], (unsigned long long)__double_as_longlong(v));
  }
  if (np_red) np_red[t] = v;
}

int launch_dens_red(const Dims &d, const double *np, double *np_red, const int *bcnd, int ntype,
                    double *np_mx_host, cudaStream_t s) {
  unsigned long long *mx = (unsigned long long *)scratch("dens_red_mx", sizeof(unsigned long long) * LEPIC_NPART);
  if (!mx) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(mx, 0, sizeof(unsigned long long) * LEPIC_NPART, s));
  k_dens_red<<<grid_for(d.cnt() * ntype, 256), 256, 0, s>>>(d, np, np_red, bcnd, ntype, mx);
  LEPIC_CUDA(cudaGetLastError());
  unsigned long long h[LEPIC_NPART];
  LEPIC_CUDA(cudaMemcpyAsync(h, mx, sizeof(h), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  for (int p = 0; p < ntype; ++p) {
    double v;
    memcpy(&v, &h[p], sizeof(double));
    np_mx_host[p] = v;
  }
  return LEPIC_OK;
}

// ------------------------------------------------------------- E field
// Pass 1: central differences on nodes with bcnd <= 0 (Src/Efield.f90:18-42).
__global__ void k_efield_interior(Dims d, double hx, double hy, double hz, const double *phi,
                                  double *Ei, const int *bcnd) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long nx = d.n1 + 1, ny = d.n2 + 1, nz = d.n3 + 1;
  if (t >= nx * ny * nz) return;
  int ix = 1 + (int)(t % nx), iy = 1 + (int)((t / nx) % ny), iz = 1 + (int)(t / (nx * ny));
  long long q = d.g(ix, iy, iz);
  if (bcnd[q] > 0) return;
  const long long sy = d.N1, sz = d.N1 * d.N2;
  Ei[3 * q + 0] = -(phi[q + 1] - phi[q - 1]) / (2.0 * hx);
  Ei[3 * q + 1] = -(phi[q + sy] - phi[q - sy]) / (2.0 * hy);
  Ei[3 * q + 2] = -(phi[q + sz] - phi[q - sz]) / (2.0 * hz);
}

// Pass 2: every non-plasma node's own values -- Neumann plane, periodic
// planes (values at iy = 1 / iz = 1) and wall extrapolation
// (Src/Efield.f90:47-187).  Reads only pass-1 values of its neighbours.
__global__ void k_efield_boundary(Dims d, double hx, double hy, double hz, const double *phi,
                                  double *Ei, const int *bcnd) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long nx = d.n1 + 1, ny = d.n2 + 1, nz = d.n3 + 1;
  if (t >= nx * ny * nz) return;
  int ix = 1 + (int)(t % nx), iy = 1 + (int)((t / nx) % ny), iz = 1 + (int)(t / (nx * ny));
  long long q = d.g(ix, iy, iz);
  int bc = bcnd[q];
  if (bc == -1) return;
  const long long sy = d.N1, sz = d.N1 * d.N2;
  const int n2 = d.n2, n3 = d.n3;
  if (bc == -2) {
    Ei[3 * d.g(1, iy, iz) + 0] = 0.0;
    if (iy > 1 && iy < n2 + 1 && iz > 1 && iz < n3 + 1) {
      Ei[3 * d.g(1, iy, iz) + 1] = -(phi[d.g(1, iy + 1, iz)] - phi[d.g(1, iy - 1, iz)]) / (2.0 * hy);
      Ei[3 * d.g(1, iy, iz) + 2] = -(phi[d.g(1, iy, iz + 1)] - phi[d.g(1, iy, iz - 1)]) / (2.0 * hz);
      return;
    }
  }
  if (bc == 0 || bc == -2) {
    if (iy == 1) Ei[3 * q + 1] = -(phi[d.g(ix, 2, iz)] - phi[d.g(ix, n2, iz)]) / (2.0 * hy);
    if (iz == 1) Ei[3 * q + 2] = -(phi[d.g(ix, iy, 2)] - phi[d.g(ix, iy, n3)]) / (2.0 * hz);
    return;
  }
  double ex = Ei[3 * q + 0], ey = Ei[3 * q + 1], ez = Ei[3 * q + 2];
  const double cx = -(phi[q + 1] - phi[q - 1]) / (2.0 * hx);
  const double cy = -(phi[q + sy] - phi[q - sy]) / (2.0 * hy);
  const double cz = -(phi[q + sz] - phi[q - sz]) / (2.0 * hz);
  // The extrapolation reads two nodes deep; nodes whose second neighbour
  // would leave the array keep their value (the reference reads past it).
  const bool xp2 = ix + 2 <= d.n1 + 2, xm2 = ix - 2 >= 0;
  const bool yp2 = iy + 2 <= d.n2 + 2, ym2 = iy - 2 >= 0;
  const bool zp2 = iz + 2 <= d.n3 + 2, zm2 = iz - 2 >= 0;
  if (bcnd[q + 1] <= 0 && xp2) {
    ex = 2.0 * Ei[3 * (q + 1)] - Ei[3 * (q + 2)];
    ey = cy;
    ez = cz;
  }
  if (bcnd[q - 1] <= 0 && xm2) {
    ex = 2.0 * Ei[3 * (q - 1)] - Ei[3 * (q - 2)];
    ey = cy;
    ez = cz;
  }
  if (bcnd[q + sy] <= 0 && yp2) {
    ex = cx;
    ey = 2.0 * Ei[3 * (q + sy) + 1] - Ei[3 * (q + 2 * sy) + 1];
    ez = cz;
  }
  if (bcnd[q - sy] <= 0 && ym2) {
    ex = cx;
    ey = 2.0 * Ei[3 * (q - sy) + 1] - Ei[3 * (q - 2 * sy) + 1];
    ez = cz;
  }
  if (bcnd[q + sz] <= 0 && zp2) {
    ex = cx;
    ey = cy;
    ez = 2.0 * Ei[3 * (q + sz) + 2] - Ei[3 * (q + 2 * sz) + 2];
  }
  if (bcnd[q - sz] <= 0 && zm2) {
    ex = cx;
    ey = cy;
    ez = 2.0 * Ei[3 * (q - sz) + 2] - Ei[3 * (q - 2 * sz) + 2];
  }
  Ei[3 * q + 0] = ex;
  Ei[3 * q + 1] = ey;
  Ei[3 * q + 2] = ez;
}

// Pass 3: periodic copies into the n+1 planes and the ghost planes
// (Src/Efield.f90:72-99), reading pass-2 values.
__global__ void k_efield_pbc_copy(Dims d, double *Ei, const int *bcnd) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long nx = d.n1 + 1, ny = d.n2 + 1, nz = d.n3 + 1;
  if (t >= nx * ny * nz) return;
  int ix = 1 + (int)(t % nx), iy = 1 + (int)((t / nx) % ny), iz = 1 + (int)(t / (nx * ny));
  int bc = bcnd[d.g(ix, iy, iz)];
  if (!(bc == 0 || bc == -2)) return;
  if (bc == -2 && iy > 1 && iy < d.n2 + 1 && iz > 1 && iz < d.n3 + 1) return;
  const int n2 = d.n2, n3 = d.n3;
  auto E = [&](int c, int a, int b, int e) -> double & { return Ei[3 * d.g(a, b, e) + c]; };
  if (iy == 1) {
    E(1, ix, 0, iz) = E(1, ix, n2, iz);
    E(1, ix, n2 + 1, iz) = E(1, ix, 1, iz);
    E(1, ix, n2 + 2, iz) = E(1, ix, 2, iz);
    E(0, ix, 0, iz) = E(0, ix, n2, iz);
    E(0, ix, n2 + 2, iz) = E(0, ix, 2, iz);
    E(2, ix, 0, iz) = E(2, ix, n2, iz);
    E(2, ix, n2 + 2, iz) = E(2, ix, 2, iz);
  }
  if (iz == 1) {
    E(2, ix, iy, 0) = E(2, ix, iy, n3);
    E(2, ix, iy, n3 + 1) = E(2, ix, iy, 1);
    E(2, ix, iy, n3 + 2) = E(2, ix, iy, 2);
    E(0, ix, iy, 0) = E(0, ix, iy, n3);
    E(0, ix, iy, n3 + 2) = E(0, ix, iy, 2);
    E(1, ix, iy, 0) = E(1, ix, iy, n3);
    E(1, ix, iy, n3 + 2) = E(1, ix, iy, 2);
  }
}

int launch_efield(const Dims &d, const double h[3], const double *phi, double *Ei, const int *bcnd,
                  cudaStream_t s) {
  long long nn = (long long)(d.n1 + 1) * (d.n2 + 1) * (d.n3 + 1);
  int tm = timer_start("efield_f64", s);
  k_efield_interior<<<grid_for(nn, 256), 256, 0, s>>>(d, h[0], h[1], h[2], phi, Ei, bcnd);
  k_efield_boundary<<<grid_for(nn, 256), 256, 0, s>>>(d, h[0], h[1], h[2], phi, Ei, bcnd);
  k_efield_pbc_copy<<<grid_for(nn, 256), 256, 0, s>>>(d, Ei, bcnd);
  timer_stop(tm, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

// cell_wall(ix,iy,iz) for ix in 0..n1+1: all 8 nodes of the cell are walls
// (bcnd >= 1), the loss test of Src/part_expmover.f90:258-262 and the load
// rejection of Src/load_part.f90:147-151.
__global__ void k_cell_wall(Dims d, const int *bcnd, unsigned char *cw) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long C1 = d.N1 - 1, C2 = d.N2 - 1, C3 = d.N3 - 1;
  if (t >= C1 * C2 * C3) return;
  int ix = (int)(t % C1), iy = (int)((t / C1) % C2), iz = (int)(t / (C1 * C2));
  const long long sy = d.N1, sz = d.N1 * d.N2;
  long long q = d.g(ix, iy, iz);
  bool w = bcnd[q] >= 1 && bcnd[q + 1] >= 1 && bcnd[q + 1 + sy] >= 1 && bcnd[q + sy] >= 1 &&
           bcnd[q + sz] >= 1 && bcnd[q + 1 + sz] >= 1 && bcnd[q + 1 + sy + sz] >= 1 &&
           bcnd[q + sy + sz] >= 1;
  cw[t] = w ? 1 : 0;
}

// Src/main.f90:859-949 (one rank, one thread slice): the potential of the
// dielectric walls' nodes rises by the surface charge over the capacitance
// per cell Ca, species by species in ptype order: Q/(2 Ca) on Y = const
// planes (sum_q_xz), Q/Ca on X = const planes (sum_q_yz).  With periodic z
// planes the sums of rows 1 and n3+1 count twice, row 0 reads twice row n3
// and row n3+2 twice row 2 (the boundary cell collects half the charge).
__global__ void k_dielectric_phi(Dims d, double *phi, const int *__restrict__ bcnd,
                                 const int *__restrict__ dtype, int ngrid, const double *__restrict__ qxz,
                                 const double *__restrict__ qyz, int ntype, double Ca, int pbc) {
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= d.cnt()) return;
  const int igrid = bcnd[t];
  if (igrid <= 0 || igrid > ngrid) return;
  const int dt = dtype[igrid];
  if (dt < 2 || dt > 4) return;
  const int ix = (int)(t % d.N1), iy = (int)((t / d.N1) % d.N2), iz = (int)(t / (d.N1 * d.N2));
  int jz = iz;
  bool twice = false;
  if (pbc == 1) {
    twice = true;
    if (iz == 0)
      jz = d.n3;
    else if (iz == d.n3 + 2)
      jz = 2;
    else if (iz != 1 && iz != d.n3 + 1)
      twice = false;
  }
  const long long nxz = d.N1 * d.N3, nyz = 2 * d.N2 * d.N3;
  double v = phi[t];
  for (int p = 0; p < ntype; ++p) {
    if (dt == 2) {
      const double q = qxz[p * nxz + ix + d.N1 * jz];
      v = v + (twice ? 2.0 * q : q) / (2.0 * Ca);
    } else {
      const double q = qyz[p * nyz + (dt - 3) + 2 * (iy + d.N2 * jz)];
      v = v + (twice ? 2.0 * q : q) / Ca;
    }
  }
  phi[t] = v;
}

int launch_dielectric_phi(const Dims &d, double *phi, const int *bcnd, const lepic_phys_t &P, int ngrid,
                          double Ca, cudaStream_t s) {
  if (!P.dtype || !P.sum_q_xz || !P.sum_q_yz || !(Ca > 0.0) || d.n3 < 2) return LEPIC_ERR_ARG;
  k_dielectric_phi<<<grid_for(d.cnt(), 256), 256, 0, s>>>(d, phi, bcnd, P.dtype, ngrid, P.sum_q_xz,
                                                          P.sum_q_yz, P.ntype, Ca, P.flag_pbc);
  LEPIC_CUDA(cudaGetLastError());
  // Src/main.f90:912-914: the counters restart from zero
  LEPIC_CUDA(cudaMemsetAsync(P.sum_q_xz, 0, sizeof(double) * P.ntype * d.N1 * d.N3, s));
  LEPIC_CUDA(cudaMemsetAsync(P.sum_q_yz, 0, sizeof(double) * P.ntype * 2 * d.N2 * d.N3, s));
  return LEPIC_OK;
}

int launch_cell_wall(const Dims &d, const int *bcnd, unsigned char *cw, cudaStream_t s) {
  long long nc = (d.N1 - 1) * (d.N2 - 1) * (d.N3 - 1);
  k_cell_wall<<<grid_for(nc, 256), 256, 0, s>>>(d, bcnd, cw);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

}  // namespace lepic
