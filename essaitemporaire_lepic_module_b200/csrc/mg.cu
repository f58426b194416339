// Poisson solve of Src/pdesolver.f90 + Src/mg.f90 + Src/sors.f90 as ONE
// persistent cooperative kernel: every V-cycle, every level, every
// red-black sweep, the residual-ratio exit test of sor_rb and the outer
// res/alpha < eps loop run on the device; the host sees a single launch.
//
// Schedule (identical to the reference, one MPI rank):
//   for each V-cycle k: down leg sor_rb(level l, dig<0) + restriction,
//   coarsest sor_rb(dig=0) (up to 1e6 sweeps in cycle 1 until res <= eps,
//   4 afterwards) + prolongation, up leg sor_rb(dig>0) + prolongation.
//   sor_rb stops after 4 sweeps or when res/res_prev <= 0.6.
//
// Bit-exactness: node updates of one colour are independent, and every
// expression keeps the Fortran evaluation order (the file is compiled with
// --fmad=false), so the iterates equal the CPU oracle's.  The L1 residual is
// summed per block in a fixed tree and then over blocks in block order by
// every block, so all blocks take the same exit decision and the result is
// deterministic run to run.
//
// Levels with few nodes (<= SMALL_NODES) are smoothed by block 0 alone with
// __syncthreads, avoiding grid-wide barriers on the tiny coarse grids.
//
// Periodic planes in y and z (bcnd 0) and the Neumann plane at x = 0
// (bcnd -2) run in a second instance of the kernel (GEN): the node rules of
// Src/sors.f90:113-125, the ghost-plane refresh after each colour
// (Src/sors.f90:157-231) and the restriction's periodic wraps
// (Src/mg.f90:314-805); the Dirichlet instance is unchanged.
#include <cooperative_groups.h>

#include "lepic_internal.cuh"

namespace cg = cooperative_groups;

namespace lepic {

namespace {

constexpr int MG_MAX = 13;
constexpr int MG_BLOCK = 512;
constexpr long long SMALL_NODES = 20000;

struct MGLev {
  int n1, n2, n3;
  long long N1, N2;   // node extents n+3 in x, y
  long long R1, R2;   // rhs extents n+2
  double aw, ae, an, as, at, ab, ac;
  double *u;          // (n+3)^3
  double *b;          // (n+2)^3
  int *bc;            // (n+3)^3
  double *rf;         // (n+3)^3 fine residual scratch (levels that restrict)
  double *rp;         // (n1+2)(n2+2) residual plane r_pbc of the last z plane (GEN)
  __device__ long long g(int i, int j, int k) const { return i + N1 * (j + N2 * (long long)k); }
  __device__ long long r(int i, int j, int k) const { return i + R1 * (j + R2 * (long long)k); }
  __device__ long long nodes() const { return (long long)(n1 + 1) * (n2 + 1) * (n3 + 1); }
};

struct MGArgs {
  MGLev L[MG_MAX + 1];
  int ng, ncycl;
  int pbc, nmn;       // periodic planes in y and z; Neumann plane at x = 0 (GEN only)
  double alpha, eps, omega;
  double *partial;    // [gridDim.x]
  double *shared_d;   // [4]: small-level results
  int *out_i;         // [0] k, [1] status, [2..] iterations per level of last cycle
  double *out_d;      // [0] ktot, [1] res
};

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// deterministic block sum (fixed tree); result valid in all threads
__device__ double block_sum(double v, double *sh) {
  int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  int nw = blockDim.x >> 5;
  double t = (threadIdx.x < nw) ? sh[threadIdx.x] : 0.0;
  if (w == 0) t = warp_sum(t);
  if (threadIdx.x == 0) sh[32] = t;
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}

// Warps that share a loop: warp gw of nw (the whole grid or block 0).
struct Warps {
  int gw, nw;
};
__device__ __forceinline__ Warps grid_warps() {
  return {(int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), (int)((gridDim.x * blockDim.x) >> 5)};
}
__device__ __forceinline__ Warps block_warps() { return {(int)(threadIdx.x >> 5), (int)(blockDim.x >> 5)}; }

// The grid rows (j, k), j in [j0, j0 + nj), k in [k0, k0 + nk), dealt
// round-robin to the warps; body(j, k) runs on all 32 lanes of the warp, which
// split the row along i (coalesced, one 32-bit division per row).
template <class F>
__device__ __forceinline__ void for_rows(const Warps &w, int j0, int nj, int k0, int nk, F &&body) {
  const int rows = nj * nk;
  for (int r = w.gw; r < rows; r += w.nw) {
    const int kk = r / nj;
    body(j0 + (r - kk * nj), k0 + kk);
  }
}

// one colour of a red-black sweep
// colour 0 = red ((i+j+k) odd), 1 = black (Src/sors.f90:87-106, 249-267).
// GEN: Neumann nodes (-2) drop the west neighbour and take the east one
// twice; periodic nodes (0) on the last y or z plane are not updated.
template <bool GEN>
__device__ __forceinline__ void sweep_colour(const MGLev &L, double omega, int colour, const Warps &w) {
  const int lane = threadIdx.x & 31;
  const long long sy = L.N1, sz = L.N1 * L.N2;
  for_rows(w, 1, L.n2 + 1, 1, L.n3 + 1, [&](int j, int k) {
    int ks = (k % 2 == 0) ? 0 : 1;
    int is;
    if (colour == 0) is = (j % 2 == 0) ? 1 : 2;
    else is = (j % 2 == 0) ? 2 : 1;
    is = is + ks;
    if (is > 2) is = 1;
    for (int i = is + 2 * lane; i <= L.n1 + 1; i += 64) {
      long long q = L.g(i, j, k);
      const int bq = L.bc[q];
      if (bq > 0) continue;
      if (GEN) {
        if (bq == -2) {
          double tt = L.b[L.r(i, j, k)] - L.an * L.u[q + sy] - L.as * L.u[q - sy] - 2.0 * L.ae * L.u[q + 1] -
                      L.at * L.u[q + sz] - L.ab * L.u[q - sz];
          L.u[q] = (1.0 - omega) * L.u[q] + omega * tt / L.ac;
          continue;
        }
        if (bq == 0 && (k == L.n3 + 1 || j == L.n2 + 1)) continue;
      }
      double tt = L.b[L.r(i, j, k)] - L.aw * L.u[q - 1] - L.an * L.u[q + sy] - L.as * L.u[q - sy] -
                  L.ae * L.u[q + 1] - L.at * L.u[q + sz] - L.ab * L.u[q - sz];
      L.u[q] = (1.0 - omega) * L.u[q] + omega * tt / L.ac;
    }
  });
}

// Periodic ghost planes (Src/sors.f90:157-231), first phase: y ghosts of
// every z plane; second phase (after a barrier): z ghosts of every y row.
// A ghost is refreshed where the node next to it is periodic or Neumann.
__device__ __forceinline__ void ghosts_y(const MGLev &L, const Warps &w) {
  const int lane = threadIdx.x & 31;
  for_rows(w, 0, 1, 0, L.n3 + 3, [&](int, int k) {
    for (int i = lane; i <= L.n1 + 2; i += 32) {
      const int b1 = L.bc[L.g(i, 1, k)], bn = L.bc[L.g(i, L.n2 + 1, k)];
      if (b1 == 0 || b1 == -2) L.u[L.g(i, 0, k)] = L.u[L.g(i, L.n2, k)];
      if (bn == 0 || bn == -2) L.u[L.g(i, L.n2 + 1, k)] = L.u[L.g(i, 1, k)];
    }
  });
}
__device__ __forceinline__ void ghosts_z(const MGLev &L, const Warps &w) {
  const int lane = threadIdx.x & 31;
  for_rows(w, 0, L.n2 + 3, 0, 1, [&](int j, int) {
    for (int i = lane; i <= L.n1 + 2; i += 32) {
      const int b1 = L.bc[L.g(i, j, 1)], bm = L.bc[L.g(i, j, L.n3 + 1)];
      if (b1 == 0 || b1 == -2) L.u[L.g(i, j, 0)] = L.u[L.g(i, j, L.n3)];
      if (bm == 0 || bm == -2) L.u[L.g(i, j, L.n3 + 1)] = L.u[L.g(i, j, 1)];
    }
  });
}

// sum of |residual| over the plasma nodes of this thread's rows
__device__ __forceinline__ double residual_part(const MGLev &L, const Warps &w) {
  const int lane = threadIdx.x & 31;
  const long long sy = L.N1, sz = L.N1 * L.N2;
  double acc = 0.0;
  for_rows(w, 1, L.n2 + 1, 1, L.n3 + 1, [&](int j, int k) {
    for (int i = 1 + lane; i <= L.n1 + 1; i += 32) {
      long long q = L.g(i, j, k);
      if (L.bc[q] != -1) continue;
      double rij = L.b[L.r(i, j, k)] - (L.aw * L.u[q - 1] + L.an * L.u[q + sy] + L.as * L.u[q - sy] +
                                        L.ae * L.u[q + 1] + L.ac * L.u[q] + L.at * L.u[q + sz] +
                                        L.ab * L.u[q - sz]);
      acc += fabs(rij);
    }
  });
  return acc;
}

// Src/sors.f90:1-535, whole grid.  Returns res, ksor (uniform in all threads).
template <bool GEN>
__device__ void sor_rb(const MGArgs &a, const MGLev &L, int kmg, int dig, double eps_abs,
                       cg::grid_group &grid, double *sh, double &res_out, int &ksor_out) {
  const bool pbc = GEN && a.pbc;
  long long nr = 4;
  if (kmg == 1 && dig == 0) nr = 1000000;
  const double eta = 0.6;
  if (L.nodes() <= SMALL_NODES) {
    if (blockIdx.x == 0) {
      double res_s = 0.0, res = 0.0;
      int ksor = 0;
      const Warps w = block_warps();
      for (long long l = 1; l <= nr; ++l) {
        for (int colour = 0; colour < 2; ++colour) {
          sweep_colour<GEN>(L, a.omega, colour, w);
          __syncthreads();
          if (pbc) {
            ghosts_y(L, w);
            __syncthreads();
            ghosts_z(L, w);
            __syncthreads();
          }
        }
        res = block_sum(residual_part(L, w), sh);
        ksor++;
        bool stop = (dig == 0) ? (res <= eps_abs) : (res_s > 0.0 && (res / res_s) <= eta);
        if (stop) break;
        res_s = res;
      }
      if (threadIdx.x == 0) {
        a.shared_d[0] = res;
        a.shared_d[1] = (double)ksor;
      }
      __threadfence();
    }
    grid.sync();
    res_out = a.shared_d[0];
    ksor_out = (int)a.shared_d[1];
    grid.sync();  // everyone has read shared_d before it is reused
    return;
  }
  const Warps w = grid_warps();
  double res_s = 0.0, res = 0.0;
  int ksor = 0;
  for (long long l = 1; l <= nr; ++l) {
    for (int colour = 0; colour < 2; ++colour) {
      sweep_colour<GEN>(L, a.omega, colour, w);
      grid.sync();
      if (pbc) {
        ghosts_y(L, w);
        grid.sync();
        ghosts_z(L, w);
        grid.sync();
      }
    }
    double part = block_sum(residual_part(L, w), sh);
    if (threadIdx.x == 0) a.partial[blockIdx.x] = part;
    grid.sync();
    // every block sums the partials in the same fixed order
    double v = 0.0;
    if (threadIdx.x < 32) {
      for (int bI = threadIdx.x; bI < (int)gridDim.x; bI += 32) v += a.partial[bI];
      v = warp_sum(v);
      if (threadIdx.x == 0) sh[33] = v;
    }
    __syncthreads();
    res = sh[33];
    __syncthreads();
    ksor++;
    bool stop = (dig == 0) ? (res <= eps_abs) : (res_s > 0.0 && (res / res_s) <= eta);
    if (stop) break;
    res_s = res;
  }
  res_out = res;
  ksor_out = ksor;
}

// Src/mg.f90:808-847 (getres), Dirichlet form
__device__ __forceinline__ double getres(const MGLev &L, long long q, double urhs) {
  const long long sy = L.N1, sz = L.N1 * L.N2;
  double uij = L.u[q], un = L.u[q + sy], us = L.u[q - sy], ue = L.u[q + 1];
  double ut = L.u[q + sz], ub = L.u[q - sz], uw = L.u[q - 1];
  return urhs - (L.aw * uw + L.ae * ue + L.an * un + L.as * us + L.ac * uij + L.at * ut + L.ab * ub);
}

__device__ __forceinline__ int fmap(int ic, int ncell) {
  return ic == ncell / 2 + 2 ? ncell + 2 : (ic == 0 ? 0 : 2 * ic - 1);
}

// Src/mg.f90:248-805 (restriction), fine F -> coarse C
__device__ void restriction(const MGLev &F, const MGLev &C, cg::grid_group &grid) {
  const Warps w = grid_warps();
  const int lane = threadIdx.x & 31;
  for_rows(w, 1, F.n2 + 1, 1, F.n3 + 1, [&](int j, int k) {
    for (int i = 1 + lane; i <= F.n1 + 1; i += 32) {
      long long q = F.g(i, j, k);
      F.rf[q] = (F.bc[q] > 0) ? 0.0 : getres(F, q, F.b[F.r(i, j, k)]);
    }
  });
  grid.sync();
  const long long sy = F.N1, sz = F.N1 * F.N2;
  for_rows(w, 0, C.n2 + 3, 0, C.n3 + 3, [&](int j, int k) {
    for (int i = lane; i <= C.n1 + 2; i += 32) {
      long long qc = C.g(i, j, k);
      int bc2 = F.bc[F.g(fmap(i, F.n1), fmap(j, F.n2), fmap(k, F.n3))];
      C.bc[qc] = bc2;
      C.u[qc] = 0.0;
      if (i <= C.n1 + 1 && j <= C.n2 + 1 && k <= C.n3 + 1) {
        double re = 0.0;
        if (i >= 1 && j >= 1 && k >= 1 && bc2 <= 0) {
          long long q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
          const double *R = F.rf;
          double r000 = R[q];
          double rpp0 = R[q + 1 + sy], rp00 = R[q + 1], rpm0 = R[q + 1 - sy];
          double r0m0 = R[q - sy], rmm0 = R[q - 1 - sy], rm00 = R[q - 1];
          double rmp0 = R[q - 1 + sy], r0p0 = R[q + sy];
          double r00p = R[q + sz], rppp = R[q + 1 + sy + sz], rp0p = R[q + 1 + sz];
          double rpmp = R[q + 1 - sy + sz], r0mp = R[q - sy + sz];
          double rmmp = R[q - 1 - sy + sz], rm0p = R[q - 1 + sz];
          double rmpp = R[q - 1 + sy + sz], r0pp = R[q + sy + sz];
          double r00m = R[q - sz], rppm = R[q + 1 + sy - sz], rp0m = R[q + 1 - sz];
          double rpmm = R[q + 1 - sy - sz], r0mm = R[q - sy - sz];
          double rmmm = R[q - 1 - sy - sz], rm0m = R[q - 1 - sz];
          double rmpm = R[q - 1 + sy - sz], r0pm = R[q + sy - sz];
          re = (8.0 * r000 + 4.0 * (rp00 + rm00 + r0p0 + r0m0 + r00p + r00m) +
                2.0 * (rpp0 + rmp0 + rpm0 + rmm0 + rp0p + rm0p + r0pp + r0mp + rp0m + rm0m +
                       r0pm + r0mm) +
                rppp + rmpp + rpmp + rmmp + rppm + rmpm + rpmm + rmmm) /
               64.0;
        }
        C.b[C.r(i, j, k)] = re;
      }
    }
  });
  grid.sync();
}

// Src/mg.f90:808-847 (getres) with its Neumann form: on the plane ir = 1
// with flag_nmn the west term is dropped (aw = uw = 0) and ae doubled.
__device__ __forceinline__ double getres_n(const MGLev &L, long long q, double urhs, bool neumann) {
  const long long sy = L.N1, sz = L.N1 * L.N2;
  double uij = L.u[q], un = L.u[q + sy], us = L.u[q - sy], ue = L.u[q + 1];
  double ut = L.u[q + sz], ub = L.u[q - sz];
  double uw, aw = L.aw, ae = L.ae;
  if (neumann) {
    uw = 0.0;
    aw = 0.0;
    ae = 2.0 * ae;
  } else {
    uw = L.u[q - 1];
  }
  return urhs - (aw * uw + ae * ue + L.an * un + L.as * us + L.ac * uij + L.at * ut + L.ab * ub);
}

// Src/mg.f90:248-805 (restriction) with periodic planes in y and z and/or
// the Neumann plane.  (1) the fine residual of every node 1..n+1 (no wall
// mask: the gather tests the neighbours' bcnd as the reference does);
// (2) with periodic planes, the residual plane r_pbc of the last fine z plane
// as the reference's loop over coarse nodes leaves it (j outer, i inner, a
// later write replacing an earlier one: every fine node takes the value of
// the last coarse node that writes it); (3) the 27-point gather, where a
// neighbour at jr-1 = 0 takes the residual of its periodic image jr = n2 in
// the terms the reference wraps and one at kr-1 = 0 takes r_pbc.  Residuals
// outside 1..n+1 (a wrapped term at ir+1 = n1+2) are zero.
__device__ void restriction_gen(const MGArgs &a, const MGLev &F, const MGLev &C, cg::grid_group &grid) {
  const Warps w = grid_warps();
  const int lane = threadIdx.x & 31;
  const int n1 = F.n1, n2 = F.n2, m = F.n3;
  const bool nmn = a.nmn != 0, pbc = a.pbc != 0;
  for_rows(w, 1, n2 + 1, 1, m + 1, [&](int j, int k) {
    for (int i = 1 + lane; i <= n1 + 1; i += 32) {
      long long q = F.g(i, j, k);
      F.rf[q] = getres_n(F, q, F.b[F.r(i, j, k)], nmn && i == 1);
    }
  });
  grid.sync();
  auto G = [&](int x, int y, int z) -> double {
    if (x < 1 || x > n1 + 1 || y < 1 || y > n2 + 1 || z < 1 || z > m + 1) return 0.0;
    return F.rf[F.g(x, y, z)];
  };
  auto BC = [&](int x, int y, int z) -> int { return F.bc[F.g(x, y, z)]; };
  const long long RP1 = n1 + 2;
  if (pbc) {
    for_rows(w, 1, n2 + 1, 0, 1, [&](int b, int) {
      for (int x = 1 + lane; x <= n1 + 1; x += 32) {
        double v = 0.0;
        bool done = false;
        // coarse writers of (x, b): jr, ir odd within one node, latest first
        for (int jr = ((b + 1) & 1) ? b + 1 : b; jr >= b - 1 && !done; jr -= 2) {
          if (jr < 1 || jr > n2 + 1) continue;
          for (int ir = ((x + 1) & 1) ? x + 1 : x; ir >= x - 1 && !done; ir -= 2) {
            if (ir < 1 || ir > n1 + 1) continue;
            const int dx = x - ir, dy = b - jr;
            const bool le = BC(ir, jr, m + 1) <= 0;
            bool wr;
            if (dx == -1) wr = ir != 1 && (dy == -1 ? jr != 1 : (dy == 1 ? jr != n2 + 1 : true));
            else if (dx == 1) wr = ir != n1 + 1 && (dy == -1 ? jr != 1 : (dy == 1 ? jr != n2 + 1 : true));
            else wr = dy == -1 ? ((le ? ir != 1 : true) && jr != 1) : (dy == 1 ? jr != n2 + 1 : true);
            if (wr) {
              v = le ? F.rf[F.g(x, b, m)] : 0.0;
              done = true;
            }
          }
        }
        F.rp[x + RP1 * b] = v;
      }
    });
    grid.sync();
  }
  auto RP = [&](int x, int y) -> double { return pbc ? F.rp[x + RP1 * y] : 0.0; };
  for_rows(w, 0, C.n2 + 3, 0, C.n3 + 3, [&](int j, int k) {
    for (int i = lane; i <= C.n1 + 2; i += 32) {
      long long qc = C.g(i, j, k);
      int bc2 = F.bc[F.g(fmap(i, F.n1), fmap(j, F.n2), fmap(k, F.n3))];
      C.bc[qc] = bc2;
      C.u[qc] = 0.0;
      if (i > C.n1 + 1 || j > C.n2 + 1 || k > C.n3 + 1) continue;
      double re = 0.0;
      if (i >= 1 && j >= 1 && k >= 1 && bc2 <= 0) {
        const int ir = 2 * i - 1, jr = 2 * j - 1, kr = 2 * k - 1;
        const bool xl = ir != 1, xr = ir != n1 + 1, yl = jr != 1, yr = jr != n2 + 1, zr = kr != m + 1;
        const bool z0 = kr == 1;
        double r000 = G(ir, jr, kr);
        double rpp0 = (xr && yr && BC(ir + 1, jr + 1, kr) <= 0) ? G(ir + 1, jr + 1, kr) : 0.0;
        double rp00 = (xr && BC(ir + 1, jr, kr) <= 0) ? G(ir + 1, jr, kr) : 0.0;
        double rpm0 = 0.0;
        if (BC(ir + 1, jr - 1, kr) <= 0) {
          if (xr && yl) rpm0 = G(ir + 1, jr - 1, kr);
          else if (!yl) rpm0 = G(ir + 1, n2, kr);
        }
        double r0m0 = 0.0;
        if (BC(ir, jr - 1, kr) <= 0) r0m0 = yl ? G(ir, jr - 1, kr) : G(ir, n2, kr);
        double rmm0 = 0.0;
        if (BC(ir - 1, jr - 1, kr) <= 0 && xl) rmm0 = yl ? G(ir - 1, jr - 1, kr) : G(ir - 1, n2, kr);
        double rm00 = (xl && BC(ir - 1, jr, kr) <= 0) ? G(ir - 1, jr, kr) : 0.0;
        double rmp0 = (xl && yr && BC(ir - 1, jr + 1, kr) <= 0) ? G(ir - 1, jr + 1, kr) : 0.0;
        double r0p0 = (yr && BC(ir, jr + 1, kr) <= 0) ? G(ir, jr + 1, kr) : 0.0;
        double r00p = (zr && BC(ir, jr, kr + 1) <= 0) ? G(ir, jr, kr + 1) : 0.0;
        double rppp = (xr && yr && zr && BC(ir + 1, jr + 1, kr + 1) <= 0) ? G(ir + 1, jr + 1, kr + 1) : 0.0;
        double rp0p = (xr && zr && BC(ir + 1, jr, kr + 1) <= 0) ? G(ir + 1, jr, kr + 1) : 0.0;
        double rpmp = 0.0;
        if (BC(ir + 1, jr - 1, kr + 1) <= 0) {
          if (xr && yl && zr) rpmp = G(ir + 1, jr - 1, kr + 1);
          else if (!yl && zr) rpmp = G(ir + 1, n2, kr + 1);
        }
        double r0mp = 0.0;
        if (BC(ir, jr - 1, kr + 1) <= 0 && zr) r0mp = yl ? G(ir, jr - 1, kr + 1) : G(ir, n2, kr + 1);
        double rmmp = 0.0;
        if (BC(ir - 1, jr - 1, kr + 1) <= 0 && xl && zr)
          rmmp = yl ? G(ir - 1, jr - 1, kr + 1) : G(ir - 1, n2, kr + 1);
        double rm0p = (xl && zr && BC(ir - 1, jr, kr + 1) <= 0) ? G(ir - 1, jr, kr + 1) : 0.0;
        double rmpp = (xl && yr && zr && BC(ir - 1, jr + 1, kr + 1) <= 0) ? G(ir - 1, jr + 1, kr + 1) : 0.0;
        double r0pp = (yr && zr && BC(ir, jr + 1, kr + 1) <= 0) ? G(ir, jr + 1, kr + 1) : 0.0;
        double r00m = 0.0;
        if (BC(ir, jr, kr - 1) <= 0) r00m = z0 ? RP(ir, jr) : G(ir, jr, kr - 1);
        double rppm = 0.0;
        if (BC(ir + 1, jr + 1, kr - 1) <= 0 && xr && yr) rppm = z0 ? RP(ir + 1, jr + 1) : G(ir + 1, jr + 1, kr - 1);
        double rp0m = 0.0;
        if (BC(ir + 1, jr, kr - 1) <= 0 && xr) rp0m = z0 ? RP(ir + 1, jr) : G(ir + 1, jr, kr - 1);
        double rpmm = 0.0;
        if (BC(ir + 1, jr - 1, kr - 1) <= 0) {
          if (z0) rpmm = (xr && yl) ? RP(ir + 1, jr - 1) : 0.0;
          else if (yl) rpmm = xr ? G(ir + 1, jr - 1, kr - 1) : 0.0;
          else rpmm = G(ir + 1, n2, kr - 1);
        }
        double r0mm = 0.0;
        if (BC(ir, jr - 1, kr - 1) <= 0) {
          if (z0) r0mm = yl ? RP(ir, jr - 1) : 0.0;
          else r0mm = yl ? G(ir, jr - 1, kr - 1) : G(ir, n2, kr - 1);
        }
        double rmmm = 0.0;
        if (BC(ir - 1, jr - 1, kr - 1) <= 0 && xl) {
          if (z0) rmmm = yl ? RP(ir - 1, jr - 1) : 0.0;
          else rmmm = yl ? G(ir - 1, jr - 1, kr - 1) : G(ir - 1, n2, kr - 1);
        }
        double rm0m = 0.0;
        if (BC(ir - 1, jr, kr - 1) <= 0 && xl) rm0m = z0 ? RP(ir - 1, jr) : G(ir - 1, jr, kr - 1);
        double rmpm = 0.0;
        if (BC(ir - 1, jr + 1, kr - 1) <= 0 && xl && yr) rmpm = z0 ? RP(ir - 1, jr + 1) : G(ir - 1, jr + 1, kr - 1);
        double r0pm = 0.0;
        if (BC(ir, jr + 1, kr - 1) <= 0 && yr) r0pm = z0 ? RP(ir, jr + 1) : G(ir, jr + 1, kr - 1);
        re = (8.0 * r000 + 4.0 * (rp00 + rm00 + r0p0 + r0m0 + r00p + r00m) +
              2.0 * (rpp0 + rmp0 + rpm0 + rmm0 + rp0p + rm0p + r0pp + r0mp + rp0m + rm0m + r0pm + r0mm) +
              rppp + rmpp + rpmp + rmmp + rppm + rmpm + rpmm + rmmm) /
             64.0;
      }
      C.b[C.r(i, j, k)] = re;
    }
  });
  grid.sync();
}

// Src/mg.f90:849-939 (prolongation): coarse C added into fine F
__device__ void prolongation(const MGLev &F, const MGLev &C, cg::grid_group &grid) {
  const Warps w = grid_warps();
  const int lane = threadIdx.x & 31;
  const long long sy = F.N1, sz = F.N1 * F.N2;
  const long long cy = C.N1, cz = C.N1 * C.N2;
  for_rows(w, 1, C.n2 + 1, 1, C.n3 + 1, [&](int j, int k) {
    for (int i = 1 + lane; i <= C.n1 + 1; i += 32) {
      long long c = C.g(i, j, k);
      const double *E = C.u;
      double r000 = E[c], r0m0 = E[c - cy], rmm0 = E[c - 1 - cy], rm00 = E[c - 1];
      double r00m = E[c - cz], r0mm = E[c - cy - cz], rmmm = E[c - 1 - cy - cz], rm0m = E[c - 1 - cz];
      long long q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
      double *U = F.u;
      const int *B = F.bc;
      if (B[q] <= 0) U[q] = U[q] + r000;
      if (B[q - sy] <= 0) U[q - sy] = U[q - sy] + (r000 + r0m0) / 2.0;
      if (B[q - 1 - sy] <= 0) U[q - 1 - sy] = U[q - 1 - sy] + (r000 + r0m0 + rmm0 + rm00) / 4.0;
      if (B[q - 1] <= 0) U[q - 1] = U[q - 1] + (r000 + rm00) / 2.0;
      if (B[q - sz] <= 0) U[q - sz] = U[q - sz] + (r000 + r00m) / 2.0;
      if (B[q - sy - sz] <= 0) U[q - sy - sz] = U[q - sy - sz] + (r000 + r00m + r0mm + r0m0) / 4.0;
      if (B[q - 1 - sz] <= 0) U[q - 1 - sz] = U[q - 1 - sz] + (r000 + r00m + rm0m + rm00) / 4.0;
      if (B[q - 1 - sy - sz] <= 0)
        U[q - 1 - sy - sz] =
            U[q - 1 - sy - sz] + (r000 + r00m + rm0m + rm00 + r0m0 + r0mm + rmmm + rmm0) / 8.0;
    }
  });
  grid.sync();
}

template <bool GEN>
__global__ void __launch_bounds__(MG_BLOCK) k_pdesolver(const MGArgs *__restrict__ ap) {
  cg::grid_group grid = cg::this_grid();
  const MGArgs &a = *ap;
  __shared__ double sh[40];
  const int ng = a.ng;
  int k = 1;
  double res_s = 0.0, ktot = 0.0, r = 0.0;
  int status = 0;
  bool converged = false;
  while (!converged) {
    int iter[MG_MAX + 1];
    for (int i = 0; i <= MG_MAX; ++i) iter[i] = 0;
    const double eps_abs = a.alpha * a.eps;
    for (int ig = 1; ig <= 2 * ng - 1; ++ig) {
      int ksor = 0;
      if (ig < ng) {
        int il = ig;
        sor_rb<GEN>(a, a.L[il], k, ig - ng, eps_abs, grid, sh, r, ksor);
        iter[il] += ksor;
        if (GEN)
          restriction_gen(a, a.L[il], a.L[il + 1], grid);
        else
          restriction(a.L[il], a.L[il + 1], grid);
      } else if (ig == ng) {
        sor_rb<GEN>(a, a.L[ng], k, 0, eps_abs, grid, sh, r, ksor);
        iter[ng] += ksor;
        if (ng >= 2) prolongation(a.L[ng - 1], a.L[ng], grid);
      } else {
        int il = 2 * ng - ig;
        sor_rb<GEN>(a, a.L[il], k, ig - ng, eps_abs, grid, sh, r, ksor);
        iter[il] += ksor;
        if (il >= 2) prolongation(a.L[il - 1], a.L[il], grid);
      }
    }
    for (int i = 1; i <= ng; ++i) ktot = ktot + (double)(float)iter[i] / exp2((double)(2 * (i - 1)));
    r = r / a.alpha;
    if (k == 1) {
      res_s = r;
    } else if (fabs(r / res_s) > 10.0) {
      status = LEPIC_ERR_DIVERGED;
      converged = true;
    }
    if (r < a.eps || k == a.ncycl) converged = true;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      for (int i = 1; i <= ng; ++i) a.out_i[2 + i] = iter[i];
    }
    k = k + 1;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out_i[0] = k;
    a.out_i[1] = status;
    a.out_d[0] = ktot;
    a.out_d[1] = r;
  }
}

}  // namespace

int launch_pdesolver(const Dims &d, const double h[3], double *u, const double *b, const int *bcnd,
                     int ncycl, double eps, double omega, int ng, double eps0, int *k_out,
                     double *ktot_out, double *res_out, cudaStream_t s, int pbc, int nmn) {
  if (ng < 1 || ng > MG_MAX) return LEPIC_ERR_ARG;
  const bool gen = pbc || nmn;
  int n[3] = {d.n1, d.n2, d.n3};
  for (int a = 0; a < 3; ++a)
    if (n[a] % (1 << (ng - 1))) return LEPIC_ERR_ARG;
  Ctx &c = ctx();
  MGArgs A;
  memset(&A, 0, sizeof(A));
  A.ng = ng;
  A.ncycl = ncycl;
  A.eps = eps;
  A.omega = omega;
  A.pbc = pbc ? 1 : 0;
  A.nmn = nmn ? 1 : 0;
  char nm[32];
  for (int l = 1; l <= ng; ++l) {
    MGLev &L = A.L[l];
    L.n1 = n[0] >> (l - 1);
    L.n2 = n[1] >> (l - 1);
    L.n3 = n[2] >> (l - 1);
    L.N1 = L.n1 + 3;
    L.N2 = L.n2 + 3;
    L.R1 = L.n1 + 2;
    L.R2 = L.n2 + 2;
    double hl[3];
    for (int q = 0; q < 3; ++q) hl[q] = h[q] * (double)(1 << (l - 1));
    L.aw = eps0 / (hl[0] * hl[0]);
    L.ae = L.aw;
    L.an = eps0 / (hl[1] * hl[1]);
    L.as = L.an;
    L.at = eps0 / (hl[2] * hl[2]);
    L.ab = L.at;
    L.ac = -(L.an + L.as + L.aw + L.ae + L.at + L.ab);
    long long nn = (long long)(L.n1 + 3) * (L.n2 + 3) * (L.n3 + 3);
    long long nr = (long long)(L.n1 + 2) * (L.n2 + 2) * (L.n3 + 2);
    if (l == 1) {
      L.u = u;
      L.b = const_cast<double *>(b);
      L.bc = const_cast<int *>(bcnd);
    } else {
      snprintf(nm, sizeof nm, "mg_e%d", l);
      L.u = (double *)scratch(nm, sizeof(double) * nn);
      snprintf(nm, sizeof nm, "mg_r%d", l);
      L.b = (double *)scratch(nm, sizeof(double) * nr);
      snprintf(nm, sizeof nm, "mg_bc%d", l);
      L.bc = (int *)scratch(nm, sizeof(int) * nn);
      if (!L.u || !L.b || !L.bc) return LEPIC_ERR_CUDA;
    }
    if (l < ng) {
      snprintf(nm, sizeof nm, "mg_rf%d", l);
      L.rf = (double *)scratch(nm, sizeof(double) * nn);
      if (!L.rf) return LEPIC_ERR_CUDA;
      LEPIC_CUDA(cudaMemsetAsync(L.rf, 0, sizeof(double) * nn, s));
      if (gen) {
        snprintf(nm, sizeof nm, "mg_rp%d", l);
        L.rp = (double *)scratch(nm, sizeof(double) * (size_t)(L.n1 + 2) * (L.n2 + 2));
        if (!L.rp) return LEPIC_ERR_CUDA;
      }
    }
  }
  double ac = A.L[1].ac;
  A.alpha = fabs((double)((n[0] + 1) * (n[1] + 1) * (n[2] + 1)) * ac) * 1.0;
  void *kern = gen ? (void *)k_pdesolver<true> : (void *)k_pdesolver<false>;
  int occ = 0;
  LEPIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, MG_BLOCK, 0));
  if (occ < 1) return LEPIC_ERR_CUDA;
  int blocks = c.sms * (occ < 2 ? occ : 2);
  A.partial = (double *)scratch("mg_partial", sizeof(double) * blocks);
  A.shared_d = (double *)scratch("mg_shared", sizeof(double) * 4);
  A.out_i = (int *)scratch("mg_out_i", sizeof(int) * (MG_MAX + 4));
  A.out_d = (double *)scratch("mg_out_d", sizeof(double) * 2);
  if (!A.partial || !A.shared_d || !A.out_i || !A.out_d) return LEPIC_ERR_CUDA;
  MGArgs *dA = (MGArgs *)scratch("mg_args", sizeof(MGArgs));
  if (!dA) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemcpyAsync(dA, &A, sizeof(MGArgs), cudaMemcpyHostToDevice, s));
  void *args[] = {&dA};
  int tm = timer_start("pdesolver_f64", s);
  LEPIC_CUDA(cudaLaunchCooperativeKernel(kern, dim3(blocks), dim3(MG_BLOCK), args, 0, s));
  timer_stop(tm, s);
  int hi[MG_MAX + 4];
  double hd[2];
  LEPIC_CUDA(cudaMemcpyAsync(hi, A.out_i, sizeof(hi), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(hd, A.out_d, sizeof(hd), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (k_out) *k_out = hi[0];
  if (ktot_out) *ktot_out = hd[0];
  if (res_out) *res_out = hd[1];
  return hi[1];
}

}  // namespace lepic

// ---------------------------------------------------------------------------
// Allocation-free variant of the Poisson solve.
//
// Some callers cannot call cudaMalloc once their time loop runs: a Fortran
// driver (or a framework such as PyTorch) that owns the device memory through
// its own pool hands every buffer in and forbids allocations inside the loop,
// because cudaMalloc synchronises the whole device and fails once the pool has
// claimed the memory.  lepic_dev_pdesolver_noalloc runs the same cooperative
// kernel as lepic_dev_pdesolver, but carves all of its scratch (the level
// arrays e, r, bcnd and the fine residuals of levels 2..ng, the block partial
// sums, the argument block and the outputs) out of one file-scope device array
// of MG_NOALLOC_BYTES bytes, which every GPU that loads the library holds until
// the process exits.  The caller still passes u, b and bcnd.
// ---------------------------------------------------------------------------
namespace lepic {
namespace {

constexpr size_t MG_NOALLOC_BYTES = 8u << 20;  // 8 MiB: grids up to 64^3 cells
static __device__ __align__(256) unsigned char g_mg_noalloc_scratch[MG_NOALLOC_BYTES];

constexpr int MG_NOALLOC_MAX_DEVICES = 64;
unsigned char *g_noalloc_ptr[MG_NOALLOC_MAX_DEVICES] = {nullptr};

inline size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

}  // namespace

}  // namespace lepic

extern "C" int lepic_dev_pdesolver_noalloc(const lepic_grid_t *g, double *u, const double *b,
                                           int ncycl, double eps, double omega, int ng,
                                           const lepic_phys_t *P, int *k_out, double *ktot_out,
                                           double *res_out, void *stream) {
  using namespace lepic;
  if (!g || !P) return LEPIC_ERR_ARG;
  if (P->flag_pbc || P->flag_nmn) return LEPIC_ERR_UNSUPPORTED;
  if (ng < 1 || ng > MG_MAX) return LEPIC_ERR_ARG;
  const int n[3] = {g->n[0], g->n[1], g->n[2]};
  for (int a = 0; a < 3; ++a)
    if (n[a] < 1 || n[a] % (1 << (ng - 1))) return LEPIC_ERR_ARG;
  cudaStream_t s = (cudaStream_t)stream;
  int dev = 0;
  LEPIC_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= MG_NOALLOC_MAX_DEVICES) return LEPIC_ERR_ARG;
  // Set-up, once per device with that device current: the host-side name of
  // the __device__ array is not a device address, so look the address up.
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_mg_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_mg_noalloc_scratch)");
    g_noalloc_ptr[dev] = (unsigned char *)p;
  }
  unsigned char *base = g_noalloc_ptr[dev];
  int sms = 0, occ = 0;
  LEPIC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  LEPIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_pdesolver<false>, MG_BLOCK, 0));
  if (occ < 1 || sms < 1) return LEPIC_ERR_CUDA;
  const int blocks = sms * (occ < 2 ? occ : 2);

  MGArgs A;
  memset(&A, 0, sizeof(A));
  A.ng = ng;
  A.ncycl = ncycl;
  A.eps = eps;
  A.omega = omega;
  // carve the scratch array; rf regions are recorded to be zeroed
  size_t off = 0;
  auto carve = [&](size_t bytes) -> unsigned char * {
    size_t at = off;
    off = align256(off + bytes);
    return off <= MG_NOALLOC_BYTES ? base + at : nullptr;
  };
  MGArgs *dA = (MGArgs *)carve(sizeof(MGArgs));
  A.partial = (double *)carve(sizeof(double) * blocks);
  A.shared_d = (double *)carve(sizeof(double) * 4);
  A.out_i = (int *)carve(sizeof(int) * (MG_MAX + 4));
  A.out_d = (double *)carve(sizeof(double) * 2);
  double *rf_ptr[MG_MAX + 1] = {nullptr};
  size_t rf_bytes[MG_MAX + 1] = {0};
  bool fits = dA && A.partial && A.shared_d && A.out_i && A.out_d;
  for (int l = 1; l <= ng && fits; ++l) {
    MGLev &L = A.L[l];
    L.n1 = n[0] >> (l - 1);
    L.n2 = n[1] >> (l - 1);
    L.n3 = n[2] >> (l - 1);
    L.N1 = L.n1 + 3;
    L.N2 = L.n2 + 3;
    L.R1 = L.n1 + 2;
    L.R2 = L.n2 + 2;
    double hl[3];
    for (int q = 0; q < 3; ++q) hl[q] = g->h[q] * (double)(1 << (l - 1));
    L.aw = P->eps0 / (hl[0] * hl[0]);
    L.ae = L.aw;
    L.an = P->eps0 / (hl[1] * hl[1]);
    L.as = L.an;
    L.at = P->eps0 / (hl[2] * hl[2]);
    L.ab = L.at;
    L.ac = -(L.an + L.as + L.aw + L.ae + L.at + L.ab);
    const size_t nn = (size_t)(L.n1 + 3) * (L.n2 + 3) * (L.n3 + 3);
    const size_t nr = (size_t)(L.n1 + 2) * (L.n2 + 2) * (L.n3 + 2);
    if (l == 1) {
      L.u = u;
      L.b = const_cast<double *>(b);
      L.bc = const_cast<int *>(g->bcnd);
    } else {
      L.u = (double *)carve(sizeof(double) * nn);
      L.b = (double *)carve(sizeof(double) * nr);
      L.bc = (int *)carve(sizeof(int) * nn);
      fits = fits && L.u && L.b && L.bc;
    }
    if (l < ng) {
      L.rf = (double *)carve(sizeof(double) * nn);
      rf_ptr[l] = L.rf;
      rf_bytes[l] = sizeof(double) * nn;
      fits = fits && L.rf;
    }
  }
  if (!fits) {
    fprintf(stderr,
            "lepic_dev_pdesolver_noalloc: a %dx%dx%d grid with %d levels needs more than the %zu "
            "bytes of static scratch (grids up to 64^3 cells fit); use lepic_dev_pdesolver\n",
            n[0], n[1], n[2], ng, MG_NOALLOC_BYTES);
    return LEPIC_ERR_SCRATCH_LIMIT;
  }
  A.alpha = fabs((double)((n[0] + 1) * (n[1] + 1) * (n[2] + 1)) * A.L[1].ac) * 1.0;
  // the shared array keeps the previous call's contents: clear the fine
  // residual arrays whose ghost entries the restriction may read
  for (int l = 1; l < ng; ++l) LEPIC_CUDA(cudaMemsetAsync(rf_ptr[l], 0, rf_bytes[l], s));
  LEPIC_CUDA(cudaMemcpyAsync(dA, &A, sizeof(MGArgs), cudaMemcpyHostToDevice, s));
  void *args[] = {&dA};
  LEPIC_CUDA(cudaLaunchCooperativeKernel((void *)k_pdesolver<false>, dim3(blocks), dim3(MG_BLOCK), args, 0, s));
  int hi[MG_MAX + 4];
  double hd[2];
  LEPIC_CUDA(cudaMemcpyAsync(hi, A.out_i, sizeof(hi), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(hd, A.out_d, sizeof(hd), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (k_out) *k_out = hi[0];
  if (ktot_out) *ktot_out = hd[0];
  if (res_out) *res_out = hd[1];
  return hi[1];
}
