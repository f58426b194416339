// Mixed-precision Poisson solve: FP32 multigrid V-cycles inside an FP64
// iterative-refinement loop, as one persistent cooperative kernel.
//
//   repeat:  r = b - A u          (FP64, plasma nodes; L1 norm -> exit test
//                                   res/alpha < eps of Src/pdesolver.f90:91-111)
//            A e = r  approx.     (one FP32 V-cycle, zero initial guess)
//            u = u + e            (FP64)
//
// The operators are the reference's (Src/mg.h, Src/sors.f90 red-black SOR,
// Src/mg.f90 27-point full-weighting restriction and trilinear
// prolongation), evaluated in FP32 on the correction; only the residual and
// the accumulation of u are FP64, so u converges to the FP64 solution while
// the V-cycle moves half the bytes.  The level masks are injected from the
// finest mask once per call.
//
// The fine levels are swept by the whole grid (warps take grid rows, lanes
// split a row, grid-wide barriers between phases).  The coarse levels, from
// the first one whose arrays fit in shared memory down to the coarsest, live
// in block 0's shared memory for the whole call: each V-cycle block 0 loads
// the restricted right-hand side of the top coarse level, runs the coarse
// part of the cycle on chip with block barriers only, and stores the
// correction back for the grid to prolongate.
#include <cooperative_groups.h>

#include <cstring>

#include "lepic_internal.cuh"

namespace cg = cooperative_groups;

namespace lepic {

namespace {

constexpr int XM_MAX = 13;
constexpr int XM_BLOCK = 512;
constexpr size_t XM_SMEM_BUDGET = 160 * 1024;  // coarse levels in block 0's shared memory

struct XLev {
  int n1, n2, n3;
  int N1, N2;          // n+3
  int R1, R2;          // n+2
  float aw, ae, an, as, at, ab, ac;
  float *e;            // (n+3)^3 correction
  float *r;            // (n+2)^3 right-hand side
  float *rf;           // (n+3)^3 residual scratch
  int *bc;             // (n+3)^3 mask (level 1: caller's bcnd)
  __device__ long long g(int i, int j, int k) const { return i + (long long)N1 * (j + (long long)N2 * k); }
  __device__ long long rr(int i, int j, int k) const { return i + (long long)R1 * (j + (long long)R2 * k); }
  __host__ __device__ long long nn() const { return (long long)N1 * N2 * (n3 + 3); }
  __host__ __device__ long long nr() const { return (long long)R1 * R2 * (n3 + 2); }
};

struct XArgs {
  XLev L[XM_MAX + 1];
  int ng, ls;          // levels 1..ls on the grid, ls+1..ng in shared memory
  int max_refine, nu_pre, nu_post, coarse_sweeps;
  float omega;
  double aw, ae, an, as, at, ab, ac;  // FP64 finest coefficients
  double *u;
  const double *b;
  double alpha, eps;
  double *partial;
  int *out_i;      // [0] refinement iterations, [1] status
  double *out_d;   // [0] res/alpha, [1] first res/alpha
  // shared-memory offsets (bytes) of e, r, rf, bc of the coarse levels
  unsigned so_e[XM_MAX + 1], so_r[XM_MAX + 1], so_rf[XM_MAX + 1], so_bc[XM_MAX + 1];
};

__device__ __forceinline__ double wsum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ double bsum(double v, double *sh) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  v = wsum(v);
  __syncthreads();
  if (lane == 0) sh[w] = v;
  __syncthreads();
  double t = (threadIdx.x < (blockDim.x >> 5)) ? sh[threadIdx.x] : 0.0;
  if (w == 0) t = wsum(t);
  if (threadIdx.x == 0) sh[32] = t;
  __syncthreads();
  double r = sh[32];
  __syncthreads();
  return r;
}

// deterministic grid-wide sum of one value per thread
__device__ double grid_sum(const XArgs &a, double v, cg::grid_group &grid, double *sh) {
  double part = bsum(v, sh);
  if (threadIdx.x == 0) a.partial[blockIdx.x] = part;
  grid.sync();
  double s = 0.0;
  if (threadIdx.x < 32) {
    for (int bI = threadIdx.x; bI < (int)gridDim.x; bI += 32) s += a.partial[bI];
    s = wsum(s);
    if (threadIdx.x == 0) sh[33] = s;
  }
  __syncthreads();
  s = sh[33];
  __syncthreads();
  grid.sync();  // partials may be reused
  return s;
}

// red-black colour start: colour 0 = red ((i+j+k) odd), 1 = black
// (Src/sors.f90:87-106, 249-267)
__device__ __forceinline__ int colour_start(int colour, int j, int k) {
  int is = (colour == 0) ? ((j % 2 == 0) ? 1 : 2) : ((j % 2 == 0) ? 2 : 1);
  is += (k % 2 == 0) ? 0 : 1;
  return is > 2 ? 1 : is;
}

__device__ __forceinline__ void relax(const XLev &L, float omega, float rac, int i, int j, int k) {
  const long long sy = L.N1, sz = (long long)L.N1 * L.N2;
  const long long q = L.g(i, j, k);
  if (L.bc[q] > 0) return;
  const float tt = L.r[L.rr(i, j, k)] - L.aw * L.e[q - 1] - L.an * L.e[q + sy] - L.as * L.e[q - sy] -
                   L.ae * L.e[q + 1] - L.at * L.e[q + sz] - L.ab * L.e[q - sz];
  L.e[q] = (1.f - omega) * L.e[q] + omega * tt * rac;
}

__device__ __forceinline__ float fine_residual(const XLev &F, int i, int j, int k) {
  const long long sy = F.N1, sz = (long long)F.N1 * F.N2;
  const long long q = F.g(i, j, k);
  if (F.bc[q] > 0) return 0.f;
  return F.r[F.rr(i, j, k)] - (F.aw * F.e[q - 1] + F.ae * F.e[q + 1] + F.an * F.e[q + sy] +
                               F.as * F.e[q - sy] + F.ac * F.e[q] + F.at * F.e[q + sz] + F.ab * F.e[q - sz]);
}

// 27-point full weighting of the fine residual onto coarse node (i,j,k)
// (Src/mg.f90:248-805); C.e cleared
__device__ __forceinline__ void restrict_node(const XLev &F, const XLev &C, int i, int j, int k) {
  const long long qc = C.g(i, j, k);
  C.e[qc] = 0.f;
  if (i > C.n1 + 1 || j > C.n2 + 1 || k > C.n3 + 1) return;
  float re = 0.f;
  if (i >= 1 && j >= 1 && k >= 1 && C.bc[qc] <= 0) {
    const long long sy = F.N1, sz = (long long)F.N1 * F.N2;
    const long long q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
    const float *R = F.rf;
    re = (8.f * R[q] + 4.f * (R[q + 1] + R[q - 1] + R[q + sy] + R[q - sy] + R[q + sz] + R[q - sz]) +
          2.f * (R[q + 1 + sy] + R[q - 1 + sy] + R[q + 1 - sy] + R[q - 1 - sy] + R[q + 1 + sz] + R[q - 1 + sz] +
                 R[q + sy + sz] + R[q - sy + sz] + R[q + 1 - sz] + R[q - 1 - sz] + R[q + sy - sz] +
                 R[q - sy - sz]) +
          R[q + 1 + sy + sz] + R[q - 1 + sy + sz] + R[q + 1 - sy + sz] + R[q - 1 - sy + sz] + R[q + 1 + sy - sz] +
          R[q - 1 + sy - sz] + R[q + 1 - sy - sz] + R[q - 1 - sy - sz]) *
         (1.f / 64.f);
  }
  C.r[C.rr(i, j, k)] = re;
}

// trilinear prolongation of coarse node (i,j,k) added into F (Src/mg.f90:849-939)
__device__ __forceinline__ void prolong_node(const XLev &F, const XLev &C, int i, int j, int k) {
  const long long sy = F.N1, sz = (long long)F.N1 * F.N2, cy = C.N1, cz = (long long)C.N1 * C.N2;
  const long long c = C.g(i, j, k);
  const float *E = C.e;
  const float r000 = E[c], r0m0 = E[c - cy], rmm0 = E[c - 1 - cy], rm00 = E[c - 1];
  const float r00m = E[c - cz], r0mm = E[c - cy - cz], rmmm = E[c - 1 - cy - cz], rm0m = E[c - 1 - cz];
  const long long q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
  float *U = F.e;
  const int *B = F.bc;
  if (B[q] <= 0) U[q] += r000;
  if (B[q - sy] <= 0) U[q - sy] += (r000 + r0m0) * 0.5f;
  if (B[q - 1 - sy] <= 0) U[q - 1 - sy] += (r000 + r0m0 + rmm0 + rm00) * 0.25f;
  if (B[q - 1] <= 0) U[q - 1] += (r000 + rm00) * 0.5f;
  if (B[q - sz] <= 0) U[q - sz] += (r000 + r00m) * 0.5f;
  if (B[q - sy - sz] <= 0) U[q - sy - sz] += (r000 + r00m + r0mm + r0m0) * 0.25f;
  if (B[q - 1 - sz] <= 0) U[q - 1 - sz] += (r000 + r00m + rm0m + rm00) * 0.25f;
  if (B[q - 1 - sy - sz] <= 0)
    U[q - 1 - sy - sz] += (r000 + r00m + rm0m + rm00 + r0m0 + r0mm + rmmm + rmm0) * 0.125f;
}

__device__ __forceinline__ int fmapx(int ic, int ncell) {
  return ic == ncell / 2 + 2 ? ncell + 2 : (ic == 0 ? 0 : 2 * ic - 1);
}

// ------------------------------------------------------------ grid-wide
// The rows (j, k), j in [j0, j0 + nj), k in [k0, k0 + nk), dealt round-robin
// to all warps of the grid; body(j, k) runs on all lanes, which split the row
// along i (coalesced, one 32-bit division per row).
template <class F>
__device__ __forceinline__ void grid_rows(int j0, int nj, int k0, int nk, F &&body) {
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int rows = nj * nk;
  for (int r = gw; r < rows; r += nw) {
    const int kk = r / nj;
    body(j0 + (r - kk * nj), k0 + kk);
  }
}

__device__ void g_smooth(const XLev &L, float omega, int nsweep, cg::grid_group &grid) {
  const int lane = threadIdx.x & 31;
  const float rac = 1.f / L.ac;
  for (int s = 0; s < nsweep; ++s) {
    for (int colour = 0; colour < 2; ++colour) {
      grid_rows(1, L.n2 + 1, 1, L.n3 + 1, [&](int j, int k) {
        for (int i = colour_start(colour, j, k) + 2 * lane; i <= L.n1 + 1; i += 64) relax(L, omega, rac, i, j, k);
      });
      grid.sync();
    }
  }
}

__device__ void g_restrict(const XLev &F, const XLev &C, cg::grid_group &grid) {
  const int lane = threadIdx.x & 31;
  grid_rows(1, F.n2 + 1, 1, F.n3 + 1, [&](int j, int k) {
    for (int i = 1 + lane; i <= F.n1 + 1; i += 32) F.rf[F.g(i, j, k)] = fine_residual(F, i, j, k);
  });
  grid.sync();
  grid_rows(0, C.n2 + 3, 0, C.n3 + 3, [&](int j, int k) {
    for (int i = lane; i <= C.n1 + 2; i += 32) restrict_node(F, C, i, j, k);
  });
  grid.sync();
}

__device__ void g_prolong(const XLev &F, const XLev &C, cg::grid_group &grid) {
  const int lane = threadIdx.x & 31;
  grid_rows(1, C.n2 + 1, 1, C.n3 + 1, [&](int j, int k) {
    for (int i = 1 + lane; i <= C.n1 + 1; i += 32) prolong_node(F, C, i, j, k);
  });
  grid.sync();
}

// ------------------------------------------------------ block 0, on chip
// flat loop over the nodes (i, j, k) of a box, 32-bit index arithmetic
template <class F>
__device__ __forceinline__ void block_box(int i0, int ni, int j0, int nj, int k0, int nk, F &&body) {
  const int tot = ni * nj * nk;
  for (int t = threadIdx.x; t < tot; t += blockDim.x) {
    const int row = t / ni, k = row / nj;
    body(i0 + (t - row * ni), j0 + (row - k * nj), k0 + k);
  }
}

__device__ void b_smooth(const XLev &L, float omega, int nsweep) {
  const float rac = 1.f / L.ac;
  const int half = (L.n1 + 2) / 2;
  for (int s = 0; s < nsweep; ++s) {
    for (int colour = 0; colour < 2; ++colour) {
      block_box(0, half, 1, L.n2 + 1, 1, L.n3 + 1, [&](int ii, int j, int k) {
        const int i = colour_start(colour, j, k) + 2 * ii;
        if (i <= L.n1 + 1) relax(L, omega, rac, i, j, k);
      });
      __syncthreads();
    }
  }
}

__device__ void b_restrict(const XLev &F, const XLev &C) {
  block_box(1, F.n1 + 1, 1, F.n2 + 1, 1, F.n3 + 1,
            [&](int i, int j, int k) { F.rf[F.g(i, j, k)] = fine_residual(F, i, j, k); });
  __syncthreads();
  block_box(0, C.n1 + 3, 0, C.n2 + 3, 0, C.n3 + 3, [&](int i, int j, int k) { restrict_node(F, C, i, j, k); });
  __syncthreads();
}

__device__ void b_prolong(const XLev &F, const XLev &C) {
  block_box(1, C.n1 + 1, 1, C.n2 + 1, 1, C.n3 + 1, [&](int i, int j, int k) { prolong_node(F, C, i, j, k); });
  __syncthreads();
}

// the coarse levels' view in block 0's shared memory
__device__ __forceinline__ XLev smem_level(const XArgs &a, int l, unsigned char *sm) {
  XLev S = a.L[l];
  S.e = reinterpret_cast<float *>(sm + a.so_e[l]);
  S.r = reinterpret_cast<float *>(sm + a.so_r[l]);
  S.rf = reinterpret_cast<float *>(sm + a.so_rf[l]);
  S.bc = reinterpret_cast<int *>(sm + a.so_bc[l]);
  return S;
}

// the coarse part of the V-cycle, block 0 only: r of level ls+1 in, e out
__device__ void coarse_cycle(const XArgs &a, unsigned char *sm) {
  const int top = a.ls + 1, ng = a.ng;
  {
    const XLev G = a.L[top], S = smem_level(a, top, sm);
    for (long long t = threadIdx.x; t < G.nr(); t += blockDim.x) S.r[t] = G.r[t];
    for (long long t = threadIdx.x; t < G.nn(); t += blockDim.x) S.e[t] = 0.f;
  }
  __syncthreads();
  for (int l = top; l < ng; ++l) {
    const XLev F = smem_level(a, l, sm), C = smem_level(a, l + 1, sm);
    b_smooth(F, a.omega, a.nu_pre);
    b_restrict(F, C);
  }
  b_smooth(smem_level(a, ng, sm), a.omega, a.coarse_sweeps);
  for (int l = ng - 1; l >= top; --l) {
    const XLev F = smem_level(a, l, sm), C = smem_level(a, l + 1, sm);
    b_prolong(F, C);
    b_smooth(F, a.omega, a.nu_post);
  }
  {
    const XLev G = a.L[top], S = smem_level(a, top, sm);
    for (long long t = threadIdx.x; t < G.nn(); t += blockDim.x) G.e[t] = S.e[t];
  }
  __threadfence();
}

__global__ void __launch_bounds__(XM_BLOCK) k_refine_mixed(const XArgs *__restrict__ ap) {
  cg::grid_group grid = cg::this_grid();
  const XArgs &a = *ap;
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ double sh[40];
  const int lane = threadIdx.x & 31;
  const int ng = a.ng, ls = a.ls;
  // level masks by injection from the finest mask (Src/mg.f90:429-436)
  for (int l = 2; l <= ng; ++l) {
    const XLev &F = a.L[l - 1], &C = a.L[l];
    grid_rows(0, C.n2 + 3, 0, C.n3 + 3, [&](int j, int k) {
      for (int i = lane; i <= C.n1 + 2; i += 32)
        C.bc[C.g(i, j, k)] = F.bc[F.g(fmapx(i, F.n1), fmapx(j, F.n2), fmapx(k, F.n3))];
    });
    grid.sync();
  }
  if (blockIdx.x == 0 && ls < ng) {
    // coarse masks and zero residual halos, resident for the whole call
    for (int l = ls + 1; l <= ng; ++l) {
      const XLev G = a.L[l], S = smem_level(a, l, smem);
      for (long long t = threadIdx.x; t < G.nn(); t += blockDim.x) {
        S.bc[t] = G.bc[t];
        S.rf[t] = 0.f;
      }
    }
    __syncthreads();
  }
  const XLev &L1 = a.L[1];
  const long long sy = L1.N1, sz = (long long)L1.N1 * L1.N2;
  double res = 0.0, res0 = -1.0;
  int it = 0, status = 0;
  for (;;) {
    // FP64 residual, FP32 copy as the V-cycle right-hand side, e = 0
    double acc = 0.0;
    grid_rows(1, L1.n2 + 1, 1, L1.n3 + 1, [&](int j, int k) {
      for (int i = 1 + lane; i <= L1.n1 + 1; i += 32) {
        const long long q = L1.g(i, j, k);
        double rv = 0.0;
        const int bc = L1.bc[q];
        if (bc <= 0) {
          const double *u = a.u;
          rv = a.b[L1.rr(i, j, k)] - (a.aw * u[q - 1] + a.an * u[q + sy] + a.as * u[q - sy] +
                                      a.ae * u[q + 1] + a.ac * u[q] + a.at * u[q + sz] + a.ab * u[q - sz]);
          if (bc == -1) acc += fabs(rv);
        }
        L1.r[L1.rr(i, j, k)] = (float)rv;
      }
    });
    grid_rows(0, L1.n2 + 3, 0, L1.n3 + 3, [&](int j, int k) {
      for (int i = lane; i <= L1.n1 + 2; i += 32) L1.e[L1.g(i, j, k)] = 0.f;
    });
    res = grid_sum(a, acc, grid, sh) / a.alpha;
    if (res0 < 0.0) res0 = res;
    if (res < a.eps) break;
    if (it >= a.max_refine) {
      status = LEPIC_ERR_NOT_CONVERGED;
      break;
    }
    if (it > 0 && res > 10.0 * res0) {
      status = LEPIC_ERR_DIVERGED;
      break;
    }
    // FP32 V-cycle on the correction: grid levels down, coarse levels on
    // chip, grid levels up
    for (int l = 1; l <= ls && l < ng; ++l) {
      g_smooth(a.L[l], a.omega, a.nu_pre, grid);
      g_restrict(a.L[l], a.L[l + 1], grid);
    }
    if (ls < ng) {
      if (blockIdx.x == 0) coarse_cycle(a, smem);
      grid.sync();
    } else {
      g_smooth(a.L[ng], a.omega, a.coarse_sweeps, grid);
    }
    for (int l = (ls < ng ? ls : ng - 1); l >= 1; --l) {
      g_prolong(a.L[l], a.L[l + 1], grid);
      g_smooth(a.L[l], a.omega, a.nu_post, grid);
    }
    // u += e (FP64)
    grid_rows(1, L1.n2 + 1, 1, L1.n3 + 1, [&](int j, int k) {
      for (int i = 1 + lane; i <= L1.n1 + 1; i += 32) {
        const long long q = L1.g(i, j, k);
        if (L1.bc[q] <= 0) a.u[q] = a.u[q] + (double)L1.e[q];
      }
    });
    grid.sync();
    ++it;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out_i[0] = it;
    a.out_i[1] = status;
    a.out_d[0] = res;
    a.out_d[1] = res0;
  }
}

size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

}  // namespace

int launch_pdesolver_mixed(const Dims &d, const double h[3], double *u, const double *b, const int *bcnd,
                           double eps, double omega, int ng, double eps0, int max_refine, int nu_pre,
                           int nu_post, int coarse_sweeps, int *iters, double *res_out, cudaStream_t s) {
  if (ng < 1 || ng > XM_MAX) return LEPIC_ERR_ARG;
  const int n[3] = {d.n1, d.n2, d.n3};
  for (int q = 0; q < 3; ++q)
    if (n[q] % (1 << (ng - 1))) return LEPIC_ERR_ARG;
  Ctx &c = ctx();
  XArgs A;
  memset(&A, 0, sizeof(A));
  A.ng = ng;
  A.max_refine = max_refine;
  A.nu_pre = nu_pre;
  A.nu_post = nu_post;
  A.coarse_sweeps = coarse_sweeps;
  A.omega = (float)omega;
  A.u = u;
  A.b = b;
  A.eps = eps;
  char nm[32];
  for (int l = 1; l <= ng; ++l) {
    XLev &L = A.L[l];
    L.n1 = n[0] >> (l - 1);
    L.n2 = n[1] >> (l - 1);
    L.n3 = n[2] >> (l - 1);
    L.N1 = L.n1 + 3;
    L.N2 = L.n2 + 3;
    L.R1 = L.n1 + 2;
    L.R2 = L.n2 + 2;
    double hl[3];
    for (int q = 0; q < 3; ++q) hl[q] = h[q] * (double)(1 << (l - 1));
    const double aw = eps0 / (hl[0] * hl[0]), an = eps0 / (hl[1] * hl[1]), at = eps0 / (hl[2] * hl[2]);
    const double ac = -(an + an + aw + aw + at + at);
    if (l == 1) {
      A.aw = A.ae = aw;
      A.an = A.as = an;
      A.at = A.ab = at;
      A.ac = ac;
    }
    L.aw = L.ae = (float)aw;
    L.an = L.as = (float)an;
    L.at = L.ab = (float)at;
    L.ac = (float)ac;
    const size_t nn = (size_t)L.nn(), nr = (size_t)L.nr();
    snprintf(nm, sizeof nm, "xm_e%d", l);
    L.e = (float *)scratch(nm, sizeof(float) * nn);
    snprintf(nm, sizeof nm, "xm_r%d", l);
    L.r = (float *)scratch(nm, sizeof(float) * nr);
    snprintf(nm, sizeof nm, "xm_rf%d", l);
    L.rf = (float *)scratch(nm, sizeof(float) * nn);
    if (l == 1) {
      L.bc = const_cast<int *>(bcnd);
    } else {
      snprintf(nm, sizeof nm, "xm_bc%d", l);
      L.bc = (int *)scratch(nm, sizeof(int) * nn);
    }
    if (!L.e || !L.r || !L.rf || !L.bc) return LEPIC_ERR_CUDA;
    LEPIC_CUDA(cudaMemsetAsync(L.rf, 0, sizeof(float) * nn, s));
    LEPIC_CUDA(cudaMemsetAsync(L.e, 0, sizeof(float) * nn, s));
  }
  // the coarse levels that fit in shared memory (level 1 stays on the grid)
  size_t smem = 0;
  A.ls = ng;
  for (int l = ng; l >= 2; --l) {
    const XLev &L = A.L[l];
    const size_t need = align16(4 * L.nn()) * 3 + align16(4 * L.nr());
    if (smem + need > XM_SMEM_BUDGET) break;
    A.so_e[l] = (unsigned)smem;
    A.so_rf[l] = (unsigned)(smem + align16(4 * L.nn()));
    A.so_bc[l] = (unsigned)(smem + 2 * align16(4 * L.nn()));
    A.so_r[l] = (unsigned)(smem + 3 * align16(4 * L.nn()));
    smem += need;
    A.ls = l - 1;
  }
  if (A.ls == ng) smem = 0;
  A.alpha = fabs((double)((n[0] + 1) * (n[1] + 1) * (n[2] + 1)) * A.ac) * 1.0;
  LEPIC_CUDA(cudaFuncSetAttribute(k_refine_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  LEPIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_refine_mixed, XM_BLOCK, smem));
  if (occ < 1) return LEPIC_ERR_CUDA;
  const int blocks = c.sms * (occ < 2 ? occ : 2);
  A.partial = (double *)scratch("xm_partial", sizeof(double) * blocks);
  A.out_i = (int *)scratch("xm_out_i", sizeof(int) * 4);
  A.out_d = (double *)scratch("xm_out_d", sizeof(double) * 2);
  XArgs *dA = (XArgs *)scratch("xm_args", sizeof(XArgs));
  if (!A.partial || !A.out_i || !A.out_d || !dA) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemcpyAsync(dA, &A, sizeof(XArgs), cudaMemcpyHostToDevice, s));
  void *args[] = {&dA};
  int tm = timer_start("pdesolver_mixed", s);
  LEPIC_CUDA(cudaLaunchCooperativeKernel((void *)k_refine_mixed, dim3(blocks), dim3(XM_BLOCK), args, smem, s));
  timer_stop(tm, s);
  int hi[4];
  double hd[2];
  LEPIC_CUDA(cudaMemcpyAsync(hi, A.out_i, sizeof(hi), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(hd, A.out_d, sizeof(hd), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (iters) *iters = hi[0];
  if (res_out) *res_out = hd[0];
  return hi[1];
}

}  // namespace lepic

extern "C" int lepic_dev_pdesolver_mixed(const lepic_grid_t *g, double *u, const double *b, double eps,
                                         double omega, int ng, const lepic_phys_t *P, int max_refine,
                                         int nu_pre, int nu_post, int coarse_sweeps, int *iters,
                                         double *res, void *stream) {
  if (!g || !P) return LEPIC_ERR_ARG;
  if (P->flag_pbc || P->flag_nmn) return LEPIC_ERR_UNSUPPORTED;
  return lepic::launch_pdesolver_mixed(lepic::Dims(g->n), g->h, u, b, g->bcnd, eps, omega, ng, P->eps0,
                                       max_refine, nu_pre, nu_post, coarse_sweeps, iters, res,
                                       (cudaStream_t)stream);
}
