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
  int max_refine, nu_fine_pre, nu_fine_post, nu_pre, nu_post, coarse_sweeps;  // sweeps: finest level, the others
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

// deterministic grid-wide sum of one value per thread.  The block partials
// alternate between two halves of a.partial (parity), so one barrier
// suffices: a half is rewritten two sums later, after further barriers.
__device__ double grid_sum(const XArgs &a, double v, int parity, cg::grid_group &grid, double *sh) {
  double *part = a.partial + (parity & 1) * gridDim.x;
  double p = bsum(v, sh);
  if (threadIdx.x == 0) part[blockIdx.x] = p;
  grid.sync();
  double s = 0.0;
  if (threadIdx.x < 32) {
    for (int bI = threadIdx.x; bI < (int)gridDim.x; bI += 32) s += part[bI];
    s = wsum(s);
    if (threadIdx.x == 0) sh[33] = s;
  }
  __syncthreads();
  s = sh[33];
  __syncthreads();
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
// (Src/mg.f90:248-805): loads only; 0 outside the interior and on walls
__device__ __forceinline__ float restrict_value(const XLev &F, const XLev &C, int i, int j, int k) {
  if (i < 1 || j < 1 || k < 1 || i > C.n1 + 1 || j > C.n2 + 1 || k > C.n3 + 1) return 0.f;
  if (C.bc[C.g(i, j, k)] > 0) return 0.f;
  const long long sy = F.N1, sz = (long long)F.N1 * F.N2;
  const long long q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
  const float *R = F.rf;
  return (8.f * R[q] + 4.f * (R[q + 1] + R[q - 1] + R[q + sy] + R[q - sy] + R[q + sz] + R[q - sz]) +
          2.f * (R[q + 1 + sy] + R[q - 1 + sy] + R[q + 1 - sy] + R[q - 1 - sy] + R[q + 1 + sz] + R[q - 1 + sz] +
                 R[q + sy + sz] + R[q - sy + sz] + R[q + 1 - sz] + R[q - 1 - sz] + R[q + sy - sz] +
                 R[q - sy - sz]) +
          R[q + 1 + sy + sz] + R[q - 1 + sy + sz] + R[q + 1 - sy + sz] + R[q - 1 - sy + sz] + R[q + 1 + sy - sz] +
          R[q - 1 + sy - sz] + R[q + 1 - sy - sz] + R[q - 1 - sy - sz]) *
         (1.f / 64.f);
}

// coarse node (i,j,k), i,j,k in 0..n+2: right-hand side from the fine
// residual, correction cleared
__device__ __forceinline__ void restrict_store(const XLev &C, int i, int j, int k, float re) {
  C.e[C.g(i, j, k)] = 0.f;
  if (i <= C.n1 + 1 && j <= C.n2 + 1 && k <= C.n3 + 1) C.r[C.rr(i, j, k)] = re;
}

__device__ __forceinline__ void restrict_node(const XLev &F, const XLev &C, int i, int j, int k) {
  restrict_store(C, i, j, k, restrict_value(F, C, i, j, k));
}

// trilinear prolongation of coarse node (i,j,k) added into F
// (Src/mg.f90:849-939): the 8 coarse values, the 8 fine masks and the 8 fine
// values are loaded before the 8 stores
__device__ __forceinline__ void prolong_node(const XLev &F, const XLev &C, int i, int j, int k) {
  const long long sy = F.N1, sz = (long long)F.N1 * F.N2, cy = C.N1, cz = (long long)C.N1 * C.N2;
  const long long c = C.g(i, j, k);
  const float *E = C.e;
  const float r000 = E[c], r0m0 = E[c - cy], rmm0 = E[c - 1 - cy], rm00 = E[c - 1];
  const float r00m = E[c - cz], r0mm = E[c - cy - cz], rmmm = E[c - 1 - cy - cz], rm0m = E[c - 1 - cz];
  const long long q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
  float *U = F.e;
  const int *B = F.bc;
  const long long o[8] = {0, -sy, -1 - sy, -1, -sz, -sy - sz, -1 - sz, -1 - sy - sz};
  int bm[8];
  float uv[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) {
    bm[t] = B[q + o[t]];
    uv[t] = U[q + o[t]];
  }
  const float add[8] = {r000,
                        (r000 + r0m0) * 0.5f,
                        (r000 + r0m0 + rmm0 + rm00) * 0.25f,
                        (r000 + rm00) * 0.5f,
                        (r000 + r00m) * 0.5f,
                        (r000 + r00m + r0mm + r0m0) * 0.25f,
                        (r000 + r00m + rm0m + rm00) * 0.25f,
                        (r000 + r00m + rm0m + rm00 + r0m0 + r0mm + rmmm + rmm0) * 0.125f};
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (bm[t] <= 0) U[q + o[t]] = uv[t] + add[t];
}

__device__ __forceinline__ int fmapx(int ic, int ncell) {
  return ic == ncell / 2 + 2 ? ncell + 2 : (ic == 0 ? 0 : 2 * ic - 1);
}

// The rows (j, k), j in [j0, j0 + nj), k in [k0, k0 + nk), dealt round-robin
// to all warps of the grid; body(j, k) runs on all lanes, which split the row
// along i.
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

// ------------------------------------------------------------ grid-wide
// The grid levels are small enough to stay in L2 (a 128^3 level of FP32
// arrays is 9 MB each), so a phase costs the latency of its dependent loads,
// not bandwidth.  Each thread therefore takes XU slots of a flat index range
// at once (slot t, t + nth, ...), issues every load of all XU slots before
// the first arithmetic, then computes and stores: one round trip to L2 per
// XU slots instead of two per node.
constexpr int XU = 2;

struct Slots {
  int tid, nth;
};
__device__ __forceinline__ Slots slots() {
  return {(int)(blockIdx.x * blockDim.x + threadIdx.x), (int)(gridDim.x * blockDim.x)};
}

// one red-black half-sweep of level L (slots: (m, j, k), i = start + 2m);
// with u, the finest level's last half-sweep also adds the new correction of
// its nodes to the FP64 solution
__device__ __noinline__ void g_half_sweep(const XLev &L, float omega, int colour, Slots S, double *u = nullptr) {
  const int half = (L.n1 + 2) / 2, nrow = L.n2 + 1;
  const int total = half * nrow * (L.n3 + 1);
  const long long sy = L.N1, sz = (long long)L.N1 * L.N2;
  const float rac = 1.f / L.ac;
  for (int base = S.tid; base < total; base += XU * S.nth) {
    long long q[XU], rq[XU];
    bool ok[XU];
#pragma unroll
    for (int v = 0; v < XU; ++v) {
      const int t = base + v * S.nth;
      ok[v] = false;
      q[v] = rq[v] = 0;
      if (t < total) {
        const int row = t / half, m = t - row * half;
        const int k = row / nrow + 1, j = row - (k - 1) * nrow + 1;
        const int i = colour_start(colour, j, k) + 2 * m;
        if (i <= L.n1 + 1) {
          ok[v] = true;
          q[v] = L.g(i, j, k);
          rq[v] = L.rr(i, j, k);
        }
      }
    }
    int bc[XU];
    float r[XU], c0[XU], ew[XU], en[XU], es[XU], ee[XU], et[XU], eb[XU];
#pragma unroll
    for (int v = 0; v < XU; ++v) {
      if (!ok[v]) continue;
      const long long w = q[v];
      bc[v] = L.bc[w];
      r[v] = L.r[rq[v]];
      c0[v] = L.e[w];
      ew[v] = L.e[w - 1];
      en[v] = L.e[w + sy];
      es[v] = L.e[w - sy];
      ee[v] = L.e[w + 1];
      et[v] = L.e[w + sz];
      eb[v] = L.e[w - sz];
    }
    double uo[XU];
    if (u) {
#pragma unroll
      for (int v = 0; v < XU; ++v)
        if (ok[v] && bc[v] <= 0) uo[v] = u[q[v]];
    }
#pragma unroll
    for (int v = 0; v < XU; ++v) {
      if (!ok[v] || bc[v] > 0) continue;
      const float tt = r[v] - L.aw * ew[v] - L.an * en[v] - L.as * es[v] - L.ae * ee[v] - L.at * et[v] -
                       L.ab * eb[v];
      const float en1 = (1.f - omega) * c0[v] + omega * tt * rac;
      L.e[q[v]] = en1;
      if (u) u[q[v]] = uo[v] + (double)en1;
    }
  }
}

// u += e on the nodes of one colour (their correction is final)
__device__ __noinline__ void g_add_colour(const XLev &L, int colour, Slots S, double *u) {
  const int half = (L.n1 + 2) / 2, nrow = L.n2 + 1;
  const int total = half * nrow * (L.n3 + 1);
  for (int base = S.tid; base < total; base += XU * S.nth) {
    long long q[XU];
    bool ok[XU];
#pragma unroll
    for (int v = 0; v < XU; ++v) {
      const int t = base + v * S.nth;
      ok[v] = false;
      q[v] = 0;
      if (t < total) {
        const int row = t / half, m = t - row * half;
        const int k = row / nrow + 1, j = row - (k - 1) * nrow + 1;
        const int i = colour_start(colour, j, k) + 2 * m;
        if (i <= L.n1 + 1) {
          ok[v] = true;
          q[v] = L.g(i, j, k);
        }
      }
    }
    int bc[XU];
    float ev[XU];
    double uo[XU];
#pragma unroll
    for (int v = 0; v < XU; ++v) {
      if (!ok[v]) continue;
      bc[v] = L.bc[q[v]];
      ev[v] = L.e[q[v]];
      uo[v] = u[q[v]];
    }
#pragma unroll
    for (int v = 0; v < XU; ++v)
      if (ok[v] && bc[v] <= 0) u[q[v]] = uo[v] + (double)ev[v];
  }
}

// nsweep red-black sweeps; with u (finest level, last smoothing of the
// cycle) the last half-sweep also accumulates u += e on every node
__device__ __noinline__ void g_smooth(const XLev &L, float omega, int nsweep, cg::grid_group &grid, double *u = nullptr) {
  const Slots S = slots();
  for (int s = 0; s < nsweep; ++s) {
    for (int colour = 0; colour < 2; ++colour) {
      const bool last = u && s == nsweep - 1 && colour == 1;
      g_half_sweep(L, omega, colour, S, last ? u : nullptr);
      if (last) g_add_colour(L, 0, S, u);
      grid.sync();
    }
  }
}

// fine residual rf = r - A e on the interior nodes (0 on walls)
__device__ __noinline__ void g_residual(const XLev &F, Slots S) {
  const int ni = F.n1 + 1, nj = F.n2 + 1;
  const int total = ni * nj * (F.n3 + 1);
  const long long sy = F.N1, sz = (long long)F.N1 * F.N2;
  for (int base = S.tid; base < total; base += XU * S.nth) {
    long long q[XU], rq[XU];
    bool ok[XU];
#pragma unroll
    for (int u = 0; u < XU; ++u) {
      const int t = base + u * S.nth;
      ok[u] = t < total;
      q[u] = rq[u] = 0;
      if (ok[u]) {
        const int row = t / ni, i = t - row * ni + 1;
        const int k = row / nj + 1, j = row - (k - 1) * nj + 1;
        q[u] = F.g(i, j, k);
        rq[u] = F.rr(i, j, k);
      }
    }
    int bc[XU];
    float r[XU], c0[XU], ew[XU], en[XU], es[XU], ee[XU], et[XU], eb[XU];
#pragma unroll
    for (int u = 0; u < XU; ++u) {
      if (!ok[u]) continue;
      const long long v = q[u];
      bc[u] = F.bc[v];
      r[u] = F.r[rq[u]];
      c0[u] = F.e[v];
      ew[u] = F.e[v - 1];
      en[u] = F.e[v + sy];
      es[u] = F.e[v - sy];
      ee[u] = F.e[v + 1];
      et[u] = F.e[v + sz];
      eb[u] = F.e[v - sz];
    }
#pragma unroll
    for (int u = 0; u < XU; ++u) {
      if (!ok[u]) continue;
      F.rf[q[u]] = bc[u] > 0 ? 0.f
                             : r[u] - (F.aw * ew[u] + F.ae * ee[u] + F.an * en[u] + F.as * es[u] +
                                       F.ac * c0[u] + F.at * et[u] + F.ab * eb[u]);
    }
  }
}

__device__ __noinline__ void g_restrict(const XLev &F, const XLev &C, cg::grid_group &grid) {
  const Slots S = slots();
  g_residual(F, S);
  grid.sync();
  const int ni = C.n1 + 3, nj = C.n2 + 3;
  const int total = ni * nj * (C.n3 + 3);
  // one coarse node per iteration: its 27 loads are already independent
  for (int t = S.tid; t < total; t += S.nth) {
    const int row = t / ni, i = t - row * ni;
    const int k = row / nj, j = row - k * nj;
    restrict_node(F, C, i, j, k);
  }
  grid.sync();
}

__device__ __noinline__ void g_prolong(const XLev &F, const XLev &C, cg::grid_group &grid) {
  const Slots S = slots();
  const int ni = C.n1 + 1, nj = C.n2 + 1;
  const int total = ni * nj * (C.n3 + 1);
  // one coarse node per iteration: its 24 loads are already independent
  for (int t = S.tid; t < total; t += S.nth) {
    const int row = t / ni, i = t - row * ni + 1;
    const int k = row / nj + 1, j = row - (k - 1) * nj + 1;
    prolong_node(F, C, i, j, k);
  }
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
__device__ __noinline__ void coarse_cycle(const XArgs &a, unsigned char *sm) {
  const int top = a.ls + 1, ng = a.ng;
  {
    // four independent loads in flight per thread
    const XLev G = a.L[top], S = smem_level(a, top, sm);
    const int nr = (int)G.nr(), nt = (int)blockDim.x;
    for (int t0 = threadIdx.x; t0 < nr; t0 += 4 * nt) {
      float v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) v[u] = t0 + u * nt < nr ? G.r[t0 + u * nt] : 0.f;
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (t0 + u * nt < nr) S.r[t0 + u * nt] = v[u];
    }
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

// FP64 residual b - A u of the finest level on its interior nodes, written
// as the FP32 right-hand side of the V-cycle (0 on walls); returns this
// thread's share of the L1 norm over the plasma nodes (bcnd = -1)
__device__ __noinline__ double g_residual_f64(const XArgs &a, const XLev &L1, Slots S) {
  constexpr int U = 2;
  const int ni = L1.n1 + 1, nj = L1.n2 + 1;
  const int total = ni * nj * (L1.n3 + 1);
  const long long sy = L1.N1, sz = (long long)L1.N1 * L1.N2;
  const double *u = a.u;
  double acc = 0.0;
  for (int base = S.tid; base < total; base += U * S.nth) {
    long long q[U], rq[U];
    bool ok[U];
#pragma unroll
    for (int v = 0; v < U; ++v) {
      const int t = base + v * S.nth;
      ok[v] = t < total;
      q[v] = rq[v] = 0;
      if (ok[v]) {
        const int row = t / ni, i = t - row * ni + 1;
        const int k = row / nj + 1, j = row - (k - 1) * nj + 1;
        q[v] = L1.g(i, j, k);
        rq[v] = L1.rr(i, j, k);
      }
    }
    int bc[U];
    double bv[U], c0[U], uw[U], un[U], us[U], ue[U], ut[U], ub[U];
#pragma unroll
    for (int v = 0; v < U; ++v) {
      if (!ok[v]) continue;
      const long long w = q[v];
      bc[v] = L1.bc[w];
      bv[v] = a.b[rq[v]];
      c0[v] = u[w];
      uw[v] = u[w - 1];
      un[v] = u[w + sy];
      us[v] = u[w - sy];
      ue[v] = u[w + 1];
      ut[v] = u[w + sz];
      ub[v] = u[w - sz];
    }
#pragma unroll
    for (int v = 0; v < U; ++v) {
      if (!ok[v]) continue;
      double rv = 0.0;
      if (bc[v] <= 0) {
        rv = bv[v] - (a.aw * uw[v] + a.an * un[v] + a.as * us[v] + a.ae * ue[v] + a.ac * c0[v] + a.at * ut[v] +
                      a.ab * ub[v]);
        if (bc[v] == -1) acc += fabs(rv);
      }
      L1.r[rq[v]] = (float)rv;
    }
  }
  return acc;
}

__global__ void __launch_bounds__(XM_BLOCK, 1) k_refine_mixed(const XArgs *__restrict__ ap) {
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
  const Slots S = slots();
  double res = 0.0, res0 = -1.0;
  int it = 0, status = 0;
  for (;;) {
    // FP64 residual, FP32 copy as the V-cycle right-hand side, e = 0
    const double acc = g_residual_f64(a, L1, S);
    for (long long t = S.tid; t < L1.nn(); t += S.nth) L1.e[t] = 0.f;
    res = grid_sum(a, acc, it, grid, sh) / a.alpha;
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
    // chip, grid levels up; the last smoothing of level 1 also applies
    // u += e (FP64)
    for (int l = 1; l <= ls && l < ng; ++l) {
      g_smooth(a.L[l], a.omega, l == 1 ? a.nu_fine_pre : a.nu_pre, grid);
      g_restrict(a.L[l], a.L[l + 1], grid);
    }
    bool added = false;
    if (ls < ng) {
      if (blockIdx.x == 0) coarse_cycle(a, smem);
      grid.sync();
    } else {
      added = ng == 1 && a.coarse_sweeps > 0;
      g_smooth(a.L[ng], a.omega, a.coarse_sweeps, grid, added ? a.u : nullptr);
    }
    for (int l = (ls < ng ? ls : ng - 1); l >= 1; --l) {
      g_prolong(a.L[l], a.L[l + 1], grid);
      const int nu = l == 1 ? a.nu_fine_post : a.nu_post;
      const bool fin = l == 1 && nu > 0;
      g_smooth(a.L[l], a.omega, nu, grid, fin ? a.u : nullptr);
      added = added || fin;
    }
    if (!added) {
      g_add_colour(L1, 0, S, a.u);
      g_add_colour(L1, 1, S, a.u);
      grid.sync();
    }
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
                           double eps, double omega, int ng, double eps0, int max_refine, int nu_fine_pre,
                           int nu_fine_post, int nu_pre, int nu_post, int coarse_sweeps, int *iters,
                           double *res_out, cudaStream_t s) {
  if (ng < 1 || ng > XM_MAX) return LEPIC_ERR_ARG;
  const int n[3] = {d.n1, d.n2, d.n3};
  for (int q = 0; q < 3; ++q)
    if (n[q] % (1 << (ng - 1))) return LEPIC_ERR_ARG;
  Ctx &c = ctx();
  XArgs A;
  memset(&A, 0, sizeof(A));
  A.ng = ng;
  A.max_refine = max_refine;
  A.nu_fine_pre = nu_fine_pre;
  A.nu_fine_post = nu_fine_post;
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
  A.partial = (double *)scratch("xm_partial", sizeof(double) * 2 * blocks);
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
                                         int nu_fine_pre, int nu_fine_post, int nu_pre, int nu_post,
                                         int coarse_sweeps, int *iters, double *res, void *stream) {
  if (!g || !P) return LEPIC_ERR_ARG;
  if (P->flag_pbc || P->flag_nmn) return LEPIC_ERR_UNSUPPORTED;
  if (nu_fine_pre < 0 || nu_fine_post < 0 || nu_pre < 0 || nu_post < 0 || coarse_sweeps < 0 || max_refine < 0)
    return LEPIC_ERR_ARG;
  return lepic::launch_pdesolver_mixed(lepic::Dims(g->n), g->h, u, b, g->bcnd, eps, omega, ng, P->eps0,
                                       max_refine, nu_fine_pre, nu_fine_post, nu_pre, nu_post, coarse_sweeps,
                                       iters, res, (cudaStream_t)stream);
}
