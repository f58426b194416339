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
// the V-cycle moves half the bytes.
//
// Wall nodes are marked in the FP32 right-hand side itself: r = +inf on a
// wall or ghost node (never updated; its correction stays 0), so the FP32
// levels carry no mask arrays.  The coarse masks are the reference's
// injection (Src/mg.f90:429-436): a coarse node is a wall when the fine node
// it sits on is one.
//
// Grid levels (those too large for one SM's shared memory) are processed in
// 3D tiles of 32 x 8 x 8 nodes staged in shared memory by the tensor memory
// accelerator: per tile a block loads the boxes of e and r covering the tile
// and two halo layers with cp.async.bulk.tensor (double-buffered: the next
// tile's copy is in flight while the current one is computed, completion on
// an mbarrier), and works on chip:
//   sweep      red nodes of tile + 1 halo layer, then black nodes of the tile
//              (a full red-black sweep per grid phase; the halo's red values
//              are computed redundantly by the neighbouring tiles);
//   restrict   the fine residual on tile + 1 halo layer, then the 27-point
//              weighting onto the coarse nodes whose fine twin lies in the
//              tile (one grid phase instead of two);
//   prolong    the coarse correction's box is staged as well and added before
//              the first post-sweep of the level, in the same phase.
// The last post-sweep of level 1 also adds the correction to u (FP64).  The
// coarse levels, from the first one whose arrays fit in shared memory down
// to the coarsest, run in block 0 alone for each V-cycle, with block
// barriers only, in the same shared memory.
//
// Every wait on a tile copy is bounded (one second); a copy that never
// completes sets LEPIC_ERR_TIMEOUT in the device error word, the block stops
// issuing copies and computing, and still meets every grid barrier.
#include <cooperative_groups.h>
#include <cuda.h>

#include <cstring>

#include "lepic_internal.cuh"

namespace cg = cooperative_groups;

namespace lepic {

namespace {

constexpr int XM_MAX = 13;      // multigrid levels
constexpr int GMAX = 6;         // levels in global memory (tiled)
constexpr int XM_BLOCK = 512;
constexpr size_t XM_SMEM_COARSE = 160 * 1024;   // budget of the on-chip coarse levels

// tile of updated nodes; the last tile of a row takes the remainder, up to
// T + 1 nodes (the node n + 1).  TX = 32 puts every fine box on a 16-byte
// boundary (column 32 t) and every coarse box too (column 16 t); a row of one
// colour of the tile and its halo (at most 18 nodes) is one warp's.  (A
// 24-node tile with a row per half-warp was slower at 128^3: 6 tiles per
// row of 129 nodes instead of 4.)
constexpr int TX = 32, TY = 8, TZ = 8;
// staged boxes: the fine box is the tile with two halo layers on each side
// (one more for a last tile), the coarse box covers what the fine box's
// nodes interpolate from
constexpr int BX = TX + 8, BY = TY + 5, BZ = TZ + 5;
constexpr int CBX = TX / 2 + 4, CBY = TY / 2 + 4, CBZ = TZ / 2 + 4;
constexpr int BXY = BX * BY;
constexpr unsigned BOX_BYTES = BX * BY * BZ * 4u;
constexpr unsigned CBOX_BYTES = CBX * CBY * CBZ * 4u;
constexpr unsigned BOX_STRIDE = (BOX_BYTES + 127u) / 128u * 128u;
constexpr unsigned CBOX_STRIDE = (CBOX_BYTES + 127u) / 128u * 128u;
constexpr unsigned STAGE_BYTES = 2 * BOX_STRIDE + CBOX_STRIDE;  // e box, r box, coarse e box
constexpr unsigned TILE_SMEM = 2 * STAGE_BYTES + BOX_STRIDE;     // two stages + the residual box

// A level in global memory: FP32 e and r over nodes 0..n+2 per axis, node
// (i, j, k) at column i + 1 of a row padded to a multiple of 4 floats (so
// that every tile box starts on a 16-byte boundary, x = 32 t).
struct GLev {
  int n1, n2, n3;
  int P1;              // row pitch, floats
  int ntx, nty, ntz;   // tiles per axis
  float aw, an, at, ac;
  float *e[2];         // the correction, two buffers (a sweep reads one, writes the other)
  float *r;
  __host__ __device__ long long g(int i, int j, int k) const {
    return (long long)(i + 1) + (long long)P1 * (j + (long long)(n2 + 3) * k);
  }
  __host__ __device__ long long nn() const { return (long long)P1 * (n2 + 3) * (n3 + 3); }
};

// A coarse level in block 0's shared memory: nodes 0..n+2, x fastest.
struct SLev {
  int n1, n2, n3;
  int N1, N2;          // n + 3
  float aw, an, at, ac;
  float *e, *r, *rf;
  __device__ int g(int i, int j, int k) const { return i + N1 * (j + N2 * k); }
};

struct XArgs {
  GLev G[GMAX + 2];    // levels 1..min(ls + 1, ng): the grid levels and the exchange level
  SLev S[XM_MAX + 1];  // levels ls + 1..ng on chip (pointers are shared-memory offsets, set per block)
  unsigned so_e[XM_MAX + 1], so_r[XM_MAX + 1], so_rf[XM_MAX + 1];
  int ng, ls;          // levels 1..ls on the grid, ls+1..ng in shared memory
  int max_refine, nu_fine_pre, nu_fine_post, nu_pre, nu_post, coarse_sweeps;
  float omega;
  double aw, an, at, ac;  // FP64 finest coefficients (ae = aw, as = an, ab = at)
  double *u;
  const double *b;
  const int *bcnd;
  double alpha, eps;
  double *partial;
  int *out_i;      // [0] refinement iterations, [1] status
  double *out_d;   // [0] res/alpha, [1] first res/alpha
  int *err;        // device error word
};

// tensor maps of the tile boxes (a __grid_constant__ kernel parameter)
struct XMaps {
  CUtensorMap fe[GMAX + 1][2], fr[GMAX + 1];  // fine boxes of e (both buffers) and r, levels 1..ls
  CUtensorMap ce[GMAX + 2][2];                // coarse boxes of e, levels 2..ls + 1
};

__device__ __forceinline__ bool wall(float r) { return isinf(r); }

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

// ------------------------------------------------------------ tile copies
__device__ __forceinline__ void tma_box(uint32_t dst, const CUtensorMap *m, int x, int y, int z, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
      "[%5];" ::"r"(dst),
      "l"(reinterpret_cast<unsigned long long>(m)), "r"(x), "r"(y), "r"(z), "r"(bar)
      : "memory");
}

// The dynamic shared memory of the kernel: the tile stages (grid phases) or
// the coarse levels (block 0's coarse cycle).  Box pointers are formed from
// this symbol so that the compiler addresses them as shared memory.
extern __shared__ __align__(128) unsigned char xm_smem[];

// The double-buffered tile copies of one block.
struct Pipe {
  int base;               // offset of the first 128-byte boundary in xm_smem
  uint32_t bar[2];        // mbarriers in shared memory
  unsigned uses[2];       // completed phases per mbarrier
  bool fail;
};

enum { K_SWEEP = 1, K_PRO = 2, K_RESTRICT = 4, K_ADDU = 8 };

struct Tile {
  int tx, ty, tz;
  int i0, j0, k0;   // node of box index 0 on each axis
  int w, h, d;      // tile nodes per axis
};

__device__ __forceinline__ Tile tile_of(const GLev &L, int tau) {
  Tile t;
  t.tx = tau % L.ntx;
  const int q = tau / L.ntx;
  t.ty = q % L.nty;
  t.tz = q / L.nty;
  t.i0 = TX * t.tx - 1;
  t.j0 = TY * t.ty - 1;
  t.k0 = TZ * t.tz - 1;
  t.w = t.tx == L.ntx - 1 ? L.n1 + 1 - TX * t.tx : TX;
  t.h = t.ty == L.nty - 1 ? L.n2 + 1 - TY * t.ty : TY;
  t.d = t.tz == L.ntz - 1 ? L.n3 + 1 - TZ * t.tz : TZ;
  return t;
}

// thread 0: the copies of tile tau of level l into stage s; ein / cin: the
// e buffers read (level l, level l + 1)
__device__ void issue(const XMaps &maps, int l, int kind, const GLev &L, int tau, Pipe &pp, int s, int ein,
                      int cin) {
  const Tile t = tile_of(L, tau);
  const unsigned bytes = 2 * BOX_BYTES + ((kind & K_PRO) ? CBOX_BYTES : 0u);
  // earlier generic accesses of this stage come before the asynchronous copy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(pp.bar[s]), "r"(bytes) : "memory");
  const uint32_t dst = smem_addr(xm_smem + pp.base + s * STAGE_BYTES);
  tma_box(dst, &maps.fe[l][ein], TX * t.tx, t.j0, t.k0, pp.bar[s]);
  tma_box(dst + BOX_STRIDE, &maps.fr[l], TX * t.tx, t.j0, t.k0, pp.bar[s]);
  if (kind & K_PRO)
    tma_box(dst + 2 * BOX_STRIDE, &maps.ce[l + 1][cin], (TX / 2) * t.tx, (TY / 2) * t.ty - 1, (TZ / 2) * t.tz - 1,
            pp.bar[s]);
}

// The rows (y, z) of the region [x0, x0 + nx) x [y0, y0 + ny) x [z0, z0 + nz)
// dealt to the warps of the block, the lanes along x: body(x, y, z).  The
// row coordinates advance by the warp count without divisions.
template <class F>
__device__ __forceinline__ void box_rows(int x0, int nx, int y0, int ny, int z0, int nz, F &&body) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  int zz = wp / ny, yy = wp - zz * ny;
#pragma unroll 2
  for (; zz < nz;) {
    const int y = y0 + yy, z = z0 + zz;
    for (int x = x0 + lane; x < x0 + nx; x += 32) body(x, y, z);
    yy += nw;
    while (yy >= ny) {
      yy -= ny;
      ++zz;
    }
  }
}

// one red-black colour (red = (i + j + k) odd, Src/sors.f90:87-106) of the box
// region [x0, x0 + nx) x ... relaxed in place (the Src/sors.f90 update, in
// FP32): each warp takes a row (at most 32 nodes of one colour: nx <= 64),
// its rows advance by the warp count.  Every load of a node is issued before
// its wall test; walls keep their value.
__device__ __forceinline__ void relax_colour(float *E, const float *R, const Tile &t, int x0, int nx, int y0, int ny,
                                             int z0, int nz, bool red, float aw, float an, float at, float om,
                                             float rac) {
  const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int p0 = (t.i0 + x0 + t.j0 + y0 + t.k0 + z0 + (red ? 1 : 0)) & 1;   // 1: the row's first node is off colour
  int zz = wp / ny, yy = wp - zz * ny;
#pragma unroll 2
  for (; zz < nz;) {
    const int bx = x0 + ((p0 + yy + zz) & 1) + 2 * lane;
    const int q = bx + BX * (y0 + yy + BY * (z0 + zz));
    if (bx < x0 + nx) {
      const float rv = R[q], e0 = E[q], ew = E[q - 1], ee = E[q + 1], en = E[q + BX], es = E[q - BX],
                  et = E[q + BXY], eb = E[q - BXY];
      const float tt = rv - aw * ew - an * en - an * es - aw * ee - at * et - at * eb;
      const float v = (1.f - om) * e0 + om * tt * rac;
      if (!wall(rv)) E[q] = v;
    }
    yy += nw;
    while (yy >= ny) {
      yy -= ny;
      ++zz;
    }
  }
}

// 27-point full weighting (Src/mg.f90:696-702) of the residual box around q
__device__ __forceinline__ float weigh27(const float *F, int q) {
  const int sy = BX, sz = BXY;
  return (8.f * F[q] + 4.f * (F[q + 1] + F[q - 1] + F[q + sy] + F[q - sy] + F[q + sz] + F[q - sz]) +
          2.f * (F[q + 1 + sy] + F[q - 1 + sy] + F[q + 1 - sy] + F[q - 1 - sy] + F[q + 1 + sz] + F[q - 1 + sz] +
                 F[q + sy + sz] + F[q - sy + sz] + F[q + 1 - sz] + F[q - 1 - sz] + F[q + sy - sz] +
                 F[q - sy - sz]) +
          F[q + 1 + sy + sz] + F[q - 1 + sy + sz] + F[q + 1 - sy + sz] + F[q - 1 - sy + sz] + F[q + 1 + sy - sz] +
          F[q - 1 + sy - sz] + F[q + 1 - sy - sz] + F[q - 1 - sy - sz]) *
         (1.f / 64.f);
}

// the work of one staged tile (stage s): sweep / prolong+sweep / restrict;
// eout: the e buffer of level l written
__device__ void tile_work(const GLev &L, const GLev &C, double *u, float omega, int kind, const Tile &t, int base,
                          int s, int eout, int cout) {
  float *E = reinterpret_cast<float *>(xm_smem + base + s * STAGE_BYTES);
  const float *R = reinterpret_cast<const float *>(xm_smem + base + s * STAGE_BYTES + BOX_STRIDE);
  const float aw = L.aw, an = L.an, at = L.at, ac = L.ac;
  const int n1 = L.n1, n2 = L.n2, n3 = L.n3;
  if (kind & K_PRO) {
    // trilinear prolongation (Src/mg.f90:849-939) of the coarse box onto
    // every non-wall node of the fine box inside the grid: a fine node on a
    // coarse node takes its value, one between coarse nodes their mean
    const float *CE = reinterpret_cast<const float *>(xm_smem + base + s * STAGE_BYTES + 2 * BOX_STRIDE);
    const int cx0 = (TX / 2) * t.tx - 1, cy0 = (TY / 2) * t.ty - 1, cz0 = (TZ / 2) * t.tz - 1;
    box_rows(0, t.w + 4, 0, t.h + 4, 0, t.d + 4, [&](int bx, int by, int bz) {
      const int i = t.i0 + bx, j = t.j0 + by, k = t.k0 + bz;
      if (i < 0 || j < 0 || k < 0 || i > n1 + 1 || j > n2 + 1 || k > n3 + 1) return;
      const int q = bx + BX * (by + BY * bz);
      if (wall(R[q])) return;
      const int c = (((i + 1) >> 1) - cx0) + CBX * ((((j + 1) >> 1) - cy0) + CBY * (((k + 1) >> 1) - cz0));
      // weights of the upper neighbour per axis: 0.5 between coarse nodes, 0 on one
      const float wx = (i & 1) ? 0.f : 0.5f, wy = (j & 1) ? 0.f : 0.5f, wz = (k & 1) ? 0.f : 0.5f;
      const float vx = 1.f - wx, vy = 1.f - wy, vz = 1.f - wz;
      const float s0 = vx * CE[c] + wx * CE[c + 1];
      const float s1 = vx * CE[c + CBX] + wx * CE[c + 1 + CBX];
      const float s2 = vx * CE[c + CBX * CBY] + wx * CE[c + 1 + CBX * CBY];
      const float s3 = vx * CE[c + CBX + CBX * CBY] + wx * CE[c + 1 + CBX + CBX * CBY];
      E[q] += vz * (vy * s0 + wy * s1) + wz * (vy * s2 + wy * s3);
    });
    __syncthreads();
  }
  if (kind & K_SWEEP) {
    const float om = omega, rac = 1.f / ac;
    // red on the tile and one halo layer, then black on the tile
    relax_colour(E, R, t, 1, t.w + 2, 1, t.h + 2, 1, t.d + 2, true, aw, an, at, om, rac);
    __syncthreads();
    relax_colour(E, R, t, 2, t.w, 2, t.h, 2, t.d, false, aw, an, at, om, rac);
    __syncthreads();
  }
  if (kind & K_RESTRICT) {
    // residual on the tile and one halo layer (0 on walls), then the coarse
    // nodes whose fine twin (2I-1, 2J-1, 2K-1) lies in the tile (the first
    // and last tiles of a row also set the coarse ghost nodes)
    float *RF = reinterpret_cast<float *>(xm_smem + base + 2 * STAGE_BYTES);
    box_rows(1, t.w + 2, 1, t.h + 2, 1, t.d + 2, [&](int bx, int by, int bz) {
      const int q = bx + BX * (by + BY * bz);
      const float rv = R[q], e0 = E[q], ew = E[q - 1], ee = E[q + 1], en = E[q + BX], es = E[q - BX],
                  et = E[q + BXY], eb = E[q - BXY];
      const float v = rv - (aw * ew + aw * ee + an * en + an * es + ac * e0 + at * et + at * eb);
      RF[q] = wall(rv) ? 0.f : v;
    });
    __syncthreads();
    float *Cr = C.r, *Ce = C.e[cout];
    const int m1 = C.n1, m2 = C.n2, m3 = C.n3, P1 = C.P1;
    const int I0 = t.tx == 0 ? 0 : (TX / 2) * t.tx + 1, I1 = t.tx == L.ntx - 1 ? m1 + 2 : (TX / 2) * (t.tx + 1);
    const int J0 = t.ty == 0 ? 0 : (TY / 2) * t.ty + 1, J1 = t.ty == L.nty - 1 ? m2 + 2 : (TY / 2) * (t.ty + 1);
    const int K0 = t.tz == 0 ? 0 : (TZ / 2) * t.tz + 1, K1 = t.tz == L.ntz - 1 ? m3 + 2 : (TZ / 2) * (t.tz + 1);
    box_rows(I0, I1 - I0 + 1, J0, J1 - J0 + 1, K0, K1 - K0 + 1, [&](int I, int J, int K) {
      float rv = INFINITY;
      if (I >= 1 && J >= 1 && K >= 1 && I <= m1 + 1 && J <= m2 + 1 && K <= m3 + 1) {
        const int q = (2 * I - 1 - t.i0) + BX * ((2 * J - 1 - t.j0) + BY * (2 * K - 1 - t.k0));
        if (!wall(R[q])) rv = weigh27(RF, q);
      }
      const long long o = (long long)(I + 1) + (long long)P1 * (J + (long long)(m2 + 3) * K);
      Cr[o] = rv;
      Ce[o] = 0.f;
    });
  } else {
    // the tile's correction back to the grid (and, last post-sweep of
    // level 1, into the FP64 solution)
    float *Le = L.e[eout];
    const int P1 = L.P1;
    const long long U1 = (long long)n1 + 3, U2 = (long long)n2 + 3;
    box_rows(2, t.w, 2, t.h, 2, t.d, [&](int bx, int by, int bz) {
      const int q = bx + BX * (by + BY * bz);
      const int i = t.i0 + bx, j = t.j0 + by, k = t.k0 + bz;
      const float ev = E[q];
      Le[(long long)(i + 1) + (long long)P1 * (j + (long long)(n2 + 3) * k)] = ev;
      if ((kind & K_ADDU) && !wall(R[q])) {
        double *uq = u + i + U1 * (j + U2 * k);
        *uq = *uq + (double)ev;
      }
    });
  }
}

// One pass of `kind` over the tiles of grid level l, ending at a grid
// barrier.  cur: bit m = the e buffer of level m that holds its correction;
// a sweep reads it and writes the other one, which becomes current (no
// block reads what another block of the same phase writes).
__device__ __noinline__ void tile_pass(const XArgs &a, const XMaps &maps, int l, int kind, Pipe &pp,
                                       cg::grid_group &grid, unsigned &cur) {
  // the level descriptors in shared memory for the whole pass
  __shared__ GLev sL, sC;
  __shared__ double *su;
  __shared__ float som;
  if (threadIdx.x == 0) {
    sL = a.G[l];
    if (kind & K_RESTRICT) sC = a.G[l + 1];
    su = a.u;
    som = a.omega;
  }
  __syncthreads();
  const GLev &L = sL;
  const int NT = L.ntx * L.nty * L.ntz;
  const int ein = (cur >> l) & 1, cin = (cur >> (l + 1)) & 1;
  const int eout = (kind & K_RESTRICT) ? ein : ein ^ 1;
  int tau = blockIdx.x;
  if (tau < NT && threadIdx.x == 0 && !pp.fail) issue(maps, l, kind, L, tau, pp, 0, ein, cin);
  for (int m = 0; tau < NT; tau += gridDim.x, ++m) {
    const int s = m & 1;
    const int nxt = tau + gridDim.x;
    if (nxt < NT && threadIdx.x == 0 && !pp.fail) issue(maps, l, kind, L, nxt, pp, s ^ 1, ein, cin);
    __shared__ int ok;
    if (threadIdx.x == 0) {
      ok = !pp.fail && mbar_wait(pp.bar[s], pp.uses[s] & 1u);
      if (!ok && !pp.fail) {
        pp.fail = true;
        raise_err(a.err, LEPIC_ERR_TIMEOUT, l);
      }
    }
    __syncthreads();
    pp.uses[s] += 1;
    if (ok) tile_work(L, sC, su, som, kind, tile_of(L, tau), pp.base, s, eout, cin);
    __syncthreads();
  }
  if (!(kind & K_RESTRICT)) cur ^= 1u << l;
  // this phase's stores before the next phase's copies read them
  asm volatile("fence.proxy.async.global;" ::: "memory");
  grid.sync();
}

// ------------------------------------------------------ block 0, on chip
// flat loop over the nodes (i, j, k) of a box, 32-bit index arithmetic
template <class F>
__device__ __forceinline__ void block_box(int i0, int ni, int j0, int nj, int k0, int nk, F &&body) {
  const int tot = ni * nj * nk;
  int t = threadIdx.x;
  if (t >= tot) return;
  // (i, j, k) of the thread's first element, then stepped by the block size
  // with carries instead of two integer divisions per element
  const int row0 = t / ni;
  int i = t - row0 * ni, k = row0 / nj, j = row0 - k * nj;
  const int bd = blockDim.x, srow = bd / ni, si = bd - srow * ni;   // bd = srow ni + si
  const int sk = srow / nj, sj = srow - sk * nj;                    // srow = sk nj + sj
  for (; t < tot; t += bd) {
    body(i0 + i, j0 + j, k0 + k);
    i += si;
    j += sj;
    k += sk;
    if (i >= ni) {
      i -= ni;
      ++j;
    }
    if (j >= nj) {
      j -= nj;
      ++k;
    }
  }
}

// red-black colour start: colour 0 = red ((i+j+k) odd), 1 = black
// (Src/sors.f90:87-106, 249-267)
__device__ __forceinline__ int colour_start(int colour, int j, int k) {
  int is = (colour == 0) ? ((j % 2 == 0) ? 1 : 2) : ((j % 2 == 0) ? 2 : 1);
  is += (k % 2 == 0) ? 0 : 1;
  return is > 2 ? 1 : is;
}

__device__ void b_smooth(const SLev &L, float omega, int nsweep) {
  const float rac = 1.f / L.ac;
  const int half = (L.n1 + 2) / 2;
  const int sy = L.N1, sz = L.N1 * L.N2;
  for (int s = 0; s < nsweep; ++s) {
    for (int colour = 0; colour < 2; ++colour) {
      block_box(0, half, 1, L.n2 + 1, 1, L.n3 + 1, [&](int ii, int j, int k) {
        const int i = colour_start(colour, j, k) + 2 * ii;
        if (i > L.n1 + 1) return;
        const int q = L.g(i, j, k);
        const float rv = L.r[q];
        if (wall(rv)) return;
        const float tt = rv - L.aw * L.e[q - 1] - L.an * L.e[q + sy] - L.an * L.e[q - sy] - L.aw * L.e[q + 1] -
                         L.at * L.e[q + sz] - L.at * L.e[q - sz];
        L.e[q] = (1.f - omega) * L.e[q] + omega * tt * rac;
      });
      __syncthreads();
    }
  }
}

__device__ void b_restrict(const SLev &F, const SLev &C) {
  const int sy = F.N1, sz = F.N1 * F.N2;
  // the residual on every node, 0 on ghosts and walls
  block_box(0, F.n1 + 3, 0, F.n2 + 3, 0, F.n3 + 3, [&](int i, int j, int k) {
    const int q = F.g(i, j, k);
    float v = 0.f;
    if (i >= 1 && j >= 1 && k >= 1 && i <= F.n1 + 1 && j <= F.n2 + 1 && k <= F.n3 + 1) {
      const float rv = F.r[q];
      if (!wall(rv))
        v = rv - (F.aw * F.e[q - 1] + F.aw * F.e[q + 1] + F.an * F.e[q + sy] + F.an * F.e[q - sy] + F.ac * F.e[q] +
                  F.at * F.e[q + sz] + F.at * F.e[q - sz]);
    }
    F.rf[q] = v;
  });
  __syncthreads();
  block_box(0, C.n1 + 3, 0, C.n2 + 3, 0, C.n3 + 3, [&](int i, int j, int k) {
    float rv = INFINITY;
    if (i >= 1 && j >= 1 && k >= 1 && i <= C.n1 + 1 && j <= C.n2 + 1 && k <= C.n3 + 1) {
      const int q = F.g(2 * i - 1, 2 * j - 1, 2 * k - 1);
      if (!wall(F.r[q])) {
        const float *R = F.rf;
        rv = (8.f * R[q] + 4.f * (R[q + 1] + R[q - 1] + R[q + sy] + R[q - sy] + R[q + sz] + R[q - sz]) +
              2.f * (R[q + 1 + sy] + R[q - 1 + sy] + R[q + 1 - sy] + R[q - 1 - sy] + R[q + 1 + sz] +
                     R[q - 1 + sz] + R[q + sy + sz] + R[q - sy + sz] + R[q + 1 - sz] + R[q - 1 - sz] +
                     R[q + sy - sz] + R[q - sy - sz]) +
              R[q + 1 + sy + sz] + R[q - 1 + sy + sz] + R[q + 1 - sy + sz] + R[q - 1 - sy + sz] +
              R[q + 1 + sy - sz] + R[q - 1 + sy - sz] + R[q + 1 - sy - sz] + R[q - 1 - sy - sz]) *
             (1.f / 64.f);
      }
    }
    const int o = C.g(i, j, k);
    C.r[o] = rv;
    C.e[o] = 0.f;
  });
  __syncthreads();
}

// trilinear prolongation of C into F on F's non-wall nodes 0..n+1
__device__ void b_prolong(const SLev &F, const SLev &C) {
  block_box(0, F.n1 + 2, 0, F.n2 + 2, 0, F.n3 + 2, [&](int i, int j, int k) {
    const int q = F.g(i, j, k);
    if (wall(F.r[q])) return;
    const int ci = (i + 1) >> 1, cj = (j + 1) >> 1, ck = (k + 1) >> 1;
    const int ex = (i & 1) ^ 1, ey = (j & 1) ^ 1, ez = (k & 1) ^ 1;
    const int c0 = C.g(ci, cj, ck);
    float s = 0.f;
#pragma unroll
    for (int dz = 0; dz < 2; ++dz)
#pragma unroll
      for (int dy = 0; dy < 2; ++dy)
#pragma unroll
        for (int dx = 0; dx < 2; ++dx)
          if (dx <= ex && dy <= ey && dz <= ez) s += C.e[c0 + dx + C.N1 * (dy + C.N2 * dz)];
    const int ne = ex + ey + ez;
    F.e[q] += s * (ne == 0 ? 1.f : (ne == 1 ? 0.5f : (ne == 2 ? 0.25f : 0.125f)));
  });
  __syncthreads();
}

// the coarse levels' view in block 0's shared memory
__device__ __forceinline__ SLev smem_level(const XArgs &a, int l, unsigned char *sm) {
  SLev S = a.S[l];
  S.e = reinterpret_cast<float *>(sm + a.so_e[l]);
  S.r = reinterpret_cast<float *>(sm + a.so_r[l]);
  S.rf = reinterpret_cast<float *>(sm + a.so_rf[l]);
  return S;
}

// the coarse part of the V-cycle, block 0 only: r of level ls+1 in from the
// grid (its exchange arrays), e out
__device__ __noinline__ void coarse_cycle(const XArgs &a, unsigned char *sm) {
  const int top = a.ls + 1, ng = a.ng;
  {
    const GLev &G = a.G[top];
    const SLev S = smem_level(a, top, sm);
    block_box(0, S.N1, 0, S.N2, 0, S.n3 + 3, [&](int i, int j, int k) {
      const int q = S.g(i, j, k);
      S.r[q] = G.r[G.g(i, j, k)];
      S.e[q] = 0.f;
    });
  }
  __syncthreads();
  for (int l = top; l < ng; ++l) {
    const SLev F = smem_level(a, l, sm), C = smem_level(a, l + 1, sm);
    b_smooth(F, a.omega, a.nu_pre);
    b_restrict(F, C);
  }
  b_smooth(smem_level(a, ng, sm), a.omega, a.coarse_sweeps);
  for (int l = ng - 1; l >= top; --l) {
    const SLev F = smem_level(a, l, sm), C = smem_level(a, l + 1, sm);
    b_prolong(F, C);
    b_smooth(F, a.omega, a.nu_post);
  }
  {
    const GLev &G = a.G[top];
    const SLev S = smem_level(a, top, sm);
    block_box(0, S.N1, 0, S.N2, 0, S.n3 + 3, [&](int i, int j, int k) { G.e[0][G.g(i, j, k)] = S.e[S.g(i, j, k)]; });
  }
  asm volatile("fence.proxy.async.global;" ::: "memory");
}

// ------------------------------------------------------------ level 1, FP64
// FP64 residual b - A u of the finest level on its interior nodes, written
// as the FP32 right-hand side of the V-cycle (+inf on walls), the correction
// cleared; returns this thread's share of the L1 norm over the plasma nodes
// (bcnd = -1).  (A flat node index per thread, with two integer divisions per
// node, made this phase 7 % of the 128^3 solve slower.)
__device__ __noinline__ double g_residual_f64(const XArgs &a, const GLev &L1, float *e1) {
  // one grid row (j, k) per warp at a time, the lanes along i: coalesced
  // loads, no division per node, the arguments in registers
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int ni = L1.n1 + 1, nj = L1.n2 + 1, nk = L1.n3 + 1;
  const long long sy = L1.n1 + 3, sz = (long long)(L1.n1 + 3) * (L1.n2 + 3);
  const long long ry = L1.n1 + 2, rz = (long long)(L1.n1 + 2) * (L1.n2 + 2);
  const double *__restrict__ u = a.u;
  const double *__restrict__ bb = a.b;
  const int *__restrict__ bcnd = a.bcnd;
  const double aw = a.aw, an = a.an, at = a.at, ac = a.ac;
  float *__restrict__ r1 = L1.r;
  float *__restrict__ e = e1;
  double acc = 0.0;
  for (int row = gw; row < nj * nk; row += nw) {
    const int k = row / nj + 1, j = row - (k - 1) * nj + 1;
    const long long w0 = sy * j + sz * k, r0 = ry * j + rz * k, o0 = L1.g(0, j, k);
#pragma unroll 2
    for (int i = 1 + lane; i <= ni; i += 32) {
      const long long w = w0 + i;
      const int bc = bcnd[w];
      const double bv = bb[r0 + i], c0 = u[w], uw = u[w - 1], un = u[w + sy], us = u[w - sy], ue = u[w + 1],
                   ut = u[w + sz], ub = u[w - sz];
      float rf = INFINITY;
      if (bc <= 0) {
        const double rv = bv - (aw * uw + an * un + an * us + aw * ue + ac * c0 + at * ut + at * ub);
        if (bc == -1) acc += fabs(rv);
        rf = (float)rv;
      }
      r1[o0 + i] = rf;
      e[o0 + i] = 0.f;
    }
  }
  return acc;
}

// r = +inf on the ghost nodes of level 1 (never updated, correction 0):
// one grid row (j, k) per warp, the whole row on the ghost planes j, k = 0,
// n + 2, else its two end nodes
__device__ __noinline__ void g_ghosts(const GLev &L) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5), nw = (int)((gridDim.x * blockDim.x) >> 5);
  const int N1 = L.n1 + 3, N2 = L.n2 + 3, N3 = L.n3 + 3;
  for (int row = gw; row < N2 * N3; row += nw) {
    const int k = row / N2, j = row - k * N2;
    const bool face = j == 0 || k == 0 || j == N2 - 1 || k == N3 - 1;
    for (int t = lane; t < (face ? N1 : 2); t += 32) {
      const int i = face ? t : (t == 0 ? 0 : N1 - 1);
      const long long q = L.g(i, j, k);
      L.r[q] = INFINITY;
      L.e[0][q] = 0.f;
      L.e[1][q] = 0.f;
    }
  }
}

// u += e on the non-wall nodes of level 1 (when no post-sweep of level 1 did it)
__device__ __noinline__ void g_add_u(const XArgs &a, const GLev &L1, const float *e1) {
  const int tid = (int)(blockIdx.x * blockDim.x + threadIdx.x), nth = (int)(gridDim.x * blockDim.x);
  const int ni = L1.n1 + 1, nj = L1.n2 + 1;
  const int total = ni * nj * (L1.n3 + 1);
  for (int t = tid; t < total; t += nth) {
    const int row = t / ni, i = t - row * ni + 1;
    const int k = row / nj + 1, j = row - (k - 1) * nj + 1;
    const long long o = L1.g(i, j, k);
    if (!wall(L1.r[o])) {
      double *uq = a.u + i + (long long)(L1.n1 + 3) * (j + (long long)(L1.n2 + 3) * k);
      *uq = *uq + (double)e1[o];
    }
  }
}

__global__ void __launch_bounds__(XM_BLOCK, 1)
    k_refine_mixed(const XArgs *__restrict__ ap, const __grid_constant__ XMaps maps) {
  cg::grid_group grid = cg::this_grid();
  const XArgs &a = *ap;
  __shared__ double sh[40];
  __shared__ __align__(8) unsigned long long bars[2];
  const int ng = a.ng, ls = a.ls;
  Pipe pp;
  pp.base = (int)((128u - (smem_addr(xm_smem) & 127u)) & 127u);
  pp.bar[0] = smem_addr(&bars[0]);
  pp.bar[1] = smem_addr(&bars[1]);
  pp.uses[0] = pp.uses[1] = 0;
  pp.fail = false;
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pp.bar[0]) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(pp.bar[1]) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  unsigned char *smem = xm_smem + pp.base;
  unsigned cur = 0;   // bit l: the e buffer of level l holding its correction
  const GLev &L1 = a.G[1];
  g_ghosts(L1);
  asm volatile("fence.proxy.async.global;" ::: "memory");
  grid.sync();
  double res = 0.0, res0 = -1.0;
  int it = 0, status = 0;
  for (;;) {
    // FP64 residual, FP32 copy as the V-cycle right-hand side, e = 0
    const double acc = g_residual_f64(a, L1, L1.e[(cur >> 1) & 1]);
    asm volatile("fence.proxy.async.global;" ::: "memory");
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
    // FP32 V-cycle on the correction: grid levels down (sweeps, fused
    // residual + restriction), coarse levels on chip, grid levels up (the
    // first post-sweep prolongs), the last sweep of level 1 adds u += e
    const int ldown = ls < ng ? ls : ng - 1;   // the last level restricted from
    for (int l = 1; l <= ldown; ++l) {
      const int nu = l == 1 ? a.nu_fine_pre : a.nu_pre;
      for (int s = 0; s < nu; ++s) tile_pass(a, maps, l, K_SWEEP, pp, grid, cur);
      tile_pass(a, maps, l, K_RESTRICT, pp, grid, cur);
    }
    bool added = false;
    if (ls < ng) {
      if (blockIdx.x == 0) coarse_cycle(a, smem);
      grid.sync();
    } else {
      // the coarsest level is a grid level: its sweeps (ng = 1: the last one
      // adds u += e)
      for (int s = 0; s < a.coarse_sweeps; ++s) {
        const bool last = ng == 1 && s == a.coarse_sweeps - 1;
        tile_pass(a, maps, ng, K_SWEEP | (last ? K_ADDU : 0), pp, grid, cur);
        added = added || last;
      }
    }
    for (int l = (ls < ng ? ls : ng - 1); l >= 1; --l) {
      const int nu = l == 1 ? a.nu_fine_post : a.nu_post;
      if (nu == 0) {
        tile_pass(a, maps, l, K_PRO, pp, grid, cur);
        continue;
      }
      for (int s = 0; s < nu; ++s) {
        const bool last = l == 1 && s == nu - 1;
        tile_pass(a, maps, l, K_SWEEP | (s == 0 ? K_PRO : 0) | (last ? K_ADDU : 0), pp, grid, cur);
        added = added || last;
      }
    }
    if (!added) {
      g_add_u(a, L1, L1.e[(cur >> 1) & 1]);
      grid.sync();
    }
    ++it;
  }
  if (pp.fail && threadIdx.x == 0) {
    // copies possibly in flight: one more bounded wait on each stage
    mbar_wait(pp.bar[0], pp.uses[0] & 1u);
    mbar_wait(pp.bar[1], pp.uses[1] & 1u);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    a.out_i[0] = it;
    a.out_i[1] = status;
    a.out_d[0] = res;
    a.out_d[1] = res0;
  }
}

size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// tensor map of array `base` of level L with a box of bx x by x bz floats
int box_map(CUtensorMap *m, float *base, const GLev &L, unsigned bx, unsigned by, unsigned bz) {
  EncodeTiledFn fn = encode_tiled();
  if (!fn) {
    fprintf(stderr, "lepic_gpu: cuTensorMapEncodeTiled not available\n");
    return LEPIC_ERR_CUDA;
  }
  const cuuint64_t dims[3] = {(cuuint64_t)L.P1, (cuuint64_t)(L.n2 + 3), (cuuint64_t)(L.n3 + 3)};
  const cuuint64_t strides[2] = {(cuuint64_t)L.P1 * 4, (cuuint64_t)L.P1 * (L.n2 + 3) * 4};
  const cuuint32_t box[3] = {bx, by, bz};
  const cuuint32_t es[3] = {1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, base, dims, strides, box, es,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    fprintf(stderr, "lepic_gpu: cuTensorMapEncodeTiled failed (%d) for a %d x %d x %d level\n", (int)r, L.n1, L.n2,
            L.n3);
    return LEPIC_ERR_CUDA;
  }
  return LEPIC_OK;
}

}  // namespace

// the status of the last solve (not converged, diverged) into the device
// error word, for a caller that does not wait for the solve
__global__ void k_solve_status(const int *out_i, int *err) {
  if (out_i[1] != 0) raise_err(err, out_i[1], out_i[0]);
}

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
  A.bcnd = bcnd;
  A.eps = eps;
  A.err = c.d_err;
  // coefficients per level (Src/mg.h) and the coarse levels that fit in
  // shared memory (level 1 stays on the grid)
  float co[XM_MAX + 1][4];
  for (int l = 1; l <= ng; ++l) {
    double hl[3];
    for (int q = 0; q < 3; ++q) hl[q] = h[q] * (double)(1 << (l - 1));
    const double aw = eps0 / (hl[0] * hl[0]), an = eps0 / (hl[1] * hl[1]), at = eps0 / (hl[2] * hl[2]);
    const double ac = -(an + an + aw + aw + at + at);
    if (l == 1) {
      A.aw = aw;
      A.an = an;
      A.at = at;
      A.ac = ac;
    }
    co[l][0] = (float)aw;
    co[l][1] = (float)an;
    co[l][2] = (float)at;
    co[l][3] = (float)ac;
  }
  size_t csm = 0;
  A.ls = ng;
  for (int l = ng; l >= 2; --l) {
    const size_t nn = (size_t)(n[0] / (1 << (l - 1)) + 3) * (n[1] / (1 << (l - 1)) + 3) * (n[2] / (1 << (l - 1)) + 3);
    const size_t need = align16(4 * nn) * 3;
    if (csm + need > XM_SMEM_COARSE) break;
    A.so_e[l] = (unsigned)csm;
    A.so_r[l] = (unsigned)(csm + align16(4 * nn));
    A.so_rf[l] = (unsigned)(csm + 2 * align16(4 * nn));
    csm += need;
    A.ls = l - 1;
  }
  if (A.ls == ng) csm = 0;
  const int ngl = A.ls < ng ? A.ls + 1 : ng;   // levels with global arrays
  if (A.ls > GMAX) {
    fprintf(stderr, "lepic_gpu: mixed solve: %d grid levels (at most %d)\n", A.ls, GMAX);
    return LEPIC_ERR_UNSUPPORTED;
  }
  char nm[32];
  for (int l = 1; l <= ng; ++l) {
    const int m1 = n[0] >> (l - 1), m2 = n[1] >> (l - 1), m3 = n[2] >> (l - 1);
    if (l <= ngl) {
      GLev &L = A.G[l];
      L.n1 = m1;
      L.n2 = m2;
      L.n3 = m3;
      L.P1 = (m1 + 4 + 3) & ~3;
      L.ntx = (m1 + TX - 1) / TX;
      L.nty = (m2 + TY - 1) / TY;
      L.ntz = (m3 + TZ - 1) / TZ;
      L.aw = co[l][0];
      L.an = co[l][1];
      L.at = co[l][2];
      L.ac = co[l][3];
      for (int q = 0; q < 2; ++q) {
        snprintf(nm, sizeof nm, "xm_e%d_%d", l, q);
        L.e[q] = (float *)scratch(nm, sizeof(float) * (size_t)L.nn());
        if (!L.e[q]) return LEPIC_ERR_CUDA;
        // the nodes a sweep never writes (ghosts; walls stay at the 0 the
        // residual or the restriction gave them) hold 0 in both buffers
        LEPIC_CUDA(cudaMemsetAsync(L.e[q], 0, sizeof(float) * (size_t)L.nn(), s));
      }
      snprintf(nm, sizeof nm, "xm_r%d", l);
      L.r = (float *)scratch(nm, sizeof(float) * (size_t)L.nn());
      if (!L.r) return LEPIC_ERR_CUDA;
    }
    if (l > A.ls) {
      SLev &S = A.S[l];
      S.n1 = m1;
      S.n2 = m2;
      S.n3 = m3;
      S.N1 = m1 + 3;
      S.N2 = m2 + 3;
      S.aw = co[l][0];
      S.an = co[l][1];
      S.at = co[l][2];
      S.ac = co[l][3];
    }
  }
  XMaps M;
  memset(&M, 0, sizeof(M));
  for (int l = 1; l <= ngl; ++l) {
    const GLev &L = A.G[l];
    if (l <= A.ls) {
      int rc = box_map(&M.fe[l][0], L.e[0], L, BX, BY, BZ);
      if (!rc) rc = box_map(&M.fe[l][1], L.e[1], L, BX, BY, BZ);
      if (!rc) rc = box_map(&M.fr[l], L.r, L, BX, BY, BZ);
      if (rc) return rc;
    }
    if (l >= 2) {
      int rc = box_map(&M.ce[l][0], L.e[0], L, CBX, CBY, CBZ);
      if (!rc) rc = box_map(&M.ce[l][1], L.e[1], L, CBX, CBY, CBZ);
      if (rc) return rc;
    }
  }
  A.alpha = fabs((double)((n[0] + 1) * (n[1] + 1) * (n[2] + 1)) * A.ac) * 1.0;
  const size_t smem = (csm > TILE_SMEM ? csm : TILE_SMEM) + 128;
  LEPIC_CUDA(cudaFuncSetAttribute(k_refine_mixed, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int occ = 0;
  LEPIC_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_refine_mixed, XM_BLOCK, smem));
  if (occ < 1) return LEPIC_ERR_CUDA;
  const int blocks = c.sms;
  A.partial = (double *)scratch("xm_partial", sizeof(double) * 2 * blocks);
  A.out_i = (int *)scratch("xm_out_i", sizeof(int) * 4);
  A.out_d = (double *)scratch("xm_out_d", sizeof(double) * 2);
  XArgs *dA = (XArgs *)scratch("xm_args", sizeof(XArgs));
  if (!A.partial || !A.out_i || !A.out_d || !dA) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemcpyAsync(dA, &A, sizeof(XArgs), cudaMemcpyHostToDevice, s));
  void *args[] = {&dA, &M};
  int tm = timer_start("pdesolver_mixed", s);
  LEPIC_CUDA(cudaLaunchCooperativeKernel((void *)k_refine_mixed, dim3(blocks), dim3(XM_BLOCK), args, smem, s));
  timer_stop(tm, s);
  if (!iters && !res_out) {
    // no wait: the solve's status goes to the device error word
    k_solve_status<<<1, 1, 0, s>>>(A.out_i, ctx().d_err);
    LEPIC_CUDA(cudaGetLastError());
    return LEPIC_OK;
  }
  int hi[4];
  double hd[2];
  LEPIC_CUDA(cudaMemcpyAsync(hi, A.out_i, sizeof(hi), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(hd, A.out_d, sizeof(hd), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (iters) *iters = hi[0];
  if (res_out) *res_out = hd[0];
  // a copy that timed out stays in the device error word (lepic_dev_check)
  return hi[1];
}

int pdesolver_mixed_stats(int *iters, double *res, cudaStream_t s) {
  if (!iters || !res) return LEPIC_ERR_ARG;
  const int *oi = (const int *)scratch("xm_out_i", sizeof(int) * 4);
  const double *od = (const double *)scratch("xm_out_d", sizeof(double) * 2);
  if (!oi || !od) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemcpyAsync(iters, oi, sizeof(int), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(res, od, sizeof(double), cudaMemcpyDeviceToHost, s));
  return LEPIC_OK;
}

}  // namespace lepic

extern "C" int lepic_dev_pdesolver_mixed_stats(int *iters, double *res, void *stream) {
  return lepic::pdesolver_mixed_stats(iters, res, (cudaStream_t)stream);
}

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
