// Mixed-precision particle kernels of the device-resident step loop.
//
// Particle state per species (28 B per particle instead of 48):
//   cell  int32   c = (ix-1) | (iy-1) << 10 | (iz-1) << 20, ix = INT(x/h)+1
//                 of the reference (Src/part_expmover.f90:89-91)
//   p32   float   6 planes: fx, fy, fz in [0,1) (x = (ix-1+fx) h) and
//                 vx, vy, vz in m/s
// The push is the reference's gather + Boris + leapfrog
// (Src/part_expmover.f90:89-246) in FP32 on an FP32 copy of E packed as one
// float4 per node; the position update is done on the in-cell offset
// (f += v dt/h, cell += floor(f)), which keeps ~7 significant digits of the
// position inside its cell.
//
// Deposition (Src/part_expmover.f90:591-656) of the new position: seven of
// the eight CIC weights are rounded to integers in units of 2^-20 and the
// eighth is the remainder, so every particle deposits exactly 2^20 units and
// integer sums are exact and independent of the summation order.  The sort orders particles by 8x8x8-cell tiles; one
// block pushes the particles of one tile and sums their weights with 32-bit
// shared-memory adds into a node tile covering the tile's cells plus one halo
// cell on each side.  The node tile is added to the FP64 grid (one atomic per
// non-zero node) and cleared after every FLUSH_PARTICLES particles, so a
// node's sum stays within [-5, 2^20] x FLUSH_PARTICLES however the particles
// are placed and is read back unambiguously modulo 2^32.  Particles outside the box (drifted since the sort, moved by
// hole filling, appended by collisions) add their integer weights to the grid
// directly.  kdep and kq are applied in FP64 to the integer sums.
//
// A thread moves four consecutive particles with 16-byte loads and stores
// and merges the weights of those that end in the same cell before touching
// shared memory.
#include <type_traits>
#include <cstring>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int MBK = 256;
constexpr int TC = LEPIC_TILE_CELLS;       // tile edge in cells
constexpr int TN = TC + 3;                 // node tile edge (halo cell each side)
constexpr int TT = TN * TN * TN;
constexpr int CHUNK = 4 * MBK;             // particles per block iteration
constexpr int FLUSH_PARTICLES = 3072;      // node sums <= 3072 * 2^20 = 0xC0000000
static_assert(FLUSH_PARTICLES % CHUNK == 0, "flush windows are whole chunks");
static_assert(qsum_window_ok(FLUSH_PARTICLES), "window sums are read back modulo 2^32");
constexpr int CB = LEPIC_CELL_BITS, CM = LEPIC_CELL_MAX - 1;

__device__ __forceinline__ unsigned lmask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

struct MixedConst {
  float dth0, dth1, dth2;     // dt / h per direction
  float k1;                   // dt q / (2 m)
  float kk;                   // Boris rotation factor 2 k1 / (1 + (k1 |B|)^2)
  float Bx, By, Bz;
  int boris, flag_pbc, flag_nmn, ngrid;
  double Nm, mass, kdep;      // kdep = Nm / (h1 h2 h3)
  int ntx, nty, ntiles;       // tile grid
  Dielectric die;             // dielectric walls (die.dtype nullptr: none)
};

// The charge of a particle lost on a dielectric wall (Src/part_expmover.f90:
// 302-348) from its cell coordinates: new cell (ax, ay, az) (z already
// wrapped with periodic planes) with offsets (fx, fy, fz) in [0, 1), clamped
// to (cx, cy, cz).  The reference's weight (ix h - x) / h is
// cx - (ax - 1 + fx) here, evaluated in FP64.
// Out of line and with its arguments by value: the branch is rare, and the
// kernel parameters' addresses are never taken (which would copy them to
// local memory).
__device__ __noinline__ void dielectric_charge_cells(Dielectric die, long long N1, long long N2, int igrid,
                                                     int ax, int ay, int az, float fx, float fy, float fz,
                                                     int cx, int cy, int cz) {
  const int dt = die.dtype[igrid];
  if (dt <= 1) return;
  const double pz = (double)cz - ((double)(az - 1) + (double)fz);
  if (dt == 2) {
    const double px = (double)cx - ((double)(ax - 1) + (double)fx);
    double *q = die.qxz;
    const long long NX = N1;
    atomicAdd(&q[cx + NX * cz], die.k3 * px * pz);
    atomicAdd(&q[cx + 1 + NX * cz], die.k3 * (1.0 - px) * pz);
    atomicAdd(&q[cx + 1 + NX * (cz + 1)], die.k3 * (1.0 - px) * (1.0 - pz));
    atomicAdd(&q[cx + NX * (cz + 1)], die.k3 * px * (1.0 - pz));
  } else if (dt == 3 || dt == 4) {
    const double py = (double)cy - ((double)(ay - 1) + (double)fy);
    double *q = die.qyz + (dt - 3);
    const long long NY = N2;
    atomicAdd(&q[2 * (cy + NY * cz)], die.k3 * py * pz);
    atomicAdd(&q[2 * (cy + 1 + NY * cz)], die.k3 * (1.0 - py) * pz);
    atomicAdd(&q[2 * (cy + 1 + NY * (cz + 1))], die.k3 * (1.0 - py) * (1.0 - pz));
    atomicAdd(&q[2 * (cy + NY * (cz + 1))], die.k3 * py * (1.0 - pz));
  }
}

// FP32 copy of the B-field map (Src/part_expmover.f90:148-203): one float4
// (Bx, By, Bz, |B|) per map node, map nodes indexed like Bi(4, 0:nB1+2, ...).
struct MixedBMap {
  const float4 *B;
  int own;                    // 1: own grid of spacing h_B; 0: the node grid
  int nb1, nb2, nb3;
  long long N1, N2;           // nB1 + 3, nB2 + 3
  float r0, r1, r2;           // h / h_B per direction
};

// The block's box in shared memory: the nodes bx..bx+TN-1 (and likewise in
// y, z) of the tile's cells plus one halo cell on each side.
struct Tile {
  unsigned *acc;              // node weight sums (nullptr: no box, global only)
  const float4 *E;            // E at the box nodes
  const unsigned char *cw;    // all-wall flags of the box cells
  int bx, by, bz;             // grid coordinates of box node (0,0,0)
  const float4 *B;            // B map at the box nodes (map on the node grid)
};

// sum of k_i e_i, i = 0..7, rounded as a chain of multiply-adds in order
__device__ __forceinline__ float gather8(float k0, float k1, float k2, float k3, float k4, float k5, float k6,
                                         float k7, float e0, float e1, float e2, float e3, float e4, float e5,
                                         float e6, float e7) {
  float s = __fmul_rn(k0, e0);
  s = __fmaf_rn(k1, e1, s);
  s = __fmaf_rn(k2, e2, s);
  s = __fmaf_rn(k3, e3, s);
  s = __fmaf_rn(k4, e4, s);
  s = __fmaf_rn(k5, e5, s);
  s = __fmaf_rn(k6, e6, s);
  return __fmaf_rn(k7, e7, s);
}

// box-local coordinates of cell (ix,iy,iz) when the cell's 8 nodes are in the
// box (a block with no box, the untiled tail, has neither acc nor E)
__device__ __forceinline__ bool in_box(const Tile &T, int ix, int iy, int iz, int &lx, int &ly, int &lz) {
  lx = ix - T.bx;
  ly = iy - T.by;
  lz = iz - T.bz;
  return (T.acc || T.E) && (unsigned)lx < (unsigned)(TN - 1) && (unsigned)ly < (unsigned)(TN - 1) &&
         (unsigned)lz < (unsigned)(TN - 1);
}

// 8 weights of the cell with base node (jx,jy,jz) into the tile when the
// cell lies in the box, else into the FP64 grid
__device__ __forceinline__ void deposit8(const Dims &d, const Tile &T, int jx, int jy, int jz, const int w[8],
                                         double kdep, const double *__restrict__ kq, double *__restrict__ np) {
  int lx, ly, lz;
  if (in_box(T, jx, jy, jz, lx, ly, lz)) {
    // shared-memory reductions on 32-bit addresses
    const uint32_t a0 = smem_addr(T.acc) + 4u * (uint32_t)(lx + TN * (ly + TN * lz));
    const uint32_t to[8] = {0, 1, 1 + TN, TN, TN * TN, 1 + TN * TN, 1 + TN + TN * TN, TN + TN * TN};
#pragma unroll
    for (int c = 0; c < 8; ++c)
      asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a0 + 4u * to[c]), "r"((unsigned)w[c]) : "memory");
  } else {
    const long long q = d.g(jx, jy, jz), sy = d.N1, sz = d.N1 * d.N2;
    const long long o[8] = {0, 1, 1 + sy, sy, sz, 1 + sz, 1 + sy + sz, sy + sz};
#pragma unroll
    for (int c = 0; c < 8; ++c) atomicAdd(&np[q + o[c]], __ldg(&kq[q + o[c]]) * (kdep * ((double)w[c] * QI)));
  }
}

// the node tile into the FP64 grid (non-zero nodes), then cleared
__device__ void flush_tile(const Dims &d, const Tile &T, double kdep, const double *__restrict__ kq,
                           double *__restrict__ np) {
  for (int e = threadIdx.x; e < TT; e += blockDim.x) {
    const unsigned v = T.acc[e];
    if (v) {
      const int lx = e % TN, ly = (e / TN) % TN, lz = e / (TN * TN);
      const int gx = T.bx + lx, gy = T.by + ly, gz = T.bz + lz;
      if (gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2) {
        const long long node = d.g(gx, gy, gz);
        const double val = qsum_value(v, FLUSH_PARTICLES);
        atomicAdd(&np[node], __ldg(&kq[node]) * (kdep * (val * QI)));
      }
      T.acc[e] = 0u;
    }
  }
}

// Four consecutive particles i0..i0+3 (i0 a multiple of 4) and which of
// them lie in the range being pushed.
struct Quad {
  int4 c4;
  char4 f4;
  float4 P[6];
  bool in[4];
};

__device__ __forceinline__ void quad_range(Quad &Q, long long i0, long long lo, long long hi) {
#pragma unroll
  for (int k = 0; k < 4; ++k) Q.in[k] = (i0 + k >= lo) && (i0 + k < hi);
}

// from HBM (i0 + 3 < cap: cap is a multiple of 4)
__device__ __forceinline__ void load_quad(Quad &Q, long long i0, long long lo, long long hi,
                                          const int *__restrict__ cell, const float *__restrict__ p,
                                          long long cap, const signed char *__restrict__ flag) {
  quad_range(Q, i0, lo, hi);
  if (i0 < hi) {
    Q.c4 = *reinterpret_cast<const int4 *>(cell + i0);
    Q.f4 = *reinterpret_cast<const char4 *>(flag + i0);
#pragma unroll
    for (int a = 0; a < 6; ++a) Q.P[a] = *reinterpret_cast<const float4 *>(p + a * cap + i0);
  } else {
    Q.c4 = make_int4(-1, -1, -1, -1);
    Q.f4 = make_char4(0, 0, 0, 0);
#pragma unroll
    for (int a = 0; a < 6; ++a) Q.P[a] = make_float4(0.f, 0.f, 0.f, 0.f);
  }
}

// B of the map at a particle in cell (ix, iy, iz) at offsets (fx, fy, fz):
// on the node grid from the E gather's node g0 and weights k[0..7] (in the
// box Eb = T.E or in HBM); on its own grid at map index INT(x/h_B)+1 with its
// own weights.  False when |B| at the left map node is not above 1e-5 T.
__device__ __forceinline__ bool bmap_gather_mixed(const MixedBMap &m, const Tile &T, bool boxed, long long g0,
                                                  long long sy, long long sz, int ix, int iy, int iz, float fx,
                                                  float fy, float fz, const float (&kE)[8], float &Bx, float &By,
                                                  float &Bz) {
  const float4 *Bb;
  float k[8];
#pragma unroll
  for (int a = 0; a < 8; ++a) k[a] = kE[a];
  if (m.own) {
    const float xb = ((float)(ix - 1) + fx) * m.r0, yb = ((float)(iy - 1) + fy) * m.r1,
                zb = ((float)(iz - 1) + fz) * m.r2;
    int bx = (int)xb, by = (int)yb, bz = (int)zb;
    bx = bx < 0 ? 0 : (bx > m.nb1 ? m.nb1 : bx);
    by = by < 0 ? 0 : (by > m.nb2 ? m.nb2 : by);
    bz = bz < 0 ? 0 : (bz > m.nb3 ? m.nb3 : bz);
    const float gx = xb - (float)bx, gy = yb - (float)by, gz = zb - (float)bz;
    const float px = 1.f - gx, py = 1.f - gy, pz = 1.f - gz;
    k[0] = px * py * pz;
    k[1] = (1.f - px) * py * pz;
    k[2] = (1.f - px) * (1.f - py) * pz;
    k[3] = px * (1.f - py) * pz;
    k[4] = px * py * (1.f - pz);
    k[5] = (1.f - px) * py * (1.f - pz);
    k[6] = (1.f - px) * (1.f - py) * (1.f - pz);
    k[7] = px * (1.f - py) * (1.f - pz);
    Bb = m.B;
    g0 = (bx + 1) + m.N1 * ((by + 1) + m.N2 * (long long)(bz + 1));
    sy = m.N1;
    sz = m.N1 * m.N2;
  } else {
    Bb = boxed ? T.B : m.B;
  }
  const float4 b0 = Bb[g0];
  if (!(b0.w > 1.e-5f)) return false;
  const float4 b1 = Bb[g0 + 1], b2 = Bb[g0 + 1 + sy], b3 = Bb[g0 + sy], b4 = Bb[g0 + sz], b5 = Bb[g0 + 1 + sz],
               b6 = Bb[g0 + 1 + sy + sz], b7 = Bb[g0 + sy + sz];
  Bx = k[0] * b0.x + k[1] * b1.x + k[2] * b2.x + k[3] * b3.x + k[4] * b4.x + k[5] * b5.x + k[6] * b6.x + k[7] * b7.x;
  By = k[0] * b0.y + k[1] * b1.y + k[2] * b2.y + k[3] * b3.y + k[4] * b4.y + k[5] * b5.y + k[6] * b6.y + k[7] * b7.y;
  Bz = k[0] * b0.z + k[1] * b1.z + k[2] * b2.z + k[3] * b3.z + k[4] * b4.z + k[5] * b5.z + k[6] * b6.z + k[7] * b7.z;
  return true;
}

// Deposit of a lane's up to four particles (jx < 0: none) at cells (jx, jy,
// jz) and offsets (gx, gy, gz): the particles that end in the lane's first
// particle's cell are merged before touching shared memory
__device__ __forceinline__ void deposit_quad(const Dims &d, const Tile &T, const int (&jx)[4], const int (&jy)[4],
                                             const int (&jz)[4], const float (&gx)[4], const float (&gy)[4],
                                             const float (&gz)[4], double kdep, const double *__restrict__ kq,
                                             double *__restrict__ np) {
  // the first particle's cell by selects (an index into jx would put the
  // arrays in local memory)
  int ax = -1, ay = 0, az = 0;
#pragma unroll
  for (int k = 0; k < 4; ++k)
    if (ax < 0 && jx[k] >= 0) {
      ax = jx[k];
      ay = jy[k];
      az = jz[k];
    }
  if (ax < 0) return;
  int wa[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (jx[k] < 0) continue;
    int w[8];
    qweights(gx[k], gy[k], gz[k], w);
    if (jx[k] == ax && jy[k] == ay && jz[k] == az) {
#pragma unroll
      for (int cc = 0; cc < 8; ++cc) wa[cc] += w[cc];
    } else {
      deposit8(d, T, jx[k], jy[k], jz[k], w, kdep, kq, np);
    }
  }
  deposit8(d, T, ax, ay, az, wa, kdep, kq, np);
}

// The deposit of a lane's up to four particles given by their packed cells
// (cc < 0: none) and offsets: those in the first particle's cell are summed,
// then the first-cell sums of the warp's lanes are merged per run of lanes
// starting in one cell (sorted particles: one to three runs per warp), so
// that a cell's 8 shared words take one add per run instead of one per lane;
// the others are added one by one.  All 32 lanes must call this.
__device__ __forceinline__ void deposit_quad_warp(const Dims &d, const Tile &T, const int (&cc)[4],
                                                  const float (&gx)[4], const float (&gy)[4], const float (&gz)[4],
                                                  double kdep, const double *__restrict__ kq,
                                                  double *__restrict__ np) {
  int a = -1;
#pragma unroll
  for (int k = 0; k < 4; ++k) a = (a < 0) ? cc[k] : a;
  int wa[8] = {0, 0, 0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if (cc[k] < 0) continue;
    int w[8];
    qweights(gx[k], gy[k], gz[k], w);
    if (cc[k] == a) {
#pragma unroll
      for (int c = 0; c < 8; ++c) wa[c] += w[c];
    } else {
      deposit8(d, T, (cc[k] & CM) + 1, ((cc[k] >> CB) & CM) + 1, (cc[k] >> (2 * CB)) + 1, w, kdep, kq, np);
    }
  }
  // the packed cell is the run key (one value per cell, -1: none)
  if (warp_run_sum<8, int>((long long)a, wa))
    deposit8(d, T, (a & CM) + 1, ((a >> CB) & CM) + 1, (a >> (2 * CB)) + 1, wa, kdep, kq, np);
}

// Push + loss test + deposit of the particle quad Q starting at i0;
// particles outside the range are not touched.  Every lane of the warp must
// call this (warp-wide hole appends).  BMAP: B from the map m.
template <bool BMAP, bool DIE, bool DEP = true>
__device__ __forceinline__ void push_quad(const Dims &d, const MixedConst &c, const MixedBMap &m, const Tile &T,
                                          long long i0, Quad &Q, const float4 *__restrict__ E4,
                                          const int *__restrict__ bcnd, const unsigned char *__restrict__ cw,
                                          int *__restrict__ cell, float *__restrict__ p, long long cap,
                                          signed char *__restrict__ flag, const double *__restrict__ kq,
                                          double *__restrict__ np, int *__restrict__ holes,
                                          int *__restrict__ nholes, double *__restrict__ acc,
                                          int *__restrict__ err) {
  const unsigned full = 0xffffffffu;
  const int n1 = d.n1, n2 = d.n2, n3 = d.n3;
  int4 &c4 = Q.c4;
  const char4 f4 = Q.f4;
  float4 *P = Q.P;
  const bool *in = Q.in;
  const bool full4 = in[0] && in[1] && in[2] && in[3];
  bool hole[4] = {false, false, false, false};
  int jx[4], jy[4], jz[4];
  float gxs[4], gys[4], gzs[4];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    jx[k] = -1;
    jy[k] = jz[k] = 0;
    gxs[k] = gys[k] = gzs[k] = 0.f;
    if (!in[k]) continue;
    const int cc = (&c4.x)[k];
    float vx = (&P[3].x)[k], vy = (&P[4].x)[k], vz = (&P[5].x)[k];
    if ((&f4.x)[k] == 1) {
      // killed in a collision: removed here (Src/part_expmover.f90:70-84)
      atomicAdd(&acc[1], -(0.5 * c.Nm * c.mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz)));
      hole[k] = true;
      continue;
    }
    const int ix = (cc & CM) + 1, iy = ((cc >> CB) & CM) + 1, iz = (cc >> (2 * CB)) + 1;
    if (cc < 0 || ix > n1 || iy > n2 || iz > n3) {
      raise_err(err, LEPIC_ERR_CELL, (int)(i0 + k));
      hole[k] = true;
      continue;
    }
    float fx = (&P[0].x)[k], fy = (&P[1].x)[k], fz = (&P[2].x)[k];
    // gather: left-node weights 1 - f (Src/part_expmover.f90:89-108)
    const float px = 1.f - fx, py = 1.f - fy, pz = 1.f - fz;
    const float k0 = px * py * pz, ka = (1.f - px) * py * pz, kb = (1.f - px) * (1.f - py) * pz,
                kc = px * (1.f - py) * pz, kd = px * py * (1.f - pz), ke = (1.f - px) * py * (1.f - pz),
                kf = (1.f - px) * (1.f - py) * (1.f - pz), kg = px * (1.f - py) * (1.f - pz);
    // from the box in shared memory when the cell is in it (shared-memory
    // loads on 32-bit addresses), else from HBM
    long long g0, sy, sz;
    float4 e0, e1, e2, e3, e4, e5, e6, e7;
    int lx, ly, lz;
    const bool boxed = in_box(T, ix, iy, iz, lx, ly, lz);
    if (boxed) {
      g0 = lx + TN * (ly + TN * lz);
      sy = TN;
      sz = TN * TN;
      const uint32_t a0 = smem_addr(T.E) + 16u * (uint32_t)g0;
      e0 = lds4(a0);
      e1 = lds4(a0 + 16u);
      e2 = lds4(a0 + 16u * (1 + TN));
      e3 = lds4(a0 + 16u * TN);
      e4 = lds4(a0 + 16u * TN * TN);
      e5 = lds4(a0 + 16u * (1 + TN * TN));
      e6 = lds4(a0 + 16u * (1 + TN + TN * TN));
      e7 = lds4(a0 + 16u * (TN + TN * TN));
    } else {
      g0 = d.g(ix, iy, iz);
      sy = d.N1;
      sz = d.N1 * d.N2;
      const float4 *q = E4 + g0;
      e0 = __ldg(q);
      e1 = __ldg(q + 1);
      e2 = __ldg(q + 1 + sy);
      e3 = __ldg(q + sy);
      e4 = __ldg(q + sz);
      e5 = __ldg(q + 1 + sz);
      e6 = __ldg(q + 1 + sy + sz);
      e7 = __ldg(q + sy + sz);
    }
    // the weighted sums as explicit multiply-adds in node order: the same
    // rounding whichever path loaded the nodes and whichever kernel pushes
    const float Ex = gather8(k0, ka, kb, kc, kd, ke, kf, kg, e0.x, e1.x, e2.x, e3.x, e4.x, e5.x, e6.x, e7.x);
    const float Ey = gather8(k0, ka, kb, kc, kd, ke, kf, kg, e0.y, e1.y, e2.y, e3.y, e4.y, e5.y, e6.y, e7.y);
    const float Ez = gather8(k0, ka, kb, kc, kd, ke, kf, kg, e0.z, e1.z, e2.z, e3.z, e4.z, e5.z, e6.z, e7.z);
    const float k1 = c.k1;
    float Bx = c.Bx, By = c.By, Bz = c.Bz, kk = c.kk;
    bool boris = c.boris;
    if (BMAP && boris) {
      const float kE[8] = {k0, ka, kb, kc, kd, ke, kf, kg};
      boris = bmap_gather_mixed(m, T, boxed, g0, sy, sz, ix, iy, iz, fx, fy, fz, kE, Bx, By, Bz);
      const float B_tot = sqrtf(Bx * Bx + By * By + Bz * Bz);
      kk = k1 * (2.f / (1.f + (k1 * B_tot) * (k1 * B_tot)));
    }
    if (boris) {
      // Src/part_expmover.f90:128-160
      const float v1x = vx + k1 * Ex, v1y = vy + k1 * Ey, v1z = vz + k1 * Ez;
      const float v3x = v1x + k1 * (v1y * Bz - v1z * By);
      const float v3y = v1y + k1 * (v1z * Bx - v1x * Bz);
      const float v3z = v1z + k1 * (v1x * By - v1y * Bx);
      vx = v1x + kk * (v3y * Bz - v3z * By) + k1 * Ex;
      vy = v1y + kk * (v3z * Bx - v3x * Bz) + k1 * Ey;
      vz = v1z + kk * (v3x * By - v3y * Bx) + k1 * Ez;
    } else {
      vx = vx + 2.f * k1 * Ex;
      vy = vy + 2.f * k1 * Ey;
      vz = vz + 2.f * k1 * Ez;
    }
    // position on the in-cell offset; the cell moves by floor(f)
    fx = fx + vx * c.dth0;
    fy = fy + vy * c.dth1;
    fz = fz + vz * c.dth2;
    int sx = 0, syi = 0, szi = 0;
    if (!(fx >= 0.f && fx < 1.f)) {
      sx = __float2int_rd(fx);
      fx -= (float)sx;
      if (fx >= 1.f) { fx = 0.f; sx += 1; }
    }
    if (!(fy >= 0.f && fy < 1.f)) {
      syi = __float2int_rd(fy);
      fy -= (float)syi;
      if (fy >= 1.f) { fy = 0.f; syi += 1; }
    }
    if (!(fz >= 0.f && fz < 1.f)) {
      szi = __float2int_rd(fz);
      fz -= (float)szi;
      if (fz >= 1.f) { fz = 0.f; szi += 1; }
    }
    int ax = ix + sx, ay = iy + syi, az = iz + szi;
    int cx = ax, cy = ay, cz = az;
    bool lost = false;
    if (sx | syi | szi) {
      // a new cell: the loss test on the clamped cell before any periodic
      // wrap, as Src/part_expmover.f90:250-275 (the cell a particle stays in
      // passed the test when the particle entered it), then the wrap of the
      // particles that stay (:460-465)
      cx = ax < 0 ? 0 : (ax > n1 + 1 ? n1 + 1 : ax);
      cy = ay < 0 ? 0 : (ay > n2 + 1 ? n2 + 1 : ay);
      cz = az < 0 ? 0 : (az > n3 + 1 ? n3 + 1 : az);
      int lx, ly, lz;
      const bool wall = in_box(T, cx, cy, cz, lx, ly, lz) ? T.cw[lx + (TN - 1) * (ly + (TN - 1) * lz)] != 0
                                                          : cw[d.c(cx, cy, cz)] != 0;
      if (c.flag_nmn == 1 && ax < 1 && !wall) {
        // specular reflection at the Neumann plane x = 0 (Src/part_expmover.f90:
        // 437-446): x = (ax - 1 + fx) h < 0 becomes -x, vx changes sign
        const float g = 1.f - fx;
        ax = 1 - ax;
        if (g >= 1.f) {
          fx = 0.f;
          ax += 1;
        } else {
          fx = g;
        }
        vx = -vx;
      }
      lost = wall || ax < 1 || ax > n1;
      if (c.flag_pbc == 1) {
        if (!lost) {
          if (ay > n2) ay -= n2;
          if (ay < 1) ay += n2;
          if (az > n3) az -= n3;
          if (az < 1) az += n3;
        }
      } else {
        lost = lost || ay < 1 || ay > n2 || az < 1 || az > n3;
      }
    }
    if (lost) {
      // lost at a wall (Src/part_expmover.f90:275-433): every cell outside
      // 1..n has only wall nodes in a closed box; a cell inside 1..n is lost
      // when all of its 8 nodes are walls
      const double Eki = 0.5 * c.Nm * c.mass * ((double)vx * vx + (double)vy * vy + (double)vz * vz);
      const int igrid = bcnd[d.g(cx, cy, cz)];
      atomicAdd(&acc[0], Eki);
      if (igrid >= 0 && igrid <= c.ngrid) {
        atomicAdd(&acc[2 + 2 * igrid], 1.0);
        atomicAdd(&acc[3 + 2 * igrid], Eki);
        if (DIE) {
          // periodic planes: z wraps for the wall charge, y does not
          // (Src/part_expmover.f90:306-316)
          int aw = az, cw_z = cz;
          if (c.flag_pbc == 1 && (az > n3 || az < 1)) {
            aw = az > n3 ? az - n3 : az + n3;
            cw_z = aw < 0 ? 0 : (aw > n3 + 1 ? n3 + 1 : aw);
          }
          const Dielectric die = {c.die.dtype, c.die.qxz, c.die.qyz, c.die.k3};
          dielectric_charge_cells(die, d.N1, d.N2, igrid, ax, ay, aw, fx, fy, fz, cx, cy, cw_z);
        }
      }
      hole[k] = true;
    } else {
      (&c4.x)[k] = (ax - 1) | (ay - 1) << CB | (az - 1) << (2 * CB);
      jx[k] = ax;
      jy[k] = ay;
      jz[k] = az;
      gxs[k] = fx;
      gys[k] = fy;
      gzs[k] = fz;
    }
    (&P[0].x)[k] = fx;
    (&P[1].x)[k] = fy;
    (&P[2].x)[k] = fz;
    (&P[3].x)[k] = vx;
    (&P[4].x)[k] = vy;
    (&P[5].x)[k] = vz;
  }
  // write back (a hole's slot is dead: what is written there is never read)
  if (full4) {
    *reinterpret_cast<int4 *>(cell + i0) = c4;
#pragma unroll
    for (int a = 0; a < 6; ++a) *reinterpret_cast<float4 *>(p + a * cap + i0) = P[a];
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (in[k]) {
        cell[i0 + k] = (&c4.x)[k];
#pragma unroll
        for (int a = 0; a < 6; ++a) p[a * cap + i0 + k] = (&P[a].x)[k];
      }
  }
  // holes: flag 2 and a warp-aggregated append to the hole list
  const int lane = threadIdx.x & 31;
  if (__any_sync(full, hole[0] | hole[1] | hole[2] | hole[3])) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      if (hole[k]) flag[i0 + k] = 2;
      const unsigned hm = __ballot_sync(full, hole[k]);
      if (hm) {
        const int leader = __ffs(hm) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(nholes, __popc(hm));
        base = __shfl_sync(full, base, leader);
        if (hole[k]) holes[base + __popc(hm & lmask_lt())] = (int)(i0 + k);
      }
    }
  }
  if (DEP) deposit_quad(d, T, jx, jy, jz, gxs, gys, gzs, c.kdep, kq, np);
}

// A thread's next quad (cell, six FP32 planes, flags) copied into shared
// memory by cp.async while it pushes the current one: plane a of thread j at
// s_stage[a][j] (16 bytes per thread and plane, conflict-free), the flags
// after the seven planes.  Each thread reads back only what it copied, so no
// barrier orders the copies.
constexpr int STAGE_BYTES = MBK * (7 * 16 + 4);
extern __shared__ __align__(16) unsigned char mx_stage[];

// PARTS blocks per tile, each taking a part of the tile's particles: more
// blocks than the resident slots by that factor, so the SMs idle less while
// a launch's last blocks finish (the push: 0.8 % faster with two parts; the
// deposit, whose parts each flush their node tile, keeps one).  Block b: tile
// b / PARTS, its range [tile_off[t], min(tile_off[t+1], N)) cut at multiples
// of 4 (no quad is shared by two blocks).
constexpr int PUSH_PARTS = 2;
template <int PARTS>
__device__ __forceinline__ void part_range(const int *__restrict__ tile_off, long long N, int b, int &t,
                                           long long &lo, long long &hi) {
  t = b / PARTS;
  const int part = b - t * PARTS;
  const long long a = tile_off[t];
  long long e = tile_off[t + 1];
  if (e > N) e = N;
  const long long n = e > a ? e - a : 0;
  auto cut = [&](int k) {
    if (k == 0) return a;
    if (k == PARTS) return e > a ? e : a;
    long long c = (a + n * k / PARTS + 3) & ~3LL;
    return c < a ? a : (c > e ? (e > a ? e : a) : c);
  };
  lo = cut(part);
  hi = cut(part + 1);
}

// one block per tile: the particles [tile_off[t], tile_off[t+1]) of the last
// sort, clipped to the current count; E and the wall flags of the tile's box
// are read into shared memory once, and each thread's next quad is in flight
// (cp.async) while it pushes the current one, so the particle loads do not
// stall the warps.  The push only: k_deposit_tiles deposits the pushed
// particles of the tile afterwards (one kernel doing both was 6 % slower: its
// shared-memory adds and flush barriers sat between the push's memory
// accesses)
template <bool BMAP, bool DIE>
__global__ void __launch_bounds__(MBK, 3) k_push_tiles(
    Dims d, MixedConst c, MixedBMap m, const float4 *__restrict__ E4, const int *__restrict__ bcnd,
    const unsigned char *__restrict__ cw, int *__restrict__ cell, float *__restrict__ p, long long cap,
    const int *__restrict__ count, signed char *__restrict__ flag, const int *__restrict__ tile_off,
    const double *__restrict__ kq, double *__restrict__ np, int *__restrict__ holes, int *__restrict__ nholes,
    double *__restrict__ acc, int *__restrict__ err) {
  __shared__ float4 s_E[TT];
  __shared__ unsigned char s_cw[(TN - 1) * (TN - 1) * (TN - 1)];
  __shared__ float4 s_B[BMAP ? TT : 1];
  float4 *s_st = reinterpret_cast<float4 *>(mx_stage);   // [7][MBK]
  char4 *s_fl = reinterpret_cast<char4 *>(mx_stage + 7 * 16 * MBK);
  int t;
  long long lo, hi;
  part_range<PUSH_PARTS>(tile_off, *count, blockIdx.x, t, lo, hi);
  const int tx = t % c.ntx, ty = (t / c.ntx) % c.nty, tz = t / (c.ntx * c.nty);
  const Tile T{nullptr, s_E, s_cw, tx * TC, ty * TC, tz * TC, s_B};
  const long long first = lo & ~3LL;
  // the copies of this thread's quad at i0 (i0 < hi: i0 + 3 < cap, 16-byte
  // aligned as i0 is a multiple of 4)
  auto fetch = [&](long long i0) {
    if (i0 < hi) {
      cp_async16(&s_st[threadIdx.x], cell + i0);
#pragma unroll
      for (int a = 0; a < 6; ++a) cp_async16(&s_st[(a + 1) * MBK + threadIdx.x], p + a * cap + i0);
      cp_async4(&s_fl[threadIdx.x], flag + i0);
    }
    asm volatile("cp.async.commit_group;" ::: "memory");
  };
  fetch(first + 4 * threadIdx.x);
  for (int e = threadIdx.x; e < TT; e += MBK) {
    const int lx = e % TN, ly = (e / TN) % TN, lz = e / (TN * TN);
    const int gx = T.bx + lx, gy = T.by + ly, gz = T.bz + lz;
    const bool ing = gx <= d.n1 + 2 && gy <= d.n2 + 2 && gz <= d.n3 + 2;
    s_E[e] = ing ? __ldg(E4 + d.g(gx, gy, gz)) : make_float4(0.f, 0.f, 0.f, 0.f);
    if (BMAP && !m.own) s_B[e] = ing ? __ldg(m.B + d.g(gx, gy, gz)) : make_float4(0.f, 0.f, 0.f, 0.f);
  }
  for (int e = threadIdx.x; e < (TN - 1) * (TN - 1) * (TN - 1); e += MBK) {
    const int lx = e % (TN - 1), ly = (e / (TN - 1)) % (TN - 1), lz = e / ((TN - 1) * (TN - 1));
    const int gx = T.bx + lx, gy = T.by + ly, gz = T.bz + lz;
    // cells beyond n+1 exist only when n is not a multiple of the tile edge:
    // they lie outside the grid and count as walls
    s_cw[e] = (gx <= d.n1 + 1 && gy <= d.n2 + 1 && gz <= d.n3 + 1) ? cw[d.c(gx, gy, gz)] : (unsigned char)1;
  }
  __syncthreads();
  for (long long base = first; base < hi; base += CHUNK) {
    Quad Q;
    const long long i0 = base + 4 * threadIdx.x;
    quad_range(Q, i0, lo, hi);
    asm volatile("cp.async.wait_group 0;" ::: "memory");
    if (i0 < hi) {
      Q.c4 = *reinterpret_cast<const int4 *>(&s_st[threadIdx.x]);
#pragma unroll
      for (int a = 0; a < 6; ++a) Q.P[a] = s_st[(a + 1) * MBK + threadIdx.x];
      Q.f4 = s_fl[threadIdx.x];
    } else {
      Q.c4 = make_int4(-1, -1, -1, -1);
      Q.f4 = make_char4(0, 0, 0, 0);
#pragma unroll
      for (int a = 0; a < 6; ++a) Q.P[a] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    fetch(i0 + CHUNK);
    push_quad<BMAP, DIE, false>(d, c, m, T, i0, Q, E4, bcnd, cw, cell, p, cap, flag, kq, np, holes, nholes, acc,
                                err);
  }
  asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// The deposit of a tile's pushed particles (those the push kept: holes, flag
// 2, skipped) into a 32-bit node tile in shared memory, flushed into the FP64
// grid after every FLUSH_PARTICLES particles.  Two node tiles take turns: the
// one a window filled is flushed while the next window adds into the other,
// so a window ends with one block barrier.
__global__ void __launch_bounds__(MBK, 4) k_deposit_tiles(Dims d, int ntx, int nty, double kdep,
                                                        const int *__restrict__ cell, const float *__restrict__ p,
                                                        long long cap, const int *__restrict__ count,
                                                        const signed char *__restrict__ flag,
                                                        const int *__restrict__ tile_off,
                                                        const double *__restrict__ kq, double *__restrict__ np) {
  __shared__ unsigned s_acc[2 * TT];
  int t;
  long long lo, hi;
  part_range<1>(tile_off, *count, blockIdx.x, t, lo, hi);
  const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
  Tile T{s_acc, nullptr, nullptr, tx * TC, ty * TC, tz * TC, nullptr};
  for (int e = threadIdx.x; e < 2 * TT; e += MBK) s_acc[e] = 0u;
  __syncthreads();
  int chunks = 0;
  for (long long base = lo & ~3LL; base < hi; base += CHUNK) {
    const long long i0 = base + 4 * threadIdx.x;
    int cc[4] = {-1, -1, -1, -1};
    float gx[4] = {0.f, 0.f, 0.f, 0.f}, gy[4] = {0.f, 0.f, 0.f, 0.f}, gz[4] = {0.f, 0.f, 0.f, 0.f};
    if (i0 < hi) {
      const int4 c4 = *reinterpret_cast<const int4 *>(cell + i0);
      const char4 f4 = *reinterpret_cast<const char4 *>(flag + i0);
      const float4 P0 = *reinterpret_cast<const float4 *>(p + i0);
      const float4 P1 = *reinterpret_cast<const float4 *>(p + cap + i0);
      const float4 P2 = *reinterpret_cast<const float4 *>(p + 2 * cap + i0);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        if (i0 + k >= lo && i0 + k < hi && (&f4.x)[k] != 2) {
          cc[k] = (&c4.x)[k];
          gx[k] = (&P0.x)[k];
          gy[k] = (&P1.x)[k];
          gz[k] = (&P2.x)[k];
        }
      }
    }
    deposit_quad_warp(d, T, cc, gx, gy, gz, kdep, kq, np);
    if (++chunks == FLUSH_PARTICLES / CHUNK && base + CHUNK < hi) {
      chunks = 0;
      // every add of this window is in T.acc, and every thread has flushed
      // (and cleared) the other tile after the previous barrier
      __syncthreads();
      const Tile F = T;
      T.acc = (T.acc == s_acc) ? s_acc + TT : s_acc;
      flush_tile(d, F, kdep, kq, np);
    }
  }
  __syncthreads();
  flush_tile(d, T, kdep, kq, np);
}

// particles past the last tile (appended since the sort), or all of them
// when no sort has run: deposited straight into the FP64 grid
template <bool BMAP, bool DIE>
__global__ void __launch_bounds__(MBK, 3) k_push_deposit_tail(
    Dims d, MixedConst c, MixedBMap m, const float4 *__restrict__ E4, const int *__restrict__ bcnd,
    const unsigned char *__restrict__ cw, int *__restrict__ cell, float *__restrict__ p, long long cap,
    const int *__restrict__ count, signed char *__restrict__ flag, const int *__restrict__ tile_off,
    const double *__restrict__ kq, double *__restrict__ np, int *__restrict__ holes, int *__restrict__ nholes,
    double *__restrict__ acc, int *__restrict__ err) {
  const Tile T{nullptr, nullptr, nullptr, 0, 0, 0, nullptr};
  const long long N = *count;
  const long long lo = tile_off ? tile_off[c.ntiles] : 0;
  const long long first = lo & ~3LL;
  for (long long base = first + (long long)blockIdx.x * CHUNK; base < N; base += (long long)gridDim.x * CHUNK) {
    Quad Q;
    const long long i0 = base + 4 * threadIdx.x;
    load_quad(Q, i0, lo, N, cell, p, cap, flag);
    push_quad<BMAP, DIE>(d, c, m, T, i0, Q, E4, bcnd, cw, cell, p, cap, flag, kq, np, holes, nholes, acc, err);
  }
}

// hole filling for the mixed layout (the FP64 kernels of the same name in
// step.cu do the same on the FP64 layout)
__global__ void k_fillm_lists(const int *__restrict__ count, const int *__restrict__ holes,
                              const signed char *__restrict__ flag, int *side, int *tailA, int *holeH) {
  const int N = *count, L = side[0], Np = N - L;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < L; t += stride) {
    const int tail = Np + (int)t;
    if (flag[tail] != 2) tailA[atomicAdd(&side[1], 1)] = tail;
    const int h = holes[t];
    if (h < Np) holeH[atomicAdd(&side[2], 1)] = h;
  }
}

__global__ void k_fillm_move(int *__restrict__ cell, float *__restrict__ p, long long cap,
                             const int *__restrict__ count, signed char *__restrict__ flag, const int *side,
                             const int *__restrict__ tailA, const int *__restrict__ holeH) {
  const int N = *count, L = side[0], Np = N - L, na = side[1];
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < na; t += stride) {
    const long long src = tailA[t], dst = holeH[t];
    cell[dst] = cell[src];
#pragma unroll
    for (int a = 0; a < 6; ++a) p[a * cap + dst] = p[a * cap + src];
    flag[dst] = 0;
  }
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < L; t += stride)
    flag[Np + t] = 0;
}

__global__ void k_fillm_count(int *count, const int *side) { *count = *count - side[0]; }

// ---------------------------------------------------------------- sort
// sort key: tile (x-fastest over tiles) * 512 + cell inside the tile
__device__ __forceinline__ int tile_key(int cc, int ntx, int nty) {
  const int cx = cc & CM, cy = (cc >> CB) & CM, cz = cc >> (2 * CB);
  const int tile = (cx / TC) + ntx * ((cy / TC) + nty * (cz / TC));
  return tile * (TC * TC * TC) + (cx % TC) + TC * ((cy % TC) + TC * (cz % TC));
}

__global__ void k_tile_offsets(const int *__restrict__ off, int ntiles, int *__restrict__ tile_off) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t <= ntiles) tile_off[t] = off[(long long)t * (TC * TC * TC)];
}

// Scatter of the counting sort, one block per chunk of SC_N consecutive
// particles.  The block groups its particles by key in shared memory (open
// addressing on the key, the per-key count giving each particle its rank),
// reserves one range per distinct key with a single atomic on that key's
// cursor, stages the particles in key order and writes them out so that
// consecutive threads store consecutive slots of a key's range.
constexpr int SC_T = 256, SC_U = 4, SC_N = SC_T * SC_U, SC_H = 1024, SC_HBITS = 10;
constexpr size_t SC_SMEM = sizeof(int) * (4 * SC_H + 2 * SC_N) + sizeof(float) * 6 * SC_N;
static_assert(SC_H >= SC_N, "the table holds every distinct key of a chunk");

__global__ void __launch_bounds__(SC_T, 4) k_msort_scatter(const int *__restrict__ cell, const float *__restrict__ p,
                                                           int *__restrict__ cell_o, float *__restrict__ p_o,
                                                           long long cap, const int *__restrict__ count, int ntx,
                                                           int nty, int *__restrict__ cursor) {
  extern __shared__ __align__(16) int smi[];
  int *hkey = smi, *hcnt = hkey + SC_H, *hoff = hcnt + SC_H, *hbase = hoff + SC_H;
  int *sdest = hbase + SC_H, *scell = sdest + SC_N;
  float *sp = reinterpret_cast<float *>(scell + SC_N);
  __shared__ int wsum[SC_T / 32];
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const long long N = *count;
  const long long c0 = (long long)blockIdx.x * SC_N;
  if (c0 >= N) return;  // uniform over the block
  for (int q = t; q < SC_H; q += SC_T) {
    hkey[q] = -1;
    hcnt[q] = 0;
  }
  __syncthreads();
  // every load of the chunk first (cells and the six planes), so that their
  // latency overlaps the grouping and the cursor atomics
  int cc[SC_U], slot[SC_U], rank[SC_U];
  float pv[SC_U][6];
#pragma unroll
  for (int u = 0; u < SC_U; ++u) {
    const long long idx = c0 + u * SC_T + t;
    const bool in = idx < N;
    cc[u] = in ? cell[idx] : 0;
#pragma unroll
    for (int a = 0; a < 6; ++a) pv[u][a] = in ? p[a * cap + idx] : 0.f;
  }
#pragma unroll
  for (int u = 0; u < SC_U; ++u) {
    const long long idx = c0 + u * SC_T + t;
    slot[u] = -1;
    rank[u] = 0;
    if (idx < N) {
      const int key = tile_key(cc[u], ntx, nty);
      unsigned h = ((unsigned)key * 2654435761u) >> (32 - SC_HBITS);
      // at most SC_N distinct keys per chunk: a free or matching slot exists
      for (int probe = 0; probe < SC_H; ++probe) {
        const int prev = atomicCAS(&hkey[h], -1, key);
        if (prev == -1 || prev == key) break;
        h = (h + 1) & (SC_H - 1);
      }
      slot[u] = (int)h;
      rank[u] = atomicAdd(&hcnt[h], 1);
    }
  }
  __syncthreads();
  {
    // exclusive scan of the slot counts (four slots per thread), then one
    // range per distinct key from its global cursor
    constexpr int PER = SC_H / SC_T;
    int v[PER];
    int sum = 0;
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      v[j] = hcnt[t * PER + j];
      sum += v[j];
    }
    int incl = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wsum[warp] = incl;
    __syncthreads();
    int run = incl - sum;
    for (int w = 0; w < warp; ++w) run += wsum[w];
#pragma unroll
    for (int j = 0; j < PER; ++j) {
      hoff[t * PER + j] = run;
      run += v[j];
      if (v[j]) hbase[t * PER + j] = atomicAdd(&cursor[hkey[t * PER + j]], v[j]);
    }
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < SC_U; ++u) {
    if (slot[u] < 0) continue;
    const int lpos = hoff[slot[u]] + rank[u];
    sdest[lpos] = hbase[slot[u]] + rank[u];
    scell[lpos] = cc[u];
#pragma unroll
    for (int a = 0; a < 6; ++a) sp[a * SC_N + lpos] = pv[u][a];
  }
  __syncthreads();
  const int nv = N - c0 < SC_N ? (int)(N - c0) : SC_N;
  for (int lp = t; lp < nv; lp += SC_T) {
    const long long dst = sdest[lp];
    cell_o[dst] = scell[lp];
#pragma unroll
    for (int a = 0; a < 6; ++a) p_o[a * cap + dst] = sp[a * SC_N + lp];
  }
}

// Counts per key of the counting sort, one block per chunk of SC_N
// particles: the chunk's keys are counted in a shared-memory table (open
// addressing) and each distinct key adds its count to the global histogram
// once, instead of one atomic per warp run.
__global__ void __launch_bounds__(SC_T) k_msort_hist(const int *__restrict__ cell, const int *__restrict__ count,
                                                     int ntx, int nty, int *__restrict__ cnt) {
  __shared__ int hkey[SC_H], hcnt[SC_H];
  const int t = threadIdx.x;
  const long long N = *count;
  const long long c0 = (long long)blockIdx.x * SC_N;
  if (c0 >= N) return;  // uniform over the block
  for (int q = t; q < SC_H; q += SC_T) {
    hkey[q] = -1;
    hcnt[q] = 0;
  }
  int key[SC_U];
#pragma unroll
  for (int u = 0; u < SC_U; ++u) {
    const long long idx = c0 + u * SC_T + t;
    key[u] = idx < N ? cell[idx] : -1;
  }
  __syncthreads();
#pragma unroll
  for (int u = 0; u < SC_U; ++u) {
    if (key[u] < 0) continue;
    const int k = tile_key(key[u], ntx, nty);
    unsigned h = ((unsigned)k * 2654435761u) >> (32 - SC_HBITS);
    for (int probe = 0; probe < SC_H; ++probe) {
      const int prev = atomicCAS(&hkey[h], -1, k);
      if (prev == -1 || prev == k) break;
      h = (h + 1) & (SC_H - 1);
    }
    atomicAdd(&hcnt[h], 1);
  }
  __syncthreads();
  for (int q = t; q < SC_H; q += SC_T)
    if (hcnt[q]) atomicAdd(&cnt[hkey[q]], hcnt[q]);
}

// E (3, nodes) FP64 -> one float4 (Ex, Ey, Ez, 0) per node
__global__ void k_pack_e32(const double *__restrict__ Ei, float4 *__restrict__ E4, long long nodes) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < nodes) E4[i] = make_float4((float)Ei[3 * i], (float)Ei[3 * i + 1], (float)Ei[3 * i + 2], 0.f);
}

// FP64 SoA (x,y,z,vx,vy,vz) -> mixed layout
__global__ void k_f64_to_mixed(Dims d, double h0, double h1, double h2, const double *__restrict__ pin,
                               long long capin, int *__restrict__ cell, float *__restrict__ p,
                               long long cap, long long n, int *err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = pin[i], y = pin[capin + i], z = pin[2 * capin + i];
  int ix = (int)(x / h0) + 1, iy = (int)(y / h1) + 1, iz = (int)(z / h2) + 1;
  if (ix < 1 || ix > d.n1 || iy < 1 || iy > d.n2 || iz < 1 || iz > d.n3 || !(x >= 0 && y >= 0 && z >= 0)) {
    raise_err(err, LEPIC_ERR_CELL, (int)i);
    ix = ix < 1 ? 1 : (ix > d.n1 ? d.n1 : ix);
    iy = iy < 1 ? 1 : (iy > d.n2 ? d.n2 : iy);
    iz = iz < 1 ? 1 : (iz > d.n3 ? d.n3 : iz);
  }
  cell[i] = (ix - 1) | (iy - 1) << CB | (iz - 1) << (2 * CB);
  const float fx = (float)(x / h0 - (ix - 1)), fy = (float)(y / h1 - (iy - 1)), fz = (float)(z / h2 - (iz - 1));
  p[i] = fx >= 1.f ? 0.99999994f : fx;
  p[cap + i] = fy >= 1.f ? 0.99999994f : fy;
  p[2 * cap + i] = fz >= 1.f ? 0.99999994f : fz;
  p[3 * cap + i] = (float)pin[3 * capin + i];
  p[4 * cap + i] = (float)pin[4 * capin + i];
  p[5 * cap + i] = (float)pin[5 * capin + i];
}

// mixed layout -> FP64 SoA (positions x = (ix-1+f) h)
__global__ void k_mixed_to_f64(Dims d, double h0, double h1, double h2, const int *__restrict__ cell,
                               const float *__restrict__ p, long long cap, double *__restrict__ pout,
                               long long capout, long long n) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int cc = cell[i];
  const int ix = cc & CM, iy = (cc >> CB) & CM, iz = cc >> (2 * CB);
  pout[i] = ((double)ix + (double)p[i]) * h0;
  pout[capout + i] = ((double)iy + (double)p[cap + i]) * h1;
  pout[2 * capout + i] = ((double)iz + (double)p[2 * cap + i]) * h2;
  pout[3 * capout + i] = p[3 * cap + i];
  pout[4 * capout + i] = p[4 * cap + i];
  pout[5 * capout + i] = p[5 * cap + i];
}

// GPU particle loader for the mixed layout: the draws of k_load_uniform
// (Philox4x32-10 per sample: positions uniform in the loading box outside
// all-wall cells, co-located species, Maxwellian velocities of the
// load_gauss form of Src/load_part.f90:233-244) written as cell + FP32
// offsets and velocities, so that large workloads need no FP64 copy.
struct LoadMixed {
  double xl, ym, zm, h0, h1, h2;
  double vt[LEPIC_NPART];
  int ntype;
  unsigned k0, k1;
  int *cell[LEPIC_NPART];
  float *p[LEPIC_NPART];
  long long cap[LEPIC_NPART];
};

__global__ void k_load_uniform_mixed(Dims d, LoadMixed c, long long n, const unsigned char *__restrict__ cw,
                                     int *err) {
  const long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double x = 0, y = 0, z = 0;
  int ix = 1, iy = 1, iz = 1;
  bool ok = false;
  for (uint32_t tr = 0; tr < 64 && !ok; ++tr) {
    U4 r = philox4x32_10({(uint32_t)j, (uint32_t)(j >> 32), tr, 0xA5A5u}, c.k0, c.k1);
    x = u01(r.x) * c.xl;
    y = u01(r.y) * c.ym;
    z = u01(r.z) * c.zm;
    ix = (int)(x / c.h0) + 1;
    iy = (int)(y / c.h1) + 1;
    iz = (int)(z / c.h2) + 1;
    ok = !cw[d.c(ix, iy, iz)];
  }
  if (!ok) raise_err(err, LEPIC_ERR_CELL, (int)j);
  ix = ix > d.n1 ? d.n1 : ix;
  iy = iy > d.n2 ? d.n2 : iy;
  iz = iz > d.n3 ? d.n3 : iz;
  const int cc = (ix - 1) | (iy - 1) << CB | (iz - 1) << (2 * CB);
  float fx = (float)(x / c.h0 - (ix - 1)), fy = (float)(y / c.h1 - (iy - 1)), fz = (float)(z / c.h2 - (iz - 1));
  fx = fx >= 1.f ? 0.99999994f : fx;
  fy = fy >= 1.f ? 0.99999994f : fy;
  fz = fz >= 1.f ? 0.99999994f : fz;
  for (int q = 0; q < c.ntype; ++q) {
    U4 r = philox4x32_10({(uint32_t)j, (uint32_t)(j >> 32), 1000u + q, 0x5A5Au}, c.k0, c.k1);
    const double vt = c.vt[q];
    double s1, c1, s2, c2;
    sincos(2.0 * 3.141592653589793 * u01(r.y), &s1, &c1);
    sincos(2.0 * 3.141592653589793 * u01(r.w), &s2, &c2);
    const double vp = vt * sqrt(-log(u01(r.x)));
    const double vq = vt * sqrt(-log(u01(r.z)));
    float *P = c.p[q];
    const long long cap = c.cap[q];
    c.cell[q][j] = cc;
    P[j] = fx;
    P[cap + j] = fy;
    P[2 * cap + j] = fz;
    P[3 * cap + j] = (float)(vp * c1);
    P[4 * cap + j] = (float)(vp * s1);
    P[5 * cap + j] = (float)(vq * c2);
  }
}

// CIC deposition of a mixed-layout species with the integer weights of the
// push (the initial charge of a loaded state)
__global__ void k_deposit_mixed(Dims d, double kdep, const int *__restrict__ cell, const float *__restrict__ p,
                                long long cap, const int *__restrict__ count, const double *__restrict__ kq,
                                double *__restrict__ np, int *err) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= *count) return;
  const int cc = cell[i];
  const int ix = (cc & CM) + 1, iy = ((cc >> CB) & CM) + 1, iz = (cc >> (2 * CB)) + 1;
  if (cc < 0 || ix > d.n1 || iy > d.n2 || iz > d.n3) {
    raise_err(err, LEPIC_ERR_CELL, (int)i);
    return;
  }
  int w[8];
  qweights(p[i], p[cap + i], p[2 * cap + i], w);
  const Tile T{nullptr, nullptr, nullptr, 0, 0, 0, nullptr};
  deposit8(d, T, ix, iy, iz, w, kdep, kq, np);
}

bool aligned16(const void *q) { return ((uintptr_t)q & 15u) == 0; }

// the FP32 copy (Bx, By, Bz, |B|) of the FP64 map Bi(4, ...)
__global__ void k_pack_b32(const double *__restrict__ Bi, long long nodes, float4 *__restrict__ B4) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nodes; q += stride)
    B4[q] = make_float4((float)Bi[4 * q], (float)Bi[4 * q + 1], (float)Bi[4 * q + 2], (float)Bi[4 * q + 3]);
}

int check_layout(const lepic_grid_t &g, const lepic_species_mixed_t &sp) {
  if (g.n[0] > LEPIC_CELL_MAX || g.n[1] > LEPIC_CELL_MAX || g.n[2] > LEPIC_CELL_MAX) return LEPIC_ERR_UNSUPPORTED;
  if (sp.cap % 4 || !aligned16(sp.cell) || !aligned16(sp.p) || !aligned16(sp.cell_alt) || !aligned16(sp.p_alt) ||
      ((uintptr_t)sp.flag_dead & 3u))
    return LEPIC_ERR_ARG;
  return LEPIC_OK;
}

}  // namespace

int launch_push_deposit_mixed(const lepic_grid_t &g, const float *E4, lepic_species_mixed_t &sp,
                              int ptype, int ngrid, const lepic_phys_t &P, double *np, double *acc,
                              int n_hint, cudaStream_t s) {
  Dims d(g.n);
  const int p = ptype - 1;
  if (!sp.flag_dead || !aligned16(E4)) return LEPIC_ERR_ARG;
  if (int rc = check_layout(g, sp)) return rc;
  MixedConst c;
  memset(&c, 0, sizeof(c));
  c.dth0 = (float)(P.dt / g.h[0]);
  c.dth1 = (float)(P.dt / g.h[1]);
  c.dth2 = (float)(P.dt / g.h[2]);
  c.k1 = (float)(P.dt * P.charge[p] / (2.0 * P.mass[p]));
  {
    const float k1 = c.k1, Bx = (float)P.Bconst[0], By = (float)P.Bconst[1], Bz = (float)P.Bconst[2];
    const float B_tot = sqrtf(Bx * Bx + By * By + Bz * Bz);
    c.kk = k1 * (2.f / (1.f + (k1 * B_tot) * (k1 * B_tot)));
  }
  c.Bx = (float)P.Bconst[0];
  c.By = (float)P.Bconst[1];
  c.Bz = (float)P.Bconst[2];
  c.boris = (P.flag_B == 1) ? 1 : 0;
  if (P.flag_B_pos == 1 && P.charge[p] > 0.0) c.boris = 0;
  c.flag_pbc = P.flag_pbc;
  c.flag_nmn = P.flag_nmn;
  c.ngrid = ngrid;
  c.die = dielectric_from_phys(P, g.n, ptype);
  c.Nm = P.Nm[p];
  c.mass = P.mass[p];
  c.kdep = P.Nm[p] / (g.h[0] * g.h[1] * g.h[2]);
  c.ntx = (d.n1 + TC - 1) / TC;
  c.nty = (d.n2 + TC - 1) / TC;
  c.ntiles = LEPIC_TILES(g.n);
  const size_t cap = (size_t)sp.cap;
  char nm[32];
  snprintf(nm, sizeof nm, "work_list%d", p);
  int *holes = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "mixed_tail%d", p);
  int *tailA = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "mixed_hh%d", p);
  int *holeH = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "mixed_side%d", p);
  int *side = (int *)scratch(nm, sizeof(int) * 4);
  if (!holes || !tailA || !holeH || !side) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(side, 0, sizeof(int) * 4, s));
  // B-field map: an FP32 copy made at every call (the map may change
  // between calls; (n_B+3)^3 x 48 B of traffic)
  MixedBMap m;
  memset(&m, 0, sizeof(m));
  {
    BMapF64 m64;
    if (int rc = bmap_from_phys(P, g.n, m64)) return rc;
    if (m64.B) {
      const long long nodes = m64.N1 * m64.N2 * (long long)(m64.nb3 + 3);
      float4 *B4 = (float4 *)scratch("bmap_f32", sizeof(float4) * (size_t)nodes);
      if (!B4) return LEPIC_ERR_CUDA;
      k_pack_b32<<<ctx().sms * 4, 256, 0, s>>>(m64.B, nodes, B4);
      LEPIC_CUDA(cudaGetLastError());
      m.B = B4;
      m.own = m64.own;
      m.nb1 = m64.nb1;
      m.nb2 = m64.nb2;
      m.nb3 = m64.nb3;
      m.N1 = m64.N1;
      m.N2 = m64.N2;
      if (m.own) {
        m.r0 = (float)(g.h[0] / m64.h0);
        m.r1 = (float)(g.h[1] / m64.h1);
        m.r2 = (float)(g.h[2] / m64.h2);
      }
    }
  }
  const float4 *E = reinterpret_cast<const float4 *>(E4);
  int t0 = timer_start("push_mixed", s);
  // the tail: at most what was appended since the sort unless never sorted
  long long tail = sp.tile_off ? (long long)ctx().sms * 2 : grid_for(n_hint > 0 ? n_hint : sp.cap, CHUNK);
  if (tail > (long long)ctx().sms * 8) tail = (long long)ctx().sms * 8;
  // four instances: B map or uniform B, dielectric walls or none (the
  // uniform kernels without walls keep their registers)
  auto run = [&](auto bmap, auto die) {
    constexpr bool B = decltype(bmap)::value, D = decltype(die)::value;
    if (sp.tile_off) {
      LEPIC_CUDA(cudaFuncSetAttribute(k_push_tiles<B, D>, cudaFuncAttributeMaxDynamicSharedMemorySize, STAGE_BYTES));
      k_push_tiles<B, D><<<c.ntiles * PUSH_PARTS, MBK, STAGE_BYTES, s>>>(d, c, m, E, g.bcnd, g.cell_wall, sp.cell, sp.p, sp.cap,
                                                            sp.count, sp.flag_dead, sp.tile_off, g.kq, np, holes,
                                                            side, acc, ctx().d_err);
    }
    return LEPIC_OK;
  };
  const bool die = c.die.dtype != nullptr;
  int rc;
  if (m.B && die)
    rc = run(std::true_type{}, std::true_type{});
  else if (m.B)
    rc = run(std::true_type{}, std::false_type{});
  else if (die)
    rc = run(std::false_type{}, std::true_type{});
  else
    rc = run(std::false_type{}, std::false_type{});
  timer_stop(t0, s);
  if (rc) return rc;
  int td = timer_start("deposit_mixed_tiles", s);
  if (sp.tile_off)
    k_deposit_tiles<<<c.ntiles, MBK, 0, s>>>(d, c.ntx, c.nty, c.kdep, sp.cell, sp.p, sp.cap, sp.count, sp.flag_dead,
                                             sp.tile_off, g.kq, np);
  timer_stop(td, s);
  // the tail (appended since the sort): push and deposit in one pass
  int t2 = timer_start("push_deposit_mixed_tail", s);
  auto run_tail = [&](auto bmap, auto die) {
    constexpr bool B = decltype(bmap)::value, D = decltype(die)::value;
    k_push_deposit_tail<B, D><<<(int)tail, MBK, 0, s>>>(d, c, m, E, g.bcnd, g.cell_wall, sp.cell, sp.p, sp.cap,
                                                        sp.count, sp.flag_dead, sp.tile_off, g.kq, np, holes,
                                                        side, acc, ctx().d_err);
  };
  if (m.B && die)
    run_tail(std::true_type{}, std::true_type{});
  else if (m.B)
    run_tail(std::true_type{}, std::false_type{});
  else if (die)
    run_tail(std::false_type{}, std::true_type{});
  else
    run_tail(std::false_type{}, std::false_type{});
  timer_stop(t2, s);
  LEPIC_CUDA(cudaGetLastError());
  int t1 = timer_start("fill_holes_mixed", s);
  const int fb = ctx().sms * 2;
  k_fillm_lists<<<fb, 256, 0, s>>>(sp.count, holes, sp.flag_dead, side, tailA, holeH);
  k_fillm_move<<<fb, 256, 0, s>>>(sp.cell, sp.p, sp.cap, sp.count, sp.flag_dead, side, tailA, holeH);
  k_fillm_count<<<1, 1, 0, s>>>(sp.count, side);
  timer_stop(t1, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int launch_sort_mixed(const lepic_grid_t &g, lepic_species_mixed_t &sp, int n_hint, cudaStream_t s) {
  Dims d(g.n);
  if (int rc = check_layout(g, sp)) return rc;
  const int ntx = (d.n1 + TC - 1) / TC, nty = (d.n2 + TC - 1) / TC;
  const int ntiles = LEPIC_TILES(g.n);
  const long long nkeys = (long long)ntiles * TC * TC * TC;
  int *cnt = (int *)scratch("msort_cnt", sizeof(int) * (size_t)(nkeys + 1));
  if (!cnt) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(nkeys + 1), s));
  const int nthreads = n_hint > 0 ? n_hint : sp.cap;
  int t0 = timer_start("sort_hist_mixed", s);
  k_msort_hist<<<grid_for(nthreads, SC_N), SC_T, 0, s>>>(sp.cell, sp.count, ntx, nty, cnt);
  timer_stop(t0, s);
  int t1 = timer_start("sort_scan_mixed", s);
  int rc = exclusive_scan_i32(cnt, cnt, nkeys + 1, s);
  timer_stop(t1, s);
  if (rc) return rc;
  if (sp.tile_off) k_tile_offsets<<<grid_for(ntiles + 1, 256), 256, 0, s>>>(cnt, ntiles, sp.tile_off);
  // the start of every cell, kept for charged-target collisions
  if (sp.cell_off)
    LEPIC_CUDA(cudaMemcpyAsync(sp.cell_off, cnt, sizeof(int) * (size_t)(nkeys + 1), cudaMemcpyDeviceToDevice, s));
  LEPIC_CUDA(cudaFuncSetAttribute(k_msort_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SC_SMEM));
  int t2 = timer_start("sort_scatter_mixed", s);
  k_msort_scatter<<<grid_for(nthreads, SC_N), SC_T, SC_SMEM, s>>>(sp.cell, sp.p, sp.cell_alt, sp.p_alt, sp.cap,
                                                                  sp.count, ntx, nty, cnt);
  timer_stop(t2, s);
  LEPIC_CUDA(cudaGetLastError());
  int *tc = sp.cell;
  sp.cell = sp.cell_alt;
  sp.cell_alt = tc;
  float *tp = sp.p;
  sp.p = sp.p_alt;
  sp.p_alt = tp;
  return LEPIC_OK;
}

int launch_load_uniform_mixed(const lepic_grid_t &g, lepic_species_mixed_t *sp, int ntype, long long n,
                              const lepic_phys_t &P, unsigned long long seed, cudaStream_t s) {
  Dims d(g.n);
  if (ntype < 1 || ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  LoadMixed c;
  memset(&c, 0, sizeof(c));
  c.xl = P.x_load;
  c.ym = P.ymax;
  c.zm = P.zmax;
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  for (int q = 0; q < LEPIC_NPART; ++q) c.vt[q] = P.vt0[q];
  c.ntype = ntype;
  c.k0 = (unsigned)(seed & 0xffffffffu);
  c.k1 = (unsigned)(seed >> 32);
  for (int q = 0; q < ntype; ++q) {
    if (int rc = check_layout(g, sp[q])) return rc;
    if (n > sp[q].cap) return LEPIC_ERR_CAPACITY;
    c.cell[q] = sp[q].cell;
    c.p[q] = sp[q].p;
    c.cap[q] = sp[q].cap;
  }
  if (n > 0) k_load_uniform_mixed<<<grid_for(n, 256), 256, 0, s>>>(d, c, n, g.cell_wall, ctx().d_err);
  LEPIC_CUDA(cudaGetLastError());
  const int nn = (int)n;
  for (int q = 0; q < ntype; ++q) {
    LEPIC_CUDA(cudaMemcpyAsync(sp[q].count, &nn, sizeof(int), cudaMemcpyHostToDevice, s));
    if (sp[q].tile_off) LEPIC_CUDA(cudaMemsetAsync(sp[q].tile_off, 0, sizeof(int) * (LEPIC_TILES(g.n) + 1), s));
  }
  return check_err(s);
}

int launch_deposit_mixed(const lepic_grid_t &g, const lepic_species_mixed_t &sp, int ptype, const lepic_phys_t &P,
                         double *np, int n_hint, cudaStream_t s) {
  Dims d(g.n);
  const double kdep = P.Nm[ptype - 1] / (g.h[0] * g.h[1] * g.h[2]);
  const int nthreads = n_hint > 0 ? n_hint : sp.cap;
  k_deposit_mixed<<<grid_for(nthreads, 256), 256, 0, s>>>(d, kdep, sp.cell, sp.p, sp.cap, sp.count, g.kq, np,
                                                        ctx().d_err);
  LEPIC_CUDA(cudaGetLastError());
  return check_err(s);
}

int launch_pack_e32(const double *Ei, float *E4, long long nodes, cudaStream_t s) {
  if (!aligned16(E4)) return LEPIC_ERR_ARG;
  k_pack_e32<<<grid_for(nodes, 256), 256, 0, s>>>(Ei, reinterpret_cast<float4 *>(E4), nodes);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int launch_convert_f64_to_mixed(const lepic_grid_t &g, const lepic_species_f64_t &in, lepic_species_mixed_t &out,
                                long long n, cudaStream_t s) {
  Dims d(g.n);
  if (n > out.cap) return LEPIC_ERR_CAPACITY;
  if (n > 0)
    k_f64_to_mixed<<<grid_for(n, 256), 256, 0, s>>>(d, g.h[0], g.h[1], g.h[2], in.p, in.cap, out.cell, out.p,
                                                   out.cap, n, ctx().d_err);
  int nn = (int)n;
  LEPIC_CUDA(cudaMemcpyAsync(out.count, &nn, sizeof(int), cudaMemcpyHostToDevice, s));
  if (out.tile_off) LEPIC_CUDA(cudaMemsetAsync(out.tile_off, 0, sizeof(int) * (LEPIC_TILES(g.n) + 1), s));
  return check_err(s);
}

int launch_convert_mixed_to_f64(const lepic_grid_t &g, const lepic_species_mixed_t &in, double *out,
                                long long capout, long long n, cudaStream_t s) {
  Dims d(g.n);
  if (n > 0)
    k_mixed_to_f64<<<grid_for(n, 256), 256, 0, s>>>(d, g.h[0], g.h[1], g.h[2], in.cell, in.p, in.cap, out,
                                                   capout, n);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

}  // namespace lepic

extern "C" {

int lepic_dev_push_deposit_mixed(const lepic_grid_t *g, const float *E4, lepic_species_mixed_t *s,
                                 int ptype, int ngrid, const lepic_phys_t *P, double *np, double *acc,
                                 int n_hint, void *stream) {
  if (!g || !s || !P || ptype < 1 || !acc || !E4 || !np) return LEPIC_ERR_ARG;
  return lepic::launch_push_deposit_mixed(*g, E4, *s, ptype, ngrid, *P, np, acc, n_hint, (cudaStream_t)stream);
}

int lepic_dev_sort_mixed(const lepic_grid_t *g, lepic_species_mixed_t *s, int n_hint, void *stream) {
  if (!g || !s) return LEPIC_ERR_ARG;
  return lepic::launch_sort_mixed(*g, *s, n_hint, (cudaStream_t)stream);
}

int lepic_dev_load_uniform_mixed(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype,
                                 long long n_per_species, const lepic_phys_t *P, unsigned long long seed,
                                 void *stream) {
  if (!g || !sp || !P || n_per_species < 0) return LEPIC_ERR_ARG;
  return lepic::launch_load_uniform_mixed(*g, sp, ntype, n_per_species, *P, seed, (cudaStream_t)stream);
}

int lepic_dev_deposit_mixed(const lepic_grid_t *g, const lepic_species_mixed_t *s, int ptype, const lepic_phys_t *P,
                            double *np, int n_hint, void *stream) {
  if (!g || !s || !P || !np || ptype < 1) return LEPIC_ERR_ARG;
  return lepic::launch_deposit_mixed(*g, *s, ptype, *P, np, n_hint, (cudaStream_t)stream);
}

int lepic_dev_pack_e32(const double *Ei, float *E4, long long nodes, void *stream) {
  if (!Ei || !E4 || nodes < 0) return LEPIC_ERR_ARG;
  return lepic::launch_pack_e32(Ei, E4, nodes, (cudaStream_t)stream);
}

int lepic_dev_f64_to_mixed(const lepic_grid_t *g, const lepic_species_f64_t *in, lepic_species_mixed_t *out,
                           long long n, void *stream) {
  if (!g || !in || !out || n < 0) return LEPIC_ERR_ARG;
  return lepic::launch_convert_f64_to_mixed(*g, *in, *out, n, (cudaStream_t)stream);
}

int lepic_dev_mixed_to_f64(const lepic_grid_t *g, const lepic_species_mixed_t *in, double *out,
                           long long capout, long long n, void *stream) {
  if (!g || !in || !out || n < 0) return LEPIC_ERR_ARG;
  return lepic::launch_convert_mixed_to_f64(*g, *in, out, capout, n, (cudaStream_t)stream);
}

}  // extern "C"
