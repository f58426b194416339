// FP64 particle kernels: Boris push + loss test + in-order compaction
// (Src/part_expmover.f90:1-482), CIC deposition (Src/part_expmover.f90:570-686)
// and the counting sort by cell (Src/sorting.f90:97-258).
//
// Particles are SoA (x, y, z, vx, vy, vz planes of `cap` doubles), so every
// pass reads and writes fully coalesced 8-byte streams.  The push and the
// deposition weights keep the Fortran expression order and the file is built
// with --fmad=false: one push of one particle reproduces the CPU oracle bit
// for bit.  Deposition and the sort scatter use atomics, so the summation
// order of rho and the order of particles inside one cell are not fixed
// (exactly as in the reference's OpenMP build).
#include <cstring>
#include <vector>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int PB = 256;

struct PushConst {
  double h0, h1, h2, dt, k1, Nm, mass;
  double Bx, By, Bz;
  int boris;        // 1: Boris, 0: leapfrog
  int flag_nmn, flag_pbc;
  double ymax, zmax;
  int ngrid;
};

// gather + Boris/leapfrog + position update of one particle; returns the
// post-push cell (clamped) for the loss test.  Src/part_expmover.f90:89-272.
// BMAP: B from the map m (else the uniform c.Bx, c.By, c.Bz).
template <bool BMAP>
__device__ __forceinline__ void push_one(const Dims &d, const PushConst &c, const BMapF64 &m,
                                         const double *__restrict__ Ei, double &xp, double &yp, double &zp,
                                         double &vx, double &vy, double &vz, int &ixn, int &iyn, int &izn) {
  int ix = (int)(xp / c.h0) + 1, iy = (int)(yp / c.h1) + 1, iz = (int)(zp / c.h2) + 1;
  double px = (ix * c.h0 - xp) / c.h0;
  double py = (iy * c.h1 - yp) / c.h1;
  double pz = (iz * c.h2 - zp) / c.h2;
  double k0 = px * py * pz;
  double kk1 = (1.0 - px) * py * pz;
  double k2 = (1.0 - px) * (1.0 - py) * pz;
  double k3 = px * (1.0 - py) * pz;
  double k4 = px * py * (1.0 - pz);
  double k5 = (1.0 - px) * py * (1.0 - pz);
  double k6 = (1.0 - px) * (1.0 - py) * (1.0 - pz);
  double k7 = px * (1.0 - py) * (1.0 - pz);
  const long long sy = d.N1, sz = d.N1 * d.N2;
  long long q = d.g(ix, iy, iz);
  const double *e0 = Ei + 3 * q, *e1 = Ei + 3 * (q + 1), *e2 = Ei + 3 * (q + 1 + sy),
               *e3 = Ei + 3 * (q + sy), *e4 = Ei + 3 * (q + sz), *e5 = Ei + 3 * (q + 1 + sz),
               *e6 = Ei + 3 * (q + 1 + sy + sz), *e7 = Ei + 3 * (q + sy + sz);
  double E[3];
#pragma unroll
  for (int a = 0; a < 3; ++a)
    E[a] = k0 * __ldg(e0 + a) + kk1 * __ldg(e1 + a) + k2 * __ldg(e2 + a) + k3 * __ldg(e3 + a) +
           k4 * __ldg(e4 + a) + k5 * __ldg(e5 + a) + k6 * __ldg(e6 + a) + k7 * __ldg(e7 + a);
  const double k1 = c.k1;
  double Bx = c.Bx, By = c.By, Bz = c.Bz;
  bool boris = c.boris;
  if (BMAP && boris) {
    const double kE[8] = {k0, kk1, k2, k3, k4, k5, k6, k7};
    boris = bmap_gather_f64(m, xp, yp, zp, ix, iy, iz, kE, Bx, By, Bz);
  }
  if (boris) {
    double B_tot = sqrt(Bx * Bx + By * By + Bz * Bz);
    double kb = k1 * (2.0 / (1.0 + (k1 * B_tot) * (k1 * B_tot)));
    double v1x = vx + k1 * E[0], v1y = vy + k1 * E[1], v1z = vz + k1 * E[2];
    double v3x = v1x + k1 * (v1y * Bz - v1z * By);
    double v3y = v1y + k1 * (v1z * Bx - v1x * Bz);
    double v3z = v1z + k1 * (v1x * By - v1y * Bx);
    double v2x = v1x + kb * (v3y * Bz - v3z * By);
    double v2y = v1y + kb * (v3z * Bx - v3x * Bz);
    double v2z = v1z + kb * (v3x * By - v3y * Bx);
    vx = v2x + k1 * E[0];
    vy = v2y + k1 * E[1];
    vz = v2z + k1 * E[2];
  } else {
    vx = vx + 2.0 * k1 * E[0];
    vy = vy + 2.0 * k1 * E[1];
    vz = vz + 2.0 * k1 * E[2];
  }
  xp = xp + c.dt * vx;
  yp = yp + c.dt * vy;
  zp = zp + c.dt * vz;
  ixn = (int)floor(xp / c.h0) + 1;
  iyn = (int)floor(yp / c.h1) + 1;
  izn = (int)floor(zp / c.h2) + 1;
  ixn = ixn < 0 ? 0 : (ixn > d.n1 + 1 ? d.n1 + 1 : ixn);
  iyn = iyn < 0 ? 0 : (iyn > d.n2 + 1 ? d.n2 + 1 : iyn);
  izn = izn < 0 ? 0 : (izn > d.n3 + 1 ? d.n3 + 1 : izn);
}

// The negative-ion bookkeeping and the secondary emission of the drop-in
// mover (Src/part_expmover.f90:76, 278-301, 353-400, 416-470).
struct MoverExtra {
  int neg;                   // this species is tag_neg
  int tag_neu, num_grd;
  const int *cex;            // flag_cex of the species, slot order (neg)
  int *cnt_cex;              // [3]
  double *cnt_dead;          // [1]
  double *beam_div;          // [4]
  double k_dead;             // Nm q of the species
  int sec;                   // secondary emission (a positive species, gam_sec > 0)
  int igrid_sec;
  double gam, vt, zg0, zg1;  // gam_sec, sqrt(2 qe |THm| / m_e), cathode planes
  double Nm1, m1;            // species 1
  double *p1;                // species 1 planes, capacity cap1, count count1
  long long cap1;
  int *count1;
  double *ploss4;            // [1]: P_loss(4, species 1)
  uint32_t k0, k1, call;     // Philox key and call counter
  double pi;
};

// Secondary electrons of an ion lost on the emissive grid: INT(gam) of
// them, one more with probability gam - INT(gam), appended behind species
// 1's count at the ion's (x, y) on the cathode plane it moved towards, with
// a flux-Maxwellian normal velocity and the Gaussian transverse velocity of
// load_gauss (Src/load_part.f90:268-291).  The reference draws from its
// serial ran2 stream; here Philox4x32-10 keyed by (ion slot, call).
__device__ void emit_secondaries(const MoverExtra &x, long long i, double xp, double yp, double vz_ion, int *err) {
  const U4 r0 = philox4x32_10({(uint32_t)i, (uint32_t)(i >> 32), x.call, 0x53454330u}, x.k0, x.k1);
  int n_sec = (int)x.gam;
  if (u01(r0.x) <= x.gam - n_sec) n_sec += 1;
  for (int k = 0; k < n_sec; ++k) {
    const U4 r = philox4x32_10({(uint32_t)i, (uint32_t)(i >> 32), x.call, 0x53454331u + (uint32_t)k}, x.k0, x.k1);
    const double vz = (vz_ion >= 0.0 ? -1.0 : 1.0) * x.vt * sqrt(-log(1.0 - u01(r.x)));
    const double vp = x.vt * sqrt(-log(1.0 - u01(r.y))), theta = 2.0 * x.pi * u01(r.z);
    const double vxs = vp * cos(theta), vys = vp * sin(theta);
    const int slot = atomicAdd(x.count1, 1);
    if (slot >= x.cap1) {
      atomicSub(x.count1, 1);
      raise_err(err, LEPIC_ERR_CAPACITY, (int)i);
      return;
    }
    double *q = x.p1 + slot;
    q[0] = xp;
    q[x.cap1] = yp;
    q[2 * x.cap1] = vz_ion < 0.0 ? x.zg0 : x.zg1;
    q[3 * x.cap1] = vxs;
    q[4 * x.cap1] = vys;
    q[5 * x.cap1] = vz;
    // P_loss(4,1) as the reference sums it (vz twice, vy not at all)
    atomicAdd(x.ploss4, 0.5 * x.Nm1 * x.m1 * (vxs * vxs + vz * vz + vz * vz));
  }
}

// Loss accumulators: acc[0] P_loss(1), acc[1] P_loss(3), acc[2+2g] p_mac
// count at label g, acc[3+2g] p_mac energy at label g.
template <bool BMAP>
__global__ void __launch_bounds__(PB) k_push_f64(Dims d, PushConst c, BMapF64 m, Dielectric die, MoverExtra x,
                                                 const double *__restrict__ Ei,
                                                 const int *__restrict__ bcnd,
                                                 const unsigned char *__restrict__ cw,
                                                 const double *__restrict__ pin, double *__restrict__ pout,
                                                 long long cap, const int *__restrict__ count,
                                                 signed char *flag_dead, int *__restrict__ keep,
                                                 double *acc, int *err) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int N = *count;
  if (i >= N) return;
  double xp = pin[i], yp = pin[cap + i], zp = pin[2 * cap + i];
  double vx = pin[3 * cap + i], vy = pin[4 * cap + i], vz = pin[5 * cap + i];
  if (flag_dead && flag_dead[i] == 1) {
    flag_dead[i] = 0;
    double Eki = 0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz);
    atomicAdd(&acc[1], -Eki);
    if (x.neg) atomicAdd(x.cnt_dead, x.k_dead);
    keep[i] = 0;
    return;
  }
  if (!(xp >= 0.0 && yp >= 0.0 && zp >= 0.0 && xp < (d.n1 + 1) * c.h0 && yp < (d.n2 + 1) * c.h1 &&
        zp < (d.n3 + 1) * c.h2)) {
    raise_err(err, LEPIC_ERR_CELL, (int)i);
    keep[i] = 0;
    return;
  }
  int ix, iy, iz;
  push_one<BMAP>(d, c, m, Ei, xp, yp, zp, vx, vy, vz, ix, iy, iz);
  // negative ions leave through the Neumann plane (no specular reflection),
  // counted at label 0 (Src/part_expmover.f90:278-280, 300)
  const bool neu_loss = x.neg && xp < 0.0 && c.flag_nmn == 1;
  if (neu_loss || cw[d.c(ix, iy, iz)]) {
    double Eki = 0.5 * c.Nm * c.mass * (vx * vx + vy * vy + vz * vz);
    int igrid = neu_loss ? 0 : bcnd[d.g(ix, iy, iz)];
    atomicAdd(&acc[0], Eki);
    if (igrid >= 0 && igrid <= c.ngrid) {
      dielectric_charge(die, d, igrid, xp, yp, zp, ix, iy, iz, c.h0, c.h1, c.h2, c.flag_pbc, c.zmax);
      if (x.sec && igrid == x.igrid_sec) emit_secondaries(x, i, xp, yp, vz, err);
      atomicAdd(&acc[2 + 2 * igrid], 1.0);
      atomicAdd(&acc[3 + 2 * igrid], Eki);
      if (x.neg && igrid == x.num_grd) {
        const int f = x.cex[i];
        atomicAdd(&x.cnt_cex[0], 1);
        if (abs(f) == x.tag_neu) atomicAdd(&x.cnt_cex[1], 1);
        if (f == -x.tag_neu) atomicAdd(&x.cnt_cex[2], 1);
        double theta = atan(vy / vx);
        atomicAdd(&x.beam_div[0], theta);
        atomicAdd(&x.beam_div[1], theta * theta);
        theta = atan(vz / vx);
        atomicAdd(&x.beam_div[2], theta);
        atomicAdd(&x.beam_div[3], theta * theta);
      }
    }
    keep[i] = 0;
    return;
  }
  if (c.flag_nmn == 1 && xp <= 0.0) {
    xp = -xp;
    vx = -vx;
  }
  if (c.flag_pbc == 1) {
    if (yp >= c.ymax) yp = yp - c.ymax;
    if (yp <= 0.0) yp = c.ymax + yp;
    if (zp >= c.zmax) zp = zp - c.zmax;
    if (zp <= 0.0) zp = c.zmax + zp;
  }
  pout[i] = xp;
  pout[cap + i] = yp;
  pout[2 * cap + i] = zp;
  pout[3 * cap + i] = vx;
  pout[4 * cap + i] = vy;
  pout[5 * cap + i] = vz;
  keep[i] = 1;
}

// scatter kept particles to their compacted (in-order) slot, with their
// flag_cex when given (the negative-ion species)
__global__ void k_compact(const double *__restrict__ pin, double *__restrict__ pout, long long cap,
                          const int *__restrict__ count, const int *__restrict__ keep,
                          const int *__restrict__ pos, const int *__restrict__ cex_in, int *__restrict__ cex_out) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= *count) return;
  if (!keep[i]) return;
  long long j = pos[i];
#pragma unroll
  for (int c = 0; c < 6; ++c) pout[c * cap + j] = pin[c * cap + i];
  if (cex_in) cex_out[j] = cex_in[i];
}

__global__ void k_set_count(int *count, const int *keep, const int *pos) {
  int N = *count;
  if (N > 0) *count = pos[N - 1] + keep[N - 1];
}

// CIC deposition: np += kq * k1 * w (Src/part_expmover.f90:591-656)
__global__ void __launch_bounds__(PB) k_deposit_f64(Dims d, double h0, double h1, double h2, double k1,
                                                    const double *__restrict__ p, long long cap,
                                                    const int *__restrict__ count,
                                                    const double *__restrict__ kq, double *np,
                                                    int *err) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= *count) return;
  double xp = p[i], yp = p[cap + i], zp = p[2 * cap + i];
  if (!(xp >= 0.0 && yp >= 0.0 && zp >= 0.0 && xp < (d.n1 + 1) * h0 && yp < (d.n2 + 1) * h1 &&
        zp < (d.n3 + 1) * h2)) {
    raise_err(err, LEPIC_ERR_CELL, (int)i);
    return;
  }
  int ix = (int)(xp / h0) + 1, iy = (int)(yp / h1) + 1, iz = (int)(zp / h2) + 1;
  double px = (ix * h0 - xp) / h0;
  double py = (iy * h1 - yp) / h1;
  double pz = (iz * h2 - zp) / h2;
  const long long sy = d.N1, sz = d.N1 * d.N2;
  long long q = d.g(ix, iy, iz);
  atomicAdd(&np[q], kq[q] * (k1 * px * py * pz));
  atomicAdd(&np[q + 1], kq[q + 1] * (k1 * (1.0 - px) * py * pz));
  atomicAdd(&np[q + 1 + sy], kq[q + 1 + sy] * (k1 * (1.0 - px) * (1.0 - py) * pz));
  atomicAdd(&np[q + sy], kq[q + sy] * (k1 * px * (1.0 - py) * pz));
  atomicAdd(&np[q + sz], kq[q + sz] * (k1 * px * py * (1.0 - pz)));
  atomicAdd(&np[q + 1 + sz], kq[q + 1 + sz] * (k1 * (1.0 - px) * py * (1.0 - pz)));
  atomicAdd(&np[q + 1 + sy + sz], kq[q + 1 + sy + sz] * (k1 * (1.0 - px) * (1.0 - py) * (1.0 - pz)));
  atomicAdd(&np[q + sy + sz], kq[q + sy + sz] * (k1 * px * (1.0 - py) * (1.0 - pz)));
}

__device__ __forceinline__ unsigned lane_le() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_le;" : "=r"(m));
  return m;
}

// Runs of equal keys in consecutive lanes (particles are nearly sorted, so a
// warp usually holds one or two cells): head lane, run start and length.
struct Run {
  bool head;
  int start, len;
};
__device__ __forceinline__ Run lane_run(int key) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  int prev = __shfl_up_sync(full, key, 1);
  Run r;
  r.head = (lane == 0) || (prev != key);
  unsigned heads = __ballot_sync(full, r.head);
  r.start = 31 - __clz(heads & lane_le());
  // next head above the run start (none: the run ends at lane 31)
  unsigned above = (r.start == 31) ? 0u : (heads & ~((2u << r.start) - 1u));
  r.len = (above ? __ffs(above) - 1 : 32) - r.start;
  return r;
}

// cell key ic = (ix-1) + n1((iy-1) + n2(iz-1)) + 1 and its histogram, one
// atomic per run of equal keys in a warp
__global__ void k_sort_keys(Dims d, double h0, double h1, double h2, const double *__restrict__ p,
                            long long cap, const int *__restrict__ count, int *key, int *cnt,
                            int pl_max, int *err) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int N = *count;
  int ic = -1;
  if (i < N) {
    int ix = (int)(p[i] / h0) + 1, iy = (int)(p[cap + i] / h1) + 1, iz = (int)(p[2 * cap + i] / h2) + 1;
    ic = (ix - 1) + d.n1 * ((iy - 1) + d.n2 * (iz - 1)) + 1;
    if (ic < 1 || ic > pl_max) {
      raise_err(err, LEPIC_ERR_CELL, (int)i);
      ic = pl_max;
    }
    key[i] = ic;
  }
  Run r = lane_run(ic);
  if (r.head && ic >= 0) atomicAdd(&cnt[ic], r.len);
}

// scatter to cursor[key]: the run head reserves len slots, lanes take them in
// lane order
__global__ void k_sort_scatter(const double *__restrict__ p, double *__restrict__ q, long long cap,
                               const int *__restrict__ count, const int *__restrict__ key, int *cursor) {
  const unsigned full = 0xffffffffu;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const int N = *count;
  const int k = (i < N) ? key[i] : -1;
  Run r = lane_run(k);
  int base = 0;
  if (r.head && k >= 0) base = atomicAdd(&cursor[k], r.len);
  base = __shfl_sync(full, base, r.start);
  if (i < N) {
    const long long j = base + ((threadIdx.x & 31) - r.start);
#pragma unroll
    for (int c = 0; c < 6; ++c) q[c * cap + j] = p[c * cap + i];
  }
}

// ---------------------------------------------------------------- scan
constexpr int SB = 1024;  // elements per scan block (512 threads x 2)

__global__ void k_scan_block(const int *in, int *out, long long n, int *bsum) {
  __shared__ int s[SB];
  long long base = (long long)blockIdx.x * SB;
  int t = threadIdx.x;
  s[2 * t] = (base + 2 * t < n) ? in[base + 2 * t] : 0;
  s[2 * t + 1] = (base + 2 * t + 1 < n) ? in[base + 2 * t + 1] : 0;
  // inclusive Hillis-Steele over SB elements with 512 threads
  for (int off = 1; off < SB; off <<= 1) {
    __syncthreads();
    int a0 = (2 * t >= off) ? s[2 * t - off] : 0;
    int a1 = (2 * t + 1 >= off) ? s[2 * t + 1 - off] : 0;
    __syncthreads();
    s[2 * t] += a0;
    s[2 * t + 1] += a1;
  }
  __syncthreads();
  // exclusive output
  if (base + 2 * t < n) out[base + 2 * t] = s[2 * t] - ((base + 2 * t < n) ? in[base + 2 * t] : 0);
  if (base + 2 * t + 1 < n) out[base + 2 * t + 1] = s[2 * t + 1] - in[base + 2 * t + 1];
  if (t == 0 && bsum) bsum[blockIdx.x] = s[SB - 1];
}

__global__ void k_scan_add(int *out, long long n, const int *boff) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] += boff[i / SB];
}

}  // namespace

// Exclusive prefix sum of n ints (three-phase block scan, recursive on the
// block totals).  in and out may alias.
int exclusive_scan_i32(const int *in, int *out, long long n, cudaStream_t s) {
  if (n <= 0) return LEPIC_OK;
  long long nb = (n + SB - 1) / SB;
  if (nb == 1) {
    k_scan_block<<<1, SB / 2, 0, s>>>(in, out, n, nullptr);
    LEPIC_CUDA(cudaGetLastError());
    return LEPIC_OK;
  }
  static thread_local int depth = 0;
  char nm[32];
  snprintf(nm, sizeof nm, "scan_bsum%d", depth);
  int *bsum = (int *)scratch(nm, sizeof(int) * (size_t)nb);
  snprintf(nm, sizeof nm, "scan_boff%d", depth);
  int *boff = (int *)scratch(nm, sizeof(int) * (size_t)nb);
  if (!bsum || !boff) return LEPIC_ERR_CUDA;
  k_scan_block<<<(unsigned)nb, SB / 2, 0, s>>>(in, out, n, bsum);
  LEPIC_CUDA(cudaGetLastError());
  depth++;
  int rc = exclusive_scan_i32(bsum, boff, nb, s);
  depth--;
  if (rc) return rc;
  k_scan_add<<<grid_for(n, 256), 256, 0, s>>>(out, n, boff);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int launch_part_mover(const lepic_grid_t &g, const double *Ei, lepic_species_f64_t &sp, int ptype,
                      int ntype, int ngrid, const lepic_phys_t &P, double *p_mac, double *P_loss,
                      cudaStream_t s, const int *dtype_dev, double *qxz_dev, double *qyz_dev,
                      const MoverExtras *ex) {
  Dims d(g.n);
  const int p = ptype - 1;
  PushConst c;
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  c.dt = P.dt;
  c.k1 = P.dt * P.charge[p] / (2.0 * P.mass[p]);
  c.Nm = P.Nm[p];
  c.mass = P.mass[p];
  c.Bx = P.Bconst[0];
  c.By = P.Bconst[1];
  c.Bz = P.Bconst[2];
  c.boris = (P.flag_B == 1) ? 1 : 0;
  if (P.flag_B_pos == 1 && P.charge[p] > 0.0) c.boris = 0;
  c.flag_nmn = P.flag_nmn;
  c.flag_pbc = P.flag_pbc;
  c.ymax = P.ymax;
  c.zmax = P.zmax;
  c.ngrid = ngrid;
  BMapF64 m;
  if (int rc = bmap_from_phys(P, g.n, m)) return rc;
  Dielectric die = dielectric_from_phys(P, g.n, ptype);
  if (dtype_dev) {
    if (!qxz_dev || !qyz_dev) return LEPIC_ERR_ARG;
    die.dtype = dtype_dev;
    die.qxz = qxz_dev;
    die.qyz = qyz_dev;
    die.k3 = P.Nm[p] * P.charge[p];
  }
  MoverExtra x;
  memset(&x, 0, sizeof(x));
  x.pi = P.pi;
  int *cex_out = nullptr;
  if (ex && ex->tag_neg == ptype) {
    if (!ex->cex || !ex->cex_out || !ex->cnt_cex || !ex->cnt_dead || !ex->beam_div) return LEPIC_ERR_ARG;
    x.neg = 1;
    x.tag_neu = ex->tag_neu;
    x.num_grd = ex->num_grd;
    x.cex = ex->cex;
    x.cnt_cex = ex->cnt_cex;
    x.cnt_dead = ex->cnt_dead;
    x.beam_div = ex->beam_div;
    x.k_dead = P.Nm[p] * P.charge[p];
    cex_out = ex->cex_out;
  }
  if (ex && ex->gam_sec > 0.0 && P.charge[p] > 0.0) {
    if (!ex->e1 || !ex->ploss4) return LEPIC_ERR_ARG;
    x.sec = 1;
    x.igrid_sec = ex->igrid_sec;
    x.gam = ex->gam_sec;
    x.vt = sqrt(2.0 * P.qe * fabs(ex->THm) / fabs(P.mass[0]));
    x.zg0 = ex->zg_sec[0];
    x.zg1 = ex->zg_sec[1];
    x.Nm1 = P.Nm[0];
    x.m1 = P.mass[0];
    x.p1 = ex->e1->p;
    x.cap1 = ex->e1->cap;
    x.count1 = ex->e1->count;
    x.ploss4 = ex->ploss4;
    x.k0 = ex->key0;
    x.k1 = ex->key1;
    x.call = ex->call;
  }
  const long long cap = sp.cap;
  int nacc = 2 + 2 * (ngrid + 1);
  double *acc = (double *)scratch("push_acc", sizeof(double) * nacc);
  int *keep = (int *)scratch("push_keep", sizeof(int) * (size_t)(cap > 0 ? cap : 1));
  int *pos = (int *)scratch("push_pos", sizeof(int) * (size_t)(cap > 0 ? cap : 1));
  if (!acc || !keep || !pos) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(acc, 0, sizeof(double) * nacc, s));
  int N = 0;
  LEPIC_CUDA(cudaMemcpyAsync(&N, sp.count, sizeof(int), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (N > 0) {
    int t0 = timer_start("push_f64", s);
    if (m.B)
      k_push_f64<true><<<grid_for(N, PB), PB, 0, s>>>(d, c, m, die, x, Ei, g.bcnd, g.cell_wall, sp.p, sp.p_alt,
                                                      cap, sp.count, sp.flag_dead, keep, acc, ctx().d_err);
    else
      k_push_f64<false><<<grid_for(N, PB), PB, 0, s>>>(d, c, m, die, x, Ei, g.bcnd, g.cell_wall, sp.p, sp.p_alt,
                                                       cap, sp.count, sp.flag_dead, keep, acc, ctx().d_err);
    timer_stop(t0, s);
    LEPIC_CUDA(cudaGetLastError());
    int t1 = timer_start("compact_scan", s);
    int rc = exclusive_scan_i32(keep, pos, N, s);
    timer_stop(t1, s);
    if (rc) return rc;
    int t2 = timer_start("compact_f64", s);
    k_compact<<<grid_for(N, PB), PB, 0, s>>>(sp.p_alt, sp.p, cap, sp.count, keep, pos, x.neg ? x.cex : nullptr,
                                             cex_out);
    timer_stop(t2, s);
    k_set_count<<<1, 1, 0, s>>>(sp.count, keep, pos);
    LEPIC_CUDA(cudaGetLastError());
  }
  std::vector<double> h(nacc);
  LEPIC_CUDA(cudaMemcpyAsync(h.data(), acc, sizeof(double) * nacc, cudaMemcpyDeviceToHost, s));
  int rc = check_err(s);
  if (P_loss) {
    P_loss[0 + 4 * p] += h[0];
    P_loss[2 + 4 * p] += h[1];
  }
  if (p_mac) {
    for (int ig = 0; ig <= ngrid; ++ig) {
      p_mac[p + (long long)ntype * (0 + 2LL * ig)] += h[2 + 2 * ig];
      p_mac[p + (long long)ntype * (1 + 2LL * ig)] += h[3 + 2 * ig];
    }
  }
  return rc;
}

int launch_deposit(const lepic_grid_t &g, const lepic_species_f64_t &sp, int ptype,
                   const lepic_phys_t &P, double *np, cudaStream_t s) {
  Dims d(g.n);
  const int p = ptype - 1;
  const double k1 = P.Nm[p] / (g.h[0] * g.h[1] * g.h[2]);
  // grid sized for the capacity; threads beyond the device count exit
  int t0 = timer_start("deposit_f64", s);
  k_deposit_f64<<<grid_for(sp.cap, PB), PB, 0, s>>>(d, g.h[0], g.h[1], g.h[2], k1, sp.p, sp.cap,
                                                     sp.count, g.kq, np, ctx().d_err);
  timer_stop(t0, s);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int launch_sort(const lepic_grid_t &g, lepic_species_f64_t &sp, int *Plist, int pl_max,
                cudaStream_t s) {
  Dims d(g.n);
  int N = 0;
  LEPIC_CUDA(cudaMemcpyAsync(&N, sp.count, sizeof(int), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  int *cnt = (int *)scratch("sort_cnt", sizeof(int) * (size_t)(pl_max + 1));
  if (!cnt) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(int) * (size_t)(pl_max + 1), s));
  if (N > 0) {
    int t0 = timer_start("sort_keys", s);
    k_sort_keys<<<grid_for(N, PB), PB, 0, s>>>(d, g.h[0], g.h[1], g.h[2], sp.p, sp.cap, sp.count,
                                               sp.key, cnt, pl_max, ctx().d_err);
    timer_stop(t0, s);
    LEPIC_CUDA(cudaGetLastError());
  }
  int t1 = timer_start("sort_scan", s);
  int rc = exclusive_scan_i32(cnt, Plist, pl_max + 1, s);
  timer_stop(t1, s);
  if (rc) return rc;
  if (N > 0) {
    int t2 = timer_start("sort_scatter", s);
    k_sort_scatter<<<grid_for(N, PB), PB, 0, s>>>(sp.p, sp.p_alt, sp.cap, sp.count, sp.key, Plist);
    timer_stop(t2, s);
    LEPIC_CUDA(cudaGetLastError());
    double *t = sp.p;
    sp.p = sp.p_alt;
    sp.p_alt = t;
  }
  // Plist now holds inclusive end offsets (cursor after the scatter);
  // Plist(0) = 0 like the reference.
  LEPIC_CUDA(cudaMemsetAsync(Plist, 0, sizeof(int), s));
  return check_err(s);
}

}  // namespace lepic

namespace lepic {

namespace {

// Uniform loading with Maxwellian velocities (the GPU counterpart of
// Src/load_part.f90:91-194): sample j draws its position from a Philox
// stream keyed by j alone, so all species of sample j sit at the same
// position like the reference's co-located pairs; positions in all-wall cells
// are redrawn (bounded retries).  Velocities use the load_gauss form
// vp = vt sqrt(-ln u1), theta = 2 pi u2.
struct LoadConst {
  double xl, ym, zm, h0, h1, h2;
  double vt[LEPIC_NPART];
  int ntype;
  unsigned k0, k1;
};

struct SpPtrsL {
  double *p[LEPIC_NPART];
  long long cap[LEPIC_NPART];
};

__global__ void k_load_uniform(Dims d, LoadConst c, SpPtrsL S, long long n,
                               const unsigned char *__restrict__ cw, int *err) {
  long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j >= n) return;
  double x = 0, y = 0, z = 0;
  bool ok = false;
  for (uint32_t tr = 0; tr < 64 && !ok; ++tr) {
    U4 r = philox4x32_10({(uint32_t)j, (uint32_t)(j >> 32), tr, 0xA5A5u}, c.k0, c.k1);
    x = u01(r.x) * c.xl;
    y = u01(r.y) * c.ym;
    z = u01(r.z) * c.zm;
    int ix = (int)(x / c.h0) + 1, iy = (int)(y / c.h1) + 1, iz = (int)(z / c.h2) + 1;
    ok = !cw[d.c(ix, iy, iz)];
  }
  if (!ok) raise_err(err, LEPIC_ERR_CELL, (int)j);
  for (int p = 0; p < c.ntype; ++p) {
    U4 r = philox4x32_10({(uint32_t)j, (uint32_t)(j >> 32), 1000u + p, 0x5A5Au}, c.k0, c.k1);
    const double vt = c.vt[p];
    double s1, c1, s2, c2;
    sincos(2.0 * 3.141592653589793 * u01(r.y), &s1, &c1);
    sincos(2.0 * 3.141592653589793 * u01(r.w), &s2, &c2);
    double vp = vt * sqrt(-log(u01(r.x)));
    double vq = vt * sqrt(-log(u01(r.z)));
    double *q = S.p[p];
    const long long cap = S.cap[p];
    q[j] = x;
    q[cap + j] = y;
    q[2 * cap + j] = z;
    q[3 * cap + j] = vp * c1;
    q[4 * cap + j] = vp * s1;
    q[5 * cap + j] = vq * c2;
  }
}

}  // namespace

int launch_load_uniform(const lepic_grid_t &g, lepic_species_f64_t *sp, int ntype, long long n,
                        const lepic_phys_t &P, unsigned long long seed, cudaStream_t s) {
  Dims d(g.n);
  LoadConst c;
  memset(&c, 0, sizeof(c));
  c.xl = P.x_load;
  c.ym = P.ymax;
  c.zm = P.zmax;
  c.h0 = g.h[0];
  c.h1 = g.h[1];
  c.h2 = g.h[2];
  for (int p = 0; p < LEPIC_NPART; ++p) c.vt[p] = P.vt0[p];
  c.ntype = ntype;
  c.k0 = (unsigned)(seed & 0xffffffffu);
  c.k1 = (unsigned)(seed >> 32);
  SpPtrsL S;
  memset(&S, 0, sizeof(S));
  for (int p = 0; p < ntype; ++p) {
    if (n > sp[p].cap) return LEPIC_ERR_CAPACITY;
    S.p[p] = sp[p].p;
    S.cap[p] = sp[p].cap;
  }
  if (n > 0) k_load_uniform<<<grid_for(n, PB), PB, 0, s>>>(d, c, S, n, g.cell_wall, ctx().d_err);
  LEPIC_CUDA(cudaGetLastError());
  int nn = (int)n;
  for (int p = 0; p < ntype; ++p)
    LEPIC_CUDA(cudaMemcpyAsync(sp[p].count, &nn, sizeof(int), cudaMemcpyHostToDevice, s));
  return check_err(s);
}

}  // namespace lepic
