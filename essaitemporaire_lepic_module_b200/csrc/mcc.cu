// Null-collision Monte Carlo (Src/collisions.f90) against neutral targets
// (MC: a Maxwellian partner) and charged targets (DSMC: a particle of the
// target species in the incident's cell).
//
// The reference draws Nc = N * nu_max * ns_coll * dt incident particles with
// replacement from a serial ran2 stream and tests each against
// sum_r nu_r / nu_max.  Here every particle draws its own Bernoulli trial
// with probability Pmax = nu_max * ns_coll * dt from a Philox4x32-10 counter
// keyed by (seed, call, species, particle, sub-stream): the expected number
// of collisions of each process, nu_r * ns_coll * dt per particle, is the
// same, and no two threads ever touch the same particle.
//
// Two passes: the select pass appends the candidates (a fraction Pmax of
// the particle indices; no particle data is read) to a list -- for small
// Pmax by geometric skipping (k_mcc_select_skip: one draw per candidate),
// else one Philox test per particle (k_mcc_select) -- and k_mcc_collide then
// runs the collision physics densely on the candidates only.  The physics follows Src/collisions.f90:437-998 step
// for step: Maxwellian neutral target (load_gauss form), relative energy in
// the centre-of-mass frame, linear interpolation of sigma on the merged
// energy grid, elastic / excitation scattering, ionization with
// equal-momentum byproducts on equally spaced angles rotated by `scatter`,
// and charge exchange by velocity swap.  Ionization products are appended at
// the end of their species' arrays.  The kernels are templated on the
// particle layout (FP64 SoA or mixed cell + FP32 offsets).
//
// Charged targets (Src/collisions.f90:335-423, 524-531): the partner is a
// uniformly chosen particle of the target species in the incident's cell, or
// in the first non-empty of the cells ici+1, ici-1, ici+n1, ici-n1,
// ici+n1 n2, ici-n1 n2 (the reference's linear cell index), found through
// the per-cell offsets of that species' last sort; the target density is the
// mean of the species' density grid over the cell's 8 nodes.  The collision
// may change the target's velocity (elastic, excitation, charge exchange) or
// remove it (other reactions).  The reference runs the collisions one after
// another, so a target drawn by two incident particles takes part in both,
// the second seeing the velocity the first left.  Here the incident
// particles collide concurrently in rounds: a collision claims its target
// with the round's tag (one word per particle, cleared per call); one that
// finds its target claimed in the same round changes nothing, goes to the
// next round's list and is evaluated again from its own draws (same target,
// same uniform) once the first collision is done -- the order of a serial
// loop in which the winner came first.  Every drawn collision happens; the
// rounds end when no collision is left over (lost_claims counts those still
// left at the round cap, and stays zero while a target is hit by fewer
// collisions than there are rounds).
#include <vector>

#include "lepic_internal.cuh"

namespace lepic {

namespace {

constexpr int MB = 256;
constexpr int MAXR = 48;  // reactions per incident species (hydrogen.dat's electrons: 40)
constexpr int MAXBY = 4;  // byproducts per reaction
// DSMC rounds per species and call (a target hit by more collisions than
// this in one call leaves the excess undone, counted as lost_claims), and
// rounds launched between two reads of the count left
constexpr int DSMC_ROUNDS = 256;
constexpr int DSMC_BATCH = 8;

// one reaction of the incident species; the table lives in device memory
// (runtime-indexed arrays in the kernel's parameters would be copied to
// every thread's local memory)
struct Reac {
  int ind;                      // 1-based reaction index
  int tt;                       // target species (1-based)
  int rt, n_by, n_re;
  int dsmc;                     // 1: charged target (DSMC)
  int by[MAXBY];
  double Eth, np_t;
};

struct MCCConst {
  int ptype, nr;
  double Pmax, nu_max, qe, pi;
  double m_p;                   // |mass| of incident
  const Reac *R;                // device Reac[nr]
  int any_dsmc;
  double mass[LEPIC_NPART];     // signed masses
  double vt0[LEPIC_NPART];
  int npt, npt_mx;
  unsigned int k0, k1, c2, c3;  // Philox key and counter words
  // region counters of Src/collisions.f90:1005-1013 (drop-in path only)
  int n_rg, ncol_mx;
  int ixl[LEPIC_NM_RG], ixr[LEPIC_NM_RG], iyl, iyr, izl, izr;
  double w_rg[LEPIC_NM_RG];     // 1 / np_tot_rg(ptype, i_rg)
  double h0, h1, h2;
  // event log of the differentiable window (nullptr: not recorded)
  lepic_win_event_t *log;
  int *nlog;
  int log_cap, step;
  // energy and source bookkeeping of the drop-in path (RegionCount)
  double *ploss3;
  int *sxy, *sxz;
  int iz_pl, iy_pl, n1, n2, n3;
  double Nm[LEPIC_NPART];
};

// FP64 SoA layout
struct AccF64 {
  double *p[LEPIC_NPART];
  int *count[LEPIC_NPART];
  long long cap[LEPIC_NPART];
  __device__ void load_v(int P, long long i, double &vx, double &vy, double &vz) const {
    const double *q = p[P];
    vx = q[3 * cap[P] + i];
    vy = q[4 * cap[P] + i];
    vz = q[5 * cap[P] + i];
  }
  __device__ void store_v(int P, long long i, double vx, double vy, double vz) const {
    double *q = p[P];
    q[3 * cap[P] + i] = vx;
    q[4 * cap[P] + i] = vy;
    q[5 * cap[P] + i] = vz;
  }
  // new particle j of species B at the position of (P, i)
  __device__ void append(int P, long long i, int B, long long j, double vx, double vy, double vz) const {
    const double *s = p[P];
    double *d = p[B];
    const long long cs = cap[P], cb = cap[B];
    d[j] = s[i];
    d[cb + j] = s[cs + i];
    d[2 * cb + j] = s[2 * cs + i];
    d[3 * cb + j] = vx;
    d[4 * cb + j] = vy;
    d[5 * cb + j] = vz;
  }
  __device__ void cell_of(const MCCConst &c, int P, long long i, int &ix, int &iy, int &iz) const {
    const double *q = p[P];
    ix = (int)(q[i] / c.h0) + 1;
    iy = (int)(q[cap[P] + i] / c.h1) + 1;
    iz = (int)(q[2 * cap[P] + i] / c.h2) + 1;
  }
  __device__ bool live(int, long long) const { return true; }
};

// mixed layout: cell + FP32 offsets and velocities
struct AccMixed {
  int *cell[LEPIC_NPART];
  float *p[LEPIC_NPART];
  int *count[LEPIC_NPART];
  long long cap[LEPIC_NPART];
  __device__ void load_v(int P, long long i, double &vx, double &vy, double &vz) const {
    const float *q = p[P];
    vx = q[3 * cap[P] + i];
    vy = q[4 * cap[P] + i];
    vz = q[5 * cap[P] + i];
  }
  __device__ void store_v(int P, long long i, double vx, double vy, double vz) const {
    float *q = p[P];
    q[3 * cap[P] + i] = (float)vx;
    q[4 * cap[P] + i] = (float)vy;
    q[5 * cap[P] + i] = (float)vz;
  }
  __device__ void append(int P, long long i, int B, long long j, double vx, double vy, double vz) const {
    const float *s = p[P];
    float *d = p[B];
    const long long cs = cap[P], cb = cap[B];
    cell[B][j] = cell[P][i];
    d[j] = s[i];
    d[cb + j] = s[cs + i];
    d[2 * cb + j] = s[2 * cs + i];
    d[3 * cb + j] = (float)vx;
    d[4 * cb + j] = (float)vy;
    d[5 * cb + j] = (float)vz;
  }
  __device__ void cell_of(const MCCConst &c, int P, long long i, int &ix, int &iy, int &iz) const {
    const int cc = cell[P][i];
    ix = (cc & (LEPIC_CELL_MAX - 1)) + 1;
    iy = ((cc >> LEPIC_CELL_BITS) & (LEPIC_CELL_MAX - 1)) + 1;
    iz = (cc >> (2 * LEPIC_CELL_BITS)) + 1;
  }
  __device__ bool live(int, long long) const { return true; }
};

// the differentiable window's particles (lepic_win_species_t): the mixed
// layout in FP32 or FP64 planes, slots kept, the window history in bl; a
// particle takes part in the collisions of `step` when it is not lost and
// was not created by them
constexpr int WIN_ALIVE = 0x7fff;
template <class T>
struct AccWin {
  int *cell[LEPIC_NPART];
  T *p[LEPIC_NPART];
  int *bl[LEPIC_NPART];
  int *count[LEPIC_NPART];
  long long cap[LEPIC_NPART];
  int step;
  __device__ void load_v(int P, long long i, double &vx, double &vy, double &vz) const {
    const T *q = p[P];
    vx = q[3 * cap[P] + i];
    vy = q[4 * cap[P] + i];
    vz = q[5 * cap[P] + i];
  }
  __device__ void store_v(int P, long long i, double vx, double vy, double vz) const {
    T *q = p[P];
    q[3 * cap[P] + i] = (T)vx;
    q[4 * cap[P] + i] = (T)vy;
    q[5 * cap[P] + i] = (T)vz;
  }
  __device__ void append(int P, long long i, int B, long long j, double vx, double vy, double vz) const {
    const T *s = p[P];
    T *d = p[B];
    const long long cs = cap[P], cb = cap[B];
    cell[B][j] = cell[P][i];
    d[j] = s[i];
    d[cb + j] = s[cs + i];
    d[2 * cb + j] = s[2 * cs + i];
    d[3 * cb + j] = (T)vx;
    d[4 * cb + j] = (T)vy;
    d[5 * cb + j] = (T)vz;
    bl[B][j] = (step & 0xffff) | (WIN_ALIVE << 16);
  }
  __device__ void cell_of(const MCCConst &c, int P, long long i, int &ix, int &iy, int &iz) const {
    const int cc = cell[P][i];
    ix = (cc & (LEPIC_CELL_MAX - 1)) + 1;
    iy = ((cc >> LEPIC_CELL_BITS) & (LEPIC_CELL_MAX - 1)) + 1;
    iz = (cc >> (2 * LEPIC_CELL_BITS)) + 1;
  }
  __device__ bool live(int P, long long i) const {
    const int b = bl[P][i];
    return (b >> 16) == WIN_ALIVE && (short)(b & 0xffff) < step;
  }
};

// DSMC state: per species density grids, per-cell offsets of the last sort
// (FP64 sort: Plist, inclusive ends at the reference's linear cell index;
// mixed sort: exclusive starts at the 8x8x8-tile key), flag_dead and claims
struct Targets {
  const double *np[LEPIC_NPART];
  const int *off[LEPIC_NPART];
  signed char *fd[LEPIC_NPART];
  int *claim[LEPIC_NPART];
  int tile, n1, n2, n3, ntx, nty;
  long long pl_max;
  // [0] incident particles with no target, [1] collisions left at the round
  // cap, [2] collisions deferred to a later round (target taken first)
  unsigned long long *stat;
};

// a particle of species T in cell ici (1-based linear index) or its six
// neighbours in the reference's order; -1 when none
__device__ __forceinline__ long long pick_target(const Targets &D, int T, long long ici, uint32_t rnd) {
  const int *off = D.off[T];
  if (!off) return -1;
  const long long n12 = (long long)D.n1 * D.n2, ncell = n12 * D.n3;
  const long long cand[7] = {ici, ici + 1, ici - 1, ici + D.n1, ici - D.n1, ici + n12, ici - n12};
  for (int k = 0; k < 7; ++k) {
    const long long ic = cand[k];
    if (ic < 1 || ic > D.pl_max) continue;
    long long lo, hi;
    if (!D.tile) {
      lo = off[ic - 1];
      hi = off[ic];
    } else {
      if (ic > ncell) continue;
      const long long l = ic - 1;
      const int cx = (int)(l % D.n1), cy = (int)((l / D.n1) % D.n2), cz = (int)(l / n12);
      const long long tile = (cx >> 3) + (long long)D.ntx * ((cy >> 3) + (long long)D.nty * (cz >> 3));
      const long long key = tile * 512 + (cx & 7) + 8 * ((cy & 7) + 8 * (cz & 7));
      lo = off[key];
      hi = off[key + 1];
    }
    if (hi > lo) {
      long long idx = lo + (long long)((double)(hi - lo) * u01(rnd));
      return idx < hi ? idx : hi - 1;
    }
  }
  return -1;
}

// Src/collisions.f90:1022-1050
__device__ __forceinline__ void scatter(double &vx1, double &vy1, double &vz1, double vx, double vy,
                                        double vz, double costheta, double phi) {
  double sintheta = sqrt(fmax(1.0 - costheta * costheta, 0.0));
  double sinphi, cosphi;
  sincos(phi, &sinphi, &cosphi);
  double v = sqrt(vx * vx + vy * vy + vz * vz);
  if (v == 0.0) return;
  if (fabs(vy) > fabs(vz)) {
    double vv = sqrt(vx * vx + vy * vy);
    vx1 = vx * costheta + (vy * v * sinphi + vx * vz * cosphi) / vv * sintheta;
    vy1 = vy * costheta + (-vx * v * sinphi + vy * vz * cosphi) / vv * sintheta;
    vz1 = vz * costheta - vv * cosphi * sintheta;
  } else {
    double vv = sqrt(vx * vx + vz * vz);
    vx1 = vx * costheta + (vz * v * sinphi - vy * vx * cosphi) / vv * sintheta;
    vy1 = vy * costheta + vv * cosphi * sintheta;
    vz1 = vz * costheta - (vx * v * sinphi + vy * vz * cosphi) / vv * sintheta;
  }
}

// the interval j of the merged grid with Er[j-1] < E <= Er[j], or -1 when
// E <= Er[0] or E > Er[npt-1] (sigma 0), Src/collisions.f90:485-507
__device__ __forceinline__ int energy_segment(const double *__restrict__ Er, int npt, double E) {
  if (!(E > Er[0]) || E > Er[npt - 1]) return -1;
  int lo = 0, hi = npt - 1;  // Er[lo] < E <= Er[hi]
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (E > Er[mid]) lo = mid;
    else hi = mid;
  }
  return hi;
}

// linear interpolation of one table in interval j (Src/collisions.f90:510-521)
__device__ __forceinline__ double sigma_in(const double *__restrict__ Er, const double *__restrict__ sig, int j,
                                           double E) {
  const double EL = Er[j - 1], ER = Er[j], sL = sig[j - 1], sR = sig[j];
  return sL + (E - EL) * (sR - sL) / (ER - EL);
}

__device__ __forceinline__ unsigned lanemask_lt_m() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// pass 1: Bernoulli(Pmax) per particle, candidates appended to a list
__global__ void __launch_bounds__(MB) k_mcc_select(MCCConst c, const int *__restrict__ count,
                                                   int *__restrict__ cand, int *__restrict__ ncand) {
  const unsigned full = 0xffffffffu;
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  bool hit = false;
  if (i < *count) {
    U4 r0 = philox4x32_10({(uint32_t)i, 0u, c.c2, c.c3}, c.k0, c.k1);
    hit = u01(r0.x) < c.Pmax;
  }
  const unsigned m = __ballot_sync(full, hit);
  if (m) {
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(ncand, __popc(m));
    base = __shfl_sync(full, base, leader);
    if (hit) cand[base + __popc(m & lanemask_lt_m())] = (int)i;
  }
}

// pass 1 for small Pmax: the same Bernoulli(Pmax) sample of the particle
// indices drawn by geometric skipping.  Within each segment of `seg`
// particles the gaps between successive candidates are independent
// geometric variables, floor(ln U / ln(1 - Pmax)), so one uniform per
// candidate replaces one per particle.  The draws use Philox counters
// (segment, 16 + k) that the per-particle streams (particle, 0..2) of the
// collision pass never use.  The segment is sized for about four candidates
// per thread (a short serial chain, few threads when Pmax is tiny).
constexpr double SKIP_PMAX = 0.25;  // above it: one draw per particle
constexpr int SEL_BUF = 256;        // picks per warp between two reservations

int skip_segment(double Pmax) {
  int seg = 256;
  while (seg < 65536 && seg * Pmax < 4.0) seg *= 2;
  return seg;
}

__global__ void __launch_bounds__(MB) k_mcc_select_skip(MCCConst c, const int *__restrict__ count,
                                                        double inv_log1m, int seg_len, int *__restrict__ cand,
                                                        int *__restrict__ ncand) {
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const long long seg = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  const long long N = *count;
  const long long lo = seg * seg_len;
  const long long hi = lo + seg_len < N ? lo + seg_len : N;
  long long pos = lo - 1;
  bool live = lo < hi;
  uint32_t draw = 0;
  U4 r = {0u, 0u, 0u, 0u};
  int left = 0;
  // the warp's picks gather in shared memory and reserve their range of the
  // list with one atomic per SEL_BUF picks instead of one per round
  __shared__ int sbuf[MB / 32][SEL_BUF];
  int *wbuf = sbuf[threadIdx.x >> 5];
  int nb = 0;   // picks in the warp's buffer (the same in every lane)
  auto flush = [&]() {
    __syncwarp();
    int base = 0;
    if (lane == 0) base = atomicAdd(ncand, nb);
    base = __shfl_sync(full, base, 0);
    for (int k = lane; k < nb; k += 32) cand[base + k] = wbuf[k];
    __syncwarp();
    nb = 0;
  };
  while (__any_sync(full, live)) {
    long long pick = -1;
    if (live) {
      if (left == 0) {
        r = philox4x32_10({(uint32_t)seg, 16u + draw, c.c2, c.c3}, c.k0, c.k1);
        ++draw;
        left = 4;
      }
      const uint32_t v = r.x;
      r.x = r.y;
      r.y = r.z;
      r.z = r.w;
      --left;
      const double gap = floor(log(u01(v)) * inv_log1m);
      pos = gap < (double)seg_len ? pos + 1 + (long long)gap : hi;
      if (pos < hi) pick = pos;
      else live = false;
    }
    const unsigned m = __ballot_sync(full, pick >= 0);
    if (m) {
      if (nb + 32 > SEL_BUF) flush();
      if (pick >= 0) wbuf[nb + __popc(m & lanemask_lt_m())] = (int)pick;
      nb += __popc(m);
    }
  }
  if (nb) flush();
}

// pass 2: the collision physics on the candidates (grid-stride over warps so
// every lane of a warp reaches the warp-wide counter reductions)
// the partner of the incident particle for target species tt: velocity,
// reduced mass, relative speed and energy, centre-of-mass velocity
// (Src/collisions.f90:437-470); idx: the DSMC target's slot
struct TState {
  double tvx, tvy, tvz, mu, vr, vxc, vyc, vzc, Ekr;
  long long idx;
  bool ok;
};

// DSMC rounds: `tag` marks the claims of this round (claims of earlier
// rounds hold smaller tags); a collision whose target carries this round's
// tag appends its particle to `defer` (counter *ndefer) for the next round.
// first: the first round of the call (the only one that counts misses).
struct Round {
  int *defer;
  int *ndefer;
  int tag;
  int first;
};

// The scattering of a colliding candidate i of reaction sel
// (Src/collisions.f90:743-1020), from the state its selection recorded:
// the incident's velocity before, the partner, the tags of a charged target
// and the two draws of r0 that set the scattering angles.
template <class Acc, bool DSMC>
__device__ __forceinline__ void mcc_apply(const MCCConst &c, const Acc &S, const Targets &D, long long i, int sel, bool tgt,
                          double vx0, double vy0, double vz0, const TState &ts, uint32_t r0z, uint32_t r0w,
                          signed char *flag_dead, int *add, double *cnt_col, int *err) {
  const int P = c.ptype - 1;
  U4 ctr = {(uint32_t)i, 0u, c.c2, c.c3};
  const U4 r0 = {0u, 0u, r0z, r0w};
    const int rt = c.R[sel].rt;
    const int T = c.R[sel].tt - 1;
    const double mu_t = ts.mu, vr_t = ts.vr, vxc = ts.vxc, vyc = ts.vyc, vzc = ts.vzc;
    // the window's record of this collision
    lepic_win_event_t *ev = nullptr;
    if (c.log) {
      const int k = atomicAdd(c.nlog, 1);
      if (k < c.log_cap) {
        ev = c.log + k;
        ev->step = c.step;
        ev->P = P;
        ev->i = (int)i;
        ev->r = sel;
        ev->rt = rt;
        ev->nby = c.R[sel].n_by;
        ev->ind = c.R[sel].ind;
        ev->tv[0] = ts.tvx;
        ev->tv[1] = ts.tvy;
        ev->tv[2] = ts.tvz;
        ev->vold[0] = vx0;
        ev->vold[1] = vy0;
        ev->vold[2] = vz0;
        ev->m_t = fabs(c.mass[T]);
        ev->Eth = c.R[sel].Eth;
        for (int a = 0; a < MAXBY; ++a) {
          ev->by[a] = -1;
          ev->slot[a] = -1;
        }
      } else {
        raise_err(err, LEPIC_ERR_CAPACITY, -1);
      }
    }
    // P_loss(3, B) += the kinetic energy change of a particle of species
    // B set to (nx, ny, nz) from a speed squared of o2 (0: created)
    auto energy = [&](int B, double nx, double ny, double nz, double o2) {
      if (c.ploss3)
        atomicAdd(&c.ploss3[B], 0.5 * c.Nm[B] * c.mass[B] * (nx * nx + ny * ny + nz * nz - o2));
    };
    auto speed2 = [&](int B, long long k) {
      double ox, oy, oz;
      S.load_v(B, k, ox, oy, oz);
      return ox * ox + oy * oy + oz * oz;
    };
    if (rt == 4) {
      // charge exchange (Src/collisions.f90:948-998): the incident takes
      // the target's velocity, a charged target the incident's
      for (int a = 0; a < c.R[sel].n_by; ++a) {
        const int bt = c.R[sel].by[a];
        if (c.mass[bt - 1] <= 0) continue;
        if (ev && bt == c.ptype) ev->by[a] = bt - 1;
        if (bt == c.ptype) {
          if (c.ploss3) energy(P, ts.tvx, ts.tvy, ts.tvz, speed2(P, i));
          S.store_v(P, i, ts.tvx, ts.tvy, ts.tvz);
        } else if (tgt && bt - 1 == T) {
          if (c.ploss3) energy(T, vx0, vy0, vz0, speed2(T, ts.idx));
          S.store_v(T, ts.idx, vx0, vy0, vz0);
        }
      }
    } else {
      double Ee = 0.5 * mu_t * (vr_t * vr_t) - c.R[sel].Eth * c.qe;
      if (Ee < 0.0) {
        raise_err(err, LEPIC_ERR_NEG_ENERGY, (int)i);
        Ee = 0.0;
      }
      const int nby = c.R[sel].n_by;
      double sum_mass = 0.0;
      for (int a = 0; a < nby; ++a) sum_mass = sum_mass + 1.0 / fabs(c.mass[c.R[sel].by[a] - 1]);
      if (ev) ev->sum_mass = sum_mass;
      const double th_add = 2.0 * c.pi / (double)nby;
      const double cos_th = 1.0 - 2.0 * u01(r0.z);
      double th = acos(cos_th);
      const double phi = 2.0 * c.pi * u01(r0.w);
      double sin_ph, cos_ph;
      sincos(phi, &sin_ph, &cos_ph);
      ctr.y = 2u;
      const U4 r2 = philox4x32_10(ctr, c.k0, c.k1);
      const double cos_th_s = 1.0 - 2.0 * u01(r2.x);
      const double phi_s = 2.0 * c.pi * u01(r2.y);
      bool incident_reused = false;
      for (int a = 0; a < nby; ++a) {
        double sth, cth;
        sincos(th, &sth, &cth);
        th = th + th_add;
        const double ex = cth, ey = sth * sin_ph, ez = sth * cos_ph;
        double ex1 = 0, ey1 = 0, ez1 = 0;
        scatter(ex1, ey1, ez1, ex, ey, ez, cos_th_s, phi_s);
        const int bt = c.R[sel].by[a];
        if (c.mass[bt - 1] <= 0) continue;
        if (ev) {
          ev->by[a] = bt - 1;
          ev->e1[a][0] = (float)ex1;
          ev->e1[a][1] = (float)ey1;
          ev->e1[a][2] = (float)ez1;
        }
        const double mb = fabs(c.mass[bt - 1]);
        const double vp = sqrt(2.0 * (Ee / sum_mass) / (mb * mb));
        const double nvx = vxc + vp * ex1, nvy = vyc + vp * ey1, nvz = vzc + vp * ez1;
        const bool reuse = (a == 0 && bt == c.ptype) || ((rt == 1 || rt == 3) && bt == c.ptype);
        if (reuse) {
          if (c.ploss3) energy(P, nvx, nvy, nvz, speed2(P, i));
          S.store_v(P, i, nvx, nvy, nvz);
          incident_reused = true;
        } else if ((rt == 1 || rt == 3) && tgt && bt - 1 == T) {
          // elastic / excitation keep a charged target (Src/collisions.f90:843-851)
          if (c.ploss3) energy(T, nvx, nvy, nvz, speed2(T, ts.idx));
          S.store_v(T, ts.idx, nvx, nvy, nvz);
        } else {
          const int B = bt - 1;
          const int slot = atomicAdd(&add[B], 1);
          const long long j = (long long)*S.count[B] + slot;
          if (j >= S.cap[B]) {
            raise_err(err, LEPIC_ERR_CAPACITY, B);
          } else {
            S.append(P, i, B, j, nvx, nvy, nvz);
            if (ev) ev->slot[a] = (int)j;
            energy(B, nvx, nvy, nvz, 0.0);
            if (c.sxy) {
              // the new particle's source count on the two plot planes
              int sx, sy, sz;
              S.cell_of(c, P, i, sx, sy, sz);
              if (sz == c.iz_pl) atomicAdd(&c.sxy[sx + (c.n1 + 3) * (sy + (long long)(c.n2 + 3) * B)], 1);
              if (sy == c.iy_pl) atomicAdd(&c.sxz[sx + (c.n1 + 3) * (sz + (long long)(c.n3 + 3) * B)], 1);
            }
          }
        }
      }
      if (!incident_reused && flag_dead) flag_dead[i] = 1;
      // other reactions remove a charged target (Src/collisions.f90:913-938)
      if (tgt && rt != 1 && rt != 3 && D.fd[T]) D.fd[T][ts.idx] = 1;
    }
    if (cnt_col) {
      int ix, iy, iz;
      S.cell_of(c, P, i, ix, iy, iz);
      for (int gq = 0; gq < c.n_rg; ++gq) {
        if (ix >= c.ixl[gq] && ix <= c.ixr[gq] && iy >= c.iyl && iy <= c.iyr && iz >= c.izl &&
            iz <= c.izr) {
          atomicAdd(&cnt_col[(c.R[sel].ind - 1) + (long long)c.ncol_mx * gq], c.w_rg[gq]);
          break;
        }
      }
    }
}

// The colliding candidates of a warp wait in a queue in shared memory until
// 32 of them can be scattered at once, one per lane (the selection leaves
// most lanes of a warp without a collision).  Per warp QCAP entries, fields
// in separate arrays: 11 doubles, 2 indices, 4 words.
constexpr int QCAP = 64;
constexpr int Q_WARP_BYTES = QCAP * (11 * 8 + 2 * 8 + 4 * 4);
constexpr int Q_SMEM = (MB / 32) * Q_WARP_BYTES;

struct QEntry {
  long long i;
  int sel, tgt;
  double v0[3];
  TState ts;
  uint32_t r0z, r0w;
};

struct WarpQueue {
  double *d;      // [11][QCAP]
  long long *l;   // [2][QCAP]
  int *w;         // [4][QCAP]
  __device__ __forceinline__ void put(int k, const QEntry &e) const {
    d[k] = e.v0[0];
    d[QCAP + k] = e.v0[1];
    d[2 * QCAP + k] = e.v0[2];
    d[3 * QCAP + k] = e.ts.tvx;
    d[4 * QCAP + k] = e.ts.tvy;
    d[5 * QCAP + k] = e.ts.tvz;
    d[6 * QCAP + k] = e.ts.mu;
    d[7 * QCAP + k] = e.ts.vr;
    d[8 * QCAP + k] = e.ts.vxc;
    d[9 * QCAP + k] = e.ts.vyc;
    d[10 * QCAP + k] = e.ts.vzc;
    l[k] = e.i;
    l[QCAP + k] = e.ts.idx;
    w[k] = e.sel;
    w[QCAP + k] = e.tgt;
    w[2 * QCAP + k] = (int)e.r0z;
    w[3 * QCAP + k] = (int)e.r0w;
  }
  __device__ __forceinline__ void get(int k, QEntry &e) const {
    e.v0[0] = d[k];
    e.v0[1] = d[QCAP + k];
    e.v0[2] = d[2 * QCAP + k];
    e.ts.tvx = d[3 * QCAP + k];
    e.ts.tvy = d[4 * QCAP + k];
    e.ts.tvz = d[5 * QCAP + k];
    e.ts.mu = d[6 * QCAP + k];
    e.ts.vr = d[7 * QCAP + k];
    e.ts.vxc = d[8 * QCAP + k];
    e.ts.vyc = d[9 * QCAP + k];
    e.ts.vzc = d[10 * QCAP + k];
    e.ts.Ekr = 0.0;
    e.ts.ok = true;
    e.i = l[k];
    e.ts.idx = l[QCAP + k];
    e.sel = w[k];
    e.tgt = w[QCAP + k];
    e.r0z = (uint32_t)w[2 * QCAP + k];
    e.r0w = (uint32_t)w[3 * QCAP + k];
  }
};

template <class Acc, bool DSMC>
__global__ void __launch_bounds__(MB, 2) k_mcc_collide(MCCConst c, Acc S, Targets D, const int *__restrict__ cand,
                                                    const int *__restrict__ ncand_p,
                                                    const double *__restrict__ Er,
                                                    const double *__restrict__ sig, signed char *flag_dead,
                                                    int *add, unsigned long long *counts, double *cnt_col,
                                                    int *err, Round rd) {
  const unsigned full = 0xffffffffu;
  const int P = c.ptype - 1;
  const int ncand = *ncand_p;
  const int lane = threadIdx.x & 31;
  const long long warp0 = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  extern __shared__ __align__(16) unsigned char q_smem[];
  unsigned char *qb = q_smem + (threadIdx.x >> 5) * Q_WARP_BYTES;
  const WarpQueue Q{reinterpret_cast<double *>(qb), reinterpret_cast<long long *>(qb + 11 * 8 * QCAP),
                    reinterpret_cast<int *>(qb + 13 * 8 * QCAP)};
  int qn = 0;   // entries in the warp's queue (the same in every lane)
  for (long long wb = warp0 * 32; wb < ncand; wb += nwarps * 32) {
    const long long t = wb + lane;
    int sel = -1;
    QEntry qe;
    if (t < ncand) {
      const long long i = cand[t];
      U4 ctr = {(uint32_t)i, 0u, c.c2, c.c3};
      const U4 r0 = philox4x32_10(ctr, c.k0, c.k1);
      double vx0, vy0, vz0;
      S.load_v(P, i, vx0, vy0, vz0);
      ctr.y = 1u;
      const U4 r1 = philox4x32_10(ctr, c.k0, c.k1);
      // the incident's cell (DSMC only)
      int cix = 1, ciy = 1, ciz = 1;
      long long ici = 0;
      if (DSMC) {
        S.cell_of(c, P, i, cix, ciy, ciz);
        ici = (cix - 1) + (long long)D.n1 * ((ciy - 1) + (long long)D.n2 * (ciz - 1)) + 1;
      }
      ctr.y = 3u;
      const U4 r3 = DSMC ? philox4x32_10(ctr, c.k0, c.k1) : U4{0u, 0u, 0u, 0u};
      // the partner for target species tt: a Maxwellian neutral
      // (Src/collisions.f90:437-449; the same draws for every neutral
      // species) or a particle of a charged species (DSMC)
      auto partner = [&](int tt, bool charged) {
        TState t;
        t.idx = -1;
        t.ok = true;
        if (DSMC && charged) {
          t.idx = pick_target(D, tt - 1, ici, r3.x);
          t.ok = t.idx >= 0;
          if (!t.ok) return t;
          S.load_v(tt - 1, t.idx, t.tvx, t.tvy, t.tvz);
        } else {
          const double vt = c.vt0[tt - 1];
          const double vp = vt * sqrt(-log(u01(r1.x)));
          double s1, c1;
          sincos(2.0 * c.pi * u01(r1.y), &s1, &c1);
          t.tvx = vp * c1;
          t.tvy = vp * s1;
          const double vp2 = vt * sqrt(-log(u01(r1.z)));
          t.tvz = vp2 * cos(2.0 * c.pi * u01(r1.w));
        }
        const double mt = fabs(c.mass[tt - 1]);
        t.mu = c.m_p * mt / (c.m_p + mt);
        t.vr = sqrt((vx0 - t.tvx) * (vx0 - t.tvx) + (vy0 - t.tvy) * (vy0 - t.tvy) + (vz0 - t.tvz) * (vz0 - t.tvz));
        t.Ekr = (0.5 * t.mu * (t.vr * t.vr)) / c.qe;
        const double sm = c.m_p + mt;
        t.vxc = (c.m_p * vx0 + mt * t.tvx) / sm;
        t.vyc = (c.m_p * vy0 + mt * t.tvy) / sm;
        t.vzc = (c.m_p * vz0 + mt * t.tvz) / sm;
        if (t.Ekr > Er[c.npt - 1]) raise_err(err, LEPIC_ERR_EKR_TABLE, (int)i);
        return t;
      };
      TState ts;
      ts.ok = false;
      int cur_tt = -1, seg = -1;
      unsigned missed = 0u;
      // nu_r / nu_max of reaction r; the partner and the interval of the
      // merged energy grid (shared by all tables) change with the target
      // species only
      auto nu_of = [&](int r) -> double {
        const int tt = c.R[r].tt;
        if (tt != cur_tt) {
          ts = partner(tt, c.R[r].dsmc != 0);
          if (!ts.ok) missed |= 1u << tt;
          seg = ts.ok ? energy_segment(Er, c.npt, ts.Ekr) : -1;
          cur_tt = tt;
        }
        if (seg < 0) return 0.0;
        const double sp = sigma_in(Er, sig + (long long)c.npt_mx * (c.R[r].ind - 1), seg, ts.Ekr);
        double np_t = c.R[r].np_t;
        if (DSMC && c.R[r].dsmc) {
          // the target density at the incident's cell (Src/collisions.f90:524-531)
          const double *g = D.np[tt - 1];
          const long long N1 = D.n1 + 3, N2 = D.n2 + 3;
          const long long q = cix + N1 * (ciy + N2 * (long long)ciz), sy = N1, sz = N1 * N2;
          np_t = 0.125 * (g[q] + g[q + 1] + g[q + sy] + g[q + 1 + sy] + g[q + sz] + g[q + 1 + sz] + g[q + sy + sz] +
                          g[q + 1 + sy + sz]);
        }
        return np_t * sp * ts.vr / c.nu_max;
      };
      // pass 1: sum_r nu_r; pass 2 (a collision): the partial sums up to the
      // drawn u over the reactions in ascending order of nu_r, as the
      // reference sorts them (Src/collisions.f90:711-737).  The order
      // matters when sum_r nu_r exceeds 1 (nu_max held at nu_uplim): the
      // smallest frequencies then keep their full share.
      double sum_nu = 0.0;
      for (int r = 0; r < c.nr; ++r) sum_nu += nu_of(r);
      if (DSMC && missed && rd.first) atomicAdd(&D.stat[0], (unsigned long long)__popc(missed));
      const double u = u01(r0.y);
      if (u <= sum_nu && S.live(P, i)) {
        double nu[MAXR];
        unsigned char ord[MAXR];
        cur_tt = -1;
        for (int r = 0; r < c.nr; ++r) {
          // insertion by value; equal values keep the table order
          const double v = nu_of(r);
          int k = r;
          while (k > 0 && nu[k - 1] > v) {
            nu[k] = nu[k - 1];
            ord[k] = ord[k - 1];
            --k;
          }
          nu[k] = v;
          ord[k] = (unsigned char)r;
        }
        double s = 0.0;
        for (int k = 0; k < c.nr; ++k) {
          s += nu[k];
          if (u <= s) {
            sel = ord[k];
            break;
          }
        }
      }
      const bool tgt = DSMC && sel >= 0 && c.R[sel].dsmc;
      if (sel >= 0) {
        if (c.R[sel].tt != cur_tt) ts = partner(c.R[sel].tt, tgt);
        // a charged target takes part in one collision per round; a later
        // collision on it is evaluated again in the next round
        if (tgt && atomicExch(&D.claim[c.R[sel].tt - 1][ts.idx], rd.tag) == rd.tag) {
          rd.defer[atomicAdd(rd.ndefer, 1)] = (int)i;
          atomicAdd(&D.stat[2], 1ull);
          sel = -1;
        }
      }
      if (sel >= 0) {
        qe.i = i;
        qe.sel = sel;
        qe.tgt = tgt ? 1 : 0;
        qe.v0[0] = vx0;
        qe.v0[1] = vy0;
        qe.v0[2] = vz0;
        qe.ts = ts;
        qe.r0z = r0.z;
        qe.r0w = r0.w;
      }
    }
    {
      // the warp's colliding candidates into its queue; 32 of them
      // scattered at once when the queue holds that many, and the rest
      // after the warp's last candidates (one call site, uniform over the
      // warp)
      const unsigned m = __ballot_sync(full, sel >= 0);
      if (sel >= 0) Q.put(qn + __popc(m & lanemask_lt_m()), qe);
      qn += __popc(m);
      __syncwarp();
      const bool last = wb + nwarps * 32 >= ncand;
      while (qn >= 32 || (last && qn > 0)) {
        const int k = qn < 32 ? qn : 32;
        if (lane < k) {
          QEntry f;
          Q.get(lane, f);
          mcc_apply<Acc, DSMC>(c, S, D, f.i, f.sel, f.tgt != 0, f.v0[0], f.v0[1], f.v0[2], f.ts, f.r0z, f.r0w,
                               flag_dead, add, cnt_col, err);
        }
        __syncwarp();
        if (lane < qn - k) {
          QEntry g;
          Q.get(k + lane, g);
          Q.put(lane, g);
        }
        qn -= k;
        __syncwarp();
      }
    }
    // warp-aggregated collision counters
    if (__ballot_sync(full, sel >= 0)) {
      for (int r = 0; r < c.nr; ++r) {
        const unsigned m = __ballot_sync(full, sel == r);
        if (lane == 0 && m) atomicAdd(&counts[c.R[r].ind - 1], (unsigned long long)__popc(m));
      }
    }
  }
}

// the appended products enter the counts; appends beyond the capacity were
// not written (LEPIC_ERR_CAPACITY is raised), so a count stops at its capacity
struct Counts {
  int *count[LEPIC_NPART];
  long long cap[LEPIC_NPART];
};

__global__ void k_mcc_finalize(Counts C, const int *add, int ntype) {
  int *const *cs = C.count;
  const long long *caps = C.cap;
  for (int p = 0; p < ntype && p < LEPIC_NPART; ++p)
    if (cs[p]) {
      const long long v = (long long)*cs[p] + add[p];
      *cs[p] = (int)(v < caps[p] ? v : caps[p]);
    }
}

// Host part shared by both layouts: nu_max, Pmax and the per-species
// constants (Src/collisions.f90:97-165).
// The differentiable window's collisions: the log they are recorded in.
struct WinLog {
  lepic_win_event_t *log;
  int *nlog;   // device int: records written (continues across calls)
  int cap, step;
};

template <class Acc>
int run_collisions(const lepic_grid_t &g, Acc S, int *const *counts_dev, signed char *const *flag_dead,
                   int ntype, const lepic_tables_t &T, const lepic_phys_t &P, unsigned long long seed,
                   unsigned long long call_index, double *nu_max, long long *counts, cudaStream_t s,
                   const RegionCount *rg, const char *tname, lepic_targets_t *tg, int tile,
                   const WinLog *wlog = nullptr) {
  if (ntype < 1 || ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  // DSMC state: density grids and sort offsets from the caller, claims here
  Targets D;
  memset(&D, 0, sizeof(D));
  D.tile = tile;
  D.n1 = g.n[0];
  D.n2 = g.n[1];
  D.n3 = g.n[2];
  D.ntx = (g.n[0] + 7) / 8;
  D.nty = (g.n[1] + 7) / 8;
  // cell indices beyond n1 n2 n3 hold no particles: every Plist covering the
  // grid's cells is read within its bounds
  D.pl_max = (long long)g.n[0] * g.n[1] * g.n[2];
  D.stat = (unsigned long long *)scratch("mcc_dsmc_stat", 3 * sizeof(unsigned long long));
  if (!D.stat) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(D.stat, 0, 3 * sizeof(unsigned long long), s));
  int tag = 0;                  // claim tag of the last DSMC round launched
  unsigned long long left_over = 0;
  for (int q = 0; q < ntype; ++q) {
    D.fd[q] = flag_dead[q];
    if (tg) {
      D.np[q] = tg->np[q];
      D.off[q] = tg->cell_off[q];
    }
  }
  auto CI = [&](int icol, int info) { return T.col_info_h[(icol - 1) + (long long)T.ncol * (info - 1)]; };
  int *add = (int *)scratch("mcc_add", sizeof(int) * LEPIC_NPART);
  unsigned long long *cnt = (unsigned long long *)scratch("mcc_cnt", sizeof(unsigned long long) * 64);
  int *ncand = (int *)scratch("mcc_ncand", sizeof(int) * LEPIC_NPART);
  if (!add || !cnt || !ncand || T.ncol > 64) return LEPIC_ERR_CUDA;
  LEPIC_CUDA(cudaMemsetAsync(add, 0, sizeof(int) * LEPIC_NPART, s));
  LEPIC_CUDA(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long) * 64, s));
  LEPIC_CUDA(cudaMemsetAsync(ncand, 0, sizeof(int) * LEPIC_NPART, s));
  std::vector<double> Eth(T.ncol > 0 ? T.ncol : 1, 0.0);
  if (T.ncol > 0)
    LEPIC_CUDA(cudaMemcpyAsync(Eth.data(), T.sig_Eth, sizeof(double) * T.ncol, cudaMemcpyDeviceToHost, s));
  std::vector<int> Nh(ntype, 0);
  for (int p = 0; p < ntype; ++p)
    LEPIC_CUDA(cudaMemcpyAsync(&Nh[p], counts_dev[p], sizeof(int), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaStreamSynchronize(s));
  for (int p = 1; p <= ntype; ++p) {
    nu_max[p - 1] = 0.0;
    const int pn = T.p_ncol[p - 1];
    if (pn == 0 || P.mass[p - 1] <= 0) continue;
    if (pn > MAXR) {
      fprintf(stderr, "lepic_gpu: collisions: species %d has %d reactions (at most %d)\n", p, pn, MAXR);
      return LEPIC_ERR_UNSUPPORTED;
    }
    MCCConst c;
    memset(&c, 0, sizeof(c));
    Reac hr[MAXR];
    memset(hr, 0, sizeof(hr));
    c.ptype = p;
    c.nr = pn;
    c.qe = P.qe;
    c.pi = P.pi;
    c.m_p = fabs(P.mass[p - 1]);
    for (int q = 0; q < LEPIC_NPART; ++q) {
      c.mass[q] = P.mass[q];
      c.vt0[q] = P.vt0[q];
    }
    double num = 0.0;
    for (int r = 0; r < pn; ++r) {
      const int ind = T.sig_list[(p - 1) + LEPIC_NPART * r];
      const int n_re = CI(ind, 1), n_by = CI(ind, 2);
      if (n_by > MAXBY || n_re > 2) {
        fprintf(stderr, "lepic_gpu: collisions: reaction %d has %d reactants and %d byproducts (at most 2 and %d)\n",
                ind, n_re, n_by, MAXBY);
        return LEPIC_ERR_UNSUPPORTED;
      }
      const int tt = CI(ind, 2 + n_re);
      if (wlog) {
        // the window keeps every particle's slot: no charged targets, and
        // the incident survives (elastic, excitation, charge exchange, or
        // a reaction whose first byproduct is the incident's species)
        const int rt = CI(ind, 3 + n_re + n_by);
        const bool kept = rt == 1 || rt == 3 || rt == 4 || (n_by > 0 && CI(ind, 3 + n_re) == p);
        if (P.charge[tt - 1] != 0.0 || !kept) {
          fprintf(stderr, "lepic_gpu: window collisions: reaction %d (charged target or incident removed)\n", ind);
          return LEPIC_ERR_UNSUPPORTED;
        }
      }
      if (P.charge[tt - 1] != 0.0 && tt == p) {
        // the incident would have to be claimed as well as its target
        fprintf(stderr, "lepic_gpu: collisions: reaction %d has a charged target of the incident's own species\n",
                ind);
        return LEPIC_ERR_UNSUPPORTED;
      }
      if (P.charge[tt - 1] != 0.0) {
        // a charged target: its density grid and sort offsets are needed
        if (tt > ntype || !D.np[tt - 1] || !D.off[tt - 1] || !D.fd[tt - 1]) {
          fprintf(stderr,
                  "lepic_gpu: collisions: reaction %d has the charged target species %d without its density "
                  "grid, sort offsets or flag_dead (lepic_targets_t)\n",
                  ind, tt);
          return LEPIC_ERR_UNSUPPORTED;
        }
        hr[r].dsmc = 1;
        c.any_dsmc = 1;
        if (!D.claim[tt - 1]) {
          char cn[32];
          snprintf(cn, sizeof cn, "mcc_claim%d", tt - 1);
          D.claim[tt - 1] = (int *)scratch(cn, sizeof(int) * (size_t)S.cap[tt - 1]);
          if (!D.claim[tt - 1]) return LEPIC_ERR_CUDA;
          LEPIC_CUDA(cudaMemsetAsync(D.claim[tt - 1], 0, sizeof(int) * (size_t)S.cap[tt - 1], s));
        }
      }
      hr[r].ind = ind;
      hr[r].tt = tt;
      hr[r].n_re = n_re;
      hr[r].n_by = n_by;
      for (int a = 0; a < n_by; ++a) hr[r].by[a] = CI(ind, 3 + n_re + a);
      hr[r].rt = CI(ind, 3 + n_re + n_by);
      hr[r].Eth = Eth[ind - 1];
      hr[r].np_t = P.np_mx[tt - 1];
      num = num + P.np_mx[tt - 1] * T.sigv_mx[(p - 1) + LEPIC_NPART * (ind - 1)];
    }
    nu_max[p - 1] = num < P.nu_uplim[p - 1] ? num : P.nu_uplim[p - 1];
    const double Pmax = nu_max[p - 1] * (double)(float)P.ns_coll * P.dt;
    if (Pmax > 1.0) return LEPIC_ERR_PMAX;
    if (Nh[p - 1] == 0 || nu_max[p - 1] <= 0.0) continue;
    c.Pmax = Pmax;
    c.nu_max = nu_max[p - 1];
    c.npt = T.npt;
    c.npt_mx = T.npt_mx;
    c.k0 = (unsigned)(seed & 0xffffffffu);
    c.k1 = (unsigned)(seed >> 32);
    c.c2 = (unsigned)(call_index & 0xffffffffu);
    c.c3 = (unsigned)((call_index >> 32) << 8) | (unsigned)p;
    c.h0 = g.h[0];
    c.h1 = g.h[1];
    c.h2 = g.h[2];
    if (wlog) {
      c.log = wlog->log;
      c.nlog = wlog->nlog;
      c.log_cap = wlog->cap;
      c.step = wlog->step;
    }
    double *cc = nullptr;
    if (rg && rg->cnt_col_dev) {
      c.n_rg = rg->n_rg;
      c.ncol_mx = rg->ncol_mx;
      for (int q = 0; q < LEPIC_NM_RG; ++q) {
        c.ixl[q] = rg->ixl[q];
        c.ixr[q] = rg->ixr[q];
        c.w_rg[q] = rg->w[p - 1][q];
      }
      c.iyl = rg->iyl;
      c.iyr = rg->iyr;
      c.izl = rg->izl;
      c.izr = rg->izr;
      cc = rg->cnt_col_dev;
    }
    if (rg) {
      c.ploss3 = rg->ploss3_dev;
      c.sxy = rg->sour_xy_dev;
      c.sxz = rg->sour_xz_dev;
      c.iz_pl = rg->iz_pl;
      c.iy_pl = rg->iy_pl;
      for (int q = 0; q < LEPIC_NPART; ++q) c.Nm[q] = P.Nm[q];
    }
    c.n1 = g.n[0];
    c.n2 = g.n[1];
    c.n3 = g.n[2];
    // the reaction table of this species, in device memory
    char rn[32];
    snprintf(rn, sizeof rn, "mcc_reac%d", p - 1);
    Reac *R = (Reac *)scratch(rn, sizeof(Reac) * MAXR);
    if (!R) return LEPIC_ERR_CUDA;
    LEPIC_CUDA(cudaMemcpyAsync(R, hr, sizeof(Reac) * (size_t)pn, cudaMemcpyHostToDevice, s));
    c.R = R;
    // the candidate list shares the species' work list with the push (hole
    // list), sized by the capacity, so that the step loop allocates nothing
    // after its first push
    char nm[32];
    snprintf(nm, sizeof nm, "work_list%d", p - 1);
    int *cand = (int *)scratch(nm, sizeof(int) * (size_t)S.cap[p - 1]);
    if (!cand) return LEPIC_ERR_CUDA;
    char sname[32];
    snprintf(sname, sizeof sname, "%s_select", tname);
    int tm = timer_start(sname, s);
    if (Pmax < SKIP_PMAX) {
      const int seg = skip_segment(Pmax);
      const long long nseg = (Nh[p - 1] + seg - 1) / seg;
      k_mcc_select_skip<<<grid_for(nseg, MB), MB, 0, s>>>(c, counts_dev[p - 1], 1.0 / log1p(-Pmax), seg, cand,
                                                          ncand + (p - 1));
    } else {
      k_mcc_select<<<grid_for(Nh[p - 1], MB), MB, 0, s>>>(c, counts_dev[p - 1], cand, ncand + (p - 1));
    }
    timer_stop(tm, s);
    tm = timer_start(tname, s);
    LEPIC_CUDA(cudaFuncSetAttribute(k_mcc_collide<Acc, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, Q_SMEM));
    LEPIC_CUDA(cudaFuncSetAttribute(k_mcc_collide<Acc, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, Q_SMEM));
    if (c.any_dsmc) {
      // rounds until no collision is deferred: the list of round r is read
      // from one buffer while the deferrals of the round go to the other
      // (the candidate list and a deferral list of the same capacity);
      // rc[r] counts the collisions of round r >= 1
      snprintf(nm, sizeof nm, "mcc_defer%d", p - 1);
      int *defer = (int *)scratch(nm, sizeof(int) * (size_t)S.cap[p - 1]);
      int *rc = (int *)scratch("mcc_round_cnt", sizeof(int) * (DSMC_ROUNDS + 1));
      if (!defer || !rc) return LEPIC_ERR_CUDA;
      LEPIC_CUDA(cudaMemsetAsync(rc, 0, sizeof(int) * (DSMC_ROUNDS + 1), s));
      int r = 0;
      for (;;) {
        // a batch of rounds without a host round trip (an empty round
        // returns at once), then the count left for the next round
        const int stop = r + DSMC_BATCH < DSMC_ROUNDS ? r + DSMC_BATCH : DSMC_ROUNDS;
        for (; r < stop; ++r) {
          Round rd;
          rd.defer = (r & 1) ? cand : defer;
          rd.ndefer = rc + r + 1;
          rd.tag = ++tag;
          rd.first = r == 0;
          const int *in = (r & 1) ? defer : cand;
          const int *nin = r == 0 ? ncand + (p - 1) : rc + r;
          k_mcc_collide<Acc, true><<<ctx().sms * 8, MB, Q_SMEM, s>>>(c, S, D, in, nin, T.sig_Er, T.sig,
                                                                flag_dead[p - 1], add, cnt, cc, ctx().d_err, rd);
          LEPIC_CUDA(cudaGetLastError());
        }
        int left = 0;
        LEPIC_CUDA(cudaMemcpyAsync(&left, rc + r, sizeof(int), cudaMemcpyDeviceToHost, s));
        LEPIC_CUDA(cudaStreamSynchronize(s));
        if (left == 0) break;
        if (r >= DSMC_ROUNDS) {
          left_over += (unsigned long long)left;
          break;
        }
      }
    } else {
      Round rd{nullptr, nullptr, 0, 1};
      k_mcc_collide<Acc, false><<<ctx().sms * 8, MB, Q_SMEM, s>>>(c, S, D, cand, ncand + (p - 1), T.sig_Er, T.sig,
                                                             flag_dead[p - 1], add, cnt, cc, ctx().d_err, rd);
    }
    timer_stop(tm, s);
    LEPIC_CUDA(cudaGetLastError());
  }
  Counts fc;
  memset(&fc, 0, sizeof(fc));
  for (int q = 0; q < ntype; ++q) {
    fc.count[q] = counts_dev[q];
    fc.cap[q] = S.cap[q];
  }
  k_mcc_finalize<<<1, 1, 0, s>>>(fc, add, ntype);
  LEPIC_CUDA(cudaGetLastError());
  unsigned long long hc[64], hs[3];
  LEPIC_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
  LEPIC_CUDA(cudaMemcpyAsync(hs, D.stat, sizeof(hs), cudaMemcpyDeviceToHost, s));
  const int rc = check_err(s);
  if (counts)
    for (int q = 0; q < T.ncol; ++q) counts[q] += (long long)hc[q];
  if (tg) {
    tg->missed += (long long)hs[0];
    tg->lost_claims += (long long)left_over;
    tg->replayed += (long long)hs[2];
  }
  return rc;
}

}  // namespace

int launch_collisions(const lepic_grid_t &g, lepic_species_f64_t *sp, int ntype,
                      const lepic_tables_t &T, const lepic_phys_t &P, unsigned long long seed,
                      unsigned long long call_index, double *nu_max, long long *counts,
                      cudaStream_t s, const RegionCount *rg, lepic_targets_t *tg) {
  if (ntype < 1 || ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  AccF64 S;
  memset(&S, 0, sizeof(S));
  int *cnts[LEPIC_NPART] = {nullptr};
  signed char *fd[LEPIC_NPART] = {nullptr};
  for (int p = 0; p < ntype; ++p) {
    S.p[p] = sp[p].p;
    S.count[p] = sp[p].count;
    S.cap[p] = sp[p].cap;
    cnts[p] = sp[p].count;
    fd[p] = sp[p].flag_dead;
  }
  return run_collisions(g, S, cnts, fd, ntype, T, P, seed, call_index, nu_max, counts, s, rg, "mcc_f64", tg, 0);
}

int launch_collisions_mixed(const lepic_grid_t &g, lepic_species_mixed_t *sp, int ntype,
                            const lepic_tables_t &T, const lepic_phys_t &P, unsigned long long seed,
                            unsigned long long call_index, double *nu_max, long long *counts,
                            cudaStream_t s, lepic_targets_t *tg) {
  if (ntype < 1 || ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  AccMixed S;
  memset(&S, 0, sizeof(S));
  int *cnts[LEPIC_NPART] = {nullptr};
  signed char *fd[LEPIC_NPART] = {nullptr};
  for (int p = 0; p < ntype; ++p) {
    S.cell[p] = sp[p].cell;
    S.p[p] = sp[p].p;
    S.count[p] = sp[p].count;
    S.cap[p] = sp[p].cap;
    cnts[p] = sp[p].count;
    fd[p] = sp[p].flag_dead;
  }
  return run_collisions(g, S, cnts, fd, ntype, T, P, seed, call_index, nu_max, counts, s, nullptr,
                        "mcc_mixed", tg, 1);
}

// the differentiable window's collisions, recorded in the log (ws in FP32 or
// FP64 planes, fp64 taken from ws[0])
template <class R>
int run_window_collisions(const lepic_grid_t &g, lepic_win_species_t *ws, int ntype, const lepic_tables_t &T,
                          const lepic_phys_t &P, unsigned long long seed, unsigned long long call_index,
                          double *nu_max, long long *counts, const WinLog &wl, cudaStream_t s) {
  AccWin<R> S;
  memset(&S, 0, sizeof(S));
  int *cnts[LEPIC_NPART] = {nullptr};
  signed char *fd[LEPIC_NPART] = {nullptr};
  for (int p = 0; p < ntype; ++p) {
    S.cell[p] = ws[p].cell;
    S.p[p] = (R *)ws[p].p;
    S.bl[p] = ws[p].bl;
    S.count[p] = ws[p].count;
    S.cap[p] = ws[p].cap;
    cnts[p] = ws[p].count;
  }
  S.step = wl.step;
  return run_collisions(g, S, cnts, fd, ntype, T, P, seed, call_index, nu_max, counts, s, nullptr,
                        ws[0].fp64 ? "mcc_window_f64" : "mcc_window", nullptr, 1, &wl);
}

}  // namespace lepic

extern "C" int lepic_dev_win_collisions(const lepic_grid_t *g, lepic_win_species_t *ws, int ntype,
                                        const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                                        unsigned long long call_index, int step, lepic_win_event_t *log,
                                        int log_cap, int *nlog, double *nu_max, long long *counts, void *stream) {
  if (!g || !ws || !T || !P || !log || !nlog || ntype < 1 || ntype > LEPIC_NPART || log_cap < 0 || step < 0)
    return LEPIC_ERR_ARG;
  for (int p = 1; p < ntype; ++p)
    if (ws[p].fp64 != ws[0].fp64) return LEPIC_ERR_ARG;
  lepic::WinLog wl{log, nlog, log_cap, step};
  if (ws[0].fp64)
    return lepic::run_window_collisions<double>(*g, ws, ntype, *T, *P, seed, call_index, nu_max, counts, wl,
                                                (cudaStream_t)stream);
  return lepic::run_window_collisions<float>(*g, ws, ntype, *T, *P, seed, call_index, nu_max, counts, wl,
                                             (cudaStream_t)stream);
}

extern "C" int lepic_dev_collisions_mixed(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype,
                                          const lepic_tables_t *T, const lepic_phys_t *P,
                                          unsigned long long seed, unsigned long long call_index,
                                          double *nu_max, long long *counts, void *stream) {
  if (!g || !sp || !T || !P || ntype < 1) return LEPIC_ERR_ARG;
  return lepic::launch_collisions_mixed(*g, sp, ntype, *T, *P, seed, call_index, nu_max, counts,
                                        (cudaStream_t)stream, nullptr);
}

extern "C" int lepic_dev_collisions_mixed_targets(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype,
                                                  const lepic_tables_t *T, const lepic_phys_t *P,
                                                  unsigned long long seed, unsigned long long call_index,
                                                  double *nu_max, long long *counts, lepic_targets_t *tg,
                                                  void *stream) {
  if (!g || !sp || !T || !P || !tg || ntype < 1) return LEPIC_ERR_ARG;
  return lepic::launch_collisions_mixed(*g, sp, ntype, *T, *P, seed, call_index, nu_max, counts,
                                        (cudaStream_t)stream, tg);
}
