// C ABI of the library: the device API (lepic_dev_*) and the Fortran
// drop-in routines with the reference's names and argument lists.
#include <cmath>
#include <cstring>
#include <vector>

#include "lepic_internal.cuh"

using namespace lepic;

// Fortran COMMON blocks (Src/particle_info.h:53-70, Src/constants.h).  Weak,
// so that the Fortran program's own COMMON storage wins when both exist.
extern "C" {
__attribute__((weak)) lepic_part_info_int_t part_info_int_ = {};
__attribute__((weak)) lepic_part_info_dp_1_t part_info_dp_1_ = {};
__attribute__((weak)) lepic_part_info_dp_2_t part_info_dp_2_ = {};
__attribute__((weak)) lepic_part_info_dp_3_t part_info_dp_3_ = {};
__attribute__((weak)) lepic_constants_t constants_ = {};
}

namespace {

thread_local int g_last = 0;

inline cudaStream_t S(void *s) { return (cudaStream_t)s; }

void record(int rc) {
  if (rc && !g_last) g_last = rc;
}

// lepic_phys_t from the COMMON blocks (what the Fortran routines read)
lepic_phys_t phys_from_common(int ntype) {
  lepic_phys_t P;
  memset(&P, 0, sizeof(P));
  P.ntype = ntype;
  for (int p = 0; p < LEPIC_NPART; ++p) {
    P.charge[p] = part_info_dp_1_.charge[p];
    P.mass[p] = part_info_dp_1_.mass[p];
    P.vt0[p] = part_info_dp_1_.vt0[p];
    P.Nm[p] = part_info_dp_2_.Nm[p];
    P.np_mx[p] = part_info_dp_3_.np_mx[p];
    P.nu_uplim[p] = part_info_dp_3_.nu_uplim[p];
  }
  P.dt = part_info_dp_2_.dt;
  P.xmax = part_info_dp_2_.xmax;
  P.ymax = part_info_dp_2_.ymax;
  P.zmax = part_info_dp_2_.zmax;
  P.x_load = part_info_dp_2_.x_load;
  P.qe = constants_.qe;
  P.eps0 = constants_.eps0;
  P.pi = constants_.pi;
  P.flag_B = part_info_int_.flag_B;
  P.flag_B_pos = part_info_int_.flag_B_pos;
  P.flag_pbc = part_info_int_.flag_pbc;
  P.flag_nmn = part_info_int_.flag_nmn;
  P.ns_coll = part_info_int_.ns_coll;
  P.n_cell = part_info_int_.n_cell;
  P.np_cell = part_info_int_.np_cell;
  return P;
}

// LEPIC_OK or the status of a failed runtime call
int cuda_ok(cudaError_t e, const char *what) { return e == cudaSuccess ? LEPIC_OK : cuda_status(e, what); }

// heating region and rate from the COMMON blocks
lepic_heat_t heat_from_common() {
  lepic_heat_t H;
  memset(&H, 0, sizeof(H));
  H.ixl_pow = part_info_int_.ixl_pow;
  H.ixr_pow = part_info_int_.ixr_pow;
  H.flag_circxh = part_info_int_.flag_circxh;
  H.flag_ahp = part_info_int_.flag_ahp;
  H.R_ahp = part_info_dp_2_.R_ahp;
  H.nudt = part_info_dp_2_.nudt;
  H.Pabs = part_info_dp_2_.Pabs;
  H.nu_h = part_info_dp_2_.nu_h;
  return H;
}

// Temporary device copy of a host table the call builds itself.
template <class T>
T *upload(const char *name, const T *h, size_t n, cudaStream_t s) {
  T *d = (T *)scratch(name, sizeof(T) * (n ? n : 1));
  if (d && n && mirror_h2d(d, h, sizeof(T) * n, s)) return nullptr;
  return d;
}

// Device view of a Fortran host array for one drop-in call.  Without
// residency: a named staging buffer, filled from the host unless the call
// only writes it (WRITE), copied back by host_back.  With residency: the
// array's device mirror, marked device-newer unless the call only reads it.
enum Use { READ, WRITE, UPDATE };

template <class T>
T *dev_view(const char *name, const T *h, size_t n, Use u, cudaStream_t s, int *rc) {
  *rc = LEPIC_OK;
  if (residency_on()) {
    T *d = (T *)mirror_array(h, sizeof(T) * n, u != READ, s, rc);
    if (!d && !*rc) *rc = LEPIC_ERR_CUDA;
    return d;
  }
  T *d = (T *)scratch(name, sizeof(T) * (n ? n : 1));
  if (!d) {
    *rc = LEPIC_ERR_CUDA;
    return nullptr;
  }
  if (u != WRITE) *rc = mirror_h2d(d, h, sizeof(T) * n, s);
  return *rc ? nullptr : d;
}

// Results of a call back into the host array (a mirror keeps them).
template <class T>
int host_back(T *h, const T *d, size_t n, cudaStream_t s) {
  if (residency_on()) return LEPIC_OK;
  return mirror_d2h(h, d, sizeof(T) * n, s);
}

// Per-call staging of one host species slice vxp(6, 1:np, ptype, 1): SoA
// copies under slot-numbered scratch names.
struct StagedSpecies {
  lepic_species_f64_t s;
  double *aos = nullptr;
  int n = 0;
};

int stage_species(StagedSpecies &st, const double *vxp_h, int np, int nmax, int slot,
                  const signed char *flag_dead_h, cudaStream_t s) {
  char nm[48];
  long long cap = nmax;
  snprintf(nm, sizeof nm, "dropin_p%d", slot);
  st.s.p = (double *)scratch(nm, sizeof(double) * 6 * cap);
  snprintf(nm, sizeof nm, "dropin_q%d", slot);
  st.s.p_alt = (double *)scratch(nm, sizeof(double) * 6 * cap);
  snprintf(nm, sizeof nm, "dropin_cnt%d", slot);
  st.s.count = (int *)scratch(nm, sizeof(int));
  snprintf(nm, sizeof nm, "dropin_key%d", slot);
  st.s.key = (int *)scratch(nm, sizeof(int) * cap);
  snprintf(nm, sizeof nm, "dropin_aos%d", slot);
  st.aos = (double *)scratch(nm, sizeof(double) * 6 * cap);
  snprintf(nm, sizeof nm, "dropin_fd%d", slot);
  st.s.flag_dead = (signed char *)scratch(nm, cap);
  st.s.cap = nmax;
  st.n = np;
  if (!st.s.p || !st.s.p_alt || !st.s.count || !st.s.key || !st.aos || !st.s.flag_dead)
    return LEPIC_ERR_CUDA;
  int rc = mirror_h2d(st.s.count, &st.n, sizeof(int), s);
  if (!rc && np > 0) rc = mirror_h2d(st.aos, vxp_h, sizeof(double) * 6 * (size_t)np, s);
  if (!rc) rc = aos_to_soa(st.aos, st.s.p, 0, np, cap, s);
  if (rc) return rc;
  if (flag_dead_h) return mirror_h2d(st.s.flag_dead, flag_dead_h, (size_t)nmax, s);
  LEPIC_CUDA(cudaMemsetAsync(st.s.flag_dead, 0, (size_t)nmax, s));
  return LEPIC_OK;
}

int unstage_species(StagedSpecies &st, double *vxp_h, int *np_out, signed char *flag_dead_h,
                    int nmax, cudaStream_t s) {
  int n = 0;
  int rc = mirror_d2h(&n, st.s.count, sizeof(int), s);
  if (rc) return rc;
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (n > nmax) n = nmax;
  rc = soa_to_aos(st.s.p, st.aos, n, st.s.cap, s);
  if (!rc && n > 0) rc = mirror_d2h(vxp_h, st.aos, sizeof(double) * 6 * (size_t)n, s);
  if (!rc && flag_dead_h) rc = mirror_d2h(flag_dead_h, st.s.flag_dead, (size_t)nmax, s);
  if (rc) return rc;
  LEPIC_CUDA(cudaStreamSynchronize(s));
  if (np_out) *np_out = n;
  return LEPIC_OK;
}

// One species slice on the device for a drop-in call: staged, or the
// slice's mirror under residency.
struct SpeciesView {
  lepic_species_f64_t s{};
  StagedSpecies st;
  double *vxp_h = nullptr;
  bool resident = false;
};

int acquire_species(SpeciesView &v, double *vxp_h, int np, int nmax, int slot, signed char *fd_h,
                    cudaStream_t s) {
  v.vxp_h = vxp_h;
  v.resident = residency_on();
  if (v.resident) return mirror_species(vxp_h, np, nmax, fd_h, s, &v.s);
  int rc = stage_species(v.st, vxp_h, np, nmax, slot, fd_h, s);
  v.s = v.st.s;
  return rc;
}

// After the call: `wrote` = the call changed the particles (and flag_dead,
// when fd_h names it); np_out receives the count.
int release_species(SpeciesView &v, int *np_out, signed char *fd_h, int nmax, bool wrote,
                    cudaStream_t s) {
  if (v.resident) return mirror_species_done(v.vxp_h, v.s, wrote, wrote && fd_h, np_out, s);
  v.st.s = v.s;
  if (!wrote) return LEPIC_OK;
  return unstage_species(v.st, v.vxp_h, np_out, fd_h, nmax, s);
}

// Geometry for the drop-ins: bcnd, kq and the cell-wall mask.  Under
// residency the mask is kept until the bcnd mirror is reloaded.
int stage_grid(lepic_grid_t &g, const int *n, const double *h, const int *bcnd_h, const double *kq_h,
               cudaStream_t s) {
  Dims d(n);
  for (int a = 0; a < 3; ++a) {
    g.n[a] = n[a];
    g.h[a] = h ? h[a] : 0.0;
  }
  int rc = LEPIC_OK;
  g.bcnd = dev_view("dropin_bcnd", bcnd_h, (size_t)d.cnt(), READ, s, &rc);
  if (!g.bcnd) return rc;
  g.kq = nullptr;
  if (kq_h) {
    g.kq = dev_view("dropin_kq", kq_h, (size_t)d.cnt(), READ, s, &rc);
    if (!g.kq) return rc;
  }
  const size_t cells = (size_t)((d.N1 - 1) * (d.N2 - 1) * (d.N3 - 1));
  if (residency_on()) {
    static const int *cw_bcnd = nullptr;
    static const unsigned char *cw_buf = nullptr;
    static unsigned long long cw_gen = 0;
    static size_t cw_cells = 0;
    unsigned char *cw = (unsigned char *)scratch("mirror_cw", cells);
    if (!cw) return LEPIC_ERR_CUDA;
    unsigned long long gen = mirror_generation(bcnd_h);
    g.cell_wall = cw;
    if (cw == cw_buf && g.bcnd == cw_bcnd && gen == cw_gen && cells == cw_cells) return LEPIC_OK;
    rc = launch_cell_wall(d, g.bcnd, cw, s);
    if (rc) return rc;
    cw_bcnd = g.bcnd;
    cw_buf = cw;
    cw_gen = gen;
    cw_cells = cells;
    return LEPIC_OK;
  }
  unsigned char *cw = (unsigned char *)scratch("dropin_cw", cells);
  if (!cw) return LEPIC_ERR_CUDA;
  g.cell_wall = cw;
  return launch_cell_wall(d, g.bcnd, cw, s);
}

}  // namespace

extern "C" {

int lepic_gpu_last_error(void) {
  int r = g_last;
  g_last = 0;
  return r;
}

const char *lepic_gpu_strerror(int code) {
  switch (code) {
    case LEPIC_OK: return "ok";
    case LEPIC_ERR_CAPACITY: return "particle array capacity (nmax) exceeded";
    case LEPIC_ERR_DIVERGED: return "PDE solver is diverging";
    case LEPIC_ERR_PMAX: return "collision probability greater than 1";
    case LEPIC_ERR_EKR_TABLE: return "collision energy above the cross-section table";
    case LEPIC_ERR_NEG_ENERGY: return "negative collision energy";
    case LEPIC_ERR_UNSUPPORTED: return "option not supported by the GPU path";
    case LEPIC_ERR_FEW_COLL: return "collision time step too small for electrons";
    case LEPIC_ERR_CUDA: return "CUDA runtime error";
    case LEPIC_ERR_ARG: return "invalid argument";
    case LEPIC_ERR_CELL: return "particle outside the grid";
    case LEPIC_ERR_NOT_CONVERGED: return "iteration cap reached";
    case LEPIC_ERR_SCRATCH_LIMIT: return "grid too large for the static scratch of the allocation-free solve";
    default: return "unknown status";
  }
}

const char *lepic_build_info(void) {
  static char buf[128];
  snprintf(buf, sizeof buf, "lepic_gpu sm_100a nvcc %d.%d (FP64 kernels without fmad)", __CUDACC_VER_MAJOR__,
           __CUDACC_VER_MINOR__);
  return buf;
}

namespace lepic {
namespace {
// one block: thread 0 waits on an mbarrier phase that nothing completes, at
// most limit_ns, then records LEPIC_ERR_TIMEOUT as a tile-copy wait does
__global__ void k_wait_selftest(unsigned long long limit_ns, int *err) {
  __shared__ __align__(8) unsigned long long bar;
  const uint32_t b = smem_addr(&bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0 && !mbar_wait_ns(b, 0u, limit_ns)) raise_err(err, LEPIC_ERR_TIMEOUT, 0);
}
}  // namespace
}  // namespace lepic

int lepic_dev_wait_selftest(long long limit_ns, void *stream) {
  if (limit_ns <= 0 || limit_ns > 2000000000LL) return LEPIC_ERR_ARG;
  lepic::k_wait_selftest<<<1, 32, 0, S(stream)>>>((unsigned long long)limit_ns, ctx().d_err);
  LEPIC_CUDA(cudaGetLastError());
  return LEPIC_OK;
}

int lepic_dev_check_async(void *stream, int *host) {
  if (!host) return LEPIC_ERR_ARG;
  Ctx &c = ctx();
  LEPIC_CUDA(cudaMemcpyAsync(host, c.d_err, 2 * sizeof(int), cudaMemcpyDeviceToHost, S(stream)));
  LEPIC_CUDA(cudaMemsetAsync(c.d_err, 0, 2 * sizeof(int), S(stream)));
  return LEPIC_OK;
}

int lepic_dev_check(void *stream, int *detail) {
  Ctx &c = ctx();
  const int rc = check_err(S(stream));
  if (detail) *detail = rc ? c.h_err[1] : 0;
  return rc;
}

int lepic_dev_info(int *sm_count, char *name, int name_len) {
  Ctx &c = ctx();
  if (sm_count) *sm_count = c.sms;
  if (name && name_len > 0) {
    strncpy(name, c.prop.name, (size_t)name_len - 1);
    name[name_len - 1] = 0;
  }
  return c.sms > 0 ? LEPIC_OK : LEPIC_ERR_CUDA;
}

// ------------------------------------------------------------ device API
int lepic_dev_calc_rho(const lepic_grid_t *g, double *np, double *rhs, int ntype,
                       const lepic_phys_t *P, void *stream) {
  if (!g || !P || ntype < 1 || ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  return launch_calc_rho(Dims(g->n), np, rhs, g->bcnd, ntype, *P, S(stream));
}

int lepic_dev_calc_efield(const lepic_grid_t *g, const double *phi, double *Ei, void *stream) {
  if (!g) return LEPIC_ERR_ARG;
  return launch_efield(Dims(g->n), g->h, phi, Ei, g->bcnd, S(stream));
}

int lepic_dev_pdesolver(const lepic_grid_t *g, double *u, const double *b, int ncycl, double eps,
                        double omega, int ng, const lepic_phys_t *P, int *k, double *ktot,
                        double *res, void *stream) {
  if (!g || !P) return LEPIC_ERR_ARG;
  return launch_pdesolver(Dims(g->n), g->h, u, b, g->bcnd, ncycl, eps, omega, ng, P->eps0, k, ktot,
                          res, S(stream), P->flag_pbc, P->flag_nmn);
}

int lepic_dev_part_mover(const lepic_grid_t *g, const double *Ei, lepic_species_f64_t *s, int ptype,
                         int ntype, int ngrid, const lepic_phys_t *P, double *p_mac,
                         double *P_loss, void *stream) {
  if (!g || !s || !P || ptype < 1 || ptype > ntype) return LEPIC_ERR_ARG;
  return launch_part_mover(*g, Ei, *s, ptype, ntype, ngrid, *P, p_mac, P_loss, S(stream));
}

int lepic_dev_charge_deposition(const lepic_grid_t *g, const lepic_species_f64_t *s, int ptype,
                                const lepic_phys_t *P, double *np, void *stream) {
  if (!g || !s || !P || ptype < 1) return LEPIC_ERR_ARG;
  return launch_deposit(*g, *s, ptype, *P, np, S(stream));
}

int lepic_dev_part_sorting(const lepic_grid_t *g, lepic_species_f64_t *s, int *Plist, int pl_max,
                           void *stream) {
  if (!g || !s || pl_max < 1) return LEPIC_ERR_ARG;
  return launch_sort(*g, *s, Plist, pl_max, S(stream));
}

int lepic_dev_collisions(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype,
                         const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                         unsigned long long call_index, double *nu_max, long long *counts,
                         void *stream) {
  if (!g || !sp || !T || !P || ntype < 1) return LEPIC_ERR_ARG;
  return launch_collisions(*g, sp, ntype, *T, *P, seed, call_index, nu_max, counts, S(stream));
}

int lepic_dev_collisions_targets(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype,
                                 const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                                 unsigned long long call_index, double *nu_max, long long *counts,
                                 lepic_targets_t *tg, void *stream) {
  if (!g || !sp || !T || !P || !tg || ntype < 1) return LEPIC_ERR_ARG;
  return launch_collisions(*g, sp, ntype, *T, *P, seed, call_index, nu_max, counts, S(stream), nullptr, tg);
}

int lepic_dev_load_uniform(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype,
                           long long n_per_species, const lepic_phys_t *P, unsigned long long seed,
                           void *stream) {
  if (!g || !sp || !P || ntype < 1 || ntype > LEPIC_NPART || n_per_species < 0) return LEPIC_ERR_ARG;
  return launch_load_uniform(*g, sp, ntype, n_per_species, *P, seed, S(stream));
}

int lepic_dev_dielectric_phi(const lepic_grid_t *g, double *phi, const lepic_phys_t *P, int ngrid, double Ca,
                             void *stream) {
  if (!g || !phi || !P || P->ntype < 1 || P->ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  return launch_dielectric_phi(Dims(g->n), phi, g->bcnd, *P, ngrid, Ca, S(stream));
}

int lepic_dev_cell_wall(const int *n, const int *bcnd, unsigned char *cell_wall, void *stream) {
  if (!n || !bcnd || !cell_wall) return LEPIC_ERR_ARG;
  return launch_cell_wall(Dims(n), bcnd, cell_wall, S(stream));
}

int lepic_dev_dens_red(const lepic_grid_t *g, const double *np, double *np_red, int ntype,
                       double *np_mx, void *stream) {
  if (!g || ntype < 1 || ntype > LEPIC_NPART) return LEPIC_ERR_ARG;
  return launch_dens_red(Dims(g->n), np, np_red, g->bcnd, ntype, np_mx, S(stream));
}

// ------------------------------------------------------------ drop-ins
// Every drop-in runs on the legacy default stream and leaves its status in
// the thread's error word.  Array arguments go through dev_view /
// acquire_species, so the same bodies serve the per-call copy mode and the
// residency mode.
void calc_rho_(const int *n, double *np, double *rhs_dom, const int *bcnd, const int *ntype,
               const int *nproc, const int *nproc_mpi, const int *mpi_rank) {
  (void)mpi_rank;
  if (*nproc != 1 || *nproc_mpi != 1) return record(LEPIC_ERR_UNSUPPORTED);
  cudaStream_t s = 0;
  Dims d(n);
  lepic_phys_t P = phys_from_common(*ntype);
  size_t nn = (size_t)d.cnt() * (size_t)*ntype;
  int rc = LEPIC_OK;
  // periodic stitching writes np
  double *np_d = dev_view("dropin_np", np, nn, P.flag_pbc ? UPDATE : READ, s, &rc);
  if (!np_d) return record(rc);
  const int *bc_d = dev_view("dropin_bcnd", bcnd, (size_t)d.cnt(), READ, s, &rc);
  if (!bc_d) return record(rc);
  double *rhs_d = dev_view("dropin_rhs", rhs_dom, (size_t)d.rcnt(), WRITE, s, &rc);
  if (!rhs_d) return record(rc);
  rc = launch_calc_rho(d, np_d, rhs_d, bc_d, *ntype, P, s);
  if (rc) return record(rc);
  rc = host_back(rhs_dom, rhs_d, (size_t)d.rcnt(), s);
  if (!rc && P.flag_pbc) rc = host_back(np, np_d, nn, s);
  record(rc);
  record(check_err(s));
}

void dens_red_(const int *n, const double *np, double *np_red, const int *bcnd, const int *ntype,
               const int *nproc, const int *nproc_mpi) {
  if (*nproc != 1 || *nproc_mpi != 1) return record(LEPIC_ERR_UNSUPPORTED);
  cudaStream_t s = 0;
  Dims d(n);
  size_t nn = (size_t)d.cnt() * (size_t)*ntype;
  int rc = LEPIC_OK;
  const double *np_d = dev_view("dropin_np", np, nn, READ, s, &rc);
  if (!np_d) return record(rc);
  const int *bc_d = dev_view("dropin_bcnd", bcnd, (size_t)d.cnt(), READ, s, &rc);
  if (!bc_d) return record(rc);
  double *red_d = dev_view("dropin_npred", np_red, nn, WRITE, s, &rc);
  if (!red_d) return record(rc);
  double mx[LEPIC_NPART] = {0};
  rc = launch_dens_red(d, np_d, red_d, bc_d, *ntype, mx, s);
  if (rc) return record(rc);
  record(host_back(np_red, red_d, nn, s));
  for (int p = 0; p < *ntype; ++p) part_info_dp_3_.np_mx[p] = mx[p];
  record(check_err(s));
}

void pdesolver_(double *u, const double *b, const int *bcnd, const double *h, const int *n,
                const int *ncycl, const double *eps, const double *omega, int *k, double *ktot,
                double *res, const int *ng, const int *rank, const int *nproc) {
  (void)rank;
  if (*nproc != 1) return record(LEPIC_ERR_UNSUPPORTED);
  cudaStream_t s = 0;
  Dims d(n);
  // u(0:n1+2,0:n2+2,-1:n3+2): skip the z = -1 ghost plane (MPI halo only)
  double *u0 = u + d.N1 * d.N2;
  int rc = LEPIC_OK;
  double *u_d = dev_view("dropin_u", u0, (size_t)d.cnt(), UPDATE, s, &rc);
  if (!u_d) return record(rc);
  const double *b_d = dev_view("dropin_b", b, (size_t)d.rcnt(), READ, s, &rc);
  if (!b_d) return record(rc);
  const int *bc_d = dev_view("dropin_bcnd", bcnd, (size_t)d.cnt(), READ, s, &rc);
  if (!bc_d) return record(rc);
  rc = launch_pdesolver(d, h, u_d, b_d, bc_d, *ncycl, *eps, *omega, *ng, constants_.eps0, k, ktot,
                        res, s, part_info_int_.flag_pbc, part_info_int_.flag_nmn);
  record(host_back(u0, u_d, (size_t)d.cnt(), s));
  record(rc);
  record(check_err(s));
}

void calc_efield_(const int *n, const double *h, const double *phi, double *Ei, const int *bcnd) {
  cudaStream_t s = 0;
  Dims d(n);
  int rc = LEPIC_OK;
  const double *phi_d = dev_view("dropin_u", phi, (size_t)d.cnt(), READ, s, &rc);
  if (!phi_d) return record(rc);
  // nodes the routine does not write keep the caller's values
  double *E_d = dev_view("dropin_E", Ei, 3 * (size_t)d.cnt(), UPDATE, s, &rc);
  if (!E_d) return record(rc);
  const int *bc_d = dev_view("dropin_bcnd", bcnd, (size_t)d.cnt(), READ, s, &rc);
  if (!bc_d) return record(rc);
  rc = launch_efield(d, h, phi_d, E_d, bc_d, s);
  if (rc) return record(rc);
  record(host_back(Ei, E_d, 3 * (size_t)d.cnt(), s));
  record(check_err(s));
}

void part_mover_(const int *n, const double *h, const double *Ei, const double *Bi, double *p_mac,
                 double *P_loss, double *vxp, const int *bcnd, const int *nmax, const int *ntype,
                 const int *ngrid, signed char *flag_dead, const int *nproc, int *np_tot,
                 const int *iproc, const int *ptype, int *flag_cex, int *cnt_cex, double *cnt_dead,
                 double *beam_div, double *sum_q_xz, double *sum_q_yz, const int *dtype,
                 int *iseed, const int *n_B, const double *h_B) {
  if (*nproc != 1 || *iproc != 1) return record(LEPIC_ERR_UNSUPPORTED);
  lepic_phys_t P = phys_from_common(*ntype);
  cudaStream_t s = 0;
  Dims d(n);
  lepic_grid_t g;
  int rc = stage_grid(g, n, h, bcnd, nullptr, s);
  if (rc) return record(rc);
  if (P.flag_B == 1) {
    // Bi(4,0:n_B(1)+2,0:n_B(2)+2,0:n_B(3)+2): Bi(1:3,1,1,1) is the uniform
    // field when n_B(1) = 1, else the whole array is the map
    const long long e1 = 4, e2 = 4LL * (n_B[0] + 3), e3 = 4LL * (n_B[0] + 3) * (n_B[1] + 3);
    if (n_B[0] == 1) {
      for (int c = 0; c < 3; ++c) P.Bconst[c] = Bi[c + e1 + e2 + e3];
    } else {
      const size_t nb = 4 * (size_t)(n_B[0] + 3) * (n_B[1] + 3) * (n_B[2] + 3);
      P.Bmap = dev_view("dropin_Bi", Bi, nb, READ, s, &rc);
      if (!P.Bmap) return record(rc);
      for (int c = 0; c < 3; ++c) {
        P.n_B[c] = n_B[c];
        P.h_B[c] = h_B[c];
      }
    }
  }
  const int p = *ptype - 1;
  double *vxp_p = vxp + 6LL * *nmax * p;
  signed char *fd_p = flag_dead + (long long)*nmax * p;
  const double *E_d = dev_view("dropin_E", Ei, 3 * (size_t)d.cnt(), READ, s, &rc);
  if (!E_d) return record(rc);
  // dielectric walls: the surface charges of this species' lost particles
  // (sum_q_xz(0:n1+2,0:n3+2,ntype,nproc), sum_q_yz(2,0:n2+2,0:n3+2,ntype,nproc))
  const bool die = part_info_int_.flag_die == 1 && dtype && sum_q_xz && sum_q_yz;
  const size_t nxz = (size_t)(n[0] + 3) * (n[2] + 3), nyz = 2 * (size_t)(n[1] + 3) * (n[2] + 3);
  const int *dt_d = nullptr;
  double *qxz_d = nullptr, *qyz_d = nullptr;
  if (die) {
    dt_d = upload("dropin_dtype", dtype, (size_t)*ngrid + 1, s);
    qxz_d = (double *)scratch("dropin_qxz", sizeof(double) * nxz);
    qyz_d = (double *)scratch("dropin_qyz", sizeof(double) * nyz);
    if (!dt_d || !qxz_d || !qyz_d) return record(LEPIC_ERR_CUDA);
    rc = cuda_ok(cudaMemsetAsync(qxz_d, 0, sizeof(double) * nxz, s), "memset");
    if (!rc) rc = cuda_ok(cudaMemsetAsync(qyz_d, 0, sizeof(double) * nyz, s), "memset");
    if (rc) return record(rc);
  }
  // negative ions (this species is tag_neg): flag_cex(1:nmax) follows the
  // particles; cnt_cex(3), cnt_dead(1), beam_div(4) accumulate
  // (Src/part_expmover.f90:76, 278-301, 416-470)
  MoverExtras ex;
  memset(&ex, 0, sizeof(ex));
  ex.tag_neg = part_info_int_.tag_neg;
  ex.tag_neu = part_info_int_.tag_neu;
  ex.num_grd = part_info_int_.num_grd;
  const bool neg = ex.tag_neg == *ptype;
  double *xacc = nullptr;   // cnt_dead, beam_div(4), P_loss(4,1)
  int *xcnt = nullptr;      // cnt_cex(3)
  if (neg) {
    if (!flag_cex || !cnt_cex || !cnt_dead || !beam_div) return record(LEPIC_ERR_ARG);
    ex.cex = upload("dropin_cex", flag_cex, (size_t)*nmax, s);
    ex.cex_out = (int *)scratch("dropin_cex_out", sizeof(int) * (size_t)*nmax);
    if (!ex.cex || !ex.cex_out) return record(LEPIC_ERR_CUDA);
  }
  // secondary emission from positive ions on the emissive grid, appended to
  // the electrons (species 1) (Src/part_expmover.f90:353-400)
  const bool sec = part_info_dp_1_.gam_sec > 0.0 && P.charge[p] > 0.0;
  if (neg || sec) {
    xacc = (double *)scratch("dropin_xacc", sizeof(double) * 6);
    xcnt = (int *)scratch("dropin_xcnt", sizeof(int) * 3);
    if (!xacc || !xcnt) return record(LEPIC_ERR_CUDA);
    rc = cuda_ok(cudaMemsetAsync(xacc, 0, sizeof(double) * 6, s), "memset");
    if (!rc) rc = cuda_ok(cudaMemsetAsync(xcnt, 0, sizeof(int) * 3, s), "memset");
    if (rc) return record(rc);
    ex.cnt_dead = xacc;
    ex.beam_div = xacc + 1;
    ex.ploss4 = xacc + 5;
    ex.cnt_cex = xcnt;
  }
  SpeciesView v1;
  if (sec) {
    if (!iseed) return record(LEPIC_ERR_ARG);
    ex.gam_sec = part_info_dp_1_.gam_sec;
    ex.THm = part_info_dp_1_.THm;
    ex.zg_sec[0] = part_info_dp_1_.zg_sec[0];
    ex.zg_sec[1] = part_info_dp_1_.zg_sec[1];
    ex.igrid_sec = part_info_int_.igrid_sec;
    // the draws are keyed by the caller's ran2 seed, which then advances one
    // ran2 step so that the next call draws differently
    ex.key0 = (uint32_t)*iseed;
    ex.key1 = 0x4C455049u;
    ex.call = (uint32_t)*ptype;
    {
      const int ia = 16807, im = 2147483647, iq = 127773, ir = 2836;
      const int k = *iseed / iq;
      *iseed = ia * (*iseed - k * iq) - ir * k;
      if (*iseed < 0) *iseed += im;
    }
    if (p == 0) return record(LEPIC_ERR_ARG);
    rc = acquire_species(v1, vxp, np_tot[0], *nmax, 1, nullptr, s);
    if (rc) return record(rc);
    ex.e1 = &v1.s;
  }
  SpeciesView v;
  rc = acquire_species(v, vxp_p, np_tot[p], *nmax, 0, fd_p, s);
  if (rc) return record(rc);
  rc = launch_part_mover(g, E_d, v.s, *ptype, *ntype, *ngrid, P, p_mac, P_loss, s, dt_d, qxz_d, qyz_d,
                         (neg || sec) ? &ex : nullptr);
  record(rc);
  record(release_species(v, &np_tot[p], fd_p, *nmax, true, s));
  if (sec) record(release_species(v1, &np_tot[0], nullptr, *nmax, true, s));
  if ((neg || sec) && !rc) {
    double hx[6];
    int hc[3];
    rc = cuda_ok(cudaMemcpyAsync(hx, xacc, sizeof(hx), cudaMemcpyDeviceToHost, s), "copy");
    if (!rc) rc = cuda_ok(cudaMemcpyAsync(hc, xcnt, sizeof(hc), cudaMemcpyDeviceToHost, s), "copy");
    if (!rc && neg)
      rc = cuda_ok(cudaMemcpyAsync(flag_cex, ex.cex_out, sizeof(int) * (size_t)np_tot[p], cudaMemcpyDeviceToHost, s),
                   "copy");
    if (!rc) rc = cuda_ok(cudaStreamSynchronize(s), "sync");
    record(rc);
    if (!rc && neg) {
      *cnt_dead += hx[0];
      for (int a = 0; a < 4; ++a) beam_div[a] += hx[1 + a];
      for (int a = 0; a < 3; ++a) cnt_cex[a] += hc[a];
    }
    if (!rc && sec && P_loss) P_loss[3] += hx[5];
  }
  if (die && !rc) {
    std::vector<double> hxz(nxz), hyz(nyz);
    rc = cuda_ok(cudaMemcpyAsync(hxz.data(), qxz_d, sizeof(double) * nxz, cudaMemcpyDeviceToHost, s), "copy");
    if (!rc) rc = cuda_ok(cudaMemcpyAsync(hyz.data(), qyz_d, sizeof(double) * nyz, cudaMemcpyDeviceToHost, s), "copy");
    if (!rc) rc = cuda_ok(cudaStreamSynchronize(s), "sync");
    record(rc);
    if (!rc) {
      for (size_t q = 0; q < nxz; ++q) sum_q_xz[q + nxz * p] += hxz[q];
      for (size_t q = 0; q < nyz; ++q) sum_q_yz[q + nyz * p] += hyz[q];
    }
  }
}

void charge_deposition_(const int *n, const double *h, const double *vxp, const int *nmax,
                        const int *ntype, const double *kq, double *np, const int *nproc,
                        const int *np_tot, double *sum_dEk, int *Nh, const int *iproc,
                        const int *ptype) {
  if (*nproc != 1 || *iproc != 1) return record(LEPIC_ERR_UNSUPPORTED);
  cudaStream_t s = 0;
  Dims d(n);
  lepic_phys_t P = phys_from_common(*ntype);
  lepic_grid_t g;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = n[a];
    g.h[a] = h[a];
  }
  g.bcnd = nullptr;
  g.cell_wall = nullptr;
  int rc = LEPIC_OK;
  g.kq = dev_view("dropin_kq", kq, (size_t)d.cnt(), READ, s, &rc);
  if (!g.kq) return record(rc);
  const int p = *ptype - 1;
  double *np_slice = np + (long long)d.cnt() * p;
  double *np_d = dev_view("dropin_npdep", np_slice, (size_t)d.cnt(), UPDATE, s, &rc);
  if (!np_d) return record(rc);
  SpeciesView v;
  // the routine reads the particles only
  rc = acquire_species(v, const_cast<double *>(vxp) + 6LL * *nmax * p, np_tot[p], *nmax, 0, nullptr, s);
  if (rc) return record(rc);
  rc = launch_deposit(g, v.s, *ptype, P, np_d, s);
  record(rc);
  // heating-region statistics of the electrons (Src/part_expmover.f90:658-681)
  double hs[2] = {0.0, 0.0};
  if (!rc && *ptype == 1 && part_info_dp_2_.Pabs > 0.0 && sum_dEk && Nh) {
    const lepic_heat_t H = heat_from_common();
    double *st = (double *)scratch("dropin_heat_stats", 2 * sizeof(double));
    rc = st ? LEPIC_OK : LEPIC_ERR_CUDA;
    if (!rc) rc = cuda_ok(cudaMemsetAsync(st, 0, 2 * sizeof(double), s), "memset");
    if (!rc) rc = launch_heat_stats(g, &v.s, nullptr, P, H, st, s);
    if (!rc) rc = cuda_ok(cudaMemcpyAsync(hs, st, sizeof(hs), cudaMemcpyDeviceToHost, s), "copy");
    record(rc);
  }
  record(release_species(v, nullptr, nullptr, *nmax, false, s));
  if (rc) return;
  record(host_back(np_slice, np_d, (size_t)d.cnt(), s));
  record(check_err(s));
  if (*ptype == 1 && part_info_dp_2_.Pabs > 0.0 && sum_dEk && Nh) {
    sum_dEk[*iproc - 1] += hs[0];
    Nh[*iproc - 1] += (int)hs[1];
  }
}

void part_injection_(const int *n, const double *h, const int *bcnd, double *vxp, int *sour_xy, int *sour_xz,
                     int *sour_yz, const int *ntype, const int *nmax, const double *I_inj, const double *xl_pow,
                     const double *xr_pow, const double *yl_pow, const double *yr_pow, const double *zl_pow,
                     const double *zr_pow, int *np_tot, const int *nproc, int *iseed, const int *nproc_mpi,
                     int *N_inj, const int *iproc, double *P_loss, const double *phi, const double *ni0) {
  (void)sour_xy;
  (void)sour_xz;
  (void)sour_yz;
  if (*nproc != 1 || *iproc != 1 || *nproc_mpi != 1) return record(LEPIC_ERR_UNSUPPORTED);
  const int nt = *ntype;
  if (nt < 1 || nt > LEPIC_NPART) return record(LEPIC_ERR_ARG);
  static unsigned long long calls = 0;
  lepic_phys_t P = phys_from_common(nt);
  lepic_inject_t I;
  memset(&I, 0, sizeof(I));
  I.opt_inj = part_info_int_.opt_inj;
  I.ns_inj = part_info_int_.ns_inj > 0 ? part_info_int_.ns_inj : 1;
  I.n_cath = part_info_int_.n_cath;
  I.dir_sec = part_info_int_.dir_sec;
  I.tag_beam = part_info_int_.tag_beam;
  I.flag_pbcz = part_info_int_.flag_pbcz;
  I.I_inj = *I_inj;
  I.xl = *xl_pow;
  I.xr = *xr_pow;
  I.yl = *yl_pow;
  I.yr = *yr_pow;
  I.zl = *zl_pow;
  I.zr = *zr_pow;
  I.THm = part_info_dp_1_.THm;
  I.zg_sec[0] = part_info_dp_1_.zg_sec[0];
  I.zg_sec[1] = part_info_dp_1_.zg_sec[1];
  for (int p = 0; p < nt; ++p) I.ni0[p] = ni0[p];
  cudaStream_t s = 0;
  Dims d(n);
  lepic_grid_t g;
  int rc = stage_grid(g, n, h, bcnd, nullptr, s);
  if (rc) return record(rc);
  const double *phi_d = dev_view("dropin_u", phi, (size_t)d.cnt(), READ, s, &rc);
  if (!phi_d) return record(rc);
  SpeciesView v[LEPIC_NPART];
  lepic_species_f64_t sp[LEPIC_NPART];
  for (int p = 0; p < nt; ++p) {
    rc = acquire_species(v[p], vxp + 6LL * *nmax * p, np_tot[p], *nmax, p, nullptr, s);
    if (rc) return record(rc);
    sp[p] = v[p].s;
  }
  // opt_inj 2: as many events as ions were lost to the walls (N_inj(2,iproc))
  const long long nev = (I.opt_inj == 2 || I.opt_inj == -2) ? (nt > 1 ? N_inj[1] : 0) : -1;
  double pl4[LEPIC_NPART] = {0};
  rc = launch_inject(g, sp, nullptr, nt, P, I, nev, (unsigned long long)(unsigned)iseed[0], calls++, nullptr, phi_d,
                     pl4, nullptr, s);
  record(rc);
  for (int p = 0; p < nt; ++p) {
    v[p].s = sp[p];
    record(release_species(v[p], &np_tot[p], nullptr, *nmax, true, s));
  }
  if (P_loss)
    for (int p = 0; p < nt; ++p) P_loss[3 + 4 * p] += pl4[p];  // P_loss(4, p, 1)
}

void eheating_(const double *h, double *vxp, const int *nmax, const int *ntype, const int *nproc, int *iseed,
               const int *np_tot, const double *vt, const int *iproc, double *P_loss) {
  if (*nproc != 1 || *iproc != 1) return record(LEPIC_ERR_UNSUPPORTED);
  static unsigned long long calls = 0;
  lepic_phys_t P = phys_from_common(*ntype);
  const lepic_heat_t H = heat_from_common();
  cudaStream_t s = 0;
  lepic_grid_t g;
  memset(&g, 0, sizeof(g));
  for (int a = 0; a < 3; ++a) g.h[a] = h[a];
  double *acc = (double *)scratch("dropin_heat_acc", 3 * sizeof(double));
  if (!acc) return record(LEPIC_ERR_CUDA);
  int rc = cuda_ok(cudaMemsetAsync(acc, 0, 3 * sizeof(double), s), "memset");
  if (rc) return record(rc);
  SpeciesView v;
  rc = acquire_species(v, vxp, np_tot[0], *nmax, 0, nullptr, s);
  if (rc) return record(rc);
  rc = launch_eheating(g, &v.s, nullptr, P, H, *vt, nullptr, (unsigned long long)(unsigned)*iseed, calls++, acc, s);
  record(rc);
  double ha[3] = {0.0, 0.0, 0.0};
  if (!rc) record(cuda_ok(cudaMemcpyAsync(ha, acc, sizeof(ha), cudaMemcpyDeviceToHost, s), "copy"));
  int np1 = np_tot[0];
  record(release_species(v, &np1, nullptr, *nmax, rc == LEPIC_OK, s));
  record(check_err(s));
  if (P_loss) P_loss[1] += ha[0];  // P_loss(2, 1, 1)
}

void part_sorting_(double *vxp, double *sorting, const int *nmax, const int *ntype, const int *n,
                   const double *h, int *Plist_thd, const int *pl_max, const int *nproc,
                   const int *np_tot, const int *ptype) {
  (void)sorting;
  (void)ntype;
  if (*nproc != 1) return record(LEPIC_ERR_UNSUPPORTED);
  cudaStream_t s = 0;
  lepic_grid_t g;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = n[a];
    g.h[a] = h[a];
  }
  g.bcnd = nullptr;
  g.kq = nullptr;
  g.cell_wall = nullptr;
  const int p = *ptype - 1;
  const size_t npl = (size_t)(*pl_max + 1);
  int *pl_h = Plist_thd + (long long)npl * p;
  int rc = LEPIC_OK;
  int *pl_d = dev_view("dropin_plist", pl_h, npl, WRITE, s, &rc);
  if (!pl_d) return record(rc);
  SpeciesView v;
  rc = acquire_species(v, vxp + 6LL * *nmax * p, np_tot[p], *nmax, 0, nullptr, s);
  if (rc) return record(rc);
  rc = launch_sort(g, v.s, pl_d, *pl_max, s);
  record(rc);
  int np_out = 0;
  record(release_species(v, &np_out, nullptr, *nmax, true, s));
  if (rc) return;
  record(host_back(pl_h, pl_d, npl, s));
  record(check_err(s));
}

void collisions_(const int *it, double *vxp, const int *n, const double *h, const int *ntype,
                 const int *nmax, const double *sig, const double *sig_Er, const int *sig_list,
                 const double *sig_Eex, const int *ncol_mx, const int *npt_mx, double *cnt_col,
                 double *P_loss, int *sour_xy, int *sour_xz, const int *Plist, const int *pl_max,
                 const double *sigv_mx, const int *col_info, const double *np_red,
                 signed char *flag_dead, int *flag_cex, const int *nproc, int *np_tot, int *iseed,
                 const int *nproc_mpi, const int *mpi_rank, double *ss2D_xy, double *ss2D_xz,
                 double *ss2D_yz, const int *flag_diag) {
  (void)flag_cex;
  (void)mpi_rank;
  (void)ss2D_xy;
  (void)ss2D_xz;
  (void)ss2D_yz;
  // flag_diag = 1 turns the routine into a diagnostic pass over every
  // particle (the source maps ss2D_*, no collision): not built here
  if (*nproc != 1 || *nproc_mpi != 1 || *flag_diag != 0) return record(LEPIC_ERR_UNSUPPORTED);
  const int nt = *ntype;
  if (nt < 1 || nt > LEPIC_NPART) return record(LEPIC_ERR_ARG);
  cudaStream_t s = 0;
  Dims d(n);
  lepic_phys_t P = phys_from_common(nt);
  lepic_grid_t g;
  for (int a = 0; a < 3; ++a) {
    g.n[a] = n[a];
    g.h[a] = h[a];
  }
  g.bcnd = nullptr;
  g.kq = nullptr;
  g.cell_wall = nullptr;
  const int ncol = part_info_int_.ncol;
  if (ncol <= 0) return;
  // tables (ordering output, reference layouts)
  lepic_tables_t T;
  memset(&T, 0, sizeof(T));
  T.ncol = ncol;
  T.npt = part_info_int_.sig_npt_mx;
  T.npt_mx = *npt_mx;
  int rc = LEPIC_OK;
  T.sig_Er = dev_view("dropin_sigEr", sig_Er, (size_t)*npt_mx, READ, s, &rc);
  if (!T.sig_Er) return record(rc);
  T.sig = dev_view("dropin_sig", sig, (size_t)*npt_mx * *ncol_mx, READ, s, &rc);
  if (!T.sig) return record(rc);
  T.sig_Eth = dev_view("dropin_sigEth", sig_Eex, (size_t)*ncol_mx, READ, s, &rc);  // sig_Eex(:,ind_Eth)
  if (!T.sig_Eth) return record(rc);
  std::vector<int> ci((size_t)ncol * 10);
  for (int c = 0; c < ncol; ++c)
    for (int q = 0; q < 10; ++q) ci[c + (size_t)ncol * q] = col_info[c + (size_t)*ncol_mx * q];
  T.col_info_h = ci.data();
  std::vector<int> sl((size_t)LEPIC_NPART * ncol);
  std::vector<double> sv((size_t)LEPIC_NPART * ncol);
  for (int c = 0; c < ncol; ++c)
    for (int q = 0; q < LEPIC_NPART; ++q) {
      sl[q + LEPIC_NPART * (size_t)c] = sig_list[q + LEPIC_NPART * (size_t)c];
      sv[q + LEPIC_NPART * (size_t)c] = sigv_mx[q + LEPIC_NPART * (size_t)c];
    }
  T.sig_list = sl.data();
  T.sigv_mx = sv.data();
  T.p_ncol = part_info_int_.p_ncol;
  // region counters (Src/collisions.f90:153-157, 1005-1013)
  RegionCount rgc;
  memset(&rgc, 0, sizeof(rgc));
  rgc.n_rg = part_info_int_.n_rg;
  rgc.ncol_mx = *ncol_mx;
  for (int q = 0; q < LEPIC_NM_RG; ++q) {
    rgc.ixl[q] = part_info_int_.ixl_rg[q];
    rgc.ixr[q] = part_info_int_.ixr_rg[q];
  }
  rgc.iyl = part_info_int_.iyl_rg;
  rgc.iyr = part_info_int_.iyr_rg;
  rgc.izl = part_info_int_.izl_rg;
  rgc.izr = part_info_int_.izr_rg;
  if (rgc.n_rg > 0) {
    // the region populations read np_red on the host
    rc = mirror_to_host(np_red, sizeof(double) * (size_t)d.cnt() * nt, s);
    if (rc) return record(rc);
  }
  for (int p = 0; p < nt; ++p) {
    double kk = h[0] * h[1] * h[2] / part_info_dp_2_.Nm[p];
    for (int q = 0; q < rgc.n_rg && q < LEPIC_NM_RG; ++q) {
      double sum = 0.0;
      for (int iz = rgc.izl; iz <= rgc.izr; ++iz)
        for (int iy = rgc.iyl; iy <= rgc.iyr; ++iy)
          for (int ix = rgc.ixl[q]; ix <= rgc.ixr[q]; ++ix) sum += np_red[d.g(ix, iy, iz) + d.cnt() * p];
      int np_rg = (int)(kk * sum);
      rgc.w[p][q] = np_rg != 0 ? 1.0 / np_rg : 0.0;
    }
  }
  size_t ncc = (size_t)*ncol_mx * (size_t)(rgc.n_rg > 0 ? rgc.n_rg : 1);
  std::vector<double> cc_h(ncc, 0.0);
  for (int q = 0; q < rgc.n_rg; ++q)
    for (int c = 0; c < *ncol_mx; ++c)
      cc_h[c + (size_t)*ncol_mx * q] = cnt_col[c + (size_t)*ncol_mx * (size_t)(*nproc) * q];
  rgc.cnt_col_dev = upload("dropin_cntcol", cc_h.data(), ncc, s);
  if (!rgc.cnt_col_dev) return record(LEPIC_ERR_CUDA);
  // P_loss(3, :, 1) and the source planes sour_xy / sour_xz of the created
  // particles (Src/collisions.f90:862-869, 894-902, 982-990)
  const size_t nsxy = (size_t)(n[0] + 3) * (n[1] + 3) * nt, nsxz = (size_t)(n[0] + 3) * (n[2] + 3) * nt;
  rgc.ploss3_dev = (double *)scratch("dropin_ploss3", sizeof(double) * LEPIC_NPART);
  if (!rgc.ploss3_dev) return record(LEPIC_ERR_CUDA);
  rc = cuda_ok(cudaMemsetAsync(rgc.ploss3_dev, 0, sizeof(double) * LEPIC_NPART, s), "memset");
  if (rc) return record(rc);
  if (sour_xy && sour_xz) {
    rgc.sour_xy_dev = dev_view("dropin_sourxy", sour_xy, nsxy, UPDATE, s, &rc);
    if (!rgc.sour_xy_dev) return record(rc);
    rgc.sour_xz_dev = dev_view("dropin_sourxz", sour_xz, nsxz, UPDATE, s, &rc);
    if (!rgc.sour_xz_dev) return record(rc);
  }
  rgc.iz_pl = part_info_int_.iz_pl;
  rgc.iy_pl = n[1] / 2 + 1;
  SpeciesView v[LEPIC_NPART];
  lepic_species_f64_t sp[LEPIC_NPART];
  for (int p = 0; p < nt; ++p) {
    rc = acquire_species(v[p], vxp + 6LL * *nmax * p, np_tot[p], *nmax, p,
                         flag_dead + (long long)*nmax * p, s);
    if (rc) return record(rc);
    sp[p] = v[p].s;
  }
  // charged targets (DSMC): the per-cell offsets Plist(0:pl_max,ntype) of the
  // last part_sorting and the densities np_red of dens_red
  lepic_targets_t tg;
  memset(&tg, 0, sizeof(tg));
  bool charged = false;
  for (int c = 0; c < ncol; ++c) {
    const int n_re = ci[c];
    const int tt = ci[c + (size_t)ncol * (2 + n_re - 1)];
    if (tt >= 1 && tt <= nt && P.charge[tt - 1] != 0.0) charged = true;
  }
  if (charged) {
    // Plist must cover every cell index of the grid
    if ((long long)*pl_max < (long long)n[0] * n[1] * n[2]) return record(LEPIC_ERR_ARG);
    const int *pl_d = dev_view("dropin_plist", Plist, (size_t)(*pl_max + 1) * nt, READ, s, &rc);
    if (!pl_d) return record(rc);
    const double *nr_d = dev_view("dropin_npred", np_red, (size_t)d.cnt() * nt, READ, s, &rc);
    if (!nr_d) return record(rc);
    for (int p = 0; p < nt; ++p) {
      tg.cell_off[p] = pl_d + (size_t)(*pl_max + 1) * p;
      tg.np[p] = nr_d + (size_t)d.cnt() * p;
    }
  }
  double nu_max[LEPIC_NPART] = {0};
  long long counts[64] = {0};
  unsigned long long seed = (unsigned long long)(unsigned)iseed[0];
  rc = launch_collisions(g, sp, nt, T, P, seed, (unsigned long long)*it, nu_max, counts, s, &rgc, &tg);
  for (int p = 0; p < nt; ++p) {
    v[p].s = sp[p];
    record(release_species(v[p], &np_tot[p], flag_dead + (long long)*nmax * p, *nmax, true, s));
  }
  if (rgc.n_rg > 0) {
    record(mirror_d2h(cc_h.data(), rgc.cnt_col_dev, sizeof(double) * ncc, s));
    if (cudaStreamSynchronize(s) != cudaSuccess) record(LEPIC_ERR_CUDA);
    for (int q = 0; q < rgc.n_rg; ++q)
      for (int c = 0; c < *ncol_mx; ++c)
        cnt_col[c + (size_t)*ncol_mx * (size_t)(*nproc) * q] = cc_h[c + (size_t)*ncol_mx * q];
  }
  if (rgc.sour_xy_dev) {
    record(host_back(sour_xy, rgc.sour_xy_dev, nsxy, s));
    record(host_back(sour_xz, rgc.sour_xz_dev, nsxz, s));
  }
  double pl3[LEPIC_NPART] = {0};
  record(mirror_d2h(pl3, rgc.ploss3_dev, sizeof(pl3), s));
  if (cudaStreamSynchronize(s) != cudaSuccess) record(LEPIC_ERR_CUDA);
  if (P_loss)
    for (int p = 0; p < nt; ++p) P_loss[2 + 4 * p] += pl3[p];  // P_loss(3, p, 1)
  for (int p = 0; p < nt; ++p) part_info_dp_3_.nu_max[p] = nu_max[p];
  record(rc);
}

}  // extern "C"
