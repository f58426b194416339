/*
 * lepic_gpu.h -- C ABI of the B200 (sm_100a) PIC-MCC hot path.
 *
 * Two layers, both plain C (pointers and sizes only, no CUDA or torch types):
 *
 * 1. Drop-in replacements for the legacy Fortran routines of the reference.
 *    The names carry the trailing underscore of gfortran/ifx external
 *    symbols and every argument is a pointer, so a Fortran build that links
 *    this library in place of the original objects calls them unchanged
 *    (the routines are external subroutines with implicit interfaces).
 *    Arrays are the Fortran host arrays (column-major, reference index
 *    bases); each call copies its inputs to the GPU, runs the kernels and
 *    copies its outputs back, or, with residency on (lepic_gpu_set_residency),
 *    works on device mirrors of the arrays that persist between calls.
 *    Physics constants are read from the Fortran
 *    COMMON blocks declared below, exactly as the Fortran routines read them.
 *    Contract: OMP_NUM_THREADS=1 (nproc = 1) and one MPI rank.
 *
 * 2. A device API (lepic_dev_*) on device pointers and a CUDA stream handle
 *    (passed as void*), used by the host step loop and the PyTorch binding.
 *
 * Errors: every entry point returns / records an int status (0 = OK, codes
 * below).  The drop-ins cannot return a value to Fortran, so they record it;
 * lepic_gpu_last_error() reads and clears it.  GPU kernels never trap: they
 * set a device error word that the host turns into these codes.
 */
#ifndef LEPIC_GPU_H
#define LEPIC_GPU_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LEPIC_NPART 10
#define LEPIC_NM_RG 5

/* status codes (shared with the CPU oracle) */
#define LEPIC_OK 0
#define LEPIC_ERR_CAPACITY 1      /* particle array full (reference: nmax)        */
#define LEPIC_ERR_DIVERGED 2      /* Poisson residual grew > 10x (pdesolver)      */
#define LEPIC_ERR_PMAX 3          /* null-collision probability > 1               */
#define LEPIC_ERR_EKR_TABLE 4     /* collision energy above the sigma table       */
#define LEPIC_ERR_NEG_ENERGY 5    /* negative CM energy after threshold           */
#define LEPIC_ERR_UNSUPPORTED 6   /* option outside the GPU path (dielectrics...) */
#define LEPIC_ERR_FEW_COLL 7      /* collision time step too small for electrons  */
#define LEPIC_ERR_CUDA 20         /* CUDA runtime error                          */
#define LEPIC_ERR_ARG 21          /* invalid argument / size                     */
#define LEPIC_ERR_CELL 22         /* particle outside the grid (device check)    */
#define LEPIC_ERR_NOT_CONVERGED 23 /* iteration cap reached                      */
#define LEPIC_ERR_SCRATCH_LIMIT 24 /* grid too large for the static scratch of
                                      lepic_dev_pdesolver_noalloc               */
#define LEPIC_ERR_TIMEOUT 25       /* a bounded device wait ran out (a tile copy
                                      that never completed)                     */

/* ------------------------------------------------------------------------ */
/* Fortran COMMON blocks of Src/particle_info.h:53-70 and Src/constants.h,   */
/* member for member.  The library defines them as weak symbols; when linked */
/* into the Fortran program its COMMON storage takes precedence.             */
/* ------------------------------------------------------------------------ */
typedef struct {
  int np_cell, ncol, sig_npt_mx, flag_pdf, n_cell, nbak, flag_restart, ixl_pow, ixr_pow, flag_B,
      ns_heat, ns_coll, p_ncol[LEPIC_NPART], nscol, p_nscol[LEPIC_NPART], n_rg, flag_pbc, n_holes,
      flag_grd, ind_g, nB, cnt_seg, tag_neg, cnt_neg, tag_neu, flag_nmn, num_grd, ptype_pdf, ns_flx,
      nhy, nhz, ixl_rg[LEPIC_NM_RG], ns_inj, ixr_rg[LEPIC_NM_RG], iyl_rg, iyr_rg, izl_rg, izr_rg,
      flag_heat, flag_inj, opt_inj, flag_B_pos, ixg, ix_PE, omp_rank_max, mpi_rank_max, flag_die,
      flag_thr, ix_pl, iz_pl, ix_thr, flag_convP, ig_die[5], flag_pbcz, tag_beam, every, cnt_plt,
      flag_bak, igrid_sec, dir_sec, n_cath, flag_circxh, flag_ahp, flag_gridB, plt_src, flag_RFpot;
} lepic_part_info_int_t;

typedef struct {
  double charge[LEPIC_NPART], mass[LEPIC_NPART], Ti[LEPIC_NPART], vt0[LEPIC_NPART], k_eps0,
      B_scale[5], B0[5], dL[5], x0[5], y0[5], z0[5], jne, RNeta, THm, x_thr, y_thr, tseq,
      tseq_init, tseq_final, gam_sec, zg_sec[2];
} lepic_part_info_dp_1_t;

typedef struct {
  double Pabs, n0, ngas, Nm[LEPIC_NPART], dt, xmax, ymax, zmax, x_load, nu_h, Lgy, Lgz, Sg, Lhy,
      Lhz, xg1, Bmax, nudt, R_ahp;
} lepic_part_info_dp_2_t;

typedef struct {
  double np_mx[LEPIC_NPART], nu_max[LEPIC_NPART], nu_uplim[LEPIC_NPART];
} lepic_part_info_dp_3_t;

typedef struct {
  double qe, eps0, c, pi, amu;
} lepic_constants_t;

extern lepic_part_info_int_t part_info_int_;
extern lepic_part_info_dp_1_t part_info_dp_1_;
extern lepic_part_info_dp_2_t part_info_dp_2_;
extern lepic_part_info_dp_3_t part_info_dp_3_;
extern lepic_constants_t constants_;

/* ------------------------------------------------------------------------ */
/* Drop-in routines (layer 1).  Each cites the reference routine it replaces. */
/* ------------------------------------------------------------------------ */

/* Src/calc_rho.f90:1 -- rhs_dom = -sum_species charge*np (+ periodic
 * stitching of np).  np(0:n1+2,0:n2+2,0:n3+2,ntype,nproc),
 * rhs_dom(0:n1+1,0:n2+1,0:n3+1), bcnd(0:n1+2,0:n2+2,0:n3+2). */
void calc_rho_(const int *n, double *np, double *rhs_dom, const int *bcnd, const int *ntype,
               const int *nproc, const int *nproc_mpi, const int *mpi_rank);

/* Src/calc_rho.f90:116 -- np_red = sum over threads, np_mx = max over plasma
 * nodes (written to COMMON /part_info_dp_3/ np_mx). */
void dens_red_(const int *n, const double *np, double *np_red, const int *bcnd, const int *ntype,
               const int *nproc, const int *nproc_mpi);

/* Src/pdesolver.f90:1 -- multigrid V-cycles with red-black SOR smoothing
 * until res/alpha < eps.  u(0:n1+2,0:n2+2,-1:n3+2) (warm start, Dirichlet
 * values on walls), b(0:n1+1,0:n2+1,0:n3+1) = -rho. */
void pdesolver_(double *u, const double *b, const int *bcnd, const double *h, const int *n,
                const int *ncycl, const double *eps, const double *omega, int *k, double *ktot,
                double *res, const int *ng, const int *rank, const int *nproc);

/* Src/Efield.f90:1 -- E = -grad(phi) with wall extrapolation.
 * phi(0:n1+2,0:n2+2,0:n3+2), Ei(3,0:n1+2,0:n2+2,0:n3+2). */
void calc_efield_(const int *n, const double *h, const double *phi, double *Ei, const int *bcnd);

/* Src/part_expmover.f90:1 as called at Src/main.f90:1250-1252 (26
 * arguments) -- trilinear gather, Boris (uniform B with n_B(1) = 1, else the
 * B-field map Bi(4,0:n_B(1)+2,...) of spacing h_B) or leapfrog, position
 * update, loss test and in-order compaction of species ptype.  With
 * flag_die = 1 in COMMON /part_info_int/ the charge of the particles lost
 * on dielectric walls (dtype(igrid) = 2: Y = const plane, 3 / 4: X = const
 * planes) is added to sum_q_xz(0:n1+2,0:n3+2,ntype,nproc) and
 * sum_q_yz(2,0:n2+2,0:n3+2,ntype,nproc) (Src/part_expmover.f90:302-348).
 * For ptype = tag_neg (COMMON /part_info_int/) the negative-ion bookkeeping
 * (Src/part_expmover.f90:76, 278-301, 416-470): flag_cex(1:nmax) follows the
 * compaction, a negative ion reaching x < 0 with flag_nmn = 1 is lost at
 * label 0, cnt_dead += Nm q per killed particle, and a particle lost on
 * num_grd counts in cnt_cex(1:3) and adds its divergence angles to
 * beam_div(1:4).  With gam_sec > 0 a positive species lost on igrid_sec emits
 * secondary electrons into species 1 (vxp(:,np_tot(1)+1:,1), P_loss(4,1);
 * Src/part_expmover.f90:353-400); the draws come from Philox keyed by *iseed,
 * which then advances one ran2 step, not from the reference's ran2 stream. */
void part_mover_(const int *n, const double *h, const double *Ei, const double *Bi, double *p_mac,
                 double *P_loss, double *vxp, const int *bcnd, const int *nmax, const int *ntype,
                 const int *ngrid, signed char *flag_dead, const int *nproc, int *np_tot,
                 const int *iproc, const int *ptype, int *flag_cex, int *cnt_cex, double *cnt_dead,
                 double *beam_div, double *sum_q_xz, double *sum_q_yz, const int *dtype,
                 int *iseed, const int *n_B, const double *h_B);

/* Src/part_expmover.f90:570 -- CIC deposition with kq into np(..,ptype,iproc);
 * for ptype 1 with Pabs > 0 also the heating-region statistics:
 * sum_dEk(iproc) += kinetic energy and Nh(iproc) += number of the electrons
 * in the heating region (Src/part_expmover.f90:658-681). */
void charge_deposition_(const int *n, const double *h, const double *vxp, const int *nmax,
                        const int *ntype, const double *kq, double *np, const int *nproc,
                        const int *np_tot, double *sum_dEk, int *Nh, const int *iproc,
                        const int *ptype);

/* Src/sorting.f90:97 -- counting sort of species ptype by cell.  Plist_thd
 * (0:pl_max,ntype,nproc) receives the inclusive end offset of every cell.
 * Within one cell the order is unspecified (the reference's OpenMP atomic
 * capture scatter is not stable either). */
void part_sorting_(double *vxp, double *sorting, const int *nmax, const int *ntype, const int *n,
                   const double *h, int *Plist_thd, const int *pl_max, const int *nproc,
                   const int *np_tot, const int *ptype);

/* Src/collisions.f90:1 -- null-collision Monte Carlo against neutral
 * targets (MC) and charged targets (DSMC, picked in the incident's cell with
 * Plist from part_sorting_ and weighted by np_red from dens_red).  Same 29
 * arguments.  The GPU draws from a Philox4x32-10 counter
 * stream keyed by iseed(1) instead of the serial ran2 stream, so results
 * agree with the reference statistically (collision counts per process,
 * moments), not bit for bit.  cnt_col(ncol_mx,nproc,nm_rg) region counters
 * are accumulated like the reference; the sour_xy, sour_xz and ss2D planes are left
 * untouched (flag_diag = 1 is unsupported). */
void collisions_(const int *it, double *vxp, const int *n, const double *h, const int *ntype,
                 const int *nmax, const double *sig, const double *sig_Er, const int *sig_list,
                 const double *sig_Eex, const int *ncol_mx, const int *npt_mx, double *cnt_col,
                 double *P_loss, int *sour_xy, int *sour_xz, const int *Plist, const int *pl_max,
                 const double *sigv_mx, const int *col_info, const double *np_red,
                 signed char *flag_dead, int *flag_cex, const int *nproc, int *np_tot, int *iseed,
                 const int *nproc_mpi, const int *mpi_rank, double *ss2D_xy, double *ss2D_xz,
                 double *ss2D_yz, const int *flag_diag);

/* Src/part_expmover.f90:484 (eheating) -- Maxwellian electron heating of
 * species 1 in the heating region ixl_pow <= ix <= ixr_pow (COMMON
 * /part_info_int/ ixl_pow, ixr_pow, flag_circxh, flag_ahp; /part_info_dp_2/
 * R_ahp, nudt): each electron there gets, with probability nudt, a new
 * Maxwellian velocity of thermal speed *vt; P_loss(2,1,iproc) gains the
 * energy change.  Draws come from a Philox4x32-10 stream keyed by iseed(1)
 * and a call counter, not ran2: the reference's statistics, not its
 * sequence. */
void eheating_(const double *h, double *vxp, const int *nmax, const int *ntype, const int *nproc, int *iseed,
               const int *np_tot, const double *vt, const int *iproc, double *P_loss);

/* Src/part_injection.f90:1 -- injection of electron-ion pairs (opt_inj 1:
 * uniform in the injection box, -1: cosine / flat-top profile, 2: as many
 * events as ions were lost to the walls, N_inj(2,iproc)), of an electron beam
 * (+-3) or of cathode electrons (+-4), appended behind np_tot; P_loss(4,:)
 * gains the injected power.  COMMON: opt_inj, ns_inj, n_cath, dir_sec,
 * tag_beam, flag_pbcz, THm, zg_sec, dt, Nm, vt0.  Draws come from a Philox
 * stream keyed by iseed(1) and a call counter, not ran2.  The sour_xy,
 * sour_xz, sour_yz planes are left untouched. */
void part_injection_(const int *n, const double *h, const int *bcnd, double *vxp, int *sour_xy, int *sour_xz,
                     int *sour_yz, const int *ntype, const int *nmax, const double *I_inj, const double *xl_pow,
                     const double *xr_pow, const double *yl_pow, const double *yr_pow, const double *zl_pow,
                     const double *zr_pow, int *np_tot, const int *nproc, int *iseed, const int *nproc_mpi,
                     int *N_inj, const int *iproc, double *P_loss, const double *phi, const double *ni0);

/* Status of the last drop-in call on this thread, then cleared. */
int lepic_gpu_last_error(void);
/* Human-readable text for a status code. */
const char *lepic_gpu_strerror(int code);

/* ------------------------------------------------------------------------ */
/* Residency of the drop-ins' arrays.  No counterpart in the reference (its  */
/* arrays live in host memory only).  Off by default: each drop-in copies    */
/* its array arguments to the GPU and its results back, so a Fortran build   */
/* links the library with no source change.  On: every host array a drop-in */
/* touches keeps a device mirror keyed by its host address range, filled    */
/* from the host on first use and kept between calls; results stay on the   */
/* device until the caller asks for them.  The Fortran loop then adds:       */
/*   call lepic_gpu_set_residency(1)          once, before the time loop    */
/*   lepic_gpu_mirror_zero(np slice)          for np(:,:,:,ptype,iproc)=0,  */
/*                                            Src/main.f90:1273             */
/*   lepic_gpu_mirror_copy(phi, phi_dom(0,0,0)) for the one-rank             */
/*                                            MPI_ALLGATHERV, main.f90:977  */
/*   lepic_gpu_sync_to_host()                 before host code reads the    */
/*                                            arrays (write_data, backups,  */
/*                                            diagnostics, main.f90:1294+)  */
/*   lepic_gpu_update_device(a, bytes)        after host code writes an     */
/*                                            array a drop-in reads         */
/* np_tot(ptype, 1) is updated on the host by every call.  Particles that   */
/* host code appends behind np_tot (part_injection, part_flux_injection)    */
/* are uploaded by the next call that sees the larger np_tot.  A host array */
/* with a mirror must not be freed before lepic_gpu_release covers it.      */
/* One device per process; the registry is guarded by a lock.               */
/* ------------------------------------------------------------------------ */

/* on = 1 turns residency on; on = 0 syncs every mirror to the host and frees
 * them. */
int lepic_gpu_set_residency(int on);
int lepic_gpu_residency(void);
/* Copy every device-newer mirror (arrays, particle slices with their
 * flag_dead) back to its host array. */
int lepic_gpu_sync_to_host(void);
/* The same for the mirrors overlapping host range [h, h + bytes). */
int lepic_gpu_update_host(const void *h, size_t bytes);
/* Host code wrote [h, h + bytes): reload that range into its mirrors (a
 * particle slice mirror is dropped and rebuilt from the host by its next
 * call). */
int lepic_gpu_update_device(const void *h, size_t bytes);
/* Sync and free the mirrors overlapping [h, h + bytes) / all mirrors. */
int lepic_gpu_release(const void *h, size_t bytes);
int lepic_gpu_release_all(void);
/* Device counterparts of host statements on mirrored arrays (host memset /
 * memcpy when residency is off).  The copy's ranges must not overlap. */
int lepic_gpu_mirror_zero(void *h, size_t bytes);
int lepic_gpu_mirror_copy(void *dst, const void *src, size_t bytes);
/* Bytes the drop-in layer moved host->device and device->host since the
 * library loaded, and the number of live mirrors. */
int lepic_gpu_mirror_stats(long long *h2d_bytes, long long *d2h_bytes, int *mirrors);

/* ------------------------------------------------------------------------ */
/* Device API (layer 2): device pointers, stream as void*.  No counterpart   */
/* in the reference (which has no device boundary); each function names the  */
/* reference routine whose semantics it implements.                          */
/* ------------------------------------------------------------------------ */

/* Physics constants for the device API: the subset of the COMMON blocks the
 * hot path reads, one struct. */
typedef struct {
  int ntype, n_neu;
  double charge[LEPIC_NPART], mass[LEPIC_NPART], vt0[LEPIC_NPART], Nm[LEPIC_NPART],
      np_mx[LEPIC_NPART], nu_uplim[LEPIC_NPART];
  double dt, xmax, ymax, zmax, x_load;
  double qe, eps0, pi;
  int flag_B, flag_B_pos, flag_pbc, flag_nmn;
  int ns_coll, n_cell, np_cell;
  double Bconst[3];
  /* B-field map (Src/main.f90:361-431, read by Src/part_expmover.f90:148-203),
   * used when flag_B = 1 and Bmap is not NULL (n_B(1) > 1 in the reference);
   * Bconst is then ignored.  Bmap = Bi(4, 0:n_B(1)+2, 0:n_B(2)+2, 0:n_B(3)+2)
   * column-major, component fastest, Bi(4,...) = |B| (device pointer for the
   * device API).  A map with n_B = n lies on the node grid and reuses the
   * E-field weights; any other n_B is its own grid of spacing h_B.  A
   * particle whose left map node has |B| <= 1e-5 T takes the leapfrog step. */
  const double *Bmap;
  int n_B[3];
  double h_B[3];
  /* Dielectric walls (Src/part_expmover.f90:302-348), device pointers, all
   * NULL when there are none: dtype(0:ngrid) (2: Y = const plane, 3 and 4:
   * X = const planes) and the surface-charge sums of every species,
   * sum_q_xz(0:n1+2,0:n3+2,ntype) and sum_q_yz(2,0:n2+2,0:n3+2,ntype), to
   * which the FP64 pushes add the charge of the particles lost on them. */
  const int *dtype;
  double *sum_q_xz;
  double *sum_q_yz;
} lepic_phys_t;

/* Cross-section tables after Src/read_reactions.f90:ordering, device copies. */
typedef struct {
  int ncol, npt, npt_mx;
  const double *sig_Er;   /* [npt] device                                    */
  const double *sig;      /* sig(npt_mx, ncol) device, column-major          */
  const double *sig_Eth;  /* [ncol] device                                   */
  const int *col_info;    /* col_info(ncol, 10) device, column-major         */
  const int *sig_list;    /* host: sig_list(10, ncol)                        */
  const int *p_ncol;      /* host: [10]                                      */
  const double *sigv_mx;  /* host: sigv_mx(10, ncol)                         */
  const int *col_info_h;  /* host copy of col_info                           */
} lepic_tables_t;

/* Grid geometry on the device. */
typedef struct {
  int n[3];
  double h[3];
  const int *bcnd;        /* (n1+3)(n2+3)(n3+3) device                        */
  const double *kq;       /* same shape, device                               */
  const unsigned char *cell_wall; /* (n1+2)(n2+2)(n3+2): 1 if all 8 nodes of
                                     cell (ix,iy,iz), ix in 0..n1+1, are walls */
} lepic_grid_t;

/* One species' FP64 particles on the device: SoA, component c of particle i
 * at p[c*cap + i], c = x,y,z,vx,vy,vz.  count: device int. */
typedef struct {
  double *p;
  double *p_alt;          /* second buffer of the same size (sort target)    */
  int *count;             /* device int                                       */
  int *key;               /* device int[cap] scratch                          */
  signed char *flag_dead; /* device int8[cap] or NULL                         */
  int cap;
} lepic_species_f64_t;

/* One species in the mixed-precision layout (28 B per particle): cell[i] =
 * (ix-1) | (iy-1) << 10 | (iz-1) << 20 with ix = INT(x/h)+1 (so each grid
 * dimension is at most 1024 cells), and p[a*cap + i] for a = fx, fy, fz
 * (in-cell offsets in [0,1), x = (ix-1+fx) h) and vx, vy, vz (m/s), all FP32.
 * *_alt: sort targets of the same size.  cap must be a multiple of 4 and the
 * arrays 16-byte aligned (the push moves particles in groups of four).  The
 * sort orders particles by 8x8x8-cell tiles (cells in x-fastest order inside
 * a tile, tiles in x-fastest order) and writes the particle offset of every
 * tile to tile_off (device int[LEPIC_TILES(n)+1], zero-filled by the caller
 * before the first sort); the push deposits each tile's particles through an
 * on-chip node tile. */
typedef struct {
  int *cell;
  float *p;
  int *cell_alt;
  float *p_alt;
  int *count;             /* device int                                       */
  signed char *flag_dead; /* device int8[cap]                                 */
  int *tile_off;          /* device int[LEPIC_TILES(n)+1]                     */
  int cap;
  int *cell_off;          /* device int[LEPIC_TILES(n)*512+1] or NULL: the sort
                             writes the start of every cell (tile-key order)  */
} lepic_species_mixed_t;

/* Packed cell index of the mixed layout and the 8x8x8-cell tiles. */
#define LEPIC_CELL_BITS 10
#define LEPIC_CELL_MAX (1 << LEPIC_CELL_BITS)
#define LEPIC_TILE_CELLS 8
#define LEPIC_TILES(n)                                                        \
  ((((n)[0] + 7) / 8) * (((n)[1] + 7) / 8) * (((n)[2] + 7) / 8))

/* Src/calc_rho.f90:1 on device grids (nproc = 1). */
int lepic_dev_calc_rho(const lepic_grid_t *g, double *np, double *rhs, int ntype,
                       const lepic_phys_t *P, void *stream);

/* Src/Efield.f90:1 on device grids. */
int lepic_dev_calc_efield(const lepic_grid_t *g, const double *phi, double *Ei, void *stream);

/* Src/pdesolver.f90:1 as one persistent cooperative kernel (all V-cycles,
 * all levels, no host round trips).  u: (n+3)^3 device potential (z from 0),
 * b: (n+2)^3.  Blocks until done; k/ktot/res returned like the reference.
 * P->flag_pbc: periodic planes in y and z (bcnd 0); P->flag_nmn: the Neumann
 * plane at x = 0 (bcnd -2), as Src/sors.f90 and Src/mg.f90 treat them. */
int lepic_dev_pdesolver(const lepic_grid_t *g, double *u, const double *b, int ncycl, double eps,
                        double omega, int ng, const lepic_phys_t *P, int *k, double *ktot,
                        double *res, void *stream);

/* No counterpart in the reference.  The Poisson solve of lepic_dev_pdesolver
 * for callers that cannot call cudaMalloc inside their time loop: drivers whose
 * device memory is owned by their own pool (a Fortran host that hands every
 * buffer in, or a framework allocator such as PyTorch's) and that forbid
 * allocations there, since cudaMalloc synchronises the device and fails once
 * the pool holds the memory.  This variant allocates nothing: its scratch is
 * one static 8 MiB device array per GPU that loads the library, held until
 * the process exits, which fits grids up to 64^3 cells; larger grids return
 * LEPIC_ERR_SCRATCH_LIMIT.  The first call on each device looks up the
 * array's device address (cudaGetSymbolAddress) and should be made before any
 * stream capture.  Every call waits on the stream until its solve is done and
 * reads k, ktot and res back from the device into host memory of its own
 * stack.  All calls share the array and it keeps the last call's
 * contents (what must start at zero is cleared per call); calls that overlap
 * on the GPU, on any stream, race.  u, b and g->bcnd are the caller's device
 * buffers exactly as for lepic_dev_pdesolver; Dirichlet walls only (periodic
 * or Neumann planes return LEPIC_ERR_UNSUPPORTED). */
int lepic_dev_pdesolver_noalloc(const lepic_grid_t *g, double *u, const double *b, int ncycl,
                                double eps, double omega, int ng, const lepic_phys_t *P, int *k,
                                double *ktot, double *res, void *stream);

/* Src/main.f90:859-949 with one rank: the potential of the dielectric walls'
 * nodes (dtype 2, 3, 4 of P->dtype) rises by the surface charge of every
 * species over the capacitance per cell Ca (F; the input Ca times h(1) h(3),
 * Src/main.f90:572) -- Q/(2 Ca) on Y = const planes, Q/Ca on X = const
 * planes, with the periodic-z doubling of the boundary rows -- and the sums
 * P->sum_q_xz / P->sum_q_yz are cleared.  phi device (0:n1+2,0:n2+2,0:n3+2).
 * Multi-rank callers sum the per-rank sums first (the MPI_ALLREDUCE of
 * Src/main.f90:888-892). */
int lepic_dev_dielectric_phi(const lepic_grid_t *g, double *phi, const lepic_phys_t *P, int ngrid, double Ca,
                             void *stream);

/* Src/part_expmover.f90:1-482 for one species: push + loss + in-order
 * compaction.  Ei device (3,(n+3)^3).  p_mac: host (ntype,2,0:ngrid),
 * P_loss: host (4,ntype), accumulated. */
int lepic_dev_part_mover(const lepic_grid_t *g, const double *Ei, lepic_species_f64_t *s,
                         int ptype, int ntype, int ngrid, const lepic_phys_t *P, double *p_mac,
                         double *P_loss, void *stream);

/* Src/part_expmover.f90:55-272 (gather, Boris, loss test of part_mover)
 * fused with Src/part_expmover.f90:591-656 (CIC deposition of the new
 * position) for one species, in place, for the device-resident step loop.
 * Lost and killed particles are removed by moving tail particles into their
 * slots (order not kept; the periodic sort restores cell order).  np: device
 * grid of this species (accumulated); acc: device doubles [2 + 2(ngrid+1)]
 * accumulating P_loss(1), P_loss(3) and p_mac(count, energy) per wall label.
 * n_hint: an upper bound of the species' count (grid size), <= 0 = capacity.
 * With P->dtype set, the surface charge of the particles lost on dielectric
 * walls is added to P->sum_q_xz / P->sum_q_yz. */
int lepic_dev_push_deposit(const lepic_grid_t *g, const double *Ei, lepic_species_f64_t *s,
                           int ptype, int ngrid, const lepic_phys_t *P, double *np, double *acc,
                           int n_hint, void *stream);

/* Mixed-precision counterpart of lepic_dev_push_deposit (same reference
 * lines): FP32 gather from E4 (one float4 Ex,Ey,Ez,0 per node, (n+3)^3
 * nodes, from lepic_dev_pack_e32), FP32 Boris, position update on the
 * in-cell offset, CIC weights of the new position quantized to 2^-24 (each
 * particle deposits exactly 1) and summed exactly in integers per sorted
 * tile on chip, then added into the FP64 grid np.  Requires a closed box
 * (cells outside 1..n are walls).  n_hint: an upper bound of the count, used
 * only before the first sort (<= 0: capacity).  Dielectric walls of P as in
 * lepic_dev_push_deposit (weights from the FP32 offsets, summed in FP64). */
int lepic_dev_push_deposit_mixed(const lepic_grid_t *g, const float *E4, lepic_species_mixed_t *s,
                                 int ptype, int ngrid, const lepic_phys_t *P, double *np, double *acc,
                                 int n_hint, void *stream);
/* Src/sorting.f90:97-258 for the mixed layout: counting sort on the stored
 * cell in tile order (swaps the buffers inside *s, writes s->tile_off). */
int lepic_dev_sort_mixed(const lepic_grid_t *g, lepic_species_mixed_t *s, int n_hint, void *stream);
/* GPU particle loader for the mixed layout: the same Philox draws as
 * lepic_dev_load_uniform written as cell + FP32 offsets and velocities (no
 * FP64 copy); clears s->tile_off. */
int lepic_dev_load_uniform_mixed(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype,
                                 long long n_per_species, const lepic_phys_t *P, unsigned long long seed,
                                 void *stream);
/* CIC deposition of a mixed-layout species into np (accumulated), with the
 * integer weights of lepic_dev_push_deposit_mixed (exact charge). */
int lepic_dev_deposit_mixed(const lepic_grid_t *g, const lepic_species_mixed_t *s, int ptype,
                            const lepic_phys_t *P, double *np, int n_hint, void *stream);
/* E4[i] = (float)Ei(1:3, i), 0 for the nodes i < nodes (FP32 field of the
 * mixed push; E4 16-byte aligned). */
int lepic_dev_pack_e32(const double *Ei, float *E4, long long nodes, void *stream);
/* Layout conversions FP64 SoA <-> mixed (n particles). */
int lepic_dev_f64_to_mixed(const lepic_grid_t *g, const lepic_species_f64_t *in, lepic_species_mixed_t *out,
                           long long n, void *stream);
int lepic_dev_mixed_to_f64(const lepic_grid_t *g, const lepic_species_mixed_t *in, double *out,
                           long long capout, long long n, void *stream);
/* Mixed-precision Poisson solve for the operator of Src/pdesolver.f90:1
 * (Dirichlet walls; periodic or Neumann planes return LEPIC_ERR_UNSUPPORTED):
 * FP64 residual r = b - A u, FP32 multigrid V-cycle on
 * A e = r (red-black sweeps: nu_fine_pre / nu_fine_post on the finest level,
 * nu_pre / nu_post on the coarser ones, coarse_sweeps on the coarsest), u += e
 * in FP64, until sum|r| / alpha < eps, with the sum over plasma nodes and the
 * alpha of the reference's exit test (or max_refine refinements).  One
 * cooperative launch.  iters: refinements done; res: the final
 * sum|r| / alpha; the call waits for the solve and returns its status.  With
 * iters and res both NULL it does not wait: a solve that does not converge
 * or diverges records its status in the device error word
 * (lepic_dev_check / lepic_dev_check_async), and
 * lepic_dev_pdesolver_mixed_stats copies its refinements and residual out
 * later in stream order. */
int lepic_dev_pdesolver_mixed(const lepic_grid_t *g, double *u, const double *b, double eps,
                              double omega, int ng, const lepic_phys_t *P, int max_refine,
                              int nu_fine_pre, int nu_fine_post, int nu_pre, int nu_post,
                              int coarse_sweeps, int *iters, double *res, void *stream);
/* Enqueues on `stream` copies of the last mixed solve's refinements and
 * residual on this device into *iters and *res (pinned host memory); no
 * wait: they hold the values once the stream has passed this point. */
int lepic_dev_pdesolver_mixed_stats(int *iters, double *res, void *stream);
/* lepic_dev_collisions for species in the mixed layout (same physics; the
 * post-collision velocities are stored in FP32). */
int lepic_dev_collisions_mixed(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype,
                               const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                               unsigned long long call_index, double *nu_max, long long *counts,
                               void *stream);

/* Src/part_expmover.f90:570-686 for one species, accumulating into np
 * (device grid of that species). */
int lepic_dev_charge_deposition(const lepic_grid_t *g, const lepic_species_f64_t *s, int ptype,
                                const lepic_phys_t *P, double *np, void *stream);

/* Src/sorting.f90:97-258 for one species: counting sort by cell.  Plist:
 * device int[pl_max+1] receiving inclusive end offsets. */
int lepic_dev_part_sorting(const lepic_grid_t *g, lepic_species_f64_t *s, int *Plist, int pl_max,
                           void *stream);

/* Src/collisions.f90:1-212 + collision_OMP for neutral targets, Philox
 * per-particle null collisions.  sp[ntype]; counts[ncol] host, accumulated
 * (collisions per reaction); nu_max[ntype] host output. */
int lepic_dev_collisions(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype,
                         const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                         unsigned long long call_index, double *nu_max, long long *counts,
                         void *stream);

/* Particle injection (Src/part_injection.f90, Src/main.f90:1261-1267). */
typedef struct {
  int opt_inj;            /* 1, -1, 2, +-3, +-4 (see part_injection_)        */
  int ns_inj;             /* steps between injections                        */
  int n_cath, dir_sec, tag_beam, flag_pbcz;
  double I_inj;           /* injected current, A                             */
  double xl, xr, yl, yr, zl, zr; /* injection box xl_pow..zr_pow, m          */
  double THm;             /* beam / cathode energy, eV                        */
  double zg_sec[2];       /* emissive planes of the cathodes, m              */
  double ni0[LEPIC_NPART]; /* probability that an event injects a species    */
} lepic_inject_t;

/* The injection on the device particles of either layout: n_events events
 * (n_events < 0: the current I_inj ns_inj dt / (qe Nm(1)), rounded
 * stochastically).  np: per-species device density grids to deposit the new
 * particles into (the step loop, whose deposition ran before), or NULL.
 * phi: device potential (beam power), or NULL.  P_loss4 (host [ntype]) and
 * injected (host [ntype]) accumulate. */
int lepic_dev_inject(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype, const lepic_phys_t *P,
                     const lepic_inject_t *I, long long n_events, unsigned long long seed, unsigned long long call,
                     double *const *np, const double *phi, double *P_loss4, long long *injected, void *stream);
int lepic_dev_inject_mixed(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype, const lepic_phys_t *P,
                           const lepic_inject_t *I, long long n_events, unsigned long long seed,
                           unsigned long long call, double *const *np, const double *phi, double *P_loss4,
                           long long *injected, void *stream);

/* Electron heating region and rate: ixl_pow, ixr_pow, flag_circxh, flag_ahp,
 * R_ahp (Src/main.f90:313, 612-614), nudt = nu_h ns_heat dt (Src/main.f90:
 * 564), Pabs and nu_h (absorbed power, W, and heating frequency, 1/s). */
typedef struct {
  int ixl_pow, ixr_pow, flag_circxh, flag_ahp;
  double R_ahp, nudt, Pabs, nu_h;
} lepic_heat_t;

/* Src/part_expmover.f90:484-568 (eheating) on the device electrons (species
 * 1, either layout).  vt: thermal speed; with stats (device double[2] from
 * lepic_dev_heat_stats: sum Ek, Nh) and H->Pabs > 0 the speed is the
 * self-consistent one of Src/main.f90:1206-1227 instead, computed on the
 * device.  Philox draws keyed by seed, counter (particle, call).  acc: device
 * double[3]; acc[0] += energy change (P_loss(2)), acc[1] += electrons heated,
 * acc[2] = the thermal speed used. */
int lepic_dev_eheating(const lepic_grid_t *g, lepic_species_f64_t *e, const lepic_phys_t *P,
                       const lepic_heat_t *H, double vt, const double *stats, unsigned long long seed,
                       unsigned long long call, double *acc, void *stream);
int lepic_dev_eheating_mixed(const lepic_grid_t *g, lepic_species_mixed_t *e, const lepic_phys_t *P,
                             const lepic_heat_t *H, double vt, const double *stats, unsigned long long seed,
                             unsigned long long call, double *acc, void *stream);
/* Src/part_expmover.f90:658-681: stats[0] += kinetic energy, stats[1] +=
 * number of the electrons in the heating region (device double[2]). */
int lepic_dev_heat_stats(const lepic_grid_t *g, const lepic_species_f64_t *e, const lepic_phys_t *P,
                         const lepic_heat_t *H, double *stats, void *stream);
int lepic_dev_heat_stats_mixed(const lepic_grid_t *g, const lepic_species_mixed_t *e, const lepic_phys_t *P,
                               const lepic_heat_t *H, double *stats, void *stream);

/* Charged targets (DSMC, Src/collisions.f90:335-423, 524-531) for the
 * collision calls below.  Per species: np[p], the device density grid of the
 * last deposition (np_red, (n1+3)(n2+3)(n3+3)); cell_off[p], the device
 * per-cell offsets of that species' last sort: for the FP64 layout the Plist
 * of lepic_dev_part_sorting (inclusive ends at the reference's linear cell
 * index, pl_max+1 entries), for the mixed layout the cell_off of
 * lepic_species_mixed_t (exclusive starts at the 8x8x8-tile key).  A target
 * is a particle of its species in the incident's cell, else in the first
 * non-empty neighbour cell in the reference's order; the species must not
 * have moved since that sort.  The target density is the mean of np over the
 * cell's 8 nodes; nu_max uses P->np_mx of the target species (dens_red's
 * maximum, set by the caller).  A collision may change the target's
 * velocity or remove it (flag_dead of the target species).  The reference
 * runs its collisions one after another; here they run concurrently in
 * rounds, and a collision whose target another collision of the same round
 * took is evaluated again in the next round, from its own draws, against the
 * target as that collision left it, so every drawn collision happens.  A
 * charged target of the incident's own species is LEPIC_ERR_UNSUPPORTED.
 * The outputs accumulate: missed, incident particles that found no target in
 * reach (the reference's err_coll); lost_claims, collisions still deferred
 * after 256 rounds (not done; zero unless one target is drawn by more than
 * 256 collisions of a call); replayed, the deferrals. */
typedef struct {
  const double *np[LEPIC_NPART];
  const int *cell_off[LEPIC_NPART];
  long long missed, lost_claims, replayed;
} lepic_targets_t;
int lepic_dev_collisions_targets(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype,
                                 const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                                 unsigned long long call_index, double *nu_max, long long *counts,
                                 lepic_targets_t *tg, void *stream);
int lepic_dev_collisions_mixed_targets(const lepic_grid_t *g, lepic_species_mixed_t *sp, int ntype,
                                       const lepic_tables_t *T, const lepic_phys_t *P, unsigned long long seed,
                                       unsigned long long call_index, double *nu_max, long long *counts,
                                       lepic_targets_t *tg, void *stream);

/* Differentiable window of the collisional step (no counterpart in the
 * reference).  The particles of each species keep their slots for the whole
 * window, in the mixed layout (packed cell, offsets in [0,1) and velocities as
 * six planes of `cap`, FP32 or FP64): lam holds the adjoint (d J / d x in
 * J per m for x, y, z, d J / d v for vx, vy, vz), bl the particle's window
 * history: born = (short)(bl & 0xffff) the step whose collisions created it
 * (-1: present at the start), lost = bl >> 16 the step whose push took it to
 * a wall (0x7fff: not lost).  A lost particle keeps its state from before that
 * push. */
typedef struct {
  int *cell;
  void *p;
  void *lam;
  int *bl;
  int *count;             /* device int                                       */
  int cap;
  int fp64;               /* 1: p and lam are double planes, 0: float         */
  const int *tile_off;    /* FP32 window: the slot offsets of the 8^3-cell
                             tiles of the sort the particles are in
                             (LEPIC_TILES(n) + 1 device ints), or NULL; the
                             deposit and the push adjoint then scatter tile
                             by tile through shared memory (any slot order
                             gives the same result, the sort's order makes
                             it fast)                                         */
  int tile_end;           /* tile_off[LEPIC_TILES(n)] (a host copy): slots
                             from here on are scattered untiled               */
  int pad;
} lepic_win_species_t;

/* One collision of the window's MCC (neutral targets), recorded by the
 * forward pass and replayed by later passes: the incident (species P, slot i)
 * collided at `step` through reaction `r` (position in the species' list;
 * `ind` the global 1-based index, `rt` its type) with a target of velocity
 * tv and mass m_t; vold is the incident's velocity before.  Byproduct a of
 * species by[a] (-1: not a particle, a neutral) got the velocity
 * v_cm + vp e1[a], vp = sqrt(2 (E_cm - Eth) / sum_mass) / |m_b|, and lives in
 * slot[a] (-1: the incident itself). */
typedef struct {
  int step, P, i, r;
  int rt, nby, ind, pad;
  int by[4];
  int slot[4];
  float e1[4][3];
  double tv[3];
  double vold[3];
  double m_t, Eth;
  double sum_mass;        /* sum over the byproducts of 1 / |mass|            */
  double pad2;
} lepic_win_event_t;

/* GPU particle loader (counterpart of Src/load_part.f90:91-194 for the
 * large workloads): n_per_species samples, positions uniform in
 * [0,x_load) x [0,ymax) x [0,zmax) outside all-wall cells, shared by all
 * species of a sample (co-located pairs), Maxwellian velocities with vt0.
 * Draws come from a Philox4x32-10 stream keyed by seed (not ran2). */
int lepic_dev_load_uniform(const lepic_grid_t *g, lepic_species_f64_t *sp, int ntype,
                           long long n_per_species, const lepic_phys_t *P, unsigned long long seed,
                           void *stream);

/* Per-cell all-wall mask of the loss test (Src/part_expmover.f90:258-262):
 * cell_wall((n1+2)(n2+2)(n3+2)) from bcnd, both device. */
int lepic_dev_cell_wall(const int *n, const int *bcnd, unsigned char *cell_wall, void *stream);

/* Src/calc_rho.f90:116 (dens_red) on device grids; np_mx host [ntype];
 * np_red may be NULL (only np_mx wanted). */
int lepic_dev_dens_red(const lepic_grid_t *g, const double *np, double *np_red, int ntype,
                       double *np_mx, void *stream);

/* Adjoint window (no counterpart in the reference).  Differentiable K-step
 * window of the collisionless FP64 step for one species in the FP64 SoA
 * layout p[a*cap + i] (x,y,z,vx,vy,vz): particles keep their slots and
 * alive[i] (int8, 1 = alive) marks those still in the domain.
 *   win_push:    gather + Boris + leapfrog of the alive particles with E
 *                (3,(n+3)^3); a particle reaching a wall cell gets alive = 0.
 *   win_deposit: CIC deposition of the alive particles into np (accumulated,
 *                kq applied).
 * Adjoint of step n, in reverse order (see the window driver):
 *   adj_push:    p = state before push n, alive_before/after = the flags
 *                before/after it; lam (6,lcap) holds (lx, lv) of the outputs
 *                and receives (lx, lv) of the inputs without the deposit
 *                term; lE (3,(n+3)^3) += gather^T of the field adjoint;
 *                *dBz += d/dBz (one device double).
 *   adj_efield:  lphi = G^T lE (E = G phi of lepic_dev_calc_efield, Dirichlet
 *                walls); lphi is overwritten, lE is modified (wall
 *                extrapolations are moved onto the nodes they read).
 *   adj_rhs:     b ((n+2)^3) = lphi on plasma nodes: the right-hand side of
 *                the adjoint Poisson solve A mu = b, solved by
 *                lepic_dev_pdesolver with u = mu = 0 on walls.
 *   adj_walls:   dV[label-1] += dJ/dV_label for labels 1..nlabel (device
 *                doubles) from lphi and mu; lnp = -q mu.
 *   adj_deposit: lam (lx) += deposit^T(lnp) at the state before push n. */
int lepic_dev_win_push(const lepic_grid_t *g, const double *Ei, double *p, int cap, int n, signed char *alive,
                       int ptype, const lepic_phys_t *P, void *stream);
int lepic_dev_win_deposit(const lepic_grid_t *g, const double *p, int cap, int n, const signed char *alive,
                          int ptype, const lepic_phys_t *P, double *np, void *stream);
int lepic_dev_adj_push(const lepic_grid_t *g, const double *Ei, const double *p, int cap, int n,
                       const signed char *alive_before, const signed char *alive_after, double *lam, int lcap,
                       int ptype, const lepic_phys_t *P, double *lE, double *dBz, void *stream);
int lepic_dev_adj_efield(const lepic_grid_t *g, double *lE, double *lphi, void *stream);
int lepic_dev_adj_rhs(const lepic_grid_t *g, const double *lphi, double *b, void *stream);
int lepic_dev_adj_walls(const lepic_grid_t *g, const lepic_phys_t *P, int ptype, const double *lphi,
                        const double *mu, double *lnp, double *dV, int nlabel, void *stream);

/* The differentiable window of the collisional step (no counterpart in the
 * reference; the forward operations are those of the step loop:
 * Src/part_expmover.f90:89-250, 570-686, Src/collisions.f90:437-998), one
 * species per call, FP32 or FP64 planes (ws->fp64).  Step n: deposit, field
 * solve, E^n, collisions, push.  E: the FP32 node field (float4 per node,
 * lepic_dev_pack_e32) for FP32 planes, the FP64 field (3 per node) for FP64.
 *   cw_deposit:     np += the CIC charge of the particles of step n (created
 *                   before it, not lost before its push), kq applied.
 *   cw_push:        gather + Boris + leapfrog of step n; a particle reaching a
 *                   wall cell is lost at n (it keeps its state from before the
 *                   push) and *wall_acc += its kinetic energy (J, weight Nm).
 *   cw_reverse:     the push of step n undone for the particles it kept
 *                   (x^n = x^{n+1} - dt v^{n+1/2}, inverse rotation with E^n).
 *   cw_adj_push:    adjoint of the push of step n at (x^n, v+): lam from
 *                   (dJ/dx^{n+1}, dJ/dv^{n+1/2}) to the push's part of dJ/dx^n
 *                   and dJ/dv+; lE += gather^T (device (3,(n+3)^3)), *dBz +=;
 *                   a particle lost at n starts from wflux Nm m v^{n+1/2}.
 *   cw_adj_deposit: lam(x) += -q kdep sum kq mu grad w for the particles
 *                   deposited at step n (mu: the adjoint potential).
 * The collisions of step n (neutral targets only; the incident survives
 * every reaction) are drawn by lepic_dev_win_collisions, which records each
 * in log (the step's records continue at *nlog, at most log_cap), or applied
 * again from records by cw_replay (which writes the incident's velocity
 * before into vold); cw_adj_collide is the records' adjoint, after which the
 * incidents hold their velocities before again. */
int lepic_dev_cw_deposit(const lepic_grid_t *g, const lepic_win_species_t *ws, int ptype, const lepic_phys_t *P,
                         int step, double *np, void *stream);
int lepic_dev_cw_push(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                      const lepic_phys_t *P, int step, double *wall_acc, void *stream);
int lepic_dev_cw_reverse(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                         const lepic_phys_t *P, int step, void *stream);
int lepic_dev_cw_adj_push(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                          const lepic_phys_t *P, int step, double wflux, double *lE, double *dBz, void *stream);
/* One backward step, fused: cw_adj_deposit of step + 1 (mu of that step;
 * NULL: none), cw_reverse of step, cw_adj_push of step -- what the three
 * calls do in that order, with the particle state read once (FP32 window
 * with tile offsets: one kernel per tile). */
int lepic_dev_cw_back(const lepic_grid_t *g, const void *E, lepic_win_species_t *ws, int ptype,
                      const lepic_phys_t *P, int step, const double *mu, double wflux, double *lE, double *dBz,
                      void *stream);
int lepic_dev_cw_adj_deposit(const lepic_grid_t *g, lepic_win_species_t *ws, int ptype, const lepic_phys_t *P,
                             int step, const double *mu, void *stream);
int lepic_dev_win_collisions(const lepic_grid_t *g, lepic_win_species_t *ws, int ntype, const lepic_tables_t *T,
                             const lepic_phys_t *P, unsigned long long seed, unsigned long long call_index, int step,
                             lepic_win_event_t *log, int log_cap, int *nlog, double *nu_max, long long *counts,
                             void *stream);
int lepic_dev_cw_replay(const lepic_grid_t *g, lepic_win_species_t *ws, int ntype, const lepic_phys_t *P,
                        lepic_win_event_t *events, int ne, void *stream);
int lepic_dev_cw_adj_collide(const lepic_grid_t *g, lepic_win_species_t *ws, int ntype, const lepic_phys_t *P,
                             const lepic_win_event_t *events, int ne, void *stream);
int lepic_dev_adj_deposit(const lepic_grid_t *g, const double *p, int cap, int n, const signed char *alive,
                          const double *lnp, double *lam, int lcap, int ptype, const lepic_phys_t *P,
                          void *stream);

/* Per-kernel device timers (CUDA events around each named launch).  No
 * counterpart in the reference (its MSTIMER buckets, Src/utils.f90:503-527,
 * time host phases).  read: names '\n'-separated into buf, total ms and
 * launch count per name; returns the number of names. */
void lepic_timing_enable(int on);
void lepic_timing_reset(void);
int lepic_timing_read(char *buf, int buflen, double *ms, long long *launches, int max_names);

/* Number of SMs, device name; 0 on success. */
int lepic_dev_info(int *sm_count, char *name, int name_len);
/* Status of the kernels launched so far: synchronises `stream`, returns the
 * first status a kernel recorded in the device error word since the last
 * check (0 = none) and clears it; detail: the recorded particle index or
 * value.  The device API's launch functions do not all wait for their
 * kernels, so a step loop calls this once per step (as sim.Simulation
 * does).  No counterpart in the reference (it stops the run in place,
 * Src/utils.f90:529-546). */
int lepic_dev_check(void *stream, int *detail);
/* lepic_dev_check without the wait: enqueues on `stream` a copy of the device
 * error word (status, detail) into host[0], host[1] (pinned host memory) and
 * clears it.  The host reads host[] once the stream has passed this point (an
 * event recorded after the call), so a step loop sees a step's status a step
 * or two later without stalling its launches.  Statuses recorded by kernels
 * on other streams between the copy and the clear are lost. */
int lepic_dev_check_async(void *stream, int *host);
/* The failure path of the bounded device waits, for tests: one block whose
 * first thread waits on an mbarrier phase that nothing completes, at most
 * limit_ns (0 < limit_ns <= 2e9) nanoseconds of %globaltimer, then records
 * LEPIC_ERR_TIMEOUT in the device error word as the library's tile-copy
 * waits do when a copy never lands; the context stays usable.  Returns the
 * launch status; the recorded one is read with lepic_dev_check.  No
 * counterpart in the reference. */
int lepic_dev_wait_selftest(long long limit_ns, void *stream);
/* Library build identification (nvcc version, arch). */
const char *lepic_build_info(void);

#ifdef __cplusplus
}
#endif
#endif
