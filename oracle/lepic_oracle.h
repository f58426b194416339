/*
 * CPU FP64 oracle for the LePIC 3D PIC-MCC timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the parity checker: it is a
 * strict-IEEE (no fast-math, no FMA contraction) restatement of the legacy
 * Fortran routines under Src/ of the reference, kept in their loop order and
 * operation order so that a GPU kernel that evaluates the same expressions in
 * the same order reproduces it bit for bit.  Only tests/, the smoke check and
 * the CPU-baseline leg of bench.py load it; the product never links it.
 *
 * Parity pins: the reference ships no golden vectors for the hot path.  The
 * geometry mask (Src/generate_boundary.f90) and the E-field stencil
 * (Src/Efield.f90) are pinned against the reference's committed output planes
 * DATA/DATA_2D/{bcnd,phi,Ex,Ey,Ez}_*.mco (see tests/golden/make_golden.py).
 * Every other routine is "parity unpinned" against the reference itself and
 * is pinned by analytic known-answer tests instead (manufactured Poisson
 * solution, gyration of the Boris push, charge conservation of CIC, counting
 * sort invariants, constant cross-section collision rate).
 *
 * Layout conventions (all column-major like the Fortran arrays, one OpenMP
 * thread slice, i.e. nproc = 1, nproc_mpi = 1):
 *   node grids   g(0:n1+2, 0:n2+2, 0:n3+2)        index ix + N1*(iy + N2*iz)
 *   rhs grid     b(0:n1+1, 0:n2+1, 0:n3+1)
 *   Ei           Ei(3, 0:n1+2, 0:n2+2, 0:n3+2)    component fastest
 *   vxp          vxp(6, nmax, ntype)              x,y,z,vx,vy,vz per particle
 *   np           np(0:n1+2, 0:n2+2, 0:n3+2, ntype)
 *   potential u  u(0:n1+2, 0:n2+2, 0:n3+2)  (the reference's extra z = -1
 *                ghost plane only serves MPI halos and is never read with one
 *                rank, so it is dropped here).
 */
#ifndef LEPIC_ORACLE_H
#define LEPIC_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_NPART 10

/* Physics constants and flags that the reference keeps in COMMON blocks
 * (Src/particle_info.h:53-70, Src/constants.h). */
typedef struct OPhys {
  int ntype;                       /* charged species count                 */
  int n_neu;                       /* neutral species after the charged ones */
  double charge[ORACLE_NPART];     /* C                                     */
  double mass[ORACLE_NPART];       /* kg (neutrals negative, as reference)   */
  double vt0[ORACLE_NPART];        /* sqrt(2 q T / m)                       */
  double Nm[ORACLE_NPART];         /* macroparticle weight                  */
  double np_mx[ORACLE_NPART];      /* target density (neutrals: ngas n/n0)  */
  double nu_uplim[ORACLE_NPART];
  double dt, xmax, ymax, zmax, x_load;
  double qe, eps0, pi;
  int flag_B;                      /* 1: magnetised                         */
  int flag_B_pos;                  /* 1: positive ions not magnetised       */
  int flag_pbc, flag_nmn;
  int ns_coll, n_cell, np_cell;
  double Bconst[3];                /* Bi(1:3,1,1,1) with n_B(1)=1           */
  const double *Bmap;              /* Bi(4,0:nB1+2,0:nB2+2,0:nB3+2) or NULL  */
  int n_B[3];                      /* map grid (n_B(1) > 1 with a map)       */
  double h_B[3];                   /* map spacing (xmax/n_B(1), ...)         */
} OPhys;

/* Electron heating region and rate (COMMON /part_info_int/ ixl_pow, ixr_pow,
 * flag_circxh, flag_ahp; /part_info_dp_2/ R_ahp, nudt, Pabs). */
typedef struct OHeat {
  int ixl_pow, ixr_pow, flag_circxh, flag_ahp;
  double R_ahp, nudt, Pabs;
} OHeat;

/* Particle injection (Src/part_injection.f90): the COMMON values it reads. */
typedef struct OInject {
  int opt_inj, ns_inj, n_cath, dir_sec, tag_beam, flag_pbcz;
  double I_inj, xl, xr, yl, yr, zl, zr, THm, zg_sec[2];
} OInject;

/* Cross-section tables after Src/read_reactions.f90:ordering. */
typedef struct OTables {
  int ncol;                        /* reactions                              */
  int npt;                         /* sig_npt_mx: merged energy points       */
  int npt_mx;                      /* leading dimension of sig               */
  const double *sig_Er;            /* [npt]                                  */
  const double *sig;               /* sig(npt_mx, ncol) column-major         */
  const double *sig_Eth;           /* sig_Eex(:,ind_Eth) [ncol]              */
  const int *col_info;             /* col_info(ncol, 10) column-major        */
  const int *sig_list;             /* sig_list(10, ncol) column-major        */
  const int *p_ncol;               /* [10]                                   */
  const double *sigv_mx;           /* sigv_mx(10, ncol) column-major         */
} OTables;

/* error codes shared with the product's error word */
#define ORACLE_OK 0
#define ORACLE_ERR_CAPACITY 1
#define ORACLE_ERR_DIVERGED 2
#define ORACLE_ERR_PMAX 3
#define ORACLE_ERR_EKR_TABLE 4
#define ORACLE_ERR_NEG_ENERGY 5
#define ORACLE_ERR_UNSUPPORTED 6
#define ORACLE_ERR_FEW_COLL 7
#define ORACLE_ERR_BAD_PICK 8

double oracle_ran2(int *irand);
void oracle_load_gauss(double *vx, double *vy, double vt, const double rnd[2],
                       double pi);
int oracle_load_part(const int n[3], const double h[3], const int *bcnd,
                     double *np, double *vxp, int ntype, int nmax,
                     const double *kq, const double *ni0, int *np_tot,
                     int *iseed, const OPhys *P);
void oracle_make_kq(const int n[3], const int *bcnd, double *kq);
void oracle_calc_rho(const int n[3], double *np, double *rhs, const int *bcnd,
                     int ntype, const OPhys *P);
void oracle_dens_red(const int n[3], const double *np, double *np_red,
                     const int *bcnd, int ntype, double *np_mx_out);
int oracle_pdesolver(double *u, const double *b, const int *bcnd,
                     const double h[3], const int n[3], int ncycl, double eps,
                     double omega, int *k, double *ktot, double *res, int ng,
                     const OPhys *P);
void oracle_calc_efield(const int n[3], const double h[3], const double *phi,
                        double *Ei, const int *bcnd);
void oracle_dielectric_phi(const int n[3], double *phi, const int *bcnd,
                           const int *dtype, int ngrid, double *qxz,
                           double *qyz, int ntype, double Ca, int flag_pbc);
/* The negative-ion bookkeeping and the secondary emission of the mover
 * (Src/part_expmover.f90:76, 278-301, 353-400, 416-470): COMMON values and
 * the caller's arrays.  tag_neg 0: no negative ions; gam_sec <= 0: no
 * secondary emission. */
typedef struct OMoverExtra {
  int tag_neg, tag_neu, num_grd;
  int *flag_cex;                   /* flag_cex(1:nmax) of species tag_neg    */
  int *cnt_cex;                    /* cnt_cex(1:3)                           */
  double *cnt_dead;                /* cnt_dead(1)                            */
  double *beam_div;                /* beam_div(1:4)                          */
  double gam_sec, THm, zg_sec[2];
  int igrid_sec;
  int *iseed;                      /* ran2 state of the secondary draws      */
} OMoverExtra;

int oracle_part_mover(const int n[3], const double h[3], const double *Ei,
                      double *p_mac, double *P_loss, double *vxp,
                      const int *bcnd, int nmax, int ntype, int ngrid,
                      signed char *flag_dead, int *np_tot, int ptype,
                      const OPhys *P, const int *dtype, double *sum_q_xz,
                      double *sum_q_yz, const OMoverExtra *X);
void oracle_charge_deposition(const int n[3], const double h[3],
                              const double *vxp, int nmax, int ntype,
                              const double *kq, double *np, const int *np_tot,
                              int ptype, const OPhys *P);
void oracle_part_sorting(double *vxp, int nmax, int ntype, const int n[3],
                         const double h[3], int *Plist, int pl_max,
                         const int *np_tot, int ptype);
int oracle_ordering(int ncol, const int *sig_npt, const double *sig_tmp_E,
                    const double *sig_tmp_s, int npt_in_mx, const double *Eth,
                    const int *col_info, const double *mass, int ntype,
                    double qe, double *sig_Er, double *sig, int npt_mx,
                    int *npt_out, int *sig_list, int *p_ncol, double *sigv_mx);
int oracle_collisions(double *vxp, const int n[3], const double h[3], int ntype,
                      int nmax, const OTables *T, signed char *flag_dead,
                      int *np_tot, int *iseed, const OPhys *P, double *nu_max,
                      long long *cnt_col, int *Nc_out, const int *Plist,
                      int pl_max, const double *np_red, long long *err_coll);
void oracle_scatter(double *vx1, double *vy1, double *vz1, double vx, double vy,
                    double vz, double costheta, double phi);
int oracle_part_injection(const int n[3], const double h[3], const int *bcnd, double *vxp, int ntype,
                          int nmax, int *np_tot, int *iseed, int N_inj_ions, double *P_loss,
                          const double *phi, const double *ni0, const OPhys *P, const OInject *I);
void oracle_eheating(const double h[3], double *vxp, int nmax, int *iseed, const int *np_tot,
                     double vt, double *P_loss, const OPhys *P, const OHeat *H, int *nheated);
void oracle_heat_stats(const double h[3], const double *vxp, int nmax, const int *np_tot,
                       const OPhys *P, const OHeat *H, double *sum_dEk, int *Nh);

#ifdef __cplusplus
}
#endif
#endif
