/*
 * rs_oracle.h -- CPU FP64 restatement of RSPACE kukan's real-space Kohn-Sham
 * hot path.  TEST INFRASTRUCTURE ONLY: the parity tests, the smoke check and
 * the CPU-baseline leg of bench.py link this; the product library never does.
 *
 * Conventions shared with the CUDA library (rspacedist_b200/csrc):
 *   - grid point p = (iz*ny + iy)*nx + ix, 0-based, x fastest: the column-major
 *     order of kukan's svecre(ncpx,ncpy,ncpz,...) (pseudocalc8f.F90:1012);
 *   - band arrays are band-major: psi[b*N + p];
 *   - sphere lists lst[a*num_list + ii] hold 0-based point indices (lstvec2-1);
 *   - projector tables v[(a*nprjmx + j)*num_list + ii] (vnlocp layout);
 *   - <p|psi> coefficients rp[(b*natom + a)*nprjmx + j] (rspsep layout);
 *   - D / S matrices m[(a*nprjmx + i)*nprjmx + j] == dij(j,i,a) of Fortran.
 *
 * "Strict" routines fix the floating-point evaluation order: every
 * `acc + a*b` of the Fortran source is one fma(a, b, acc) (what gfortran
 * emits with FMA contraction and no reassociation), evaluated left to right.
 * Long dot products use the fixed block tree rs_tree_dot (see rs_oracle.c),
 * which the CUDA reductions reproduce exactly.
 */
#ifndef RS_ORACLE_H
#define RS_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

/* ---- tools ---- */
void orc_fdcoef(int nf, double a[9]);
void orc_lap_coefs(int nf, double dx, double dy, double dz,
                   double cx[9], double cy[9], double cz[9]);
double orc_tree_dot(long n, const double* a, const double* b);
double orc_tree_dot_f(long n, const float* a, const float* b);

/* ---- H*psi pieces ---- */
void orc_kslaplacian(int nx, int ny, int nz, int nf, double dx, double dy, double dz,
                     const double* psi, const double* veff, double* out, int nb);
void orc_precondition(int nx, int ny, int nz, const double* in, double* out, int nb);
void orc_nl_dot(int natom, int nprjmx, int num_list, const int* nprj, const int* natinf,
                const int* lst, const double* v, const double* psi, long N, int nb,
                double* rp);
void orc_nl_apply(int natom, int nprjmx, int num_list, const int* nprj, const int* natinf,
                  const int* lst, const double* v, const double* mat, double dvol,
                  const double* rp, long N, int nb, double* out);
void orc_hpsi(int nx, int ny, int nz, int nf, double dx, double dy, double dz,
              const double* veff, int natom, int nprjmx, int num_list, const int* nprj,
              const int* natinf, const int* lst, const double* v, const double* dij,
              const double* rp, const double* psi, double* hpsi, int nb);
void orc_spsi(long N, int natom, int nprjmx, int num_list, const int* nprj,
              const int* natinf, const int* lst, const double* v, const double* sss,
              double dvol, const double* rp, const double* psi, double* spsi, int nb);
void orc_grad_coefs(int nf, double h, double a[5]);
void orc_gradient(int nx, int ny, int nz, int nf, double h, int axis,
                  const double* psi, double* out);

/* ---- density / interpolation / Hartree ---- */
void orc_density(long N, int nb, const double* occ, const double* psi, double* rho);
void orc_interp_c2d(int nx, int ny, int nz, int nf, const double* in, double* out);
/* interpolation weights aweight(j, k) for nmesh = 2 (interpolation8f.F90):
 * aw[k][j + nf - 1], k = dense parity, j = -nf+1..nf */
void orc_interp_weights(int nf, double aw[2][16]);

/* ---- potentials and mixing (rs_oracle_scf.c) ---- */
/* trans_d2c_vh / trans_d2c_vxc for nperi=3, one rank: interpolation mode 2
 * (interpolation8f.F90:98-214) + overlap_interpolation nflag=2
 * (overlap_interpolation8f.F90:492-892) + division by nmesh^3.  in: dense
 * (2nx, 2ny, 2nz); out: coarse (nx, ny, nz). */
void orc_interp_d2c(int nx, int ny, int nz, int nf, const double* in, double* out);
/* vxpot_lda_pz (vxpot8f.F90:126-155): Perdew-Zunger LDA potential and energy
 * density per point. */
void orc_vxc_pz(long n, const double* rho, double* vx, double* ex);
/* scf_potentials' veff sum (scf_potentials8f.F90:256-267, no bias):
 * veff = vx + (vloc + vh). */
void orc_veff_sum(long n, const double* vx, const double* vloc, const double* vh,
                  double* veff);
/* scf_diffcharge (scf_diffcharge8f.F90) + kukan8f.F90:673:
 * sqrt(sum (ri-ro)^2 dx dy dz / (8 xmax ymax zmax)), the sum in the fixed
 * block tree. */
double orc_diffcharge(long n, const double* rho_o, const double* rho_i, double dx, double dy,
                      double dz, double xmax, double ymax, double zmax);
/* scf_charge_atomicocc (scf_charge8f.F90:146-213), real bands, one spin, one
 * k point: atocc[a][ij] = sum_l fnele[l] * t, t = rp[l][a][i] rp[l][a][j]
 * (doubled for i != j), ij over i <= j with j outer (packed upper triangle),
 * each band added as fma(fnele, t, atocc) in band order. */
void orc_atomicocc(int natom, int nprjmx, const int* nprj, int M, const double* rp,
                   const double* fnele, double* atocc);
/* scf_chargemixing_broyden (scf_chargemixing8f.F90:214-657), one spin, grid
 * density only (norm-conserving atoms): modified Broyden with history nbrydn
 * and mixing ratio eta.  Dot products use the fixed block tree times dV. */
typedef struct orc_broyden orc_broyden;
orc_broyden* orc_broyden_create(long n, int nbrydn, double eta);
void orc_broyden_free(orc_broyden* b);
/* one call of scf_chargemixing: rho_i (in: last input density, out: next) */
void orc_broyden_step(orc_broyden* b, const double* rho_o, double* rho_i, double dvol);
void orc_hartree_laplacian(int nx, int ny, int nz, int nfh, double ddx, double ddy,
                           double ddz, const double* v, double* av);
int orc_hartree_cg(int nx, int ny, int nz, int nfh, double xmax, double ymax, double zmax,
                   double epsvh, int ncgmin, int ncgmax, int ncgres, const double* rho,
                   double* vh, double* dp_out);

/* ---- sphere lists (pseudocalc_01b) ---- */
int orc_sphere_lists(int natom, const double* atx, const double* aty, const double* atz,
                     const double* rcut, int nxmax, int nymax, int nzmax, double dx,
                     double dy, double dz, int npxmax, int npymax, int npzmax, int nfdg,
                     int num_list, int* natx, int* naty, int* natz, int* natinf, int* lst,
                     int* lstx, int* lsty, int* lstz);

/* ---- projector tables (pseudocalc_01a, pseudocalc_07) ---- */
/* w[j + nfdg*npmesh], j = -nfdg*npmesh .. nfdg*npmesh-1 (wxyz) */
void orc_dg_weights(int nfdg, int npmesh, double* w);
/* One species: v[(a*nprj + la)*num_list + ii] (vnlocp), lists lstx/y/z[a*num_list + ii]
 * as offsets from (natx, naty, natz); projector la uses coefficient column
 * prj_col[la] (1..6: s, s', p, p', d, d') of coef[c*(nqmx+1) + iq] and the real
 * harmonic ylm0<prj_m[la]> (1..9).  Returns 1 when out of memory. */
int orc_projector_tables(int natom, int nprj, int num_list, int nxmax, int nymax, int nzmax,
                         double dx, double dy, double dz, int npxmax, int npymax, int npzmax,
                         int nfdg, int npmesh, const double* atx, const double* aty,
                         const double* atz, const int* natx, const int* naty, const int* natz,
                         const int* natinf, const int* lstx, const int* lsty, const int* lstz,
                         const int* prj_col, const int* prj_m, int nqct, int nqmx,
                         const double* coef, double rcut, double psftrad, double psctoff,
                         double eps, int nfiltyp, double filpp, const double* wxyz, double* v);

/* ---- eigen / subspace ---- */
int orc_jacobi_eig(int n, double* a, double* w, double* z);
void orc_reorder_rank(int m, const double* sval, int* rank);
void orc_eig2(const double a[4], double w[2], double z[4]);

/* ---- band solvers (rs_oracle_solvers.c) ---- */
typedef struct {
  int nx, ny, nz, nf;
  double dx, dy, dz;
  long N;
  int natom, nprjmx, num_list;
  const int* nprj;
  const int* natinf;
  const int* lst;
  const double* v;    /* vnlocp */
  const double* dij;  /* D per atom */
  const double* sss;  /* S-term per atom, or NULL for norm-conserving S = 1 */
  const double* veff;
} orc_sys;

typedef struct {
  int northo, nsdmax, nprecon;     /* kscg */
  double epssd;
  int ndiismax;                    /* ksdiis */
  double eps_eig_diis, alambda_diis, alambda_min, alambda_max;
} orc_solver_prm;

void orc_apply_h(const orc_sys* s, const double* psi, const double* rp, double* hpsi, int nb);
void orc_apply_s(const orc_sys* s, const double* psi, const double* rp, double* spsi, int nb);
void orc_ortho(const orc_sys* s, int M, int l_inp, int cmpt, double* psi, double* spsi,
               double* rp);
int orc_rayleighritz(const orc_sys* s, int M, int l_rrb, double* psi, double* spsi,
                     double* rp, double* hpsi, double* sval);
int orc_kscg(const orc_sys* s, const orc_solver_prm* prm, int M, double* psi, double* spsi,
             double* rp, double* hpsi, double* sval, double* resid, int* itmax);
int orc_ksdiis(const orc_sys* s, const orc_solver_prm* prm, int M, int l_hsv, double* psi,
               double* spsi, double* rp, double* hpsi, double* sval, double* resid);
void orc_reorder(long N, int M, int nrp, double* sval, double* resid, double* psi,
                 double* spsi, double* rp, double* work);
void orc_force_nl(const orc_sys* s, int M, const double* psi, const double* sval,
                  const double* occ, double* fx, double* fy, double* fz);

/* fast (OpenMP, unordered) H*psi used only as the timed CPU baseline */
void orc_hpsi_fast(const orc_sys* s, const double* psi, const double* rp, double* hpsi,
                   int nb, int nthreads);

/* ---- local pseudopotential, Ewald energy, initial bands (rs_oracle_vloc.c) ---- */
void orc_bisec(double z, double r, double eps, double* a, double* b, double* c);
void orc_vloc_coef(int nradps, int nradct, const double* radial, const double* dradial,
                   const double* potc, double a, double b, double c, double rcuts, int nqct,
                   double* coef);
void orc_vloc_soft(int natom, const double* atx, const double* aty, const double* atz,
                   double cp1, double ca, double cb, double cc, double rc, int nx, int ny,
                   int nz, double dx, double dy, double dz, double xmax, double ymax,
                   double zmax, double veta, int npwx, int npwy, int npwz, double* out,
                   double* grad);
void orc_vloc_hard(int natom, const double* atx, const double* aty, const double* atz,
                   int nxmax, int nymax, int nzmax, int nmesh, double dx, double dy, double dz,
                   double xmax, double ymax, double zmax, int npxmax, int npymax, int npzmax,
                   double rcut, double psctoff, double rcuts, int nqct, const double* coef,
                   double filpp, double eps, int nfiltyp, double* dense,
                   const double* rho_dense, double* force_acc);
double orc_ewald(int natom, const double* atx, const double* aty, const double* atz,
                 double cp1, double xmax, double ymax, double zmax, double veta, int npwx,
                 int npwy, int npwz, int nrsx, int nrsy, int nrsz);
void orc_initial_wave(int natom, const double* atx, const double* aty, const double* atz,
                      double cp1, double zs_pre, int neig, int nx, int ny, int nz, double dx,
                      double dy, double dz, double xmax, double ymax, double zmax, double* psi);

#ifdef __cplusplus
}
#endif
#endif
