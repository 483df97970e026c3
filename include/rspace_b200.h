/*
 * rspace_b200.h -- C ABI of the B200 (sm_100a) replacement for RSPACE kukan's
 * real-space Kohn-Sham hot path.
 *
 * Conventions (all entry points):
 *   - every function returns RS_OK (0) or a negative RS_E* status; the message
 *     of the last failure on the calling thread is read with rs_last_error();
 *   - arrays marked (dev) are device pointers, (host) host pointers;
 *   - grid arrays are x-fastest, column-major like kukan's
 *     svecre(ncpx,ncpy,ncpz,neigmx); band b of a band array starts at b*N;
 *   - <p|psi> arrays are rp[(b*natom + a)*nprjmx + j] (rspsep layout);
 *   - D / S matrices are m[(a*nprjmx + i)*nprjmx + j] == dij(j,i,a);
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy stream);
 *   - the library computes on one GPU, the current device of the caller.
 * Reference files are cited relative to RSPACEes.v08.01/kukan/.
 */
#ifndef RSPACE_B200_H
#define RSPACE_B200_H
#ifdef __cplusplus
extern "C" {
#endif

#define RS_OK 0
#define RS_EINVAL (-1)   /* bad argument (reference: stopp with a message) */
#define RS_ECUDA (-2)    /* CUDA runtime error */
#define RS_ENOMEM (-3)   /* device allocation failed */
#define RS_ENOCONV (-4)  /* iteration limit reached without convergence */
#define RS_ENUMERIC (-5) /* negative norm / failed eigensolve (kukan stopp) */

typedef struct rs_geom rs_geom;

/* Copies the message of the last failure on this thread into buf. */
int rs_last_error(char* buf, int len);
/* Library version string, e.g. "rspace_b200 0.1 sm_100a". */
const char* rs_version(void);

/* ---- geometry: sphere lists + projector tables ------------------------- */
/* Replaces the list-vector part of pseudocalc_01b (pseudocalc8f.F90:955-1033)
 * for one rank and nperi=3.  rcut[a] = radial(nradct)*psctoff.  Writes natx..
 * (host, natom each), natinf (host, natom), lst/lstx/lsty/lstz (host,
 * natom*num_list, lst 0-based point index).  RS_EINVAL if num_list is too
 * small ("num_list is too small", pseudocalc8f.F90:1025-1028). */
int rs_sphere_lists(int natom, const double* atx, const double* aty, const double* atz,
                    const double* rcut, int nxmax, int nymax, int nzmax, double dx,
                    double dy, double dz, int npxmax, int npymax, int npzmax, int nfdg,
                    int num_list, int* natx, int* naty, int* natz, int* natinf, int* lst,
                    int* lstx, int* lsty, int* lstz);

/* Double-grid weights of pseudocalc_01a (pseudocalc8f.F90:343-629):
 * w[j + nfdg*npmesh] = wxyz(j), j = -nfdg*npmesh .. nfdg*npmesh-1 (host). */
int rs_double_grid_weights(int nfdg, int npmesh, double* w);

/* Projector tables of one species on the GPU: replaces pseudocalc_07
 * (pseudocalc8f.F90:2515-3702).  Inputs are host arrays: atom positions
 * atx/aty/atz and coarse indices natx/naty/natz, natinf and the list offsets
 * lstx/lsty/lstz (natom*num_list) from rs_sphere_lists; per projector la the
 * coefficient column prj_col[la] (1..6: the tmpspd1..6 radial channels s, s',
 * p, p', d, d') and the real harmonic prj_m[la] (1..9: ylm01..ylm09);
 * coef(0:nqmx, 0:7) column-major (Fourier-Bessel coefficients of
 * filterpseudopotentials), nqct of them used; rcut = radial(nradct), psftrad,
 * psctoff, eps, nfiltyp (1: Fermi filter with width filpp) and wxyz from
 * rs_double_grid_weights.  Output: vnlocp(num_list, nprj, natom), zero past
 * natinf, in host memory (returns when it is written) or device memory
 * (written in stream order).  The fine mesh is npmesh points per coarse
 * spacing. */
int rs_projector_tables(int natom, int nprj, int num_list, int nxmax, int nymax, int nzmax,
                        double dx, double dy, double dz, int npxmax, int npymax, int npzmax,
                        int nfdg, int npmesh, const double* atx, const double* aty,
                        const double* atz, const int* natx, const int* naty, const int* natz,
                        const int* natinf, const int* lstx, const int* lsty, const int* lstz,
                        const int* prj_col, const int* prj_m, int nqct, int nqmx,
                        const double* coef, double rcut, double psftrad, double psctoff,
                        double eps, int nfiltyp, double filpp, const double* wxyz,
                        double* vnlocp, void* stream);

/* Uploads the grid, the sphere lists and vnlocp (host, vnlocp(num_list,
 * nprjmx,natom) layout) and builds the point-major inverse lists used by the
 * fused H*psi.  Stands for the geometry arguments kukan threads through
 * kslaplacian_r / nonlocaloperation_r_0x (nonlocaloperation8f.F90:9-235). */
int rs_geom_create(rs_geom** g, int nx, int ny, int nz, int nf, double dx, double dy,
                   double dz, int natom, int nprjmx, int num_list, const int* nprj,
                   const int* natinf, const int* lst, const double* vnlocp);
int rs_geom_destroy(rs_geom* g);
/* number of inverse-list entries (sum of natinf) */
long rs_geom_entries(const rs_geom* g);

/* ---- H*psi pieces (FP64 = bit-exact with the strict oracle) ------------- */
/* out(dev) += (-1/2 lap_FD + veff) psi for nb bands: kslaplacian_r
 * (kslaplacian8f.F90:23-261, nf=4 at 207-261) with the periodic halo of
 * overlap_finitedifference_r (overlap_finitedifference8f.F90:97-139). */
int rs_kslaplacian_f64(const rs_geom* g, const double* psi, const double* veff, double* out,
                       int nb, void* stream);
int rs_kslaplacian_f32(const rs_geom* g, const float* psi, const float* veff, float* out,
                       int nb, void* stream);

/* rp(dev) = <p_j,a|psi_b>: nonlocaloperation_r_01 (nonlocaloperation8f.F90:9-53)
 * over nb bands.  FP64: one sequential fma chain per (atom, projector, band).
 * FP32 psi: FP64 accumulation, rp in FP64. */
int rs_nonlocal_dot_f64(const rs_geom* g, const double* psi, int nb, double* rp, void* stream);
int rs_nonlocal_dot_f32(const rs_geom* g, const float* psi, int nb, double* rp, void* stream);

/* out(dev) += sum_a p_a (mat_a rp_a)/dV over nb bands: nonlocaloperation_r_02
 * (nonlocaloperation8f.F90:149-235); mat = dij (nhs=1) or sss (nhs=0). */
int rs_nonlocal_apply_f64(const rs_geom* g, const double* mat, const double* rp, int nb,
                          double* out, void* stream);

/* The launch shape the FP32 H psi of g chose (rs_hpsi_f32 times the
 * candidates on its first call with at least 64 bands): nl_chunk, the band
 * chunk whose nonlocal pass runs on a side stream behind the next chunk's
 * stencil (-1: one stencil launch, then one pass), and nl_bands, the bands
 * per thread of that pass (16 or 32); both 0 before that call.  No
 * counterpart in the reference. */
int rs_hpsi_f32_tuning(const rs_geom* g, int* nl_chunk, int* nl_bands);

/* How the FP32 stencil of g stages its planes: mode 0 (the default) copies
 * them with tensor-map (TMA) loads where nx is 64, 128 or 256 and ny a
 * multiple of 2048/nx (k_stencil_f32_tma), mode 1 with per-thread cp.async
 * (k_stencil_f32_zmarch, also the form for every other grid); mode < 0 keeps
 * the current mode.  *tma is set to 1 when an nb-band call would take the
 * TMA form.  Both forms give identical results.  No counterpart in the
 * reference. */
int rs_hpsi_f32_staging(rs_geom* g, int mode, int nb, int* tma);

/* Fused H psi = nonlocal(D) + stencil + veff, one pass over psi (the H*psi of
 * kscg8f.F90:147-183 and rayleighritz_hamiltonian_r, rayleigh-ritz8f.F90:493-575).
 * hpsi(dev) is overwritten. */
int rs_hpsi_f64(const rs_geom* g, const double* veff, const double* dij, const double* rp,
                const double* psi, double* hpsi, int nb, void* stream);
int rs_hpsi_f32(const rs_geom* g, const float* veff, const double* dij, const double* rp,
                const float* psi, float* hpsi, int nb, void* stream);
/* S psi = psi + nonlocal(sss) (orthogonalization8f.F90:187-210, nhs=0). */
int rs_spsi_f64(const rs_geom* g, const double* sss, const double* rp, const double* psi,
                double* spsi, int nb, void* stream);
int rs_spsi_f32(const rs_geom* g, const double* sss, const double* rp, const float* psi,
                float* spsi, int nb, void* stream);

/* H psi through host buffers (host psi in, host hpsi out), staged through the
 * device in band chunks with copies overlapping compute: the drop-in for a
 * Fortran caller holding svecre/hsvre in host memory. */
int rs_hpsi_host_f32(const rs_geom* g, const float* veff_dev, const double* dij_dev,
                     const double* rp_dev, const float* psi_host, float* hpsi_host, int nb,
                     int chunk, void* stream);

/* ksprecondition (ksprecondition8f.F90:8-39): out = psi/2 + sum_6 nbr/12. */
int rs_precondition_f64(const rs_geom* g, const double* in, double* out, int nb, void* stream);
int rs_precondition_f32(const rs_geom* g, const float* in, float* out, int nb, void* stream);

/* ---- density / interpolation / Hartree ---------------------------------- */
/* scf_charge_smt_r (scf_charge8f.F90:290-321): rho(dev) = sum_b occ_b psi_b^2,
 * bands accumulated in order.  occ(dev). */
int rs_density_f64(long N, int nb, const double* occ, const double* psi, double* rho,
                   void* stream);
int rs_density_f32(long N, int nb, const double* occ, const float* psi, double* rho,
                   void* stream);

/* Occupation matrices of the projectors (scf_charge_atomicocc,
 * scf_charge8f.F90:146-213; real bands, one spin, one k point):
 * atocc[a][ij] = sum_l fnele[l] <p_i|psi_l> <psi_l|p_j> (doubled for i != j),
 * ij running over i <= j with j outer, nprjmx (nprjmx + 1) / 2 entries per
 * atom.  rp is rspsep as rs_nonlocal_dot returns it ([M][natom][nprjmx]), fnele
 * the occupations (device).  Every atom is handled; kukan uses the PAW ones. */
int rs_atomicocc(const rs_geom* g, const double* rp, const double* fnele, int M, double* atocc,
                 void* stream);
/* trans_c2d_smtcharge + interpolation, forward branch, nmesh=2
 * (trans8f.F90:8-47, interpolation8f.F90:8-100): out(dev) has 8*nx*ny*nz. */
int rs_interp_c2d(int nx, int ny, int nz, int nf, const double* in, double* out,
                  void* stream);
/* scf_hartee_laplacian (scf_hartree8f.F90:901-1004): av = -1/2 lap v. */
int rs_hartree_laplacian(int nx, int ny, int nz, int nfh, double ddx, double ddy, double ddz,
                         const double* v, double* av, void* stream);
/* scf_hartree + scf_hartree_cg for nperi=3 (scf_hartree8f.F90:84-89, 626-812):
 * CG on -1/2 lap V = 2 pi (rho - mean), warm start from vh(dev, in/out).
 * Work vectors come from a stream-ordered device allocation.  iters/dp
 * (host) receive the iteration count and final residual. */
int rs_hartree_cg(int nx, int ny, int nz, int nfh, double xmax, double ymax, double zmax,
                  double epsvh, int ncgmin, int ncgmax, int ncgres, const double* rho,
                  double* vh, int* iters, double* dp, void* stream);

/* ---- subspace contractions (GS / Rayleigh-Ritz) ------------------------- */
/* C(dev, FP64, column-major ldc) = alpha * A^T B where A and B hold m and n
 * bands of K grid points (band i at A + i*lda): the Gram products of
 * rayleighritz_r (rayleigh-ritz8f.F90:80, dgemm 't','n') and of the GS blocks
 * (orthogonalization8f.F90:225-228).  FP32 operands run on tcgen05 tensor
 * cores with the 3xTF32 split and FP32 accumulation over K chunks of 16384,
 * chunks summed in FP64; sym=1 (A==B, m==n) computes one triangle and
 * mirrors it; sym=2 (m==n, A and B distinct, a product known to be
 * symmetric such as Psi^T H Psi) computes the lower triangle C(i,j), i >= j,
 * and mirrors it into the upper one.  K, lda, ldb multiples of 4. */
int rs_gram_f32(int m, int n, long K, const float* A, long lda, const float* B, long ldb,
                double alpha, double* C, long ldc, int sym, void* stream);
int rs_gram_f64(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
                double alpha, double* C, long ldc, void* stream);
/* Y(dev) = X Z: band j of Y = sum_k Z(k,j) * band k of X, Z FP64 column-major
 * (kin x nout, ldz) -- the Psi <- Psi Z updates of rayleighritz_r
 * (rayleigh-ritz8f.F90:96-119).  FP32: tcgen05 3xTF32 with X read
 * MN-major; npts and ldx multiples of 4.  FP32: Y may alias X (X is packed
 * into tensor-core blocks before Y is written); FP64: Y must not alias X. */
int rs_rotate_f32(long npts, int kin, int nout, const float* X, long ldx, const double* Z,
                  long ldz, float* Y, long ldy, void* stream);
int rs_rotate_f64(long npts, int kin, int nout, const double* X, long ldx, const double* Z,
                  long ldz, double* Y, long ldy, void* stream);

/* Symmetric eigenproblem on the GPU in FP64 (parallel cyclic Jacobi): the
 * dsyev('v','l') / pdsyevd of rayleighritz_r (rayleigh-ritz8f.F90:89,
 * rayleigh-ritz8f_sclpck.F90:268).  A (dev, n x n) is destroyed; w (dev)
 * ascending eigenvalues; Z (dev, column-major) eigenvectors, each with its
 * largest-magnitude component positive.  RS_ENUMERIC without convergence
 * (kukan: 'error in matrix diagonalization'). */
int rs_syev_f64(int n, double* A, double* w, double* Z, int* sweeps, void* stream);
/* Cholesky-QR helper: G = L L^T (dev, FP64, overwritten by L) and
 * W = L^{-T} (dev, column-major upper triangular), so that Psi W is
 * S-orthonormal with the span and ordering of kukan's Gram-Schmidt.
 * RS_ENUMERIC when G is not positive definite ('wf has negative norm',
 * orthogonalization8f.F90:249). */
int rs_chol_inv_t(int n, double* G, double* W, void* stream);

/* ---- band solvers (scf_diag and what it calls) -------------------------- */
/* Solver parameters with kukan's namelist names and defaults
 * (read_input_kukan8f.F90:198-249): northo=1, nsdmax=4, nprecon_cg=1,
 * nprecon_diis=1, epssd=1e-6, ndiismax=4, eps_eig_diis=1e-14,
 * alambda_diis=0.5, alambda_min=0.1, alambda_max=1.0, nrrz=1, nchange=1,
 * ncgscf=200, nretcg=2000. */
typedef struct rs_solver_prm {
  int northo, nsdmax, nprecon_cg, nprecon_diis, ndiismax;
  int nrrz, nchange, ncgscf, nretcg;
  double epssd, eps_eig_diis, alambda_diis, alambda_min, alambda_max;
} rs_solver_prm;

/* Band arrays: psi, spsi (S psi; pass sss=NULL and spsi=psi for
 * norm-conserving S=1), hpsi (M bands each), rp (<p|psi>, M x natom x nprjmx),
 * all device; sval / resid host arrays of M doubles.  _f64 = plain FP64
 * path, _f32 = mixed path (FP32 band arrays, FP64 rp, dots and matrices);
 * veff has the band arrays' precision. */

/* orthogonalization_r_01 with l_inp=0 (orthogonalization8f.F90:93-376): all
 * bands S-orthonormalised in order by Cholesky-QR (tensor-core Gram and
 * rotation for _f32); cmpt recomputes <p|psi> and S psi first
 * (key_ortho_cmpt_innerproduct). */
int rs_orthogonalize_f64(const rs_geom* g, const double* sss, int M, double* psi, double* spsi,
                         double* rp, int cmpt, void* stream);
int rs_orthogonalize_f32(const rs_geom* g, const double* sss, int M, float* psi, float* spsi,
                         double* rp, int cmpt, void* stream);
/* orthogonalization_r_01 with l_inp=l+1: band l against bands 0..l-1 and
 * normalised (the level-1 path used inside kscg_r). */
int rs_orthogonalize_band_f64(const rs_geom* g, const double* sss, int M, int l, double* psi,
                              double* spsi, double* rp, int cmpt, void* stream);
int rs_orthogonalize_band_f32(const rs_geom* g, const double* sss, int M, int l, float* psi,
                              float* spsi, double* rp, int cmpt, void* stream);
/* rayleighritz_r (rayleigh-ritz8f.F90:22-125): l_rrb recomputes H psi into
 * hpsi first (rayleighritz_hamiltonian_r); hpsi is work space on exit. */
int rs_rayleighritz_f64(const rs_geom* g, const double* veff, const double* dij,
                        const double* sss, int M, double* psi, double* spsi, double* rp,
                        double* hpsi, int l_rrb, double* sval, void* stream);
int rs_rayleighritz_f32(const rs_geom* g, const float* veff, const double* dij,
                        const double* sss, int M, float* psi, float* spsi, double* rp,
                        float* hpsi, int l_rrb, double* sval, void* stream);
/* kscg_r (kscg8f.F90:7-489): band-by-band preconditioned CG with the 2x2
 * Rayleigh-Ritz update; itmax = max iterations over bands. */
int rs_kscg_f64(const rs_geom* g, const double* veff, const double* dij, const double* sss,
                const rs_solver_prm* prm, int M, double* psi, double* spsi, double* rp,
                double* hpsi, double* sval, double* resid, int* itmax, void* stream);
int rs_kscg_f32(const rs_geom* g, const float* veff, const double* dij, const double* sss,
                const rs_solver_prm* prm, int M, float* psi, float* spsi, double* rp,
                float* hpsi, double* sval, double* resid, int* itmax, void* stream);
/* ksdiis_r (ksdiis8f.F90:8-712): RMM-DIIS sweeps with one trial step per
 * band; l_hsv orthogonalises all bands and recomputes H psi afterwards.
 * resid is read (bands whose 2x2 solve degenerates keep their value). */
int rs_ksdiis_f64(const rs_geom* g, const double* veff, const double* dij, const double* sss,
                  const rs_solver_prm* prm, int M, int l_hsv, double* psi, double* spsi,
                  double* rp, double* hpsi, double* sval, double* resid, int* ksconv,
                  void* stream);
int rs_ksdiis_f32(const rs_geom* g, const float* veff, const double* dij, const double* sss,
                  const rs_solver_prm* prm, int M, int l_hsv, float* psi, float* spsi,
                  double* rp, float* hpsi, double* sval, double* resid, int* ksconv,
                  void* stream);
/* reorderstates (reorderstates8f.F90:8-124): stable ascending order of sval;
 * psi, spsi, rp, sval, resid permuted. */
int rs_reorder_f64(const rs_geom* g, const double* sss, int M, double* psi, double* spsi,
                   double* rp, double* sval, double* resid, void* stream);
int rs_reorder_f32(const rs_geom* g, const double* sss, int M, float* psi, float* spsi,
                   double* rp, double* sval, double* resid, void* stream);
/* scf_diag (scf_diag8f.F90:6-316), real path, one k-point and spin: RR
 * before (nrrz>0) or after (nrrz<0), CG while iscf<=ncgscf or every nretcg,
 * DIIS otherwise, reorder every nchange. */
int rs_scf_diag_f64(const rs_geom* g, const double* veff, const double* dij, const double* sss,
                    const rs_solver_prm* prm, int iscf, int M, double* psi, double* spsi,
                    double* rp, double* hpsi, double* sval, double* resid, int* ksconv,
                    int* ksitmax, void* stream);
int rs_scf_diag_f32(const rs_geom* g, const float* veff, const double* dij, const double* sss,
                    const rs_solver_prm* prm, int iscf, int M, float* psi, float* spsi,
                    double* rp, float* hpsi, double* sval, double* resid, int* ksconv,
                    int* ksitmax, void* stream);

/* ---- SCF potentials and mixing (periodic, one spin) --------------------- */
/* trans_d2c_vh / trans_d2c_vxc for nperi=3 (trans8f.F90:93-152, 415-454):
 * out(dev, coarse nx*ny*nz) = transpose of the coarse->dense interpolation
 * applied to in(dev, dense 2nx*2ny*2nz) / 8, with the periodic halo fold of
 * overlap_interpolation nflag=2.  Needs n >= 2nf on each axis. */
int rs_interp_d2c(int nx, int ny, int nz, int nf, const double* in, double* out,
                  void* stream);
/* vxpot_lda_pz (vxpot8f.F90:126-155): vx, ex(dev) from rho(dev), n points. */
int rs_vxc_pz(long n, const double* rho, double* vx, double* ex, void* stream);
/* scf_potentials' veff (scf_potentials8f.F90:256-267, no bias field):
 * veff = vx + (vloc + vh); writes the FP64 and/or the FP32 copy (either
 * pointer may be NULL, not both). */
int rs_veff_sum(long n, const double* vx, const double* vloc, const double* vh, double* veff,
                float* veff32, void* stream);
/* scf_diffcharge + kukan8f.F90:672-673: *diff(host) = sqrt(sum (rho_i -
 * rho_o)^2 dx dy dz / (8 xmax ymax zmax)); synchronises the stream. */
int rs_diffcharge(long n, const double* rho_o, const double* rho_i, double dx, double dy,
                  double dz, double xmax, double ymax, double zmax, double* diff,
                  void* stream);
/* scf_chargemixing with modified Broyden (scf_chargemixing8f.F90:59-168,
 * 214-657), grid density of one spin: a mixer keeps nbrydn (2..63) history
 * vectors of n points on the device.  Each rs_mixer_step is one call of
 * scf_chargemixing: rho_i(dev) holds the last input density and receives
 * the next one; the first step copies rho_o.  Synchronises the stream. */
typedef struct rs_mixer rs_mixer;
int rs_mixer_create(rs_mixer** m, long n, int nbrydn, double eta);
int rs_mixer_step(rs_mixer* m, const double* rho_o, double* rho_i, double dvol, void* stream);
int rs_mixer_destroy(rs_mixer* m);

/* ---- forces ------------------------------------------------------------- */
/* force_eig_r (force8f.F90:9-195), one k-point and spin: the nonlocal force
 * fxyz(dev, [3][natom]: x forces, then y, then z) = -sum_l 2 occ_l sum_ij
 * <p_i|psi_l> (D - sval_l S)_ij <p_j|d psi_l>, with d the nf-order first
 * derivative (force_r_02/03/04, force8f.F90:409-490).  dij and sss are per
 * atom [natom][nprjmx][nprjmx] (dev); sss = NULL for norm-conserving sets.
 * psi [nb][N], sval and occ (fnele) [nb] are device arrays.  The FP64 form
 * matches the strict oracle bit for bit; the FP32 form takes FP32 bands and
 * accumulates in FP64. */
int rs_force_nl_f64(const rs_geom* g, const double* dij, const double* sss, const double* psi,
                    const double* sval, const double* occ, int nb, double* fxyz, void* stream);
int rs_force_nl_f32(const rs_geom* g, const double* dij, const double* sss, const float* psi,
                    const double* sval, const double* occ, int nb, double* fxyz, void* stream);

/* rs_hartree_cg for the mixed-precision path: the same CG (restart every
 * ncgres, the same stopping rule on the residual) with p, A p and r in FP32
 * and vh, every dot product and every residual norm in FP64.  The residual
 * is recomputed in FP64 as b - A vh ("reliable update") whenever its FP32
 * recurrence has dropped tenfold since the last recomputation, and before
 * the solve stops, so the attainable accuracy is that of the FP64 solve.
 * rho and vh are FP64 as in rs_hartree_cg.  Grids with odd nx or odd nfh run
 * the FP64 iteration. */
int rs_hartree_cg_f32(int nx, int ny, int nz, int nfh, double xmax, double ymax, double zmax,
                      double epsvh, int ncgmin, int ncgmax, int ncgres, const double* rho,
                      double* vh, int* iters, double* dp, void* stream);

/* rs_hartree_cg for callers that cannot allocate device memory (a host code
 * that handed all device memory to its own pool, a framework whose caching
 * allocator owns the GPU, work issued where the driver's allocation lock must
 * not be taken).  Same arguments, results and iterates as rs_hartree_cg, but
 * the work vectors live in a fixed array inside the library (about 10.5 MB
 * per GPU, held until exit), so grids are limited to 262144 points (64^3);
 * larger grids return RS_EINVAL.  Every call looks up the array's device
 * address in the current context and runs its iterations as plain kernel
 * launches (no CUDA graph is instantiated on any stream).  Calls that overlap
 * on one GPU share the array and race.  This entry point has no counterpart
 * in the reference. */
int rs_hartree_cg_noalloc(int nx, int ny, int nz, int nfh, double xmax, double ymax,
                          double zmax, double epsvh, int ncgmin, int ncgmax, int ncgres,
                          const double* rho, double* vh, int* iters, double* dp, void* stream);

/* ---- many small cells in one launch --------------------------------------- */
/* H psi (FP32 bands) of ncell independent cells, each as rs_hpsi_f32 would
 * compute it through the per-point gather (kslaplacian_r then
 * nonlocaloperation_r_02 per cell: kslaplacian8f.F90:23-261,
 * nonlocaloperation8f.F90:149-235), in one persistent launch over a device
 * table of the cells, for sets of small cells (tens of 20-40^3 grids) that a
 * launch per cell would leave mostly idle.
 *   rs_hpsi_batch_create: plan over the geometries and band counts nb[c];
 *   rs_hpsi_batch_set_f32: per-cell device pointers (veff, D per atom,
 *     <p|psi>, psi, H psi); waits for the device, so no run may be in flight;
 *   rs_hpsi_batch_run_f32: the first run times the candidate launch shapes
 *     and keeps the fastest (rs_hpsi_batch_info reports it); with use_graph
 *     and a non-null stream the launch is captured once into a CUDA graph and
 *     replayed on later runs (a new set_f32 drops the graph).
 * Returns 0, or a negative status (rs_last_error). */
typedef struct rs_hpsi_batch rs_hpsi_batch;
int rs_hpsi_batch_create(rs_hpsi_batch** plan, int ncell, const rs_geom* const* geoms,
                         const int* nb);
int rs_hpsi_batch_set_f32(rs_hpsi_batch* plan, const float* const* veff,
                          const double* const* dij, const double* const* rp,
                          const float* const* psi, float* const* hpsi);
int rs_hpsi_batch_run_f32(rs_hpsi_batch* plan, int use_graph, void* stream);
/* the autotuned shape; returns 1 before the first run */
int rs_hpsi_batch_info(const rs_hpsi_batch* plan, int* threads_per_cta, int* bands_per_item,
                       int* ctas_per_sm);
/* fixes the launch shape instead of the first run's autotuning (threads per
 * CTA 64/128/256, bands per item 1/2/4/8, CTAs per SM 1-16); every shape
 * gives the same bits.  No counterpart in the reference. */
int rs_hpsi_batch_set_shape(rs_hpsi_batch* plan, int threads_per_cta, int bands_per_item,
                            int ctas_per_sm);
int rs_hpsi_batch_destroy(rs_hpsi_batch* plan);

/* ---- device-resident state handle (the drop-in surface of scf_diag and
 * scf_charge: kukan8f.F90:466-487, 605-622, 647-662) --------------------- */
/* One cell and one k-point/spin: psi, S psi, H psi (M x N, precision 32 =
 * the mixed path or 64 = the plain FP64 path), <p|psi> (FP64), veff, D and S
 * stay on the GPU between calls; host memory is read at upload and written
 * only for results (sval, residual_states, rho, psi for checkpoints).  All
 * work runs on the stream given to rs_create; every call returns when its
 * results are in place.  A state is used from one host thread.
 *   rs_create: grid (dx, dy, dz spacings), band count, precision;
 *   rs_upload_geometry: as rs_geom_create, plus D (natom*nprjmx^2, required
 *     with atoms) and S (same size, NULL for S = 1), host arrays;
 *   rs_set_potential: veff (host, FP64, N), stored in the state's precision;
 *   rs_upload_bands: psi (host, M x N in the state's precision); S psi starts
 *     as a copy, H psi and <p|psi> as zeros (kukan's state before its first
 *     orthogonalisation);
 *   rs_orthogonalize: rs_orthogonalize_* on the state;
 *   rs_hpsi: H psi of all bands from psi and <p|psi>;
 *   rs_diag_step: rs_scf_diag_* on the state; sval, resid host (M, in/out);
 *   rs_density: rho (host, N) = sum_b occ_b psi_b^2 with occ host (M);
 *   rs_download_bands: psi to host;
 *   rs_state_arrays: the device pointers, for the other entry points. */
typedef struct rs_state rs_state;
int rs_create(rs_state** s, int precision, int nx, int ny, int nz, int nf, double dx, double dy,
              double dz, int nbands, void* stream);
int rs_upload_geometry(rs_state* s, int natom, int nprjmx, int num_list, const int* nprj,
                       const int* natinf, const int* lst, const double* vnlocp,
                       const double* dij, const double* sss);
int rs_set_potential(rs_state* s, const double* veff);
int rs_upload_bands(rs_state* s, const void* psi);
int rs_orthogonalize(rs_state* s, int cmpt);
int rs_hpsi(rs_state* s);
int rs_diag_step(rs_state* s, const rs_solver_prm* prm, int iscf, double* sval, double* resid,
                 int* ksconv, int* ksitmax);
int rs_density(rs_state* s, const double* occ, double* rho);
int rs_download_bands(rs_state* s, void* psi);
int rs_state_arrays(rs_state* s, void** psi, void** spsi, void** hpsi, double** rp, void** veff);
int rs_destroy(rs_state* s);

/* ---- local pseudopotential, ion-ion energy, initial bands (nperi = 3) ---- */
/* Soft local part of pseudocalc_02 case (3) with its real-space images
 * (pseudocalc8f.F90:1443-1568), summed over the atoms as pseudocalc_03 does
 * (:1600-1678), on the coarse grid: vsoft (device, N) is overwritten.  Host
 * inputs: atxyz (x, y, z per atom) and prm (5 per atom: cp1 = the valence
 * charge, and a, b, c of tools_bisec (tools8f.F90:922-953), and
 * rcut = radial(nradct)); veta and new_pw{x,y,z} are kukan's Ewald
 * parameters (read_input_kukan8f.F90:273-276). */
int rs_vloc_soft(int natom, const double* atxyz, const double* prm, int nx, int ny, int nz,
                 double dx, double dy, double dz, double xmax, double ymax, double zmax,
                 double veta, int npwx, int npwy, int npwz, double* vsoft, void* stream);

/* Hard local part of pseudocalc_02 (pseudocalc8f.F90:1245-1290) on the dense
 * grid (nmesh points per coarse spacing, the list of pseudocalc_01b within
 * rcut*psctoff, :1035-1144), added to dense (device, 8N for nmesh = 2) atom by
 * atom as pseudocalc_04 does (:1682-1706).  Host inputs: atxyz, spe (species
 * index per atom), per species sprm (rcut, rcuts = rcut*psftrad, filpp) and
 * nqct, coef (nspe x (nqmx+1): the local-part Fourier-Bessel coefficients
 * coef(0:nqmx, 0) of filterpseudopotentials8f.F90:107-131); npxmax.. are the
 * coarse list half-widths of tools_listvecdim. */
int rs_vloc_hard_add(int natom, const double* atxyz, const int* spe, int nspe,
                     const double* sprm, const int* nqct, int nqmx, const double* coef, int nx,
                     int ny, int nz, double dx, double dy, double dz, double xmax, double ymax,
                     double zmax, int nmesh, int npxmax, int npymax, int npzmax,
                     double psctoff, double eps, int nfiltyp, double* dense, void* stream);

/* Ewald energy of the ions, eneat of totalenergy_space_03 case (3)
 * (totalenergy8f.F90:520-565), and, when force (host, 3 per atom) is not
 * NULL, its forces (the ion-ion part of force8f.F90:1900-1950).  Host inputs
 * atxyz and q (cp1 per atom); energy (host) in Ha.  Returns after the
 * result is on the host. */
int rs_ewald(int natom, const double* atxyz, const double* q, double xmax, double ymax,
             double zmax, double veta, int npwx, int npwy, int npwz, double* energy,
             double* force, void* stream);

/* kukan's initial bands, setup_initialwave real branch
 * (setup_initialwave8f.F90:48-130): band l of atom a is exp(-zs_a r) times
 * 1 (l < natom), x, y, z (next 3 natom) or the five d forms (when
 * neig > 4 natom), r the minimum-image distance, normalised to
 * sum psi^2 dV = 1.  zs (host, per atom) = cp1 * zs_pre; psi device
 * (neig x N). */
int rs_initial_wave_f64(int natom, const double* atxyz, const double* zs, int neig, int nx,
                        int ny, int nz, double dx, double dy, double dz, double xmax,
                        double ymax, double zmax, double* psi, void* stream);
int rs_initial_wave_f32(int natom, const double* atxyz, const double* zs, int neig, int nx,
                        int ny, int nz, double dx, double dy, double dz, double xmax,
                        double ymax, double zmax, float* psi, void* stream);

/* ---- forces by one adjoint pass over the bands --------------------------- */
/* Local-pseudopotential part of the atomic forces as the exact derivative
 * of E_loc = dV sum_p rho(p) vloc_coarse(p), vloc_coarse = d2c(c2d(soft) +
 * hard) built as rs_vloc_soft / rs_vloc_hard_add do: with d2c the adjoint of
 * c2d (over 8), F_a = dV sum_p rho_soft(p) grad soft_a(p) + dV/8
 * sum_q rho_dense(q) grad hard_a(q), where rho_dense = c2d(rho) and
 * rho_soft = d2c(rho_dense) (device, coarse and dense).  The gradients are
 * those kukan stores as dvlocd*_scw and dvlocd*_hdp (pseudocalc8f.F90:
 * 1252-1289, 1443-1568), summed as force_01 does (force8f.F90:2016-2109) but
 * recomputed instead of stored; the reciprocal part runs as a separable
 * transform of rho_soft.  Arguments as rs_vloc_soft (prm) and
 * rs_vloc_hard_add (spe .. coef, nmesh .. nfiltyp); force: host, 3 per atom
 * (Ha/bohr), returned after it is on the host. */
int rs_force_local(int natom, const double* atxyz, const double* prm, const int* spe, int nspe,
                   const double* sprm, const int* nqct, int nqmx, const double* coef, int nx,
                   int ny, int nz, double dx, double dy, double dz, double xmax, double ymax,
                   double zmax, double veta, int npwx, int npwy, int npwz, int nmesh,
                   int npxmax, int npymax, int npzmax, double psctoff, double eps,
                   int nfiltyp, const double* rho_soft, const double* rho_dense, double* force,
                   void* stream);

/* Projector part of the atomic forces as the exact derivative of the
 * discrete energy: F_a = 2 sum_l occ_l sum_ij (D_a - sval_l S_a)_ij
 * <p_i|psi_l> <grad p_j|psi_l> (the quantity force_eig_r forms with
 * finite-difference band derivatives, force8f.F90:9-195).  The projector
 * values and gradients are recomputed at every sphere-list point from the
 * radial tables, nothing per projector is stored: tabs (host, ntab x nr) on
 * the radial grid i*dr, linearly interpolated and zero from r >= rcut; per
 * projector j its table prj_tab[j], angular momentum prj_l[j] and real
 * harmonic prj_form[j] (0: s; 1-3: x, y, z; 4-8: x^2-y^2, -zx, 3z^2-r^2, -yz,
 * xy, each over r^l, normalised as pseudocalc8f.F90:2962-2970), times
 * dx dy dz.  Host lists: atxyz (3 per atom), natxyz ([3][natom]), natinf,
 * lstxyz ([3][natom*num_list] offsets), lst (natom*num_list point indices)
 * from rs_sphere_lists.  Device: dij, sss ([natom][nprj][nprj], sss NULL for
 * NC), psi [nb][N], sval, occ [nb].  force: host, 3 per atom (Ha/bohr);
 * rp: NULL or device [nb][natom][nprj], the recomputed <p|psi>.  Returns
 * after force is on the host. */
int rs_force_adjoint_f64(int natom, int nprj, int num_list, const double* atxyz,
                         const int* natxyz, const int* natinf, const int* lstxyz, const int* lst,
                         int ntab, int nr, double dr, const double* tabs, const int* prj_tab,
                         const int* prj_l, const int* prj_form, double rcut, int nx, int ny,
                         int nz, double dx, double dy, double dz, const double* dij,
                         const double* sss, const double* psi, const double* sval,
                         const double* occ, int nb, double* force, double* rp, void* stream);
int rs_force_adjoint_f32(int natom, int nprj, int num_list, const double* atxyz,
                         const int* natxyz, const int* natinf, const int* lstxyz, const int* lst,
                         int ntab, int nr, double dr, const double* tabs, const int* prj_tab,
                         const int* prj_l, const int* prj_form, double rcut, int nx, int ny,
                         int nz, double dx, double dy, double dz, const double* dij,
                         const double* sss, const float* psi, const double* sval,
                         const double* occ, int nb, double* force, double* rp, void* stream);

/* ---- fixed-tree reductions (shared order with the oracle) --------------- */
/* out(dev, 1 double) = sum_i a_i b_i in the documented block tree. */
int rs_dot_f64(long n, const double* a, const double* b, double* out, void* stream);
int rs_dot_f32(long n, const float* a, const float* b, double* out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
