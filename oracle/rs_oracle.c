/*
 * rs_oracle.c -- CPU FP64 restatement of the RSPACE kukan hot path.
 *
 * TEST INFRASTRUCTURE: only tests/, __graft_entry__.smoke() and the
 * cpu_baseline / reference legs of bench.py load this file's shared object.
 * It is the checker, never the product.  Reference files are cited relative
 * to RSPACEes.v08.01/kukan/.
 *
 * Evaluation order: each Fortran `s = s + a*b` is fma(a, b, s) evaluated in
 * source order (gfortran's FMA contraction without reassociation), so the
 * stencil, projector, density and interpolation routines reproduce a
 * single-threaded run of the reference bit for bit.  Long reductions that the
 * reference splits over OpenMP threads (order undefined there) use the fixed
 * tree of orc_tree_dot, which the CUDA reductions reproduce exactly.
 */
#include "rs_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static inline long wrap(long i, long n) {
  i %= n;
  return i < 0 ? i + n : i;
}

/* tools_definefdcoef (tools8f.F90:144-237). */
void orc_fdcoef(int nf, double a[9]) {
  for (int i = 0; i < 9; ++i) a[i] = 0.0;
  switch (nf) {
    case 1: a[0] = -2.0; a[1] = 1.0; break;
    case 2: a[0] = -5.0 / 2.0; a[1] = 4.0 / 3.0; a[2] = -1.0 / 12.0; break;
    case 3: a[0] = -49.0 / 18.0; a[1] = 3.0 / 2.0; a[2] = -3.0 / 20.0; a[3] = 1.0 / 90.0; break;
    case 4:
      a[0] = -205.0 / 72.0; a[1] = 8.0 / 5.0; a[2] = -1.0 / 5.0; a[3] = 8.0 / 315.0;
      a[4] = -1.0 / 560.0;
      break;
    case 5:
      a[0] = -36883.0 / 12600.0; a[1] = 5.0 / 3.0; a[2] = -5.0 / 21.0; a[3] = 5.0 / 126.0;
      a[4] = -5.0 / 1008.0; a[5] = 1.0 / 3150.0;
      break;
    case 6:
      a[0] = -5369.0 / 1800.0; a[1] = 12.0 / 7.0; a[2] = -15.0 / 56.0; a[3] = 10.0 / 189.0;
      a[4] = -1.0 / 112.0; a[5] = 2.0 / 1925.0; a[6] = -1.0 / 16632.0;
      break;
    default: break; /* nf=7,8 are decimal tables in the reference; not used here */
  }
}

/* xx(m)=acfd(m)/dx/dx*(-0.5d0)  (kslaplacian8f.F90:40-66). */
void orc_lap_coefs(int nf, double dx, double dy, double dz, double cx[9], double cy[9],
                   double cz[9]) {
  double a[9];
  orc_fdcoef(nf, a);
  for (int m = 0; m < 9; ++m) {
    cx[m] = a[m] / dx / dx * (-0.5);
    cy[m] = a[m] / dy / dy * (-0.5);
    cz[m] = a[m] / dz / dz * (-0.5);
  }
}

/* ------------------------------------------------------------------------ */
/* Fixed reduction tree shared with the CUDA kernels (csrc/reduce.cuh):
 *   chunk c covers [4096c, 4096c+4096); lane t in 0..255 accumulates
 *   elements 4096c + t + 256k, k = 0..15, with fma from 0; the 256 lane sums
 *   fold as eight 32-lane shuffle trees (offsets 16,8,4,2,1) followed by an
 *   8-way tree over the warp sums (offsets 4,2,1).  The chunk sums are folded
 *   the same way: lane t accumulates chunk sums t, t+256, ... (plain adds from
 *   0), then the same 256-lane tree. */
#define TREE_LANES 256
#define TREE_PER_LANE 16
#define TREE_CHUNK (TREE_LANES * TREE_PER_LANE)

static double tree_fold(double* s) {
  for (int w = 0; w < 8; ++w)
    for (int off = 16; off >= 1; off >>= 1)
      for (int l = 0; l < off; ++l) s[32 * w + l] = s[32 * w + l] + s[32 * w + l + off];
  double ws[8];
  for (int w = 0; w < 8; ++w) ws[w] = s[32 * w];
  for (int off = 4; off >= 1; off >>= 1)
    for (int l = 0; l < off; ++l) ws[l] = ws[l] + ws[l + off];
  return ws[0];
}

static double tree_final(long nblk, const double* part) {
  double s[TREE_LANES];
  for (int t = 0; t < TREE_LANES; ++t) {
    double acc = 0.0;
    for (long k = t; k < nblk; k += TREE_LANES) acc = acc + part[k];
    s[t] = acc;
  }
  return tree_fold(s);
}

double orc_tree_dot(long n, const double* a, const double* b) {
  long nblk = (n + TREE_CHUNK - 1) / TREE_CHUNK;
  if (nblk == 0) return 0.0;
  double* part = (double*)malloc(sizeof(double) * nblk);
  for (long c = 0; c < nblk; ++c) {
    double s[TREE_LANES];
    for (int t = 0; t < TREE_LANES; ++t) {
      double acc = 0.0;
      for (int k = 0; k < TREE_PER_LANE; ++k) {
        long i = c * TREE_CHUNK + (long)k * TREE_LANES + t;
        if (i < n) acc = fma(a[i], b[i], acc);
      }
      s[t] = acc;
    }
    part[c] = tree_fold(s);
  }
  double r = tree_final(nblk, part);
  free(part);
  return r;
}

double orc_tree_dot_f(long n, const float* a, const float* b) {
  long nblk = (n + TREE_CHUNK - 1) / TREE_CHUNK;
  if (nblk == 0) return 0.0;
  double* part = (double*)malloc(sizeof(double) * nblk);
  for (long c = 0; c < nblk; ++c) {
    double s[TREE_LANES];
    for (int t = 0; t < TREE_LANES; ++t) {
      double acc = 0.0;
      for (int k = 0; k < TREE_PER_LANE; ++k) {
        long i = c * TREE_CHUNK + (long)k * TREE_LANES + t;
        if (i < n) acc = fma((double)a[i], (double)b[i], acc);
      }
      s[t] = acc;
    }
    part[c] = tree_fold(s);
  }
  double r = tree_final(nblk, part);
  free(part);
  return r;
}

/* ------------------------------------------------------------------------ */
/* kslaplacian_r (kslaplacian8f.F90:23-557; nf=4 at 207-261): three passes
 * x, y, z accumulated into out.  The periodic halo that
 * overlap_finitedifference_r builds with one rank and nperi=3
 * (overlap_finitedifference8f.F90:97-139) is the (i mod n) index used here. */
void orc_kslaplacian(int nx, int ny, int nz, int nf, double dx, double dy, double dz,
                     const double* psi, const double* veff, double* out, int nb) {
  double cx[9], cy[9], cz[9];
  orc_lap_coefs(nf, dx, dy, dz, cx, cy, cz);
  const long N = (long)nx * ny * nz;
  for (int b = 0; b < nb; ++b) {
    const double* v = psi + (long)b * N;
    double* o = out + (long)b * N;
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const long p = ((long)iz * ny + iy) * nx + ix;
          const long row = ((long)iz * ny + iy) * nx;
          double acc = o[p];
          for (int m = nf; m >= 1; --m) acc = fma(cx[m], v[row + wrap(ix - m, nx)], acc);
          const double diag = cx[0] + cy[0] + cz[0] + veff[p];
          acc = fma(diag, v[p], acc);
          for (int m = 1; m <= nf; ++m) acc = fma(cx[m], v[row + wrap(ix + m, nx)], acc);
          /* y pass */
          for (int m = nf; m >= 1; --m)
            acc = fma(cy[m], v[((long)iz * ny + wrap(iy - m, ny)) * nx + ix], acc);
          for (int m = 1; m <= nf; ++m)
            acc = fma(cy[m], v[((long)iz * ny + wrap(iy + m, ny)) * nx + ix], acc);
          /* z pass */
          for (int m = nf; m >= 1; --m)
            acc = fma(cz[m], v[(wrap(iz - m, nz) * ny + iy) * nx + ix], acc);
          for (int m = 1; m <= nf; ++m)
            acc = fma(cz[m], v[(wrap(iz + m, nz) * ny + iy) * nx + ix], acc);
          o[p] = acc;
        }
  }
}

/* ksprecondition (ksprecondition8f.F90:8-39): 1/2 psi + 1/12 * 6 neighbours. */
void orc_precondition(int nx, int ny, int nz, const double* in, double* out, int nb) {
  const double c = 1.0 / 12.0;
  const long N = (long)nx * ny * nz;
  for (int b = 0; b < nb; ++b) {
    const double* v = in + (long)b * N;
    double* o = out + (long)b * N;
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const long p = ((long)iz * ny + iy) * nx + ix;
          double t = c * v[((long)iz * ny + iy) * nx + wrap(ix - 1, nx)];
          t = fma(c, v[((long)iz * ny + wrap(iy - 1, ny)) * nx + ix], t);
          t = fma(c, v[(wrap(iz - 1, nz) * ny + iy) * nx + ix], t);
          t = fma(0.5, v[p], t);
          t = fma(c, v[(wrap(iz + 1, nz) * ny + iy) * nx + ix], t);
          t = fma(c, v[((long)iz * ny + wrap(iy + 1, ny)) * nx + ix], t);
          t = fma(c, v[((long)iz * ny + iy) * nx + wrap(ix + 1, nx)], t);
          o[p] = t;
        }
  }
}

/* nonlocaloperation_r_01 (nonlocaloperation8f.F90:9-53): <p_j,a|psi_b>,
 * a sequential gather-dot per (atom, projector, band). */
void orc_nl_dot(int natom, int nprjmx, int num_list, const int* nprj, const int* natinf,
                const int* lst, const double* v, const double* psi, long N, int nb,
                double* rp) {
  for (int b = 0; b < nb; ++b) {
    const double* x = psi + (long)b * N;
    for (int a = 0; a < natom; ++a) {
      const int* l = lst + (long)a * num_list;
      for (int j = 0; j < nprjmx; ++j) {
        double t = 0.0;
        if (j < nprj[a]) {
          const double* vj = v + ((long)a * nprjmx + j) * num_list;
          for (int ii = 0; ii < natinf[a]; ++ii) t = fma(vj[ii], x[l[ii]], t);
        }
        rp[((long)b * natom + a) * nprjmx + j] = t;
      }
    }
  }
}

/* nonlocaloperation_r_02 (nonlocaloperation8f.F90:149-235):
 * t_i = (sum_j rp_j m(j,i)) / dV, avr = sum_i t_i p_i, scatter-add in atom
 * order.  mat is dij (nhs=1) or sss (nhs=0), one matrix per atom. */
void orc_nl_apply(int natom, int nprjmx, int num_list, const int* nprj, const int* natinf,
                  const int* lst, const double* v, const double* mat, double dvol,
                  const double* rp, long N, int nb, double* out) {
  const double dxyzin = 1.0 / dvol;
  double* t = (double*)malloc(sizeof(double) * (nprjmx > 0 ? nprjmx : 1));
  for (int b = 0; b < nb; ++b) {
    double* o = out + (long)b * N;
    for (int a = 0; a < natom; ++a) {
      const int P = nprj[a];
      if (P <= 0) continue;
      const double* r = rp + ((long)b * natom + a) * nprjmx;
      const double* m = mat + (long)a * nprjmx * nprjmx;
      for (int i = 0; i < P; ++i) {
        double s = 0.0;
        for (int j = 0; j < P; ++j) s = fma(r[j], m[i * nprjmx + j], s);
        t[i] = s * dxyzin;
      }
      const int* l = lst + (long)a * num_list;
      const double* va = v + (long)a * nprjmx * num_list;
      for (int ii = 0; ii < natinf[a]; ++ii) {
        double avr = t[0] * va[ii];
        for (int j = 1; j < P; ++j) avr = fma(t[j], va[(long)j * num_list + ii], avr);
        o[l[ii]] = o[l[ii]] + avr;
      }
    }
  }
  free(t);
}

/* H psi exactly as kscg_r / rayleighritz_hamiltonian_r build it
 * (kscg8f.F90:147-183): hpsi = 0, nonlocal D-term, then the stencil passes. */
void orc_hpsi(int nx, int ny, int nz, int nf, double dx, double dy, double dz,
              const double* veff, int natom, int nprjmx, int num_list, const int* nprj,
              const int* natinf, const int* lst, const double* v, const double* dij,
              const double* rp, const double* psi, double* hpsi, int nb) {
  const long N = (long)nx * ny * nz;
  memset(hpsi, 0, sizeof(double) * N * nb);
  orc_nl_apply(natom, nprjmx, num_list, nprj, natinf, lst, v, dij, dx * dy * dz, rp, N, nb,
               hpsi);
  orc_kslaplacian(nx, ny, nz, nf, dx, dy, dz, psi, veff, hpsi, nb);
}

/* S psi as orthogonalization_r_01 builds it (orthogonalization8f.F90:187-210):
 * spsi = psi, then the sss-term (nhs=0). */
void orc_spsi(long N, int natom, int nprjmx, int num_list, const int* nprj,
              const int* natinf, const int* lst, const double* v, const double* sss,
              double dvol, const double* rp, const double* psi, double* spsi, int nb) {
  memcpy(spsi, psi, sizeof(double) * N * nb);
  orc_nl_apply(natom, nprjmx, num_list, nprj, natinf, lst, v, sss, dvol, rp, N, nb, spsi);
}

/* force_r_02/03/04 (force8f.F90:409-1612, nf=4 at 468-490): first-derivative
 * stencil avre = -a_nf v(+nf) ... - a_1 v(+1) + a_1 v(-1) ... + a_nf v(-nf). */
void orc_grad_coefs(int nf, double h, double a[5]) {
  for (int m = 0; m < 5; ++m) a[m] = 0.0;
  if (nf == 1) { a[1] = -0.5 / h; }
  if (nf == 2) { a[2] = 1.0 / 12.0 / h; a[1] = -8.0 / 12.0 / h; }
  if (nf == 3) { a[3] = -1.0 / 60.0 / h; a[2] = 9.0 / 60.0 / h; a[1] = -45.0 / 60.0 / h; }
  if (nf >= 4) {
    a[4] = 3.0 / 840.0 / h; a[3] = -32.0 / 840.0 / h;
    a[2] = 168.0 / 840.0 / h; a[1] = -672.0 / 840.0 / h;
  }
}

void orc_gradient(int nx, int ny, int nz, int nf, double h, int axis, const double* psi,
                  double* out) {
  double a[5];
  orc_grad_coefs(nf, h, a);
  const int nfu = nf > 4 ? 4 : nf;
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const long p = ((long)iz * ny + iy) * nx + ix;
        long pm[5], pp[5];
        for (int m = 1; m <= nfu; ++m) {
          if (axis == 0) {
            pm[m] = ((long)iz * ny + iy) * nx + wrap(ix - m, nx);
            pp[m] = ((long)iz * ny + iy) * nx + wrap(ix + m, nx);
          } else if (axis == 1) {
            pm[m] = ((long)iz * ny + wrap(iy - m, ny)) * nx + ix;
            pp[m] = ((long)iz * ny + wrap(iy + m, ny)) * nx + ix;
          } else {
            pm[m] = (wrap(iz - m, nz) * ny + iy) * nx + ix;
            pp[m] = (wrap(iz + m, nz) * ny + iy) * nx + ix;
          }
        }
        double acc = -(a[nfu] * psi[pp[nfu]]);
        for (int m = nfu - 1; m >= 1; --m) acc = fma(-a[m], psi[pp[m]], acc);
        for (int m = 1; m <= nfu; ++m) acc = fma(a[m], psi[pm[m]], acc);
        out[p] = acc;
      }
}

/* ------------------------------------------------------------------------ */
/* scf_charge_smt_r (scf_charge8f.F90:290-321): rho += (f*psi)*psi, bands in order. */
void orc_density(long N, int nb, const double* occ, const double* psi, double* rho) {
  for (long p = 0; p < N; ++p) rho[p] = 0.0;
  for (int b = 0; b < nb; ++b) {
    const double f = occ[b];
    const double* x = psi + (long)b * N;
    for (long p = 0; p < N; ++p) rho[p] = fma(f * x[p], x[p], rho[p]);
  }
}

/* interpolation, forward branch (interpolation8f.F90:8-100) with nmesh=2 and
 * the periodic halo of overlap_interpolation; Lagrange weights of order 2nf
 * from interpolation8f.F90:36-44. */
void orc_interp_weights(int nf, double aw[2][16]) {
  for (int k = 0; k < 2; ++k) {
    const double r = ((double)k + 0.5) * 0.5;
    for (int j = -nf + 1; j <= nf; ++j) {
      double w = 1.0;
      for (int i = -nf + 1; i <= nf; ++i)
        if (i != j) w = w * (r - (double)i) / ((double)j - (double)i);
      aw[k][j + nf - 1] = w;
    }
  }
}

void orc_interp_c2d(int nx, int ny, int nz, int nf, const double* in, double* out) {
  double aw[2][16];
  orc_interp_weights(nf, aw);
  const int Nx = 2 * nx, Ny = 2 * ny, Nz = 2 * nz;
  double* t1 = (double*)malloc(sizeof(double) * (long)Nx * ny * nz);
  double* t2 = (double*)malloc(sizeof(double) * (long)Nx * Ny * nz);
  for (int jz = 0; jz < nz; ++jz)
    for (int jy = 0; jy < ny; ++jy)
      for (int jd = 0; jd < Nx; ++jd) {
        const int k = (jd + 1) % 2, l0 = (jd + 1) / 2 - 1;
        double acc = 0.0;
        for (int i = -nf + 1; i <= nf; ++i)
          acc = fma(aw[k][i + nf - 1], in[((long)jz * ny + jy) * nx + wrap(l0 + i, nx)], acc);
        t1[((long)jz * ny + jy) * Nx + jd] = acc;
      }
  for (int jz = 0; jz < nz; ++jz)
    for (int jd = 0; jd < Ny; ++jd)
      for (int jx = 0; jx < Nx; ++jx) {
        const int k = (jd + 1) % 2, l0 = (jd + 1) / 2 - 1;
        double acc = 0.0;
        for (int i = -nf + 1; i <= nf; ++i)
          acc = fma(aw[k][i + nf - 1], t1[((long)jz * ny + wrap(l0 + i, ny)) * Nx + jx], acc);
        t2[((long)jz * Ny + jd) * Nx + jx] = acc;
      }
  for (int jd = 0; jd < Nz; ++jd)
    for (int jy = 0; jy < Ny; ++jy)
      for (int jx = 0; jx < Nx; ++jx) {
        const int k = (jd + 1) % 2, l0 = (jd + 1) / 2 - 1;
        double acc = 0.0;
        for (int i = -nf + 1; i <= nf; ++i)
          acc = fma(aw[k][i + nf - 1], t2[(wrap(l0 + i, nz) * Ny + jy) * Nx + jx], acc);
        out[((long)jd * Ny + jy) * Nx + jx] = acc;
      }
  free(t1);
  free(t2);
}

/* scf_hartee_laplacian (scf_hartree8f.F90:901-1004, nfh=4 branch): the x pass
 * starts from the first product, diagonal = hadx+hady+hadz. */
void orc_hartree_laplacian(int nx, int ny, int nz, int nfh, double ddx, double ddy,
                           double ddz, const double* v, double* av) {
  double a[9], cx[9], cy[9], cz[9];
  orc_fdcoef(nfh, a);
  for (int m = 1; m < 9; ++m) {
    cx[m] = a[m] / ddx / ddx * (-0.5);
    cy[m] = a[m] / ddy / ddy * (-0.5);
    cz[m] = a[m] / ddz / ddz * (-0.5);
  }
  const double hadx = a[0] / (ddx * ddx) * (-0.5);
  const double hady = a[0] / (ddy * ddy) * (-0.5);
  const double hadz = a[0] / (ddz * ddz) * (-0.5);
  const double diag = hadx + hady + hadz;
  for (int iz = 0; iz < nz; ++iz)
    for (int iy = 0; iy < ny; ++iy)
      for (int ix = 0; ix < nx; ++ix) {
        const long p = ((long)iz * ny + iy) * nx + ix;
        const long row = ((long)iz * ny + iy) * nx;
        double acc = cx[nfh] * v[row + wrap(ix - nfh, nx)];
        for (int m = nfh - 1; m >= 1; --m) acc = fma(cx[m], v[row + wrap(ix - m, nx)], acc);
        acc = fma(diag, v[p], acc);
        for (int m = 1; m <= nfh; ++m) acc = fma(cx[m], v[row + wrap(ix + m, nx)], acc);
        for (int m = nfh; m >= 1; --m)
          acc = fma(cy[m], v[((long)iz * ny + wrap(iy - m, ny)) * nx + ix], acc);
        for (int m = 1; m <= nfh; ++m)
          acc = fma(cy[m], v[((long)iz * ny + wrap(iy + m, ny)) * nx + ix], acc);
        for (int m = nfh; m >= 1; --m)
          acc = fma(cz[m], v[(wrap(iz - m, nz) * ny + iy) * nx + ix], acc);
        for (int m = 1; m <= nfh; ++m)
          acc = fma(cz[m], v[(wrap(iz + m, nz) * ny + iy) * nx + ix], acc);
        av[p] = acc;
      }
}

/* scf_hartree + scf_hartree_cg (scf_hartree8f.F90:84-89, 626-812) for nperi=3:
 * b = 2*pi*rho minus its mean, warm start from vh, running A.x in avhs,
 * restart every ncgres, stop on sqrt(r.r dV / Omega) <= epsvh.
 * Returns the iteration count. */
int orc_hartree_cg(int nx, int ny, int nz, int nfh, double xmax, double ymax, double zmax,
                   double epsvh, int ncgmin, int ncgmax, int ncgres, const double* rho,
                   double* vh, double* dp_out) {
  const long N = (long)nx * ny * nz;
  const double pi = acos(-1.0);
  const double ddx = 2.0 * xmax / nx, ddy = 2.0 * ymax / ny, ddz = 2.0 * zmax / nz;
  double* b = (double*)malloc(sizeof(double) * N);
  double* r = (double*)malloc(sizeof(double) * N);
  double* p = (double*)malloc(sizeof(double) * N);
  double* ap = (double*)malloc(sizeof(double) * N);
  double* avhs = (double*)malloc(sizeof(double) * N);
  double* q = (double*)malloc(sizeof(double) * N);
  double* one = (double*)malloc(sizeof(double) * N);
  for (long i = 0; i < N; ++i) {
    b[i] = 2.0 * pi * rho[i];
    q[i] = b[i] * ddx * ddy * ddz;
    one[i] = 1.0;
  }
  double bve = orc_tree_dot(N, q, one);
  bve = bve / (8.0 * xmax * ymax * zmax);
  for (long i = 0; i < N; ++i) b[i] = b[i] - bve;
  orc_hartree_laplacian(nx, ny, nz, nfh, ddx, ddy, ddz, vh, ap);
  for (long i = 0; i < N; ++i) {
    avhs[i] = ap[i];
    r[i] = b[i] - ap[i];
    p[i] = r[i];
  }
  int loop = 0;
  double dp = 0.0;
  for (;;) {
    ++loop;
    orc_hartree_laplacian(nx, ny, nz, nfh, ddx, ddy, ddz, p, ap);
    const double r1r = orc_tree_dot(N, r, r);
    const double pap = orc_tree_dot(N, p, ap);
    const double alph = r1r / pap;
    for (long i = 0; i < N; ++i) {
      vh[i] = fma(alph, p[i], vh[i]);
      avhs[i] = fma(alph, ap[i], avhs[i]);
    }
    for (long i = 0; i < N; ++i) r[i] = b[i] - avhs[i];
    const double r2r = orc_tree_dot(N, r, r);
    double beta = r2r / r1r;
    if (loop % ncgres == 0) beta = 0.0;
    for (long i = 0; i < N; ++i) p[i] = fma(beta, p[i], r[i]);
    dp = sqrt(r2r * ddx * ddy * ddz / (8.0 * xmax * ymax * zmax));
    if (loop < ncgmin) continue;
    if (loop >= ncgmax) break;
    if (dp > epsvh) continue;
    break;
  }
  if (dp_out) *dp_out = dp;
  free(b); free(r); free(p); free(ap); free(avhs); free(q); free(one);
  return loop;
}

/* ------------------------------------------------------------------------ */
/* pseudocalc_01b list vectors (pseudocalc8f.F90:691-693, 955-1033), one rank,
 * nperi=3.  rcut[a] is radial(nradct)*psctoff.  Returns 0, or -1 when an
 * atom's list exceeds num_list (the reference's stopp at :1025-1028). */
int orc_sphere_lists(int natom, const double* atx, const double* aty, const double* atz,
                     const double* rcut, int nxmax, int nymax, int nzmax, double dx,
                     double dy, double dz, int npxmax, int npymax, int npzmax, int nfdg,
                     int num_list, int* natx, int* naty, int* natz, int* natinf, int* lst,
                     int* lstx, int* lsty, int* lstz) {
  const double xmax = nxmax * dx, ymax = nymax * dy, zmax = nzmax * dz;
  const int ncpx = 2 * nxmax, ncpy = 2 * nymax, ncpz = 2 * nzmax;
  int status = 0;
  for (int a = 0; a < natom; ++a) {
    natx[a] = (int)((atx[a] + xmax + 0.5 * dx) / dx) - nxmax;
    naty[a] = (int)((aty[a] + ymax + 0.5 * dy) / dy) - nymax;
    natz[a] = (int)((atz[a] + zmax + 0.5 * dz) / dz) - nzmax;
    const double tx = atx[a] - (natx[a] * dx - 0.5 * dx);
    const double ty = aty[a] - (naty[a] * dy - 0.5 * dy);
    const double tz = atz[a] - (natz[a] * dz - 0.5 * dz);
    int l0 = 0;
    for (int iz = -npzmax + 1; iz <= npzmax; ++iz)
      for (int iy = -npymax + 1; iy <= npymax; ++iy)
        for (int ix = -npxmax + 1; ix <= npxmax; ++ix) {
          int hit = 0;
          for (int jz = -nfdg; jz <= nfdg && !hit; ++jz)
            for (int jy = -nfdg; jy <= nfdg && !hit; ++jy)
              for (int jx = -nfdg; jx <= nfdg && !hit; ++jx) {
                const double x = (ix + jx) * dx - tx;
                const double y = (iy + jy) * dy - ty;
                const double z = (iz + jz) * dz - tz;
                const double r = sqrt(x * x + y * y + z * z);
                if (r < rcut[a]) hit = 1;
              }
          if (!hit) continue;
          int i = ix + natx[a] + nxmax, j = iy + naty[a] + nymax, k = iz + natz[a] + nzmax;
          while (i > 2 * nxmax) i -= 2 * nxmax;
          while (i < 1) i += 2 * nxmax;
          while (j > 2 * nymax) j -= 2 * nymax;
          while (j < 1) j += 2 * nymax;
          while (k > 2 * nzmax) k -= 2 * nzmax;
          while (k < 1) k += 2 * nzmax;
          if (l0 >= num_list) { status = -1; continue; }
          lst[(long)a * num_list + l0] = ((k - 1) * ncpy + (j - 1)) * ncpx + (i - 1);
          if (lstx) lstx[(long)a * num_list + l0] = ix;
          if (lsty) lsty[(long)a * num_list + l0] = iy;
          if (lstz) lstz[(long)a * num_list + l0] = iz;
          ++l0;
        }
    natinf[a] = l0;
  }
  return status;
}

/* ------------------------------------------------------------------------ */
/* Cyclic Jacobi eigensolver for a symmetric n x n matrix (row-major a, only
 * read).  Stands in for LAPACK dsyev in rayleighritz_r (rayleigh-ritz8f.F90:89):
 * eigenvalues ascending in w, eigenvectors as columns of z (z[i*n+k] is
 * component i of vector k), each with its largest-magnitude component made
 * positive.  Returns the number of sweeps, or -1 without convergence. */
int orc_jacobi_eig(int n, double* a_in, double* w, double* z) {
  double* a = (double*)malloc(sizeof(double) * n * n);
  memcpy(a, a_in, sizeof(double) * n * n);
  for (int i = 0; i < n * n; ++i) z[i] = 0.0;
  for (int i = 0; i < n; ++i) z[i * n + i] = 1.0;
  int sweep = 0;
  for (; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        tot += a[i * n + j] * a[i * n + j];
        if (i != j) off += a[i * n + j] * a[i * n + j];
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < n - 1; ++p)
      for (int q = p + 1; q < n; ++q) {
        const double apq = a[p * n + q];
        if (apq == 0.0) continue;
        const double theta = (a[q * n + q] - a[p * n + p]) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < n; ++k) {
          const double akp = a[k * n + p], akq = a[k * n + q];
          a[k * n + p] = c * akp - s * akq;
          a[k * n + q] = s * akp + c * akq;
        }
        for (int k = 0; k < n; ++k) {
          const double apk = a[p * n + k], aqk = a[q * n + k];
          a[p * n + k] = c * apk - s * aqk;
          a[q * n + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < n; ++k) {
          const double zkp = z[k * n + p], zkq = z[k * n + q];
          z[k * n + p] = c * zkp - s * zkq;
          z[k * n + q] = s * zkp + c * zkq;
        }
        /* the annihilated pair is zero by construction; its computed value
           is rounding noise of size eps*|a_pp| */
        a[p * n + q] = 0.0;
        a[q * n + p] = 0.0;
      }
  }
  for (int i = 0; i < n; ++i) w[i] = a[i * n + i];
  /* sort ascending (stable selection) */
  for (int i = 0; i < n - 1; ++i) {
    int m = i;
    for (int j = i + 1; j < n; ++j)
      if (w[j] < w[m]) m = j;
    if (m != i) {
      double t = w[i]; w[i] = w[m]; w[m] = t;
      for (int k = 0; k < n; ++k) {
        double u = z[k * n + i]; z[k * n + i] = z[k * n + m]; z[k * n + m] = u;
      }
    }
  }
  for (int j = 0; j < n; ++j) {
    int im = 0;
    for (int i = 1; i < n; ++i)
      if (fabs(z[i * n + j]) > fabs(z[im * n + j])) im = i;
    if (z[im * n + j] < 0)
      for (int i = 0; i < n; ++i) z[i * n + j] = -z[i * n + j];
  }
  free(a);
  return sweep < 100 ? sweep : -1;
}

/* Closed-form eigen-decomposition of a symmetric 2x2 (row-major a) standing in
 * for the 2-dimensional dsyev calls of ksdiis_r (ksdiis8f.F90:427,477).
 * Eigenvalues ascending; vector k is (z[k], z[2+k]) with its largest
 * component positive (ties: the first).  The CUDA band kernels use the same
 * formula. */
void orc_eig2(const double a[4], double w[2], double z[4]) {
  const double p = a[0], q = a[3], r = 0.5 * (a[1] + a[2]);
  const double mean = 0.5 * (p + q), half = 0.5 * (p - q);
  const double rad = sqrt(half * half + r * r);
  w[0] = mean - rad;
  w[1] = mean + rad;
  if (r == 0.0) {
    if (p <= q) { z[0] = 1.0; z[2] = 0.0; z[1] = 0.0; z[3] = 1.0; }
    else        { z[0] = 0.0; z[2] = 1.0; z[1] = 1.0; z[3] = 0.0; }
    return;
  }
  /* vector for w[1]: (r, w1 - p) or (w1 - q, r), whichever is better conditioned */
  double u0, u1;
  if (half >= 0.0) { u0 = half + rad; u1 = r; }
  else             { u0 = r; u1 = rad - half; }
  const double nu = sqrt(u0 * u0 + u1 * u1);
  u0 /= nu; u1 /= nu;
  double v0 = -u1, v1 = u0; /* orthogonal vector for w[0] */
  if (fabs(u1) > fabs(u0) ? u1 < 0.0 : u0 < 0.0) { u0 = -u0; u1 = -u1; }
  if (fabs(v1) > fabs(v0) ? v1 < 0.0 : v0 < 0.0) { v0 = -v0; v1 = -v1; }
  z[0] = v0; z[2] = v1;
  z[1] = u0; z[3] = u1;
}

/* reorderstates rank (reorderstates8f.F90:38-50): a stable ascending rank. */
void orc_reorder_rank(int m, const double* sval, int* rank) {
  for (int j = 0; j < m; ++j) rank[j] = 0;
  rank[0] = 0;
  for (int j = 1; j < m; ++j)
    for (int i = 0; i < j; ++i) {
      if (sval[i] > sval[j]) rank[i] += 1;
      else rank[j] += 1;
    }
}
