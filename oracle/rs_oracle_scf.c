/*
 * rs_oracle_scf.c -- CPU restatement of the SCF potential and mixing steps of
 * kukan (TEST INFRASTRUCTURE ONLY, see rs_oracle.h): the dense-to-coarse
 * transfer, the PZ LDA potential, the veff sum, the SCF charge difference
 * and the modified Broyden charge mixing.  Same conventions as rs_oracle.c.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

/* ------------------------------------------------------------------------ */
/* interpolation(..., is=2) (interpolation8f.F90:98-214), nperi=3: the dense
 * halo is zero, so only interior dense points contribute; each pass sums its
 * contributions in the reference's loop order (offset i outer, dense index
 * inner, ascending).  Coarse arrays carry the halo -nf+1..n+nf (offset
 * nf-1).  Then v/nmesh^3 and the periodic fold of overlap_interpolation
 * nflag=2 (overlap_interpolation8f.F90:559-622 for x, and the y and z
 * branches after it): x, then y, then z, each over the full halo'd extent
 * of the other two axes. */
void orc_interp_d2c(int nx, int ny, int nz, int nf, const double* in, double* out) {
  double aw[2][16];
  orc_interp_weights(nf, aw);
  const int nf1 = nf - 1;
  const int Nx = 2 * nx, Ny = 2 * ny, Nz = 2 * nz;
  const int Hx = nx + 2 * nf, Hy = ny + 2 * nf, Hz = nz + 2 * nf;
  double* t2 = (double*)malloc(sizeof(double) * (long)Nx * Ny * Hz);  /* [cz][jy][jx] */
  double* t1 = (double*)malloc(sizeof(double) * (long)Nx * Hy * Hz);  /* [cz][cy][jx] */
  double* v = (double*)malloc(sizeof(double) * (long)Hx * Hy * Hz);   /* [cz][cy][cx] */
  /* z pass: dense (jx, jy, jz) -> (jx, jy, cz) */
  for (int cz = -nf1; cz <= nz + nf; ++cz)
    for (int jy = 1; jy <= Ny; ++jy)
      for (int jx = 1; jx <= Nx; ++jx) {
        double acc = 0.0;
        for (int iz = -nf1; iz <= nf; ++iz) {
          const int l = cz - iz;
          for (int jz = 2 * l; jz <= 2 * l + 1; ++jz)
            if (jz >= 1 && jz <= Nz)
              acc = fma(aw[jz % 2][iz + nf1],
                        in[((long)(jz - 1) * Ny + (jy - 1)) * Nx + (jx - 1)], acc);
        }
        t2[((long)(cz + nf1) * Ny + (jy - 1)) * Nx + (jx - 1)] = acc;
      }
  /* y pass */
  for (int cz = -nf1; cz <= nz + nf; ++cz)
    for (int cy = -nf1; cy <= ny + nf; ++cy)
      for (int jx = 1; jx <= Nx; ++jx) {
        double acc = 0.0;
        for (int iy = -nf1; iy <= nf; ++iy) {
          const int l = cy - iy;
          for (int jy = 2 * l; jy <= 2 * l + 1; ++jy)
            if (jy >= 1 && jy <= Ny)
              acc = fma(aw[jy % 2][iy + nf1],
                        t2[((long)(cz + nf1) * Ny + (jy - 1)) * Nx + (jx - 1)], acc);
        }
        t1[((long)(cz + nf1) * Hy + (cy + nf1)) * Nx + (jx - 1)] = acc;
      }
  /* x pass */
  for (int cz = -nf1; cz <= nz + nf; ++cz)
    for (int cy = -nf1; cy <= ny + nf; ++cy)
      for (int cx = -nf1; cx <= nx + nf; ++cx) {
        double acc = 0.0;
        for (int ix = -nf1; ix <= nf; ++ix) {
          const int l = cx - ix;
          for (int jx = 2 * l; jx <= 2 * l + 1; ++jx)
            if (jx >= 1 && jx <= Nx)
              acc = fma(aw[jx % 2][ix + nf1],
                        t1[((long)(cz + nf1) * Hy + (cy + nf1)) * Nx + (jx - 1)], acc);
        }
        v[((long)(cz + nf1) * Hy + (cy + nf1)) * Hx + (cx + nf1)] = acc / 8.0;
      }
#define V(a, b, c) v[((long)((c) + nf1) * Hy + ((b) + nf1)) * Hx + ((a) + nf1)]
  for (int c = -nf1; c <= nz + nf; ++c)
    for (int b = -nf1; b <= ny + nf; ++b)
      for (int o = 1; o <= nf; ++o) {
        V(o, b, c) = V(o, b, c) + V(nx + o, b, c);
        V(nx - nf + o, b, c) = V(nx - nf + o, b, c) + V(-nf + o, b, c);
      }
  for (int c = -nf1; c <= nz + nf; ++c)
    for (int o = 1; o <= nf; ++o)
      for (int a = -nf1; a <= nx + nf; ++a) {
        V(a, o, c) = V(a, o, c) + V(a, ny + o, c);
        V(a, ny - nf + o, c) = V(a, ny - nf + o, c) + V(a, -nf + o, c);
      }
  for (int o = 1; o <= nf; ++o)
    for (int b = -nf1; b <= ny + nf; ++b)
      for (int a = -nf1; a <= nx + nf; ++a) {
        V(a, b, o) = V(a, b, o) + V(a, b, nz + o);
        V(a, b, nz - nf + o) = V(a, b, nz - nf + o) + V(a, b, -nf + o);
      }
  for (int c = 1; c <= nz; ++c)
    for (int b = 1; b <= ny; ++b)
      for (int a = 1; a <= nx; ++a) out[((long)(c - 1) * ny + (b - 1)) * nx + (a - 1)] = V(a, b, c);
#undef V
  free(t2);
  free(t1);
  free(v);
}

/* ------------------------------------------------------------------------ */
/* vxpot_lda_pz, written as the Fortran groups it (x**2.0d0 as x*x, pi as the
 * double nearest pi, which dacos(-1.0d0) returns). */
void orc_vxc_pz(long n, const double* rho, double* vx, double* ex) {
  const double pi = 3.141592653589793;
  const double third = 1.0 / 3.0;
  for (long i = 0; i < n; ++i) {
    if (rho[i] > 1.0e-15) {
      const double rs = pow(3.0 / (4.0 * pi * rho[i]), 1.0 / 3.0);
      double exc, v;
      if (rs >= 1.0) {
        const double den = 1.0 + 1.0529 * sqrt(rs) + 0.3334 * rs;
        exc = -0.1423 / den;
        v = exc - rs / 3.0 * (0.1423 * (0.3334 + 0.52645 / sqrt(rs)) / (den * den));
      } else {
        exc = -0.048 + 0.0311 * log(rs) - 0.0116 * rs + 0.002 * rs * log(rs);
        v = exc - rs / 3.0 * (0.0311 / rs - 0.0096 + 0.002 * log(rs));
      }
      const double cx = 0.75 * pow(2.25 / (pi * pi), third);
      exc = exc - cx / rs;
      ex[i] = exc;
      vx[i] = v - cx / rs - rs / 3.0 * (cx / (rs * rs));
    } else {
      vx[i] = 0.0;
      ex[i] = 0.0;
    }
  }
}

void orc_veff_sum(long n, const double* vx, const double* vloc, const double* vh,
                  double* veff) {
  for (long i = 0; i < n; ++i) veff[i] = vx[i] + (vloc[i] + vh[i]);
}

double orc_diffcharge(long n, const double* rho_o, const double* rho_i, double dx, double dy,
                      double dz, double xmax, double ymax, double zmax) {
  double* d = (double*)malloc(sizeof(double) * (n > 0 ? n : 1));
  for (long i = 0; i < n; ++i) d[i] = rho_i[i] - rho_o[i];
  const double s = orc_tree_dot(n, d, d);
  free(d);
  return sqrt(s * dx * dy * dz / (8.0 * xmax * ymax * zmax));
}

/* Occupation matrices of the projectors, restated from scf_charge_atomicocc
 * (scf_charge8f.F90:146-213) for nrc = 0, nums = nspv = 1, numk = 1: the loop
 * order there is band l, then j, then i <= j, and every atom's matrix is a
 * sum over bands in order. */
void orc_atomicocc(int natom, int nprjmx, const int* nprj, int M, const double* rp,
                   const double* fnele, double* atocc) {
  const int npack = nprjmx * (nprjmx + 1) / 2;
  for (long k = 0; k < (long)natom * npack; ++k) atocc[k] = 0.0;
  for (int a = 0; a < natom; ++a) {
    double* occ = atocc + (long)a * npack;
    for (int l = 0; l < M; ++l) {
      const double* r = rp + ((long)l * natom + a) * nprjmx;
      int ij = 0;
      for (int j = 0; j < nprj[a]; ++j)
        for (int i = 0; i <= j; ++i) {
          double t = r[i] * r[j];
          if (i != j) t = 2.0 * t;
          occ[ij] = fma(fnele[l], t, occ[ij]);
          ++ij;
        }
    }
  }
}

/* ------------------------------------------------------------------------ */
/* Modified Broyden mixing, restated from scf_chargemixing
 * (scf_chargemixing8f.F90:59-168) and scf_chargemixing_broyden (:214-657)
 * for one spin and the grid density.  History slots keep the reference's
 * numbering: f(1..nbrydn), u(2..nbrydn), amat1(2..,2..), amat3(2..).
 * Each "a - b*c" update of the Fortran is fma(-b, c, a). */
struct orc_broyden {
  long n;
  int nbrydn, lbrydn;
  double eta;
  double* f;     /* [nbrydn+1][n] */
  double* u;     /* [nbrydn+1][n] */
  double* g;     /* [n] */
  double* prev;  /* [n] rhosmt_brydn */
  double* w1;    /* [n] work */
  double* w2;    /* [n] work */
  double* amat1; /* [(nbrydn+1)^2] */
  double* amat3; /* [nbrydn+1] */
};

orc_broyden* orc_broyden_create(long n, int nbrydn, double eta) {
  orc_broyden* b = (orc_broyden*)calloc(1, sizeof(orc_broyden));
  const long m = nbrydn + 1;
  b->n = n; b->nbrydn = nbrydn; b->lbrydn = 0; b->eta = eta;
  b->f = (double*)calloc(m * n, sizeof(double));
  b->u = (double*)calloc(m * n, sizeof(double));
  b->g = (double*)calloc(n, sizeof(double));
  b->prev = (double*)calloc(n, sizeof(double));
  b->w1 = (double*)calloc(n, sizeof(double));
  b->w2 = (double*)calloc(n, sizeof(double));
  b->amat1 = (double*)calloc(m * m, sizeof(double));
  b->amat3 = (double*)calloc(m, sizeof(double));
  return b;
}

void orc_broyden_free(orc_broyden* b) {
  if (!b) return;
  free(b->f); free(b->u); free(b->g); free(b->prev); free(b->w1); free(b->w2);
  free(b->amat1); free(b->amat3);
  free(b);
}

/* sum (x1 - x0) * (y1 - y0) dV over the grid, in the block tree */
static double bdot_diff(const orc_broyden* b, const double* x1, const double* x0,
                        const double* y1, const double* y0, double dvol) {
  for (long i = 0; i < b->n; ++i) b->w1[i] = x1[i] - x0[i];
  const double* yy = y1;
  if (y0) {
    for (long i = 0; i < b->n; ++i) b->w2[i] = y1[i] - y0[i];
    yy = b->w2;
  }
  return orc_tree_dot(b->n, b->w1, yy) * dvol;
}

void orc_broyden_step(orc_broyden* b, const double* rho_o, double* rho_i, double dvol) {
  const long n = b->n;
  const int nb = b->nbrydn;
  const int M1 = nb + 1;
  double* F[64];
  double* U[64];
  for (int k = 0; k <= nb && k < 64; ++k) {
    F[k] = b->f + (long)k * n;
    U[k] = b->u + (long)k * n;
  }
#define A1(i, j) b->amat1[(long)(i) * M1 + (j)]
  b->lbrydn += 1;
  if (b->lbrydn == 1) {
    for (long x = 0; x < n; ++x) rho_i[x] = rho_o[x];
    return;
  }
  if (b->lbrydn == 2) {
    memset(b->amat1, 0, sizeof(double) * M1 * M1);
    memset(b->amat3, 0, sizeof(double) * M1);
  }
  const int m = b->lbrydn - 1 < nb ? b->lbrydn - 1 : nb;
  double t1[64][64], t2[64];
  if (m > 1)
    for (long x = 0; x < n; ++x) U[m][x] = -b->g[x];
  for (long x = 0; x < n; ++x) {  /* scf_chargemixing_broyden_vecs, nspv=1 */
    F[m][x] = rho_o[x] - rho_i[x];
    b->g[x] = (rho_o[x] - rho_i[x]) * b->eta;
  }
  if (m > 1) {
    for (int i = 2; i <= nb; ++i)
      for (int j = 2; j <= nb; ++j) t1[i][j] = A1(i, j);
    for (int i = 2; i <= m; ++i) {
      const double t = bdot_diff(b, F[m], F[m - 1], F[i], F[i - 1], dvol);
      t1[m][i] = t; t1[i][m] = t;
      A1(m, i) = t; A1(i, m) = t;
    }
    for (int i = 2; i <= m; ++i) t2[i] = bdot_diff(b, F[i], F[i - 1], F[m], NULL, dvol);
    b->amat3[m] = bdot_diff(b, F[m], F[m - 1], F[m], F[m - 1], dvol);
    for (int j = 2; j <= m; ++j) {
      for (int i = 2; i <= m; ++i) t1[j][i] = t1[j][i] / b->amat3[j];
      t2[j] = t2[j] / b->amat3[j];
    }
    for (long x = 0; x < n; ++x) U[m][x] = U[m][x] + b->g[x] + rho_i[x] - b->prev[x];
    for (int j = 2; j <= m - 1; ++j)
      for (long x = 0; x < n; ++x) U[m][x] = fma(-t1[j][m], U[j][x], U[m][x]);
  }
  double* bv = b->w1;
  for (long x = 0; x < n; ++x) {
    b->prev[x] = rho_i[x];
    bv[x] = b->g[x];
  }
  for (int j = 2; j <= m; ++j)
    for (long x = 0; x < n; ++x) bv[x] = fma(-t2[j], U[j][x], bv[x]);
  for (long x = 0; x < n; ++x) rho_i[x] = rho_i[x] + bv[x];
  if (m == nb) {
    t2[2] = 1.0;
    for (int i = 3; i <= m; ++i) {
      t2[i] = 0.0;
      for (int j = 2; j <= i - 1; ++j) t2[i] = fma(-t1[j][i], t2[j], t2[i]);
      for (long x = 0; x < n; ++x) U[i][x] = fma(-t2[i], U[2][x], U[i][x]);
    }
    for (int i = 2; i <= m; ++i) {
      memcpy(F[i - 1], F[i], sizeof(double) * n);
      if (i > 2) memcpy(U[i - 1], U[i], sizeof(double) * n);
    }
    for (int j = 2; j <= m - 1; ++j) {
      for (int i = 2; i <= m - 1; ++i) A1(i, j) = A1(i + 1, j + 1);
      b->amat3[j] = b->amat3[j + 1];
    }
  }
#undef A1
}
