/*
 * rs_oracle_proj.c -- CPU FP64 restatement of kukan's projector-table
 * generation: the double-grid weights of pseudocalc_01a
 * (pseudocalc8f.F90:343-629) and the Fourier-filtered projectors on the fine
 * mesh with their double-grid contraction onto the sphere lists of
 * pseudocalc_07 (pseudocalc8f.F90:2515-3702), for one species.
 *
 * TEST INFRASTRUCTURE ONLY (see rs_oracle.h).  Loops, index ranges and the
 * order of every sum follow the Fortran source; products are plain
 * multiplications (no contraction), sums run left to right.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

/* pseudocalc_01a: Lagrange weight of the coarse node 0 at the fine offset
 * r = |j + 1/2| / npmesh (even npmesh) or |j| / npmesh (odd), piecewise over
 * the intervals (k-1, k], k = 1..nfdg, with the nodes k+nfdg-1 .. k-nfdg
 * (0 excluded) multiplied from the largest down, divided by the product of
 * their negatives (144, -240, 720, -5040 for nfdg = 4). */
void orc_dg_weights(int nfdg, int npmesh, double* w) {
  const int n = nfdg * npmesh;
  int js = -n;
  const int je = n - 1;
  double tmp1 = 0.5;
  int ntmp1 = 1;
  if (npmesh % 2 == 1) {
    js = -n + 1;
    tmp1 = 0.0;
    ntmp1 = 0;
  }
  const double tmp = 1.0 / npmesh;
  for (int j = -n; j <= je; ++j) w[j + n] = 0.0;
  for (int j = js; j <= je; ++j) {
    const double r = fabs(j * tmp + tmp1 * tmp);
    int k = 1;
    while (k < nfdg && abs(2 * j + ntmp1) > 2 * k * npmesh) ++k;
    double p = 1.0, d = 1.0;
    for (int m = k + nfdg - 1; m >= 1; --m) {
      p = p * (r - m);
      d = d * (double)(-m);
    }
    for (int m = 1; m <= nfdg - k; ++m) {
      p = p * (r + m);
      d = d * (double)m;
    }
    w[j + n] = p / d;
  }
}

/* the Fermi filter of mathfunctions8f.F90:21-36 (fwght = 1) */
static double fermidis(double r, double t, double rc) {
  const double a = (r - rc) / t;
  if (fabs(a) < 1.0e2) return 1.0 / (exp(a) + 1.0);
  return a > 0.0 ? 0.0 : 1.0;
}

/* normalisation of the real harmonic ylm01..ylm09 (pseudocalc8f.F90:2553-2560) */
static double ylm_norm(int m) {
  const double pi = acos(-1.0);
  if (m == 1) return sqrt(1.0 / 4.0 / pi);
  if (m <= 4) return sqrt(3.0 / 4.0 / pi);
  if (m == 5) return sqrt(15.0 / 16.0 / pi);
  if (m == 7) return sqrt(5.0 / 16.0 / pi);
  return sqrt(15.0 / 4.0 / pi);
}

int orc_projector_tables(int natom, int nprj, int num_list, int nxmax, int nymax, int nzmax,
                         double dx, double dy, double dz, int npxmax, int npymax, int npzmax,
                         int nfdg, int npmesh, const double* atx, const double* aty,
                         const double* atz, const int* natx, const int* naty, const int* natz,
                         const int* natinf, const int* lstx, const int* lsty, const int* lstz,
                         const int* prj_col, const int* prj_m, int nqct, int nqmx,
                         const double* coef, double rcut, double psftrad, double psctoff,
                         double eps, int nfiltyp, double filpp, const double* wxyz, double* v) {
  const double pi = acos(-1.0);
  const double dpx = dx / npmesh, dpy = dy / npmesh, dpz = dz / npmesh;
  const double dpxyz = dpx * dpy * dpz;
  const int npxd = npxmax * npmesh, npyd = npymax * npmesh, npzd = npzmax * npmesh;
  const double twopicbin = 1.0 / ((2.0 * pi) * (2.0 * pi) * (2.0 * pi));
  const double fourpi = 4.0 * pi;
  const int nxs = npmesh * (npxmax + nfdg) - (npmesh + 1) / 2;
  const int nys = npmesh * (npymax + nfdg) - (npmesh + 1) / 2;
  const int nzs = npmesh * (npzmax + nfdg) - (npmesh + 1) / 2;
  const long sx = 2L * nxs, sy = 2L * nys, sz = 2L * nzs;
  const long nspd = sx * sy * sz;
  const int q1 = nqmx + 1;
  double* spd = calloc((size_t)nspd * nprj, sizeof(double));
  double* t1 = malloc(sizeof(double) * (size_t)sx * sy * 2 * npzmax);
  double* t2 = malloc(sizeof(double) * (size_t)sx * 2 * npymax * 2 * npzmax);
  double* t0 = malloc(sizeof(double) * (size_t)8 * npxmax * npymax * npzmax);
  if (!spd || !t1 || !t2 || !t0) {
    free(spd); free(t1); free(t2); free(t0);
    return 1;
  }
  double nrm[18];
  int used[7] = {0, 0, 0, 0, 0, 0, 0};
  for (int la = 0; la < nprj; ++la) {
    nrm[la] = ylm_norm(prj_m[la]);
    used[prj_col[la]] = 1;
  }
  const double rcutss = rcut * psftrad;
  const double dqq = pi / rcutss;
  const double tq = fourpi * dqq * twopicbin;
  const int n = nfdg * npmesh;
  const int js = npmesh % 2 == 1 ? -n + 1 : -n, je = n - 1;
#define SPD(kx, ky, kz, la) \
  spd[(long)(la) * nspd + ((long)((kz) + nzs - 1) * sy + ((ky) + nys - 1)) * sx + ((kx) + nxs - 1)]
  for (int na = 0; na < natom; ++na) {
    memset(spd, 0, sizeof(double) * (size_t)nspd * nprj);
    const int npatx = (int)((atx[na] + nxmax * dx + 0.5 * dpx) / dpx) - nxmax * npmesh;
    const int npaty = (int)((aty[na] + nymax * dy + 0.5 * dpy) / dpy) - nymax * npmesh;
    const int npatz = (int)((atz[na] + nzmax * dz + 0.5 * dpz) / dpz) - nzmax * npmesh;
    for (int iz = -npzd + 1; iz <= npzd; ++iz)
      for (int iy = -npyd + 1; iy <= npyd; ++iy)
        for (int ix = -npxd + 1; ix <= npxd; ++ix) {
          const int kx = ix + (npatx - npmesh * natx[na]);
          const int ky = iy + (npaty - npmesh * naty[na]);
          const int kz = iz + (npatz - npmesh * natz[na]);
          const double x = ix * dpx - (atx[na] - (npatx * dpx - 0.5 * dpx));
          const double y = iy * dpy - (aty[na] - (npaty * dpy - 0.5 * dpy));
          const double z = iz * dpz - (atz[na] - (npatz * dpz - 0.5 * dpz));
          const double r = sqrt(x * x + y * y + z * z);
          if (!(r < rcut * psctoff)) continue;
          double s[7] = {0, 0, 0, 0, 0, 0, 0};
          double ylm[10];
          double weight = 1.0;
          if (r > eps) {
            if (nfiltyp == 1) weight = fermidis(r, filpp, rcut);
            const double rin = 1.0 / r;
            ylm[1] = 1.0;
            ylm[2] = rin * x;
            ylm[3] = rin * y;
            ylm[4] = rin * z;
            ylm[5] = rin * rin * (x * x - y * y);
            ylm[6] = -rin * rin * z * x;
            ylm[7] = rin * rin * (3.0 * z * z - r * r);
            ylm[8] = -rin * rin * y * z;
            ylm[9] = rin * rin * x * y;
            for (int iq = 1; iq <= nqct; ++iq) {
              const double qqq = dqq * iq;
              const double qqq2 = qqq * qqq;
              const double qqqr = qqq * r;
              const double qqqr2 = qqqr * qqqr;
              const double qqqrin = rin / qqq;
              const double qqqr2in = qqqrin * qqqrin;
              const double qqqr3in = qqqr2in * qqqrin;
              const double sn = sin(qqqr), cs = cos(qqqr);
              const double j0 = sn * qqqrin;
              const double j1 = (sn - qqqr * cs) * qqqr2in;
              const double j2 = ((3.0 - qqqr2) * sn - 3.0 * qqqr * cs) * qqqr3in;
              for (int c = 1; c <= 6; ++c) {
                if (!used[c]) continue;
                const double jl = c <= 2 ? j0 : (c <= 4 ? j1 : j2);
                s[c] = s[c] + coef[c * q1 + iq] * jl * qqq2;
              }
            }
          } else {
            ylm[1] = 1.0;
            for (int m = 2; m <= 9; ++m) ylm[m] = 0.0;
            for (int iq = 1; iq <= nqct; ++iq) {
              const double qqq = dqq * iq;
              for (int c = 1; c <= 2; ++c)
                if (used[c]) s[c] = s[c] + coef[c * q1 + iq] * qqq * qqq;
            }
          }
          for (int la = 0; la < nprj; ++la)
            SPD(kx, ky, kz, la) = s[prj_col[la]] * tq * dpxyz * nrm[la] * ylm[prj_m[la]] * weight;
        }
    /* double-grid contraction z, y, x, then the list points */
    for (int la = 0; la < nprj; ++la) {
      for (int iz = -npzmax + 1; iz <= npzmax; ++iz)
        for (int iy = -nys + 1; iy <= nys; ++iy)
          for (int ix = -nxs + 1; ix <= nxs; ++ix) {
            const int kkz = iz * npmesh - (npmesh - 1) / 2;
            double acc = 0.0;
            for (int jz = js; jz <= je; ++jz) acc = acc + SPD(ix, iy, kkz + jz, la) * wxyz[jz + n];
            t1[((long)(iz + npzmax - 1) * sy + (iy + nys - 1)) * sx + (ix + nxs - 1)] = acc;
          }
      for (int iz = -npzmax + 1; iz <= npzmax; ++iz)
        for (int iy = -npymax + 1; iy <= npymax; ++iy)
          for (int ix = -nxs + 1; ix <= nxs; ++ix) {
            const int kky = iy * npmesh - (npmesh - 1) / 2;
            double acc = 0.0;
            for (int jy = js; jy <= je; ++jy)
              acc = acc + t1[((long)(iz + npzmax - 1) * sy + (kky + jy + nys - 1)) * sx +
                             (ix + nxs - 1)] * wxyz[jy + n];
            t2[((long)(iz + npzmax - 1) * 2 * npymax + (iy + npymax - 1)) * sx + (ix + nxs - 1)] =
                acc;
          }
      for (int iz = -npzmax + 1; iz <= npzmax; ++iz)
        for (int iy = -npymax + 1; iy <= npymax; ++iy)
          for (int ix = -npxmax + 1; ix <= npxmax; ++ix) {
            const int kkx = ix * npmesh - (npmesh - 1) / 2;
            double acc = 0.0;
            for (int jx = js; jx <= je; ++jx)
              acc = acc + t2[((long)(iz + npzmax - 1) * 2 * npymax + (iy + npymax - 1)) * sx +
                             (kkx + jx + nxs - 1)] * wxyz[jx + n];
            t0[((long)(iz + npzmax - 1) * 2 * npymax + (iy + npymax - 1)) * 2 * npxmax +
               (ix + npxmax - 1)] = acc;
          }
      for (int i = 0; i < num_list; ++i) v[((long)na * nprj + la) * num_list + i] = 0.0;
      for (int i = 0; i < natinf[na]; ++i) {
        const long e = (long)na * num_list + i;
        v[((long)na * nprj + la) * num_list + i] =
            t0[((long)(lstz[e] + npzmax - 1) * 2 * npymax + (lsty[e] + npymax - 1)) * 2 * npxmax +
               (lstx[e] + npxmax - 1)];
      }
    }
  }
#undef SPD
  free(spd); free(t1); free(t2); free(t0);
  return 0;
}
