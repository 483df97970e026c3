/*
 * rs_oracle_vloc.c -- CPU FP64 restatement of kukan's local pseudopotential,
 * ion-ion (Ewald) energy and initial bands for a periodic cell (nperi = 3):
 *
 *   orc_bisec        tools_bisec (tools8f.F90:922-953): the soft local part
 *                    b cos(a r) + c inside r_c matched to -z/r at r_c;
 *   orc_vloc_coef    the local part of filterpseudopotentials
 *                    (filterpseudopotentials8f.F90:62-69, 107-131): Fourier-
 *                    Bessel coefficients of potc - (b cos(a r) + c) on the
 *                    dataset's radial mesh;
 *   orc_vloc_soft    pseudocalc_02 case (3) and its real-space images
 *                    (pseudocalc8f.F90:1443-1568) summed over atoms as
 *                    pseudocalc_03 does (:1600-1678): the soft local
 *                    potential on the coarse grid, with its gradient with
 *                    respect to the atom positions when asked (dvlocd*_scw);
 *   orc_vloc_hard    pseudocalc_02's hard part (:1245-1290) on the dense
 *                    grid list of pseudocalc_01b (:1035-1144), added as
 *                    pseudocalc_04 does (:1682-1706);
 *   orc_ewald        totalenergy_space_03 case (3) (totalenergy8f.F90:520-565);
 *   orc_initial_wave setup_initialwave, real branch
 *                    (setup_initialwave8f.F90:48-130).
 *
 * TEST INFRASTRUCTURE ONLY (see rs_oracle.h).  Loops and the order of every
 * sum follow the Fortran source; products are plain multiplications, sums
 * run left to right.  One departure, exact in FP64: real-space image terms
 * with veta*r >= 6 are skipped.  There erf(veta r) rounds to 1.0, so the
 * reference's (erf(veta r) - 1)/r adds exactly zero (the reference loops
 * over all 23^3 images).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

static const double kEtaRCut = 6.0;

void orc_bisec(double z, double r, double eps, double* a_out, double* b_out, double* c_out) {
  const double pi = acos(-1.0);
  double a0 = pi * 0.5 / r + eps;
  double a2 = 2.0 * pi * 0.5 / r - eps;
  const double fr = -r / 2.0;
  double a = 0.0;
  long l = 0;
  for (;;) {
    ++l;
    a = (a0 + a2) * 0.5;
    const double f0 = tan(a0 * r) / a0 - fr;
    const double f1 = tan(a * r) / a - fr;
    if (f0 * f1 < 0.0)
      a2 = a;
    else
      a0 = a;
    if (l > 1000000) break;
    if (!(a2 - a0 > eps)) break;
  }
  const double b = -z / r / r / a / sin(a * r);
  *a_out = a;
  *b_out = b;
  *c_out = -z / r - b * cos(a * r);
}

/* coef(iq) = sum_{ir=2..nradps} 4 pi r^2 j0(q r) vlocr(r) dr, q = pi/rcuts iq,
 * vlocr = potc - (b cos(a r) + c) for ir <= nradct and 0 beyond; j0 = 1 at
 * iq = 0.  Indices ir are 1-based as in the Fortran (array index ir-1). */
void orc_vloc_coef(int nradps, int nradct, const double* radial, const double* dradial,
                   const double* potc, double a, double b, double c, double rcuts, int nqct,
                   double* coef) {
  const double pi = acos(-1.0);
  const double fourpi = 4.0 * pi;
  double* vlocr = (double*)calloc((size_t)nradps + 1, sizeof(double));
  for (int ir = 2; ir <= nradct; ++ir) {
    const double r = radial[ir - 1];
    vlocr[ir] = potc[ir - 1] - (b * cos(a * r) + c);
  }
  for (int iq = 0; iq <= nqct; ++iq) {
    const double q = pi / rcuts * iq;
    double t = 0.0;
    for (int ir = 2; ir <= nradps; ++ir) {
      const double r = radial[ir - 1];
      const double dr = dradial[ir - 1];
      const double z = q * r;
      const double j0 = iq == 0 ? 1.0 : sin(z) / z;
      t = t + fourpi * r * r * j0 * vlocr[ir] * dr;
    }
    coef[iq] = t;
  }
  free(vlocr);
}

/* grad: NULL, or 3*natom*N doubles: the derivatives dvlocd{x,y,z}_scw of
 * each atom's soft part with respect to the point (the force uses minus
 * them), layout grad[(axis*natom + a)*N + p]. */
void orc_vloc_soft(int natom, const double* atx, const double* aty, const double* atz,
                   double cp1, double ca, double cb, double cc, double rc, int nx, int ny,
                   int nz, double dx, double dy, double dz, double xmax, double ymax,
                   double zmax, double veta, int npwx, int npwy, int npwz, double* out,
                   double* grad) {
  const long N = (long)nx * ny * nz;
  const double pi = acos(-1.0);
  const double fourpi = 4.0 * pi;
  const double omega = xmax * ymax * zmax * 8.0;
  const double omegain = 1.0 / omega;
  const double twosqrtpiin = 2.0 / sqrt(pi);
  /* images beyond these give exactly zero (veta r >= 6); the reference's
   * new_rs = 11 bounds them too */
  int nimx = (int)ceil(kEtaRCut / veta / (2.0 * xmax)) + 1;
  int nimy = (int)ceil(kEtaRCut / veta / (2.0 * ymax)) + 1;
  int nimz = (int)ceil(kEtaRCut / veta / (2.0 * zmax)) + 1;
  if (nimx > 11) nimx = 11;
  if (nimy > 11) nimy = 11;
  if (nimz > 11) nimz = 11;
  double* v = (double*)malloc(sizeof(double) * N);
  double* g = (double*)malloc(sizeof(double) * 3 * N);
  for (long p = 0; p < N; ++p) out[p] = 0.0;
  for (int na = 0; na < natom; ++na) {
    const double vlo = pi * omegain * cp1 / (veta * veta);
    for (long p = 0; p < N; ++p) {
      v[p] = vlo;
      g[p] = g[N + p] = g[2 * N + p] = 0.0;
    }
    for (int kz = 0; kz <= npwz; ++kz) {
      const double awei = kz != 0 ? 2.0 * fourpi * omegain : fourpi * omegain;
      for (int ky = -npwy; ky <= npwy; ++ky)
        for (int kx = -npwx; kx <= npwx; ++kx) {
          if (kx * kx + ky * ky + kz * kz == 0) continue;
          const double vkx = pi / xmax * kx, vky = pi / ymax * ky, vkz = pi / zmax * kz;
          const double vk2 = vkx * vkx + vky * vky + vkz * vkz;
          const double tmp = -awei * cp1 / vk2 * exp(-vk2 / (4.0 * veta * veta));
          for (int iz = 0; iz < nz; ++iz)
            for (int iy = 0; iy < ny; ++iy)
              for (int ix = 0; ix < nx; ++ix) {
                const long p = ((long)iz * ny + iy) * nx + ix;
                const double x = (ix + 1) * dx - xmax - 0.5 * dx - atx[na];
                const double y = (iy + 1) * dy - ymax - 0.5 * dy - aty[na];
                const double z = (iz + 1) * dz - zmax - 0.5 * dz - atz[na];
                const double ph = vkx * x + vky * y + vkz * z;
                const double tds = tmp * sin(ph);
                v[p] = v[p] + tmp * cos(ph);
                g[p] = g[p] - vkx * tds;
                g[N + p] = g[N + p] - vky * tds;
                g[2 * N + p] = g[2 * N + p] - vkz * tds;
              }
        }
    }
    for (int kpz = -nimz; kpz <= nimz; ++kpz)
      for (int kpy = -nimy; kpy <= nimy; ++kpy)
        for (int kpx = -nimx; kpx <= nimx; ++kpx) {
          const int near = kpx * kpx <= 1 && kpy * kpy <= 1 && kpz * kpz <= 1;
          for (long p = 0; p < N; ++p) {
            const int iz = (int)(p / ((long)nx * ny));
            const int iy = (int)((p / nx) % ny);
            const int ix = (int)(p % nx);
            const double x = (ix + 1) * dx - xmax - 0.5 * dx - atx[na] + kpx * xmax * 2.0;
            const double y = (iy + 1) * dy - ymax - 0.5 * dy - aty[na] + kpy * ymax * 2.0;
            const double z = (iz + 1) * dz - zmax - 0.5 * dz - atz[na] + kpz * zmax * 2.0;
            const double r = sqrt(x * x + y * y + z * z);
            if (veta * r >= kEtaRCut) continue;
            const double ee = exp(-(veta * r) * (veta * r));
            const double ef = erf(veta * r);
            const double rin = 1.0 / r;
            const double r2in = rin * rin;
            double tmp, derfdrr;
            if (near && r < rc) {
              tmp = cp1 * rin * ef + (cb * cos(ca * r) + cc);
              derfdrr = -cb * ca * sin(ca * r) * rin +
                        (twosqrtpiin * veta * ee * rin - ef * r2in) * cp1 * rin;
            } else {
              tmp = cp1 * rin * (ef - 1.0);
              derfdrr = cp1 * rin * (r2in + twosqrtpiin * veta * ee * rin - ef * r2in);
            }
            v[p] = v[p] + tmp;
            g[p] = g[p] + derfdrr * x;
            g[N + p] = g[N + p] + derfdrr * y;
            g[2 * N + p] = g[2 * N + p] + derfdrr * z;
          }
        }
    for (long p = 0; p < N; ++p) out[p] = out[p] + v[p];
    if (grad)
      for (int k = 0; k < 3; ++k)
        memcpy(grad + ((long)k * natom + na) * N, g + (long)k * N, sizeof(double) * N);
  }
  free(v);
  free(g);
}

static double fermidis1(double r, double t, double rc) {
  const double a = (r - rc) / t;
  if (fabs(a) < 1.0e2) return 1.0 / (exp(a) + 1.0);
  return a > 0.0 ? 0.0 : 1.0;
}

/* the hard part of one list entry at (x, y, z) from the atom: value and,
 * when g is not NULL, the gradient (dvlocd*_hdp) */
static double hard_value(double x, double y, double z, double rcut, double rcuts, int nqct,
                         const double* coef, double filpp, double eps, int nfiltyp, double* g) {
  const double pi = acos(-1.0);
  const double dqq = pi / rcuts;
  const double twopicbin = 1.0 / ((2.0 * pi) * (2.0 * pi) * (2.0 * pi));
  const double tmp = 4.0 * pi * dqq * twopicbin;
  const double r = sqrt(x * x + y * y + z * z);
  double po = 0.0, tx = 0.0, ty = 0.0, tz = 0.0, weight = 1.0, dweight = 0.0;
  if (r > eps) {
    if (nfiltyp == 1) {
      weight = fermidis1(r, filpp, rcut);
      dweight = -weight * (1.0 - weight) / filpp;
    }
    const double rin = 1.0 / r;
    for (int iq = 1; iq <= nqct; ++iq) {
      const double q = dqq * iq;
      const double q2 = q * q;
      const double qr = q * r;
      const double qrin = rin / q;
      const double s = sin(qr), c = cos(qr);
      const double j0 = s * qrin;
      const double dj0 = -(s - qr * c) * qrin * qrin * q;
      const double djq = dj0 * q2 * rin;
      po = po + coef[iq] * j0 * q2;
      tx = tx + coef[iq] * djq * x;
      ty = ty + coef[iq] * djq * y;
      tz = tz + coef[iq] * djq * z;
    }
  } else {
    for (int iq = 1; iq <= nqct; ++iq) {
      const double q = dqq * iq;
      po = po + coef[iq] * q * q;
    }
  }
  if (g) {
    /* kukan's dvlocd*_hdp (pseudocalc8f.F90:1286-1289) keep the filter
     * weight as a constant; the gradient of the value also carries the
     * weight's derivative, w' = -w (1 - w) / filpp, along r / |r| */
    const double wr = r > eps ? po * tmp * dweight / r : 0.0;
    g[0] = tx * tmp * weight + wr * x;
    g[1] = ty * tmp * weight + wr * y;
    g[2] = tz * tmp * weight + wr * z;
  }
  return po * tmp * weight;
}

/* dense grid (2nx_c... given as ndx, ndy, ndz with spacing ddx..), coarse
 * half-sizes nxmax.. and nmesh; the list box is [-npxmax*nmesh+1,
 * npxmax*nmesh] per axis.  Adds each atom's hard part to dense in atom order
 * (pseudocalc_04).  grad: NULL or the list-ordered gradients are not kept;
 * instead force_acc (3*natom, may be NULL) receives sum over the atom's list
 * of rho_dense(point) * dvlocd*_hdp * ddx ddy ddz when rho_dense is given. */
void orc_vloc_hard(int natom, const double* atx, const double* aty, const double* atz,
                   int nxmax, int nymax, int nzmax, int nmesh, double dx, double dy, double dz,
                   double xmax, double ymax, double zmax, int npxmax, int npymax, int npzmax,
                   double rcut, double psctoff, double rcuts, int nqct, const double* coef,
                   double filpp, double eps, int nfiltyp, double* dense,
                   const double* rho_dense, double* force_acc) {
  const int ndx = 2 * nxmax * nmesh, ndy = 2 * nymax * nmesh, ndz = 2 * nzmax * nmesh;
  const double ddx = dx / nmesh, ddy = dy / nmesh, ddz = dz / nmesh;
  const int bx = npxmax * nmesh, by = npymax * nmesh, bz = npzmax * nmesh;
  for (int na = 0; na < natom; ++na) {
    const int ndatx = (int)((atx[na] + xmax + 0.5 * ddx) / ddx) - nxmax * nmesh;
    const int ndaty = (int)((aty[na] + ymax + 0.5 * ddy) / ddy) - nymax * nmesh;
    const int ndatz = (int)((atz[na] + zmax + 0.5 * ddz) / ddz) - nzmax * nmesh;
    double fx = 0.0, fy = 0.0, fz = 0.0;
    for (int pass = 0; pass < 2; ++pass)
      for (int iz = -bz + 1; iz <= bz; ++iz)
        for (int iy = -by + 1; iy <= by; ++iy)
          for (int ix = -bx + 1; ix <= bx; ++ix) {
            const double x = ix * ddx - (atx[na] - (ndatx * ddx - 0.5 * ddx));
            const double y = iy * ddy - (aty[na] - (ndaty * ddy - 0.5 * ddy));
            const double z = iz * ddz - (atz[na] - (ndatz * ddz - 0.5 * ddz));
            const double r = sqrt(x * x + y * y + z * z);
            const int in = pass == 0 ? r < rcut : (r >= rcut && r < rcut * psctoff);
            if (!in) continue;
            int i = ix + ndatx + nxmax * nmesh, j = iy + ndaty + nymax * nmesh,
                k = iz + ndatz + nzmax * nmesh;
            while (i > ndx) i -= ndx;
            while (i < 1) i += ndx;
            while (j > ndy) j -= ndy;
            while (j < 1) j += ndy;
            while (k > ndz) k -= ndz;
            while (k < 1) k += ndz;
            const long p = ((long)(k - 1) * ndy + (j - 1)) * ndx + (i - 1);
            double g[3];
            const double v = hard_value(x, y, z, rcut, rcuts, nqct, coef, filpp, eps, nfiltyp, g);
            if (dense) dense[p] = dense[p] + v;
            if (rho_dense) {
              fx = fx + rho_dense[p] * g[0];
              fy = fy + rho_dense[p] * g[1];
              fz = fz + rho_dense[p] * g[2];
            }
          }
    if (force_acc) {
      force_acc[3 * na + 0] = fx * ddx * ddy * ddz;
      force_acc[3 * na + 1] = fy * ddx * ddy * ddz;
      force_acc[3 * na + 2] = fz * ddx * ddy * ddz;
    }
  }
}

/* eneat of totalenergy_space_03 case (3), one process, all atoms of one
 * species (charge cp1 each) */
double orc_ewald(int natom, const double* atx, const double* aty, const double* atz,
                 double cp1, double xmax, double ymax, double zmax, double veta, int npwx,
                 int npwy, int npwz, int nrsx, int nrsy, int nrsz) {
  const double pi = acos(-1.0);
  const double fourpi = 4.0 * pi;
  const double omega = 8.0 * xmax * ymax * zmax;
  const double omegain = 1.0 / omega;
  double e = 0.0;
  for (int l0 = 0; l0 < natom; ++l0)
    for (int l1 = 0; l1 < natom; ++l1) {
      const double x0 = atx[l0], y0 = aty[l0], z0 = atz[l0];
      for (int kz = -npwz; kz <= npwz; ++kz)
        for (int ky = -npwy; ky <= npwy; ++ky)
          for (int kx = -npwx; kx <= npwx; ++kx) {
            if (kx * kx + ky * ky + kz * kz == 0) continue;
            const double vkx = pi / xmax * kx, vky = pi / ymax * ky, vkz = pi / zmax * kz;
            const double vk2 = vkx * vkx + vky * vky + vkz * vkz;
            const double vlo0 = fourpi * omegain *
                                cos(vkx * (x0 - atx[l1]) + vky * (y0 - aty[l1]) +
                                    vkz * (z0 - atz[l1])) /
                                vk2 * exp(-vk2 / (4.0 * veta * veta));
            e = e + 0.5 * cp1 * cp1 * vlo0;
          }
      const double delta = l0 == l1 ? 1.0 : 0.0;
      const double vlo1 = -pi / omega / (veta * veta);
      const double vlo2 = -delta * 2.0 * veta / sqrt(pi);
      e = e + 0.5 * cp1 * cp1 * (vlo1 + vlo2);
      for (int kz = -nrsz; kz <= nrsz; ++kz)
        for (int ky = -nrsy; ky <= nrsy; ++ky)
          for (int kx = -nrsx; kx <= nrsx; ++kx) {
            const double x = kx * 2.0 * xmax + x0 - atx[l1];
            const double y = ky * 2.0 * ymax + y0 - aty[l1];
            const double z = kz * 2.0 * zmax + z0 - atz[l1];
            const double r = sqrt(x * x + y * y + z * z);
            if (r > 1.0e-20 && veta * r < kEtaRCut) {
              const double vlo0 = (1.0 - erf(veta * r)) / r;
              e = e + 0.5 * cp1 * cp1 * vlo0;
            }
          }
    }
  return e;
}

/* setup_initialwave, real branch, one spin and k-point: neig bands of
 * exp(-zs r) times 1, x, y, z (and the five d forms when neig > 4 natom),
 * minimum image per axis, each normalised to sum psi^2 dV = 1. */
void orc_initial_wave(int natom, const double* atx, const double* aty, const double* atz,
                      double cp1, double zs_pre, int neig, int nx, int ny, int nz, double dx,
                      double dy, double dz, double xmax, double ymax, double zmax, double* psi) {
  const double pi = acos(-1.0);
  const double sqfourpi = sqrt(1.0 / 4.0 / pi), sq3fourpi = sqrt(3.0 / 4.0 / pi);
  const double sq1516pi = sqrt(15.0 / 16.0 / pi), sq0516pi = sqrt(5.0 / 16.0 / pi);
  const double sq1504pi = sqrt(15.0 / 4.0 / pi);
  const long N = (long)nx * ny * nz;
  for (long i = 0; i < (long)neig * N; ++i) psi[i] = 0.0;
  const double zs = cp1 * zs_pre;
  const int with_d = !(neig <= natom * 4);
  for (int na = 0; na < natom; ++na)
    for (int iz = 0; iz < nz; ++iz)
      for (int iy = 0; iy < ny; ++iy)
        for (int ix = 0; ix < nx; ++ix) {
          const long p = ((long)iz * ny + iy) * nx + ix;
          double x = (ix + 1) * dx - xmax - 0.5 * dx - atx[na];
          double y = (iy + 1) * dy - ymax - 0.5 * dy - aty[na];
          double z = (iz + 1) * dz - zmax - 0.5 * dz - atz[na];
          if (x > xmax) x = x - 2.0 * xmax;
          if (x < -xmax) x = x + 2.0 * xmax;
          if (y > ymax) y = y - 2.0 * ymax;
          if (y < -ymax) y = y + 2.0 * ymax;
          if (z > zmax) z = z - 2.0 * zmax;
          if (z < -zmax) z = z + 2.0 * zmax;
          const double r = sqrt(x * x + y * y + z * z);
          const double e = exp(-zs * r);
          const double yy[9] = {sqfourpi,
                                sq3fourpi * x,
                                sq3fourpi * y,
                                sq3fourpi * z,
                                sq1516pi * (x * x - y * y),
                                -sq1504pi * z * x,
                                sq0516pi * (3.0 * z * z - r * r),
                                -sq1504pi * y * z,
                                sq1504pi * x * y};
          int band[9];
          band[0] = na;
          for (int m = 0; m < 3; ++m) band[1 + m] = natom + na * 3 + m;
          for (int m = 0; m < 5; ++m) band[4 + m] = natom * 4 + na * 5 + m;
          const int nform = with_d ? 9 : 4;
          for (int f = 0; f < nform; ++f)
            if (band[f] < neig) psi[(long)band[f] * N + p] = e * yy[f];
        }
  for (int l = 0; l < neig; ++l) {
    double s = 0.0;
    for (long p = 0; p < N; ++p) s = s + psi[(long)l * N + p] * psi[(long)l * N + p];
    const double sn = 1.0 / sqrt(s * dx * dy * dz);
    for (long p = 0; p < N; ++p) psi[(long)l * N + p] = psi[(long)l * N + p] * sn;
  }
}
