// vloc.cu -- the local pseudopotential of a periodic cell (pseudocalc_02/03/04
// for nperi = 3), the ion-ion Ewald energy and forces (totalenergy_space_03,
// force8f.F90:1900-1950) and kukan's initial bands (setup_initialwave), on the
// device.
//
// Soft part (coarse grid).  Per atom kukan evaluates
//   pi cp1 / (Omega eta^2)
//   + sum_{k != 0, kz >= 0} -awei cp1 / k^2 exp(-k^2 / 4 eta^2) cos(k.(r - R))
//   + sum_images [ r < rc : cp1 erf(eta r)/r + b cos(a r) + c
//                  else   : cp1 (erf(eta r) - 1)/r ]
// and sums the atoms (pseudocalc8f.F90:1443-1568, 1643-1665).  Here the
// reciprocal sum of all atoms is one separable transform: the structure
// factor s(k) = sum_a cp1_a exp(i k.R_a) weights each k, and
//   v(r) = Re sum_k W(k) exp(i k.r),  W(k) = T(k) conj(s(k)),
// runs as three one-axis passes (kz, then ky, then kx), about 23 complex
// multiply-adds per point instead of 6348 cosines per point and atom.  The
// real-space images run per point over the atoms with a cut-off: images with
// eta r >= 6 are skipped, where erf(eta r) rounds to 1 and kukan's term is
// exactly zero.
//
// Hard part (dense grid).  For every atom kukan lists the dense points of its
// box (+-npxmax*nmesh) within rc*psctoff (pseudocalc8f.F90:1035-1144) and
// adds the Fourier-Bessel sum sum_iq coef(iq) j0(q r) q^2 * 4 pi dq/(2 pi)^3
// times the Fermi filter (:1245-1290) in atom order (pseudocalc_04).  Here
// one thread per dense point walks the atoms in order and adds the atom's
// value when the point lies in its box and sphere.
//
// Results agree with the FP64 oracle to rounding (the sums run in another
// order, and device sin/cos/erf differ from the host's in the last bits).
#include <math.h>

#include <vector>

#include "reduce.cuh"
#include "rs_common.cuh"

namespace rs {
namespace {

constexpr double kEtaRCut = 6.0;
constexpr double kPi = 3.141592653589793238462643383279502884;

struct AtomSoft {
  double x, y, z, q, a, b, c, rc;
};

struct HardSpecies {
  double rc, rcuts, filpp;
  int nqct, coef_off;
};

struct AtomHard {
  double x, y, z;
  int ndx, ndy, ndz, spe;
};

__device__ __forceinline__ double2 cmul(double2 u, double2 v) {
  return make_double2(u.x * v.x - u.y * v.y, u.x * v.y + u.y * v.x);
}

// exp(i vk x_i) for k = kmin..kmax and the n grid points of one axis
// (x_i = (i + 1) h - xmax - h/2, vk = pi k / xmax); ph[(k - kmin) * n + i]
__global__ void k_axis_phase(int n, int kmin, int kmax, double h, double xmax, double2* ph) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long tot = (long)(kmax - kmin + 1) * n;
  if (t >= tot) return;
  const int k = kmin + (int)(t / n);
  const int i = (int)(t % n);
  const double x = (i + 1) * h - xmax - 0.5 * h;
  double s, c;
  sincos(kPi / xmax * k * x, &s, &c);
  ph[t] = make_double2(c, s);
}

// W(k) = T(k) conj(s(k)) over kz = 0..npwz, ky = -npwy..npwy, kx = -npwx..npwx
// (index ((kz * nky) + ky + npwy) * nkx + kx + npwx); W(0) = 0
__global__ void k_soft_weights(int natom, const AtomSoft* at, int npwx, int npwy, int npwz,
                               double xmax, double ymax, double zmax, double veta, double2* w) {
  const int nkx = 2 * npwx + 1, nky = 2 * npwy + 1;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)(npwz + 1) * nky * nkx) return;
  const int kz = (int)(t / ((long)nky * nkx));
  const int ky = (int)((t / nkx) % nky) - npwy;
  const int kx = (int)(t % nkx) - npwx;
  if (kx == 0 && ky == 0 && kz == 0) {
    w[t] = make_double2(0.0, 0.0);
    return;
  }
  const double omegain = 1.0 / (8.0 * xmax * ymax * zmax);
  const double awei = kz != 0 ? 2.0 * 4.0 * kPi * omegain : 4.0 * kPi * omegain;
  const double vkx = kPi / xmax * kx, vky = kPi / ymax * ky, vkz = kPi / zmax * kz;
  const double vk2 = vkx * vkx + vky * vky + vkz * vkz;
  const double tk = -awei / vk2 * exp(-vk2 / (4.0 * veta * veta));
  double cs = 0.0, sn = 0.0;
  for (int a = 0; a < natom; ++a) {
    double s, c;
    sincos(vkx * at[a].x + vky * at[a].y + vkz * at[a].z, &s, &c);
    cs += at[a].q * c;
    sn += at[a].q * s;
  }
  w[t] = make_double2(tk * cs, -tk * sn);
}

// U[(ky, kx), iz] = sum_kz W[kz, ky, kx] ez[kz, iz]
__global__ void k_soft_pass_z(int nkxy, int npwz, int nz, const double2* w, const double2* ez,
                              double2* u) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nkxy * nz) return;
  const int kxy = (int)(t / nz), iz = (int)(t % nz);
  double2 acc = make_double2(0.0, 0.0);
  for (int kz = 0; kz <= npwz; ++kz) {
    const double2 p = cmul(w[(long)kz * nkxy + kxy], ez[(long)kz * nz + iz]);
    acc.x += p.x;
    acc.y += p.y;
  }
  u[t] = acc;
}

// V[kx, iy, iz] = sum_ky U[(ky, kx), iz] ey[ky, iy]
__global__ void k_soft_pass_y(int nkx, int nky, int ny, int nz, const double2* u,
                              const double2* ey, double2* v) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nkx * ny * nz) return;
  const int kx = (int)(t / ((long)ny * nz));
  const int iy = (int)((t / nz) % ny);
  const int iz = (int)(t % nz);
  double2 acc = make_double2(0.0, 0.0);
  for (int ky = 0; ky < nky; ++ky) {
    const double2 p = cmul(u[((long)ky * nkx + kx) * nz + iz], ey[(long)ky * ny + iy]);
    acc.x += p.x;
    acc.y += p.y;
  }
  v[t] = acc;
}

// out[p] = c0 + Re sum_kx V[kx, iy, iz] ex[kx, ix]
__global__ void k_soft_pass_x(int nkx, int nx, int ny, int nz, double c0, const double2* v,
                              const double2* ex, double* out) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)nx * ny * nz) return;
  const int ix = (int)(p % nx);
  const int iy = (int)((p / nx) % ny);
  const int iz = (int)(p / ((long)nx * ny));
  double acc = 0.0;
  for (int kx = 0; kx < nkx; ++kx) {
    const double2 a = v[((long)kx * ny + iy) * nz + iz];
    const double2 e = ex[(long)kx * nx + ix];
    acc += a.x * e.x - a.y * e.y;
  }
  out[p] = c0 + acc;
}

// one image term of an atom's soft part at separation (x, y, z) and the
// derivative of the term with respect to the point
__device__ __forceinline__ double soft_image(const AtomSoft& A, bool near, double x, double y,
                                             double z, double veta, double* g) {
  const double r = sqrt(x * x + y * y + z * z);
  if (veta * r >= kEtaRCut) {
    if (g) g[0] = g[1] = g[2] = 0.0;
    return 0.0;
  }
  const double ef = erf(veta * r);
  const double rin = 1.0 / r;
  double v, d;
  if (near && r < A.rc) {
    double s, c;
    sincos(A.a * r, &s, &c);
    v = A.q * rin * ef + (A.b * c + A.c);
    if (g) {
      const double ee = exp(-(veta * r) * (veta * r));
      d = -A.b * A.a * s * rin + (2.0 / sqrt(kPi) * veta * ee * rin - ef * rin * rin) * A.q * rin;
    }
  } else {
    v = A.q * rin * (ef - 1.0);
    if (g) {
      const double ee = exp(-(veta * r) * (veta * r));
      d = A.q * rin * (rin * rin + 2.0 / sqrt(kPi) * veta * ee * rin - ef * rin * rin);
    }
  }
  if (g) {
    g[0] = d * x;
    g[1] = d * y;
    g[2] = d * z;
  }
  return v;
}

struct SoftGrid {
  int nx, ny, nz;
  double dx, dy, dz, xmax, ymax, zmax, veta;
  int nimx, nimy, nimz;
};

// out[p] += sum over atoms and images of the real-space terms
__global__ void k_soft_real(SoftGrid G, int natom, const AtomSoft* at, double* out) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)G.nx * G.ny * G.nz) return;
  const int ix = (int)(p % G.nx);
  const int iy = (int)((p / G.nx) % G.ny);
  const int iz = (int)(p / ((long)G.nx * G.ny));
  const double px = (ix + 1) * G.dx - G.xmax - 0.5 * G.dx;
  const double py = (iy + 1) * G.dy - G.ymax - 0.5 * G.dy;
  const double pz = (iz + 1) * G.dz - G.zmax - 0.5 * G.dz;
  const double rcut = kEtaRCut / G.veta;
  double acc = 0.0;
  for (int a = 0; a < natom; ++a) {
    const AtomSoft A = at[a];
    for (int kz = -G.nimz; kz <= G.nimz; ++kz) {
      const double z = pz - A.z + kz * G.zmax * 2.0;
      if (fabs(z) >= rcut) continue;
      for (int ky = -G.nimy; ky <= G.nimy; ++ky) {
        const double y = py - A.y + ky * G.ymax * 2.0;
        if (fabs(y) >= rcut) continue;
        for (int kx = -G.nimx; kx <= G.nimx; ++kx) {
          const double x = px - A.x + kx * G.xmax * 2.0;
          if (fabs(x) >= rcut) continue;
          const bool near = kx * kx <= 1 && ky * ky <= 1 && kz * kz <= 1;
          acc += soft_image(A, near, x, y, z, G.veta, nullptr);
        }
      }
    }
  }
  out[p] += acc;
}

// the Fermi filter of mathfunctions8f.F90:21-36 (fwght = 1)
__device__ __forceinline__ double fermi1(double r, double t, double rc) {
  const double a = (r - rc) / t;
  if (fabs(a) < 1.0e2) return 1.0 / (exp(a) + 1.0);
  return a > 0.0 ? 0.0 : 1.0;
}

// hard part at separation (x, y, z) from the atom (pseudocalc8f.F90:1252-1289)
__device__ double hard_value(const HardSpecies& S, const double* coef, double x, double y,
                             double z, double eps, int nfiltyp, double* g) {
  const double dqq = kPi / S.rcuts;
  const double tmp = 4.0 * kPi * dqq * (1.0 / ((2.0 * kPi) * (2.0 * kPi) * (2.0 * kPi)));
  const double r = sqrt(x * x + y * y + z * z);
  double po = 0.0, tx = 0.0, ty = 0.0, tz = 0.0, weight = 1.0, dweight = 0.0;
  if (r > eps) {
    if (nfiltyp == 1) {
      weight = fermi1(r, S.filpp, S.rc);
      dweight = -weight * (1.0 - weight) / S.filpp;
    }
    const double rin = 1.0 / r;
    for (int iq = 1; iq <= S.nqct; ++iq) {
      const double q = dqq * iq;
      const double q2 = q * q;
      const double qr = q * r;
      const double qrin = rin / q;
      double s, c;
      sincos(qr, &s, &c);
      po += coef[iq] * (s * qrin) * q2;
      if (g) {
        const double dj = -(s - qr * c) * qrin * qrin * q * q2 * rin;
        tx += coef[iq] * dj * x;
        ty += coef[iq] * dj * y;
        tz += coef[iq] * dj * z;
      }
    }
  } else {
    for (int iq = 1; iq <= S.nqct; ++iq) {
      const double q = dqq * iq;
      po += coef[iq] * q * q;
    }
  }
  if (g) {
    // the gradient of the value: kukan's dvlocd*_hdp terms (the filter
    // weight held constant, pseudocalc8f.F90:1286-1289) plus the weight's
    // own derivative w' = -w (1 - w) / filpp along r / |r|
    const double wr = r > eps ? po * tmp * dweight / r : 0.0;
    g[0] = tx * tmp * weight + wr * x;
    g[1] = ty * tmp * weight + wr * y;
    g[2] = tz * tmp * weight + wr * z;
  }
  return po * tmp * weight;
}

struct HardGrid {
  int nx, ny, nz;            // dense grid
  int nxmax, nymax, nzmax;   // coarse half sizes
  int nmesh;
  double ddx, ddy, ddz;
  int bx, by, bz;            // box half sizes on the dense grid (npxmax * nmesh)
  double psctoff, eps;
  int nfiltyp;
};

// box offsets o in [-b+1, b] with o = base (mod n), ascending
__device__ __forceinline__ int first_offset(int base, int n, int b) {
  int o = ((base + b - 1) % n + n) % n - b + 1;  // smallest o >= -b+1 congruent to base
  return o;
}

__global__ void k_hard_add(HardGrid G, int natom, const AtomHard* at, const HardSpecies* sp,
                           const double* coef, double* dense) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= (long)G.nx * G.ny * G.nz) return;
  const int i0 = (int)(p % G.nx);
  const int j0 = (int)((p / G.nx) % G.ny);
  const int k0 = (int)(p / ((long)G.nx * G.ny));
  double acc = dense[p];
  for (int a = 0; a < natom; ++a) {
    const AtomHard A = at[a];
    const HardSpecies S = sp[A.spe];
    const double lim = S.rc * G.psctoff;
    // kukan's point index (1-based) is o + ndat + nmax*nmesh, wrapped
    const int ox0 = first_offset(i0 + 1 - A.ndx - G.nxmax * G.nmesh, G.nx, G.bx);
    const int oy0 = first_offset(j0 + 1 - A.ndy - G.nymax * G.nmesh, G.ny, G.by);
    const int oz0 = first_offset(k0 + 1 - A.ndz - G.nzmax * G.nmesh, G.nz, G.bz);
    for (int oz = oz0; oz <= G.bz; oz += G.nz) {
      const double z = oz * G.ddz - (A.z - (A.ndz * G.ddz - 0.5 * G.ddz));
      for (int oy = oy0; oy <= G.by; oy += G.ny) {
        const double y = oy * G.ddy - (A.y - (A.ndy * G.ddy - 0.5 * G.ddy));
        for (int ox = ox0; ox <= G.bx; ox += G.nx) {
          const double x = ox * G.ddx - (A.x - (A.ndx * G.ddx - 0.5 * G.ddx));
          if (sqrt(x * x + y * y + z * z) < lim)
            acc += hard_value(S, coef + S.coef_off, x, y, z, G.eps, G.nfiltyp, nullptr);
        }
      }
    }
  }
  dense[p] = acc;
}

// --- Ewald ion-ion energy and forces ---------------------------------------

// structure factor of the ions over the full k box, and per k the
// reciprocal energy weight A(k) = 4 pi / Omega exp(-k^2/4eta^2) / k^2
__global__ void k_ewald_sfac(int natom, const double* xyz, const double* q, int npwx, int npwy,
                             int npwz, double xmax, double ymax, double zmax, double veta,
                             double2* sk, double* ak) {
  const int nkx = 2 * npwx + 1, nky = 2 * npwy + 1, nkz = 2 * npwz + 1;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nkz * nky * nkx) return;
  const int kz = (int)(t / ((long)nky * nkx)) - npwz;
  const int ky = (int)((t / nkx) % nky) - npwy;
  const int kx = (int)(t % nkx) - npwx;
  const double vkx = kPi / xmax * kx, vky = kPi / ymax * ky, vkz = kPi / zmax * kz;
  const double vk2 = vkx * vkx + vky * vky + vkz * vkz;
  double cs = 0.0, sn = 0.0;
  for (int a = 0; a < natom; ++a) {
    double s, c;
    sincos(vkx * xyz[3 * a] + vky * xyz[3 * a + 1] + vkz * xyz[3 * a + 2], &s, &c);
    cs += q[a] * c;
    sn += q[a] * s;
  }
  sk[t] = make_double2(cs, sn);
  ak[t] = (kx == 0 && ky == 0 && kz == 0)
              ? 0.0
              : 4.0 * kPi / (8.0 * xmax * ymax * zmax) * exp(-vk2 / (4.0 * veta * veta)) / vk2;
}

// per atom: reciprocal force sum_k A q_a k Im[conj(S) exp(i k.R_a)], and the
// real-space energy and force of its pairs (images with eta r >= 6 give
// exactly zero energy and are skipped)
__global__ void k_ewald_atom(int natom, const double* xyz, const double* q, int npwx, int npwy,
                             int npwz, double xmax, double ymax, double zmax, double veta,
                             int nimx, int nimy, int nimz, const double2* sk, const double* ak,
                             double* e_real, double* f) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const int nkx = 2 * npwx + 1, nky = 2 * npwy + 1, nkz = 2 * npwz + 1;
  const double x0 = xyz[3 * a], y0 = xyz[3 * a + 1], z0 = xyz[3 * a + 2];
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (long t = 0; t < (long)nkz * nky * nkx; ++t) {
    if (ak[t] == 0.0) continue;
    const int kz = (int)(t / ((long)nky * nkx)) - npwz;
    const int ky = (int)((t / nkx) % nky) - npwy;
    const int kx = (int)(t % nkx) - npwx;
    const double vkx = kPi / xmax * kx, vky = kPi / ymax * ky, vkz = kPi / zmax * kz;
    double s, c;
    sincos(vkx * x0 + vky * y0 + vkz * z0, &s, &c);
    const double im = sk[t].x * s - sk[t].y * c;  // Im[conj(S) e^{ik.R}]
    const double w = ak[t] * q[a] * im;
    fx += w * vkx;
    fy += w * vky;
    fz += w * vkz;
  }
  double e = 0.0;
  const double rcut = kEtaRCut / veta;
  for (int b = 0; b < natom; ++b) {
    const double qq = q[a] * q[b];
    for (int kz = -nimz; kz <= nimz; ++kz)
      for (int ky = -nimy; ky <= nimy; ++ky)
        for (int kx = -nimx; kx <= nimx; ++kx) {
          const double x = kx * 2.0 * xmax + x0 - xyz[3 * b];
          const double y = ky * 2.0 * ymax + y0 - xyz[3 * b + 1];
          const double z = kz * 2.0 * zmax + z0 - xyz[3 * b + 2];
          const double r = sqrt(x * x + y * y + z * z);
          if (r <= 1.0e-20 || r >= rcut) continue;
          const double er = erfc(veta * r);
          e += 0.5 * qq * er / r;
          // d/dr [erfc(eta r)/r] = -2 eta/sqrt(pi) exp(-eta^2 r^2)/r - erfc/r^2
          const double d = -2.0 * veta / sqrt(kPi) * exp(-veta * veta * r * r) / r - er / (r * r);
          fx -= qq * d * x / r;
          fy -= qq * d * y / r;
          fz -= qq * d * z / r;
        }
  }
  e_real[a] = e;
  f[3 * a] = fx;
  f[3 * a + 1] = fy;
  f[3 * a + 2] = fz;
}

// --- initial bands (setup_initialwave, real branch) -------------------------

struct WaveArgs {
  int natom, neig, nx, ny, nz;
  double dx, dy, dz, xmax, ymax, zmax;
  bool with_d;
};

// value of band l at point p before normalisation (0 outside its atom's form)
__device__ double wave_value(const WaveArgs& W, const double* xyz, const double* zs, int l,
                             long p) {
  int atom, form;
  if (l < W.natom) {
    atom = l;
    form = 0;
  } else if (l < 4 * W.natom) {
    atom = (l - W.natom) / 3;
    form = 1 + (l - W.natom) % 3;
  } else {
    if (!W.with_d) return 0.0;
    atom = (l - 4 * W.natom) / 5;
    form = 4 + (l - 4 * W.natom) % 5;
  }
  const int ix = (int)(p % W.nx);
  const int iy = (int)((p / W.nx) % W.ny);
  const int iz = (int)(p / ((long)W.nx * W.ny));
  double x = (ix + 1) * W.dx - W.xmax - 0.5 * W.dx - xyz[3 * atom];
  double y = (iy + 1) * W.dy - W.ymax - 0.5 * W.dy - xyz[3 * atom + 1];
  double z = (iz + 1) * W.dz - W.zmax - 0.5 * W.dz - xyz[3 * atom + 2];
  if (x > W.xmax) x = x - 2.0 * W.xmax;
  if (x < -W.xmax) x = x + 2.0 * W.xmax;
  if (y > W.ymax) y = y - 2.0 * W.ymax;
  if (y < -W.ymax) y = y + 2.0 * W.ymax;
  if (z > W.zmax) z = z - 2.0 * W.zmax;
  if (z < -W.zmax) z = z + 2.0 * W.zmax;
  const double r = sqrt(x * x + y * y + z * z);
  const double e = exp(-zs[atom] * r);
  const double s3 = sqrt(3.0 / 4.0 / kPi), s1516 = sqrt(15.0 / 16.0 / kPi);
  const double s0516 = sqrt(5.0 / 16.0 / kPi), s1504 = sqrt(15.0 / 4.0 / kPi);
  double yy;
  switch (form) {
    case 0: yy = sqrt(1.0 / 4.0 / kPi); break;
    case 1: yy = s3 * x; break;
    case 2: yy = s3 * y; break;
    case 3: yy = s3 * z; break;
    case 4: yy = s1516 * (x * x - y * y); break;
    case 5: yy = -s1504 * z * x; break;
    case 6: yy = s0516 * (3.0 * z * z - r * r); break;
    case 7: yy = -s1504 * y * z; break;
    default: yy = s1504 * x * y; break;
  }
  return e * yy;
}

// one block per band: norm[l] = 1 / sqrt(sum psi^2 dV), fixed-order tree
__global__ void k_wave_norm(WaveArgs W, const double* xyz, const double* zs, double* norm) {
  __shared__ double red[256];
  const int l = blockIdx.x;
  const long N = (long)W.nx * W.ny * W.nz;
  double s = 0.0;
  for (long p = threadIdx.x; p < N; p += blockDim.x) {
    const double v = wave_value(W, xyz, zs, l, p);
    s += v * v;
  }
  red[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) norm[l] = 1.0 / sqrt(red[0] * W.dx * W.dy * W.dz);
}

template <class T>
__global__ void k_wave_write(WaveArgs W, const double* xyz, const double* zs, const double* norm,
                             T* psi) {
  const long N = (long)W.nx * W.ny * W.nz;
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= N * W.neig) return;
  const int l = (int)(t / N);
  psi[t] = (T)(wave_value(W, xyz, zs, l, t % N) * norm[l]);
}

// --- local-part forces ------------------------------------------------------

// A[kx, iy, iz] = sum_ix rho[iz, iy, ix] ex[kx, ix]
__global__ void k_fwd_pass_x(int nkx, int nx, int ny, int nz, const double* rho,
                             const double2* ex, double2* a) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nkx * ny * nz) return;
  const int kx = (int)(t / ((long)ny * nz));
  const int iy = (int)((t / nz) % ny);
  const int iz = (int)(t % nz);
  const double* row = rho + ((long)iz * ny + iy) * nx;
  const double2* e = ex + (long)kx * nx;
  double re = 0.0, im = 0.0;
  for (int ix = 0; ix < nx; ++ix) {
    re += row[ix] * e[ix].x;
    im += row[ix] * e[ix].y;
  }
  a[t] = make_double2(re, im);
}

// B[(ky, kx), iz] = sum_iy A[kx, iy, iz] ey[ky, iy]
__global__ void k_fwd_pass_y(int nkx, int nky, int ny, int nz, const double2* a,
                             const double2* ey, double2* b) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)nky * nkx * nz) return;
  const int ky = (int)(t / ((long)nkx * nz));
  const int kx = (int)((t / nz) % nkx);
  const int iz = (int)(t % nz);
  double2 acc = make_double2(0.0, 0.0);
  for (int iy = 0; iy < ny; ++iy) {
    const double2 p = cmul(a[((long)kx * ny + iy) * nz + iz], ey[(long)ky * ny + iy]);
    acc.x += p.x;
    acc.y += p.y;
  }
  b[t] = acc;
}

// P[kz, (ky, kx)] = sum_iz B[(ky, kx), iz] ez[kz, iz]
__global__ void k_fwd_pass_z(int nkxy, int npwz, int nz, const double2* b, const double2* ez,
                             double2* pk) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)(npwz + 1) * nkxy) return;
  const int kz = (int)(t / nkxy), kxy = (int)(t % nkxy);
  double2 acc = make_double2(0.0, 0.0);
  for (int iz = 0; iz < nz; ++iz) {
    const double2 p = cmul(b[(long)kxy * nz + iz], ez[(long)kz * nz + iz]);
    acc.x += p.x;
    acc.y += p.y;
  }
  pk[t] = acc;
}

// reciprocal part: f_a -= dV q_a sum_k T_k k Im[exp(-i k.R_a) P_k]
__global__ void k_force_recip(int natom, const AtomSoft* at, int npwx, int npwy, int npwz,
                              double xmax, double ymax, double zmax, double veta, double dvol,
                              const double2* pk, double* f) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const int nkx = 2 * npwx + 1, nky = 2 * npwy + 1;
  const double omegain = 1.0 / (8.0 * xmax * ymax * zmax);
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (long t = 0; t < (long)(npwz + 1) * nky * nkx; ++t) {
    const int kz = (int)(t / ((long)nky * nkx));
    const int ky = (int)((t / nkx) % nky) - npwy;
    const int kx = (int)(t % nkx) - npwx;
    if (kx == 0 && ky == 0 && kz == 0) continue;
    const double awei = kz != 0 ? 2.0 * 4.0 * kPi * omegain : 4.0 * kPi * omegain;
    const double vkx = kPi / xmax * kx, vky = kPi / ymax * ky, vkz = kPi / zmax * kz;
    const double vk2 = vkx * vkx + vky * vky + vkz * vkz;
    const double tk = -awei / vk2 * exp(-vk2 / (4.0 * veta * veta));
    double s, c;
    sincos(vkx * at[a].x + vky * at[a].y + vkz * at[a].z, &s, &c);
    const double im = c * pk[t].y - s * pk[t].x;  // Im[(c - i s) P]
    const double w = -dvol * at[a].q * tk * im;
    fx += w * vkx;
    fy += w * vky;
    fz += w * vkz;
  }
  f[3 * a] = fx;
  f[3 * a + 1] = fy;
  f[3 * a + 2] = fz;
}

__device__ void block_sum3(double* v, double* red) {
  for (int k = 0; k < 3; ++k) red[k * 256 + threadIdx.x] = v[k];
  __syncthreads();
  for (int w = 128; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w)
      for (int k = 0; k < 3; ++k) red[k * 256 + threadIdx.x] += red[k * 256 + threadIdx.x + w];
    __syncthreads();
  }
  for (int k = 0; k < 3; ++k) v[k] = red[k * 256];
}

// real-space part: f_a += dV sum_p rho(p) sum_images grad term; one block per atom
__global__ void __launch_bounds__(256) k_force_real(SoftGrid G, const AtomSoft* at,
                                                    const double* rho, double* f) {
  __shared__ double red[3 * 256];
  const int a = blockIdx.x;
  const AtomSoft A = at[a];
  const long N = (long)G.nx * G.ny * G.nz;
  const double rcut = kEtaRCut / G.veta;
  double acc[3] = {0.0, 0.0, 0.0};
  for (long p = threadIdx.x; p < N; p += blockDim.x) {
    const int ix = (int)(p % G.nx);
    const int iy = (int)((p / G.nx) % G.ny);
    const int iz = (int)(p / ((long)G.nx * G.ny));
    const double px = (ix + 1) * G.dx - G.xmax - 0.5 * G.dx - A.x;
    const double py = (iy + 1) * G.dy - G.ymax - 0.5 * G.dy - A.y;
    const double pz = (iz + 1) * G.dz - G.zmax - 0.5 * G.dz - A.z;
    const double rp = rho[p];
    for (int kz = -G.nimz; kz <= G.nimz; ++kz) {
      const double z = pz + kz * G.zmax * 2.0;
      if (fabs(z) >= rcut) continue;
      for (int ky = -G.nimy; ky <= G.nimy; ++ky) {
        const double y = py + ky * G.ymax * 2.0;
        if (fabs(y) >= rcut) continue;
        for (int kx = -G.nimx; kx <= G.nimx; ++kx) {
          const double x = px + kx * G.xmax * 2.0;
          if (fabs(x) >= rcut) continue;
          double g[3];
          soft_image(A, kx * kx <= 1 && ky * ky <= 1 && kz * kz <= 1, x, y, z, G.veta, g);
          acc[0] += rp * g[0];
          acc[1] += rp * g[1];
          acc[2] += rp * g[2];
        }
      }
    }
  }
  block_sum3(acc, red);
  if (threadIdx.x == 0) {
    const double dv = G.dx * G.dy * G.dz;
    f[3 * a] = acc[0] * dv;
    f[3 * a + 1] = acc[1] * dv;
    f[3 * a + 2] = acc[2] * dv;
  }
}

// hard part: f_a += ddV sum over the atom's dense box points within
// rc*psctoff of rho_dense * grad(hard); one block per atom
__global__ void __launch_bounds__(256) k_force_hard(HardGrid G, const AtomHard* at,
                                                    const HardSpecies* sp, const double* coef,
                                                    const double* rho, double* f) {
  __shared__ double red[3 * 256];
  const int a = blockIdx.x;
  const AtomHard A = at[a];
  const HardSpecies S = sp[A.spe];
  const double lim = S.rc * G.psctoff;
  const int wx = 2 * G.bx, wy = 2 * G.by, wz = 2 * G.bz;
  const long box = (long)wx * wy * wz;
  double acc[3] = {0.0, 0.0, 0.0};
  for (long t = threadIdx.x; t < box; t += blockDim.x) {
    const int ox = (int)(t % wx) - G.bx + 1;
    const int oy = (int)((t / wx) % wy) - G.by + 1;
    const int oz = (int)(t / ((long)wx * wy)) - G.bz + 1;
    const double x = ox * G.ddx - (A.x - (A.ndx * G.ddx - 0.5 * G.ddx));
    const double y = oy * G.ddy - (A.y - (A.ndy * G.ddy - 0.5 * G.ddy));
    const double z = oz * G.ddz - (A.z - (A.ndz * G.ddz - 0.5 * G.ddz));
    if (!(sqrt(x * x + y * y + z * z) < lim)) continue;
    const long i = wrapi((long)ox + A.ndx + G.nxmax * G.nmesh - 1, G.nx);
    const long j = wrapi((long)oy + A.ndy + G.nymax * G.nmesh - 1, G.ny);
    const long k = wrapi((long)oz + A.ndz + G.nzmax * G.nmesh - 1, G.nz);
    double g[3];
    hard_value(S, coef + S.coef_off, x, y, z, G.eps, G.nfiltyp, g);
    const double r = rho[(k * G.ny + j) * G.nx + i];
    acc[0] += r * g[0];
    acc[1] += r * g[1];
    acc[2] += r * g[2];
  }
  block_sum3(acc, red);
  if (threadIdx.x == 0) {
    const double dv = G.ddx * G.ddy * G.ddz;
    f[3 * a] = acc[0] * dv;
    f[3 * a + 1] = acc[1] * dv;
    f[3 * a + 2] = acc[2] * dv;
  }
}

int nimages(double veta, double len) {
  int n = (int)ceil(kEtaRCut / veta / len) + 1;
  return n > 11 ? 11 : n;
}

template <class T>
int initial_wave(int natom, const double* atxyz, const double* zs, int neig, int nx, int ny,
                 int nz, double dx, double dy, double dz, double xmax, double ymax, double zmax,
                 T* psi, cudaStream_t st) {
  if (natom <= 0 || neig <= 0 || nx <= 0 || ny <= 0 || nz <= 0 || !atxyz || !zs || !psi)
    return fail(RS_EINVAL, "rs_initial_wave: bad arguments");
  if (neig > 9 * natom)
    return fail(RS_EINVAL, "rs_initial_wave: at most 9 initial bands per atom");
  WaveArgs W{natom, neig, nx, ny, nz, dx, dy, dz, xmax, ymax, zmax, !(neig <= 4 * natom)};
  double* d = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * (4 * (size_t)natom + neig), st));
  double* dxyz = d;
  double* dzs = d + 3 * natom;
  double* norm = d + 4 * natom;
  cudaMemcpyAsync(dxyz, atxyz, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dzs, zs, sizeof(double) * natom, cudaMemcpyHostToDevice, st);
  k_wave_norm<<<neig, 256, 0, st>>>(W, dxyz, dzs, norm);
  const long tot = (long)nx * ny * nz * neig;
  k_wave_write<T><<<div_up(tot, 256), 256, 0, st>>>(W, dxyz, dzs, norm, psi);
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(d, st);
  if (e != cudaSuccess) return cuda_status(e, "k_wave_write");
  return RS_OK;
}

}  // namespace
}  // namespace rs

extern "C" int rs_vloc_soft(int natom, const double* atxyz, const double* prm, int nx, int ny,
                            int nz, double dx, double dy, double dz, double xmax, double ymax,
                            double zmax, double veta, int npwx, int npwy, int npwz,
                            double* vsoft, void* stream) {
  using namespace rs;
  if (natom < 0 || nx <= 0 || ny <= 0 || nz <= 0 || npwx < 0 || npwy < 0 || npwz < 0 ||
      veta <= 0.0 || !vsoft || (natom > 0 && (!atxyz || !prm)))
    return fail(RS_EINVAL, "rs_vloc_soft: bad arguments");
  cudaStream_t st = as_stream(stream);
  std::vector<AtomSoft> h(natom);
  double qsum = 0.0;
  for (int a = 0; a < natom; ++a) {
    h[a] = AtomSoft{atxyz[3 * a], atxyz[3 * a + 1], atxyz[3 * a + 2], prm[5 * a],
                    prm[5 * a + 1], prm[5 * a + 2], prm[5 * a + 3], prm[5 * a + 4]};
    qsum += prm[5 * a];
  }
  const int nkx = 2 * npwx + 1, nky = 2 * npwy + 1, nkz = npwz + 1;
  const long nk = (long)nkz * nky * nkx;
  const size_t n_at = sizeof(AtomSoft) * (natom > 0 ? natom : 1);
  const size_t n_c = sizeof(double2) * (nk + (long)nkx * nx + (long)nky * ny + (long)nkz * nz +
                                        (long)nky * nkx * nz + (long)nkx * ny * nz);
  char* buf = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&buf, n_at + n_c, st));
  AtomSoft* dat = (AtomSoft*)buf;
  double2* w = (double2*)(buf + n_at);
  double2* ex = w + nk;
  double2* ey = ex + (long)nkx * nx;
  double2* ez = ey + (long)nky * ny;
  double2* u = ez + (long)nkz * nz;
  double2* v = u + (long)nky * nkx * nz;
  if (natom > 0)
    cudaMemcpyAsync(dat, h.data(), sizeof(AtomSoft) * natom, cudaMemcpyHostToDevice, st);
  k_axis_phase<<<div_up((long)nkx * nx, 256), 256, 0, st>>>(nx, -npwx, npwx, dx, xmax, ex);
  k_axis_phase<<<div_up((long)nky * ny, 256), 256, 0, st>>>(ny, -npwy, npwy, dy, ymax, ey);
  k_axis_phase<<<div_up((long)nkz * nz, 256), 256, 0, st>>>(nz, 0, npwz, dz, zmax, ez);
  k_soft_weights<<<div_up(nk, 128), 128, 0, st>>>(natom, dat, npwx, npwy, npwz, xmax, ymax, zmax,
                                                  veta, w);
  k_soft_pass_z<<<div_up((long)nky * nkx * nz, 256), 256, 0, st>>>(nky * nkx, npwz, nz, w, ez, u);
  k_soft_pass_y<<<div_up((long)nkx * ny * nz, 256), 256, 0, st>>>(nkx, nky, ny, nz, u, ey, v);
  const double c0 = kPi / (8.0 * xmax * ymax * zmax) * qsum / (veta * veta);
  const long N = (long)nx * ny * nz;
  k_soft_pass_x<<<div_up(N, 256), 256, 0, st>>>(nkx, nx, ny, nz, c0, v, ex, vsoft);
  SoftGrid G{nx, ny, nz, dx, dy, dz, xmax, ymax, zmax, veta,
             nimages(veta, 2.0 * xmax), nimages(veta, 2.0 * ymax), nimages(veta, 2.0 * zmax)};
  if (natom > 0) k_soft_real<<<div_up(N, 128), 128, 0, st>>>(G, natom, dat, vsoft);
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_status(e, "rs_vloc_soft");
  return RS_OK;
}

extern "C" int rs_vloc_hard_add(int natom, const double* atxyz, const int* spe, int nspe,
                                const double* sprm, const int* nqct, int nqmx, const double* coef,
                                int nx, int ny, int nz, double dx, double dy, double dz,
                                double xmax, double ymax, double zmax, int nmesh, int npxmax,
                                int npymax, int npzmax, double psctoff, double eps, int nfiltyp,
                                double* dense, void* stream) {
  using namespace rs;
  if (natom < 0 || nspe <= 0 || nqmx < 0 || nx <= 0 || ny <= 0 || nz <= 0 || nmesh < 1 ||
      !dense || (natom > 0 && (!atxyz || !spe || !sprm || !nqct || !coef)))
    return fail(RS_EINVAL, "rs_vloc_hard_add: bad arguments");
  if (natom == 0) return RS_OK;
  cudaStream_t st = as_stream(stream);
  const int nxmax = nx / 2, nymax = ny / 2, nzmax = nz / 2;
  const double ddx = dx / nmesh, ddy = dy / nmesh, ddz = dz / nmesh;
  std::vector<AtomHard> ha(natom);
  for (int a = 0; a < natom; ++a) {
    if (spe[a] < 0 || spe[a] >= nspe) return fail(RS_EINVAL, "rs_vloc_hard_add: bad species");
    const double x = atxyz[3 * a], y = atxyz[3 * a + 1], z = atxyz[3 * a + 2];
    // ndatx of pseudocalc_01b (pseudocalc8f.F90:693-695)
    ha[a] = AtomHard{x, y, z, (int)((x + xmax + 0.5 * ddx) / ddx) - nxmax * nmesh,
                     (int)((y + ymax + 0.5 * ddy) / ddy) - nymax * nmesh,
                     (int)((z + zmax + 0.5 * ddz) / ddz) - nzmax * nmesh, spe[a]};
  }
  std::vector<HardSpecies> hs(nspe);
  for (int s = 0; s < nspe; ++s) {
    if (nqct[s] < 0 || nqct[s] > nqmx) return fail(RS_EINVAL, "rs_vloc_hard_add: nqct > nqmx");
    hs[s] = HardSpecies{sprm[3 * s], sprm[3 * s + 1], sprm[3 * s + 2], nqct[s], s * (nqmx + 1)};
  }
  const size_t b1 = sizeof(AtomHard) * natom, b2 = sizeof(HardSpecies) * nspe;
  const size_t b3 = sizeof(double) * (size_t)nspe * (nqmx + 1);
  char* buf = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&buf, b1 + b2 + b3 + 64, st));
  AtomHard* dat = (AtomHard*)buf;
  HardSpecies* dsp = (HardSpecies*)(buf + ((b1 + 15) & ~(size_t)15));
  double* dcoef = (double*)(buf + ((((b1 + 15) & ~(size_t)15) + b2 + 15) & ~(size_t)15));
  cudaMemcpyAsync(dat, ha.data(), b1, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dsp, hs.data(), b2, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dcoef, coef, b3, cudaMemcpyHostToDevice, st);
  HardGrid G{nx * nmesh, ny * nmesh, nz * nmesh, nxmax, nymax, nzmax, nmesh, ddx, ddy, ddz,
             npxmax * nmesh, npymax * nmesh, npzmax * nmesh, psctoff, eps, nfiltyp};
  const long Nd = (long)G.nx * G.ny * G.nz;
  k_hard_add<<<div_up(Nd, 128), 128, 0, st>>>(G, natom, dat, dsp, dcoef, dense);
  const cudaError_t e = cudaGetLastError();
  cudaFreeAsync(buf, st);
  if (e != cudaSuccess) return cuda_status(e, "k_hard_add");
  return RS_OK;
}

extern "C" int rs_ewald(int natom, const double* atxyz, const double* q, double xmax, double ymax,
                        double zmax, double veta, int npwx, int npwy, int npwz, double* energy,
                        double* force, void* stream) {
  using namespace rs;
  if (natom <= 0 || !atxyz || !q || !energy || veta <= 0.0 || npwx < 0 || npwy < 0 || npwz < 0)
    return fail(RS_EINVAL, "rs_ewald: bad arguments");
  cudaStream_t st = as_stream(stream);
  const long nk = (long)(2 * npwx + 1) * (2 * npwy + 1) * (2 * npwz + 1);
  double* d = nullptr;
  const size_t words = 3 * (size_t)natom + natom + 2 * nk + nk + natom + 3 * (size_t)natom;
  RS_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * words, st));
  double* dxyz = d;
  double* dq = dxyz + 3 * natom;
  double2* sk = (double2*)(dq + natom);
  double* ak = (double*)(sk + nk);
  double* er = ak + nk;
  double* df = er + natom;
  cudaMemcpyAsync(dxyz, atxyz, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dq, q, sizeof(double) * natom, cudaMemcpyHostToDevice, st);
  k_ewald_sfac<<<div_up(nk, 128), 128, 0, st>>>(natom, dxyz, dq, npwx, npwy, npwz, xmax, ymax,
                                                zmax, veta, sk, ak);
  k_ewald_atom<<<div_up(natom, 64), 64, 0, st>>>(
      natom, dxyz, dq, npwx, npwy, npwz, xmax, ymax, zmax, veta, nimages(veta, 2.0 * xmax),
      nimages(veta, 2.0 * ymax), nimages(veta, 2.0 * zmax), sk, ak, er, df);
  std::vector<double> h_sk(2 * nk), h_ak(nk), h_er(natom), h_f(3 * natom);
  cudaMemcpyAsync(h_sk.data(), sk, sizeof(double) * 2 * nk, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(h_ak.data(), ak, sizeof(double) * nk, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(h_er.data(), er, sizeof(double) * natom, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(h_f.data(), df, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(d, st);
  const cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "rs_ewald");
  // E = 1/2 sum_k A |S|^2 + sum_a e_real[a] + 1/2 (sum q)^2 (-pi/(Omega eta^2))
  //     - sum_a q_a^2 eta/sqrt(pi), in FP64 on the host in a fixed order
  const double omega = 8.0 * xmax * ymax * zmax;
  double er_k = 0.0;
  for (long t = 0; t < nk; ++t)
    er_k += 0.5 * h_ak[t] * (h_sk[2 * t] * h_sk[2 * t] + h_sk[2 * t + 1] * h_sk[2 * t + 1]);
  double qs = 0.0, q2 = 0.0, er_r = 0.0;
  for (int a = 0; a < natom; ++a) {
    qs += q[a];
    q2 += q[a] * q[a];
    er_r += h_er[a];
  }
  *energy = er_k + er_r - 0.5 * qs * qs * kPi / omega / (veta * veta) -
            q2 * veta / sqrt(kPi);
  if (force)
    for (int i = 0; i < 3 * natom; ++i) force[i] = h_f[i];
  return RS_OK;
}

extern "C" int rs_initial_wave_f64(int natom, const double* atxyz, const double* zs, int neig,
                                   int nx, int ny, int nz, double dx, double dy, double dz,
                                   double xmax, double ymax, double zmax, double* psi,
                                   void* stream) {
  return rs::initial_wave<double>(natom, atxyz, zs, neig, nx, ny, nz, dx, dy, dz, xmax, ymax,
                                  zmax, psi, rs::as_stream(stream));
}

extern "C" int rs_initial_wave_f32(int natom, const double* atxyz, const double* zs, int neig,
                                   int nx, int ny, int nz, double dx, double dy, double dz,
                                   double xmax, double ymax, double zmax, float* psi,
                                   void* stream) {
  return rs::initial_wave<float>(natom, atxyz, zs, neig, nx, ny, nz, dx, dy, dz, xmax, ymax,
                                 zmax, psi, rs::as_stream(stream));
}

extern "C" int rs_force_local(int natom, const double* atxyz, const double* prm, const int* spe,
                              int nspe, const double* sprm, const int* nqct, int nqmx,
                              const double* coef, int nx, int ny, int nz, double dx, double dy,
                              double dz, double xmax, double ymax, double zmax, double veta,
                              int npwx, int npwy, int npwz, int nmesh, int npxmax, int npymax,
                              int npzmax, double psctoff, double eps, int nfiltyp,
                              const double* rho_soft, const double* rho_dense, double* force,
                              void* stream) {
  using namespace rs;
  if (natom <= 0 || nspe <= 0 || nqmx < 0 || nx <= 0 || ny <= 0 || nz <= 0 || nmesh < 1 ||
      veta <= 0.0 || npwx < 0 || npwy < 0 || npwz < 0 || !atxyz || !prm || !spe || !sprm ||
      !nqct || !coef || !rho_soft || !rho_dense || !force)
    return fail(RS_EINVAL, "rs_force_local: bad arguments");
  cudaStream_t st = as_stream(stream);
  const int nxmax = nx / 2, nymax = ny / 2, nzmax = nz / 2;
  const double ddx = dx / nmesh, ddy = dy / nmesh, ddz = dz / nmesh;
  std::vector<AtomSoft> hsoft(natom);
  std::vector<AtomHard> hhard(natom);
  for (int a = 0; a < natom; ++a) {
    if (spe[a] < 0 || spe[a] >= nspe) return fail(RS_EINVAL, "rs_force_local: bad species");
    const double x = atxyz[3 * a], y = atxyz[3 * a + 1], z = atxyz[3 * a + 2];
    hsoft[a] = AtomSoft{x, y, z, prm[5 * a], prm[5 * a + 1], prm[5 * a + 2], prm[5 * a + 3],
                        prm[5 * a + 4]};
    hhard[a] = AtomHard{x, y, z, (int)((x + xmax + 0.5 * ddx) / ddx) - nxmax * nmesh,
                        (int)((y + ymax + 0.5 * ddy) / ddy) - nymax * nmesh,
                        (int)((z + zmax + 0.5 * ddz) / ddz) - nzmax * nmesh, spe[a]};
  }
  std::vector<HardSpecies> hs(nspe);
  for (int s = 0; s < nspe; ++s) {
    if (nqct[s] < 0 || nqct[s] > nqmx) return fail(RS_EINVAL, "rs_force_local: nqct > nqmx");
    hs[s] = HardSpecies{sprm[3 * s], sprm[3 * s + 1], sprm[3 * s + 2], nqct[s], s * (nqmx + 1)};
  }
  const int nkx = 2 * npwx + 1, nky = 2 * npwy + 1, nkz = npwz + 1;
  const long nk = (long)nkz * nky * nkx;
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  const size_t bs = up(sizeof(AtomSoft) * natom), bh = up(sizeof(AtomHard) * natom);
  const size_t bsp = up(sizeof(HardSpecies) * nspe);
  const size_t bc = up(sizeof(double) * (size_t)nspe * (nqmx + 1));
  const size_t bph = up(sizeof(double2) * ((long)nkx * nx + (long)nky * ny + (long)nkz * nz));
  const size_t ba = up(sizeof(double2) * (long)nkx * ny * nz);
  const size_t bb = up(sizeof(double2) * (long)nky * nkx * nz);
  const size_t bp = up(sizeof(double2) * nk);
  const size_t bf = up(sizeof(double) * 9 * natom);
  char* buf = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&buf, bs + bh + bsp + bc + bph + ba + bb + bp + bf, st));
  char* q = buf;
  AtomSoft* dsoft = (AtomSoft*)q; q += bs;
  AtomHard* dhard = (AtomHard*)q; q += bh;
  HardSpecies* dsp = (HardSpecies*)q; q += bsp;
  double* dcoef = (double*)q; q += bc;
  double2* ex = (double2*)q;
  double2* ey = ex + (long)nkx * nx;
  double2* ez = ey + (long)nky * ny;
  q += bph;
  double2* A = (double2*)q; q += ba;
  double2* B = (double2*)q; q += bb;
  double2* Pk = (double2*)q; q += bp;
  double* df = (double*)q;
  cudaMemcpyAsync(dsoft, hsoft.data(), sizeof(AtomSoft) * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dhard, hhard.data(), sizeof(AtomHard) * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dsp, hs.data(), sizeof(HardSpecies) * nspe, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(dcoef, coef, sizeof(double) * nspe * (nqmx + 1), cudaMemcpyHostToDevice, st);
  k_axis_phase<<<div_up((long)nkx * nx, 256), 256, 0, st>>>(nx, -npwx, npwx, dx, xmax, ex);
  k_axis_phase<<<div_up((long)nky * ny, 256), 256, 0, st>>>(ny, -npwy, npwy, dy, ymax, ey);
  k_axis_phase<<<div_up((long)nkz * nz, 256), 256, 0, st>>>(nz, 0, npwz, dz, zmax, ez);
  k_fwd_pass_x<<<div_up((long)nkx * ny * nz, 256), 256, 0, st>>>(nkx, nx, ny, nz, rho_soft, ex, A);
  k_fwd_pass_y<<<div_up((long)nky * nkx * nz, 256), 256, 0, st>>>(nkx, nky, ny, nz, A, ey, B);
  k_fwd_pass_z<<<div_up(nk, 256), 256, 0, st>>>(nky * nkx, npwz, nz, B, ez, Pk);
  k_force_recip<<<div_up(natom, 64), 64, 0, st>>>(natom, dsoft, npwx, npwy, npwz, xmax, ymax,
                                                  zmax, veta, dx * dy * dz, Pk, df);
  SoftGrid G{nx, ny, nz, dx, dy, dz, xmax, ymax, zmax, veta,
             nimages(veta, 2.0 * xmax), nimages(veta, 2.0 * ymax), nimages(veta, 2.0 * zmax)};
  k_force_real<<<natom, 256, 0, st>>>(G, dsoft, rho_soft, df + 3 * natom);
  HardGrid H{nx * nmesh, ny * nmesh, nz * nmesh, nxmax, nymax, nzmax, nmesh, ddx, ddy, ddz,
             npxmax * nmesh, npymax * nmesh, npzmax * nmesh, psctoff, eps, nfiltyp};
  k_force_hard<<<natom, 256, 0, st>>>(H, dhard, dsp, dcoef, rho_dense, df + 6 * natom);
  std::vector<double> hf(9 * (size_t)natom);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(hf.data(), df, sizeof(double) * 9 * natom, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "rs_force_local");
  // recip + real + hard, per atom and axis
  for (int i = 0; i < 3 * natom; ++i) force[i] = hf[i] + hf[3 * natom + i] + hf[6 * natom + i];
  return RS_OK;
}
