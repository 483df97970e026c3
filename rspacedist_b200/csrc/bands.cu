// bands.cu -- band solvers of scf_diag on the GPU: Gram-Schmidt in the S
// metric, Rayleigh-Ritz, band-by-band preconditioned CG (kscg_r), RMM-DIIS
// (ksdiis_r), reordering (reorderstates) and the dispatcher (scf_diag).
//
// Vectors are T = double (plain FP64 path) or T = float (mixed path: FP32
// wavefunctions, FP64 dots, coefficients and small matrices).  With T =
// double every per-band vector operation is the fma the Fortran statement
// contracts to and every dot product uses the fixed tree of reduce.cuh, so
// the CG and DIIS band updates reproduce the strict CPU restatement bit for
// bit; the block orthogonalisation (Cholesky-QR) and Rayleigh-Ritz go through
// GEMMs and an eigensolver and agree to rounding.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <type_traits>
#include <vector>

#include "reduce.cuh"
#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {

// kernels implemented elsewhere
template <class T>
int launch_nl_dot(const rs_geom* g, const T* psi, int nb, double* rp, cudaStream_t st);
template <class T, int MODE>
int launch_gather(const rs_geom* g, const double* mat, const double* rp, const T* psi,
                  const T* veff, T* out, int nb, cudaStream_t st);
int launch_hpsi_f32_fast(const rs_geom* g, const float* veff, const double* dij,
                         const double* rp, const float* psi, float* hpsi, int nb,
                         cudaStream_t st, bool local_only = false);
bool hpsi_f32_fast_ok(const rs_geom* g, int nb);
bool spsi_f32_fast_ok(const rs_geom* g);
int launch_spsi_f32_fast(const rs_geom* g, const double* sss, const double* rp, const float* psi,
                         float* out, int nb, cudaStream_t st);
int gram_f32(int m, int n, long K, const float* A, long lda, const float* B, long ldb,
             double alpha, double* C, long ldc, int sym, cudaStream_t st);
int gram_f64(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
             double alpha, double* C, long ldc, cudaStream_t st);
int gram_f64_beta(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
                  double alpha, double beta, double* C, long ldc, cudaStream_t st);
int rotate_f32(long npts, int kin, int nout, const float* X, long ldx, const double* Z, long ldz,
               float* Y, long ldy, cudaStream_t st);
int rotate_f64(long npts, int kin, int nout, const double* X, long ldx, const double* Z, long ldz,
               double* Y, long ldy, cudaStream_t st);
int syev_jacobi(int n, double* A, double* w, double* Z, int max_sweeps, cudaStream_t st,
                int* sweeps_out);
int chol_inv_t(int n, double* G, double* W, cudaStream_t st);

namespace {

// ------------------------------------------------------------ vector kernels
// out[j] = tree_dot(Y_j, x) * dx * dy * dz  (j < cnt), partial pass
template <class T>
__global__ void k_bdot_partial(long n, const T* __restrict__ Y, long ldy, const T* __restrict__ x,
                               long nblk, double* __restrict__ part) {
  __shared__ double ws[8];
  const int j = blockIdx.y;
  const T* y = Y + (long)j * ldy;
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < n) acc = fma((double)y[i], (double)x[i], acc);
  }
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) part[(long)j * nblk + blockIdx.x] = s;
}

__global__ void k_bdot_final(long nblk, const double* __restrict__ part, double dx, double dy,
                             double dz, int scale, double* __restrict__ out) {
  __shared__ double ws[8];
  const int j = blockIdx.x;
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + part[(long)j * nblk + k];
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) out[j] = scale ? s * dx * dy * dz : s;
}

// x -= sum_{j<cnt} c[j] y_j, j in order (orthogonalization_r_03 / multr)
template <class T>
__global__ void k_subcomb(long n, T* __restrict__ x, const T* __restrict__ Y, long ldy,
                          const double* __restrict__ c, int cnt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = (double)x[i];
  for (int j = 0; j < cnt; ++j) v = fma(-c[j], (double)Y[(long)j * ldy + i], v);
  x[i] = (T)v;
}
// double-precision rp vectors
__global__ void k_subcomb_d(long n, double* __restrict__ x, const double* __restrict__ Y,
                            long ldy, const double* __restrict__ c, int cnt) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = x[i];
  for (int j = 0; j < cnt; ++j) v = fma(-c[j], Y[(long)j * ldy + i], v);
  x[i] = v;
}

// x *= 1/sqrt(*nrm) for up to three vectors (the third is the rp vector)
template <class T>
__global__ void k_scale3(long n, T* __restrict__ a, T* __restrict__ b, long nrp,
                         double* __restrict__ r, const double* __restrict__ tmp) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const double t = *tmp;
  if (i < n) {
    a[i] = (T)((double)a[i] * t);
    if (b) b[i] = (T)((double)b[i] * t);
  }
  if (i < nrp) r[i] = r[i] * t;
}

// tmp = 1/sqrt(vecnor); status 1 when vecnor <= 0 (kukan's 'negative norm')
__global__ void k_invsqrt(const double* __restrict__ vecnor, double* __restrict__ tmp,
                          int* __restrict__ status) {
  const double v = *vecnor;
  if (!(v > 0.0)) {
    *status = 1;
    *tmp = 1.0;
  } else {
    *tmp = 1.0 / sqrt(v);
  }
}

// rvec = -(h - lambda s)   (kscg_r_02)
template <class T>
__global__ void k_resid(long n, const T* __restrict__ h, const T* __restrict__ s,
                        const double* __restrict__ lam, T* __restrict__ r) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  r[i] = (T)(-fma(-*lam, (double)s[i], (double)h[i]));
}


// kscg_r_03 on the grid vectors and the rp vectors
template <class T>
__global__ void k_cg_dir(long n, T* __restrict__ pvec, const T* __restrict__ rv,
                         T* __restrict__ pv, T* __restrict__ spv, const T* __restrict__ asv,
                         long nrp, double* __restrict__ rpp, const double* __restrict__ rrp,
                         const double* __restrict__ sc /* ratio at sc[0] */) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const double ratio = sc[0];
  if (i < n) {
    const T p = (T)fma(ratio, (double)pv[i], (double)rv[i]);
    pv[i] = p;
    pvec[i] = p;
    if (spv) spv[i] = (T)fma(ratio, (double)spv[i], (double)asv[i]);
  }
  if (i < nrp) rpp[i] = fma(ratio, rpp[i], rrp[i]);
}

// kscg_r_05 rotation x = alph x + beta y on psi, hpsi, spsi and rp
template <class T>
__global__ void k_cg_rot(long n, T* __restrict__ psi, const T* __restrict__ p, T* __restrict__ h,
                         const T* __restrict__ ap, T* __restrict__ s, const T* __restrict__ as,
                         long nrp, double* __restrict__ rp, const double* __restrict__ rpl,
                         const double* __restrict__ sc /* alph, beta at sc[0..1] */) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const double al = sc[0], be = sc[1];
  if (i < n) {
    psi[i] = (T)fma(be, (double)p[i], al * (double)psi[i]);
    h[i] = (T)fma(be, (double)ap[i], al * (double)h[i]);
    if (s) s[i] = (T)fma(be, (double)as[i], al * (double)s[i]);
  }
  if (i < nrp) rp[i] = fma(be, rpl[i], al * rp[i]);
}


// ------------------------------------------------------------ scalar kernels
// device scalars of one band step
struct Sc {
  double valre, r1rr, r2rr, ratio, vecnor, tmp, pap, sapre, ab[2];
  double s[4];            // DIIS line-search sums
  double lam;             // DIIS step
  double rs[4], rr[4];    // 2x2 matrices, rs[i*2+j]
  double c[2];            // DIIS combination
  double coef_dummy;
  int status;
};

__global__ void k_cg_ratio(Sc* sc) { sc->ratio = sc->r2rr / sc->r1rr; }

// kscg_r_05: 2x2 Rayleigh-Ritz in span{psi, p}
__global__ void k_cg_alphabeta(Sc* sc, const double* __restrict__ sval) {
  const double sv = *sval, pap = sc->pap, sapre = sc->sapre, eps = 1.0e-14;
  double alph = 1.0, beta = 0.0;
  const double gamma = (sv + pap) * 0.5 - sqrt((sv - pap) * (sv - pap) * 0.25 + sapre * sapre);
  if (fabs((sv - gamma) / gamma) > eps) {
    const double den = sqrt(sapre * sapre + (sv - gamma) * (sv - gamma));
    alph = sapre / den;
    beta = -(sv - gamma) / den;
  }
  if (alph < eps) {
    alph = -alph;
    beta = -beta;
  }
  sc->ab[0] = alph;
  sc->ab[1] = beta;
}

// DIIS step length (ksdiis8f.F90:285-320)
__device__ void diis_lambda(Sc* sc, const double* __restrict__ sval, double a1, double dx,
                            double dy, double dz, double lmin, double lmax) {
  const double sv = *sval;
  const double aaa = 2.0 * fma(-sv, sc->s[1], sc->s[0]) * dx * dy * dz;
  const double valre = sc->s[2] / sc->s[3];
  const double bbb = fma(-aaa, a1, valre - sv) / (a1 * a1);
  double al = 0.5 * aaa / bbb;
  if (al > lmax) al = lmax;
  if (al < lmin) al = lmin;
  sc->lam = al;
}

__device__ void eig2(const double a[4], double w[2], double z[4]) {
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
  double u0, u1;
  if (half >= 0.0) { u0 = half + rad; u1 = r; }
  else             { u0 = r; u1 = rad - half; }
  const double nu = sqrt(u0 * u0 + u1 * u1);
  u0 /= nu; u1 /= nu;
  double v0 = -u1, v1 = u0;
  if (fabs(u1) > fabs(u0) ? u1 < 0.0 : u0 < 0.0) { u0 = -u0; u1 = -u1; }
  if (fabs(v1) > fabs(v0) ? v1 < 0.0 : v0 < 0.0) { v0 = -v0; v1 = -v1; }
  z[0] = v0; z[2] = v1;
  z[1] = u0; z[3] = u1;
}

// DIIS 2x2 subspace solve (ksdiis8f.F90:405-548); rs/rr already scaled
__device__ void diis_solve(Sc* sc, double eps_eig, double* __restrict__ resid) {
  double rs[4], rr[4], rs0[4];
  for (int k = 0; k < 4; ++k) { rs[k] = sc->rs[k]; rr[k] = sc->rr[k]; rs0[k] = rs[k]; }
  double w[2], z[4], eig[2], vec[4];
  eig2(rs, w, z);
  for (int k = 0; k < 2; ++k) {
    eig[k] = w[1 - k];
    vec[0 * 2 + k] = z[0 * 2 + (1 - k)];
    vec[1 * 2 + k] = z[1 * 2 + (1 - k)];
  }
  int nmat = 0, k = 0;
  while (k < 2) {
    ++nmat; ++k;
    if (eig[nmat - 1] < eps_eig) --nmat;
  }
  double c[2];
  if (nmat > 1) {
    for (int i = 0; i < 2; ++i) {
      const double sq = sqrt(eig[i]);
      vec[0 * 2 + i] /= sq;
      vec[1 * 2 + i] /= sq;
    }
    double t[4] = {0, 0, 0, 0}, r2[4] = {0, 0, 0, 0};
    for (int kk = 0; kk < 2; ++kk)
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) t[kk * 2 + j] = fma(rr[kk * 2 + i], vec[i * 2 + j], t[kk * 2 + j]);
    for (int kk = 0; kk < 2; ++kk)
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i < 2; ++i) r2[kk * 2 + j] = fma(vec[i * 2 + kk], t[i * 2 + j], r2[kk * 2 + j]);
    double w2[2], z2[4], v2[4];
    eig2(r2, w2, z2);
    for (int kk = 0; kk < 2; ++kk) {
      v2[0 * 2 + kk] = z2[0 * 2 + (1 - kk)];
      v2[1 * 2 + kk] = z2[1 * 2 + (1 - kk)];
    }
    *resid = w2[0];
    for (int j = 0; j < 2; ++j) {
      double acc = 0.0;
      for (int i = 0; i < 2; ++i) acc = fma(vec[j * 2 + i], v2[i * 2 + 1], acc);
      c[j] = acc;
    }
    double nrm = 0.0;
    for (int j = 0; j < 2; ++j)
      for (int i = 0; i < 2; ++i) nrm = fma(c[i] * rs0[i * 2 + j], c[j], nrm);
    const double sq = sqrt(nrm);
    c[0] /= sq;
    c[1] /= sq;
  } else {
    c[0] = 0.0;
    c[1] = 1.0;
  }
  sc->c[0] = c[0];
  sc->c[1] = c[1];
}

// scale row/column 2 of the DIIS matrices by tmp (rs(2,2) twice)
__device__ void diis_scale_mats(Sc* sc) {
  const double t = sc->tmp;
  for (int i = 0; i < 2; ++i) { sc->rs[1 * 2 + i] *= t; sc->rr[1 * 2 + i] *= t; }
  for (int i = 0; i < 2; ++i) { sc->rs[i * 2 + 1] *= t; sc->rr[i * 2 + 1] *= t; }
}

__global__ void k_copy_d(double* dst, const double* src) { *dst = *src; }

// ------------------------------------------------------------ band-batched DIIS
// ksdiis_r updates every band from its own vectors only, so one step of the
// band loop runs for a block of bands at once: vectors of band j of the
// block sit at offset j*n, its scalars in sc[j].  Each band sees the same
// operations and tree orders as in the band-by-band loop.
static_assert(sizeof(Sc) % sizeof(double) == 0, "Sc fields are addressed as doubles");
constexpr long kScStride = sizeof(Sc) / sizeof(double);

// out[j*ostride] = tree_dot(A_j, B_j) (times dV when scale)
template <class T>
__global__ void k_pdot_partial(long n, const T* __restrict__ A, const T* __restrict__ Bv,
                               long nblk, double* __restrict__ part) {
  __shared__ double ws[8];
  const int j = blockIdx.y;
  const T* a = A + (long)j * n;
  const T* b = Bv + (long)j * n;
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < n) acc = fma((double)a[i], (double)b[i], acc);
  }
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) part[(long)j * nblk + blockIdx.x] = s;
}

__global__ void k_pdot_final(long nblk, const double* __restrict__ part, double dx, double dy,
                             double dz, int scale, double* __restrict__ out, long ostride) {
  __shared__ double ws[8];
  const int j = blockIdx.x;
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + part[(long)j * nblk + k];
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) out[(long)j * ostride] = scale ? s * dx * dy * dz : s;
}

// c_j = a_j + d_j b_j, d_j = sign * dp[j*dstride]  (ksdiis_r_01); V
// consecutive values per thread (V divides n)
template <class T, int V>
__global__ void k_axpy_b(long n, const T* __restrict__ a, const T* __restrict__ b,
                         const double* __restrict__ dp, long dstride, double sign,
                         T* __restrict__ c) {
  const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) * V;
  if (i >= n) return;
  const long o = (long)blockIdx.y * n + i;
  const T d = (T)(sign * dp[(long)blockIdx.y * dstride]);
  const Pack<T, V> av = ldpk<T, V>(a + o), bv = ldpk<T, V>(b + o);
  Pack<T, V> cv;
#pragma unroll
  for (int k = 0; k < V; ++k) cv.v[k] = fma(d, bv.v[k], av.v[k]);
  stpk<T, V>(c + o, cv);
}

// ---- fused DIIS passes.  Each forms the trial vectors of ksdiis_r on the
// fly, with the same T-precision formula in every pass (the step, eigenvalue
// and combination coefficients rounded to T once; for T = double the Fortran
// statement's FMA), and accumulates every dot product it needs in FP64 in the
// fixed tree order, so each band sees the same values as with the vectors
// stored.  The FP32 path so forms its vectors in FP32 arithmetic, which keeps
// the passes clear of FP32<->FP64 conversions.  part layout: [dot][band][chunk].
//
// Trial-step sums (ksdiis8f.F90:285-300) with a1 = alambda_diis:
//   rvre.hs, rvre.ss, ph1.hph1, ph1.sph1 with ph1 = ps + a1 rvre,
//   hph1 = hs + a1 avre, sph1 = ss + a1 asvre (ph1 when S = 1).
template <class T, bool SP>
__global__ void k_diis_dots_a(long n, const T* __restrict__ ps, const T* __restrict__ rvre,
                              const T* __restrict__ hs, const T* __restrict__ avre,
                              const T* __restrict__ ss, const T* __restrict__ asvre,
                              const double* __restrict__ a1p, long nblk,
                              double* __restrict__ part) {
  __shared__ double ws[8];
  const int j = blockIdx.y, nb = gridDim.y;
  const long off = (long)j * n;
  const T a1 = (T)*a1p;
  double acc[4] = {0.0, 0.0, 0.0, 0.0};
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
#pragma unroll 4
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < n) {
      const long o = off + i;
      const T rt = rvre[o], ht = hs[o], pt = ps[o];
      const T st = SP ? ss[o] : pt;
      const T p1 = fma(a1, rt, pt);
      const T h1 = fma(a1, avre[o], ht);
      const T s1 = SP ? fma(a1, asvre[o], st) : p1;
      const double r = (double)rt, h = (double)ht, s = (double)st;
      acc[0] = fma(r, h, acc[0]);
      acc[1] = fma(r, s, acc[1]);
      acc[2] = fma((double)p1, (double)h1, acc[2]);
      acc[3] = fma((double)p1, (double)s1, acc[3]);
    }
  }
#pragma unroll
  for (int d = 0; d < 4; ++d) {
    const double v = tree_fold256(acc[d], ws);
    if (threadIdx.x == 0) part[((long)d * nb + j) * nblk + blockIdx.x] = v;
  }
}

// DIIS matrix sums (ksdiis8f.F90:321-404) with the step lam of band j:
//   ps.ss, rvv0.rvv0, ps.sph1, rvv0.rvv1, ph1.sph1, rvv1.rvv1 with
//   ph1 = ps + lam rvre, hph1 = hs + lam avre, sph1 = ss + lam asvre,
//   rvv1 = hph1 - sval sph1, and the first residual rvv0 = hs - sval ss
//   formed again as ksdiis_r_01 formed it (so it is never stored).
template <class T, bool SP>
__global__ void k_diis_dots_b(long n, const T* __restrict__ ps, const T* __restrict__ rvre,
                              const T* __restrict__ hs, const T* __restrict__ avre,
                              const T* __restrict__ ss, const T* __restrict__ asvre,
                              const Sc* __restrict__ sc, const double* __restrict__ sval,
                              long nblk, double* __restrict__ part) {
  __shared__ double ws[8];
  const int j = blockIdx.y, nb = gridDim.y;
  const long off = (long)j * n;
  const T lam = (T)sc[j].lam, ev = (T)(-1.0 * sval[j]);
  double acc[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
#pragma unroll 4
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < n) {
      const long o = off + i;
      const T pt = ps[o];
      const T st = SP ? ss[o] : pt;
      const T ht = hs[o];
      const double p = (double)pt, s = (double)st;
      const double v0 = (double)fma(ev, st, ht);
      const T p1 = fma(lam, rvre[o], pt);
      const T h1 = fma(lam, avre[o], ht);
      const T s1 = SP ? fma(lam, asvre[o], st) : p1;
      const double v1 = (double)fma(ev, s1, h1);
      acc[0] = fma(p, s, acc[0]);
      acc[1] = fma(v0, v0, acc[1]);
      acc[2] = fma(p, (double)s1, acc[2]);
      acc[3] = fma(v0, v1, acc[3]);
      acc[4] = fma((double)p1, (double)s1, acc[4]);
      acc[5] = fma(v1, v1, acc[5]);
    }
  }
#pragma unroll
  for (int d = 0; d < 6; ++d) {
    const double v = tree_fold256(acc[d], ws);
    if (threadIdx.x == 0) part[((long)d * nb + j) * nblk + blockIdx.x] = v;
  }
}

// chunk sums -> out[d][j * ostride] (times dV where scale[d]); grid (nb, ndot)
struct DotOuts {
  double* out[6];
  int scale[6];
};
__global__ void k_dots_final(long nblk, const double* __restrict__ part, double dx, double dy,
                             double dz, DotOuts o, long ostride) {
  __shared__ double ws[8];
  const int j = blockIdx.x, d = blockIdx.y, nb = gridDim.x;
  const double* p = part + ((long)d * nb + j) * nblk;
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + p[k];
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) o.out[d][(long)j * ostride] = o.scale[d] ? s * dx * dy * dz : s;
}

// The DIIS combination (ksdiis8f.F90:549-600) of band j with the normalised
// trial vectors: y1 = tmp * (y + lam dy), new = c1 y1 + c0 y for psi, S psi
// (with an S metric) and, when upd_h, H psi.  V consecutive values per thread
// (V divides n).
template <class T, bool SP, int V>
__device__ __forceinline__ void diis_comb_vec(long o, T* y, const T* __restrict__ dy, double lam,
                                              double t, double c0, double c1) {
  const Pack<T, V> yv = ldpk<T, V>(y + o), dv = ldpk<T, V>(dy + o);
  const T lt = (T)lam, tt = (T)t, c0t = (T)c0, c1t = (T)c1;
  Pack<T, V> nv;
#pragma unroll
  for (int k = 0; k < V; ++k) {
    const T a = yv.v[k];
    const T a1 = fma(lt, dv.v[k], a) * tt;
    nv.v[k] = fma(c1t, a1, c0t * a);
  }
  stpk<T, V>(y + o, nv);
}
template <class T, bool SP, int V>
__global__ void k_diis_comb(long n, T* ps, const T* __restrict__ rvre, T* hs,
                            const T* __restrict__ avre, T* ss, const T* __restrict__ asvre,
                            const Sc* __restrict__ sc, int upd_h) {
  const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) * V;
  if (i >= n) return;
  const Sc& q = sc[blockIdx.y];
  const double lam = q.lam, t = q.tmp, c0 = q.c[0], c1 = q.c[1];
  const long o = (long)blockIdx.y * n + i;
  diis_comb_vec<T, SP, V>(o, ps, rvre, lam, t, c0, c1);
  if (SP) diis_comb_vec<T, SP, V>(o, ss, asvre, lam, t, c0, c1);
  if (upd_h) diis_comb_vec<T, SP, V>(o, hs, avre, lam, t, c0, c1);
}
__global__ void k_diis_comb_rp(long n, double* rps, const double* __restrict__ rpsep,
                               const Sc* __restrict__ sc) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Sc& q = sc[blockIdx.y];
  const long o = (long)blockIdx.y * n + i;
  const double r = rps[o];
  const double r1 = fma(q.lam, rpsep[o], r) * q.tmp;
  double acc = 0.0;
  acc = fma(q.c[0], r, acc);
  acc = fma(q.c[1], r1, acc);
  rps[o] = acc;
}

__global__ void k_diis_lambda_b(int nb, Sc* sc, const double* __restrict__ sval, double a1,
                                double dx, double dy, double dz, double lmin, double lmax) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nb) diis_lambda(sc + j, sval + j, a1, dx, dy, dz, lmin, lmax);
}

// the symmetric entries of the 2x2 matrices, then tmp = 1/sqrt(rs(2,2))
__global__ void k_diis_norm_b(int nb, Sc* sc) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nb) return;
  Sc* s = sc + j;
  s->rs[1 * 2 + 0] = s->rs[0 * 2 + 1];
  s->rr[1 * 2 + 0] = s->rr[0 * 2 + 1];
  s->tmp = 1.0 / sqrt(s->rs[3]);
}

__global__ void k_diis_scale_mats_b(int nb, Sc* sc) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nb) diis_scale_mats(sc + j);
}

__global__ void k_diis_solve_b(int nb, Sc* sc, double eps_eig, double* __restrict__ resid) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nb) diis_solve(sc + j, eps_eig, resid + j);
}

// dst band dband[k] = src band sband[k] for k = blockIdx.y (bands of n
// values, V consecutive values per thread, V divides n)
template <class T, int V>
__global__ void k_move_bands(long n, const int* __restrict__ sband, const T* __restrict__ src,
                             const int* __restrict__ dband, T* __restrict__ dst) {
  const long e = ((long)blockIdx.x * blockDim.x + threadIdx.x) * V;
  if (e >= n) return;
  const int k = blockIdx.y;
  stpk<T, V>(dst + (long)dband[k] * n + e, ldpk<T, V>(src + (long)sband[k] * n + e));
}

// T[b][a][i] = sum_j S_a(i, j) <p_j|psi_b> with S_a(i, j) = m[(a*P + i)*P + j]
// (the projector sums of S psi before the 1/dV, in the order of k_tcoef_f32)
__global__ void k_s_rp(int M, int natom, int P, const int* __restrict__ nprj,
                       const double* __restrict__ m, const double* __restrict__ rp,
                       double* __restrict__ T) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M * natom * P) return;
  const int i = (int)(idx % P);
  const long ba = idx / P;
  const int a = (int)(ba % natom);
  const int pa = nprj[a];
  const double* r = rp + ba * P;
  const double* s = m + ((long)a * P + i) * P;
  double acc = 0.0;
  if (i < pa)
    for (int j = 0; j < pa; ++j) acc = fma(r[j], s[j], acc);
  T[idx] = acc;
}

// A(i, j) = A(j, i) for i < j (column-major M x M): the upper triangle
// becomes the mirror of the lower one
__global__ void k_mirror_lower(int M, double* A) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)M * M) return;
  const int i = (int)(idx % M), j = (int)(idx / M);
  if (i < j) A[(long)j * M + i] = A[(long)i * M + j];
}

}  // namespace

// ============================================================ the solver
template <class T>
struct BandCtx {
  const rs_geom* g;
  const T* veff;
  const double* dij;
  const double* sss;  // nullptr: S = 1 (spsi aliases psi)
  int M;
  T* psi;
  T* spsi;
  double* rp;
  T* hpsi;
  cudaStream_t st;
  long N;
  int nrp;
  double dx, dy, dz;
  // work
  double* part = nullptr;
  long nblk = 0;
  double* coef = nullptr;  // M+1
  Sc* sc = nullptr;
  T* w[8] = {};
  double* wrp[6] = {};
  int status_err = RS_OK;

  bool sep() const { return sss != nullptr; }

  int init(int nvec, int nrpv) {
    N = g->N;
    nrp = g->natom * g->nprjmx;
    dx = g->dx; dy = g->dy; dz = g->dz;
    nblk = tree_chunks(N);
    RS_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * nblk * (M + 2), st));
    RS_CUDA(cudaMallocAsync((void**)&coef, sizeof(double) * (M + 2), st));
    RS_CUDA(cudaMallocAsync((void**)&sc, sizeof(Sc), st));
    RS_CUDA(cudaMemsetAsync(sc, 0, sizeof(Sc), st));
    for (int k = 0; k < nvec; ++k) {
      RS_CUDA(cudaMallocAsync((void**)&w[k], sizeof(T) * N, st));
      RS_CUDA(cudaMemsetAsync(w[k], 0, sizeof(T) * N, st));
    }
    for (int k = 0; k < nrpv; ++k) {
      RS_CUDA(cudaMallocAsync((void**)&wrp[k], sizeof(double) * (nrp > 0 ? nrp : 1), st));
      RS_CUDA(cudaMemsetAsync(wrp[k], 0, sizeof(double) * (nrp > 0 ? nrp : 1), st));
    }
    return RS_OK;
  }
  void release() {
    if (part) cudaFreeAsync(part, st);
    if (coef) cudaFreeAsync(coef, st);
    if (sc) cudaFreeAsync(sc, st);
    for (auto& p : w)
      if (p) { cudaFreeAsync(p, st); p = nullptr; }
    for (auto& p : wrp)
      if (p) { cudaFreeAsync(p, st); p = nullptr; }
  }

  T* band(T* base, int l) const { return base + (long)l * N; }
  double* rpb(double* base, int l) const { return base + (long)l * nrp; }

  // out[j] = dot(Y_j, x) (times dV when scale)
  int bdot(const T* Y, int cnt, const T* x, double* out, int scale = 1) {
    if (cnt <= 0) return RS_OK;
    dim3 grid((unsigned)nblk, cnt);
    k_bdot_partial<T><<<grid, kTreeLanes, 0, st>>>(N, Y, N, x, nblk, part);
    k_bdot_final<<<cnt, kTreeLanes, 0, st>>>(nblk, part, dx, dy, dz, scale, out);
    RS_LAUNCH_CHECK("bdot");
    return RS_OK;
  }
  void subcomb(T* x, const T* Y, const double* c, int cnt) {
    if (cnt > 0) k_subcomb<T><<<div_up(N, 256), 256, 0, st>>>(N, x, Y, N, c, cnt);
  }
  void subcomb_rp(double* x, const double* Y, const double* c, int cnt) {
    if (cnt > 0 && nrp > 0) k_subcomb_d<<<div_up(nrp, 256), 256, 0, st>>>(nrp, x, Y, nrp, c, cnt);
  }
  int apply_h(const T* x, const double* r, T* out, int nb) {
    if constexpr (sizeof(T) == 4)
      return launch_hpsi_f32_fast(g, (const float*)veff, dij, r, (const float*)x, (float*)out, nb, st);
    else
      return launch_gather<double, 1>(g, dij, r, (const double*)x, (const double*)veff,
                                      (double*)out, nb, st);
  }
  int apply_s(const T* x, const double* r, T* out, int nb) {
    if (!sss) {
      if (out != x) RS_CUDA(cudaMemcpyAsync(out, x, sizeof(T) * N * nb, cudaMemcpyDeviceToDevice, st));
      return RS_OK;
    }
    if constexpr (sizeof(T) == 4) {
      if (spsi_f32_fast_ok(g))
        return launch_spsi_f32_fast(g, sss, r, (const float*)x, (float*)out, nb, st);
    }
    return launch_gather<T, 2>(g, sss, r, x, nullptr, out, nb, st);
  }
  int nl_dot(const T* x, double* r, int nb) {
    if (g->natom == 0) return RS_OK;
    return launch_nl_dot<T>(g, x, nb, r, st);
  }
  int precond(const T* in, T* out) { return launch_precondition<T>(g, in, out, 1, st); }
  unsigned gN() const { return div_up(std::max(N, (long)nrp), 256); }

  // normalise x (and sx, r) by 1/sqrt(dot(x, sx) dV)
  int normalize(T* x, T* sx, double* r) {
    int rc;
    if ((rc = bdot(sx, 1, x, &sc->vecnor))) return rc;
    k_invsqrt<<<1, 1, 0, st>>>(&sc->vecnor, &sc->tmp, &sc->status);
    k_scale3<T><<<gN(), 256, 0, st>>>(N, x, sep() ? sx : nullptr, nrp, r, &sc->tmp);
    RS_LAUNCH_CHECK("normalize");
    return RS_OK;
  }

  // orthogonalization_r_01 for the single band l (l_inp = l+1), level-1 GS
  int ortho_band(int l, bool cmpt) {
    int rc;
    T* x = band(psi, l);
    T* sx = band(spsi, l);
    double* r = rpb(rp, l);
    if (cmpt) {
      if ((rc = nl_dot(x, r, 1))) return rc;
      if (sep() && (rc = apply_s(x, r, sx, 1))) return rc;
    }
    if (l > 0) {
      // coef[j] = dot(spsi_j, psi_l) dV
      if ((rc = bdot(spsi, l, x, coef))) return rc;
      subcomb(x, psi, coef, l);
      if (sep()) subcomb(sx, spsi, coef, l);
      subcomb_rp(r, rp, coef, l);
    }
    return normalize(x, sx, r);
  }

  // Cholesky-QR of all bands in the S metric (block GS of
  // orthogonalization_r_01 with l_inp=0): G = dV Psi^T S Psi = L L^T,
  // Psi <- Psi L^-T, S Psi and <p|Psi> likewise.
  int ortho_all(bool cmpt) {
    int rc;
    // FP32 with an S metric: dV Psi^T S Psi = dV Psi^T Psi + <p|Psi>^T S <p|Psi>
    // (the nonlocal part of S psi is sum_a |p> S_a <p|psi> / dV), so the Gram
    // needs <p|Psi> but not S Psi, which rotate_all forms afterwards
    const bool split = sizeof(T) == 4 && sep() && nrp > 0;
    if (cmpt) {
      if ((rc = nl_dot(psi, rp, M))) return rc;
      if (sep() && !split && (rc = apply_s(psi, rp, spsi, M))) return rc;
    }
    double *G = nullptr, *W = nullptr;
    RS_CUDA(cudaMallocAsync((void**)&G, sizeof(double) * 2 * (size_t)M * M, st));
    W = G + (size_t)M * M;
    const double dv = dx * dy * dz;
    if constexpr (sizeof(T) == 4) {
      // the Cholesky reads the lower triangle only: one triangle of tile pairs
      if (split) {
        rc = gram_f32(M, M, N, (const float*)psi, N, (const float*)psi, N, dv, G, M, 1, st);
        double* Ts = nullptr;
        if (!rc) {
          cudaError_t e = cudaMallocAsync((void**)&Ts, sizeof(double) * (size_t)nrp * M, st);
          if (e != cudaSuccess) rc = cuda_status(e, "ortho_all: S <p|psi>");
        }
        if (!rc) {
          k_s_rp<<<div_up((long)nrp * M, 256), 256, 0, st>>>(M, g->natom, g->nprjmx, g->d_nprj,
                                                              sss, rp, Ts);
          rc = gram_f64_beta(M, M, nrp, rp, nrp, Ts, nrp, 1.0, 1.0, G, M, st);
        }
        if (Ts) cudaFreeAsync(Ts, st);
      } else {
        rc = gram_f32(M, M, N, (const float*)psi, N, (const float*)spsi, N, dv, G, M,
                      spsi == psi ? 1 : 2, st);
      }
    } else {
      rc = gram_f64(M, M, N, (const double*)psi, N, (const double*)spsi, N, dv, G, M, st);
    }
    if (!rc) rc = chol_inv_t(M, G, W, st);
    if (!rc) rc = rotate_all(W);
    cudaFreeAsync(G, st);
    return rc;
  }

  // Psi <- Psi Z, S Psi <- S Psi Z, <p|Psi> <- <p|Psi> Z (Z FP64 M x M).
  // The FP32 rotation packs its operand into tensor-core blocks before the
  // product reads anything, so it writes the result over Psi in place.  On
  // the FP32 path S Psi Z is formed as S (Psi Z) from the rotated Psi and
  // <p|Psi> Z (S is linear; one S pass costs a sixth of a rotation); the
  // FP64 path rotates S Psi, its product (a library GEMM) through a work
  // array.
  int rotate_all(const double* Z) {
    int rc = RS_OK;
    T* arrs[2] = {psi, sep() ? spsi : nullptr};
    if constexpr (sizeof(T) == 4) {
      rc = rotate_f32(N, M, M, (const float*)psi, N, Z, M, (float*)psi, N, st);
      if (!rc && nrp > 0) rc = rotate_rp(Z);
      if (!rc && sep()) rc = apply_s(psi, rp, spsi, M);
      return rc;
    } else {
      T* tmp = nullptr;
      RS_CUDA(cudaMallocAsync((void**)&tmp, sizeof(T) * (size_t)N * M, st));
      for (T* a : arrs) {
        if (!a || rc) continue;
        rc = rotate_f64(N, M, M, (const double*)a, N, Z, M, (double*)tmp, N, st);
        if (!rc) {
          cudaError_t e = cudaMemcpyAsync(a, tmp, sizeof(T) * (size_t)N * M,
                                          cudaMemcpyDeviceToDevice, st);
          if (e != cudaSuccess) rc = cuda_status(e, "rotate copy");
        }
      }
      cudaFreeAsync(tmp, st);
    }
    if (rc || nrp == 0) return rc;
    return rotate_rp(Z);
  }
  // <p|Psi> <- <p|Psi> Z (FP64)
  int rotate_rp(const double* Z) {
    double* tr = nullptr;
    RS_CUDA(cudaMallocAsync((void**)&tr, sizeof(double) * (size_t)nrp * M, st));
    int rc = rotate_f64(nrp, M, M, rp, nrp, Z, M, tr, nrp, st);
    if (!rc) RS_CUDA(cudaMemcpyAsync(rp, tr, sizeof(double) * (size_t)nrp * M,
                                     cudaMemcpyDeviceToDevice, st));
    cudaFreeAsync(tr, st);
    return rc;
  }

  int check_status() {
    int h = 0;
    RS_CUDA(cudaMemcpyAsync(&h, &sc->status, sizeof(int), cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaStreamSynchronize(st));
    if (h) return fail(RS_ENUMERIC, "band solver: vector has negative norm");
    return RS_OK;
  }
};

template <class T>
static int kscg(BandCtx<T>& c, const rs_solver_prm* prm, double* sval_h, double* resid_h,
                int* itmax) {
  int rc = c.init(7, 4);
  if (rc) return rc;
  const long N = c.N;
  T *rvec = c.w[0], *pvec = c.w[1], *pv = c.w[2], *rv = c.w[3], *spv = c.w[4], *asv = c.w[5],
    *av = c.w[6];
  double *rrp = c.wrp[0], *rpp = c.wrp[1], *rpl = c.wrp[2], *dsval = c.wrp[3];
  double* dval = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&dval, sizeof(double) * (c.M + 1), c.st));
  const int nsdmax1 = 10, nsdmax2 = 200;
  int itm = 0;
  for (int l = 0; l < c.M && !rc; ++l) {
    T* psl = c.band(c.psi, l);
    T* ssl = c.band(c.spsi, l);
    T* hsl = c.band(c.hpsi, l);
    double* rpsl = c.rpb(c.rp, l);
    for (int loop = 0; loop < prm->northo && !rc; ++loop) rc = c.ortho_band(l, prm->northo == 2);
    if (!rc) rc = c.apply_h(psl, rpsl, hsl, 1);
    int iiter = 0;
    bool conv = false;
    while (!rc && iiter < prm->nsdmax && !conv) {
      ++iiter;
      bool reset = (iiter == 1) || (iiter == nsdmax1);
      if (nsdmax2 > 0) reset = reset || ((iiter - 1) % nsdmax2 == 0);
      if (reset) {
        const double one = 1.0;
        cudaMemcpyAsync(&c.sc->r2rr, &one, sizeof(double), cudaMemcpyHostToDevice, c.st);
        cudaMemsetAsync(pvec, 0, sizeof(T) * N, c.st);
        cudaMemsetAsync(rvec, 0, sizeof(T) * N, c.st);
        cudaMemsetAsync(pv, 0, sizeof(T) * N, c.st);
        cudaMemsetAsync(spv, 0, sizeof(T) * N, c.st);
        if (c.nrp) cudaMemsetAsync(rpp, 0, sizeof(double) * c.nrp, c.st);
      }
      k_copy_d<<<1, 1, 0, c.st>>>(&c.sc->r1rr, &c.sc->r2rr);
      if ((rc = c.bdot(psl, 1, hsl, &c.sc->valre))) break;
      k_copy_d<<<1, 1, 0, c.st>>>(dval + l, &c.sc->valre);
      k_resid<T><<<div_up(N, 256), 256, 0, c.st>>>(N, hsl, ssl, &c.sc->valre, rvec);
      if (prm->nprecon_cg) rc = c.precond(rvec, rv);
      else cudaMemcpyAsync(rv, rvec, sizeof(T) * N, cudaMemcpyDeviceToDevice, c.st);
      for (int loop = 0; loop < prm->northo && !rc; ++loop) {
        if ((rc = c.bdot(c.spsi, l + 1, rv, c.coef))) break;
        c.subcomb(rv, c.psi, c.coef, l + 1);
      }
      if (rc) break;
      if ((rc = c.nl_dot(rv, rrp, 1))) break;
      if ((rc = c.apply_s(rv, rrp, asv, 1))) break;
      if ((rc = c.bdot(rv, 1, rvec, &c.sc->r2rr))) break;
      k_copy_d<<<1, 1, 0, c.st>>>(dsval + 0, &c.sc->r2rr);  // resid of this band
      k_cg_ratio<<<1, 1, 0, c.st>>>(c.sc);
      k_cg_dir<T><<<c.gN(), 256, 0, c.st>>>(N, pvec, rv, pv, c.sep() ? spv : nullptr, asv,
                                             c.nrp, rpp, rrp, &c.sc->ratio);
      if (c.nrp) cudaMemcpyAsync(rpl, rpp, sizeof(double) * c.nrp, cudaMemcpyDeviceToDevice, c.st);
      if (c.sep()) cudaMemcpyAsync(asv, spv, sizeof(T) * N, cudaMemcpyDeviceToDevice, c.st);
      else cudaMemcpyAsync(asv, pvec, sizeof(T) * N, cudaMemcpyDeviceToDevice, c.st);
      for (int loop = 0; loop < prm->northo && !rc; ++loop) {
        if ((rc = c.bdot(c.spsi, l + 1, pvec, c.coef))) break;
        c.subcomb(pvec, c.psi, c.coef, l + 1);
        if (c.sep()) c.subcomb(asv, c.spsi, c.coef, l + 1);
        else c.subcomb(asv, c.psi, c.coef, l + 1);
        c.subcomb_rp(rpl, c.rp, c.coef, l + 1);
      }
      if (rc) break;
      if ((rc = c.bdot(asv, 1, pvec, &c.sc->vecnor))) break;
      k_invsqrt<<<1, 1, 0, c.st>>>(&c.sc->vecnor, &c.sc->tmp, &c.sc->status);
      k_scale3<T><<<c.gN(), 256, 0, c.st>>>(N, pvec, asv, c.nrp, rpl, &c.sc->tmp);
      if ((rc = c.apply_h(pvec, rpl, av, 1))) break;
      if ((rc = c.bdot(pvec, 1, av, &c.sc->pap))) break;
      if ((rc = c.bdot(psl, 1, av, &c.sc->sapre))) break;
      k_cg_alphabeta<<<1, 1, 0, c.st>>>(c.sc, dval + l);
      k_cg_rot<T><<<c.gN(), 256, 0, c.st>>>(N, psl, pvec, hsl, av, c.sep() ? ssl : nullptr, asv,
                                             c.nrp, rpsl, rpl, c.sc->ab);
      double r2 = 0.0;
      int bad = 0;
      RS_CUDA(cudaMemcpyAsync(&r2, dsval, sizeof(double), cudaMemcpyDeviceToHost, c.st));
      RS_CUDA(cudaMemcpyAsync(&bad, &c.sc->status, sizeof(int), cudaMemcpyDeviceToHost, c.st));
      RS_CUDA(cudaStreamSynchronize(c.st));
      cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) { rc = cuda_status(e, "kscg"); break; }
      if (bad) { rc = fail(RS_ENUMERIC, "kscg_r: pvec has negative norm"); break; }
      resid_h[l] = r2;
      conv = sqrt(r2) < prm->epssd;
    }
    if (iiter > itm) itm = iiter;
  }
  if (!rc) {
    RS_CUDA(cudaMemcpyAsync(sval_h, dval, sizeof(double) * c.M, cudaMemcpyDeviceToHost, c.st));
    RS_CUDA(cudaStreamSynchronize(c.st));
  }
  if (itmax) *itmax = itm;
  cudaFreeAsync(dval, c.st);
  c.release();
  return rc;
}

template <class T>
static int ksdiis(BandCtx<T>& c, const rs_solver_prm* prm, int l_hsv, double* sval_h,
                  double* resid_h, int* ksconv) {
  int rc = c.init(0, 0);
  if (rc) return rc;
  const long N = c.N;
  const long nrp = c.nrp;
  const bool sp = c.sep();
  const int M = c.M;
  // a block of B bands runs each step of the band loop at once; its work
  // vectors (the residual, the preconditioned residual and its H image, plus
  // its S image with an S metric) stay within ~8 GB.  The trial vectors
  // phi1, H phi1, S phi1 and the second residual are formed on the fly by
  // the fused passes.
  const int nvec = sp ? 4 : 3;
  const long per_band = (long)nvec * N * (long)sizeof(T) + nrp * (long)sizeof(double);
  const int B = (int)std::min<long>(std::min<long>(M, 65535),
                                    std::max<long>(1, (8L << 30) / per_band));
  T* wv = nullptr;
  double* wd = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&wv, sizeof(T) * (size_t)nvec * B * N, c.st));
  const size_t nd = (size_t)B * (nrp > 0 ? nrp : 1) + 2 * (M + 1) + 1;
  cudaError_t e = cudaMallocAsync((void**)&wd, sizeof(double) * nd, c.st);
  Sc* scb = nullptr;
  double* dpart = nullptr;  // chunk sums of the fused passes: [6][B][nblk]
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&scb, sizeof(Sc) * B, c.st);
  if (e == cudaSuccess) e = cudaMemsetAsync(scb, 0, sizeof(Sc) * B, c.st);
  if (e == cudaSuccess)
    e = cudaMallocAsync((void**)&dpart, sizeof(double) * 6 * (size_t)B * c.nblk, c.st);
  if (e != cudaSuccess) rc = cuda_status(e, "ksdiis: work arrays");
  const size_t BN = (size_t)B * N;
  T* rvv0 = wv;
  T* rvre = rvv0 + BN;
  T* avre = rvre + BN;
  T* asvre = sp ? avre + BN : nullptr;
  double* rpsep = wd;
  double* dval = rpsep + (size_t)B * (nrp > 0 ? nrp : 1);
  double* dres = dval + M + 1;
  double* da1 = dres + M + 1;
  const double a1 = prm->alambda_diis;
  constexpr int V = 16 / (int)sizeof(T);
  auto aligned16 = [](const void* p) { return (uintptr_t)p % 16 == 0; };
  if (!rc) {
    cudaMemcpyAsync(dres, resid_h, sizeof(double) * M, cudaMemcpyHostToDevice, c.st);
    cudaMemcpyAsync(da1, &a1, sizeof(double), cudaMemcpyHostToDevice, c.st);
  }
  auto pdot = [&](const T* a, const T* b, int nb, double* out, long ostride, int scale) {
    dim3 grid((unsigned)c.nblk, nb);
    k_pdot_partial<T><<<grid, kTreeLanes, 0, c.st>>>(N, a, b, c.nblk, c.part);
    k_pdot_final<<<nb, kTreeLanes, 0, c.st>>>(c.nblk, c.part, c.dx, c.dy, c.dz, scale, out,
                                              ostride);
  };
  for (int b0 = 0; b0 < M && !rc; b0 += B) {
    const int nb = std::min(B, M - b0);
    T* ps = c.band(c.psi, b0);                 // phi0 (psi), overwritten by the combination
    T* ss = sp ? c.band(c.spsi, b0) : ps;      // S phi0
    T* hs = c.band(c.hpsi, b0);                // H phi0, computed afresh each sweep
    double* rps = c.rpb(c.rp, b0);
    const dim3 gv(div_up(N, 256), nb), gr(div_up(nrp > 0 ? nrp : 1, 256), nb);
    const dim3 gvv(div_up(N / V, 256), nb);
    // 16-byte vectors when a band is a whole number of them and every band
    // vector starts on a 16-byte boundary
    const bool vec = N % V == 0 && aligned16(ps) && aligned16(ss) && aligned16(hs) &&
                     aligned16(wv);
    const dim3 gd((unsigned)c.nblk, nb);
    const unsigned gs = div_up(nb, 128);
    for (int jiter = 1; jiter + 1 <= prm->ndiismax && !rc; ++jiter) {
      if ((rc = c.apply_h(ps, rps, hs, nb))) break;
      pdot(ps, hs, nb, dval + b0, 1, 1);
      // the first residual, smoothed into rvre (or rvre itself without a
      // preconditioner)
      T* r0 = prm->nprecon_diis ? rvv0 : rvre;
      if (vec) k_axpy_b<T, V><<<gvv, 256, 0, c.st>>>(N, hs, ss, dval + b0, 1, -1.0, r0);
      else k_axpy_b<T, 1><<<gv, 256, 0, c.st>>>(N, hs, ss, dval + b0, 1, -1.0, r0);
      if (prm->nprecon_diis && (rc = launch_precondition<T>(c.g, rvv0, rvre, nb, c.st))) break;
      if ((rc = c.nl_dot(rvre, rpsep, nb))) break;
      if ((rc = c.apply_h(rvre, rpsep, avre, nb))) break;
      if (sp && (rc = c.apply_s(rvre, rpsep, asvre, nb))) break;
      // trial step with alambda_diis: the four line-search sums in one pass
      if (sp)
        k_diis_dots_a<T, true><<<gd, kTreeLanes, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre, da1,
                                                            c.nblk, dpart);
      else
        k_diis_dots_a<T, false><<<gd, kTreeLanes, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre,
                                                             da1, c.nblk, dpart);
      {
        DotOuts o{};
        for (int d = 0; d < 4; ++d) { o.out[d] = &scb->s[d]; o.scale[d] = 0; }
        k_dots_final<<<dim3(nb, 4), kTreeLanes, 0, c.st>>>(c.nblk, dpart, c.dx, c.dy, c.dz, o,
                                                          kScStride);
      }
      k_diis_lambda_b<<<gs, 128, 0, c.st>>>(nb, scb, dval + b0, a1, c.dx, c.dy, c.dz,
                                            prm->alambda_min, prm->alambda_max);
      // the 2x2 DIIS matrices at the step lam, in one pass
      if (sp)
        k_diis_dots_b<T, true><<<gd, kTreeLanes, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre,
                                                            scb, dval + b0, c.nblk, dpart);
      else
        k_diis_dots_b<T, false><<<gd, kTreeLanes, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre,
                                                             scb, dval + b0, c.nblk, dpart);
      {
        DotOuts o{};
        double* outs[6] = {&scb->rs[0], &scb->rr[0], &scb->rs[1],
                           &scb->rr[1], &scb->rs[3], &scb->rr[3]};
        for (int d = 0; d < 6; ++d) { o.out[d] = outs[d]; o.scale[d] = 1; }
        k_dots_final<<<dim3(nb, 6), kTreeLanes, 0, c.st>>>(c.nblk, dpart, c.dx, c.dy, c.dz, o,
                                                          kScStride);
      }
      k_diis_norm_b<<<gs, 128, 0, c.st>>>(nb, scb);
      k_diis_scale_mats_b<<<gs, 128, 0, c.st>>>(nb, scb);
      k_diis_solve_b<<<gs, 128, 0, c.st>>>(nb, scb, prm->eps_eig_diis, dres + b0);
      // combination with the normalised trial vectors (formed again on the fly)
      // H phi is recomputed at the top of the next sweep: only the last sweep
      // leaves the combined H psi
      const int upd_h = jiter + 2 > prm->ndiismax;
      if (vec && sp)
        k_diis_comb<T, true, V><<<gvv, 256, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre, scb, upd_h);
      else if (vec)
        k_diis_comb<T, false, V><<<gvv, 256, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre, scb,
                                                        upd_h);
      else if (sp)
        k_diis_comb<T, true, 1><<<gv, 256, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre, scb, upd_h);
      else
        k_diis_comb<T, false, 1><<<gv, 256, 0, c.st>>>(N, ps, rvre, hs, avre, ss, asvre, scb,
                                                       upd_h);
      if (nrp) k_diis_comb_rp<<<gr, 256, 0, c.st>>>(nrp, rps, rpsep, scb);
      e = cudaGetLastError();
      if (e != cudaSuccess) rc = cuda_status(e, "ksdiis");
    }
  }
  if (!rc) {
    RS_CUDA(cudaMemcpyAsync(sval_h, dval, sizeof(double) * M, cudaMemcpyDeviceToHost, c.st));
    RS_CUDA(cudaMemcpyAsync(resid_h, dres, sizeof(double) * M, cudaMemcpyDeviceToHost, c.st));
    RS_CUDA(cudaStreamSynchronize(c.st));
    int conv = 1;
    for (int l = 0; l < M; ++l) conv = conv && (sqrt(resid_h[l]) <= prm->epssd);
    if (ksconv) *ksconv = conv;
  }
  if (!rc && l_hsv) {
    for (int i = 0; i < prm->northo && !rc; ++i) rc = c.ortho_all(true);
    if (!rc) rc = c.apply_h(c.psi, c.rp, c.hpsi, c.M);
  }
  if (wv) cudaFreeAsync(wv, c.st);
  if (wd) cudaFreeAsync(wd, c.st);
  if (scb) cudaFreeAsync(scb, c.st);
  if (dpart) cudaFreeAsync(dpart, c.st);
  c.release();
  return rc;
}

// rayleighritz_r: A = dV Psi^T H Psi (lower triangle), eigen, rotations
template <class T>
static int rayleighritz(BandCtx<T>& c, int l_rrb, double* sval_h) {
  c.N = c.g->N;
  c.nrp = c.g->natom * c.g->nprjmx;
  c.dx = c.g->dx; c.dy = c.g->dy; c.dz = c.g->dz;
  const int M = c.M;
  int rc = RS_OK;
  // FP32 with projectors, H psi recomputed here: dV Psi^T H Psi = dV Psi^T
  // (-1/2 lap + veff) Psi + <p|Psi>^T D <p|Psi>, so only the local part is
  // applied (hpsi is work space on exit)
  bool split = false;
  if constexpr (sizeof(T) == 4)
    split = l_rrb && c.nrp > 0 && c.g->natom > 0 && hpsi_f32_fast_ok(c.g, M);
  if (l_rrb) {
    if (split)
      rc = launch_hpsi_f32_fast(c.g, (const float*)c.veff, c.dij, c.rp, (const float*)c.psi,
                                (float*)c.hpsi, M, c.st, true);
    else
      rc = c.apply_h(c.psi, c.rp, c.hpsi, M);
    if (rc) return rc;
  }
  double *A = nullptr, *w = nullptr, *Z = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&A, sizeof(double) * ((size_t)2 * M * M + M), c.st));
  Z = A + (size_t)M * M;
  w = Z + (size_t)M * M;
  const double dv = c.dx * c.dy * c.dz;
  if constexpr (sizeof(T) == 4) {
    rc = gram_f32(M, M, c.N, (const float*)c.psi, c.N, (const float*)c.hpsi, c.N, dv, A, M, 2,
                  c.st);  // lower tile pairs: dsyev('v','l') reads the lower triangle
    if (!rc && split) {
      double* Td = nullptr;
      cudaError_t e = cudaMallocAsync((void**)&Td, sizeof(double) * (size_t)c.nrp * M, c.st);
      if (e != cudaSuccess) rc = cuda_status(e, "rayleighritz: D <p|psi>");
      if (!rc) {
        k_s_rp<<<div_up((long)c.nrp * M, 256), 256, 0, c.st>>>(M, c.g->natom, c.g->nprjmx,
                                                              c.g->d_nprj, c.dij, c.rp, Td);
        rc = gram_f64_beta(M, M, c.nrp, c.rp, c.nrp, Td, c.nrp, 1.0, 1.0, A, M, c.st);
      }
      if (Td) cudaFreeAsync(Td, c.st);
    }
  } else
    rc = gram_f64(M, M, c.N, (const double*)c.psi, c.N, (const double*)c.hpsi, c.N, dv, A, M, c.st);
  // dsyev('v','l') reads the lower triangle: mirror it
  if (!rc) {
    k_mirror_lower<<<div_up((long)M * M, 256), 256, 0, c.st>>>(M, A);
    rc = syev_jacobi(M, A, w, Z, 60, c.st, nullptr);
  }
  if (!rc) rc = c.rotate_all(Z);
  if (!rc) {
    RS_CUDA(cudaMemcpyAsync(sval_h, w, sizeof(double) * M, cudaMemcpyDeviceToHost, c.st));
    RS_CUDA(cudaStreamSynchronize(c.st));
  }
  cudaFreeAsync(A, c.st);
  return rc;
}

// reorderstates: stable ascending rank, permute psi, spsi, rp, sval, resid
template <class T>
static int reorder(BandCtx<T>& c, double* sval_h, double* resid_h) {
  const int M = c.M;
  const long N = c.g->N;
  const int nrp = c.g->natom * c.g->nprjmx;
  std::vector<int> rank(M, 0);
  for (int j = 1; j < M; ++j)
    for (int i = 0; i < j; ++i) {
      if (sval_h[i] > sval_h[j]) rank[i] += 1;
      else rank[j] += 1;
    }
  std::vector<double> t(M);
  for (int j = 0; j < M; ++j) t[rank[j]] = sval_h[j];
  std::copy(t.begin(), t.end(), sval_h);
  for (int j = 0; j < M; ++j) t[rank[j]] = resid_h[j];
  std::copy(t.begin(), t.end(), resid_h);
  // only the bands whose position changes move: they form a permutation of
  // their own, so gathering them into a buffer and scattering them to their
  // ranks reorders the arrays (nothing moves when the order already holds)
  std::vector<int> mv;  // [from..., to...]
  for (int j = 0; j < M; ++j)
    if (rank[j] != j) mv.push_back(j);
  const int K = (int)mv.size();
  if (K == 0) return RS_OK;
  for (int k = 0; k < K; ++k) mv.push_back(rank[mv[k]]);
  std::vector<int> seq(K);
  for (int k = 0; k < K; ++k) seq[k] = k;
  int* dmv = nullptr;
  void* tmp = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&dmv, sizeof(int) * 3 * K, c.st));
  RS_CUDA(cudaMallocAsync(&tmp, std::max(sizeof(T) * (size_t)N, sizeof(double) * nrp) * K, c.st));
  mv.insert(mv.end(), seq.begin(), seq.end());  // [from | to | 0..K-1]
  RS_CUDA(cudaMemcpyAsync(dmv, mv.data(), sizeof(int) * 3 * K, cudaMemcpyHostToDevice, c.st));
  const int* from = dmv;
  const int* to = dmv + K;
  const int* slot = dmv + 2 * K;
  // gather the moving bands into tmp, then scatter them to their ranks, in
  // launches of at most 65535 bands
  auto move = [&](auto* a, long n, bool vec) {
    using U = std::remove_pointer_t<decltype(a)>;
    constexpr int V = 16 / (int)sizeof(U);
    U* b = (U*)tmp;
    for (int k0 = 0; k0 < K; k0 += 65535) {
      const int kc = std::min(65535, K - k0);
      if (vec) {
        const dim3 grid(div_up(n / V, 256), kc);
        k_move_bands<U, V><<<grid, 256, 0, c.st>>>(n, from + k0, a, slot + k0, b);
      } else {
        const dim3 grid(div_up(n, 256), kc);
        k_move_bands<U, 1><<<grid, 256, 0, c.st>>>(n, from + k0, a, slot + k0, b);
      }
    }
    for (int k0 = 0; k0 < K; k0 += 65535) {
      const int kc = std::min(65535, K - k0);
      if (vec) {
        const dim3 grid(div_up(n / V, 256), kc);
        k_move_bands<U, V><<<grid, 256, 0, c.st>>>(n, slot + k0, b, to + k0, a);
      } else {
        const dim3 grid(div_up(n, 256), kc);
        k_move_bands<U, 1><<<grid, 256, 0, c.st>>>(n, slot + k0, b, to + k0, a);
      }
    }
  };
  T* arrs[2] = {c.psi, c.sep() ? c.spsi : nullptr};
  for (T* a : arrs)
    if (a) move(a, N, N % (16 / (long)sizeof(T)) == 0 && (uintptr_t)a % 16 == 0);
  if (nrp) move(c.rp, (long)nrp, false);
  cudaFreeAsync(dmv, c.st);
  cudaFreeAsync(tmp, c.st);
  cudaError_t e = cudaStreamSynchronize(c.st);
  if (e != cudaSuccess) return cuda_status(e, "reorderstates");
  return RS_OK;
}

template <class T>
static BandCtx<T> make_ctx(const rs_geom* g, const T* veff, const double* dij, const double* sss,
                           int M, T* psi, T* spsi, double* rp, T* hpsi, void* stream) {
  BandCtx<T> c;
  c.g = g; c.veff = veff; c.dij = dij; c.sss = sss; c.M = M;
  c.psi = psi; c.spsi = sss ? spsi : psi; c.rp = rp; c.hpsi = hpsi;
  c.st = as_stream(stream);
  c.N = g->N;
  c.nrp = g->natom * g->nprjmx;
  c.dx = g->dx; c.dy = g->dy; c.dz = g->dz;
  return c;
}

}  // namespace rs

#define RS_BANDS_CHECK(fn)                                                    \
  if (!g) return rs::fail(RS_EINVAL, fn ": null geometry");                  \
  if (M <= 0) return rs::fail(RS_EINVAL, fn ": no bands");                   \
  if (sss && (!spsi || spsi == psi)) return rs::fail(RS_EINVAL, fn ": S psi must be its own array")

#define RS_BANDS_IMPL(SUF, T)                                                                  \
  extern "C" int rs_orthogonalize_##SUF(const rs_geom* g, const double* sss, int M, T* psi,     \
                                        T* spsi, double* rp, int cmpt, void* stream) {          \
    RS_BANDS_CHECK("rs_orthogonalize_" #SUF);                                                  \
    auto c = rs::make_ctx<T>(g, nullptr, nullptr, sss, M, psi, spsi, rp, nullptr, stream);      \
    int rc = c.init(0, 0);                                                                     \
    if (!rc) rc = c.ortho_all(cmpt != 0);                                                       \
    c.release();                                                                               \
    return rc;                                                                                 \
  }                                                                                            \
  extern "C" int rs_orthogonalize_band_##SUF(const rs_geom* g, const double* sss, int M, int l, \
                                             T* psi, T* spsi, double* rp, int cmpt,             \
                                             void* stream) {                                    \
    RS_BANDS_CHECK("rs_orthogonalize_band_" #SUF);                                             \
    if (l < 0 || l >= M) return rs::fail(RS_EINVAL, "rs_orthogonalize_band: band out of range"); \
    auto c = rs::make_ctx<T>(g, nullptr, nullptr, sss, M, psi, spsi, rp, nullptr, stream);      \
    int rc = c.init(0, 0);                                                                     \
    if (!rc) rc = c.ortho_band(l, cmpt != 0);                                                   \
    if (!rc) rc = c.check_status();                                                            \
    c.release();                                                                               \
    return rc;                                                                                 \
  }                                                                                            \
  extern "C" int rs_rayleighritz_##SUF(const rs_geom* g, const T* veff, const double* dij,      \
                                       const double* sss, int M, T* psi, T* spsi, double* rp,   \
                                       T* hpsi, int l_rrb, double* sval, void* stream) {        \
    RS_BANDS_CHECK("rs_rayleighritz_" #SUF);                                                   \
    auto c = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);                \
    return rs::rayleighritz<T>(c, l_rrb, sval);                                                 \
  }                                                                                            \
  extern "C" int rs_kscg_##SUF(const rs_geom* g, const T* veff, const double* dij,              \
                               const double* sss, const rs_solver_prm* prm, int M, T* psi,      \
                               T* spsi, double* rp, T* hpsi, double* sval, double* resid,       \
                               int* itmax, void* stream) {                                      \
    RS_BANDS_CHECK("rs_kscg_" #SUF);                                                           \
    auto c = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);                \
    return rs::kscg<T>(c, prm, sval, resid, itmax);                                             \
  }                                                                                            \
  extern "C" int rs_ksdiis_##SUF(const rs_geom* g, const T* veff, const double* dij,            \
                                 const double* sss, const rs_solver_prm* prm, int M, int l_hsv, \
                                 T* psi, T* spsi, double* rp, T* hpsi, double* sval,            \
                                 double* resid, int* ksconv, void* stream) {                    \
    RS_BANDS_CHECK("rs_ksdiis_" #SUF);                                                         \
    auto c = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);                \
    return rs::ksdiis<T>(c, prm, l_hsv, sval, resid, ksconv);                                   \
  }                                                                                            \
  extern "C" int rs_reorder_##SUF(const rs_geom* g, const double* sss, int M, T* psi, T* spsi,  \
                                  double* rp, double* sval, double* resid, void* stream) {      \
    RS_BANDS_CHECK("rs_reorder_" #SUF);                                                        \
    auto c = rs::make_ctx<T>(g, nullptr, nullptr, sss, M, psi, spsi, rp, nullptr, stream);      \
    return rs::reorder<T>(c, sval, resid);                                                      \
  }                                                                                            \
  extern "C" int rs_scf_diag_##SUF(const rs_geom* g, const T* veff, const double* dij,          \
                                   const double* sss, const rs_solver_prm* prm, int iscf,       \
                                   int M, T* psi, T* spsi, double* rp, T* hpsi, double* sval,   \
                                   double* resid, int* ksconv, int* ksitmax, void* stream) {    \
    RS_BANDS_CHECK("rs_scf_diag_" #SUF);                                                       \
    auto c = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);                \
    const int nrrz = prm->nrrz, nchange = prm->nchange;                                         \
    bool l_rrb = false, l_rra = false, l_hsv = false, l_reo = false;                            \
    if (nrrz != 0) {                                                                           \
      l_rrb = (iscf % abs(nrrz) == 0) && nrrz > 0;                                             \
      l_rra = (iscf % abs(nrrz) == 0) && nrrz < 0;                                             \
      l_hsv = l_rra || ((iscf + 1) % nrrz == 0 && nrrz > 0);                                   \
    }                                                                                          \
    if (nchange > 0) l_reo = (iscf % nchange == 0) && !l_rra;                                  \
    int rc = RS_OK;                                                                            \
    *ksconv = 1;                                                                               \
    *ksitmax = 0;                                                                              \
    if (l_rrb) rc = rs::rayleighritz<T>(c, 1, sval);                                           \
    if (!rc) {                                                                                 \
      if (iscf <= prm->ncgscf || (prm->nretcg > 0 && iscf % prm->nretcg == 0)) {               \
        auto c2 = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);           \
        rc = rs::kscg<T>(c2, prm, sval, resid, ksitmax);                                       \
        for (int l = 0; l < M && !rc; ++l)                                                     \
          *ksconv = *ksconv && (sqrt(resid[l]) < prm->epssd || *ksitmax < prm->nsdmax);        \
      } else {                                                                                 \
        auto c2 = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);           \
        rc = rs::ksdiis<T>(c2, prm, l_hsv ? 1 : 0, sval, resid, ksconv);                       \
        *ksitmax = 1;                                                                          \
      }                                                                                        \
    }                                                                                          \
    if (!rc && l_rra) {                                                                        \
      auto c3 = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);             \
      rc = rs::rayleighritz<T>(c3, 1, sval);                                                   \
    }                                                                                          \
    if (!rc && l_reo) {                                                                        \
      auto c4 = rs::make_ctx<T>(g, veff, dij, sss, M, psi, spsi, rp, hpsi, stream);             \
      rc = rs::reorder<T>(c4, sval, resid);                                                    \
    }                                                                                          \
    return rc;                                                                                 \
  }

RS_BANDS_IMPL(f64, double)
RS_BANDS_IMPL(f32, float)
