/*
 * rs_oracle_solvers.c -- CPU FP64 restatement of kukan's band solvers:
 * block Gram-Schmidt in the S metric, Rayleigh-Ritz, band-by-band CG,
 * RMM-DIIS, state reordering and the nonlocal force.  TEST INFRASTRUCTURE
 * (see rs_oracle.c).  Dense products use orc_tree_dot per matrix element;
 * the BLAS calls of the reference have no defined summation order, so parity
 * on these routines is checked within a tolerance, not bit for bit.
 */
#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#include "rs_oracle.h"

#define DV(s) ((s)->dx * (s)->dy * (s)->dz)

void orc_apply_h(const orc_sys* s, const double* psi, const double* rp, double* hpsi, int nb) {
  orc_hpsi(s->nx, s->ny, s->nz, s->nf, s->dx, s->dy, s->dz, s->veff, s->natom, s->nprjmx,
           s->num_list, s->nprj, s->natinf, s->lst, s->v, s->dij, rp, psi, hpsi, nb);
}

void orc_apply_s(const orc_sys* s, const double* psi, const double* rp, double* spsi, int nb) {
  if (!s->sss) {
    memcpy(spsi, psi, sizeof(double) * s->N * nb);
    return;
  }
  orc_spsi(s->N, s->natom, s->nprjmx, s->num_list, s->nprj, s->natinf, s->lst, s->v, s->sss,
           DV(s), rp, psi, spsi, nb);
}

static void nl_dot(const orc_sys* s, const double* psi, double* rp, int nb) {
  orc_nl_dot(s->natom, s->nprjmx, s->num_list, s->nprj, s->natinf, s->lst, s->v, psi, s->N,
             nb, rp);
}

/* x -= sum_{j<cnt} c[j] * y_j   (orthogonalization_r_03 / multr order) */
static void sub_comb(long n, double* x, const double* y, long ystride, const double* c,
                     int cnt) {
  for (int j = 0; j < cnt; ++j) {
    const double* yj = y + (long)j * ystride;
    for (long i = 0; i < n; ++i) x[i] = fma(-c[j], yj[i], x[i]);
  }
}

static void normalize_band(const orc_sys* s, double* psi, double* spsi, double* rp,
                           int nrp) {
  double vecnor = orc_tree_dot(s->N, psi, spsi) * s->dx * s->dy * s->dz;
  const double tmp = 1.0 / sqrt(vecnor);
  for (long i = 0; i < s->N; ++i) psi[i] = psi[i] * tmp;
  if (spsi != psi)
    for (long i = 0; i < s->N; ++i) spsi[i] = spsi[i] * tmp;
  for (int i = 0; i < nrp; ++i) rp[i] = rp[i] * tmp;
}

/* orthogonalization_r_01 (orthogonalization8f.F90:93-376).  l_inp = 0 works on
 * all bands, l_inp = l (1-based) on band l alone; cmpt recomputes <p|psi> and
 * S psi first (key_ortho_cmpt_innerproduct).  spsi may alias psi when S = 1. */
void orc_ortho(const orc_sys* s, int M, int l_inp, int cmpt, double* psi, double* spsi,
               double* rp) {
  const long N = s->N;
  const int nrp = s->natom * s->nprjmx;
  int mstep = 32;
  if (M > 1024) mstep = 64;
  if (M > 2048) mstep = 128;
  if (M > 4096) mstep = 256;
  const int l_stt = l_inp == 0 ? 1 : l_inp, l_end = l_inp == 0 ? M : l_inp;
  if (cmpt) {
    for (int l = l_stt; l <= l_end; ++l) {
      nl_dot(s, psi + (long)(l - 1) * N, rp + (long)(l - 1) * nrp, 1);
      if (spsi != psi) orc_apply_s(s, psi + (long)(l - 1) * N, rp + (long)(l - 1) * nrp,
                                   spsi + (long)(l - 1) * N, 1);
    }
  }
  double* av = (double*)malloc(sizeof(double) * (M + 1));
  double* am = (double*)malloc(sizeof(double) * mstep * mstep);
  int l = l_stt;
  while (l < l_end + 1) {
    if (l > mstep && l_end - l + 1 >= mstep) {
      for (int j = 1; j <= l - 1; j += mstep) {
        /* amatr(a,b) = <psi_{l+a} | S psi_{j+b}> dV  (dgemm 't','n') */
        for (int b = 0; b < mstep; ++b)
          for (int a = 0; a < mstep; ++a)
            am[b * mstep + a] =
                orc_tree_dot(N, psi + (long)(l - 1 + a) * N, spsi + (long)(j - 1 + b) * N) *
                s->dx * s->dy * s->dz;
        /* psi_{l+a} -= sum_b psi_{j+b} amatr(a,b)  (dgemm 'n','t', alpha=1, -amatr) */
        for (int a = 0; a < mstep; ++a) {
          double c[256];
          for (int b = 0; b < mstep; ++b) c[b] = am[b * mstep + a];
          sub_comb(N, psi + (long)(l - 1 + a) * N, psi + (long)(j - 1) * N, N, c, mstep);
          if (spsi != psi)
            sub_comb(N, spsi + (long)(l - 1 + a) * N, spsi + (long)(j - 1) * N, N, c, mstep);
          sub_comb(nrp, rp + (long)(l - 1 + a) * nrp, rp + (long)(j - 1) * nrp, nrp, c, mstep);
        }
      }
      normalize_band(s, psi + (long)(l - 1) * N, spsi + (long)(l - 1) * N,
                     rp + (long)(l - 1) * nrp, nrp);
      for (int l0 = l + 1; l0 <= l + mstep - 1; ++l0) {
        for (int j = l; j <= l0 - 1; ++j)
          av[j - l] = orc_tree_dot(N, spsi + (long)(j - 1) * N, psi + (long)(l0 - 1) * N) *
                      s->dx * s->dy * s->dz;
        sub_comb(N, psi + (long)(l0 - 1) * N, psi + (long)(l - 1) * N, N, av, l0 - l);
        if (spsi != psi)
          sub_comb(N, spsi + (long)(l0 - 1) * N, spsi + (long)(l - 1) * N, N, av, l0 - l);
        sub_comb(nrp, rp + (long)(l0 - 1) * nrp, rp + (long)(l - 1) * nrp, nrp, av, l0 - l);
        normalize_band(s, psi + (long)(l0 - 1) * N, spsi + (long)(l0 - 1) * N,
                       rp + (long)(l0 - 1) * nrp, nrp);
      }
      l += mstep;
    } else {
      for (int j = 1; j <= l - 1; ++j)
        av[j - 1] = orc_tree_dot(N, spsi + (long)(j - 1) * N, psi + (long)(l - 1) * N) *
                    s->dx * s->dy * s->dz;
      sub_comb(N, psi + (long)(l - 1) * N, psi, N, av, l - 1);
      if (spsi != psi) sub_comb(N, spsi + (long)(l - 1) * N, spsi, N, av, l - 1);
      sub_comb(nrp, rp + (long)(l - 1) * nrp, rp, nrp, av, l - 1);
      normalize_band(s, psi + (long)(l - 1) * N, spsi + (long)(l - 1) * N,
                     rp + (long)(l - 1) * nrp, nrp);
      l += 1;
    }
  }
  free(av);
  free(am);
}

/* rayleighritz_r (rayleigh-ritz8f.F90:22-125): A = dV Psi^T H Psi, eigen
 * (lower triangle), Psi <- Psi Z, S Psi <- S Psi Z, <p|Psi> <- <p|Psi> Z.
 * hpsi is work space on exit, as in the reference. */
int orc_rayleighritz(const orc_sys* s, int M, int l_rrb, double* psi, double* spsi,
                     double* rp, double* hpsi, double* sval) {
  const long N = s->N;
  const int nrp = s->natom * s->nprjmx;
  if (l_rrb) orc_apply_h(s, psi, rp, hpsi, M);
  double* a = (double*)malloc(sizeof(double) * M * M);
  double* z = (double*)malloc(sizeof(double) * M * M);
  for (int j = 0; j < M; ++j)
    for (int i = j; i < M; ++i) {
      const double v = s->dx * s->dy * s->dz * orc_tree_dot(N, psi + (long)i * N,
                                                            hpsi + (long)j * N);
      a[i * M + j] = v; /* lower triangle as dsyev('v','l') reads it */
      a[j * M + i] = v;
    }
  const int st = orc_jacobi_eig(M, a, sval, z);
  double* out = (double*)malloc(sizeof(double) * (N > nrp ? N : nrp) * M);
  for (int pass = 0; pass < (spsi != psi ? 3 : 2); ++pass) {
    double* x = pass == 0 ? psi : (pass == 1 ? rp : spsi);
    const long n = pass == 1 ? nrp : N;
    for (int k = 0; k < M; ++k) {
      double* o = out + (long)k * n;
      for (long i = 0; i < n; ++i) o[i] = 0.0;
      for (int j = 0; j < M; ++j) {
        const double c = z[j * M + k];
        const double* xj = x + (long)j * n;
        for (long i = 0; i < n; ++i) o[i] = fma(xj[i], c, o[i]);
      }
    }
    memcpy(x, out, sizeof(double) * n * M);
  }
  free(out);
  free(a);
  free(z);
  return st < 0 ? -1 : 0;
}

/* kscg_r (kscg8f.F90:7-489) with helpers kscg_r_01.._05 (:1035-1230),
 * nkscg=1.  Returns 0; *itmax = max CG iterations over bands. */
int orc_kscg(const orc_sys* s, const orc_solver_prm* prm, int M, double* psi, double* spsi,
             double* rp, double* hpsi, double* sval, double* resid, int* itmax) {
  const long N = s->N;
  const int nrp = s->natom * s->nprjmx;
  const int nsdmax1 = 10, nsdmax2 = 200;
  double* rvec = (double*)calloc(N, sizeof(double));
  double* pvec = (double*)calloc(N, sizeof(double));
  double* pv = (double*)calloc(N, sizeof(double));
  double* rv = (double*)calloc(N, sizeof(double));
  double* spv = (double*)calloc(N, sizeof(double));
  double* asv = (double*)calloc(N, sizeof(double));
  double* av = (double*)calloc(N, sizeof(double));
  double* rrp = (double*)calloc(nrp, sizeof(double));
  double* rpp = (double*)calloc(nrp, sizeof(double));
  double* rpl = (double*)calloc(nrp, sizeof(double));
  double* coef = (double*)calloc(M + 1, sizeof(double));
  int itm = 0;
  for (int l = 1; l <= M; ++l) {
    double* psl = psi + (long)(l - 1) * N;
    double* ssl = spsi + (long)(l - 1) * N;
    double* hsl = hpsi + (long)(l - 1) * N;
    double* rpsl = rp + (long)(l - 1) * nrp;
    for (int loop = 0; loop < prm->northo; ++loop)
      orc_ortho(s, M, l, prm->northo == 2, psi, spsi, rp);
    orc_apply_h(s, psl, rpsl, hsl, 1);
    int iiter = 0, conv = 0;
    double r2rr = 1.0, r1rr;
    while (iiter < prm->nsdmax && !conv) {
      ++iiter;
      int reset = (iiter == 1) || (iiter == nsdmax1);
      if (nsdmax2 > 0) reset = reset || ((iiter - 1) % nsdmax2 == 0);
      if (reset) {
        r2rr = 1.0;
        memset(pvec, 0, sizeof(double) * N);
        memset(rvec, 0, sizeof(double) * N);
        memset(pv, 0, sizeof(double) * N);
        memset(spv, 0, sizeof(double) * N);
        memset(rpp, 0, sizeof(double) * nrp);
      }
      r1rr = r2rr;
      const double valre = orc_tree_dot(N, psl, hsl) * s->dx * s->dy * s->dz;
      sval[l - 1] = valre;
      for (long i = 0; i < N; ++i) rvec[i] = -fma(-valre, ssl[i], hsl[i]);
      if (prm->nprecon) orc_precondition(s->nx, s->ny, s->nz, rvec, rv, 1);
      else memcpy(rv, rvec, sizeof(double) * N);
      for (int loop = 0; loop < prm->northo; ++loop) {
        for (int j = 1; j <= l; ++j)
          coef[j - 1] = orc_tree_dot(N, spsi + (long)(j - 1) * N, rv) * s->dx * s->dy * s->dz;
        sub_comb(N, rv, psi, N, coef, l);
      }
      nl_dot(s, rv, rrp, 1);
      orc_apply_s(s, rv, rrp, asv, 1);
      r2rr = orc_tree_dot(N, rv, rvec) * s->dx * s->dy * s->dz;
      resid[l - 1] = r2rr;
      /* kscg_r_03 */
      const double ratio = r2rr / r1rr;
      for (long i = 0; i < N; ++i) {
        pv[i] = fma(ratio, pv[i], rv[i]);
        pvec[i] = pv[i];
        spv[i] = fma(ratio, spv[i], asv[i]);
      }
      for (int i = 0; i < nrp; ++i) rpp[i] = fma(ratio, rpp[i], rrp[i]);
      memcpy(rpl, rpp, sizeof(double) * nrp);
      memcpy(asv, spv, sizeof(double) * N);
      for (int loop = 0; loop < prm->northo; ++loop) {
        for (int j = 1; j <= l; ++j)
          coef[j - 1] = orc_tree_dot(N, spsi + (long)(j - 1) * N, pvec) * s->dx * s->dy * s->dz;
        sub_comb(N, pvec, psi, N, coef, l);
        sub_comb(N, asv, spsi, N, coef, l);
        sub_comb(nrp, rpl, rp, nrp, coef, l);
      }
      const double vecnor = orc_tree_dot(N, pvec, asv) * s->dx * s->dy * s->dz;
      if (!(vecnor > 0.0)) return -2; /* 'kscg_r: pvec has negative norm' */
      const double tmp = 1.0 / sqrt(vecnor);
      for (long i = 0; i < N; ++i) {
        pvec[i] = pvec[i] * tmp;
        asv[i] = asv[i] * tmp;
      }
      for (int i = 0; i < nrp; ++i) rpl[i] = rpl[i] * tmp;
      orc_apply_h(s, pvec, rpl, av, 1);
      const double pap = orc_tree_dot(N, pvec, av) * s->dx * s->dy * s->dz;
      const double sapre = orc_tree_dot(N, psl, av) * s->dx * s->dy * s->dz;
      /* kscg_r_05 */
      const double sv = sval[l - 1], eps = 1.0e-14;
      double alph = 1.0, beta = 0.0;
      const double gamma = (sv + pap) * 0.5 - sqrt((sv - pap) * (sv - pap) * 0.25 + sapre * sapre);
      if (fabs((sv - gamma) / gamma) > eps) {
        const double den = sqrt(sapre * sapre + (sv - gamma) * (sv - gamma));
        alph = sapre / den;
        beta = -(sv - gamma) / den;
      }
      if (alph < eps) { alph = -alph; beta = -beta; }
      for (long i = 0; i < N; ++i) {
        psl[i] = fma(beta, pvec[i], alph * psl[i]);
        hsl[i] = fma(beta, av[i], alph * hsl[i]);
        if (ssl != psl) ssl[i] = fma(beta, asv[i], alph * ssl[i]);
      }
      for (int i = 0; i < nrp; ++i) rpsl[i] = fma(beta, rpl[i], alph * rpsl[i]);
      conv = sqrt(resid[l - 1]) < prm->epssd;
    }
    if (iiter > itm) itm = iiter;
  }
  if (itmax) *itmax = itm;
  free(rvec); free(pvec); free(pv); free(rv); free(spv); free(asv); free(av);
  free(rrp); free(rpp); free(rpl); free(coef);
  return 0;
}

/* ksdiis_r (ksdiis8f.F90:8-712) with nitermax=2 (one trial step per band per
 * sweep) and helpers ksdiis_r_01/_03 (:1512-1570). */
int orc_ksdiis(const orc_sys* s, const orc_solver_prm* prm, int M, int l_hsv, double* psi,
               double* spsi, double* rp, double* hpsi, double* sval, double* resid) {
  const long N = s->N;
  const int nrp = s->natom * s->nprjmx;
  const int sep = spsi != psi;
  double* ph[2]; double* sph[2]; double* hph[2]; double* rv[2]; double* rph[2];
  for (int k = 0; k < 2; ++k) {
    ph[k] = (double*)malloc(sizeof(double) * N);
    sph[k] = sep ? (double*)malloc(sizeof(double) * N) : ph[k];
    hph[k] = (double*)malloc(sizeof(double) * N);
    rv[k] = (double*)malloc(sizeof(double) * N);
    rph[k] = (double*)malloc(sizeof(double) * nrp);
  }
  double* rvre = (double*)malloc(sizeof(double) * N);
  double* avre = (double*)malloc(sizeof(double) * N);
  double* asvre = (double*)malloc(sizeof(double) * N);
  double* rpsep = (double*)malloc(sizeof(double) * nrp);
  int ksconv = 1;
  for (int jiter = 1; jiter + 1 <= prm->ndiismax; ++jiter) {
    for (int l = 0; l < M; ++l) {
      memcpy(ph[0], psi + (long)l * N, sizeof(double) * N);
      if (sep) memcpy(sph[0], spsi + (long)l * N, sizeof(double) * N);
      memcpy(rph[0], rp + (long)l * nrp, sizeof(double) * nrp);
      /* iiter = 1 */
      orc_apply_h(s, ph[0], rph[0], hph[0], 1);
      double valre = orc_tree_dot(N, ph[0], hph[0]) * s->dx * s->dy * s->dz;
      sval[l] = valre;
      for (long i = 0; i < N; ++i) rv[0][i] = fma(-valre, sph[0][i], hph[0][i]);
      if (prm->nprecon) orc_precondition(s->nx, s->ny, s->nz, rv[0], rvre, 1);
      else memcpy(rvre, rv[0], sizeof(double) * N);
      nl_dot(s, rvre, rpsep, 1);
      orc_apply_h(s, rvre, rpsep, avre, 1);
      orc_apply_s(s, rvre, rpsep, asvre, 1);
      /* lambda line search */
      const double a1 = prm->alambda_diis;
      for (int i = 0; i < nrp; ++i) rph[1][i] = fma(a1, rpsep[i], rph[0][i]);
      for (long i = 0; i < N; ++i) {
        ph[1][i] = fma(a1, rvre[i], ph[0][i]);
        hph[1][i] = fma(a1, avre[i], hph[0][i]);
        if (sep) sph[1][i] = fma(a1, asvre[i], sph[0][i]);
      }
      const double s1 = orc_tree_dot(N, rvre, hph[0]);
      const double s2 = orc_tree_dot(N, rvre, sph[0]);
      const double s3 = orc_tree_dot(N, ph[1], hph[1]);
      const double s4 = orc_tree_dot(N, ph[1], sph[1]);
      const double aaa = 2.0 * fma(-sval[l], s2, s1) * s->dx * s->dy * s->dz;
      valre = s3 / s4;
      const double bbb = fma(-aaa, a1, valre - sval[l]) / (a1 * a1);
      double alambda = 0.5 * aaa / bbb;
      if (alambda > prm->alambda_max) alambda = prm->alambda_max;
      if (alambda < prm->alambda_min) alambda = prm->alambda_min;
      for (long i = 0; i < N; ++i) {
        ph[1][i] = fma(alambda, rvre[i], ph[0][i]);
        hph[1][i] = fma(alambda, avre[i], hph[0][i]);
        if (sep) sph[1][i] = fma(alambda, asvre[i], sph[0][i]);
      }
      for (int i = 0; i < nrp; ++i) rph[1][i] = fma(alambda, rpsep[i], rph[0][i]);
      for (int j = 0; j < 2; ++j)
        for (long i = 0; i < N; ++i) rv[j][i] = fma(-sval[l], sph[j][i], hph[j][i]);
      /* 2x2 S and R matrices, rsmat(i,j) = <phi_i|S phi_j>, rrmat = <R_i|R_j> */
      double rs[4], rr[4];
      for (int j = 0; j < 2; ++j)
        for (int i = 0; i <= j; ++i) {
          const double sv_ = orc_tree_dot(N, ph[i], sph[j]) * s->dx * s->dy * s->dz;
          const double rv_ = orc_tree_dot(N, rv[i], rv[j]) * s->dx * s->dy * s->dz;
          rs[i * 2 + j] = rs[j * 2 + i] = sv_;
          rr[i * 2 + j] = rr[j * 2 + i] = rv_;
        }
      const double tmp = 1.0 / sqrt(rs[3]);
      for (long i = 0; i < N; ++i) {
        ph[1][i] = ph[1][i] * tmp;
        hph[1][i] = hph[1][i] * tmp;
        if (sep) sph[1][i] = sph[1][i] * tmp;
        rv[1][i] = rv[1][i] * tmp;
      }
      for (int i = 0; i < nrp; ++i) rph[1][i] = rph[1][i] * tmp;
      for (int i = 0; i < 2; ++i) { rs[1 * 2 + i] *= tmp; rr[1 * 2 + i] *= tmp; }
      for (int i = 0; i < 2; ++i) { rs[i * 2 + 1] *= tmp; rr[i * 2 + 1] *= tmp; }
      double rs0[4];
      memcpy(rs0, rs, sizeof rs);
      double w[2], z[4], eig[2], vec[4];
      orc_eig2(rs, w, z);
      /* descending order: column k of vec is eigenvector of eig[k] */
      for (int k = 0; k < 2; ++k) {
        eig[k] = w[1 - k];
        vec[0 * 2 + k] = z[0 * 2 + (1 - k)];
        vec[1 * 2 + k] = z[1 * 2 + (1 - k)];
      }
      int nmat = 0, k = 0;
      while (k < 2) {
        ++nmat; ++k;
        /* with one trial vector the reference's column shift
           (ksdiis8f.F90:448-452) is an empty loop: only nmat drops */
        if (eig[nmat - 1] < prm->eps_eig_diis) --nmat;
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
        orc_eig2(r2, w2, z2);
        for (int kk = 0; kk < 2; ++kk) {
          v2[0 * 2 + kk] = z2[0 * 2 + (1 - kk)];
          v2[1 * 2 + kk] = z2[1 * 2 + (1 - kk)];
        }
        resid[l] = w2[0]; /* eigen(nmat) after the descending reorder */
        for (int j = 0; j < 2; ++j) {
          double acc = 0.0;
          for (int i = 0; i < 2; ++i) acc = fma(vec[j * 2 + i], v2[i * 2 + 1], acc);
          c[j] = acc;
        }
        double nrm = 0.0;
        for (int j = 0; j < 2; ++j)
          for (int i = 0; i < 2; ++i) nrm = fma(c[i] * rs0[i * 2 + j], c[j], nrm);
        const double sq = sqrt(nrm);
        c[0] /= sq; c[1] /= sq;
      } else {
        c[0] = 0.0; c[1] = 1.0;
      }
      /* ksdiis_r_03 combination */
      for (long i = 0; i < N; ++i) {
        avre[i] = fma(c[1], ph[1][i], c[0] * ph[0][i]);
        asvre[i] = fma(c[1], sph[1][i], c[0] * sph[0][i]);
        rvre[i] = fma(c[1], hph[1][i], c[0] * hph[0][i]);
      }
      for (int i = 0; i < nrp; ++i) {
        double acc = 0.0;
        acc = fma(c[0], rph[0][i], acc);
        acc = fma(c[1], rph[1][i], acc);
        rp[(long)l * nrp + i] = acc;
      }
      memcpy(psi + (long)l * N, avre, sizeof(double) * N);
      if (sep) memcpy(spsi + (long)l * N, asvre, sizeof(double) * N);
      memcpy(hpsi + (long)l * N, rvre, sizeof(double) * N);
      ksconv = ksconv && (sqrt(resid[l]) <= prm->epssd);
    }
  }
  if (l_hsv) {
    for (int i = 0; i < prm->northo; ++i) orc_ortho(s, M, 0, 1, psi, spsi, rp);
    orc_apply_h(s, psi, rp, hpsi, M);
  }
  for (int k = 0; k < 2; ++k) {
    free(ph[k]);
    if (sep) free(sph[k]);
    free(hph[k]); free(rv[k]); free(rph[k]);
  }
  free(rvre); free(avre); free(asvre); free(rpsep);
  return ksconv;
}

/* reorderstates (reorderstates8f.F90:8-124), real branch: stable ascending
 * permutation of sval, residuals, psi, S psi and <p|psi>; work holds N*M. */
void orc_reorder(long N, int M, int nrp, double* sval, double* resid, double* psi,
                 double* spsi, double* rp, double* work) {
  int* rank = (int*)malloc(sizeof(int) * M);
  orc_reorder_rank(M, sval, rank);
  double* t = (double*)malloc(sizeof(double) * M);
  for (int j = 0; j < M; ++j) t[rank[j]] = sval[j];
  memcpy(sval, t, sizeof(double) * M);
  for (int j = 0; j < M; ++j) t[rank[j]] = resid[j];
  memcpy(resid, t, sizeof(double) * M);
  for (int pass = 0; pass < 3; ++pass) {
    double* x = pass == 0 ? psi : (pass == 1 ? spsi : rp);
    const long n = pass == 2 ? nrp : N;
    if (pass == 1 && spsi == psi) continue;
    for (int j = 0; j < M; ++j) memcpy(work + (long)rank[j] * n, x + (long)j * n, sizeof(double) * n);
    memcpy(x, work, sizeof(double) * n * M);
  }
  free(t);
  free(rank);
}

/* force_eig_r (force8f.F90:9-195): F_a = -2 sum_l f_l sum_ij <p_i|psi_l>
 * (D_ij - eps_l S_ij) <p_j|d psi_l>.  S = 0 in the sum when sss is NULL. */
void orc_force_nl(const orc_sys* s, int M, const double* psi, const double* sval,
                  const double* occ, double* fx, double* fy, double* fz) {
  const long N = s->N;
  const int P = s->nprjmx, A = s->natom;
  double* rp = (double*)malloc(sizeof(double) * A * P * M);
  double* rdp = (double*)malloc(sizeof(double) * A * P);
  double* g = (double*)malloc(sizeof(double) * N);
  for (int a = 0; a < A; ++a) fx[a] = fy[a] = fz[a] = 0.0;
  nl_dot(s, psi, rp, M);
  const double hs[3] = {s->dx, s->dy, s->dz};
  for (int lmn = 0; lmn < 3; ++lmn) {
    double* f = lmn == 0 ? fx : (lmn == 1 ? fy : fz);
    for (int l = 0; l < M; ++l) {
      orc_gradient(s->nx, s->ny, s->nz, s->nf, hs[lmn], lmn, psi + (long)l * N, g);
      nl_dot(s, g, rdp, 1);
      for (int a = 0; a < A; ++a) {
        const int n = s->nprj[a];
        const double* r = rp + ((long)l * A + a) * P;
        const double* rd = rdp + (long)a * P;
        for (int j = 0; j < n; ++j)
          for (int i = 0; i < n; ++i) {
            double d = s->dij[((long)a * P + j) * P + i];
            if (s->sss) d = fma(-sval[l], s->sss[((long)a * P + j) * P + i], d);
            f[a] = fma(-(2.0 * occ[l] * (r[i] * rd[j])), d, f[a]);
          }
      }
    }
  }
  free(rp); free(rdp); free(g);
}

/* Timed CPU baseline: the same H*psi with bands split over POSIX threads
 * (per-point evaluation order unchanged). */
typedef struct {
  const orc_sys* s;
  const double* psi;
  const double* rp;
  double* hpsi;
  int b0, b1;
} hpsi_job;

static void* hpsi_worker(void* arg) {
  hpsi_job* j = (hpsi_job*)arg;
  const long N = j->s->N;
  const int nrp = j->s->natom * j->s->nprjmx;
  for (int b = j->b0; b < j->b1; ++b)
    orc_apply_h(j->s, j->psi + (long)b * N, j->rp + (long)b * nrp, j->hpsi + (long)b * N, 1);
  return NULL;
}

void orc_hpsi_fast(const orc_sys* s, const double* psi, const double* rp, double* hpsi,
                   int nb, int nthreads) {
  if (nthreads < 1) nthreads = 1;
  if (nthreads > nb) nthreads = nb;
  pthread_t th[256];
  hpsi_job jobs[256];
  if (nthreads > 256) nthreads = 256;
  for (int t = 0; t < nthreads; ++t) {
    jobs[t].s = s; jobs[t].psi = psi; jobs[t].rp = rp; jobs[t].hpsi = hpsi;
    jobs[t].b0 = (int)((long)nb * t / nthreads);
    jobs[t].b1 = (int)((long)nb * (t + 1) / nthreads);
    pthread_create(&th[t], NULL, hpsi_worker, &jobs[t]);
  }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
}
