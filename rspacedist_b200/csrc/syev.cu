// syev.cu -- FP64 dense kernels of the subspace step on the GPU:
//  * symmetric eigensolver (parallel cyclic Jacobi, round-robin pairing), the
//    replacement of dsyev / pdsyevd in rayleighritz_r
//    (rayleigh-ritz8f.F90:89; rayleigh-ritz8f_sclpck.F90:268);
//  * Cholesky factorisation and triangular inverse for Cholesky-QR, which
//    spans the same vectors in the same order as kukan's block Gram-Schmidt
//    (orthogonalization8f.F90:93-376).
#include <math.h>

#include <vector>

#include "reduce.cuh"
#include "rs_common.cuh"

namespace rs {
namespace {

// pairs of round r of the circle method over ne (even) players
__device__ __forceinline__ void rr_pair(int r, int t, int ne, int* p, int* q) {
  const int m = ne - 1;
  int a = (r + t) % m;
  int b = t == 0 ? m : (r - t + m) % m;
  *p = a < b ? a : b;
  *q = a < b ? b : a;
}

struct Rot {
  int p, q;
  double c, s;
};

// rotation angle zeroing a_pq (same formula as the CPU oracle's Jacobi)
__global__ void k_jac_params(const double* __restrict__ A, int n, int ne, int r,
                             Rot* __restrict__ rot) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= ne / 2) return;
  int p, q;
  rr_pair(r, t, ne, &p, &q);
  Rot o{p, q, 1.0, 0.0};
  if (q < n) {
    const double apq = A[(long)p * n + q];
    if (apq != 0.0) {
      const double app = A[(long)p * n + p], aqq = A[(long)q * n + q];
      const double theta = (aqq - app) / (2.0 * apq);
      const double tt = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
      const double c = 1.0 / sqrt(tt * tt + 1.0);
      o.c = c;
      o.s = tt * c;
    }
  }
  rot[t] = o;
}

// A <- J^T A J on every 2x2 block (P, Q) of the pairing, V <- V J
__global__ void k_jac_apply(double* __restrict__ A, double* __restrict__ V, int n, int npair,
                            const Rot* __restrict__ rot) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nblk = (long)npair * npair;
  if (idx < nblk) {
    const Rot P = rot[idx % npair], Q = rot[idx / npair];
    if (P.q < n && Q.q < n) {
      const double apr = A[(long)P.p * n + Q.p], aps = A[(long)P.p * n + Q.q];
      const double aqr = A[(long)P.q * n + Q.p], aqs = A[(long)P.q * n + Q.q];
      // rows: new_p = c a_p - s a_q, new_q = s a_p + c a_q
      const double rpr = P.c * apr - P.s * aqr, rps = P.c * aps - P.s * aqs;
      const double rqr = P.s * apr + P.c * aqr, rqs = P.s * aps + P.c * aqs;
      // columns; on the pair's own 2x2 block the annihilated element is set
      // to zero exactly (its computed value is rounding noise of size
      // eps*|a_pp|, which would stall convergence for large n)
      A[(long)P.p * n + Q.p] = Q.c * rpr - Q.s * rps;
      A[(long)P.p * n + Q.q] = P.p == Q.p ? 0.0 : Q.s * rpr + Q.c * rps;
      A[(long)P.q * n + Q.p] = P.p == Q.p ? 0.0 : Q.c * rqr - Q.s * rqs;
      A[(long)P.q * n + Q.q] = Q.s * rqr + Q.c * rqs;
    } else if (P.q >= n && Q.q < n && P.p < n) {
      // P pairs a real index with the dummy: only the column rotation of Q
      const double ar = A[(long)P.p * n + Q.p], as = A[(long)P.p * n + Q.q];
      A[(long)P.p * n + Q.p] = Q.c * ar - Q.s * as;
      A[(long)P.p * n + Q.q] = Q.s * ar + Q.c * as;
    } else if (Q.q >= n && P.q < n && Q.p < n) {
      const double ap = A[(long)P.p * n + Q.p], aq = A[(long)P.q * n + Q.p];
      A[(long)P.p * n + Q.p] = P.c * ap - P.s * aq;
      A[(long)P.q * n + Q.p] = P.s * ap + P.c * aq;
    }
  } else {
    const long v = idx - nblk;
    if (v >= (long)npair * n) return;
    const Rot Q = rot[v / n];
    const int i = (int)(v % n);
    if (Q.q >= n) return;
    // V column-major: column k at V + k*n
    const double vp = V[(long)Q.p * n + i], vq = V[(long)Q.q * n + i];
    V[(long)Q.p * n + i] = Q.c * vp - Q.s * vq;
    V[(long)Q.q * n + i] = Q.s * vp + Q.c * vq;
  }
}

__global__ void k_offdiag(const double* __restrict__ A, int n, double* __restrict__ out) {
  __shared__ double ws[8];
  double off = 0.0, tot = 0.0;
  for (long k = threadIdx.x; k < (long)n * n; k += blockDim.x) {
    const double a = A[k];
    tot = fma(a, a, tot);
    if (k / n != k % n) off = fma(a, a, off);
  }
  off = tree_fold256(off, ws);
  tot = tree_fold256(tot, ws);
  if (threadIdx.x == 0) {
    out[0] = off;
    out[1] = tot;
  }
}

__global__ void k_eye(double* __restrict__ V, int n) {
  const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (k < (long)n * n) V[k] = (k / n == k % n) ? 1.0 : 0.0;
}

// ascending stable order of the diagonal; columns of V permuted, each made to
// have its largest-magnitude component positive
__global__ void k_sort_eig(const double* __restrict__ A, const double* __restrict__ V, int n,
                           double* __restrict__ w, double* __restrict__ Z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double di = A[(long)i * n + i];
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const double dj = A[(long)j * n + j];
    if (dj < di || (dj == di && j < i)) ++rank;
  }
  w[rank] = di;
  const double* v = V + (long)i * n;
  int im = 0;
  for (int k = 1; k < n; ++k)
    if (fabs(v[k]) > fabs(v[im])) im = k;
  const double sg = v[im] < 0 ? -1.0 : 1.0;
  for (int k = 0; k < n; ++k) Z[(long)rank * n + k] = sg * v[k];
}

// ---------------------------------------------------------------- Cholesky
// In-place lower Cholesky of a symmetric positive definite n x n matrix
// (column-major; only the lower triangle is referenced), one CTA.
// info[0] = 0, or j+1 when the pivot of column j is not positive.
__global__ void k_potrf(double* __restrict__ A, int n, int* __restrict__ info) {
  __shared__ double piv;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int k = 0; k < n; ++k) {
    if (threadIdx.x == 0) {
      const double d = A[(long)k * n + k];
      if (!(d > 0.0)) {
        bad = k + 1;
        piv = 1.0;
      } else {
        piv = sqrt(d);
        A[(long)k * n + k] = piv;
      }
    }
    __syncthreads();
    if (bad) break;
    for (int i = k + 1 + threadIdx.x; i < n; i += blockDim.x) A[(long)k * n + i] /= piv;
    __syncthreads();
    // trailing update A[i][j] -= L[i][k] L[j][k], j in (k, i]
    const long m = n - k - 1;
    for (long e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int jj = (int)(e / m), ii = (int)(e % m);
      if (ii < jj) continue;
      const int i = k + 1 + ii, j = k + 1 + jj;
      A[(long)j * n + i] = fma(-A[(long)k * n + i], A[(long)k * n + j], A[(long)j * n + i]);
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) info[0] = bad;
}

// W = L^{-T} (upper triangular, column-major): column j of L^{-1} solved by
// forward substitution, stored as row j of W.  One thread per column.
__global__ void k_trinv_t(const double* __restrict__ L, int n, double* __restrict__ W) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  // x = L^{-1} e_j : x_i = 0 for i < j
  for (int i = 0; i < n; ++i) {
    double x = 0.0;
    if (i >= j) {
      double s = i == j ? 1.0 : 0.0;
      for (int k = j; k < i; ++k) s = fma(-L[(long)k * n + i], W[(long)k * n + j], s);
      x = s / L[(long)i * n + i];
    }
    // W(j, i) = x   (W = X^T, column-major W[i*n + j])
    W[(long)i * n + j] = x;
  }
}

}  // namespace

// A (n x n, symmetric, device) is overwritten; w (device, n) eigenvalues
// ascending, Z (device, n x n column-major) eigenvectors.  work: 2*n*n + ...
int syev_jacobi(int n, double* A, double* w, double* Z, int max_sweeps, cudaStream_t st,
                int* sweeps_out) {
  if (n <= 0) return RS_OK;
  const int ne = n + (n & 1);
  const int npair = ne / 2;
  double* V = nullptr;
  Rot* rot = nullptr;
  double* od = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&V, sizeof(double) * (size_t)n * n, st));
  RS_CUDA(cudaMallocAsync((void**)&rot, sizeof(Rot) * npair, st));
  RS_CUDA(cudaMallocAsync((void**)&od, sizeof(double) * 2, st));
  k_eye<<<div_up((long)n * n, 256), 256, 0, st>>>(V, n);
  int sweep = 0, rc = RS_OK;
  const long nwork = (long)npair * npair + (long)npair * n;
  for (; sweep < max_sweeps; ++sweep) {
    double h[2];
    k_offdiag<<<1, 256, 0, st>>>(A, n, od);
    cudaError_t e = cudaMemcpyAsync(h, od, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = cuda_status(e, "syev_jacobi"); break; }
    if (h[0] == 0.0 || h[0] <= 1e-30 * h[1]) break;
    for (int r = 0; r < ne - 1; ++r) {
      k_jac_params<<<div_up(npair, 128), 128, 0, st>>>(A, n, ne, r, rot);
      k_jac_apply<<<div_up(nwork, 256), 256, 0, st>>>(A, V, n, npair, rot);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) { rc = cuda_status(e, "k_jac_apply"); break; }
  }
  if (rc == RS_OK && sweep >= max_sweeps) rc = fail(RS_ENUMERIC, "syev: Jacobi did not converge");
  if (rc == RS_OK) {
    k_sort_eig<<<div_up(n, 128), 128, 0, st>>>(A, V, n, w, Z);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "k_sort_eig");
  }
  cudaFreeAsync(V, st);
  cudaFreeAsync(rot, st);
  cudaFreeAsync(od, st);
  if (sweeps_out) *sweeps_out = sweep;
  return rc;
}

// W = L^{-T} with G = L L^T (G overwritten by L); RS_ENUMERIC when G is not
// positive definite (kukan: 'wf has negative norm', orthogonalization8f.F90:249)
int chol_inv_t(int n, double* G, double* W, cudaStream_t st) {
  if (n <= 0) return RS_OK;
  int* info = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&info, sizeof(int), st));
  k_potrf<<<1, 1024, 0, st>>>(G, n, info);
  int h = 0;
  RS_CUDA(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  RS_CUDA(cudaStreamSynchronize(st));
  cudaFreeAsync(info, st);
  if (h) return fail(RS_ENUMERIC, "Cholesky-QR: overlap matrix not positive definite (negative norm)");
  k_trinv_t<<<div_up(n, 64), 64, 0, st>>>(G, n, W);
  RS_LAUNCH_CHECK("k_trinv_t");
  return RS_OK;
}

}  // namespace rs

extern "C" int rs_syev_f64(int n, double* A, double* w, double* Z, int* sweeps, void* stream) {
  if (n < 0) return rs::fail(RS_EINVAL, "rs_syev_f64: n < 0");
  return rs::syev_jacobi(n, A, w, Z, 60, rs::as_stream(stream), sweeps);
}

extern "C" int rs_chol_inv_t(int n, double* G, double* W, void* stream) {
  if (n < 0) return rs::fail(RS_EINVAL, "rs_chol_inv_t: n < 0");
  return rs::chol_inv_t(n, G, W, rs::as_stream(stream));
}
