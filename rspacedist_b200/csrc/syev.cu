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
#include <algorithm>

#include <cooperative_groups.h>

#include "rs_common.cuh"

namespace rs {
namespace cg = cooperative_groups;
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
__device__ __forceinline__ void jac_params(const double* __restrict__ A, int n, int ne, int r,
                                           int t, Rot* __restrict__ rot) {
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
__device__ __forceinline__ void jac_apply(double* __restrict__ A, double* __restrict__ V, int n,
                                          int npair, const Rot* __restrict__ rot, long idx) {
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

// one cyclic sweep: ne-1 rounds of (rotation parameters, apply), separated by
// grid-wide barriers of a cooperative launch (all blocks are co-resident)
constexpr int kJacThreads = 1024;
__global__ void __launch_bounds__(kJacThreads) k_jac_sweep(double* __restrict__ A, double* __restrict__ V, int n, int ne,
                            Rot* __restrict__ rot) {
  cg::grid_group grid = cg::this_grid();
  const int npair = ne / 2;
  const long nwork = (long)npair * npair + (long)npair * n;
  const long tid = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long stride = (long)gridDim.x * blockDim.x;
  for (int r = 0; r < ne - 1; ++r) {
    for (long t = tid; t < npair; t += stride) jac_params(A, n, ne, r, (int)t, rot);
    grid.sync();
    for (long idx = tid; idx < nwork; idx += stride) jac_apply(A, V, n, npair, rot, idx);
    grid.sync();
  }
}

// sums of squares of the off-diagonal and of all elements: chunk sums of the
// reduction tree (one 256-thread block per 4096 elements), then one fold
__global__ void k_offdiag_part(const double* __restrict__ A, int n, double* __restrict__ part) {
  __shared__ double ws[8];
  const long nn = (long)n * n;
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double off = 0.0, tot = 0.0;
#pragma unroll
  for (int k = 0; k < kTreePerLane; ++k) {
    const long e = base + (long)k * kTreeLanes;
    if (e < nn) {
      const double a = A[e];
      tot = fma(a, a, tot);
      if (e / n != e % n) off = fma(a, a, off);
    }
  }
  off = tree_fold256(off, ws);
  tot = tree_fold256(tot, ws);
  if (threadIdx.x == 0) {
    part[2 * blockIdx.x] = off;
    part[2 * blockIdx.x + 1] = tot;
  }
}

__global__ void k_offdiag_fold(long nblk, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double ws[8];
  double off = 0.0, tot = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) {
    off = off + part[2 * k];
    tot = tot + part[2 * k + 1];
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

// ------------------------------------------------ blocked Cholesky, L L^T = A
// A is column-major (element (i, k) at A[k*n + i]); the lower triangle is
// overwritten by L.  Block steps of kCholB columns: the diagonal block is
// factored by one CTA in shared memory, the panel below it by one thread per
// row, and the trailing lower triangle is updated in 32 x 32 tiles.
constexpr int kCholB = 64;

__global__ void k_chol_diag(double* __restrict__ A, int n, int kb, int* __restrict__ info) {
  __shared__ double a[kCholB][kCholB + 1];  // a[col][row]
  __shared__ double piv;
  const int b = min(kCholB, n - kb);
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e % b;
    a[c][r] = A[(long)(kb + c) * n + kb + r];
  }
  __syncthreads();
  for (int k = 0; k < b; ++k) {
    if (threadIdx.x == 0) {
      const double d = a[k][k];
      if (!(d > 0.0)) {
        if (info[0] == 0) info[0] = kb + k + 1;
        piv = 1.0;
      } else {
        piv = sqrt(d);
      }
      a[k][k] = piv;
    }
    __syncthreads();
    for (int i = k + 1 + threadIdx.x; i < b; i += blockDim.x) a[k][i] /= piv;
    __syncthreads();
    const int m = b - k - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int jj = e / m, ii = e % m;
      if (ii < jj) continue;
      const int i = k + 1 + ii, jc = k + 1 + jj;
      a[jc][i] = fma(-a[k][i], a[k][jc], a[jc][i]);
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e % b;
    if (r >= c) A[(long)(kb + c) * n + kb + r] = a[c][r];
  }
}

// rows i >= kb + b of the block column: L(i, kb:kb+b) = A(i, .) L_kk^{-T}
__global__ void k_chol_panel(double* __restrict__ A, int n, int kb) {
  __shared__ double l[kCholB][kCholB + 1];  // l[col][row] of L_kk
  const int b = min(kCholB, n - kb);
  for (int e = threadIdx.x; e < b * b; e += blockDim.x) {
    const int c = e / b, r = e % b;
    l[c][r] = A[(long)(kb + c) * n + kb + r];
  }
  __syncthreads();
  const int i = kb + b + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double x[kCholB];
  for (int c = 0; c < b; ++c) {
    double v = A[(long)(kb + c) * n + i];
    for (int k = 0; k < c; ++k) v = fma(-x[k], l[k][c], v);
    x[c] = v / l[c][c];
  }
  for (int c = 0; c < b; ++c) A[(long)(kb + c) * n + i] = x[c];
}

// A(i, j) -= sum_{k in block} L(i, k) L(j, k) for kb + b <= j <= i
__global__ void k_chol_trail(double* __restrict__ A, int n, int kb) {
  const int b = min(kCholB, n - kb);
  const int t0 = kb + b;
  const int ti = blockIdx.y, tj = blockIdx.x;
  if (tj > ti) return;
  __shared__ double li[kCholB][33], lj[kCholB][33];  // [k][row within tile]
  const int i0 = t0 + ti * 32, j0 = t0 + tj * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int k = ty; k < b; k += blockDim.y) {
    const int ri = i0 + tx, rj = j0 + tx;
    li[k][tx] = ri < n ? A[(long)(kb + k) * n + ri] : 0.0;
    lj[k][tx] = rj < n ? A[(long)(kb + k) * n + rj] : 0.0;
  }
  __syncthreads();
  const int i = i0 + ty, j = j0 + tx;
  if (i >= n || j >= n || j > i) return;
  double s = 0.0;
  for (int k = 0; k < b; ++k) s = fma(li[k][ty], lj[k][tx], s);
  A[(long)j * n + i] -= s;
}

// LT (row-major) = L: LT[i*n + k] = L(i, k) for k <= i
__global__ void k_lower_rows(const double* __restrict__ A, int n, double* __restrict__ LT) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long)n * n) return;
  const int i = (int)(e / n), k = (int)(e % n);
  LT[e] = k <= i ? A[(long)k * n + i] : 0.0;
}

// W (column-major) = L^{-T}: column j of X = L^{-1} by forward substitution,
// one warp per column, the sum of each step spread over the lanes; the
// column lives in shared memory (n doubles per warp)
__global__ void k_trinv_cols(const double* __restrict__ LT, int n, double* __restrict__ W) {
  extern __shared__ double xs[];
  const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
  const int j = blockIdx.x * (blockDim.x >> 5) + wib;
  if (j >= n) return;
  double* x = xs + (long)wib * n;
  for (int i = j; i < n; ++i) {
    const double* row = LT + (long)i * n;
    double s = 0.0;
    for (int k = j + lane; k < i; k += 32) s = fma(row[k], x[k], s);
    for (int off = 16; off >= 1; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    if (lane == 0) x[i] = ((i == j ? 1.0 : 0.0) - s) / row[i];
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) W[(long)i * n + j] = i >= j ? x[i] : 0.0;
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
  const long oblk = tree_chunks((long)n * n);
  RS_CUDA(cudaMallocAsync((void**)&od, sizeof(double) * (2 + 2 * oblk), st));
  k_eye<<<div_up((long)n * n, 256), 256, 0, st>>>(V, n);
  int sweep = 0, rc = RS_OK;
  // the cooperative grid: one 1024-thread block per SM (fewer blocks make
  // the grid barrier cheaper), at most one block per 1024 work items
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_jac_sweep, kJacThreads, 0);
  const long nwork = (long)npair * npair + (long)npair * n;
  const unsigned coop_grid = (unsigned)std::max(
      1L, std::min((long)nsm * std::min(std::max(per_sm, 1), 1),
                   (nwork + kJacThreads - 1) / kJacThreads));
  for (; sweep < max_sweeps; ++sweep) {
    double h[2];
    k_offdiag_part<<<(unsigned)oblk, kTreeLanes, 0, st>>>(A, n, od + 2);
    k_offdiag_fold<<<1, kTreeLanes, 0, st>>>(oblk, od + 2, od);
    cudaError_t e = cudaMemcpyAsync(h, od, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = cuda_status(e, "syev_jacobi"); break; }
    if (h[0] == 0.0 || h[0] <= 1e-30 * h[1]) break;
    {
      int nn = n, nne = ne;
      void* args[] = {&A, &V, &nn, &nne, &rot};
      e = cudaLaunchCooperativeKernel((void*)k_jac_sweep, coop_grid, kJacThreads, args, 0, st);
    }
    if (e != cudaSuccess) { rc = cuda_status(e, "k_jac_sweep"); break; }
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
  double* LT = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&info, sizeof(int), st));
  RS_CUDA(cudaMemsetAsync(info, 0, sizeof(int), st));
  for (int kb = 0; kb < n; kb += kCholB) {
    k_chol_diag<<<1, 256, 0, st>>>(G, n, kb, info);
    const int rest = n - kb - kCholB;
    if (rest > 0) {
      k_chol_panel<<<div_up(rest, 64), 64, 0, st>>>(G, n, kb);
      const unsigned nt = div_up(rest, 32);
      k_chol_trail<<<dim3(nt, nt), dim3(32, 32), 0, st>>>(G, n, kb);
    }
  }
  int h = 0;
  RS_CUDA(cudaMemcpyAsync(&h, info, sizeof(int), cudaMemcpyDeviceToHost, st));
  RS_CUDA(cudaStreamSynchronize(st));
  cudaFreeAsync(info, st);
  if (h) return fail(RS_ENUMERIC, "Cholesky-QR: overlap matrix not positive definite (negative norm)");
  RS_CUDA(cudaMallocAsync((void**)&LT, sizeof(double) * (size_t)n * n, st));
  k_lower_rows<<<div_up((long)n * n, 256), 256, 0, st>>>(G, n, LT);
  const int wpb = (int)std::max(1L, std::min(8L, (96L * 1024) / ((long)n * 8)));
  const size_t sm = sizeof(double) * (size_t)wpb * n;
  cudaError_t e = cudaSuccess;
  if (sm > 48 * 1024)
    e = cudaFuncSetAttribute(k_trinv_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e == cudaSuccess) {
    k_trinv_cols<<<div_up(n, wpb), 32 * wpb, sm, st>>>(LT, n, W);
    e = cudaGetLastError();
  }
  cudaFreeAsync(LT, st);
  if (e != cudaSuccess) return cuda_status(e, "k_trinv_cols");
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
