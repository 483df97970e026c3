// syev.cu -- FP64 dense kernels of the subspace step on the GPU:
//  * symmetric eigensolver (block Jacobi: round-robin pairing of 32-index
//    blocks, 64 x 64 subproblems in shared memory, batched FP64 tile
//    updates), the replacement of dsyev / pdsyevd in rayleighritz_r
//    (rayleigh-ritz8f.F90:89; rayleigh-ritz8f_sclpck.F90:268);
//  * Cholesky factorisation and triangular inverse for Cholesky-QR, which
//    spans the same vectors in the same order as kukan's block Gram-Schmidt
//    (orthogonalization8f.F90:93-376).
#include <math.h>

#include <vector>

#include "reduce.cuh"
#include <algorithm>

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

// ------------------------------------------------ block Jacobi eigensolver
// The padded matrix (np = nbe*32 indices, nbe even) is split into 32-index
// blocks; a sweep is nbe-1 rounds of the circle method over the blocks.  In a
// round every block pair P = (I, J) is one 64 x 64 subproblem:
//  * k_bjac_solve: one CTA runs a cyclic Jacobi sweep of the subproblem in
//    shared memory (63 rounds of 32 disjoint rotations, the rotation and the
//    exact zeroing of each annihilated element as in the scalar method),
//    writes the rotated 64 x 64 block back and keeps Q_P (the product of its
//    rotations);
//  * k_bjac_update: every other tile, A(P1, P2) <- Q_P1^T A(P1, P2) Q_P2 for
//    P1 > P2 (mirrored to (P2, P1), so A stays exactly symmetric), and the
//    eigenvectors V(:, P) <- V(:, P) Q_P.
// Padding indices have zero couplings, so their rotations are exact
// identities and the real n x n problem is untouched by them.
constexpr int JB = 32;
constexpr int JB2 = 2 * JB;
constexpr int JLD = JB2 + 1;  // padded smem row
constexpr int kBjThreads = 256;
// the subproblem sweep is latency-bound (63 dependent rounds, two barriers
// each): one rotation pair of S and two entries of Q per thread and round
constexpr int kBjSolveThreads = 1024;

__device__ __forceinline__ int bj_index(int I, int J, int k) {
  return k < JB ? I * JB + k : J * JB + (k - JB);
}

// rotation (c, s) zeroing S[p][q]: the smaller root t of t^2 + 2 theta t - 1 = 0,
// theta = (aqq - app) / (2 apq), written as t = sign(theta) 2|apq| / (|d| +
// sqrt(d^2 + 4 apq^2)) with d = aqq - app, and c = 1/sqrt(1 + t^2).  The
// sign convention is the scalar sweep's (theta = +-0 counts as positive); one
// division, one square root and one reciprocal square root per rotation,
// since these dependent long-latency steps set the pace of the 63 rounds.
__device__ __forceinline__ Rot bj_params(const double (*S)[JLD], int p, int q) {
  Rot o{p, q, 1.0, 0.0};
  const double apq = S[p][q];
  if (apq != 0.0) {
    const double app = S[p][p], aqq = S[q][q];
    const double d = aqq - app;
    const double a2 = 2.0 * fabs(apq);
    const double sgn = (d == 0.0 || (d > 0.0) == (apq > 0.0)) ? 1.0 : -1.0;
    const double tt = sgn * a2 / (fabs(d) + sqrt(d * d + a2 * a2));
    const double c = rsqrt(tt * tt + 1.0);
    o.c = c;
    o.s = tt * c;
  }
  return o;
}

__global__ void __launch_bounds__(kBjSolveThreads) k_bjac_solve(double* __restrict__ A, int np,
                                                           int nbe, int round,
                                                           double* __restrict__ Qbuf) {
  extern __shared__ double bj_sm[];
  double(*S)[JLD] = reinterpret_cast<double(*)[JLD]>(bj_sm);  // [JB2][JLD]
  double(*Q)[JLD] = S + JB2;
  __shared__ Rot rot[JB];
  const int tid = threadIdx.x;
  int I, J;
  rr_pair(round, blockIdx.x, nbe, &I, &J);
  for (int e = tid; e < JB2 * JB2; e += kBjSolveThreads) {
    const int r = e / JB2, c = e % JB2;
    S[r][c] = A[(long)bj_index(I, J, r) * np + bj_index(I, J, c)];
    Q[r][c] = r == c ? 1.0 : 0.0;
  }
  __syncthreads();
  for (int ir = 0; ir < JB2 - 1; ++ir) {
    if (tid < JB) {
      int p, q;
      rr_pair(ir, tid, JB2, &p, &q);
      rot[tid] = bj_params(S, p, q);
    }
    __syncthreads();
    // S <- J^T S J on the 2x2 blocks of every two rotations
    for (int k = tid; k < JB * JB; k += kBjSolveThreads) {
      const Rot P = rot[k % JB], R = rot[k / JB];
      const double apr = S[P.p][R.p], aps = S[P.p][R.q];
      const double aqr = S[P.q][R.p], aqs = S[P.q][R.q];
      const double rpr = P.c * apr - P.s * aqr, rps = P.c * aps - P.s * aqs;
      const double rqr = P.s * apr + P.c * aqr, rqs = P.s * aps + P.c * aqs;
      S[P.p][R.p] = R.c * rpr - R.s * rps;
      S[P.p][R.q] = P.p == R.p ? 0.0 : R.s * rpr + R.c * rps;
      S[P.q][R.p] = P.p == R.p ? 0.0 : R.c * rqr - R.s * rqs;
      S[P.q][R.q] = R.s * rqr + R.c * rqs;
    }
    // Q <- Q J
    for (int k = tid; k < JB * JB2; k += kBjSolveThreads) {
      const Rot R = rot[k / JB2];
      const int i = k % JB2;
      const double qp = Q[i][R.p], qq = Q[i][R.q];
      Q[i][R.p] = R.c * qp - R.s * qq;
      Q[i][R.q] = R.s * qp + R.c * qq;
    }
    __syncthreads();
  }
  double* Qo = Qbuf + (long)blockIdx.x * JB2 * JB2;
  for (int e = tid; e < JB2 * JB2; e += kBjSolveThreads) {
    const int r = e / JB2, c = e % JB2;
    A[(long)bj_index(I, J, r) * np + bj_index(I, J, c)] = S[r][c];
    Qo[e] = Q[r][c];  // row-major Q[r][c]
  }
}

// C (64 x 64, smem) = X^T Y or X Y for 64 x 64 smem operands; 256 threads,
// a 4 x 4 output block each (rows ty + 16 a, columns tx + 16 b)
template <bool XT>
__device__ __forceinline__ void bj_gemm(const double (*X)[JLD], const double (*Y)[JLD],
                                        double (*C)[JLD]) {
  const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int k = 0; k < JB2; ++k) {
    double x[4], y[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) x[a] = XT ? X[k][ty + 16 * a] : X[ty + 16 * a][k];
#pragma unroll
    for (int b = 0; b < 4; ++b) y[b] = Y[k][tx + 16 * b];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = fma(x[a], y[b], acc[a][b]);
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) C[ty + 16 * a][tx + 16 * b] = acc[a][b];
}

// blocks [0, ntile): A tiles (P1 > P2) of the round; then V tiles (64 rows of
// V x the 64 columns of one pair).  V is column-major: (i, k) at V[k*np + i].
__global__ void __launch_bounds__(kBjThreads) k_bjac_update(double* __restrict__ A,
                                                            double* __restrict__ V, int np,
                                                            int nbe, int round,
                                                            const double* __restrict__ Qbuf) {
  extern __shared__ double bj_sm[];
  double(*X)[JLD] = reinterpret_cast<double(*)[JLD]>(bj_sm);
  double(*Y)[JLD] = X + JB2;
  double(*T)[JLD] = Y + JB2;
  const int tid = threadIdx.x;
  const int npair = nbe / 2;
  const int ntile = npair * (npair - 1) / 2;
  const int bx = blockIdx.x;
  if (bx < ntile) {
    int p1 = (int)((sqrtf(8.f * bx + 1.f) + 1.f) * 0.5f);  // bx = p1 (p1 - 1) / 2 + p2
    while (p1 * (p1 - 1) / 2 > bx) --p1;
    while ((p1 + 1) * p1 / 2 <= bx) ++p1;
    const int p2 = bx - p1 * (p1 - 1) / 2;
    int I1, J1, I2, J2;
    rr_pair(round, p1, nbe, &I1, &J1);
    rr_pair(round, p2, nbe, &I2, &J2);
    const double* Q1 = Qbuf + (long)p1 * JB2 * JB2;
    const double* Q2 = Qbuf + (long)p2 * JB2 * JB2;
    for (int e = tid; e < JB2 * JB2; e += kBjThreads) {
      const int r = e / JB2, c = e % JB2;
      X[r][c] = Q1[e];
      Y[r][c] = A[(long)bj_index(I1, J1, r) * np + bj_index(I2, J2, c)];
    }
    __syncthreads();
    bj_gemm<true>(X, Y, T);  // T = Q1^T B
    __syncthreads();
    for (int e = tid; e < JB2 * JB2; e += kBjThreads) X[e / JB2][e % JB2] = Q2[e];
    __syncthreads();
    bj_gemm<false>(T, X, Y);  // Y = T Q2
    __syncthreads();
    for (int e = tid; e < JB2 * JB2; e += kBjThreads) {
      const int r = e / JB2, c = e % JB2;
      const double v = Y[r][c];
      A[(long)bj_index(I1, J1, r) * np + bj_index(I2, J2, c)] = v;
      A[(long)bj_index(I2, J2, c) * np + bj_index(I1, J1, r)] = v;
    }
  } else {
    const int v = bx - ntile;
    const int p = v % npair, rt = v / npair;
    int I, J;
    rr_pair(round, p, nbe, &I, &J);
    const double* Qp = Qbuf + (long)p * JB2 * JB2;
    for (int e = tid; e < JB2 * JB2; e += kBjThreads) {
      Y[e / JB2][e % JB2] = Qp[e];
      const int r = e % JB2, c = e / JB2;  // consecutive threads: consecutive rows of V
      X[r][c] = V[(long)bj_index(I, J, c) * np + rt * JB2 + r];
    }
    __syncthreads();
    bj_gemm<false>(X, Y, T);  // T = V(rows, P) Q
    __syncthreads();
    for (int e = tid; e < JB2 * JB2; e += kBjThreads) {
      const int r = e % JB2, c = e / JB2;
      V[(long)bj_index(I, J, c) * np + rt * JB2 + r] = T[r][c];
    }
  }
}

// padded copy A' (np x np) = [A 0; 0 0] and V' = I: a zero coupling is
// never rotated, so the padding indices stay exactly decoupled
__global__ void k_bjac_pad(const double* __restrict__ A, int n, int np, double* __restrict__ Ap,
                           double* __restrict__ V) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= (long)np * np) return;
  const int r = (int)(e / np), c = (int)(e % np);
  Ap[e] = (r < n && c < n) ? A[(long)r * n + c] : 0.0;
  V[e] = r == c ? 1.0 : 0.0;
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

// ascending stable order of the diagonal of the leading n x n block (row
// stride ld); columns of V permuted, each made to have its largest-magnitude
// component positive
__global__ void k_sort_eig(const double* __restrict__ A, const double* __restrict__ V, int n,
                           int ld, double* __restrict__ w, double* __restrict__ Z) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double di = A[(long)i * ld + i];
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const double dj = A[(long)j * ld + j];
    if (dj < di || (dj == di && j < i)) ++rank;
  }
  w[rank] = di;
  const double* v = V + (long)i * ld;
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
// ascending, Z (device, n x n column-major) eigenvectors.  Sweeps of the
// block method until the off-diagonal norm is below 1e-15 of the norm.
int syev_jacobi(int n, double* A, double* w, double* Z, int max_sweeps, cudaStream_t st,
                int* sweeps_out) {
  if (n <= 0) return RS_OK;
  const int nb = (n + JB - 1) / JB;
  const int nbe = std::max(2, nb + (nb & 1));
  const int np = nbe * JB;
  const int npair = nbe / 2;
  const long nn = (long)np * np;
  double *Ap = nullptr, *V = nullptr, *Qb = nullptr, *od = nullptr;
  const long oblk = tree_chunks(nn);
  RS_CUDA(cudaMallocAsync((void**)&Ap, sizeof(double) * (2 * nn + (long)npair * JB2 * JB2 +
                                                          2 + 2 * oblk), st));
  V = Ap + nn;
  Qb = V + nn;
  od = Qb + (long)npair * JB2 * JB2;
  k_bjac_pad<<<div_up(nn, 256), 256, 0, st>>>(A, n, np, Ap, V);
  const int usm = 3 * JB2 * JLD * (int)sizeof(double), ssm = 2 * JB2 * JLD * (int)sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_bjac_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       usm);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_bjac_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, ssm);
  int sweep = 0, rc = e == cudaSuccess ? RS_OK : cuda_status(e, "k_bjac_update");
  const unsigned nupd = (unsigned)(npair * (npair - 1) / 2 + npair * npair);
  for (; rc == RS_OK && sweep < max_sweeps; ++sweep) {
    double h[2];
    k_offdiag_part<<<(unsigned)oblk, kTreeLanes, 0, st>>>(Ap, np, od + 2);
    k_offdiag_fold<<<1, kTreeLanes, 0, st>>>(oblk, od + 2, od);
    e = cudaMemcpyAsync(h, od, sizeof(h), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = cuda_status(e, "syev_jacobi"); break; }
    if (h[0] == 0.0 || h[0] <= 1e-30 * h[1]) break;
    for (int r = 0; r < nbe - 1; ++r) {
      k_bjac_solve<<<npair, kBjSolveThreads, ssm, st>>>(Ap, np, nbe, r, Qb);
      k_bjac_update<<<nupd, kBjThreads, usm, st>>>(Ap, V, np, nbe, r, Qb);
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "k_bjac");
  }
  if (rc == RS_OK && sweep >= max_sweeps) rc = fail(RS_ENUMERIC, "syev: Jacobi did not converge");
  if (rc == RS_OK) {
    k_sort_eig<<<div_up(n, 128), 128, 0, st>>>(Ap, V, n, np, w, Z);
    e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "k_sort_eig");
  }
  cudaFreeAsync(Ap, st);
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
