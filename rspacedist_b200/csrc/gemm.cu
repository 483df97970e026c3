// gemm.cu -- subspace contractions of the Gram-Schmidt / Rayleigh-Ritz step.
//
//  * Gram matrices C = alpha A^T B (Psi^T H Psi, Psi^T S Psi): K = grid
//    points (millions), M, N = bands.
//  * Band rotations Y = X Z (Psi <- Psi C): K = bands.
//
// FP32 operands run on the 5th-generation tensor cores (tcgen05.mma,
// kind::tf32) with the 3xTF32 split: x = hi + lo with hi = tf32(x) and lo = x -
// hi, and A B ~ hi_A hi_B + hi_A lo_B + lo_A hi_B, accumulated in FP32 in
// TMEM.  Operands are staged global -> registers -> shared memory (where the
// split happens) in the 128-byte-swizzled canonical layouts; one thread issues
// the MMAs and commits them to an mbarrier that frees the stage.  Gram
// products split K into chunks whose FP32 partial tiles are summed in FP64 in
// a fixed order.  FP64 operands use tiled FP64 kernels (CUDA cores).
#include <math.h>

#include "rs_common.cuh"
#include "tc_ptx.cuh"

namespace rs {
namespace {

using namespace tc;

constexpr int GM = 128;        // tile rows (MMA M)
constexpr int GN = 128;        // Gram tile cols (MMA N)
constexpr int KB = 32;         // K per stage: one 128-byte swizzle row of fp32
constexpr int TILE_BYTES = GM * KB * 4;  // 16 KB

__device__ int g_tc_error;     // set when a bounded wait gives up

// byte offset of (row r, 16-byte chunk c) in a K-major SW128 tile of 128-byte rows
__device__ __forceinline__ uint32_t kmaj_off(int r, int c) {
  return (uint32_t)((r >> 3) * 1024 + (r & 7) * 128 + ((c ^ (r & 7)) << 4));
}

__device__ __forceinline__ void split_store(char* hi_base, char* lo_base, uint32_t off,
                                            float4 v) {
  float4 h, l;
  h.x = tf32_rna(v.x); l.x = v.x - h.x;
  h.y = tf32_rna(v.y); l.y = v.y - h.y;
  h.z = tf32_rna(v.z); l.z = v.z - h.z;
  h.w = tf32_rna(v.w); l.w = v.w - h.w;
  *reinterpret_cast<float4*>(hi_base + off) = h;
  *reinterpret_cast<float4*>(lo_base + off) = l;
}

// ------------------------------------------------------------------ Gram
// FP64 partial tiles P[pair][split][j][i] = sum_{k in chunk} A[i][k] B[j][k]
// for one 128 x 128 tile pair and one K chunk.  The tensor core accumulates
// at most DG stages (DG*32 terms, 3 MMA passes) in FP32 in one of two TMEM
// buffers; each finished buffer is drained into FP64 registers while the
// other one fills, so long sums never build up in FP32.
constexpr int GRAM_THREADS = 256;
constexpr int DG = 2;

__device__ __forceinline__ void drain_f64(uint32_t taddr, double* acc) {
  uint32_t r[32];
  tmem_ld32(taddr, r);
  tmem_ld_wait();
#pragma unroll
  for (int k = 0; k < 32; ++k) acc[k] += (double)__uint_as_float(r[k]);
  tmem_ld32(taddr + 32, r);
  tmem_ld_wait();
#pragma unroll
  for (int k = 0; k < 32; ++k) acc[32 + k] += (double)__uint_as_float(r[k]);
}

__global__ void __launch_bounds__(GRAM_THREADS, 1)
    k_gram_tf32x3(const float* __restrict__ A, long lda, int m, const float* __restrict__ B,
                  long ldb, int n, long K, long kchunk, int sym, int tn,
                  double* __restrict__ part) {
  extern __shared__ __align__(1024) char smem_dyn[];
  char* smem = (char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  // stage s: A hi | A lo | B hi | B lo
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  int it, jt;
  {
    const int pr = blockIdx.x;
    if (sym) {  // lower triangle it >= jt, row-major over it
      it = (int)((sqrtf(8.f * pr + 1.f) - 1.f) * 0.5f);
      while ((it + 1) * (it + 2) / 2 <= pr) ++it;
      while (it * (it + 1) / 2 > pr) --it;
      jt = pr - it * (it + 1) / 2;
    } else {
      it = pr % tn;
      jt = pr / tn;
    }
  }
  const long k0 = (long)blockIdx.y * kchunk;
  const long k1 = min(K, k0 + kchunk);
  const int nkb = (int)((k1 - k0 + KB - 1) / KB);

  if (warp == 0) tmem_alloc(&tmem_base, 2 * GN);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_relinquish();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = idesc_tf32(GM, GN, 0, 0);
  // drain role: lane quadrant q (TMEM lanes 32q..), column half h
  const int dq = warp & 3, dh = warp >> 2;
  const uint32_t dlane = (uint32_t)(dq * 32) << 16;
  double acc[64];
#pragma unroll
  for (int k = 0; k < 64; ++k) acc[k] = 0.0;

  const int lc = tid & 7;
  const int lr = tid >> 3;  // 0..31
  bool bad = false;
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb & 1;
    const int g = kb / DG;
    const long kk0 = k0 + (long)kb * KB + 4 * lc;
    float4 va[4], vb[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = lr + 32 * i;
      const int ra = it * GM + r, rb = jt * GN + r;
      const bool kin = kk0 < k1;
      va[i] = (ra < m && kin) ? __ldg(reinterpret_cast<const float4*>(A + (long)ra * lda + kk0))
                              : make_float4(0.f, 0.f, 0.f, 0.f);
      vb[i] = (rb < n && kin) ? __ldg(reinterpret_cast<const float4*>(B + (long)rb * ldb + kk0))
                              : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (kb >= 2) {
      const bool ok = mbar_wait(&mbar[s], ((kb - 2) >> 1) & 1);
      if (__syncthreads_or(!ok)) { bad = true; break; }
    }
    if (kb % DG == 0 && g >= 2) {
      // group g-2 (same TMEM buffer) has completed: fold it into FP64
      tc_fence_after();
      drain_f64(tmem + (g & 1) * GN + dh * 64 + dlane, acc);
      tc_fence_before();
    }
    char* st = smem + s * 4 * TILE_BYTES;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t off = kmaj_off(lr + 32 * i, lc);
      split_store(st, st + TILE_BYTES, off, va[i]);
      split_store(st + 2 * TILE_BYTES, st + 3 * TILE_BYTES, off, vb[i]);
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t d = tmem + (g & 1) * GN;
      const uint32_t sa = smem_u32(st);
#pragma unroll
      for (int q = 0; q < 4; ++q) {  // K = 8 per instruction, 32 bytes
        const uint64_t ahi = smem_desc_sw128(sa + q * 32, 16, 1024);
        const uint64_t alo = smem_desc_sw128(sa + TILE_BYTES + q * 32, 16, 1024);
        const uint64_t bhi = smem_desc_sw128(sa + 2 * TILE_BYTES + q * 32, 16, 1024);
        const uint64_t blo = smem_desc_sw128(sa + 3 * TILE_BYTES + q * 32, 16, 1024);
        mma_tf32(d, alo, bhi, idesc, ((kb % DG) | q) != 0);
        mma_tf32(d, ahi, blo, idesc, 1);
        mma_tf32(d, ahi, bhi, idesc, 1);
      }
      mma_commit(&mbar[s]);
    }
  }
  if (!bad && nkb > 0) {
    const int s = (nkb - 1) & 1;
    const bool ok = mbar_wait(&mbar[s], ((nkb - 1) >> 1) & 1);
    bad = __syncthreads_or(!ok);
  }
  tc_fence_after();
  if (bad) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
  } else {
    const int glast = (nkb - 1) / DG;
    if (nkb > 0 && glast >= 1) drain_f64(tmem + ((glast - 1) & 1) * GN + dh * 64 + dlane, acc);
    if (nkb > 0) drain_f64(tmem + (glast & 1) * GN + dh * 64 + dlane, acc);
    double* P = part + ((long)blockIdx.x * gridDim.y + blockIdx.y) * GM * GN;
    const int row = dq * 32 + (tid & 31);
#pragma unroll
    for (int k = 0; k < 64; ++k) P[(long)(dh * 64 + k) * GM + row] = acc[k];
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 2 * GN);
}

// C[i + j*ldc] = alpha * sum over splits (fixed order) of the FP64 partials;
// for symmetric products the upper triangle is mirrored.
__global__ void k_gram_reduce(const double* __restrict__ part, int nsplit, int m, int n, int sym,
                              int tn, double alpha, double* __restrict__ C, long ldc) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)m * n) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  int ii = i, jj = j;
  if (sym && i < j) { ii = j; jj = i; }
  const int it = ii / GM, jt = jj / GN;
  const int pr = sym ? it * (it + 1) / 2 + jt : jt * tn + it;
  const double* p = part + (long)pr * nsplit * GM * GN + (long)(jj % GN) * GM + (ii % GM);
  double s = 0.0;
  for (int sp = 0; sp < nsplit; ++sp) s += p[(long)sp * GM * GN];
  C[(long)j * ldc + i] = alpha * s;
}

// ------------------------------------------------------------------ rotation
// Y[j][p] = sum_k X[k][p] Z(k, j) for a 128-point x RN-band tile.  A = X is
// MN-major (points contiguous), B = Z^T is K-major (Zhi/Zlo given as [j][k]).
// TMEM accumulates DR stages per buffer; drained sums add up in FP32
// registers.
constexpr int RN = 128;         // output bands per tile (MMA N)
constexpr int DR = 2;
constexpr int ROT_THREADS = 256;
constexpr int ROT_A_BYTES = GM * KB * 4;   // 16 KB
constexpr int ROT_B_BYTES = RN * KB * 4;   // 16 KB
constexpr int ROT_STAGE = 2 * ROT_A_BYTES + 2 * ROT_B_BYTES;  // 64 KB

// byte offset of (point p, band k) in the MN-major tile: each k-row holds 32
// points (128 B) whose 32-byte chunks are XOR-swizzled with (k mod 4);
// 4-row atoms (512 B) step along k (SBO = 512 B), 32-point blocks of 8
// atoms (4 KB) step along the points (LBO = 4 KB)
__device__ __forceinline__ uint32_t mnmaj_off(int p, int k) {
  return (uint32_t)((p >> 5) * 4096 + (k >> 2) * 512 + (k & 3) * 128 +
                    ((((p & 31) >> 3) ^ (k & 3)) << 5) + (p & 7) * 4);
}

__device__ __forceinline__ void drain_f32(uint32_t taddr, float* acc) {
  uint32_t r[32];
  tmem_ld32(taddr, r);
  tmem_ld_wait();
#pragma unroll
  for (int k = 0; k < 32; ++k) acc[k] += __uint_as_float(r[k]);
  tmem_ld32(taddr + 32, r);
  tmem_ld_wait();
#pragma unroll
  for (int k = 0; k < 32; ++k) acc[32 + k] += __uint_as_float(r[k]);
}

__global__ void __launch_bounds__(ROT_THREADS, 1)
    k_rotate_tf32x3(const float* __restrict__ X, long ldx, long npts, int kin,
                    const float* __restrict__ Zhi, const float* __restrict__ Zlo, int kpad,
                    int nout, float* __restrict__ Y, long ldy) {
  extern __shared__ __align__(1024) char smem_dyn[];
  char* smem = (char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  const int tid = threadIdx.x, warp = tid >> 5;
  const long p0 = (long)blockIdx.x * GM;
  const int j0 = blockIdx.y * RN;
  const int nkb = (kin + KB - 1) / KB;
  if (warp == 0) tmem_alloc(&tmem_base, 2 * RN);
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 0) tmem_relinquish();
  const uint32_t tmem = tmem_base;
  constexpr uint32_t idesc = idesc_tf32(GM, RN, 1, 0);
  const int dq = warp & 3, dh = warp >> 2;
  const uint32_t dlane = (uint32_t)(dq * 32) << 16;
  float acc[64];
#pragma unroll
  for (int k = 0; k < 64; ++k) acc[k] = 0.f;
  // X loader: 32 k-rows x 32 float4 -> 4 per thread; Z loader: 128 j x 8 chunks -> 4 per thread
  const int xc = tid & 31, xr = tid >> 5;  // xr 0..7
  const int zc = tid & 7, zr = tid >> 3;   // zr 0..31
  bool bad = false;
  for (int kb = 0; kb < nkb; ++kb) {
    const int s = kb & 1;
    const int g = kb / DR;
    float4 vx[4], vzh[4], vzl[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = kb * KB + xr + 8 * i;
      const long p = p0 + 4 * xc;
      vx[i] = (k < kin && p < npts)
                  ? __ldg(reinterpret_cast<const float4*>(X + (long)k * ldx + p))
                  : make_float4(0.f, 0.f, 0.f, 0.f);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int j = j0 + zr + 32 * i;
      const long o = (long)j * kpad + kb * KB + 4 * zc;
      const bool in = j < nout;
      vzh[i] = in ? __ldg(reinterpret_cast<const float4*>(Zhi + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
      vzl[i] = in ? __ldg(reinterpret_cast<const float4*>(Zlo + o)) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (kb >= 2) {
      const bool ok = mbar_wait(&mbar[s], ((kb - 2) >> 1) & 1);
      if (__syncthreads_or(!ok)) { bad = true; break; }
    }
    if (kb % DR == 0 && g >= 2) {
      tc_fence_after();
      drain_f32(tmem + (g & 1) * RN + dh * 64 + dlane, acc);
      tc_fence_before();
    }
    char* st = smem + s * ROT_STAGE;
    char* ahi = st;
    char* alo = st + ROT_A_BYTES;
    char* bhi = st + 2 * ROT_A_BYTES;
    char* blo = bhi + ROT_B_BYTES;
#pragma unroll
    for (int i = 0; i < 4; ++i) split_store(ahi, alo, mnmaj_off(4 * xc, xr + 8 * i), vx[i]);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t off = kmaj_off(zr + 32 * i, zc);
      *reinterpret_cast<float4*>(bhi + off) = vzh[i];
      *reinterpret_cast<float4*>(blo + off) = vzl[i];
    }
    fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc_fence_after();
      const uint32_t d = tmem + (g & 1) * RN;
      const uint32_t sa = smem_u32(ahi), sl = smem_u32(alo);
      const uint32_t sb = smem_u32(bhi), sbl = smem_u32(blo);
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const uint64_t dah = smem_desc_sw128_b32(sa + q * 1024, 4096, 512);
        const uint64_t dal = smem_desc_sw128_b32(sl + q * 1024, 4096, 512);
        const uint64_t dbh = smem_desc_sw128(sb + q * 32, 16, 1024);
        const uint64_t dbl = smem_desc_sw128(sbl + q * 32, 16, 1024);
        mma_tf32(d, dal, dbh, idesc, ((kb % DR) | q) != 0);
        mma_tf32(d, dah, dbl, idesc, 1);
        mma_tf32(d, dah, dbh, idesc, 1);
      }
      mma_commit(&mbar[s]);
    }
  }
  if (!bad && nkb > 0) {
    const int s = (nkb - 1) & 1;
    const bool ok = mbar_wait(&mbar[s], ((nkb - 1) >> 1) & 1);
    bad = __syncthreads_or(!ok);
  }
  tc_fence_after();
  if (bad) {
    if (tid == 0) atomicExch(&g_tc_error, 1);
  } else {
    const int glast = (nkb - 1) / DR;
    if (nkb > 0 && glast >= 1) drain_f32(tmem + ((glast - 1) & 1) * RN + dh * 64 + dlane, acc);
    if (nkb > 0) drain_f32(tmem + (glast & 1) * RN + dh * 64 + dlane, acc);
    const long p = p0 + dq * 32 + (tid & 31);
    if (p < npts) {
#pragma unroll
      for (int k = 0; k < 64; ++k) {
        const int j = j0 + dh * 64 + k;
        if (j < nout) Y[(long)j * ldy + p] = acc[k];
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) tmem_dealloc(tmem, 2 * RN);
}

// Z (FP64, column-major kin x nout) -> Zhi/Zlo [j][kpad] FP32 with hi = tf32(z)
__global__ void k_split_z(const double* __restrict__ Z, long ldz, int kin, int nout, int kpad,
                          float* __restrict__ hi, float* __restrict__ lo) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)nout * kpad) return;
  const int k = (int)(idx % kpad), j = (int)(idx / kpad);
  const float z = k < kin ? (float)Z[(long)j * ldz + k] : 0.f;
  const float h = tf32_rna(z);
  hi[idx] = h;
  lo[idx] = z - h;
}

// ------------------------------------------------------------------ FP64
// C tile 64 x 64 per block (256 threads, 4 x 4 each), K chunk per blockIdx.y,
// partials summed in a fixed order by k_gram_reduce64.
constexpr int DT = 64;
constexpr int DK = 16;

__global__ void __launch_bounds__(256) k_gram_f64(const double* __restrict__ A, long lda, int m,
                                                  const double* __restrict__ B, long ldb, int n,
                                                  long K, long kchunk, double* __restrict__ part) {
  __shared__ double As[DK][DT + 1], Bs[DK][DT + 1];
  const int tid = threadIdx.x;
  const int ti = tid % 16, tj = tid / 16;
  const int i0 = blockIdx.x % ((m + DT - 1) / DT) * DT;
  const int j0 = blockIdx.x / ((m + DT - 1) / DT) * DT;
  const long k0 = (long)blockIdx.y * kchunk, k1 = min(K, k0 + kchunk);
  double acc[4][4] = {};
  for (long kb = k0; kb < k1; kb += DK) {
    for (int e = tid; e < DK * DT; e += 256) {
      const int kk = e % DK, r = e / DK;
      const long k = kb + kk;
      As[kk][r] = (i0 + r < m && k < k1) ? A[(long)(i0 + r) * lda + k] : 0.0;
      Bs[kk][r] = (j0 + r < n && k < k1) ? B[(long)(j0 + r) * ldb + k] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < DK; ++kk) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) { a[q] = As[kk][ti + 16 * q]; b[q] = Bs[kk][tj + 16 * q]; }
#pragma unroll
      for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
    }
    __syncthreads();
  }
  double* P = part + ((long)blockIdx.y * gridDim.x + blockIdx.x) * DT * DT;
#pragma unroll
  for (int x = 0; x < 4; ++x)
#pragma unroll
    for (int y = 0; y < 4; ++y) P[(tj + 16 * y) * DT + ti + 16 * x] = acc[x][y];
}

__global__ void k_gram_reduce64(const double* __restrict__ part, int nsplit, int ntile, int m,
                                int n, double alpha, double* __restrict__ C, long ldc) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)m * n) return;
  const int i = (int)(idx % m), j = (int)(idx / m);
  const int tiles_i = (m + DT - 1) / DT;
  const int t = (j / DT) * tiles_i + i / DT;
  double s = 0.0;
  for (int sp = 0; sp < nsplit; ++sp)
    s += part[((long)sp * ntile + t) * DT * DT + (j % DT) * DT + (i % DT)];
  C[(long)j * ldc + i] = alpha * s;
}

// Y[j][p] = sum_k X[k][p] Z(k,j); block = 128 points x 32 bands, 4 per thread in bands
__global__ void __launch_bounds__(256) k_rotate_f64(const double* __restrict__ X, long ldx,
                                                    long npts, int kin,
                                                    const double* __restrict__ Z, long ldz,
                                                    int nout, double* __restrict__ Y, long ldy) {
  __shared__ double Zs[32][33];
  const int tid = threadIdx.x;
  const long p = (long)blockIdx.x * 128 + (tid % 128);
  const int jg = tid / 128;  // 0..1
  const int j0 = blockIdx.y * 32;
  double acc[16] = {};
  for (int kb = 0; kb < kin; kb += 32) {
    for (int e = tid; e < 32 * 32; e += 256) {
      const int kk = e % 32, jj = e / 32;
      Zs[kk][jj] = (kb + kk < kin && j0 + jj < nout) ? Z[(long)(j0 + jj) * ldz + kb + kk] : 0.0;
    }
    __syncthreads();
    const int kn = min(32, kin - kb);
    if (p < npts)
      for (int kk = 0; kk < kn; ++kk) {
        const double x = X[(long)(kb + kk) * ldx + p];
#pragma unroll
        for (int q = 0; q < 16; ++q) acc[q] = fma(x, Zs[kk][jg * 16 + q], acc[q]);
      }
    __syncthreads();
  }
  if (p < npts)
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const int j = j0 + jg * 16 + q;
      if (j < nout) Y[(long)j * ldy + p] = acc[q];
    }
}

int check_tc_error(cudaStream_t st) {
  int h = 0;
  RS_CUDA(cudaMemcpyFromSymbolAsync(&h, g_tc_error, sizeof(int), 0, cudaMemcpyDeviceToHost, st));
  RS_CUDA(cudaStreamSynchronize(st));
  if (h) {
    int z = 0;
    cudaMemcpyToSymbolAsync(g_tc_error, &z, sizeof(int), 0, cudaMemcpyHostToDevice, st);
    return fail(RS_ECUDA, "tensor-core kernel: an mbarrier wait timed out");
  }
  return RS_OK;
}

}  // namespace

int gram_f32(int m, int n, long K, const float* A, long lda, const float* B, long ldb,
             double alpha, double* C, long ldc, int sym, cudaStream_t st) {
  if (m <= 0 || n <= 0) return RS_OK;
  if (K % 4 || lda % 4 || ldb % 4 ||
      ((uintptr_t)A | (uintptr_t)B) % 16)
    return fail(RS_EINVAL, "rs_gram_f32: K, lda, ldb must be multiples of 4, A/B 16-byte aligned");
  if (sym && (m != n || A != B)) sym = 0;
  const int tm = (m + GM - 1) / GM, tn = (n + GN - 1) / GN;
  const int npairs = sym ? tm * (tm + 1) / 2 : tm * tn;
  // about two CTAs' worth of work per SM, at least 4*DG stages per chunk
  long want = (296 + npairs - 1) / npairs;
  long kchunk = (K + want - 1) / want;
  kchunk = (kchunk + KB - 1) / KB * KB;
  if (kchunk < 4 * DG * KB) kchunk = 4 * DG * KB;
  long nsplit = (K + kchunk - 1) / kchunk;
  if (nsplit < 1) nsplit = 1;
  double* part = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * npairs * nsplit * GM * GN, st));
  const size_t smem = 2 * 4 * TILE_BYTES + 1024;
  RS_CUDA(cudaFuncSetAttribute(k_gram_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  dim3 grid(npairs, (unsigned)nsplit);
  k_gram_tf32x3<<<grid, GRAM_THREADS, smem, st>>>(A, lda, m, B, ldb, n, K, kchunk, sym, tm,
                                                  part);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) {
    k_gram_reduce<<<div_up((long)m * n, 256), 256, 0, st>>>(part, (int)nsplit, m, n, sym, tm,
                                                            alpha, C, ldc);
    e = cudaGetLastError();
  }
  cudaFreeAsync(part, st);
  if (e != cudaSuccess) return cuda_status(e, "k_gram_tf32x3");
  return check_tc_error(st);
}

int rotate_f32(long npts, int kin, int nout, const float* X, long ldx, const double* Z, long ldz,
               float* Y, long ldy, cudaStream_t st) {
  if (npts <= 0 || nout <= 0) return RS_OK;
  if (npts % 4 || ldx % 4 || (uintptr_t)X % 16)
    return fail(RS_EINVAL, "rs_rotate_f32: points and ldx must be multiples of 4");
  const int kpad = (kin + KB - 1) / KB * KB;
  const int npad = (nout + RN - 1) / RN * RN;
  float *zh = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&zh, sizeof(float) * 2 * (size_t)npad * kpad, st));
  float* zl = zh + (size_t)npad * kpad;
  k_split_z<<<div_up((long)npad * kpad, 256), 256, 0, st>>>(Z, ldz, kin, nout, kpad, zh, zl);
  const size_t smem = 2 * ROT_STAGE + 1024;
  RS_CUDA(cudaFuncSetAttribute(k_rotate_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  dim3 grid(div_up(npts, GM), div_up(nout, RN));
  k_rotate_tf32x3<<<grid, ROT_THREADS, smem, st>>>(X, ldx, npts, kin, zh, zl, kpad, nout, Y, ldy);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(zh, st);
  if (e != cudaSuccess) return cuda_status(e, "k_rotate_tf32x3");
  return check_tc_error(st);
}

int gram_f64(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
             double alpha, double* C, long ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0) return RS_OK;
  const int ti = (m + DT - 1) / DT, tj = (n + DT - 1) / DT;
  const int ntile = ti * tj;
  long kchunk = 8192;
  long nsplit = (K + kchunk - 1) / kchunk;
  if (nsplit < 1) nsplit = 1;
  while (nsplit * ntile > 65536 * 4) { kchunk *= 2; nsplit = (K + kchunk - 1) / kchunk; }
  double* part = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * nsplit * ntile * DT * DT, st));
  dim3 grid(ntile, (unsigned)nsplit);
  k_gram_f64<<<grid, 256, 0, st>>>(A, lda, m, B, ldb, n, K, kchunk, part);
  k_gram_reduce64<<<div_up((long)m * n, 256), 256, 0, st>>>(part, (int)nsplit, ntile, m, n,
                                                            alpha, C, ldc);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(part, st);
  if (e != cudaSuccess) return cuda_status(e, "k_gram_f64");
  return RS_OK;
}

int rotate_f64(long npts, int kin, int nout, const double* X, long ldx, const double* Z, long ldz,
               double* Y, long ldy, cudaStream_t st) {
  if (npts <= 0 || nout <= 0) return RS_OK;
  dim3 grid(div_up(npts, 128), div_up(nout, 32));
  k_rotate_f64<<<grid, 256, 0, st>>>(X, ldx, npts, kin, Z, ldz, nout, Y, ldy);
  RS_LAUNCH_CHECK("k_rotate_f64");
  return RS_OK;
}

}  // namespace rs

extern "C" int rs_gram_f32(int m, int n, long K, const float* A, long lda, const float* B,
                           long ldb, double alpha, double* C, long ldc, int sym, void* stream) {
  return rs::gram_f32(m, n, K, A, lda, B, ldb, alpha, C, ldc, sym, rs::as_stream(stream));
}
extern "C" int rs_gram_f64(int m, int n, long K, const double* A, long lda, const double* B,
                           long ldb, double alpha, double* C, long ldc, void* stream) {
  return rs::gram_f64(m, n, K, A, lda, B, ldb, alpha, C, ldc, rs::as_stream(stream));
}
extern "C" int rs_rotate_f32(long npts, int kin, int nout, const float* X, long ldx,
                             const double* Z, long ldz, float* Y, long ldy, void* stream) {
  return rs::rotate_f32(npts, kin, nout, X, ldx, Z, ldz, Y, ldy, rs::as_stream(stream));
}
extern "C" int rs_rotate_f64(long npts, int kin, int nout, const double* X, long ldx,
                             const double* Z, long ldz, double* Y, long ldy, void* stream) {
  return rs::rotate_f64(npts, kin, nout, X, ldx, Z, ldz, Y, ldy, rs::as_stream(stream));
}
