// gemm.cu -- subspace contractions of the Gram-Schmidt / Rayleigh-Ritz step.
//
//  * Gram matrices C = alpha A^T B (Psi^T H Psi, Psi^T S Psi): K = grid
//    points (millions), M, N = bands.
//  * Band rotations Y = X Z (Psi <- Psi C): K = bands.
//
// FP32 operands run on the 5th-generation tensor cores (tcgen05.mma,
// kind::tf32) with the 3xTF32 split: x = hi + lo with hi = tf32(x) and lo = x -
// hi, and A B ~ hi_A hi_B + hi_A lo_B + lo_A hi_B, accumulated in FP32 in
// TMEM.  The hi/lo pieces are packed once per call into operand blocks in
// the canonical tcgen05 layouts; a warp-specialised pipeline (bulk-copy
// producer, MMA issuer, drain warps) streams them through shared memory.
// Gram products split K into chunks whose partial tiles are summed in FP64
// in a fixed order.  FP64 operands (the plain FP64 drop-in path) go to cuBLAS
// DGEMM.
#include <cublas_v2.h>
#include <math.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <string>

#include "rs_common.cuh"
#include "tc_ptx.cuh"

namespace rs {
namespace {

using namespace tc;

constexpr int GM = 128;        // tile rows (MMA M)
constexpr int GN = 128;        // Gram tile cols (MMA N)
constexpr int KB = 32;         // K per stage: one 128-byte swizzle row of fp32

__device__ int g_tc_error;     // set when a bounded wait gives up

// Operands are packed once per call into 32 KB blocks (hi 16 KB | lo 16 KB,
// hi = tf32_rna(x), lo = x - hi, both exact in TF32) of 128 rows (MMA M or
// N) by 32 K values, in the canonical tcgen05 shared-memory layouts, so a
// pipeline stage is a plain bulk copy:
//  * K-major (Gram A and B, rotation Z): row r at byte r*128 with its 16-byte
//    chunk c stored at chunk c ^ (r mod 8) (SW128: 8-row atoms, SBO = 1 KB);
//  * MN-major (rotation X, points contiguous): see mnmaj_off.

// byte offset of (point p, band k) in the MN-major tile: each k-row holds 32
// points (128 B) whose 32-byte chunks are XOR-swizzled with (k mod 4);
// 4-row atoms (512 B) step along k (SBO = 512 B), 32-point blocks of 8
// atoms (4 KB) step along the points (LBO = 4 KB)
__device__ __forceinline__ uint32_t mnmaj_off(int p, int k) {
  return (uint32_t)((p >> 5) * 4096 + (k >> 2) * 512 + (k & 3) * 128 +
                    ((((p & 31) >> 3) ^ (k & 3)) << 5) + (p & 7) * 4);
}
// byte offset of (row r, K index k) in the K-major SW128 tile
__device__ __forceinline__ uint32_t kmaj_off(int r, int k) {
  return (uint32_t)(r * 128 + ((((k >> 2) ^ (r & 7))) << 4) + (k & 3) * 4);
}

// ------------------------------------------------------------------ pipeline
// Both tensor-core kernels run the same warp-specialised pipeline:
//  * warp 0 (one lane): producer -- keeps STAGES operand stages in flight
//    (bulk copies into shared memory, completion counted in bytes);
//  * warp 1 (one lane): issues the 12 MMAs of a stage (4 K-steps x 3 passes)
//    into one of TM_BUFS TMEM accumulators, DGRP stages per accumulator, and
//    commits them to the mbarriers that free the stage and hand the
//    accumulator to the drain warps;
//  * warps 2..: drain finished accumulators into registers (warp w reads
//    TMEM lanes 32*(w%4).. and a share of the 128 columns: a half in the
//    rotation, a quarter in the Gram, whose sums are (hi, lo) pairs) and
//    write the results.
// Every wait is bounded; a timeout raises a shared abort flag that winds all
// roles down, and the host sees g_tc_error.
constexpr int STAGES = 3;
constexpr int TM_BUFS = 4;
constexpr int DGRP = 2;
constexpr int NDRAIN = 256;                  // rotation: 8 drain warps, 64 columns each
constexpr int TC_THREADS = 64 + NDRAIN;
constexpr int GRAM_DRAIN = 512;              // Gram: 16 drain warps, 32 columns each
constexpr int GRAM_THREADS = 64 + GRAM_DRAIN;
constexpr int OPB = GM * KB * 4;      // one 128 x 32 FP32 operand tile: 16 KB
constexpr int STAGE_BYTES = 4 * OPB;  // a hi | a lo | b hi | b lo
constexpr size_t TC_SMEM = (size_t)STAGES * STAGE_BYTES + 1024;

struct PipeBars {
  uint64_t full[STAGES], empty[STAGES], tfull[TM_BUFS], tempty[TM_BUFS];
};

__device__ __forceinline__ void pipe_init(PipeBars& b, int ndrain) {
  for (int s = 0; s < STAGES; ++s) {
    mbar_init(&b.full[s], 1);
    mbar_init(&b.empty[s], 1);
  }
  for (int t = 0; t < TM_BUFS; ++t) {
    mbar_init(&b.tfull[t], 1);
    mbar_init(&b.tempty[t], ndrain);
  }
}

// untiled bulk copy global -> this CTA's shared memory (16-byte aligned, size
// a multiple of 16), completion counted on *bar
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes,
                                          uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n"
      ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// The MMA role for one stage: 3xTF32 over K = 32 into accumulator d.
// a_mn / b_mn select the MN-major layout for the operand (descriptor type 1,
// LBO 4 KB, SBO 512 B, K-steps 1 KB apart) instead of K-major SW128.
template <bool A_MN>
__device__ __forceinline__ void issue_stage(uint32_t d, uint32_t ahi, uint32_t alo, uint32_t bhi,
                                            uint32_t blo, uint32_t idesc, bool first) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    uint64_t dah, dal;
    if (A_MN) {
      dah = smem_desc_sw128_b32(ahi + q * 1024, 4096, 512);
      dal = smem_desc_sw128_b32(alo + q * 1024, 4096, 512);
    } else {
      dah = smem_desc_sw128(ahi + q * 32, 16, 1024);
      dal = smem_desc_sw128(alo + q * 32, 16, 1024);
    }
    const uint64_t dbh = smem_desc_sw128(bhi + q * 32, 16, 1024);
    const uint64_t dbl = smem_desc_sw128(blo + q * 32, 16, 1024);
    mma_tf32(d, dal, dbh, idesc, (first && q == 0) ? 0u : 1u);
    mma_tf32(d, dah, dbl, idesc, 1);
    mma_tf32(d, dah, dbh, idesc, 1);
  }
}

// ------------------------------------------------------------------ operand pieces
// Rows of K values (stride ld) -> 32 KB blocks [row tile][k block] of hi | lo
// in the K-major layout (row = band), for the K range [k0, k0 + nkb*32) cut
// at K, zero beyond `rows` and K.  One CTA per block, 256 threads, 4 float4
// each: 8 threads read one 128-byte row piece.
__global__ void __launch_bounds__(256) k_tile_rows(const float* __restrict__ x, long ld, int rows,
                                                   long k0, long K, int nkb,
                                                   char* __restrict__ out) {
  const long blk = blockIdx.x;
  const int rt = (int)(blk / nkb), kb = (int)(blk % nkb);
  char* hi = out + blk * (2 * OPB);
  char* lo = hi + OPB;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int f = threadIdx.x + 256 * i;
    const int r = f >> 3, c4 = f & 7;
    const int row = rt * GM + r;
    const long k = k0 + (long)kb * KB + 4 * c4;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (row < rows && k < K) v = __ldg(reinterpret_cast<const float4*>(x + (long)row * ld + k));
    float4 h, l;
    h.x = tf32_rna(v.x); l.x = v.x - h.x;
    h.y = tf32_rna(v.y); l.y = v.y - h.y;
    h.z = tf32_rna(v.z); l.z = v.z - h.z;
    h.w = tf32_rna(v.w); l.w = v.w - h.w;
    const uint32_t off = kmaj_off(r, 4 * c4);
    *reinterpret_cast<float4*>(hi + off) = h;
    *reinterpret_cast<float4*>(lo + off) = l;
  }
}

// X (kin rows of npts points, stride ldx) -> 32 KB blocks [point tile][k block]
// of hi | lo in the MN-major layout, zero beyond kin and npts.  One CTA per
// block, 256 threads, 4 float4 each.
__global__ void __launch_bounds__(256) k_tile_x(const float* __restrict__ X, long ldx, long npts,
                                                int kin, int nkb, char* __restrict__ xt) {
  const long blk = blockIdx.x;
  const long pt = blk / nkb;
  const int kb = (int)(blk % nkb);
  char* hi = xt + blk * (2 * OPB);
  char* lo = hi + OPB;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const int f = threadIdx.x + 256 * i;  // k = f / 32, points 4 (f % 32) ..
    const int kk = f >> 5, p4 = 4 * (f & 31);
    const int k = kb * KB + kk;
    const long p = pt * GM + p4;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (k < kin && p < npts) v = __ldg(reinterpret_cast<const float4*>(X + (long)k * ldx + p));
    float4 h, l;
    h.x = tf32_rna(v.x); l.x = v.x - h.x;
    h.y = tf32_rna(v.y); l.y = v.y - h.y;
    h.z = tf32_rna(v.z); l.z = v.z - h.z;
    h.w = tf32_rna(v.w); l.w = v.w - h.w;
    const uint32_t off = mnmaj_off(p4, kk);
    *reinterpret_cast<float4*>(hi + off) = h;
    *reinterpret_cast<float4*>(lo + off) = l;
  }
}

// Z (FP64, column-major kin x nout) -> 32 KB blocks [band tile][k block] of
// hi | lo in the K-major layout (row = output band j), zero beyond kin, nout.
__global__ void __launch_bounds__(256) k_tile_z(const double* __restrict__ Z, long ldz, int kin,
                                                int nout, int nkb, char* __restrict__ zt) {
  const long blk = blockIdx.x;
  const int jt = (int)(blk / nkb), kb = (int)(blk % nkb);
  char* hi = zt + blk * (2 * OPB);
  char* lo = hi + OPB;
  for (int e = threadIdx.x; e < GM * KB; e += 256) {
    const int kk = e % KB, jj = e / KB;
    const int k = kb * KB + kk, j = jt * GM + jj;
    const float z = (k < kin && j < nout) ? (float)Z[(long)j * ldz + k] : 0.f;
    const float h = tf32_rna(z);
    const uint32_t off = kmaj_off(jj, kk);
    *reinterpret_cast<float*>(hi + off) = h;
    *reinterpret_cast<float*>(lo + off) = z - h;
  }
}


// ------------------------------------------------------------------ Gram
// FP64 partial tiles P[pair][split][j][i] = sum_{k in chunk} A[i][k] B[j][k]
// for one 128 x 128 tile pair and one K chunk.  The product runs over K in
// pieces: each piece of A and B is first packed into hi | lo blocks
// (k_tile_rows), so a stage is two 32 KB bulk copies of contiguous memory.
// The tensor core accumulates DGRP stages (64 K terms, 3 passes) in FP32 in
// one TMEM accumulator; the drain warps fold each finished accumulator into
// compensated (hi, lo) FP32 register pairs while the next ones fill, so long
// sums never build up in plain FP32.  A diagonal pair of a symmetric product
// loads its block once.
// Compensated FP32 accumulation: (hi, lo) += x with TwoSum (Knuth), so that
// hi + lo carries the running sum to about 44 bits without FP64 conversions
// in the loop (the library is built without contraction, so the six
// additions run exactly as written).
__device__ __forceinline__ void two_sum_acc(float& hi, float& lo, float x) {
  const float s = hi + x;
  const float bp = s - hi;
  const float ap = s - bp;
  lo += (hi - ap) + (x - bp);
  hi = s;
}
__device__ __forceinline__ void drain_f64(uint32_t taddr, float* hi, float* lo) {
#pragma unroll
  for (int c = 0; c < 32; c += 16) {
    uint32_t r[16];
    tmem_ld16(taddr + c, r);
    tmem_ld_wait();
#pragma unroll
    for (int k = 0; k < 16; ++k) two_sum_acc(hi[c + k], lo[c + k], __uint_as_float(r[k]));
  }
}

// grid (pairs, splits of this piece); the CTA's partial goes to split column
// split0 + blockIdx.y of nsplit_total
__global__ void __launch_bounds__(GRAM_THREADS, 1)
    k_gram_tf32x3(const char* __restrict__ at, const char* __restrict__ bt, int nkb, int kbc,
                  int sym, int tn, int split0, int nsplit_total, double* __restrict__ part) {
  extern __shared__ __align__(1024) char smem_dyn[];
  char* smem = (char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) PipeBars bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
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
  const bool same = sym == 1 && it == jt;  // one block serves both operands
  const int kb0 = blockIdx.y * kbc;
  const int nst = max(0, min(nkb, kb0 + kbc) - kb0);
  const int ngrp = (nst + DGRP - 1) / DGRP;
  const char* ablk = at + ((long)it * nkb + kb0) * (2L * OPB);
  const char* bblk = bt + ((long)jt * nkb + kb0) * (2L * OPB);

  if (warp == 2) tmem_alloc(&tmem_base, TM_BUFS * GN);
  if (tid == 0) {
    pipe_init(bar, GRAM_DRAIN);
    abort_flag = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 2) tmem_relinquish();
  const uint32_t tmem = tmem_base;
  bool bad = false;

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    if ((tid & 31) == 0 && nst > 0) {
      const uint32_t tx = same ? 2 * OPB : 4 * OPB;
      int kb = 0;
      for (; kb < nst; ++kb) {
        const int s = kb % STAGES;
        if (kb >= STAGES &&
            !mbar_wait_or_abort(&bar.empty[s], (kb / STAGES - 1) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        char* st = smem + s * STAGE_BYTES;
        mbar_arrive_expect_tx(&bar.full[s], tx);
        bulk_load(st, ablk + (long)kb * (2 * OPB), 2 * OPB, &bar.full[s]);
        if (!same) bulk_load(st + 2 * OPB, bblk + (long)kb * (2 * OPB), 2 * OPB, &bar.full[s]);
      }
      // nothing may still write this CTA's shared memory when it exits
      for (int j = max(0, kb - STAGES); j < kb; ++j)
        if (!mbar_wait(&bar.full[j % STAGES], (j / STAGES) & 1)) bad = true;
      if (bad) abort_flag = 1;
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issue
    if ((tid & 31) == 0 && nst > 0) {
      constexpr uint32_t idesc = idesc_tf32(GM, GN, 0, 0);
      int kb = 0;
      for (; kb < nst; ++kb) {
        const int s = kb % STAGES, g = kb / DGRP, tb = g % TM_BUFS;
        if (kb % DGRP == 0 && g >= TM_BUFS &&
            !mbar_wait_or_abort(&bar.tempty[tb], (g / TM_BUFS - 1) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        if (!mbar_wait_or_abort(&bar.full[s], (kb / STAGES) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * STAGE_BYTES);
        const uint32_t sb = same ? sa : sa + 2 * OPB;
        issue_stage<false>(tmem + tb * GN, sa, sa + OPB, sb, sb + OPB, idesc, kb % DGRP == 0);
        mma_commit(&bar.empty[s]);
        if (kb % DGRP == DGRP - 1 || kb == nst - 1) mma_commit(&bar.tfull[tb]);
      }
      // no MMA may still run when the CTA exits
      if (kb > 0 && !mbar_wait(&bar.empty[(kb - 1) % STAGES], ((kb - 1) / STAGES) & 1))
        bad = true;
      if (bad) abort_flag = 1;
    }
  } else {
    // ---------------------------------------------------------- drain
    const int dq = warp & 3, dc = (warp - 2) >> 2;  // lane quadrant, column quarter
    const uint32_t dlane = (uint32_t)(dq * 32) << 16;
    float ahi[32], alo[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) ahi[k] = alo[k] = 0.f;
    for (int g = 0; g < ngrp; ++g) {
      const int tb = g % TM_BUFS;
      const bool ok = mbar_wait_or_abort(&bar.tfull[tb], (g / TM_BUFS) & 1, &abort_flag);
      if (__any_sync(0xffffffffu, !ok)) { bad = true; break; }
      tc_fence_after();
      drain_f64(tmem + tb * GN + dc * 32 + dlane, ahi, alo);
      tc_fence_before();
      mbar_arrive(&bar.tempty[tb]);
    }
    if (!bad) {
      double* P = part + ((long)blockIdx.x * nsplit_total + split0 + blockIdx.y) * GM * GN;
      const int row = dq * 32 + (tid & 31);
#pragma unroll
      for (int k = 0; k < 32; ++k)
        P[(long)(dc * 32 + k) * GM + row] = (double)ahi[k] + (double)alo[k];
    }
  }
  tc_fence_before();
  __syncthreads();
  if (bad || abort_flag) {
    if (tid == 64) atomicExch(&g_tc_error, 1);
  }
  if (warp == 2) tmem_dealloc(tmem, TM_BUFS * GN);
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
// Y[j][p] = sum_k X[k][p] Z(k, j).  The contraction is bound by operand
// delivery from L2 (about 9.5 TB/s into all SMs at 48 flop per byte), so a
// CTA computes two 128 x 128 output tiles at once: one 128-point block of X
// against two 128-band blocks of Z.  A stage is three 32 KB bulk copies,
// X hi | lo (MN-major) and the two Z hi | lo (K-major), fed to 6 MMAs per
// K step, 64 flop per byte.  Each CTA walks tile pairs t = blockIdx.x,
// blockIdx.x + gridDim.x, ... (band pair fastest, so the CTAs sharing an X
// block run together and read it from HBM once); an odd last band tile
// runs alone.  Two TMEM buffers, each two accumulators of 128 columns: the
// MMA warp fills one while the drain warps fold the other into FP32
// registers (DGRP stages per accumulator, as in the Gram), so the producer
// and the MMA warp run ahead into the next pair while the last one drains.
constexpr int RSTAGES = 2;
constexpr int RSTAGE_BYTES = 6 * OPB;
constexpr size_t ROT_SMEM = (size_t)RSTAGES * RSTAGE_BYTES + 1024;

struct RotBars {
  uint64_t full[RSTAGES], empty[RSTAGES], tfull[2], tempty[2];
};

__device__ __forceinline__ void drain_f32(uint32_t taddr, float* acc) {
#pragma unroll
  for (int c = 0; c < 64; c += 16) {
    uint32_t r[16];
    tmem_ld16(taddr + c, r);
    tmem_ld_wait();
#pragma unroll
    for (int k = 0; k < 16; ++k) acc[c + k] += __uint_as_float(r[k]);
  }
}

__global__ void __launch_bounds__(TC_THREADS, 1)
    k_rotate_tf32x3(const char* __restrict__ xt, const char* __restrict__ zt, long npts, int nkb,
                    int nout, int ntn, long ntiles, float* __restrict__ Y, long ldy) {
  extern __shared__ __align__(1024) char smem_dyn[];
  char* smem = (char*)(((uintptr_t)smem_dyn + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) RotBars bar;
  __shared__ uint32_t tmem_base;
  __shared__ volatile int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int npr = (ntn + 1) / 2;  // band-tile pairs
  const int ngrp = (nkb + DGRP - 1) / DGRP;
  const long mytiles = ntiles > blockIdx.x ? (ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

  if (warp == 2) tmem_alloc(&tmem_base, 4 * GN);
  if (tid == 0) {
    for (int q = 0; q < RSTAGES; ++q) {
      mbar_init(&bar.full[q], 1);
      mbar_init(&bar.empty[q], 1);
    }
    for (int q = 0; q < 2; ++q) {
      mbar_init(&bar.tfull[q], 1);
      mbar_init(&bar.tempty[q], NDRAIN);
    }
    abort_flag = 0;
    fence_mbar_init();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 2) tmem_relinquish();
  const uint32_t tmem = tmem_base;
  bool bad = false;
  const long nstage = mytiles * nkb;

  if (warp == 0) {
    // ---------------------------------------------------------- producer
    if ((tid & 31) == 0) {
      long c = 0;
      for (; c < nstage && !bad; ++c) {
        const long t = blockIdx.x + (c / nkb) * gridDim.x;
        const int kb = (int)(c % nkb);
        const long pt = t / npr;
        const int j1 = 2 * (int)(t % npr);
        const bool two = j1 + 1 < ntn;
        const int s = (int)(c % RSTAGES);
        if (c >= RSTAGES &&
            !mbar_wait_or_abort(&bar.empty[s], (int)(c / RSTAGES - 1) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        char* st = smem + s * RSTAGE_BYTES;
        mbar_arrive_expect_tx(&bar.full[s], (two ? 6 : 4) * OPB);
        bulk_load(st, xt + (pt * nkb + kb) * (2L * OPB), 2 * OPB, &bar.full[s]);
        bulk_load(st + 2 * OPB, zt + ((long)j1 * nkb + kb) * (2L * OPB), 2 * OPB, &bar.full[s]);
        if (two)
          bulk_load(st + 4 * OPB, zt + ((long)(j1 + 1) * nkb + kb) * (2L * OPB), 2 * OPB,
                    &bar.full[s]);
      }
      for (long j = max(0L, c - RSTAGES); j < c; ++j)
        if (!mbar_wait(&bar.full[j % RSTAGES], (int)(j / RSTAGES) & 1)) bad = true;
      if (bad) abort_flag = 1;
    }
  } else if (warp == 1) {
    // ---------------------------------------------------------- MMA issue
    if ((tid & 31) == 0) {
      constexpr uint32_t idesc = idesc_tf32(GM, GN, 1, 0);
      long c = 0;
      for (; c < nstage; ++c) {
        const long t = blockIdx.x + (c / nkb) * gridDim.x;
        const bool two = 2 * (int)(t % npr) + 1 < ntn;
        const int kb = (int)(c % nkb);
        const long G = (c / nkb) * ngrp + kb / DGRP;  // accumulator group, over all pairs
        const int tb = (int)(G & 1), s = (int)(c % RSTAGES);
        if (kb % DGRP == 0 && G >= 2 &&
            !mbar_wait_or_abort(&bar.tempty[tb], (int)(G / 2 - 1) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        if (!mbar_wait_or_abort(&bar.full[s], (int)(c / RSTAGES) & 1, &abort_flag)) {
          bad = true;
          break;
        }
        tc_fence_after();
        const uint32_t sa = smem_u32(smem + s * RSTAGE_BYTES);
        const bool first = kb % DGRP == 0;
        issue_stage<true>(tmem + (2 * tb) * GN, sa, sa + OPB, sa + 2 * OPB, sa + 3 * OPB, idesc,
                          first);
        if (two)
          issue_stage<true>(tmem + (2 * tb + 1) * GN, sa, sa + OPB, sa + 4 * OPB, sa + 5 * OPB,
                            idesc, first);
        mma_commit(&bar.empty[s]);
        if (kb % DGRP == DGRP - 1 || kb == nkb - 1) mma_commit(&bar.tfull[tb]);
      }
      if (c > 0 && !mbar_wait(&bar.empty[(c - 1) % RSTAGES], (int)((c - 1) / RSTAGES) & 1))
        bad = true;
      if (bad) abort_flag = 1;
    }
  } else {
    // ---------------------------------------------------------- drain + store
    const int dq = warp & 3, dh = (warp - 2) >> 2;
    const uint32_t dlane = (uint32_t)(dq * 32) << 16;
    long G = 0;
    for (long i = 0; i < mytiles && !bad; ++i) {
      const long t = blockIdx.x + i * gridDim.x;
      const long p = (t / npr) * GM + dq * 32 + (tid & 31);
      const int j1 = 2 * (int)(t % npr);
      const bool two = j1 + 1 < ntn;
      float acc1[64], acc2[64];
#pragma unroll
      for (int k = 0; k < 64; ++k) acc1[k] = acc2[k] = 0.f;
      for (int g = 0; g < ngrp; ++g, ++G) {
        const int tb = (int)(G & 1);
        const bool ok = mbar_wait_or_abort(&bar.tfull[tb], (int)(G / 2) & 1, &abort_flag);
        if (__any_sync(0xffffffffu, !ok)) { bad = true; break; }
        tc_fence_after();
        drain_f32(tmem + (2 * tb) * GN + dh * 64 + dlane, acc1);
        if (two) drain_f32(tmem + (2 * tb + 1) * GN + dh * 64 + dlane, acc2);
        tc_fence_before();
        mbar_arrive(&bar.tempty[tb]);
      }
      if (!bad && p < npts) {
        const int b1 = j1 * GN + dh * 64, b2 = b1 + GN;
#pragma unroll
        for (int k = 0; k < 64; ++k)
          if (b1 + k < nout) Y[(long)(b1 + k) * ldy + p] = acc1[k];
        if (two) {
#pragma unroll
          for (int k = 0; k < 64; ++k)
            if (b2 + k < nout) Y[(long)(b2 + k) * ldy + p] = acc2[k];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (bad || abort_flag) {
    if (tid == 64) atomicExch(&g_tc_error, 1);
  }
  if (warp == 2) tmem_dealloc(tmem, 4 * GN);
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

// K split of the Gram product: one CTA per SM runs (pairs x splits) CTAs in
// whole waves where it can, with chunks of at least 8 stages.
long gram_splits(int npairs, long K) {
  const long nsm = 148;
  const long maxsplit = max(1L, K / (8L * KB));
  long best = 1;
  double best_eff = -1.0;
  for (long w = 1; w <= 8; ++w) {
    const long ns = min(maxsplit, max(1L, w * nsm / npairs));
    const long ctas = (long)npairs * ns;
    const long waves = (ctas + nsm - 1) / nsm;
    const double eff = (double)ctas / (double)(waves * nsm);
    if (eff > best_eff + 1e-3) { best_eff = eff; best = ns; }
    if (ns == maxsplit) break;
  }
  return best;
}

int gram_f32(int m, int n, long K, const float* A, long lda, const float* B, long ldb,
             double alpha, double* C, long ldc, int sym, cudaStream_t st) {
  if (m <= 0 || n <= 0) return RS_OK;
  if (K % 4 || lda % 4 || ldb % 4 || ((uintptr_t)A | (uintptr_t)B) % 16)
    return fail(RS_EINVAL, "rs_gram_f32: K, lda, ldb must be multiples of 4, A/B 16-byte aligned");
  if (K <= 0 || lda < K || ldb < K)
    return fail(RS_EINVAL, "rs_gram_f32: K must be positive and at most lda, ldb");
  // sym 1: A == B, one triangle, diagonal blocks loaded once; sym 2: the
  // lower-triangle tile pairs of a product known to be symmetric (A != B)
  if (sym == 1 && (m != n || A != B || lda != ldb)) sym = 0;
  if (sym == 2 && m != n) sym = 0;
  const bool shared = sym == 1;
  keep_pool_memory();
  const int tm = (m + GM - 1) / GM, tn = (n + GN - 1) / GN;
  const int npairs = sym ? tm * (tm + 1) / 2 : tm * tn;
  // K pieces of at most 2^19 values bound the packed copies (2 x 2^19 x 8 B
  // per band); each piece runs in whole waves of K splits
  const long piece = min(K, 1L << 19);
  const long npieces = (K + piece - 1) / piece;
  const int nkb = (int)((piece + KB - 1) / KB);
  const int ns = (int)gram_splits(npairs, piece);
  const int kbc = (nkb + ns - 1) / ns;
  const int nsplit = (int)npieces * ns;
  const size_t abytes = (size_t)tm * nkb * 2 * OPB,
               bbytes = shared ? 0 : (size_t)tn * nkb * 2 * OPB;
  char* at = nullptr;
  double* part = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&at, abytes + bbytes, st));
  cudaError_t e = cudaMallocAsync((void**)&part, sizeof(double) * npairs * nsplit * GM * GN, st);
  if (e != cudaSuccess) {
    cudaFreeAsync(at, st);
    return cuda_status(e, "rs_gram_f32: work arrays");
  }
  char* bt = shared ? at : at + abytes;
  e = cudaFuncSetAttribute(k_gram_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)TC_SMEM);
  for (long pc = 0; pc < npieces && e == cudaSuccess; ++pc) {
    const long k0 = pc * piece;
    k_tile_rows<<<(unsigned)(tm * nkb), 256, 0, st>>>(A, lda, m, k0, K, nkb, at);
    if (!shared) k_tile_rows<<<(unsigned)(tn * nkb), 256, 0, st>>>(B, ldb, n, k0, K, nkb, bt);
    dim3 grid(npairs, ns);
    k_gram_tf32x3<<<grid, GRAM_THREADS, TC_SMEM, st>>>(at, bt, nkb, kbc, sym, tm, (int)pc * ns,
                                                       nsplit, part);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) {
    k_gram_reduce<<<div_up((long)m * n, 256), 256, 0, st>>>(part, nsplit, m, n, sym, tm, alpha,
                                                            C, ldc);
    e = cudaGetLastError();
  }
  cudaFreeAsync(part, st);
  cudaFreeAsync(at, st);
  if (e != cudaSuccess) return cuda_status(e, "k_gram_tf32x3");
  return check_tc_error(st);
}

// Y may be X (same layout, nout <= kin): X is read only by the packing pass,
// which completes before the product writes Y.
int rotate_f32(long npts, int kin, int nout, const float* X, long ldx, const double* Z, long ldz,
               float* Y, long ldy, cudaStream_t st) {
  if (npts <= 0 || nout <= 0) return RS_OK;
  if (npts % 4 || ldx % 4 || (uintptr_t)X % 16)
    return fail(RS_EINVAL, "rs_rotate_f32: points and ldx must be multiples of 4");
  if (kin <= 0 || ldx < npts) return fail(RS_EINVAL, "rs_rotate_f32: bad kin or ldx");
  keep_pool_memory();
  const int nkb = (kin + KB - 1) / KB;
  const long npt = div_up(npts, GM);
  const int ntn = (nout + GN - 1) / GN;
  char* xt = nullptr;
  char* zt = nullptr;
  const size_t xbytes = (size_t)npt * nkb * 2 * OPB, zbytes = (size_t)ntn * nkb * 2 * OPB;
  RS_CUDA(cudaMallocAsync((void**)&xt, xbytes + zbytes, st));
  zt = xt + xbytes;
  k_tile_x<<<(unsigned)(npt * nkb), 256, 0, st>>>(X, ldx, npts, kin, nkb, xt);
  k_tile_z<<<(unsigned)(ntn * nkb), 256, 0, st>>>(Z, ldz, kin, nout, nkb, zt);
  cudaError_t e = cudaFuncSetAttribute(k_rotate_tf32x3,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ROT_SMEM);
  if (e == cudaSuccess) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const long ntiles = npt * ((ntn + 1) / 2);  // (point tile, band-tile pair)
    const long nblk = min(ntiles, (long)nsm);
    k_rotate_tf32x3<<<(unsigned)nblk, TC_THREADS, ROT_SMEM, st>>>(xt, zt, npts, nkb, nout, ntn,
                                                                  ntiles, Y, ldy);
    e = cudaGetLastError();
  }
  cudaFreeAsync(xt, st);
  if (e != cudaSuccess) return cuda_status(e, "k_rotate_tf32x3");
  return check_tc_error(st);
}

// ------------------------------------------------------------------ FP64
// The plain FP64 path (the drop-in baseline) runs its subspace products as
// library DGEMMs: one cuBLAS handle per device, bound to the caller's stream
// for each call.  cuBLAS is deterministic run to run; its sums are not the
// oracle's order, so these products are checked to 1e-12, not bit for bit.
cublasHandle_t cublas_handle() {
  static std::mutex mu;
  static std::map<int, cublasHandle_t> handles;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto it = handles.find(dev);
  if (it != handles.end()) return it->second;
  cublasHandle_t h = nullptr;
  if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return nullptr;
  handles[dev] = h;
  return h;
}

int cublas_status(cublasStatus_t s, const char* what) {
  if (s == CUBLAS_STATUS_SUCCESS) return RS_OK;
  return fail(RS_ECUDA, std::string(what) + ": cuBLAS status " + std::to_string((int)s));
}

int gram_f64_beta(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
                  double alpha, double beta, double* C, long ldc, cudaStream_t st);

// C[i + j*ldc] = alpha sum_k A[i*lda + k] B[j*ldb + k]  (C = alpha A B^T)
int gram_f64(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
             double alpha, double* C, long ldc, cudaStream_t st) {
  return gram_f64_beta(m, n, K, A, lda, B, ldb, alpha, 0.0, C, ldc, st);
}

// C = alpha A^T B + beta C (the same operand layout as gram_f64)
int gram_f64_beta(int m, int n, long K, const double* A, long lda, const double* B, long ldb,
                  double alpha, double beta, double* C, long ldc, cudaStream_t st) {
  if (m <= 0 || n <= 0) return RS_OK;
  if (K > INT32_MAX || lda > INT32_MAX || ldb > INT32_MAX)
    return fail(RS_EINVAL, "rs_gram_f64: K and leading dimensions must fit in 32 bits");
  keep_pool_memory();
  cublasHandle_t h = cublas_handle();
  if (!h) return fail(RS_ECUDA, "rs_gram_f64: cublasCreate failed");
  int rc = cublas_status(cublasSetStream(h, st), "rs_gram_f64");
  if (!rc)
    rc = cublas_status(cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, m, n, (int)K, &alpha, A,
                                   (int)lda, B, (int)ldb, &beta, C, (int)ldc),
                       "rs_gram_f64");
  return rc;
}

// Y[j*ldy + p] = sum_k X[k*ldx + p] Z[j*ldz + k]  (Y = X Z, column-major)
int rotate_f64(long npts, int kin, int nout, const double* X, long ldx, const double* Z, long ldz,
               double* Y, long ldy, cudaStream_t st) {
  if (npts <= 0 || nout <= 0) return RS_OK;
  if (npts > INT32_MAX || ldx > INT32_MAX || ldy > INT32_MAX)
    return fail(RS_EINVAL, "rs_rotate_f64: sizes must fit in 32 bits");
  cublasHandle_t h = cublas_handle();
  if (!h) return fail(RS_ECUDA, "rs_rotate_f64: cublasCreate failed");
  int rc = cublas_status(cublasSetStream(h, st), "rs_rotate_f64");
  const double one = 1.0, zero = 0.0;
  if (!rc)
    rc = cublas_status(cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)npts, nout, kin, &one, X,
                                   (int)ldx, Z, (int)ldz, &zero, Y, (int)ldy),
                       "rs_rotate_f64");
  return rc;
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
