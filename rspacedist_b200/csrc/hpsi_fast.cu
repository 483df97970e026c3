// hpsi_fast.cu -- FP32 H*psi for the mixed-precision path, in two kernels:
//
// 1. k_stencil_f32_zmarch: (-1/2 lap + veff) psi.  One CTA owns a 64 x 32
//    tile of an xy plane of one band and marches along z.  Each thread holds
//    a 4(x) x 2(y) block of points:
//      * the nine planes z-4..z+4 of its block sit in a register queue, so
//        the z terms need no shared memory;
//      * whole planes (own blocks plus a 4-point halo) are copied into an
//        8-slot shared ring with cp.async, 3 planes ahead of the queue's
//        newest plane, so HBM latency is hidden without spending registers;
//        x terms read 2 float4 per row, y terms 8 float4 for both rows, and
//        one __syncthreads per plane protects slot reuse.
//    Tiles of one band are adjacent in launch order, so halo rows come from
//    L2 (loaded by the neighbouring tiles), and psi crosses HBM once.
// 2. k_nl_rmw_f32: the nonlocal D term on the points inside at least one
//    projector support (a fraction of the grid).  A thread owns one such
//    point and a block of 16 bands: it loads the point's projector entries
//    once and adds sum_e sum_j t[atom_e][b][j] p_e[j] to 16 bands of hpsi.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>

#include "rs_common.cuh"
#include "stencil.cuh"
#include "tc_ptx.cuh"

namespace rs {

template <class T, int MODE>
int launch_gather(const rs_geom* g, const double* mat, const double* rp, const T* psi,
                  const T* veff, T* out, int nb, cudaStream_t st);

namespace {

constexpr int TX = 64;
constexpr int TY = 32;
constexpr int NTX = TX / 4;
constexpr int NTY = TY / 2;
constexpr int NTHREADS = NTX * NTY;  // 256
constexpr int HX = TX + 8;
constexpr int HY = TY + 8;
constexpr int NL_BANDS = 16;

struct StArgs {
  int nx, ny, nz, zchunk, ntx, nty;
  float cx[5], cy[5], cz[5], c0;
  const float* psi;
  float* out;
  const float* veff;
  // Hartree form only: skip the launch when *done is set, and write this
  // CTA's share of psi . out to part[blockIdx.x]
  const int* done;
  double* part;
};

__device__ __forceinline__ int wrap_once(int i, int n) {
  return i < 0 ? i + n : (i >= n ? i - n : i);
}
__device__ __forceinline__ float4 ld4(const float* p) {
  return __ldg(reinterpret_cast<const float4*>(p));
}
__device__ __forceinline__ float4 zero4() { return make_float4(0.f, 0.f, 0.f, 0.f); }


// 16-byte asynchronous global->shared copies (cp.async, L2 only)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

constexpr int RING = 8;    // staged planes (halo'd) in shared memory
constexpr int AHEAD = 3;   // planes in flight beyond the queue's newest plane

// HARTREE: the Hartree operator of the mixed CG, A p with diagonal c0 and
// no veff, plus the p . A p partial of the CTA (one band).
template <bool HARTREE>
__global__ void __launch_bounds__(NTHREADS, 2) k_stencil_f32_zmarch(StArgs a) {
  if (HARTREE && *a.done) return;
  extern __shared__ __align__(16) float smem_raw[];
  float (*pl)[HY][HX] = reinterpret_cast<float (*)[HY][HX]>(smem_raw);  // [RING][HY][HX]
  const int tid = threadIdx.x;
  const int tx = tid % NTX, ty = tid / NTX;
  const int ntile = a.ntx * a.nty;
  const int tile = blockIdx.x % ntile;
  const int zc = blockIdx.x / ntile;
  const int band = blockIdx.y;
  const int x0 = (tile % a.ntx) * TX, y0 = (tile / a.ntx) * TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long plane = (long)nx * ny;
  const long N = plane * nz;
  const float* psi = a.psi + (long)band * N;
  float* out = a.out + (long)band * N;
  const int zs = zc * a.zchunk;
  const int ze = min(zs + a.zchunk, nz);
  const int gx = x0 + 4 * tx, gy = y0 + 2 * ty;
  const bool active = gx < nx && gy < ny;  // nx % 4 == 0, ny even
  const int w = min(TX, nx - x0), hgt = min(TY, ny - y0);
  const long own0 = (long)gy * nx + gx, own1 = own0 + nx;
  const int lx = 4 * tx + 4, ly = 2 * ty + 4;

  // the halo float4 this thread stages for every plane (or none)
  int h_src = -1, h_row = 0, h_col = 0;
  if (tid < 2 * TY) {
    const int side = tid / TY, r = tid % TY;
    if (r < hgt) {
      const int xs = side == 0 ? wrap_once(x0 - 4, nx) : wrap_once(x0 + w, nx);
      h_src = (y0 + r) * nx + xs;
      h_row = r + 4;
      h_col = side == 0 ? 0 : w + 4;
    }
  } else if (tid < 2 * TY + 8 * NTX) {
    const int j = tid - 2 * TY;
    const int c = j % NTX, rr = (j / NTX) % 4, side = j / (4 * NTX);
    if (4 * c < w) {
      const int ys = side == 0 ? wrap_once(y0 - 4 + rr, ny) : wrap_once(y0 + hgt + rr, ny);
      h_src = ys * nx + x0 + 4 * c;
      h_row = side == 0 ? rr : hgt + 4 + rr;
      h_col = 4 + 4 * c;
    }
  }
  auto plane_ptr = [&](int z) { return psi + (long)wrap_once(z, nz) * plane; };
  // one commit group per plane: this thread's own rows and its halo piece
  auto stage = [&](int z) {
    const float* pp = plane_ptr(z);
    float(*sl)[HX] = pl[z & (RING - 1)];
    if (active) {
      cp_async16(&sl[ly][lx], pp + own0);
      cp_async16(&sl[ly + 1][lx], pp + own1);
    }
    if (h_src >= 0) cp_async16(&sl[h_row][h_col], pp + h_src);
    cp_commit();
  };

  float4 q[9][2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const float* pp = plane_ptr(zs - 4 + k);
    q[k][0] = active ? ld4(pp + own0) : zero4();
    q[k][1] = active ? ld4(pp + own1) : zero4();
  }
#pragma unroll
  for (int k = 0; k < 4 + AHEAD; ++k) stage(zs + k);
  cp_wait<AHEAD>();
  __syncthreads();
#pragma unroll
  for (int k = 4; k < 8; ++k) {
    const float(*sl)[HX] = pl[(zs + k - 4) & (RING - 1)];
    q[k][0] = *reinterpret_cast<const float4*>(&sl[ly][lx]);
    q[k][1] = *reinterpret_cast<const float4*>(&sl[ly + 1][lx]);
  }
  float4 vreg[2] = {zero4(), zero4()};
  if (!HARTREE && active) {
    vreg[0] = ld4(a.veff + (long)zs * plane + own0);
    vreg[1] = ld4(a.veff + (long)zs * plane + own1);
  }
  double pacc = 0.0;  // Hartree form: p . A p over this thread's points

  // unrolled by the queue length, so the queue rotates by renaming
#pragma unroll 9
  for (int z = zs; z < ze; ++z) {
    stage(z + 4 + AHEAD);   // reuses the slot of plane z-1 (freed by the last sync)
    cp_wait<AHEAD>();       // this thread's copies of plane z+4 have landed
    const float(*cur)[HX] = pl[z & (RING - 1)];
    {
      const float(*nw)[HX] = pl[(z + 4) & (RING - 1)];
      q[8][0] = *reinterpret_cast<const float4*>(&nw[ly][lx]);
      q[8][1] = *reinterpret_cast<const float4*>(&nw[ly + 1][lx]);
    }
    const float4 vcur[2] = {vreg[0], vreg[1]};
    if (!HARTREE && active && z + 1 < ze) {
      vreg[0] = ld4(a.veff + (long)(z + 1) * plane + own0);
      vreg[1] = ld4(a.veff + (long)(z + 1) * plane + own1);
    }
    if (active) {
#pragma unroll
      for (int rr = 0; rr < 2; ++rr) {
        const float4 L = *reinterpret_cast<const float4*>(&cur[ly + rr][lx - 4]);
        const float4 R = *reinterpret_cast<const float4*>(&cur[ly + rr][lx + 4]);
        const float4 C = q[4][rr];
        const float xv[12] = {L.x, L.y, L.z, L.w, C.x, C.y, C.z, C.w, R.x, R.y, R.z, R.w};
        const float vv[4] = {vcur[rr].x, vcur[rr].y, vcur[rr].z, vcur[rr].w};
        float acc[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          float s = a.cx[4] * xv[i];
          s = fmaf(a.cx[3], xv[i + 1], s);
          s = fmaf(a.cx[2], xv[i + 2], s);
          s = fmaf(a.cx[1], xv[i + 3], s);
          s = fmaf(HARTREE ? a.c0 : a.c0 + vv[i], xv[i + 4], s);
          s = fmaf(a.cx[1], xv[i + 5], s);
          s = fmaf(a.cx[2], xv[i + 6], s);
          s = fmaf(a.cx[3], xv[i + 7], s);
          s = fmaf(a.cx[4], xv[i + 8], s);
          acc[i] = s;
        }
        // y and z terms as packed pair FMAs (each lane the scalar fma)
        float2 lo = make_float2(acc[0], acc[1]), hi = make_float2(acc[2], acc[3]);
        auto f2 = [&](const float c, const float4& v) {
          const float2 cc = make_float2(c, c);
          lo = __ffma2_rn(cc, make_float2(v.x, v.y), lo);
          hi = __ffma2_rn(cc, make_float2(v.z, v.w), hi);
        };
#pragma unroll
        for (int m = 4; m >= 1; --m) {
          const int yy = rr - m;
          f2(a.cy[m], yy == 0 ? q[4][0] : *reinterpret_cast<const float4*>(&cur[ly + yy][lx]));
        }
#pragma unroll
        for (int m = 1; m <= 4; ++m) {
          const int yy = rr + m;
          f2(a.cy[m], yy == 1 ? q[4][1] : *reinterpret_cast<const float4*>(&cur[ly + yy][lx]));
        }
#pragma unroll
        for (int m = 4; m >= 1; --m) f2(a.cz[m], q[4 - m][rr]);
#pragma unroll
        for (int m = 1; m <= 4; ++m) f2(a.cz[m], q[4 + m][rr]);
        acc[0] = lo.x; acc[1] = lo.y; acc[2] = hi.x; acc[3] = hi.y;
        *reinterpret_cast<float4*>(out + (long)z * plane + (rr ? own1 : own0)) =
            make_float4(acc[0], acc[1], acc[2], acc[3]);
        if (HARTREE) {
          pacc = fma((double)C.x, (double)acc[0], pacc);
          pacc = fma((double)C.y, (double)acc[1], pacc);
          pacc = fma((double)C.z, (double)acc[2], pacc);
          pacc = fma((double)C.w, (double)acc[3], pacc);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      q[k][0] = q[k + 1][0];
      q[k][1] = q[k + 1][1];
    }
    __syncthreads();
  }
  cp_wait<0>();
  if (HARTREE) {
    // the CTA's sum in a fixed order: lanes of a warp, then the warps
    __shared__ double ws[NTHREADS / 32];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) pacc = pacc + __shfl_down_sync(0xffffffffu, pacc, off);
    if ((tid & 31) == 0) ws[tid >> 5] = pacc;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
#pragma unroll
      for (int k = 0; k < NTHREADS / 32; ++k) t = t + ws[k];
      a.part[blockIdx.x] = t;
    }
  }
}

// ---------------------------------------------------------------------------
// k_stencil_f32_tma: the same operator and the same FMA order per point as
// k_stencil_f32_zmarch<false> (so bit-identical results), with the planes
// staged by the tensor-memory accelerator instead of per-thread cp.async.
// A tile is TYT whole rows of a plane (all NXT points of x, NXT * TYT = 2048
// points, 256 threads of 4 x 2 points), so the x halo is the tile's own row
// (periodic x wraps inside shared memory) and only the y halo is extra: one
// plane of a tile is three 2-D tensor loads of whole rows -- 4 halo rows
// above, the TYT own rows, 4 halo rows below, the halo rows wrapped
// periodically in y -- issued by one thread and counted in bytes on the
// slot's mbarrier.  Bands and z planes are rows of the tensor map too (rows
// of all bands, planes and y, NXT floats each), so z wraps by the row index.
// The kernel is issue-bound, so it spends few instructions per point:
//   * the y and z terms are packed FP32 pair FMAs (points 0,1 and 2,3 of a
//     thread's 4-point row, each lane the same fma as the scalar form);
//   * the march is unrolled by the length of the register queue (9), so the
//     queue rotates by renaming instead of 64 register moves per plane;
//   * veff is loaded two planes ahead.
// Every mbarrier wait is bounded; a wait that gives up raises *err (a
// host-mapped flag) and the CTA waits, again bounded, for the copies it
// issued before it returns.
constexpr int TRING = 8;   // staged planes
constexpr int TAHEAD = 3;  // planes in flight beyond the newest plane the queue reads

template <int NXT>
struct TmaTile {
  static constexpr int TYT = 2048 / NXT;   // own rows of a tile
  static constexpr int NTX = NXT / 4;
  static constexpr int ROWS = TYT + 8;     // with the two 4-row halos
  static constexpr int SLOT = ROWS * NXT;  // floats per staged plane
  static constexpr size_t SMEM = sizeof(float) * TRING * SLOT;
};

struct TmaArgs {
  int ny, nz, zchunk;
  float cx[5], c0;
  float2 cyy[5], czz[5];  // (cy, cy) and (cz, cz) pairs for the packed FMAs
  const float* psi;       // band 0 of the launch (also the tensor maps' base)
  float* out;
  const float* veff;
  int* err;
};

// Set by a CTA whose staging wait gave up: the CTAs that start after it
// return at once (so a broken launch ends within a few wait limits), and the
// host clears it when it reports the error.
__device__ int g_st_abort;
constexpr unsigned long long kStageWaitNs = 250000000ull;  // 0.25 s per wait

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;\n" : "=l"(t));
  return t;
}
// true once the phase of `parity` has completed; false after kStageWaitNs
// (or tc::kSpinLimit polls)
__device__ __forceinline__ bool stage_wait(uint64_t* bar, uint32_t parity) {
  if (tc::mbar_try_wait(bar, parity)) return true;
  const unsigned long long t0 = global_ns();
  for (long long i = 0; i < tc::kSpinLimit; ++i) {
    if (tc::mbar_try_wait(bar, parity)) return true;
    if (global_ns() - t0 > kStageWaitNs) break;
  }
  return false;
}
__device__ __forceinline__ void raise_stage_error(int* err) {
  atomicExch(&g_st_abort, 1);
  *reinterpret_cast<volatile int*>(err) = 1;
  __threadfence_system();
}

__device__ __forceinline__ void tma_rows(float* dst, const CUtensorMap* map, int row,
                                         uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3}], [%4];\n" ::"r"(tc::smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(0), "r"(row), "r"(tc::smem_u32(bar))
      : "memory");
}

template <int NXT>
__global__ void __launch_bounds__(NTHREADS, 2)
    k_stencil_f32_tma(const __grid_constant__ CUtensorMap core,
                      const __grid_constant__ CUtensorMap halo, TmaArgs a) {
  using T = TmaTile<NXT>;
  extern __shared__ __align__(1024) float tring[];  // [TRING][ROWS][NXT]
  __shared__ __align__(8) uint64_t full[TRING];
  __shared__ int s_abort;
  const int tid = threadIdx.x;
  const int tx = tid % T::NTX, ty = tid / T::NTX;
  const int ny = a.ny, nz = a.nz;
  const int nyt = ny / T::TYT;
  const int tile = blockIdx.x % nyt;
  const int zc = blockIdx.x / nyt;
  const int band = blockIdx.y;
  const int y0 = tile * T::TYT;
  const long plane = (long)NXT * ny;
  const long N = plane * nz;
  const float* psi = a.psi + (long)band * N;
  float* out = a.out + (long)band * N;
  const int zs = zc * a.zchunk;
  const int ze = min(zs + a.zchunk, nz);
  const int last = ze + 3;  // newest plane the march reads
  const int gx = 4 * tx, gy = y0 + 2 * ty;
  const long own0 = (long)gy * NXT + gx, own1 = own0 + NXT;
  const int ly = 2 * ty + 4;
  const int lxm = gx >= 4 ? gx - 4 : gx - 4 + NXT;   // x - 4 .. x - 1, periodic
  const int lxp = gx + 4 < NXT ? gx + 4 : gx + 4 - NXT;
  const int ytop = y0 >= 4 ? y0 - 4 : y0 - 4 + ny;
  const int ybot = y0 + T::TYT < ny ? y0 + T::TYT : y0 + T::TYT - ny;
  const int prow = band * nz;  // this band's first plane in the maps' rows / ny

  if (tid == 0) {
    // an earlier CTA gave up: leave at once (one read, so the CTA agrees)
    s_abort = *reinterpret_cast<volatile int*>(&g_st_abort);
    if (!s_abort) {
      for (int s = 0; s < TRING; ++s) tc::mbar_init(&full[s], 1);
      tc::fence_mbar_init();
    }
  }
  __syncthreads();
  if (s_abort) {
    if (tid == 0) raise_stage_error(a.err);
    return;
  }
  // thread 0: stage plane p (zs <= p <= last) into slot p % TRING
  auto stage = [&](int p) {
    const int s = p & (TRING - 1);
    float* dst = tring + s * T::SLOT;
    const int r0 = (prow + (p < nz ? p : p - nz)) * ny;
    tc::mbar_arrive_expect_tx(&full[s], (uint32_t)(T::SLOT * sizeof(float)));
    tma_rows(dst, &halo, r0 + ytop, &full[s]);
    tma_rows(dst + 4 * NXT, &core, r0 + y0, &full[s]);
    tma_rows(dst + (T::TYT + 4) * NXT, &halo, r0 + ybot, &full[s]);
  };
  auto parity = [&](int p) { return (uint32_t)(((p - zs) >> 3) & 1); };
  int issued = zs - 1;
  if (tid == 0) {
    issued = min(zs + 3 + TAHEAD, last);
    for (int p = zs; p <= issued; ++p) stage(p);
  }

  float4 q[9][2];
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    const int z = zs - 4 + k;
    const float* pp = psi + (long)(z < 0 ? z + nz : z) * plane;
    q[k][0] = ld4(pp + own0);
    q[k][1] = ld4(pp + own1);
  }
  bool ok = true;
#pragma unroll
  for (int k = 4; k < 8; ++k) {
    const int p = zs + k - 4;
    ok = ok && stage_wait(&full[p & (TRING - 1)], parity(p));
    const float* sl = tring + (p & (TRING - 1)) * T::SLOT;
    q[k][0] = *reinterpret_cast<const float4*>(sl + ly * NXT + gx);
    q[k][1] = *reinterpret_cast<const float4*>(sl + (ly + 1) * NXT + gx);
  }
  if (!ok) s_abort = 1;
  // veff of planes z and z + 1 in registers, loaded two planes ahead
  float4 vreg[2][2];
  vreg[0][0] = ld4(a.veff + (long)zs * plane + own0);
  vreg[0][1] = ld4(a.veff + (long)zs * plane + own1);
  {
    const int z1 = zs + 1 < nz ? zs + 1 : zs;
    vreg[1][0] = ld4(a.veff + (long)z1 * plane + own0);
    vreg[1][1] = ld4(a.veff + (long)z1 * plane + own1);
  }

#pragma unroll 9
  for (int z = zs; z < ze; ++z) {
    if (tid == 0 && z + 4 + TAHEAD <= last) {
      // the slot of plane z - 1, whose last reads ended at the barrier below
      tc::fence_async_smem();
      stage(z + 4 + TAHEAD);
      issued = z + 4 + TAHEAD;
    }
    const int pn = z + 4;
    if (!stage_wait(&full[pn & (TRING - 1)], parity(pn))) s_abort = 1;
    const float* cur = tring + (z & (TRING - 1)) * T::SLOT;
    {
      const float* nw = tring + (pn & (TRING - 1)) * T::SLOT;
      q[8][0] = *reinterpret_cast<const float4*>(nw + ly * NXT + gx);
      q[8][1] = *reinterpret_cast<const float4*>(nw + (ly + 1) * NXT + gx);
    }
    const float4 vcur[2] = {vreg[0][0], vreg[0][1]};
    vreg[0][0] = vreg[1][0];
    vreg[0][1] = vreg[1][1];
    if (z + 2 < ze) {
      vreg[1][0] = ld4(a.veff + (long)(z + 2) * plane + own0);
      vreg[1][1] = ld4(a.veff + (long)(z + 2) * plane + own1);
    }
#pragma unroll
    for (int rr = 0; rr < 2; ++rr) {
      const float* row = cur + (ly + rr) * NXT;
      const float4 L = *reinterpret_cast<const float4*>(row + lxm);
      const float4 R = *reinterpret_cast<const float4*>(row + lxp);
      const float4 C = q[4][rr];
      const float xv[12] = {L.x, L.y, L.z, L.w, C.x, C.y, C.z, C.w, R.x, R.y, R.z, R.w};
      const float vv[4] = {vcur[rr].x, vcur[rr].y, vcur[rr].z, vcur[rr].w};
      float acc[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        float s = a.cx[4] * xv[i];
        s = fmaf(a.cx[3], xv[i + 1], s);
        s = fmaf(a.cx[2], xv[i + 2], s);
        s = fmaf(a.cx[1], xv[i + 3], s);
        s = fmaf(a.c0 + vv[i], xv[i + 4], s);
        s = fmaf(a.cx[1], xv[i + 5], s);
        s = fmaf(a.cx[2], xv[i + 6], s);
        s = fmaf(a.cx[3], xv[i + 7], s);
        s = fmaf(a.cx[4], xv[i + 8], s);
        acc[i] = s;
      }
      float2 lo = make_float2(acc[0], acc[1]), hi = make_float2(acc[2], acc[3]);
      auto f2 = [&](const float2 c, const float4& v) {
        lo = __ffma2_rn(c, make_float2(v.x, v.y), lo);
        hi = __ffma2_rn(c, make_float2(v.z, v.w), hi);
      };
#pragma unroll
      for (int m = 4; m >= 1; --m) {
        const int yy = rr - m;
        f2(a.cyy[m],
           yy == 0 ? q[4][0] : *reinterpret_cast<const float4*>(cur + (ly + yy) * NXT + gx));
      }
#pragma unroll
      for (int m = 1; m <= 4; ++m) {
        const int yy = rr + m;
        f2(a.cyy[m],
           yy == 1 ? q[4][1] : *reinterpret_cast<const float4*>(cur + (ly + yy) * NXT + gx));
      }
#pragma unroll
      for (int m = 4; m >= 1; --m) f2(a.czz[m], q[4 - m][rr]);
#pragma unroll
      for (int m = 1; m <= 4; ++m) f2(a.czz[m], q[4 + m][rr]);
      *reinterpret_cast<float4*>(out + (long)z * plane + (rr ? own1 : own0)) =
          make_float4(lo.x, lo.y, hi.x, hi.y);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      q[k][0] = q[k + 1][0];
      q[k][1] = q[k + 1][1];
    }
    __syncthreads();
    if (s_abort) break;
  }
  if (s_abort && tid == 0) {
    // wind down: let the copies still in flight land before the CTA exits
    // (the newest TRING planes staged; older slots were reused, so their
    // phases are gone)
    for (int p = max(zs, issued - TRING + 1); p <= issued; ++p)
      stage_wait(&full[p & (TRING - 1)], parity(p));
    raise_stage_error(a.err);
  }
}

// t coefficients in atom-major order t[a][b][i] = (sum_j rp[b][a][j] m[a][i][j]) / dV
// (FP64 sum, stored FP32), so that one atom's coefficients for a block of
// bands are contiguous.
__global__ void k_tcoef_f32(int natom, int nprjmx, const int* __restrict__ nprj,
                            const double* __restrict__ mat, const double* __restrict__ rp,
                            double dxyzin, int nb, float* __restrict__ t) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)nb * natom * nprjmx;
  if (idx >= total) return;
  const int i = (int)(idx % nprjmx);
  const long ba = idx / nprjmx;
  const int at = (int)(ba % natom);
  const int b = (int)(ba / natom);
  const int P = nprj[at];
  double s = 0.0;
  if (i < P) {
    const double* r = rp + ba * nprjmx;
    const double* m = mat + ((long)at * nprjmx + i) * nprjmx;
    for (int j = 0; j < P; ++j) s = fma(r[j], m[j], s);
    s = s * dxyzin;
  }
  t[((long)at * nb + b) * nprjmx + i] = (float)s;
}

// hpsi[b][p] += sum over p's entries e of t[a_e][b] . p_e for NL_BANDS bands.
// All loads of a thread are independent of each other except through the
// entry's atom index, so many are in flight at once.
// tstride: the band count of the coefficient array (t[a][b] at (a tstride +
// b) P), so that a band range of a larger H psi runs with tco and out offset
// to its first band.
template <int NLB = NL_BANDS>
__global__ void __launch_bounds__(128) k_nl_rmw_f32(
    const int* __restrict__ cov, const int* __restrict__ cov_off, long ncov,
    const int* __restrict__ inv_atom, const float* __restrict__ inv_v,
    const float* __restrict__ tco, int P, long N, int nb, int tstride,
    float* __restrict__ out) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncov) return;
  const int b0 = blockIdx.y * NLB;
  const int nbb = min(NLB, nb - b0);
  const int p = __ldg(cov + c);
  const int e0 = __ldg(cov_off + c), e1 = __ldg(cov_off + c + 1);
  float h[NLB];
#pragma unroll
  for (int b = 0; b < NLB; ++b) h[b] = b < nbb ? out[(long)(b0 + b) * N + p] : 0.f;
  const int nq = P / 4;
  for (int e = e0; e < e1; ++e) {
    const int at = __ldg(inv_atom + e);
    float4 v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = k < nq ? ld4(inv_v + (long)e * P + 4 * k) : zero4();
    const float* tb = tco + ((long)at * tstride + b0) * P;
#pragma unroll
    for (int b = 0; b < NLB; ++b) {
      if (b < nbb) {
        float s = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          if (k < nq) {
            const float4 t = ld4(tb + (long)b * P + 4 * k);
            s = fmaf(t.x, v[k].x, s);
            s = fmaf(t.y, v[k].y, s);
            s = fmaf(t.z, v[k].z, s);
            s = fmaf(t.w, v[k].w, s);
          }
        }
        h[b] += s;
      }
    }
  }
#pragma unroll
  for (int b = 0; b < NLB; ++b)
    if (b < nbb) out[(long)(b0 + b) * N + p] = h[b];
}

// S psi in two passes.  k_entry_sums: s[b][e] = sum_j t[atom_e][b][j] p_e[j]
// for every inverse-list entry e, one FMA chain in projector order (the sum
// k_nl_rmw_f32 adds per entry); a thread owns one entry and NL_BANDS bands,
// lanes of a warp mostly share the atom, so the t loads are broadcasts.
__global__ void __launch_bounds__(128) k_entry_sums(long nent, const int* __restrict__ inv_atom,
                                                    const float* __restrict__ inv_v,
                                                    const float* __restrict__ tco, int P, int nb,
                                                    float* __restrict__ s) {
  const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  const int b0 = blockIdx.y * NL_BANDS;
  const int nbb = min(NL_BANDS, nb - b0);
  const int at = __ldg(inv_atom + e);
  const int nq = P / 4;
  float4 v[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) v[q] = q < nq ? ld4(inv_v + e * P + 4 * q) : zero4();
  const float* tb = tco + ((long)at * nb + b0) * P;
#pragma unroll
  for (int b = 0; b < NL_BANDS; ++b) {
    if (b < nbb) {
      float sum = 0.f;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        if (q < nq) {
          const float4 t = ld4(tb + (long)b * P + 4 * q);
          sum = fmaf(t.x, v[q].x, sum);
          sum = fmaf(t.y, v[q].y, sum);
          sum = fmaf(t.z, v[q].z, sum);
          sum = fmaf(t.w, v[q].w, sum);
        }
      }
      s[(long)(b0 + b) * nent + e] = sum;
    }
  }
}

// k_spsi_apply: S psi = psi + the entry sums of each point, added in the
// inverse-list order (so the same additions as k_nl_rmw_f32).  A thread owns
// 4 consecutive points (one 16-byte vector per band) and SP_BANDS bands,
// reads psi and writes S psi once; psi == out is allowed (a thread reads its
// values before writing them).
constexpr int SP_BANDS = 8;
__global__ void __launch_bounds__(128) k_spsi_apply(long N, int nb, long nent, const float* psi,
                                                    float* out, const int* __restrict__ inv_off,
                                                    const float* __restrict__ s) {
  const long p0 = ((long)blockIdx.x * blockDim.x + threadIdx.x) * 4;
  if (p0 >= N) return;
  const int b0 = blockIdx.y * SP_BANDS;
  const int nbb = min(SP_BANDS, nb - b0);
  float4 h[SP_BANDS];
#pragma unroll
  for (int b = 0; b < SP_BANDS; ++b)
    h[b] = b < nbb ? ld4(psi + (long)(b0 + b) * N + p0) : zero4();
  const int4 o4 = __ldg(reinterpret_cast<const int4*>(inv_off + p0));
  const int o[5] = {o4.x, o4.y, o4.z, o4.w, __ldg(inv_off + p0 + 4)};
  if (o[4] > o[0]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      for (int e = o[k]; e < o[k + 1]; ++e) {
#pragma unroll
        for (int b = 0; b < SP_BANDS; ++b) {
          if (b < nbb) {
            const float v = __ldg(s + (long)(b0 + b) * nent + e);
            float* hk = k == 0 ? &h[b].x : (k == 1 ? &h[b].y : (k == 2 ? &h[b].z : &h[b].w));
            *hk += v;
          }
        }
      }
    }
  }
#pragma unroll
  for (int b = 0; b < SP_BANDS; ++b)
    if (b < nbb) *reinterpret_cast<float4*>(out + (long)(b0 + b) * N + p0) = h[b];
}

}  // namespace

// true when launch_hpsi_f32_fast takes the z-march (and can stop after its
// local part) for nb bands
bool hpsi_f32_fast_ok(const rs_geom* g, int nb) {
  const bool shape_ok = g->nf == 4 && g->nx % 4 == 0 && g->ny % 2 == 0 && g->nx >= 8 &&
                        g->ny >= 8 && g->nz >= 8 && nb <= 65535;
  const bool proj_ok = g->nprjmx % 4 == 0 && g->nprjmx <= 16;
  return shape_ok && proj_ok;
}

namespace {

void stencil_args(const rs_geom* g, const float* veff, StArgs& a) {
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.zchunk = g->nz <= 160 ? g->nz : 64;
  a.ntx = (g->nx + TX - 1) / TX;
  a.nty = (g->ny + TY - 1) / TY;
  for (int m = 0; m < 5; ++m) {
    a.cx[m] = (float)g->cx[m]; a.cy[m] = (float)g->cy[m]; a.cz[m] = (float)g->cz[m];
  }
  a.c0 = (float)(g->cx[0] + g->cy[0] + g->cz[0]);
  a.veff = veff;
  a.done = nullptr;
  a.part = nullptr;
}

using EncodeTiled = PFN_cuTensorMapEncodeTiled_v12000;

// cuTensorMapEncodeTiled from the driver the runtime loaded (null if absent)
EncodeTiled tensor_map_encoder() {
  static const EncodeTiled fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) !=
            cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      p = nullptr;
    return reinterpret_cast<EncodeTiled>(p);
  }();
  return fn;
}

// the TMA form takes nx = 64, 128 or 256 (tiles of 32, 16 or 8 whole rows)
// with ny a multiple of the tile height, and row indices of n bands that fit
// in 32 bits
bool stencil_tma_shape(const rs_geom* g, int n) {
  const int nx = g->nx;
  if (nx != 64 && nx != 128 && nx != 256) return false;
  const int tyt = 2048 / nx;
  return g->ny % tyt == 0 && (long)n * g->nz * g->ny < (1L << 31);
}

// n bands of nx floats per row, ny * nz rows per band, boxes of `rows` rows
cudaError_t encode_rows(CUtensorMap* m, const float* base, int nx, long nrows, int rows) {
  const cuuint64_t dims[2] = {(cuuint64_t)nx, (cuuint64_t)nrows};
  const cuuint64_t strides[1] = {(cuuint64_t)nx * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)nx, (cuuint32_t)rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = tensor_map_encoder()(
      m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int NXT>
cudaError_t launch_stencil_tma(rs_geom* g, const StArgs& sa, const float* psi, float* out, int n,
                               cudaStream_t st) {
  using T = TmaTile<NXT>;
  cudaError_t e = cudaFuncSetAttribute(k_stencil_f32_tma<NXT>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)T::SMEM);
  if (e != cudaSuccess) return e;
  CUtensorMap core, halo;
  const long nrows = (long)n * g->nz * g->ny;
  e = encode_rows(&core, psi, NXT, nrows, T::TYT);
  if (e == cudaSuccess) e = encode_rows(&halo, psi, NXT, nrows, 4);
  if (e != cudaSuccess) return e;
  TmaArgs a;
  a.ny = g->ny; a.nz = g->nz; a.zchunk = sa.zchunk;
  for (int m = 0; m < 5; ++m) {
    a.cx[m] = sa.cx[m];
    a.cyy[m] = make_float2(sa.cy[m], sa.cy[m]);
    a.czz[m] = make_float2(sa.cz[m], sa.cz[m]);
  }
  a.c0 = sa.c0;
  a.psi = psi; a.out = out; a.veff = sa.veff;
  a.err = g->st_err_d;
  const int nzc = (g->nz + a.zchunk - 1) / a.zchunk;
  dim3 grid((g->ny / T::TYT) * nzc, n);
  k_stencil_f32_tma<NXT><<<grid, NTHREADS, T::SMEM, st>>>(core, halo, a);
  return cudaGetLastError();
}

// true when the stencil of n bands runs the TMA form; allocates its error
// flag on first use (never inside a stream capture)
bool use_stencil_tma(rs_geom* g, int n, cudaStream_t st) {
  if (g->st_copy != 0 || !stencil_tma_shape(g, n) || !tensor_map_encoder()) return false;
  if (!g->st_err_h) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs != cudaStreamCaptureStatusNone) return false;
    int* h = nullptr;
    if (cudaHostAlloc((void**)&h, sizeof(int), cudaHostAllocMapped) != cudaSuccess) return false;
    *h = 0;
    int* d = nullptr;
    if (cudaHostGetDevicePointer((void**)&d, h, 0) != cudaSuccess) {
      cudaFreeHost(h);
      return false;
    }
    g->st_err_h = h;
    g->st_err_d = d;
  }
  return true;
}

// stencil of bands [b0, b0 + n) on st
cudaError_t launch_stencil(rs_geom* g, StArgs a, const float* psi, float* hpsi, int b0, int n,
                           cudaStream_t st) {
  a.psi = psi + (long)b0 * g->N;
  a.out = hpsi + (long)b0 * g->N;
  if (use_stencil_tma(g, n, st)) {
    switch (g->nx) {
      case 64: return launch_stencil_tma<64>(g, a, a.psi, a.out, n, st);
      case 128: return launch_stencil_tma<128>(g, a, a.psi, a.out, n, st);
      default: return launch_stencil_tma<256>(g, a, a.psi, a.out, n, st);
    }
  }
  const int nzc = (g->nz + a.zchunk - 1) / a.zchunk;
  dim3 grid(a.ntx * a.nty * nzc, n);
  k_stencil_f32_zmarch<false><<<grid, NTHREADS, sizeof(float) * RING * HY * HX, st>>>(a);
  return cudaGetLastError();
}

// nonlocal pass of bands [b0, b0 + n) (t holds all nb bands' coefficients),
// nlb bands per thread (16 or 32)
void launch_nl(const rs_geom* g, const float* t, float* hpsi, int b0, int n, int nb, int nlb,
               cudaStream_t st) {
  // t[a][b0 + b] lies b0 P floats past t[a][b]: offset the base, keep the
  // stride of all nb bands
  const float* tb = t + (long)b0 * g->nprjmx;
  float* out = hpsi + (long)b0 * g->N;
  if (nlb == 32) {
    dim3 g2(div_up(g->n_cov, 128), div_up(n, 32));
    k_nl_rmw_f32<32><<<g2, 128, 0, st>>>(g->d_cov, g->d_cov_off, g->n_cov, g->d_inv_atom,
                                         g->d_inv_v32, tb, g->nprjmx, g->N, n, nb, out);
  } else {
    dim3 g2(div_up(g->n_cov, 128), div_up(n, NL_BANDS));
    k_nl_rmw_f32<<<g2, 128, 0, st>>>(g->d_cov, g->d_cov_off, g->n_cov, g->d_inv_atom,
                                      g->d_inv_v32, tb, g->nprjmx, g->N, n, nb, out);
  }
}

}  // namespace

// local_only: (-1/2 lap + veff) psi alone, without the nonlocal term (only
// where hpsi_f32_fast_ok holds).
//
// The nonlocal pass re-reads H psi at the covered points.  It runs on a side
// stream chunk by chunk behind the stencil, so that a chunk's pass overlaps
// the next chunk's stencil and finds much of the chunk's H psi still in L2.
// The chunk size (bands) is chosen once per geometry, on its first call with
// at least 64 bands, by timing the candidates on that call's own data (the
// call's result is the same whichever ran last); -1 is the unchunked form.
int launch_hpsi_f32_fast(const rs_geom* gc, const float* veff, const double* dij,
                         const double* rp, const float* psi, float* hpsi, int nb,
                         cudaStream_t st, bool local_only) {
  if (nb <= 0) return RS_OK;
  rs_geom* g = const_cast<rs_geom*>(gc);
  if (!hpsi_f32_fast_ok(g, nb)) {
    if (local_only) return fail(RS_EINVAL, "H psi: local part alone needs the z-march shape");
    return launch_gather<float, 1>(g, dij, rp, psi, veff, hpsi, nb, st);
  }
  StArgs a;
  stencil_args(g, veff, a);
  RS_CUDA(cudaFuncSetAttribute(k_stencil_f32_zmarch<false>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(sizeof(float) * RING * HY * HX)));
  if (g->st_err_h && *reinterpret_cast<volatile int*>(g->st_err_h)) {
    // raised by an earlier call on this geometry: report it once, clear it
    *g->st_err_h = 0;
    const int zero = 0;
    cudaMemcpyToSymbolAsync(g_st_abort, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    return fail(RS_ECUDA, "H psi: a plane-staging wait of k_stencil_f32_tma timed out");
  }
  if (local_only || g->natom == 0 || g->n_cov == 0) {
    const cudaError_t e = launch_stencil(g, a, psi, hpsi, 0, nb, st);
    if (e != cudaSuccess) return cuda_status(e, "k_stencil_f32 (H psi local part)");
    return RS_OK;
  }
  const long nt = (long)nb * g->natom * g->nprjmx;
  float* t = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&t, nt * sizeof(float), st));
  k_tcoef_f32<<<div_up(nt, 256), 256, 0, st>>>(g->natom, g->nprjmx, g->d_nprj, dij, rp,
                                               1.0 / (g->dx * g->dy * g->dz), nb, t);
  if (!g->nl_cs) {
    RS_CUDA(cudaStreamCreateWithFlags(&g->nl_cs, cudaStreamNonBlocking));
    RS_CUDA(cudaEventCreateWithFlags(&g->nl_ev_in, cudaEventDisableTiming));
    RS_CUDA(cudaEventCreateWithFlags(&g->nl_ev_out, cudaEventDisableTiming));
  }
  // tuning code: chunk size in bands (<= 0: unchunked) times 64, plus the
  // nonlocal band block (16 or 32)
  auto run = [&](int code) -> cudaError_t {
    const int chunk = code >= 0 ? code / 64 : -1;
    const int nlb = code >= 0 ? code % 64 : (-code) % 64;
    if (chunk <= 0 || chunk >= nb) {
      const cudaError_t e = launch_stencil(g, a, psi, hpsi, 0, nb, st);
      if (e != cudaSuccess) return e;
      launch_nl(g, t, hpsi, 0, nb, nb, nlb, st);
      return cudaGetLastError();
    }
    // small chunks split z into runs of 32 planes so that a chunk's stencil
    // still fills the GPU
    StArgs ac = a;
    if (chunk <= 16 && g->nz > 64) ac.zchunk = 32;
    for (int b0 = 0; b0 < nb; b0 += chunk) {
      const int n = std::min(chunk, nb - b0);
      const cudaError_t e = launch_stencil(g, ac, psi, hpsi, b0, n, st);
      if (e != cudaSuccess) return e;
      cudaEventRecord(g->nl_ev_in, st);
      cudaStreamWaitEvent(g->nl_cs, g->nl_ev_in, 0);
      launch_nl(g, t, hpsi, b0, n, nb, nlb, g->nl_cs);
    }
    cudaEventRecord(g->nl_ev_out, g->nl_cs);
    cudaStreamWaitEvent(st, g->nl_ev_out, 0);
    return cudaGetLastError();
  };
  cudaError_t e = cudaSuccess;
  if (g->nl_chunk == 0 && nb >= 64) {
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cs);
    if (cs == cudaStreamCaptureStatusNone) {
      // unchunked (negative codes) or chunks of 4 to 64 bands, with
      // nonlocal band blocks of 16 or 32
      const int cand[] = {-16, -32, 4 * 64 + 16, 8 * 64 + 16, 16 * 64 + 16, 16 * 64 + 32,
                          32 * 64 + 16, 32 * 64 + 32, 64 * 64 + 32};
      cudaEvent_t e0, e1;
      float best = 0.f;
      int pick = -NL_BANDS;
      cudaEventCreate(&e0);
      cudaEventCreate(&e1);
      for (int c : cand) {
        run(c);  // warm
        cudaEventRecord(e0, st);
        run(c);
        cudaEventRecord(e1, st);
        if ((e = cudaEventSynchronize(e1)) != cudaSuccess) break;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (best == 0.f || ms < best) {
          best = ms;
          pick = c;
        }
      }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      if (e == cudaSuccess) g->nl_chunk = pick;
    }
  }
  if (e == cudaSuccess) e = run(g->nl_chunk == 0 ? -NL_BANDS : g->nl_chunk);
  cudaFreeAsync(t, st);
  if (e != cudaSuccess) return cuda_status(e, "H psi (k_stencil_f32, k_nl_rmw_f32)");
  return RS_OK;
}

// the band-chunk size the FP32 H psi of this geometry picked (0: not yet
// chosen, -1: unchunked)
int hpsi_f32_nl_chunk(const rs_geom* g) { return g->nl_chunk; }

// staging of the FP32 stencil: mode 0 = TMA where the grid allows it, 1 =
// cp.async (mode < 0 leaves it); *tma = 1 when a call of nb bands would run
// the TMA form
int hpsi_f32_staging(rs_geom* g, int mode, int nb, int* tma) {
  if (mode > 1) return fail(RS_EINVAL, "rs_hpsi_f32_staging: mode must be 0 or 1");
  if (mode >= 0) g->st_copy = mode;
  *tma = (g->st_copy == 0 && stencil_tma_shape(g, nb) && hpsi_f32_fast_ok(g, nb) &&
          tensor_map_encoder() != nullptr) ? 1 : 0;
  return RS_OK;
}

// A p of the mixed Hartree CG (nfh = 4) by the H psi z-march: coefficients
// cx, cy, cz [1..4] and diag from hartree_coefs, runs of 32 z planes (so one
// grid fills the GPU), one p.Ap partial per CTA in part[0, *nparts).  The
// launch returns at once when *done is set.
bool hartree_ap_f32_ok(int nx, int ny, int nz, int nfh) {
  return nfh == 4 && nx % 4 == 0 && ny % 2 == 0 && nx >= 8 && ny >= 8 && nz >= 8;
}
// z run of the Hartree A p: 32 planes where that gives a CTA per SM, else 16
// or 8 (small grids: more CTAs at the cost of re-reading the 8 halo planes of
// each run), and the whole z extent below 48 planes
int hartree_ap_f32_zchunk(int nx, int ny, int nz) {
  if (nz <= 48) return nz;
  const long tiles = (long)((nx + TX - 1) / TX) * ((ny + TY - 1) / TY);
  for (int zc : {32, 16}) {
    if (tiles * ((nz + zc - 1) / zc) >= 148) return zc;
  }
  return 8;
}
unsigned hartree_ap_f32_ctas(int nx, int ny, int nz) {
  const int zchunk = hartree_ap_f32_zchunk(nx, ny, nz);
  return (unsigned)(((nx + TX - 1) / TX) * ((ny + TY - 1) / TY) * ((nz + zchunk - 1) / zchunk));
}
// shared-memory limit of the Hartree form; call before any stream capture
int hartree_ap_f32_attr() {
  RS_CUDA(cudaFuncSetAttribute(k_stencil_f32_zmarch<true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)(sizeof(float) * RING * HY * HX)));
  return RS_OK;
}
int launch_hartree_ap_f32(int nx, int ny, int nz, const double* cx, const double* cy,
                          const double* cz, double diag, const float* p, float* ap,
                          const int* done, double* part, cudaStream_t st) {
  StArgs a;
  a.nx = nx; a.ny = ny; a.nz = nz;
  a.zchunk = hartree_ap_f32_zchunk(nx, ny, nz);
  a.ntx = (nx + TX - 1) / TX;
  a.nty = (ny + TY - 1) / TY;
  a.cx[0] = a.cy[0] = a.cz[0] = 0.f;
  for (int m = 1; m < 5; ++m) {
    a.cx[m] = (float)cx[m]; a.cy[m] = (float)cy[m]; a.cz[m] = (float)cz[m];
  }
  a.c0 = (float)diag;
  a.psi = p; a.out = ap; a.veff = nullptr;
  a.done = done; a.part = part;
  const size_t smem = sizeof(float) * RING * HY * HX;
  k_stencil_f32_zmarch<true><<<hartree_ap_f32_ctas(nx, ny, nz), NTHREADS, smem, st>>>(a);
  RS_LAUNCH_CHECK("k_stencil_f32_zmarch (Hartree)");
  return RS_OK;
}

// S psi for FP32 bands; false when the geometry does not fit the fast path
// (the caller then uses the per-band gather)
bool spsi_f32_fast_ok(const rs_geom* g) {
  return g->nprjmx % 4 == 0 && g->nprjmx <= 16 && g->natom > 0 && g->N < (1L << 31);
}

int launch_spsi_f32_fast(const rs_geom* g, const double* sss, const double* rp, const float* psi,
                         float* out, int nb, cudaStream_t st) {
  if (nb <= 0) return RS_OK;
  const long nt = (long)nb * g->natom * g->nprjmx;
  float* t = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&t, nt * sizeof(float), st));
  k_tcoef_f32<<<div_up(nt, 256), 256, 0, st>>>(g->natom, g->nprjmx, g->d_nprj, sss, rp,
                                               1.0 / (g->dx * g->dy * g->dz), nb, t);
  cudaError_t e = cudaSuccess;
  const bool vec = g->N % 4 == 0 && ((uintptr_t)psi | (uintptr_t)out) % 16 == 0 &&
                   nb <= 65535 * SP_BANDS;
  if (vec) {
    const long ne = g->n_inv;
    float* sums = nullptr;
    if (ne > 0) {
      e = cudaMallocAsync((void**)&sums, sizeof(float) * (size_t)ne * nb, st);
      if (e == cudaSuccess) {
        dim3 g1(div_up(ne, 128), div_up(nb, NL_BANDS));
        k_entry_sums<<<g1, 128, 0, st>>>(ne, g->d_inv_atom, g->d_inv_v32, t, g->nprjmx, nb, sums);
      }
    }
    if (e == cudaSuccess) {
      dim3 g2(div_up(g->N / 4, 128), div_up(nb, SP_BANDS));
      k_spsi_apply<<<g2, 128, 0, st>>>(g->N, nb, ne > 0 ? ne : 1, psi, out, g->d_inv_off,
                                        sums);
      e = cudaGetLastError();
    }
    if (sums) cudaFreeAsync(sums, st);
    cudaFreeAsync(t, st);
    if (e != cudaSuccess) return cuda_status(e, "S psi (k_entry_sums, k_spsi_apply)");
    return RS_OK;
  }
  // otherwise out = psi, then the nonlocal sums added on the points inside a
  // projector support only (the same entries, sums and order)
  if (out != psi)
    e = cudaMemcpyAsync(out, psi, sizeof(float) * g->N * nb, cudaMemcpyDeviceToDevice, st);
  if (e == cudaSuccess && g->n_cov > 0) {
    dim3 g2(div_up(g->n_cov, 128), div_up(nb, NL_BANDS));
    k_nl_rmw_f32<<<g2, 128, 0, st>>>(g->d_cov, g->d_cov_off, g->n_cov, g->d_inv_atom,
                                      g->d_inv_v32, t, g->nprjmx, g->N, nb, nb, out);
    e = cudaGetLastError();
  }
  cudaFreeAsync(t, st);
  if (e != cudaSuccess) return cuda_status(e, "S psi (k_nl_rmw_f32)");
  return RS_OK;
}

}  // namespace rs
