// density.cu -- density build, coarse->dense interpolation, fixed-tree dot
// products and the Hartree CG Poisson solve.
#include <math.h>

#include <vector>

#include "reduce.cuh"
#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {

// ------------------------------------------------------------ tree dot
template <class T>
__global__ void k_tree_partial(long n, const T* __restrict__ a, const T* __restrict__ b,
                               double* __restrict__ part) {
  __shared__ double ws[8];
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < n) acc = fma((double)a[i], (double)b[i], acc);
  }
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// folds nblk chunk sums; scale multiplies the result (scale==1 leaves it exact)
__global__ void k_tree_final(long nblk, const double* __restrict__ part, double* __restrict__ out) {
  __shared__ double ws[8];
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + part[k];
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) *out = s;
}

template <class T>
int tree_dot(long n, const T* a, const T* b, double* out, double* part, cudaStream_t st) {
  const long nblk = tree_chunks(n);
  if (nblk == 0) {
    RS_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    return RS_OK;
  }
  k_tree_partial<T><<<(unsigned)nblk, kTreeLanes, 0, st>>>(n, a, b, part);
  k_tree_final<<<1, kTreeLanes, 0, st>>>(nblk, part, out);
  RS_LAUNCH_CHECK("tree_dot");
  return RS_OK;
}
template int tree_dot<double>(long, const double*, const double*, double*, double*, cudaStream_t);
template int tree_dot<float>(long, const float*, const float*, double*, double*, cudaStream_t);

// ------------------------------------------------------------ density
// scf_charge_smt_r (scf_charge8f.F90:309-319): rho = rho + (f*psi)*psi over
// bands in order, one thread per point.
template <class T>
__global__ void k_density(long N, int nb, const double* __restrict__ occ,
                          const T* __restrict__ psi, double* __restrict__ rho) {
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  double r = 0.0;
  for (int b = 0; b < nb; ++b) {
    const double x = (double)__ldg(psi + (long)b * N + p);
    r = fma(__ldg(occ + b) * x, x, r);
  }
  rho[p] = r;
}

// ------------------------------------------------------------ interpolation
struct InterpW {
  double w[2][16];
};

// One separable pass of interpolation8f.F90:56-95 (forward, nmesh=2): the
// output axis `axis` is doubled; dense index jd takes coarse base
// (jd+1)/2 - 1 and weight row (jd+1) mod 2.
__global__ void k_interp_pass(int nxo, int nyo, int nzo, int nxi, int nyi, int nzi, int axis,
                              int nf, InterpW W, const double* __restrict__ in,
                              double* __restrict__ out) {
  const long No = (long)nxo * nyo * nzo;
  const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= No) return;
  const int jx = (int)(q % nxo), jy = (int)((q / nxo) % nyo), jz = (int)(q / ((long)nxo * nyo));
  const int jd = axis == 0 ? jx : (axis == 1 ? jy : jz);
  const int k = (jd + 1) % 2, l0 = (jd + 1) / 2 - 1;
  const int n = axis == 0 ? nxi : (axis == 1 ? nyi : nzi);
  double acc = 0.0;
  for (int i = -nf + 1; i <= nf; ++i) {
    const int c = (int)wrapi(l0 + i, n);
    long src;
    if (axis == 0) src = ((long)jz * nyi + jy) * nxi + c;
    else if (axis == 1) src = ((long)jz * nyi + c) * nxi + jx;
    else src = ((long)c * nyi + jy) * nxi + jx;
    acc = fma(W.w[k][i + nf - 1], in[src], acc);
  }
  out[q] = acc;
}

static InterpW interp_weights(int nf) {
  InterpW W;
  for (int k = 0; k < 2; ++k) {
    const double r = ((double)k + 0.5) * 0.5;
    for (int j = -nf + 1; j <= nf; ++j) {
      double w = 1.0;
      for (int i = -nf + 1; i <= nf; ++i)
        if (i != j) w = w * (r - (double)i) / ((double)j - (double)i);
      W.w[k][j + nf - 1] = w;
    }
  }
  return W;
}

// ------------------------------------------------------------ Hartree CG
// scf_hartree_cg (scf_hartree8f.F90:626-812).  Each iteration is five
// launches: the stencil with the p.Ap chunk sums of the reduction tree, the
// tree's final fold with alpha, the x/r update with the r.r chunk sums, the
// final fold with beta, dp and the stopping test, and the direction update.
// Every sum keeps the tree order of tree_dot (a point's chunk and lane are
// those of k_tree_partial), so iterates equal the unfused sequence bit for
// bit.  r1r of an iteration equals r2r of the one before (r is unchanged in
// between) and is carried over instead of summed again.  The stopping test
// runs on the device: once it fires, the kernels of the iterations already
// queued return at once, and the host checks the flag every kCgBatch
// iterations instead of after each one.
struct CgScalars {
  double r1r, pap, r2r, alph, beta, dp, bve;
  double r2ref;  // mixed solve: r.r at the last FP64 residual
  int done, iters;
  int upd;       // mixed solve: recompute the residual in FP64 now
  unsigned ticket;  // mixed solve: update blocks finished (the last one folds r.r)
};
static_assert(sizeof(CgScalars) <= 16 * sizeof(double), "CG scalars fit the work array");

constexpr int kCgBatch = 50;  // iterations per host check (800 = 16 batches)


// ap = A p by a z-march, in k_hartree_lap's multiply-add order (x terms from
// the first product, then y, then z; scf_hartree8f.F90:949-1004).  A CTA owns a
// 32 x 16 tile of an xy plane for a run of z planes; each thread one point.
//  * halo'd planes (the tile plus NF points on each side in x and y) are
//    copied into a ring of hz_ring(NF) shared-memory slots with 8-byte
//    cp.async, HZ_AHEAD planes ahead of use; x and y terms read the ring;
//  * the z terms come from a register queue of the thread's own column
//    (planes z-NF .. z+NF), so each plane crosses HBM about once;
//  * one __syncthreads per plane orders the ring reuse.
// The staging index of every element is computed once with a full modulo,
// so any grid of at least one point per axis is handled.
constexpr int HZ_TX = 32, HZ_TY = 16, HZ_THREADS = HZ_TX * HZ_TY, HZ_AHEAD = 7;
__host__ __device__ constexpr int hz_ring(int nf) { return nf + HZ_AHEAD + 1; }
__host__ __device__ constexpr int hz_plane(int nf) { return (HZ_TX + 2 * nf) * (HZ_TY + 2 * nf); }
constexpr int HZ_STAGE_MAX = 4;  // staged elements per thread (hz_plane(6) = 44 * 28 = 1232)

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit_hz() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait_hz() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}
__device__ __forceinline__ int wrapm(long i, int n) {
  long r = i % n;
  return (int)(r < 0 ? r + n : r);
}

template <int NF>
__global__ void __launch_bounds__(HZ_THREADS, 2) k_hlap_zmarch(int nx, int ny, int nz,
                                                               int zchunk, HartreeCoefs c,
                                                               const double* __restrict__ p,
                                                               double* __restrict__ ap,
                                                               const CgScalars* __restrict__ s) {
  if (s->done) return;
  constexpr int HX = HZ_TX + 2 * NF, HY = HZ_TY + 2 * NF, PL = HX * HY, RING = hz_ring(NF);
  constexpr int NST = (PL + HZ_THREADS - 1) / HZ_THREADS;
  static_assert(NST <= HZ_STAGE_MAX, "staging slots");
  extern __shared__ double hz_sm[];  // [RING][HY][HX]
  const int tid = threadIdx.x, tx = tid % HZ_TX, ty = tid / HZ_TX;
  const int ntx = (nx + HZ_TX - 1) / HZ_TX, nty = (ny + HZ_TY - 1) / HZ_TY;
  const int tile = blockIdx.x % (ntx * nty), zc = blockIdx.x / (ntx * nty);
  const int x0 = (tile % ntx) * HZ_TX, y0 = (tile / ntx) * HZ_TY;
  const int zs = zc * zchunk, ze = min(zs + zchunk, nz);
  const long plane = (long)nx * ny;
  const int gx = x0 + tx, gy = y0 + ty;
  const bool active = gx < nx && gy < ny;
  const long own = active ? (long)gy * nx + gx : 0;
  // in-plane source offsets of this thread's staged elements (the same every plane)
  int soff[NST], doff[NST];
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int e = tid + k * HZ_THREADS;
    if (e < PL) {
      const int r = e / HX, q = e % HX;
      soff[k] = (int)((long)wrapm(y0 - NF + r, ny) * nx + wrapm(x0 - NF + q, nx));
      doff[k] = e;
    } else {
      soff[k] = -1;
      doff[k] = 0;
    }
  }
  // planes z in [zs - NF, ze + NF + HZ_AHEAD); the ring slot of plane z is
  // (z - zs + NF) mod RING, kept as a running counter
  auto wrapz = [&](int z) {
    while (z < 0) z += nz;
    while (z >= nz) z -= nz;
    return z;
  };
  auto slot = [&](int z) { return (z - zs + NF) % RING; };
  auto stage = [&](int z) {
    const double* src = p + (long)wrapz(z) * plane;
    double* dst = hz_sm + slot(z) * PL;
#pragma unroll
    for (int k = 0; k < NST; ++k)
      if (soff[k] >= 0) cp_async8(dst + doff[k], src + soff[k]);
    cp_commit_hz();
  };
  double q[2 * NF + 1];  // q[k]: plane z-NF+k at (gx, gy)
#pragma unroll
  for (int k = 0; k < NF; ++k) q[k] = __ldg(p + (long)wrapz(zs - NF + k) * plane + own);
#pragma unroll
  for (int k = 0; k < NF + HZ_AHEAD; ++k) stage(zs + k);
  const int lc = (ty + NF) * HX + tx + NF;  // this thread's point in a staged plane
  for (int z = zs; z < ze; ++z) {
    cp_wait_hz<HZ_AHEAD - 1>();  // planes up to z+NF have landed (this thread's copies)
    __syncthreads();             // ... everyone's; plane z-1's slot is free
    stage(z + NF + HZ_AHEAD);
    if (z == zs) {
#pragma unroll
      for (int k = 0; k < NF; ++k) q[NF + k] = hz_sm[slot(zs + k) * PL + lc];
    }
    q[2 * NF] = hz_sm[slot(z + NF) * PL + lc];
    const double* cur = hz_sm + slot(z) * PL;
    double acc = c.cx[NF] * cur[lc - NF];
#pragma unroll
    for (int m = NF - 1; m >= 1; --m) acc = fma(c.cx[m], cur[lc - m], acc);
    acc = fma(c.diag, cur[lc], acc);
#pragma unroll
    for (int m = 1; m <= NF; ++m) acc = fma(c.cx[m], cur[lc + m], acc);
#pragma unroll
    for (int m = NF; m >= 1; --m) acc = fma(c.cy[m], cur[lc - m * HX], acc);
#pragma unroll
    for (int m = 1; m <= NF; ++m) acc = fma(c.cy[m], cur[lc + m * HX], acc);
#pragma unroll
    for (int m = NF; m >= 1; --m) acc = fma(c.cz[m], q[NF - m], acc);
#pragma unroll
    for (int m = 1; m <= NF; ++m) acc = fma(c.cz[m], q[NF + m], acc);
    if (active) ap[(long)z * plane + own] = acc;
#pragma unroll
    for (int k = 0; k < 2 * NF; ++k) q[k] = q[k + 1];
  }
  cp_wait_hz<0>();
}

// The same z-march with two x-neighbouring points per thread, for even NF and
// even nx: 16-byte staging copies and 16-byte shared loads (x terms of both
// points from NF+1 double2 loads, y terms and the z queue as double2), about
// half the instructions per point.  64 x 16 tiles, one CTA per SM.
constexpr int HZ2_TX = 64, HZ2_TY = 16, HZ2_THREADS = (HZ2_TX / 2) * HZ2_TY, HZ2_AHEAD = 5;
__host__ __device__ constexpr int hz2_ring(int nf) { return nf + HZ2_AHEAD + 1; }
__host__ __device__ constexpr int hz2_plane(int nf) { return (HZ2_TX + 2 * nf) * (HZ2_TY + 2 * nf); }

__device__ __forceinline__ void cp_async16_hz(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}

// RES: the residual of the mixed solve instead, out32 = (float)(b - A p), only
// when s->upd is set.
template <int NF, bool RES = false>
__global__ void __launch_bounds__(HZ2_THREADS, 1) k_hlap_zmarch2(int nx, int ny, int nz,
                                                                 int zchunk, HartreeCoefs c,
                                                                 const double* __restrict__ p,
                                                                 double* __restrict__ ap,
                                                                 const CgScalars* __restrict__ s,
                                                                 const double* __restrict__ b = nullptr,
                                                                 float* __restrict__ out32 = nullptr,
                                                                 double* __restrict__ rpart = nullptr) {
  static_assert(NF % 2 == 0, "double2 path needs an even halo");
  if (s->done || (RES && !s->upd)) return;
  double racc = 0.0;  // RES: r.r of this thread's FP32 residual values
  constexpr int HX = HZ2_TX + 2 * NF, HY = HZ2_TY + 2 * NF, PL = HX * HY, RING = hz2_ring(NF);
  constexpr int PL2 = PL / 2, NST = (PL2 + HZ2_THREADS - 1) / HZ2_THREADS;
  extern __shared__ double2 hz2_sm[];  // [RING][HY][HX / 2]
  const int tid = threadIdx.x, tx = tid % (HZ2_TX / 2), ty = tid / (HZ2_TX / 2);
  const int ntx = (nx + HZ2_TX - 1) / HZ2_TX, nty = (ny + HZ2_TY - 1) / HZ2_TY;
  const int tile = blockIdx.x % (ntx * nty), zc = blockIdx.x / (ntx * nty);
  const int x0 = (tile % ntx) * HZ2_TX, y0 = (tile / ntx) * HZ2_TY;
  const int zs = zc * zchunk, ze = min(zs + zchunk, nz);
  const long plane = (long)nx * ny;
  const int gx = x0 + 2 * tx, gy = y0 + ty;
  const bool active = gx < nx && gy < ny;  // nx even: gx + 1 < nx as well
  const long own = active ? (long)gy * nx + gx : 0;
  int soff[NST], doff[NST];
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int e = tid + k * HZ2_THREADS;  // double2 index in the staged plane
    if (e < PL2) {
      const int r = e / (HX / 2), q2 = e % (HX / 2);
      soff[k] = (int)((long)wrapm(y0 - NF + r, ny) * nx + wrapm(x0 - NF + 2 * q2, nx));
      doff[k] = e;
    } else {
      soff[k] = -1;
      doff[k] = 0;
    }
  }
  auto wrapz = [&](int z) {
    while (z < 0) z += nz;
    while (z >= nz) z -= nz;
    return z;
  };
  auto slot = [&](int z) { return (z - zs + NF) % RING; };
  auto stage = [&](int z) {
    const double* src = p + (long)wrapz(z) * plane;
    double2* dst = hz2_sm + slot(z) * PL2;
#pragma unroll
    for (int k = 0; k < NST; ++k)
      if (soff[k] >= 0) cp_async16_hz(dst + doff[k], src + soff[k]);
    cp_commit_hz();
  };
  double2 q[2 * NF + 1];
#pragma unroll
  for (int k = 0; k < NF; ++k)
    q[k] = __ldg(reinterpret_cast<const double2*>(p + (long)wrapz(zs - NF + k) * plane + own));
#pragma unroll
  for (int k = 0; k < NF + HZ2_AHEAD; ++k) stage(zs + k);
  const int lc2 = (ty + NF) * (HX / 2) + tx + NF / 2;  // this thread's pair, double2 index
  for (int z = zs; z < ze; ++z) {
    cp_wait_hz<HZ2_AHEAD - 1>();
    __syncthreads();
    stage(z + NF + HZ2_AHEAD);
    if (z == zs) {
#pragma unroll
      for (int k = 0; k < NF; ++k) q[NF + k] = hz2_sm[slot(zs + k) * PL2 + lc2];
    }
    q[2 * NF] = hz2_sm[slot(z + NF) * PL2 + lc2];
    const double2* cur = hz2_sm + slot(z) * PL2;
    double v[2 * NF + 2];  // x - NF .. x + NF + 1
#pragma unroll
    for (int k = 0; k <= NF; ++k) {
      const double2 w = cur[lc2 - NF / 2 + k];
      v[2 * k] = w.x;
      v[2 * k + 1] = w.y;
    }
    double a0 = c.cx[NF] * v[0], a1 = c.cx[NF] * v[1];
#pragma unroll
    for (int m = NF - 1; m >= 1; --m) {
      a0 = fma(c.cx[m], v[NF - m], a0);
      a1 = fma(c.cx[m], v[NF + 1 - m], a1);
    }
    a0 = fma(c.diag, v[NF], a0);
    a1 = fma(c.diag, v[NF + 1], a1);
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      a0 = fma(c.cx[m], v[NF + m], a0);
      a1 = fma(c.cx[m], v[NF + 1 + m], a1);
    }
#pragma unroll
    for (int m = NF; m >= 1; --m) {
      const double2 w = cur[lc2 - m * (HX / 2)];
      a0 = fma(c.cy[m], w.x, a0);
      a1 = fma(c.cy[m], w.y, a1);
    }
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      const double2 w = cur[lc2 + m * (HX / 2)];
      a0 = fma(c.cy[m], w.x, a0);
      a1 = fma(c.cy[m], w.y, a1);
    }
#pragma unroll
    for (int m = NF; m >= 1; --m) {
      a0 = fma(c.cz[m], q[NF - m].x, a0);
      a1 = fma(c.cz[m], q[NF - m].y, a1);
    }
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      a0 = fma(c.cz[m], q[NF + m].x, a0);
      a1 = fma(c.cz[m], q[NF + m].y, a1);
    }
    if (active) {
      const long o = (long)z * plane + own;
      if (RES) {
        const double2 bb = *reinterpret_cast<const double2*>(b + o);
        const float2 r = make_float2((float)(bb.x - a0), (float)(bb.y - a1));
        *reinterpret_cast<float2*>(out32 + o) = r;
        racc = fma((double)r.x, (double)r.x, racc);
        racc = fma((double)r.y, (double)r.y, racc);
      } else {
        *reinterpret_cast<double2*>(ap + o) = make_double2(a0, a1);
      }
    }
#pragma unroll
    for (int k = 0; k < 2 * NF; ++k) q[k] = q[k + 1];
  }
  cp_wait_hz<0>();
  if (RES) {
    // this CTA's share of r.r, summed in a fixed order (lanes, then warps)
    __shared__ double rws[HZ2_THREADS / 32];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) racc = racc + __shfl_down_sync(0xffffffffu, racc, off);
    if ((tid & 31) == 0) rws[tid >> 5] = racc;
    __syncthreads();
    if (tid == 0) {
      double t = 0.0;
#pragma unroll
      for (int w = 0; w < HZ2_THREADS / 32; ++w) t = t + rws[w];
      rpart[blockIdx.x] = t;
    }
  }
}

// chunk sums of p.ap in the reduction tree's order, from the stored ap
__global__ void __launch_bounds__(kTreeLanes) k_cg_pap(long N, const double* __restrict__ p,
                                                       const double* __restrict__ ap,
                                                       double* __restrict__ part,
                                                       const CgScalars* __restrict__ s) {
  if (s->done) return;
  __shared__ double ws[8];
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double acc = 0.0;
#pragma unroll 4
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < N) acc = fma(p[i], ap[i], acc);
  }
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// pap = fold(part); alpha = r1r / pap
__global__ void k_cg_fold_alpha(long nblk, const double* __restrict__ part, CgScalars* s) {
  if (s->done) return;
  __shared__ double ws[8];
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + part[k];
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) {
    s->pap = t;
    s->alph = s->r1r / t;
  }
}

// scf_hartee_cg_03 and the residual of scf_hartee_cg_04, with the r.r chunk sums
__global__ void __launch_bounds__(kTreeLanes) k_cg_update_rr(long N, CgScalars* s,
                                                             double* __restrict__ vh,
                                                             const double* __restrict__ p,
                                                             const double* __restrict__ ap,
                                                             double* __restrict__ avhs,
                                                             const double* __restrict__ b,
                                                             double* __restrict__ r,
                                                             double* __restrict__ part) {
  if (s->done) return;
  __shared__ double ws[8];
  const double alph = s->alph;
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double acc = 0.0;
#pragma unroll 4
  for (int k = 0; k < kTreePerLane; ++k) {
    const long i = base + (long)k * kTreeLanes;
    if (i < N) {
      vh[i] = fma(alph, p[i], vh[i]);
      const double a = fma(alph, ap[i], avhs[i]);
      avhs[i] = a;
      const double ri = b[i] - a;
      r[i] = ri;
      acc = fma(ri, ri, acc);
    }
  }
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) part[blockIdx.x] = t;
}

// r2r = fold(part); beta, dp and the stopping rule of scf_hartree_cg
// (restart every ncgres; at least ncgmin, at most ncgmax iterations)
// The iteration number is kept on the device (s->iters), so a batch of
// iterations is the same sequence of launches every time and can be replayed
// as one CUDA graph.
__global__ void k_cg_fold_beta(long nblk, const double* __restrict__ part, CgScalars* s,
                               int ncgres, int ncgmin, int ncgmax, double epsvh, double ddx,
                               double ddy, double ddz, double vol) {
  if (s->done) return;
  __shared__ double ws[8];
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + part[k];
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) {
    const int loop = s->iters + 1;
    s->r2r = t;
    double beta = t / s->r1r;
    if (loop % ncgres == 0) beta = 0.0;
    s->beta = beta;
    s->dp = sqrt(t * ddx * ddy * ddz / vol);
    s->r1r = t;
    s->iters = loop;
    bool stop = false;
    if (loop >= ncgmin) {
      if (loop >= ncgmax) stop = true;
      else if (!(s->dp > epsvh)) stop = true;
    }
    if (stop) s->done = 1;
  }
}

__global__ void k_cg_bvec(long N, const double* __restrict__ rho, double two_pi, double ddx,
                          double ddy, double ddz, double* __restrict__ b, double* __restrict__ q,
                          double* __restrict__ one) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  const double bi = two_pi * rho[i];
  b[i] = bi;
  q[i] = bi * ddx * ddy * ddz;
  one[i] = 1.0;
}

// b = b - bve/(8 xmax ymax zmax)  (scf_hartree8f.F90:667-691)
__global__ void k_cg_neutral(long N, double* __restrict__ b, const double* __restrict__ bve,
                             double vol) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  b[i] = b[i] - (*bve) / vol;
}

// avhs = Av, r = b - Av, p = r  (scf_hartee_cg_01 and the copies around it)
__global__ void k_cg_init(long N, const double* __restrict__ b, const double* __restrict__ av,
                          double* __restrict__ avhs, double* __restrict__ r,
                          double* __restrict__ p) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  avhs[i] = av[i];
  const double ri = b[i] - av[i];
  r[i] = ri;
  p[i] = ri;
}

// scf_hartee_cg_05: p = r + beta p
__global__ void k_cg_dir(long N, const CgScalars* __restrict__ s, const double* __restrict__ r,
                         double* __restrict__ p) {
  if (s->done) return;
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  p[i] = fma(s->beta, p[i], r[i]);
}

// ---------------------------------------------------------------- mixed CG
// The Hartree CG of the mixed path: the same iteration as hartree_cg (kukan's
// recurrences, restart, stopping rule, device-side folds and graph batches),
// with the vectors p, A p and r in FP32 and the solution vh, every dot
// product and every residual norm in FP64.  Between two FP64 residuals the
// solution change dvh accumulates in FP32 and is then added into vh.  The A p
// stencil is the paired z-march in FP32 and also sums p.Ap, one partial per
// CTA.
template <int NF>
__global__ void __launch_bounds__(HZ2_THREADS, 1) k_hlap_zmarch2f(int nx, int ny, int nz,
                                                                  int zchunk, HartreeCoefs c,
                                                                  const float* __restrict__ p,
                                                                  float* __restrict__ ap,
                                                                  const CgScalars* __restrict__ s,
                                                                  double* __restrict__ part) {
  static_assert(NF % 2 == 0, "float2 path needs an even halo");
  if (s->done) return;
  constexpr int HX = HZ2_TX + 2 * NF, HY = HZ2_TY + 2 * NF, PL = HX * HY, RING = hz2_ring(NF);
  constexpr int PL2 = PL / 2, NST = (PL2 + HZ2_THREADS - 1) / HZ2_THREADS;
  extern __shared__ float2 hzf_sm[];  // [RING][HY][HX / 2]
  float cx[NF + 1], cy[NF + 1], cz[NF + 1];
#pragma unroll
  for (int m = 1; m <= NF; ++m) {
    cx[m] = (float)c.cx[m];
    cy[m] = (float)c.cy[m];
    cz[m] = (float)c.cz[m];
  }
  const float diag = (float)c.diag;
  const int tid = threadIdx.x, tx = tid % (HZ2_TX / 2), ty = tid / (HZ2_TX / 2);
  const int ntx = (nx + HZ2_TX - 1) / HZ2_TX, nty = (ny + HZ2_TY - 1) / HZ2_TY;
  const int tile = blockIdx.x % (ntx * nty), zc = blockIdx.x / (ntx * nty);
  const int x0 = (tile % ntx) * HZ2_TX, y0 = (tile / ntx) * HZ2_TY;
  const int zs = zc * zchunk, ze = min(zs + zchunk, nz);
  const long plane = (long)nx * ny;
  const int gx = x0 + 2 * tx, gy = y0 + ty;
  const bool active = gx < nx && gy < ny;
  const long own = active ? (long)gy * nx + gx : 0;
  int soff[NST], doff[NST];
#pragma unroll
  for (int k = 0; k < NST; ++k) {
    const int e = tid + k * HZ2_THREADS;
    if (e < PL2) {
      const int r = e / (HX / 2), q2 = e % (HX / 2);
      soff[k] = (int)((long)wrapm(y0 - NF + r, ny) * nx + wrapm(x0 - NF + 2 * q2, nx));
      doff[k] = e;
    } else {
      soff[k] = -1;
      doff[k] = 0;
    }
  }
  auto wrapz = [&](int z) {
    while (z < 0) z += nz;
    while (z >= nz) z -= nz;
    return z;
  };
  auto slot = [&](int z) { return (z - zs + NF) % RING; };
  auto stage = [&](int z) {
    const float* src = p + (long)wrapz(z) * plane;
    float2* dst = hzf_sm + slot(z) * PL2;
#pragma unroll
    for (int k = 0; k < NST; ++k)
      if (soff[k] >= 0) cp_async8(dst + doff[k], src + soff[k]);
    cp_commit_hz();
  };
  float2 q[2 * NF + 1];
  double pacc = 0.0;  // p . A p over this thread's points
#pragma unroll
  for (int k = 0; k < NF; ++k)
    q[k] = __ldg(reinterpret_cast<const float2*>(p + (long)wrapz(zs - NF + k) * plane + own));
#pragma unroll
  for (int k = 0; k < NF + HZ2_AHEAD; ++k) stage(zs + k);
  const int lc2 = (ty + NF) * (HX / 2) + tx + NF / 2;
  for (int z = zs; z < ze; ++z) {
    cp_wait_hz<HZ2_AHEAD - 1>();
    __syncthreads();
    stage(z + NF + HZ2_AHEAD);
    if (z == zs) {
#pragma unroll
      for (int k = 0; k < NF; ++k) q[NF + k] = hzf_sm[slot(zs + k) * PL2 + lc2];
    }
    q[2 * NF] = hzf_sm[slot(z + NF) * PL2 + lc2];
    const float2* cur = hzf_sm + slot(z) * PL2;
    float v[2 * NF + 2];
#pragma unroll
    for (int k = 0; k <= NF; ++k) {
      const float2 w = cur[lc2 - NF / 2 + k];
      v[2 * k] = w.x;
      v[2 * k + 1] = w.y;
    }
    float a0 = cx[NF] * v[0], a1 = cx[NF] * v[1];
#pragma unroll
    for (int m = NF - 1; m >= 1; --m) {
      a0 = fmaf(cx[m], v[NF - m], a0);
      a1 = fmaf(cx[m], v[NF + 1 - m], a1);
    }
    a0 = fmaf(diag, v[NF], a0);
    a1 = fmaf(diag, v[NF + 1], a1);
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      a0 = fmaf(cx[m], v[NF + m], a0);
      a1 = fmaf(cx[m], v[NF + 1 + m], a1);
    }
#pragma unroll
    for (int m = NF; m >= 1; --m) {
      const float2 w = cur[lc2 - m * (HX / 2)];
      a0 = fmaf(cy[m], w.x, a0);
      a1 = fmaf(cy[m], w.y, a1);
    }
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      const float2 w = cur[lc2 + m * (HX / 2)];
      a0 = fmaf(cy[m], w.x, a0);
      a1 = fmaf(cy[m], w.y, a1);
    }
#pragma unroll
    for (int m = NF; m >= 1; --m) {
      a0 = fmaf(cz[m], q[NF - m].x, a0);
      a1 = fmaf(cz[m], q[NF - m].y, a1);
    }
#pragma unroll
    for (int m = 1; m <= NF; ++m) {
      a0 = fmaf(cz[m], q[NF + m].x, a0);
      a1 = fmaf(cz[m], q[NF + m].y, a1);
    }
    if (active) {
      *reinterpret_cast<float2*>(ap + (long)z * plane + own) = make_float2(a0, a1);
      pacc = fma((double)q[NF].x, (double)a0, pacc);
      pacc = fma((double)q[NF].y, (double)a1, pacc);
    }
#pragma unroll
    for (int k = 0; k < 2 * NF; ++k) q[k] = q[k + 1];
  }
  cp_wait_hz<0>();
  // this CTA's share of p.Ap, summed in a fixed order (warps, then lanes)
  __shared__ double ws[HZ2_THREADS / 32];
#pragma unroll
  for (int off = 16; off >= 1; off >>= 1) pacc = pacc + __shfl_down_sync(0xffffffffu, pacc, off);
  if ((tid & 31) == 0) ws[tid >> 5] = pacc;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
#pragma unroll
    for (int w = 0; w < HZ2_THREADS / 32; ++w) t = t + ws[w];
    part[blockIdx.x] = t;
  }
}

// beta, dp and the stopping rule of scf_hartree_cg from r2r (shared by the
// two folds of the mixed solve)
__device__ void cg_close_iteration(CgScalars* s, double t, int loop, int ncgres, int ncgmin,
                                   int ncgmax, double epsvh, double ddx, double ddy, double ddz,
                                   double vol) {
  s->r2r = t;
  double beta = t / s->r1r;
  if (loop % ncgres == 0) beta = 0.0;
  s->beta = beta;
  s->dp = sqrt(t * ddx * ddy * ddz / vol);
  s->r1r = t;
  s->iters = loop;
  bool stop = false;
  if (loop >= ncgmin) {
    if (loop >= ncgmax) stop = true;
    else if (!(s->dp > epsvh)) stop = true;
  }
  if (stop) s->done = 1;
}

// Mixed solve, after the FP32 update: when r.r has dropped by kReliable since
// the last FP64 residual, or the stopping test would fire, ask for the
// residual to be recomputed in FP64 (reliable update) and close the
// iteration after that; otherwise close it now.  Run by the last block of
// k_cg_update_f (kTreeLanes threads) over the nblk r.r partials, in block
// order.
constexpr double kReliable = 1e-2;  // in r.r: a factor 10 in the residual norm
struct CgFoldArgs {
  int ncgres, ncgmin, ncgmax;
  double epsvh, ddx, ddy, ddz, vol;
};
__device__ void cg_fold_beta_f(long nblk, const double* part, CgScalars* s,
                               const CgFoldArgs& f, double* ws) {
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + __ldcg(part + k);
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) {
    const int loop = s->iters + 1;
    const double dp = sqrt(t * f.ddx * f.ddy * f.ddz / f.vol);
    const bool would_stop = loop >= f.ncgmin && (loop >= f.ncgmax || !(dp > f.epsvh));
    if (t < kReliable * s->r2ref || would_stop) {
      s->upd = 1;
      s->r2r = t;
    } else {
      s->upd = 0;
      cg_close_iteration(s, t, loop, f.ncgres, f.ncgmin, f.ncgmax, f.epsvh, f.ddx, f.ddy, f.ddz,
                         f.vol);
    }
  }
}

// alpha = r.r / p.Ap from the stencil's per-CTA partials (every block folds
// them in the same order), then dvh += alpha p and r -= alpha A p (FP32, the
// same alpha) and the r.r sum of this 4096-point chunk (FP64).  V consecutive
// values per lane (V divides N).  dvh, the change of the solution since the
// last FP64 residual, is added into vh (FP64) by k_cg_fold_dvh before each
// FP64 residual.  The last block to finish (a ticket in the scalars) folds
// the r.r partials and closes or hands on the iteration (cg_fold_beta_f), so
// that fold needs no launch of its own.
template <int V>
__global__ void __launch_bounds__(kTreeLanes) k_cg_update_f(long N, CgScalars* s, long npap,
                                                            const double* __restrict__ pap_part,
                                                            float* __restrict__ dvh,
                                                            const float* __restrict__ p,
                                                            const float* __restrict__ ap,
                                                            float* __restrict__ r,
                                                            double* __restrict__ part,
                                                            CgFoldArgs fa) {
  if (s->done) return;
  __shared__ double ws[8];
  __shared__ double alph_s;
  __shared__ int last_s;
  double q = 0.0;
  for (long k = threadIdx.x; k < npap; k += kTreeLanes) q = q + pap_part[k];
  q = tree_fold256(q, ws);
  if (threadIdx.x == 0) {
    alph_s = s->r1r / q;
    if (blockIdx.x == 0) {
      s->pap = q;
      s->alph = alph_s;
    }
  }
  __syncthreads();
  const float alf = (float)alph_s;
  const long base = (long)blockIdx.x * kTreeChunk + (long)threadIdx.x * V;
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < kTreePerLane / V; ++k) {
    const long i = base + (long)k * kTreeLanes * V;
    if (i < N) {
      Pack<float, V> dv = ldpk<float, V>(dvh + i), rv = ldpk<float, V>(r + i);
      const Pack<float, V> pv = ldpk<float, V>(p + i), av = ldpk<float, V>(ap + i);
#pragma unroll
      for (int c = 0; c < V; ++c) {
        dv.v[c] = fmaf(alf, pv.v[c], dv.v[c]);
        rv.v[c] = fmaf(-alf, av.v[c], rv.v[c]);
        acc = fma((double)rv.v[c], (double)rv.v[c], acc);
      }
      stpk<float, V>(dvh + i, dv);
      stpk<float, V>(r + i, rv);
    }
  }
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) {
    part[blockIdx.x] = t;
    __threadfence();
    last_s = atomicAdd(&s->ticket, 1u) == gridDim.x - 1 ? 1 : 0;
  }
  __syncthreads();
  if (!last_s) return;
  __threadfence();
  cg_fold_beta_f(gridDim.x, part, s, fa, ws);
  if (threadIdx.x == 0) s->ticket = 0;
}

// blocks of the kernels that only run at an FP64 residual (and return at once
// otherwise): a grid-stride loop over a few waves keeps the idle launches short
constexpr unsigned kGatedBlocks = 148 * 8;

// vh += dvh (FP64), dvh = 0, when an FP64 residual follows
__global__ void k_cg_fold_dvh(long N, const CgScalars* __restrict__ s, float* __restrict__ dvh,
                              double* __restrict__ vh) {
  if (s->done || !s->upd) return;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < N;
       i += (long)gridDim.x * blockDim.x) {
    vh[i] = vh[i] + (double)dvh[i];
    dvh[i] = 0.f;
  }
}

// closes an iteration whose residual was recomputed in FP64
__global__ void k_cg_fold_upd_f(long nblk, const double* __restrict__ part, CgScalars* s,
                                int ncgres, int ncgmin, int ncgmax, double epsvh, double ddx,
                                double ddy, double ddz, double vol) {
  if (s->done || !s->upd) return;
  __shared__ double ws[8];
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + part[k];
  const double t = tree_fold256(acc, ws);
  if (threadIdx.x == 0) {
    cg_close_iteration(s, t, s->iters + 1, ncgres, ncgmin, ncgmax, epsvh, ddx, ddy, ddz, vol);
    s->r2ref = t;
    s->upd = 0;
  }
}

// p = r + beta p (FP32), V consecutive values per thread (V divides N)
template <int V>
__global__ void k_cg_dir_f(long N, const CgScalars* __restrict__ s, const float* __restrict__ r,
                           float* __restrict__ p) {
  if (s->done) return;
  const long i = ((long)blockIdx.x * blockDim.x + threadIdx.x) * V;
  if (i >= N) return;
  const float beta = (float)s->beta;
  const Pack<float, V> rv = ldpk<float, V>(r + i);
  Pack<float, V> pv = ldpk<float, V>(p + i);
#pragma unroll
  for (int k = 0; k < V; ++k) pv.v[k] = fmaf(beta, pv.v[k], rv.v[k]);
  stpk<float, V>(p + i, pv);
}

__global__ void k_to_f32x2(long N, const double* __restrict__ a, const double* __restrict__ b,
                           float* __restrict__ fa, float* __restrict__ fb) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= N) return;
  fa[i] = (float)a[i];
  fb[i] = (float)b[i];
}

__global__ void k_cg_ref(CgScalars* s) {
  s->r2ref = s->r1r;
  s->upd = 0;
  s->ticket = 0;
}

constexpr size_t hz_smem(int nf) { return sizeof(double) * hz_ring(nf) * hz_plane(nf); }
constexpr size_t hz2_smem(int nf) { return sizeof(double) * hz2_ring(nf) * hz2_plane(nf); }

// shared-memory limits of the z-march kernels (above 48 KB for nfh >= 4)
int hlap_zmarch_attr(int nfh) {
  cudaError_t e = cudaSuccess;
  switch (nfh) {
    case 1: e = cudaFuncSetAttribute(k_hlap_zmarch<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz_smem(1)); break;
    case 2: e = cudaFuncSetAttribute(k_hlap_zmarch<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz_smem(2)); break;
    case 3: e = cudaFuncSetAttribute(k_hlap_zmarch<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz_smem(3)); break;
    case 4: e = cudaFuncSetAttribute(k_hlap_zmarch<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz_smem(4)); break;
    case 5: e = cudaFuncSetAttribute(k_hlap_zmarch<5>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz_smem(5)); break;
    default: e = cudaFuncSetAttribute(k_hlap_zmarch<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz_smem(6)); break;
  }
  if (e == cudaSuccess && nfh % 2 == 0) {
    switch (nfh) {
      case 2: e = cudaFuncSetAttribute(k_hlap_zmarch2<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz2_smem(2)); break;
      case 4: e = cudaFuncSetAttribute(k_hlap_zmarch2<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz2_smem(4)); break;
      default: e = cudaFuncSetAttribute(k_hlap_zmarch2<6>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz2_smem(6)); break;
    }
  }
  return e == cudaSuccess ? RS_OK : cuda_status(e, "k_hlap_zmarch");
}

bool hartree_ap_f32_ok(int nx, int ny, int nz, int nfh);
unsigned hartree_ap_f32_ctas(int nx, int ny, int nz);
int hartree_ap_f32_attr();
int launch_hartree_ap_f32(int nx, int ny, int nz, const double* cx, const double* cy,
                          const double* cz, double diag, const float* p, float* ap,
                          const int* done, double* part, cudaStream_t st);

// work32: nullptr for the FP64 solve; 4 N floats for the mixed solve (used
// when nfh and nx are even, which its paired FP32 stencil needs; other grids
// run the FP64 iteration)
// allow_graph: false keeps every batch as plain launches on any stream (no
// graph is captured or instantiated)
int hartree_cg(int nx, int ny, int nz, int nfh, double xmax, double ymax, double zmax,
               double epsvh, int ncgmin, int ncgmax, int ncgres, const double* rho, double* vh,
               double* work, int* iters, double* dp_out, cudaStream_t st,
               float* work32, bool allow_graph) {
  const long N = (long)nx * ny * nz;
  const long nblk = tree_chunks(N);
  double* b = work;
  double* r = b + N;
  double* p = r + N;
  double* ap = p + N;
  double* avhs = ap + N;
  double* part = avhs + N;
  CgScalars* sc = (CgScalars*)(part + nblk + 1);
  // q and one reuse r and p before the iteration starts
  const double ddx = 2.0 * xmax / nx, ddy = 2.0 * ymax / ny, ddz = 2.0 * zmax / nz;
  const double pi = acos(-1.0);
  const HartreeCoefs hc = hartree_coefs(nfh, ddx, ddy, ddz);
  const unsigned gN = div_up(N, 256);
  const double vol = 8.0 * xmax * ymax * zmax;
  int rc;
  RS_CUDA(cudaMemsetAsync(sc, 0, sizeof(CgScalars), st));
  k_cg_bvec<<<gN, 256, 0, st>>>(N, rho, 2.0 * pi, ddx, ddy, ddz, b, r, p);
  if ((rc = tree_dot<double>(N, r, p, &sc->bve, part, st))) return rc;
  k_cg_neutral<<<gN, 256, 0, st>>>(N, b, &sc->bve, vol);
  RS_LAUNCH_CHECK("k_cg_neutral");
  if ((rc = launch_hartree_lap(nx, ny, nz, nfh, hc, vh, ap, st))) return rc;
  k_cg_init<<<gN, 256, 0, st>>>(N, b, ap, avhs, r, p);
  if ((rc = tree_dot<double>(N, r, r, &sc->r1r, part, st))) return rc;
  // A p by the z-march stencil, then the p.Ap chunk sums (tree order)
  const bool pairs = nfh % 2 == 0 && nx % 2 == 0;
  const int ztiles = pairs ? (int)(div_up(nx, HZ2_TX) * div_up(ny, HZ2_TY))
                           : (int)(div_up(nx, HZ_TX) * div_up(ny, HZ_TY));
  // z runs of up to 64 planes, halved (down to 8) while that leaves fewer
  // CTAs than SMs: small grids trade halo re-reads for parallelism
  int zrun = 64;
  while (zrun > 8 && (long)ztiles * ((nz + zrun - 1) / zrun) < 148) zrun /= 2;
  const int nzc = (nz + zrun - 1) / zrun;
  const int zchunk = (nz + nzc - 1) / nzc;
  const unsigned gz = (unsigned)(ztiles * nzc);
  if ((rc = hlap_zmarch_attr(nfh))) return rc;
  auto lap = [&](const double* x, double* ax) {
    if (pairs) {
      switch (nfh) {
        case 2: k_hlap_zmarch2<2><<<gz, HZ2_THREADS, hz2_smem(2), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
        case 4: k_hlap_zmarch2<4><<<gz, HZ2_THREADS, hz2_smem(4), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
        default: k_hlap_zmarch2<6><<<gz, HZ2_THREADS, hz2_smem(6), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
      }
      k_cg_pap<<<(unsigned)nblk, kTreeLanes, 0, st>>>(N, x, ax, part, sc);
      return;
    }
    switch (nfh) {
      case 1: k_hlap_zmarch<1><<<gz, HZ_THREADS, hz_smem(1), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
      case 2: k_hlap_zmarch<2><<<gz, HZ_THREADS, hz_smem(2), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
      case 3: k_hlap_zmarch<3><<<gz, HZ_THREADS, hz_smem(3), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
      case 4: k_hlap_zmarch<4><<<gz, HZ_THREADS, hz_smem(4), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
      case 5: k_hlap_zmarch<5><<<gz, HZ_THREADS, hz_smem(5), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
      default: k_hlap_zmarch<6><<<gz, HZ_THREADS, hz_smem(6), st>>>(nx, ny, nz, zchunk, hc, x, ax, sc); break;
    }
    k_cg_pap<<<(unsigned)nblk, kTreeLanes, 0, st>>>(N, x, ax, part, sc);
  };
  CgScalars hs;
  hs.done = 0;
  const int lmax = ncgmax > ncgmin ? ncgmax : ncgmin;
  // batches of kCgBatch iterations; every kernel returns at once after the
  // stopping test has fired, so a batch may run past the last iteration.  On
  // a stream other than the legacy one the batch is captured once as a CUDA
  // graph and replayed.
  const bool mixed = work32 != nullptr && pairs;
  // nfh = 4 grids with x in whole 16-byte vectors take the 4 x 2 point z-march
  // of H psi for A p; the others the paired Hartree z-march
  const bool wide_ap = mixed && hartree_ap_f32_ok(nx, ny, nz, nfh);
  const unsigned nap = wide_ap ? hartree_ap_f32_ctas(nx, ny, nz) : gz;
  float *fr = nullptr, *fp = nullptr, *fap = nullptr, *fdv = nullptr;
  if (mixed) {
    fr = work32;
    fp = fr + N;
    fap = fp + N;
    fdv = fap + N;
    RS_CUDA(cudaMemsetAsync(fdv, 0, sizeof(float) * N, st));
    k_to_f32x2<<<gN, 256, 0, st>>>(N, r, p, fr, fp);
    k_cg_ref<<<1, 1, 0, st>>>(sc);
    cudaError_t e = cudaFuncSetAttribute(
        nfh == 2 ? (const void*)k_hlap_zmarch2f<2>
                 : (nfh == 4 ? (const void*)k_hlap_zmarch2f<4> : (const void*)k_hlap_zmarch2f<6>),
        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(hz2_smem(nfh) / 2));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(
          nfh == 2 ? (const void*)k_hlap_zmarch2<2, true>
                   : (nfh == 4 ? (const void*)k_hlap_zmarch2<4, true>
                               : (const void*)k_hlap_zmarch2<6, true>),
          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hz2_smem(nfh));
    if (e != cudaSuccess) return cuda_status(e, "mixed Hartree CG kernels");
    if (wide_ap && (rc = hartree_ap_f32_attr())) return rc;
  }
  // one mixed iteration: FP32 A p and update, then (when asked) the FP64
  // residual b - A vh rounded into r, its r.r, and the closing fold
  auto iter32 = [&]() {
    if (wide_ap)
      launch_hartree_ap_f32(nx, ny, nz, hc.cx, hc.cy, hc.cz, hc.diag, fp, fap, &sc->done, ap, st);
    else switch (nfh) {
      case 2: k_hlap_zmarch2f<2><<<gz, HZ2_THREADS, hz2_smem(2) / 2, st>>>(nx, ny, nz, zchunk, hc, fp, fap, sc, ap); break;
      case 4: k_hlap_zmarch2f<4><<<gz, HZ2_THREADS, hz2_smem(4) / 2, st>>>(nx, ny, nz, zchunk, hc, fp, fap, sc, ap); break;
      default: k_hlap_zmarch2f<6><<<gz, HZ2_THREADS, hz2_smem(6) / 2, st>>>(nx, ny, nz, zchunk, hc, fp, fap, sc, ap); break;
    }
    // p.Ap: one partial per stencil CTA (in the FP64 A p array, which the
    // mixed iteration leaves unused), folded by every block of the update
    const CgFoldArgs fa{ncgres, ncgmin, lmax, epsvh, ddx, ddy, ddz, vol};
    if (N % 4 == 0)
      k_cg_update_f<4><<<(unsigned)nblk, kTreeLanes, 0, st>>>(N, sc, (long)nap, ap, fdv, fp, fap,
                                                              fr, part, fa);
    else
      k_cg_update_f<1><<<(unsigned)nblk, kTreeLanes, 0, st>>>(N, sc, (long)nap, ap, fdv, fp, fap,
                                                              fr, part, fa);
    k_cg_fold_dvh<<<std::min(gN, kGatedBlocks), 256, 0, st>>>(N, sc, fdv, vh);
    // the FP64 residual rounded into r, with its r.r partials per CTA (in the
    // FP64 A p array too: the update has consumed the p.Ap partials by now)
    switch (nfh) {
      case 2: k_hlap_zmarch2<2, true><<<gz, HZ2_THREADS, hz2_smem(2), st>>>(nx, ny, nz, zchunk, hc, vh, nullptr, sc, b, fr, ap); break;
      case 4: k_hlap_zmarch2<4, true><<<gz, HZ2_THREADS, hz2_smem(4), st>>>(nx, ny, nz, zchunk, hc, vh, nullptr, sc, b, fr, ap); break;
      default: k_hlap_zmarch2<6, true><<<gz, HZ2_THREADS, hz2_smem(6), st>>>(nx, ny, nz, zchunk, hc, vh, nullptr, sc, b, fr, ap); break;
    }
    k_cg_fold_upd_f<<<1, kTreeLanes, 0, st>>>((long)gz, ap, sc, ncgres, ncgmin, lmax, epsvh,
                                              ddx, ddy, ddz, vol);
    if (N % 4 == 0) k_cg_dir_f<4><<<div_up(N / 4, 256), 256, 0, st>>>(N, sc, fr, fp);
    else k_cg_dir_f<1><<<gN, 256, 0, st>>>(N, sc, fr, fp);
  };
  auto batch = [&]() {
    for (int l = 0; l < kCgBatch; ++l) {
      if (mixed) {
        iter32();
        continue;
      }
      lap(p, ap);
      k_cg_fold_alpha<<<1, kTreeLanes, 0, st>>>(nblk, part, sc);
      k_cg_update_rr<<<(unsigned)nblk, kTreeLanes, 0, st>>>(N, sc, vh, p, ap, avhs, b, r, part);
      k_cg_fold_beta<<<1, kTreeLanes, 0, st>>>(nblk, part, sc, ncgres, ncgmin, lmax, epsvh,
                                               ddx, ddy, ddz, vol);
      k_cg_dir<<<gN, 256, 0, st>>>(N, sc, r, p);
    }
  };
  cudaGraphExec_t exec = nullptr;
  if (st != nullptr && allow_graph) {
    cudaGraph_t gph = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      batch();
      cudaError_t e = cudaStreamEndCapture(st, &gph);
      if (e == cudaSuccess && cudaGraphInstantiate(&exec, gph, 0) != cudaSuccess) exec = nullptr;
      if (gph) cudaGraphDestroy(gph);
    }
    cudaGetLastError();  // a failed capture falls back to plain launches
  }
  rc = RS_OK;
  for (int loop = 1; loop <= lmax && !hs.done; loop += kCgBatch) {
    if (exec) {
      const cudaError_t e = cudaGraphLaunch(exec, st);
      if (e != cudaSuccess) { rc = cuda_status(e, "hartree_cg graph"); break; }
    } else {
      batch();
    }
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) { rc = cuda_status(e, "hartree_cg iteration"); break; }
    if (cudaMemcpyAsync(&hs, sc, sizeof(CgScalars), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess) {
      rc = cuda_status(cudaGetLastError(), "hartree_cg");
      break;
    }
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (rc) return rc;
  if (iters) *iters = hs.iters;
  if (dp_out) *dp_out = hs.dp;
  return RS_OK;
}

}  // namespace rs

extern "C" int rs_dot_f64(long n, const double* a, const double* b, double* out, void* stream) {
  cudaStream_t st = rs::as_stream(stream);
  const long nblk = rs::tree_chunks(n);
  double* part = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * (nblk + 1), st));
  int rc = rs::tree_dot<double>(n, a, b, out, part, st);
  cudaFreeAsync(part, st);
  return rc;
}

extern "C" int rs_dot_f32(long n, const float* a, const float* b, double* out, void* stream) {
  cudaStream_t st = rs::as_stream(stream);
  const long nblk = rs::tree_chunks(n);
  double* part = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&part, sizeof(double) * (nblk + 1), st));
  int rc = rs::tree_dot<float>(n, a, b, out, part, st);
  cudaFreeAsync(part, st);
  return rc;
}

extern "C" int rs_density_f64(long N, int nb, const double* occ, const double* psi, double* rho,
                              void* stream) {
  if (N <= 0 || nb < 0) return rs::fail(RS_EINVAL, "rs_density_f64: bad sizes");
  rs::k_density<double><<<rs::div_up(N, 256), 256, 0, rs::as_stream(stream)>>>(N, nb, occ, psi,
                                                                               rho);
  RS_LAUNCH_CHECK("k_density");
  return RS_OK;
}

extern "C" int rs_density_f32(long N, int nb, const double* occ, const float* psi, double* rho,
                              void* stream) {
  if (N <= 0 || nb < 0) return rs::fail(RS_EINVAL, "rs_density_f32: bad sizes");
  rs::k_density<float><<<rs::div_up(N, 256), 256, 0, rs::as_stream(stream)>>>(N, nb, occ, psi,
                                                                              rho);
  RS_LAUNCH_CHECK("k_density");
  return RS_OK;
}

namespace rs {
namespace {
// scf_charge_atomicocc (scf_charge8f.F90:146-213), real bands, one spin: one
// thread per (atom, packed pair i <= j), the bands summed in order with one
// fma each, as the Fortran loop does.
__global__ void k_atomicocc(int natom, int nprjmx, const int* __restrict__ nprj, int M,
                            const double* __restrict__ rp, const double* __restrict__ fnele,
                            double* __restrict__ atocc) {
  const int npack = nprjmx * (nprjmx + 1) / 2;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)natom * npack) return;
  const int a = (int)(idx / npack), ij = (int)(idx % npack);
  int j = 0;
  while ((j + 1) * (j + 2) / 2 <= ij) ++j;
  const int i = ij - j * (j + 1) / 2;
  double acc = 0.0;
  if (j < nprj[a]) {
    for (int l = 0; l < M; ++l) {
      const double* r = rp + ((long)l * natom + a) * nprjmx;
      double t = r[i] * r[j];
      if (i != j) t = 2.0 * t;
      acc = fma(fnele[l], t, acc);
    }
  }
  atocc[idx] = acc;
}
}  // namespace
}  // namespace rs

extern "C" int rs_atomicocc(const rs_geom* g, const double* rp, const double* fnele, int M,
                            double* atocc, void* stream) {
  if (!g || M < 0 || (M > 0 && (!rp || !fnele)) || !atocc)
    return rs::fail(RS_EINVAL, "rs_atomicocc: bad arguments");
  const long n = (long)g->natom * (g->nprjmx * (g->nprjmx + 1) / 2);
  if (n == 0) return RS_OK;
  rs::k_atomicocc<<<rs::div_up(n, 128), 128, 0, rs::as_stream(stream)>>>(
      g->natom, g->nprjmx, g->d_nprj, M, rp, fnele, atocc);
  RS_LAUNCH_CHECK("k_atomicocc");
  return RS_OK;
}

extern "C" int rs_interp_c2d(int nx, int ny, int nz, int nf, const double* in, double* out,
                             void* stream) {
  if (nf < 1 || nf > 8 || nx < 2 * nf || ny < 2 * nf || nz < 2 * nf)
    return rs::fail(RS_EINVAL, "rs_interp_c2d: bad grid or nf");
  cudaStream_t st = rs::as_stream(stream);
  const rs::InterpW W = rs::interp_weights(nf);
  double *t1 = nullptr, *t2 = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&t1, sizeof(double) * 2L * nx * ny * nz, st));
  RS_CUDA(cudaMallocAsync((void**)&t2, sizeof(double) * 4L * nx * ny * nz, st));
  const long n1 = 2L * nx * ny * nz, n2 = 4L * nx * ny * nz, n3 = 8L * nx * ny * nz;
  rs::k_interp_pass<<<rs::div_up(n1, 256), 256, 0, st>>>(2 * nx, ny, nz, nx, ny, nz, 0, nf, W,
                                                         in, t1);
  rs::k_interp_pass<<<rs::div_up(n2, 256), 256, 0, st>>>(2 * nx, 2 * ny, nz, 2 * nx, ny, nz, 1,
                                                         nf, W, t1, t2);
  rs::k_interp_pass<<<rs::div_up(n3, 256), 256, 0, st>>>(2 * nx, 2 * ny, 2 * nz, 2 * nx, 2 * ny,
                                                         nz, 2, nf, W, t2, out);
  cudaError_t e = cudaGetLastError();
  cudaFreeAsync(t1, st);
  cudaFreeAsync(t2, st);
  if (e != cudaSuccess) return rs::cuda_status(e, "k_interp_pass");
  return RS_OK;
}

extern "C" int rs_hartree_cg_f32(int nx, int ny, int nz, int nfh, double xmax, double ymax,
                                 double zmax, double epsvh, int ncgmin, int ncgmax, int ncgres,
                                 const double* rho, double* vh, int* iters, double* dp,
                                 void* stream) {
  if (nfh < 1 || nfh > 6 || nx <= 2 * nfh || ny <= 2 * nfh || nz <= 2 * nfh)
    return rs::fail(RS_EINVAL, "rs_hartree_cg_f32: bad grid or nfh");
  if (ncgres <= 0 || ncgmax <= 0)
    return rs::fail(RS_EINVAL, "rs_hartree_cg_f32: bad iteration limits");
  if ((long)nx * ny * nz > 2147483647L)
    return rs::fail(RS_EINVAL, "rs_hartree_cg_f32: the dense grid must have fewer than 2^31 points");
  cudaStream_t st = rs::as_stream(stream);
  const long N = (long)nx * ny * nz;
  const long nblk = rs::tree_chunks(N);
  const size_t bytes64 = sizeof(double) * (5 * N + nblk + 1) + 2 * sizeof(double) * 8;
  const size_t bytes = bytes64 + sizeof(float) * 4 * N + 16;
  double* work = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&work, bytes, st));
  float* work32 = (float*)(((uintptr_t)work + bytes64 + 15) & ~(uintptr_t)15);
  int rc = rs::hartree_cg(nx, ny, nz, nfh, xmax, ymax, zmax, epsvh, ncgmin, ncgmax, ncgres, rho,
                          vh, work, iters, dp, st, work32, true);
  cudaFreeAsync(work, st);
  return rc;
}

extern "C" int rs_hartree_cg(int nx, int ny, int nz, int nfh, double xmax, double ymax,
                             double zmax, double epsvh, int ncgmin, int ncgmax, int ncgres,
                             const double* rho, double* vh, int* iters, double* dp,
                             void* stream) {
  if (nfh < 1 || nfh > 6 || nx <= 2 * nfh || ny <= 2 * nfh || nz <= 2 * nfh)
    return rs::fail(RS_EINVAL, "rs_hartree_cg: bad grid or nfh");
  if (ncgres <= 0 || ncgmax <= 0) return rs::fail(RS_EINVAL, "rs_hartree_cg: bad iteration limits");
  if ((long)nx * ny * nz > 2147483647L)
    return rs::fail(RS_EINVAL, "rs_hartree_cg: the dense grid must have fewer than 2^31 points");
  cudaStream_t st = rs::as_stream(stream);
  const long N = (long)nx * ny * nz;
  const long nblk = rs::tree_chunks(N);
  const size_t bytes = sizeof(double) * (5 * N + nblk + 1) + 2 * sizeof(double) * 8;
  double* work = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&work, bytes, st));
  int rc = rs::hartree_cg(nx, ny, nz, nfh, xmax, ymax, zmax, epsvh, ncgmin, ncgmax, ncgres, rho,
                          vh, work, iters, dp, st, nullptr, true);
  cudaFreeAsync(work, st);
  if (rc == RS_OK && iters && *iters >= ncgmax && dp && *dp > epsvh) {
    rs::set_error("rs_hartree_cg: ncgmax reached");
  }
  return rc;
}
