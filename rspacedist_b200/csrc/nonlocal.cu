// nonlocal.cu -- nonlocal projector kernels and the fused H*psi / S*psi.
//
//  * nonlocal_dot: <p_j,a|psi_b> as one sequential fma chain per
//    (atom, projector, band) over the atom's sphere list -- the order of a
//    single-threaded nonlocaloperation_r_01 (nonlocaloperation8f.F90:34-40).
//  * t coefficients: t_i = (sum_j rp_j m(j,i)) * (1/dV)
//    (nonlocaloperation8f.F90:188-204).
//  * apply / fused H*psi: the atom-ordered scatter-add of
//    nonlocaloperation_r_02 (:206-226) is evaluated as a gather over each
//    point's inverse list, whose entries are sorted by (atom, list index), so
//    every point receives its contributions in the reference's order without
//    atomics.
#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {

// ---------------------------------------------------------------- dot
// FP64: thread (j, band) of block (atom, band group) runs the reference's
// sequential fma chain over the atom's nonzero list positions only (a
// skipped position would add fma(0, x, acc) == acc).
__global__ void k_nl_dot_f64(int natom, int nprjmx, const int* __restrict__ nprj,
                             const int* __restrict__ nz_off, const int* __restrict__ nz_pt,
                             const double* __restrict__ nz_v, const double* __restrict__ psi,
                             long N, int nb, double* __restrict__ rp) {
  const int a = blockIdx.x;
  const int bpb = blockDim.x / nprjmx;
  const int j = threadIdx.x % nprjmx, bl = threadIdx.x / nprjmx;
  const int b = blockIdx.y * bpb + bl;
  if (bl >= bpb || b >= nb) return;
  double acc = 0.0;
  if (j < nprj[a]) {
    const int e0 = nz_off[a], e1 = nz_off[a + 1];
    const double* x = psi + (long)b * N;
    for (int e = e0; e < e1; ++e)
      acc = fma(__ldg(nz_v + (long)e * nprjmx + j), __ldg(x + __ldg(nz_pt + e)), acc);
  }
  rp[((long)b * natom + a) * nprjmx + j] = acc;
}

// FP32 psi: CTA (atom, 32 bands).  Chunks of 64 list positions are staged in
// shared memory (psi gathered per band along the list, projector values
// contiguous); thread (band, j-group) accumulates its dots over the chunk in
// FP32 and adds the chunk sum into an FP64 total.
constexpr int DOT_BANDS = 32;
constexpr int DOT_CHUNK = 64;
constexpr int DOT_MAXP = 16;

__global__ void __launch_bounds__(256) k_nl_dot_f32(
    int natom, int nprjmx, const int* __restrict__ nprj, const int* __restrict__ nz_off,
    const int* __restrict__ nz_pt, const float* __restrict__ nz_v, const float* __restrict__ psi,
    long N, int nb, double* __restrict__ rp) {
  __shared__ float xs[DOT_CHUNK][DOT_BANDS + 1];
  __shared__ float vs[DOT_CHUNK][DOT_MAXP];
  __shared__ int ps[DOT_CHUNK];
  const int a = blockIdx.x;
  const int b0 = blockIdx.y * DOT_BANDS;
  const int t = threadIdx.x;
  const int bl = t % DOT_BANDS, jg = t / DOT_BANDS;  // 8 j-groups
  const int P = nprj[a];
  const int e0 = nz_off[a], e1 = nz_off[a + 1];
  double tot[2] = {0.0, 0.0};
  for (int c0 = e0; c0 < e1; c0 += DOT_CHUNK) {
    const int n = min(DOT_CHUNK, e1 - c0);
    if (t < n) ps[t] = __ldg(nz_pt + c0 + t);
    for (int i = t; i < n * nprjmx && i < DOT_CHUNK * DOT_MAXP; i += blockDim.x)
      vs[i / nprjmx][i % nprjmx] = __ldg(nz_v + (long)c0 * nprjmx + i);
    __syncthreads();
    // gather: warp w takes bands w, w+8, ...; lanes run along the list
    for (int i = t; i < DOT_CHUNK * DOT_BANDS; i += blockDim.x) {
      const int e = i % DOT_CHUNK, bb = i / DOT_CHUNK;
      const int b = b0 + bb;
      xs[e][bb] = (b < nb && e < n) ? __ldg(psi + (long)b * N + ps[e]) : 0.f;
    }
    __syncthreads();
    float s0 = 0.f, s1 = 0.f;
    const int j0 = jg, j1 = jg + 8;
    for (int e = 0; e < n; ++e) {
      const float x = xs[e][bl];
      s0 = fmaf(vs[e][j0], x, s0);
      if (j1 < DOT_MAXP) s1 = fmaf(vs[e][j1], x, s1);
    }
    tot[0] += (double)s0;
    tot[1] += (double)s1;
    __syncthreads();
  }
  const int b = b0 + bl;
  if (b < nb) {
    double* r = rp + ((long)b * natom + a) * nprjmx;
    if (jg < nprjmx) r[jg] = jg < P ? tot[0] : 0.0;
    if (jg + 8 < nprjmx) r[jg + 8] = jg + 8 < P ? tot[1] : 0.0;
  }
}

// ---------------------------------------------------------------- t coefficients
template <class TC>
__global__ void k_tcoef(int natom, int nprjmx, const int* __restrict__ nprj,
                        const double* __restrict__ mat, const double* __restrict__ rp,
                        double dxyzin, int nb, TC* __restrict__ t) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)nb * natom * nprjmx;
  if (idx >= total) return;
  const int i = (int)(idx % nprjmx);
  const long ba = idx / nprjmx;
  const int a = (int)(ba % natom);
  const int P = nprj[a];
  double s = 0.0;
  if (i < P) {
    const double* r = rp + ba * nprjmx;
    const double* m = mat + ((long)a * nprjmx + i) * nprjmx;
    for (int j = 0; j < P; ++j) s = fma(r[j], m[j], s);
    s = s * dxyzin;
  }
  t[idx] = (TC)s;
}

// avr of one inverse-list entry: t_1 p_1 + t_2 p_2 + ... (first term a product)
template <class T>
__device__ __forceinline__ T entry_avr(const T* __restrict__ tv, const T* __restrict__ pv,
                                       int P) {
  T avr = tv[0] * __ldg(pv);
  for (int j = 1; j < P; ++j) avr = fma(tv[j], __ldg(pv + j), avr);
  return avr;
}

// mode 0: out = base(out) + NL                  (nonlocal apply)
// mode 1: out = NL + stencil (H psi, base 0)    (fused)
// mode 2: out = psi + NL                        (S psi)
template <class T, int MODE>
__global__ void k_nl_gather(StencilArgs<T> s, const int* __restrict__ inv_off,
                            const int* __restrict__ inv_atom, const T* __restrict__ inv_v,
                            int nprjmx, int natom, const int* __restrict__ nprj,
                            const T* __restrict__ tco, const T* __restrict__ psi,
                            const T* __restrict__ veff, T* __restrict__ out, int nb, int bpb) {
  const long N = (long)s.nx * s.ny * s.nz;
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int ix = (int)(p % s.nx), iy = (int)((p / s.nx) % s.ny),
            iz = (int)(p / ((long)s.nx * s.ny));
  const int e0 = inv_off[p], e1 = inv_off[p + 1];
  const T vloc = MODE == 1 ? veff[p] : (T)0;
  const int b0 = blockIdx.y * bpb;
  const int b1 = min(b0 + bpb, nb);
  for (int b = b0; b < b1; ++b) {
    T acc;
    if (MODE == 0) acc = out[(long)b * N + p];
    else if (MODE == 1) acc = (T)0;
    else acc = psi[(long)b * N + p];
    for (int e = e0; e < e1; ++e) {
      const int a = __ldg(inv_atom + e);
      const int P = __ldg(nprj + a);
      if (P <= 0) continue;
      const T avr = entry_avr<T>(tco + ((long)b * natom + a) * nprjmx, inv_v + (long)e * nprjmx, P);
      acc = acc + avr;
    }
    if (MODE == 1) acc = stencil_point<T>(s, psi + (long)b * N, ix, iy, iz, vloc, acc);
    out[(long)b * N + p] = acc;
  }
}

// ---------------------------------------------------------------- launchers
template <class T>
int launch_nl_dot(const rs_geom* g, const T* psi, int nb, double* rp, cudaStream_t st) {
  if (nb <= 0 || g->natom == 0) return RS_OK;
  const int P = g->nprjmx;
  if constexpr (sizeof(T) == 8) {
    const int bpb = P > 128 ? 1 : 128 / P;
    dim3 grid(g->natom, div_up(nb, bpb));
    k_nl_dot_f64<<<grid, bpb * P, 0, st>>>(g->natom, P, g->d_nprj, g->d_nz_off, g->d_nz_pt,
                                          g->d_nz_v64, (const double*)psi, g->N, nb, rp);
  } else {
    if (P > DOT_MAXP) return fail(RS_EINVAL, "nonlocal dot: more than 16 projectors per atom");
    dim3 grid(g->natom, div_up(nb, DOT_BANDS));
    k_nl_dot_f32<<<grid, 256, 0, st>>>(g->natom, P, g->d_nprj, g->d_nz_off, g->d_nz_pt,
                                       g->d_nz_v32, (const float*)psi, g->N, nb, rp);
  }
  RS_LAUNCH_CHECK("k_nl_dot");
  return RS_OK;
}

// t coefficients into a stream-ordered temporary
template <class T>
static int make_tcoef(const rs_geom* g, const double* mat, const double* rp, int nb, T** t,
                      cudaStream_t st) {
  const long n = (long)nb * g->natom * g->nprjmx;
  *t = nullptr;
  if (n == 0) return RS_OK;
  RS_CUDA(cudaMallocAsync((void**)t, n * sizeof(T), st));
  const double dxyzin = 1.0 / (g->dx * g->dy * g->dz);
  k_tcoef<T><<<div_up(n, 256), 256, 0, st>>>(g->natom, g->nprjmx, g->d_nprj, mat, rp, dxyzin,
                                             nb, *t);
  RS_LAUNCH_CHECK("k_tcoef");
  return RS_OK;
}

// ---------------------------------------------------- FP64 H psi, z-march form
// The same sums as k_nl_gather<double, 1>, in the same order, over two
// kernels:
// 1. k_nl_sum_f64: for every covered point and band, nl = 0 + avr_e1 +
//    avr_e2 + ... over the point's entries in order, written to out;
// 2. k_stencil_f64_zmarch: one CTA owns a 32 x 16 tile of an xy plane of one
//    band and marches along z.  A thread holds 2 x-points of one row; the
//    nine planes z-4..z+4 of its points sit in a register queue, and whole
//    halo'd planes are staged in an 8-slot shared ring by cp.async, 3 planes
//    ahead.  Each point starts from nl (covered points) or 0 and adds the x
//    terms with the diagonal, then y, then z, one fma each -- the order of
//    stencil_point -- so the result equals the gather's bit for bit while psi
//    crosses HBM once instead of being gathered 25 times per point.
constexpr int D_TX = 32, D_TY = 16, D_NTX = D_TX / 2;
constexpr int D_THREADS = D_NTX * D_TY;  // 256
constexpr int D_HX = D_TX + 8, D_HY = D_TY + 8;
constexpr int D_RING = 8, D_AHEAD = 3;
constexpr int NLS_BANDS = 8;

__global__ void __launch_bounds__(128) k_nl_sum_f64(
    const int* __restrict__ cov, const int* __restrict__ cov_off, long ncov,
    const int* __restrict__ inv_atom, const double* __restrict__ inv_v, int nprjmx,
    int natom, const int* __restrict__ nprj, const double* __restrict__ tco, long N, int nb,
    double* __restrict__ out) {
  const long c = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncov) return;
  const int b0 = blockIdx.y * NLS_BANDS;
  const int b1 = min(b0 + NLS_BANDS, nb);
  const int p = __ldg(cov + c);
  const int e0 = __ldg(cov_off + c), e1 = __ldg(cov_off + c + 1);
  for (int b = b0; b < b1; ++b) {
    double acc = 0.0;
    for (int e = e0; e < e1; ++e) {
      const int a = __ldg(inv_atom + e);
      const int P = __ldg(nprj + a);
      if (P <= 0) continue;
      acc = acc + entry_avr<double>(tco + ((long)b * natom + a) * nprjmx,
                                    inv_v + (long)e * nprjmx, P);
    }
    out[(long)b * N + p] = acc;
  }
}

struct St64 {
  int nx, ny, nz, zchunk, ntx, nty;
  double cx[5], cy[5], cz[5], c0;
  const double* psi;
  double* out;
  const double* veff;
  const int* inv_off;
};

__device__ __forceinline__ int wrap1(int i, int n) {
  return i < 0 ? i + n : (i >= n ? i - n : i);
}
__device__ __forceinline__ void cp16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_commit64() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait64() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

__global__ void __launch_bounds__(D_THREADS, 2) k_stencil_f64_zmarch(St64 a) {
  extern __shared__ __align__(16) double dsm[];
  double (*pl)[D_HY][D_HX] = reinterpret_cast<double (*)[D_HY][D_HX]>(dsm);
  const int tid = threadIdx.x;
  const int tx = tid % D_NTX, ty = tid / D_NTX;
  const int ntile = a.ntx * a.nty;
  const int tile = blockIdx.x % ntile;
  const int zc = blockIdx.x / ntile;
  const int band = blockIdx.y;
  const int x0 = (tile % a.ntx) * D_TX, y0 = (tile / a.ntx) * D_TY;
  const int nx = a.nx, ny = a.ny, nz = a.nz;
  const long plane = (long)nx * ny;
  const long N = plane * nz;
  const double* psi = a.psi + (long)band * N;
  double* out = a.out + (long)band * N;
  const int zs = zc * a.zchunk;
  const int ze = min(zs + a.zchunk, nz);
  const int gx = x0 + 2 * tx, gy = y0 + ty;
  const bool active = gx < nx && gy < ny;  // nx even
  const int w = min(D_TX, nx - x0), hgt = min(D_TY, ny - y0);
  const long own = (long)gy * nx + gx;
  const int lx = 2 * tx + 4, ly = ty + 4;
  // the 16-byte halo piece this thread stages for every plane (or none):
  // x halos of the tile's rows, then y halos of its columns
  int h_src = -1, h_row = 0, h_col = 0;
  if (tid < 4 * D_TY) {
    const int side = tid / (2 * D_TY), r = (tid / 2) % D_TY, ch = tid % 2;
    if (r < hgt) {
      const int xs = side == 0 ? wrap1(x0 - 4 + 2 * ch, nx) : wrap1(x0 + w + 2 * ch, nx);
      h_src = (y0 + r) * nx + xs;
      h_row = r + 4;
      h_col = side == 0 ? 2 * ch : w + 4 + 2 * ch;
    }
  } else if (tid < 4 * D_TY + 8 * D_NTX) {
    const int j = tid - 4 * D_TY;
    const int c = j % D_NTX, rr = (j / D_NTX) % 4, side = j / (4 * D_NTX);
    if (2 * c < w) {
      const int ys = side == 0 ? wrap1(y0 - 4 + rr, ny) : wrap1(y0 + hgt + rr, ny);
      h_src = ys * nx + x0 + 2 * c;
      h_row = side == 0 ? rr : hgt + 4 + rr;
      h_col = 4 + 2 * c;
    }
  }
  auto plane_ptr = [&](int z) { return psi + (long)wrap1(z, nz) * plane; };
  auto stage = [&](int z) {
    const double* pp = plane_ptr(z);
    double(*sl)[D_HX] = pl[z & (D_RING - 1)];
    if (active) cp16(&sl[ly][lx], pp + own);
    if (h_src >= 0) cp16(&sl[h_row][h_col], pp + h_src);
    cp_commit64();
  };
  double2 q[9];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    q[k] = active ? __ldg(reinterpret_cast<const double2*>(plane_ptr(zs - 4 + k) + own))
                  : make_double2(0.0, 0.0);
#pragma unroll
  for (int k = 0; k < 4 + D_AHEAD; ++k) stage(zs + k);
  cp_wait64<D_AHEAD>();
  __syncthreads();
#pragma unroll
  for (int k = 4; k < 8; ++k)
    q[k] = *reinterpret_cast<const double2*>(&pl[(zs + k - 4) & (D_RING - 1)][ly][lx]);
  for (int z = zs; z < ze; ++z) {
    stage(z + 4 + D_AHEAD);
    cp_wait64<D_AHEAD>();
    const double(*cur)[D_HX] = pl[z & (D_RING - 1)];
    q[8] = *reinterpret_cast<const double2*>(&pl[(z + 4) & (D_RING - 1)][ly][lx]);
    if (active) {
      const long p = (long)z * plane + own;
      const double2 v2 = __ldg(reinterpret_cast<const double2*>(a.veff + p));
      const int o0 = __ldg(a.inv_off + p), o1 = __ldg(a.inv_off + p + 1),
                o2 = __ldg(a.inv_off + p + 2);
      double xv[10];
#pragma unroll
      for (int k = 0; k < 10; ++k) xv[k] = cur[ly][lx - 4 + k];
      double acc[2];
      acc[0] = o1 > o0 ? out[p] : 0.0;
      acc[1] = o2 > o1 ? out[p + 1] : 0.0;
      const double vv[2] = {v2.x, v2.y};
#pragma unroll
      for (int i = 0; i < 2; ++i) {
        double s = acc[i];
#pragma unroll
        for (int m = 4; m >= 1; --m) s = fma(a.cx[m], xv[4 + i - m], s);
        s = fma(a.c0 + vv[i], xv[4 + i], s);
#pragma unroll
        for (int m = 1; m <= 4; ++m) s = fma(a.cx[m], xv[4 + i + m], s);
        acc[i] = s;
      }
#pragma unroll
      for (int m = 4; m >= 1; --m) {
        const double2 v = *reinterpret_cast<const double2*>(&cur[ly - m][lx]);
        acc[0] = fma(a.cy[m], v.x, acc[0]);
        acc[1] = fma(a.cy[m], v.y, acc[1]);
      }
#pragma unroll
      for (int m = 1; m <= 4; ++m) {
        const double2 v = *reinterpret_cast<const double2*>(&cur[ly + m][lx]);
        acc[0] = fma(a.cy[m], v.x, acc[0]);
        acc[1] = fma(a.cy[m], v.y, acc[1]);
      }
#pragma unroll
      for (int m = 4; m >= 1; --m) {
        acc[0] = fma(a.cz[m], q[4 - m].x, acc[0]);
        acc[1] = fma(a.cz[m], q[4 - m].y, acc[1]);
      }
#pragma unroll
      for (int m = 1; m <= 4; ++m) {
        acc[0] = fma(a.cz[m], q[4 + m].x, acc[0]);
        acc[1] = fma(a.cz[m], q[4 + m].y, acc[1]);
      }
      *reinterpret_cast<double2*>(out + p) = make_double2(acc[0], acc[1]);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) q[k] = q[k + 1];
    __syncthreads();
  }
  cp_wait64<0>();
}

// true when the FP64 fused H psi takes the z-march (nf = 4, x even, grid
// larger than the stencil reach on every axis)
bool hpsi_f64_zmarch_ok(const rs_geom* g, int nb) {
  return g->nf == 4 && g->nx % 2 == 0 && g->nx >= 8 && g->ny >= 8 && g->nz >= 8 &&
         nb <= 65535 && g->N < (1L << 31);
}

int launch_hpsi_f64_zmarch(const rs_geom* g, const double* t, const double* psi,
                           const double* veff, double* out, int nb, cudaStream_t st) {
  if (g->natom > 0 && g->n_cov > 0) {
    dim3 g1(div_up(g->n_cov, 128), div_up(nb, NLS_BANDS));
    k_nl_sum_f64<<<g1, 128, 0, st>>>(g->d_cov, g->d_cov_off, g->n_cov, g->d_inv_atom,
                                      g->d_inv_v64, g->nprjmx, g->natom, g->d_nprj, t, g->N, nb,
                                      out);
  }
  St64 a;
  a.nx = g->nx; a.ny = g->ny; a.nz = g->nz;
  a.zchunk = g->nz <= 160 ? g->nz : 64;
  a.ntx = (g->nx + D_TX - 1) / D_TX;
  a.nty = (g->ny + D_TY - 1) / D_TY;
  const StencilArgs<double> sa = make_stencil_args<double>(g);
  for (int m = 0; m < 5; ++m) {
    a.cx[m] = sa.cx[m]; a.cy[m] = sa.cy[m]; a.cz[m] = sa.cz[m];
  }
  a.c0 = sa.c0;
  a.psi = psi; a.out = out; a.veff = veff; a.inv_off = g->d_inv_off;
  const int nzc = (g->nz + a.zchunk - 1) / a.zchunk;
  const size_t smem = sizeof(double) * D_RING * D_HY * D_HX;
  RS_CUDA(cudaFuncSetAttribute(k_stencil_f64_zmarch, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)smem));
  dim3 grid(a.ntx * a.nty * nzc, nb);
  k_stencil_f64_zmarch<<<grid, D_THREADS, smem, st>>>(a);
  RS_LAUNCH_CHECK("k_stencil_f64_zmarch");
  return RS_OK;
}

template <class T, int MODE>
int launch_gather(const rs_geom* g, const double* mat, const double* rp, const T* psi,
                  const T* veff, T* out, int nb, cudaStream_t st) {
  if (nb <= 0) return RS_OK;
  T* t = nullptr;
  int rc = make_tcoef<T>(g, mat, rp, nb, &t, st);
  if (rc) return rc;
  if constexpr (sizeof(T) == 8 && MODE == 1) {
    if (hpsi_f64_zmarch_ok(g, nb)) {
      rc = launch_hpsi_f64_zmarch(g, t, psi, veff, out, nb, st);
      if (t) cudaFreeAsync(t, st);
      return rc;
    }
  }
  const T* inv_v;
  if constexpr (sizeof(T) == 8) inv_v = (const T*)g->d_inv_v64; else inv_v = (const T*)g->d_inv_v32;
  const int bpb = 4;
  dim3 grid(div_up(g->N, 128), div_up(nb, bpb));
  k_nl_gather<T, MODE><<<grid, 128, 0, st>>>(make_stencil_args<T>(g), g->d_inv_off,
                                             g->d_inv_atom, inv_v, g->nprjmx, g->natom,
                                             g->d_nprj, t, psi, veff, out, nb, bpb);
  cudaError_t e = cudaGetLastError();
  if (t) cudaFreeAsync(t, st);
  if (e != cudaSuccess) return cuda_status(e, "k_nl_gather");
  return RS_OK;
}

template int launch_nl_dot<double>(const rs_geom*, const double*, int, double*, cudaStream_t);
template int launch_nl_dot<float>(const rs_geom*, const float*, int, double*, cudaStream_t);
template int launch_gather<double, 0>(const rs_geom*, const double*, const double*,
                                      const double*, const double*, double*, int, cudaStream_t);
template int launch_gather<double, 1>(const rs_geom*, const double*, const double*,
                                      const double*, const double*, double*, int, cudaStream_t);
template int launch_gather<double, 2>(const rs_geom*, const double*, const double*,
                                      const double*, const double*, double*, int, cudaStream_t);
template int launch_gather<float, 1>(const rs_geom*, const double*, const double*, const float*,
                                     const float*, float*, int, cudaStream_t);
template int launch_gather<float, 2>(const rs_geom*, const double*, const double*, const float*,
                                     const float*, float*, int, cudaStream_t);

}  // namespace rs

#define RS_NEED_G(fn) \
  if (!g) return rs::fail(RS_EINVAL, fn ": null geometry")

extern "C" int rs_nonlocal_dot_f64(const rs_geom* g, const double* psi, int nb, double* rp,
                                   void* stream) {
  RS_NEED_G("rs_nonlocal_dot_f64");
  return rs::launch_nl_dot<double>(g, psi, nb, rp, rs::as_stream(stream));
}
extern "C" int rs_nonlocal_dot_f32(const rs_geom* g, const float* psi, int nb, double* rp,
                                   void* stream) {
  RS_NEED_G("rs_nonlocal_dot_f32");
  return rs::launch_nl_dot<float>(g, psi, nb, rp, rs::as_stream(stream));
}
extern "C" int rs_nonlocal_apply_f64(const rs_geom* g, const double* mat, const double* rp,
                                     int nb, double* out, void* stream) {
  RS_NEED_G("rs_nonlocal_apply_f64");
  return rs::launch_gather<double, 0>(g, mat, rp, nullptr, nullptr, out, nb,
                                      rs::as_stream(stream));
}
extern "C" int rs_hpsi_f64(const rs_geom* g, const double* veff, const double* dij,
                           const double* rp, const double* psi, double* hpsi, int nb,
                           void* stream) {
  RS_NEED_G("rs_hpsi_f64");
  return rs::launch_gather<double, 1>(g, dij, rp, psi, veff, hpsi, nb, rs::as_stream(stream));
}
extern "C" int rs_spsi_f64(const rs_geom* g, const double* sss, const double* rp,
                           const double* psi, double* spsi, int nb, void* stream) {
  RS_NEED_G("rs_spsi_f64");
  return rs::launch_gather<double, 2>(g, sss, rp, psi, nullptr, spsi, nb, rs::as_stream(stream));
}
namespace rs {
bool spsi_f32_fast_ok(const rs_geom* g);
int launch_spsi_f32_fast(const rs_geom* g, const double* sss, const double* rp, const float* psi,
                         float* out, int nb, cudaStream_t st);
}  // namespace rs
extern "C" int rs_spsi_f32(const rs_geom* g, const double* sss, const double* rp,
                           const float* psi, float* spsi, int nb, void* stream) {
  RS_NEED_G("rs_spsi_f32");
  if (rs::spsi_f32_fast_ok(g))
    return rs::launch_spsi_f32_fast(g, sss, rp, psi, spsi, nb, rs::as_stream(stream));
  return rs::launch_gather<float, 2>(g, sss, rp, psi, nullptr, spsi, nb, rs::as_stream(stream));
}
