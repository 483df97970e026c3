// stencil.cu -- periodic FD stencils: the kinetic+local operator of
// kslaplacian_r, the ksprecondition smoother, the Hartree Laplacian and the
// first-derivative stencil of force_r_02/03/04.
//
// Periodic boundaries are handled by index wrapping inside the kernels; this
// replaces overlap_finitedifference_r's halo copy for a single rank with
// nperi=3 (overlap_finitedifference8f.F90:97-139, 685-710).
#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {

// One thread per grid point, bands along blockIdx.y.  Accumulation order per
// point: x pass (including the diagonal (cx0+cy0+cz0+veff)*psi), then y, then
// z, each term one fma -- kslaplacian8f.F90:207-261 evaluated left to right.
template <class T>
__global__ void k_kslaplacian(StencilArgs<T> s, const T* __restrict__ psi,
                              const T* __restrict__ veff, T* __restrict__ out, int nb) {
  const long N = (long)s.nx * s.ny * s.nz;
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (p >= N || b >= nb) return;
  const int ix = (int)(p % s.nx), iy = (int)((p / s.nx) % s.ny), iz = (int)(p / ((long)s.nx * s.ny));
  const T* v = psi + (long)b * N;
  T acc = out[(long)b * N + p];
  acc = stencil_point<T>(s, v, ix, iy, iz, veff[p], acc);
  out[(long)b * N + p] = acc;
}

// ksprecondition (ksprecondition8f.F90:8-39).  One block per run of kPrecRows
// x-rows of one band: the row pointers and their periodic neighbours are set
// up once, threads walk x with branch wraps (no integer division per point).
constexpr int kPrecRows = 4;
template <class T>
__global__ void k_precondition(int nx, int ny, int nz, const T* __restrict__ in,
                               T* __restrict__ out, int nb) {
  const long N = (long)nx * ny * nz;
  const int b = blockIdx.y;
  const T* v = in + (long)b * N;
  T* o = out + (long)b * N;
  const T c = (T)(1.0 / 12.0), h = (T)0.5;
  const long nrow = (long)ny * nz;
  for (int r = 0; r < kPrecRows; ++r) {
    const long row = (long)blockIdx.x * kPrecRows + r;
    if (row >= nrow) return;
    const int iy = (int)(row % ny), iz = (int)(row / ny);
    const int iym = iy == 0 ? ny - 1 : iy - 1, iyp = iy == ny - 1 ? 0 : iy + 1;
    const int izm = iz == 0 ? nz - 1 : iz - 1, izp = iz == nz - 1 ? 0 : iz + 1;
    const T* r0 = v + row * nx;
    const T* rym = v + ((long)iz * ny + iym) * nx;
    const T* ryp = v + ((long)iz * ny + iyp) * nx;
    const T* rzm = v + ((long)izm * ny + iy) * nx;
    const T* rzp = v + ((long)izp * ny + iy) * nx;
    T* orow = o + row * nx;
    for (int ix = threadIdx.x; ix < nx; ix += blockDim.x) {
      const int ixm = ix == 0 ? nx - 1 : ix - 1, ixp = ix == nx - 1 ? 0 : ix + 1;
      T t = c * r0[ixm];
      t = fma(c, rym[ix], t);
      t = fma(c, rzm[ix], t);
      t = fma(h, r0[ix], t);
      t = fma(c, rzp[ix], t);
      t = fma(c, ryp[ix], t);
      t = fma(c, r0[ixp], t);
      orow[ix] = t;
    }
  }
}

// Plane-marching form of k_precondition for grids whose x-rows split into
// 16-byte vectors (V points of T).  A CTA owns TY whole x-rows of one band
// and walks a run of z planes.  Each plane, with one halo row on either side
// in y, is copied into a shared ring with 16-byte cp.async, kPzAhead planes
// ahead of the plane being smoothed, so HBM latency hides behind the copies
// in flight and every value crosses HBM once per band (the halo rows come
// from L2, loaded by the neighbouring tiles).  A thread smooths V points of
// one row from the ring: the same seven fmas in the same order as
// k_precondition.
constexpr int kPzAhead = 2;
constexpr int kPzRing = kPzAhead + 4;  // planes z-1..z+1, the ones in flight, the one issued
constexpr int kPzThreads = 256;
constexpr int kPzZChunk = 32;

__device__ __forceinline__ void pz_cp16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void pz_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void pz_wait_ahead() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(kPzAhead) : "memory");
}

template <class T>
using PzVec = Pack<T, 16 / (int)sizeof(T)>;

template <class T>
__global__ void __launch_bounds__(kPzThreads) k_precondition_zm(int nx, int ny, int nz, int ty_rows,
                                                                int nty, int zc,
                                                                const T* __restrict__ in,
                                                                T* __restrict__ out) {
  constexpr int V = 16 / (int)sizeof(T);
  extern __shared__ __align__(16) unsigned char pz_smem[];
  T* ring = reinterpret_cast<T*>(pz_smem);  // [kPzRing][ty_rows + 2][nx]
  const int nxv = nx / V;
  const int rows = ty_rows + 2;
  const long slot = (long)rows * nx;
  const int tid = threadIdx.x;
  const int tx = tid % nxv, ty = tid / nxv;  // rows past ny in the last tile stay idle
  const int ytile = blockIdx.x % nty, zt = blockIdx.x / nty;
  const int y0 = ytile * ty_rows;
  const int z0 = zt * zc, z1 = min(nz, z0 + zc);
  const long plane = (long)nx * ny;
  const T* v = in + (long)blockIdx.y * plane * nz;
  T* o = out + (long)blockIdx.y * plane * nz;
  const int nchunk = rows * nxv;
  // copy plane zz (wrapped) with its halo rows into its ring slot, one group
  auto issue = [&](int zz) {
    const int zw = zz < 0 ? zz + nz : (zz >= nz ? zz - nz : zz);
    T* dst = ring + (long)((zz - z0 + 1 + kPzRing) % kPzRing) * slot;
    const T* src = v + (long)zw * plane;
    for (int c = tid; c < nchunk; c += blockDim.x) {
      const int r = c / nxv, cx = c - r * nxv;
      int yr = y0 - 1 + r;
      yr = yr < 0 ? yr + ny : (yr >= ny ? yr - ny : yr);
      pz_cp16(dst + (long)r * nx + cx * V, src + (long)yr * nx + cx * V);
    }
    pz_commit();
  };
  // planes z0-1 .. z0+1+kPzAhead (the last one needed is z1)
  for (int zz = z0 - 1; zz <= z0 + 1 + kPzAhead; ++zz) {
    if (zz <= z1) issue(zz);
    else pz_commit();
  }
  const T c = (T)(1.0 / 12.0), h = (T)0.5;
  const int iy = y0 + ty;
  const bool active = ty < ty_rows && iy < ny;
  const int xm = tx == 0 ? nx - 1 : tx * V - 1;
  const int xp = tx == nxv - 1 ? 0 : tx * V + V;
  for (int z = z0; z < z1; ++z) {
    pz_wait_ahead();
    __syncthreads();
    // the slot of plane z+2+kPzAhead last held plane z-2, read before the barrier
    if (z + 2 + kPzAhead <= z1) issue(z + 2 + kPzAhead);
    else pz_commit();
    if (active) {
      const T* sm = ring + (long)((z - z0 + kPzRing) % kPzRing) * slot;   // plane z-1
      const T* s0 = ring + (long)((z - z0 + 1) % kPzRing) * slot;         // plane z
      const T* sp = ring + (long)((z - z0 + 2) % kPzRing) * slot;         // plane z+1
      const int r = ty + 1;
      PzVec<T> a0 = *reinterpret_cast<const PzVec<T>*>(s0 + (long)r * nx + tx * V);
      PzVec<T> aym = *reinterpret_cast<const PzVec<T>*>(s0 + (long)(r - 1) * nx + tx * V);
      PzVec<T> ayp = *reinterpret_cast<const PzVec<T>*>(s0 + (long)(r + 1) * nx + tx * V);
      PzVec<T> azm = *reinterpret_cast<const PzVec<T>*>(sm + (long)r * nx + tx * V);
      PzVec<T> azp = *reinterpret_cast<const PzVec<T>*>(sp + (long)r * nx + tx * V);
      const T left = s0[(long)r * nx + xm], right = s0[(long)r * nx + xp];
      PzVec<T> res;
#pragma unroll
      for (int k = 0; k < V; ++k) {
        const T xl = k == 0 ? left : a0.v[k - 1];
        const T xr = k == V - 1 ? right : a0.v[k + 1];
        T t = c * xl;
        t = fma(c, aym.v[k], t);
        t = fma(c, azm.v[k], t);
        t = fma(h, a0.v[k], t);
        t = fma(c, azp.v[k], t);
        t = fma(c, ayp.v[k], t);
        t = fma(c, xr, t);
        res.v[k] = t;
      }
      *reinterpret_cast<PzVec<T>*>(o + (long)z * plane + (long)iy * nx + tx * V) = res;
    }
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
}

// scf_hartee_laplacian (scf_hartree8f.F90:949-1004): the x pass starts from
// the first product; diagonal = hadx+hady+hadz with had = acfdh(0)/(d*d)*(-1/2).
__global__ void k_hartree_lap(int nx, int ny, int nz, int nf, HartreeCoefs c,
                              const double* __restrict__ v, double* __restrict__ av) {
  const long N = (long)nx * ny * nz;
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= N) return;
  const int ix = (int)(p % nx), iy = (int)((p / nx) % ny), iz = (int)(p / ((long)nx * ny));
  const long row = ((long)iz * ny + iy) * nx;
  double acc = c.cx[nf] * v[row + wrapi(ix - nf, nx)];
  for (int m = nf - 1; m >= 1; --m) acc = fma(c.cx[m], v[row + wrapi(ix - m, nx)], acc);
  acc = fma(c.diag, v[p], acc);
  for (int m = 1; m <= nf; ++m) acc = fma(c.cx[m], v[row + wrapi(ix + m, nx)], acc);
  for (int m = nf; m >= 1; --m) acc = fma(c.cy[m], v[((long)iz * ny + wrapi(iy - m, ny)) * nx + ix], acc);
  for (int m = 1; m <= nf; ++m) acc = fma(c.cy[m], v[((long)iz * ny + wrapi(iy + m, ny)) * nx + ix], acc);
  for (int m = nf; m >= 1; --m) acc = fma(c.cz[m], v[(wrapi(iz - m, nz) * ny + iy) * nx + ix], acc);
  for (int m = 1; m <= nf; ++m) acc = fma(c.cz[m], v[(wrapi(iz + m, nz) * ny + iy) * nx + ix], acc);
  av[p] = acc;
}

// force_r_02/03/04 (force8f.F90:468-490 for nf=4):
// -a_nf v(+nf) ... -a_1 v(+1) + a_1 v(-1) ... + a_nf v(-nf).
template <class T>
__global__ void k_gradient(int nx, int ny, int nz, int nf, int axis, GradCoefs g,
                           const T* __restrict__ psi, T* __restrict__ out, int nb) {
  const long N = (long)nx * ny * nz;
  const long p = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  if (p >= N || b >= nb) return;
  const int ix = (int)(p % nx), iy = (int)((p / nx) % ny), iz = (int)(p / ((long)nx * ny));
  const T* v = psi + (long)b * N;
  auto at = [&](int m) -> T {
    if (axis == 0) return v[((long)iz * ny + iy) * nx + wrapi(ix + m, nx)];
    if (axis == 1) return v[((long)iz * ny + wrapi(iy + m, ny)) * nx + ix];
    return v[(wrapi(iz + m, nz) * ny + iy) * nx + ix];
  };
  T acc = -((T)g.a[nf] * at(nf));
  for (int m = nf - 1; m >= 1; --m) acc = fma(-(T)g.a[m], at(m), acc);
  for (int m = 1; m <= nf; ++m) acc = fma((T)g.a[m], at(-m), acc);
  out[(long)b * N + p] = acc;
}

template <class T>
StencilArgs<T> make_stencil_args(const rs_geom* g) {
  StencilArgs<T> s;
  s.nx = g->nx; s.ny = g->ny; s.nz = g->nz; s.nf = g->nf;
  for (int m = 0; m < 9; ++m) {
    s.cx[m] = (T)g->cx[m]; s.cy[m] = (T)g->cy[m]; s.cz[m] = (T)g->cz[m];
  }
  s.c0 = (T)(g->cx[0] + g->cy[0] + g->cz[0]);
  return s;
}
template StencilArgs<double> make_stencil_args<double>(const rs_geom*);
template StencilArgs<float> make_stencil_args<float>(const rs_geom*);

GradCoefs grad_coefs(int nf, double h) {
  GradCoefs g;
  for (int m = 0; m < 9; ++m) g.a[m] = 0.0;
  if (nf == 1) g.a[1] = -0.5 / h;
  if (nf == 2) { g.a[2] = 1.0 / 12.0 / h; g.a[1] = -8.0 / 12.0 / h; }
  if (nf == 3) { g.a[3] = -1.0 / 60.0 / h; g.a[2] = 9.0 / 60.0 / h; g.a[1] = -45.0 / 60.0 / h; }
  if (nf >= 4) {
    g.a[4] = 3.0 / 840.0 / h; g.a[3] = -32.0 / 840.0 / h;
    g.a[2] = 168.0 / 840.0 / h; g.a[1] = -672.0 / 840.0 / h;
  }
  return g;
}

HartreeCoefs hartree_coefs(int nfh, double ddx, double ddy, double ddz) {
  double a[9];
  fd_coefs(nfh, a);
  HartreeCoefs c;
  for (int m = 0; m < 9; ++m) {
    c.cx[m] = a[m] / ddx / ddx * (-0.5);
    c.cy[m] = a[m] / ddy / ddy * (-0.5);
    c.cz[m] = a[m] / ddz / ddz * (-0.5);
  }
  const double hadx = a[0] / (ddx * ddx) * (-0.5);
  const double hady = a[0] / (ddy * ddy) * (-0.5);
  const double hadz = a[0] / (ddz * ddz) * (-0.5);
  c.diag = hadx + hady + hadz;
  return c;
}

template <class T>
int launch_kslaplacian(const rs_geom* g, const T* psi, const T* veff, T* out, int nb,
                       cudaStream_t st) {
  if (nb <= 0) return RS_OK;
  if (nb > 65535) return fail(RS_EINVAL, "kslaplacian: nb > 65535");
  dim3 grid(div_up(g->N, 256), nb);
  k_kslaplacian<T><<<grid, 256, 0, st>>>(make_stencil_args<T>(g), psi, veff, out, nb);
  RS_LAUNCH_CHECK("k_kslaplacian");
  return RS_OK;
}

template <class T>
int launch_precondition(const rs_geom* g, const T* in, T* out, int nb, cudaStream_t st) {
  if (nb <= 0) return RS_OK;
  if (nb > 65535) return fail(RS_EINVAL, "precondition: nb > 65535");
  constexpr int V = 16 / (int)sizeof(T);
  const int nxv = g->nx / V;
  const bool aligned = ((uintptr_t)in % 16 == 0) && ((uintptr_t)out % 16 == 0);
  if (g->nx % V == 0 && nxv >= 1 && nxv <= kPzThreads && aligned && in != out) {
    const int tyr = std::max(1, std::min(g->ny, kPzThreads / nxv));
    const int nty = (g->ny + tyr - 1) / tyr;
    // z runs of up to kPzZChunk planes, shorter when few bands leave SMs idle
    int zc = std::min(g->nz, kPzZChunk);
    while (zc > 4 && (long)nty * div_up(g->nz, zc) * nb < 148L * 8) zc = (zc + 1) / 2;
    const int nzc = (g->nz + zc - 1) / zc;
    const size_t smem = sizeof(T) * (size_t)kPzRing * (tyr + 2) * g->nx;
    if (smem <= 200 * 1024 && (long)nty * nzc < (1L << 31)) {
      RS_CUDA(cudaFuncSetAttribute(k_precondition_zm<T>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      dim3 grid((unsigned)(nty * nzc), nb);
      k_precondition_zm<T><<<grid, nxv * tyr, smem, st>>>(g->nx, g->ny, g->nz, tyr, nty, zc, in,
                                                           out);
      RS_LAUNCH_CHECK("k_precondition_zm");
      return RS_OK;
    }
  }
  const long nrow = (long)g->ny * g->nz;
  const int thr = g->nx >= 128 ? 128 : (g->nx + 31) / 32 * 32;
  dim3 grid((unsigned)div_up(nrow, kPrecRows), nb);
  k_precondition<T><<<grid, thr, 0, st>>>(g->nx, g->ny, g->nz, in, out, nb);
  RS_LAUNCH_CHECK("k_precondition");
  return RS_OK;
}

int launch_hartree_lap(int nx, int ny, int nz, int nfh, const HartreeCoefs& c, const double* v,
                       double* av, cudaStream_t st) {
  const long N = (long)nx * ny * nz;
  k_hartree_lap<<<div_up(N, 256), 256, 0, st>>>(nx, ny, nz, nfh, c, v, av);
  RS_LAUNCH_CHECK("k_hartree_lap");
  return RS_OK;
}

template <class T>
int launch_gradient(const rs_geom* g, int axis, const T* psi, T* out, int nb, cudaStream_t st) {
  if (nb <= 0) return RS_OK;
  const double h = axis == 0 ? g->dx : (axis == 1 ? g->dy : g->dz);
  const int nf = g->nf > 4 ? 4 : g->nf;
  dim3 grid(div_up(g->N, 256), nb);
  k_gradient<T><<<grid, 256, 0, st>>>(g->nx, g->ny, g->nz, nf, axis, grad_coefs(nf, h), psi,
                                      out, nb);
  RS_LAUNCH_CHECK("k_gradient");
  return RS_OK;
}

template int launch_kslaplacian<double>(const rs_geom*, const double*, const double*, double*,
                                        int, cudaStream_t);
template int launch_kslaplacian<float>(const rs_geom*, const float*, const float*, float*, int,
                                       cudaStream_t);
template int launch_precondition<double>(const rs_geom*, const double*, double*, int,
                                         cudaStream_t);
template int launch_precondition<float>(const rs_geom*, const float*, float*, int, cudaStream_t);
template int launch_gradient<double>(const rs_geom*, int, const double*, double*, int,
                                     cudaStream_t);
template int launch_gradient<float>(const rs_geom*, int, const float*, float*, int,
                                    cudaStream_t);

}  // namespace rs

extern "C" int rs_kslaplacian_f64(const rs_geom* g, const double* psi, const double* veff,
                                  double* out, int nb, void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_kslaplacian_f64: null geometry");
  return rs::launch_kslaplacian<double>(g, psi, veff, out, nb, rs::as_stream(stream));
}
extern "C" int rs_kslaplacian_f32(const rs_geom* g, const float* psi, const float* veff,
                                  float* out, int nb, void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_kslaplacian_f32: null geometry");
  return rs::launch_kslaplacian<float>(g, psi, veff, out, nb, rs::as_stream(stream));
}
extern "C" int rs_precondition_f64(const rs_geom* g, const double* in, double* out, int nb,
                                   void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_precondition_f64: null geometry");
  return rs::launch_precondition<double>(g, in, out, nb, rs::as_stream(stream));
}
extern "C" int rs_precondition_f32(const rs_geom* g, const float* in, float* out, int nb,
                                   void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_precondition_f32: null geometry");
  return rs::launch_precondition<float>(g, in, out, nb, rs::as_stream(stream));
}
extern "C" int rs_hartree_laplacian(int nx, int ny, int nz, int nfh, double ddx, double ddy,
                                    double ddz, const double* v, double* av, void* stream) {
  if (nx <= 2 * nfh || ny <= 2 * nfh || nz <= 2 * nfh || nfh < 1 || nfh > 6)
    return rs::fail(RS_EINVAL, "rs_hartree_laplacian: bad grid or nfh");
  return rs::launch_hartree_lap(nx, ny, nz, nfh, rs::hartree_coefs(nfh, ddx, ddy, ddz), v, av,
                                rs::as_stream(stream));
}
