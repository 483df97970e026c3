// stencil.cuh -- coefficient bundles and the per-point stencil evaluation
// shared by the stand-alone Laplacian and the fused H*psi kernels.
#pragma once
#include "rs_common.cuh"

namespace rs {

template <class T>
struct StencilArgs {
  int nx, ny, nz, nf;
  T cx[9], cy[9], cz[9];
  T c0;  // cx[0] + cy[0] + cz[0], added left to right
};

struct HartreeCoefs {
  double cx[9], cy[9], cz[9];
  double diag;
};

struct GradCoefs {
  double a[9];
};

// i in (-n, 2n) wrapped into [0, n) (stencil offsets are below the grid size:
// rs_geom_create requires 2 nf < n on every axis)
__device__ __forceinline__ int wrap_near(int i, int n) {
  return i < 0 ? i + n : (i >= n ? i - n : i);
}

// acc + (-1/2 lap + veff) psi at (ix,iy,iz): x terms with the diagonal, then
// y, then z, one fma each (kslaplacian8f.F90:207-261).
template <class T>
__device__ __forceinline__ T stencil_point(const StencilArgs<T>& s, const T* __restrict__ v,
                                           int ix, int iy, int iz, T vloc, T acc) {
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  const long plane = (long)nx * ny;
  const T* row = v + (long)iz * plane + (long)iy * nx;  // (iy, iz) row
  const T* col = v + (long)iy * nx + ix;                  // (ix, iy) column, z stride plane
  for (int m = s.nf; m >= 1; --m) acc = fma(s.cx[m], __ldg(row + wrap_near(ix - m, nx)), acc);
  const T diag = s.c0 + vloc;
  acc = fma(diag, __ldg(row + ix), acc);
  for (int m = 1; m <= s.nf; ++m) acc = fma(s.cx[m], __ldg(row + wrap_near(ix + m, nx)), acc);
  const T* pl = v + (long)iz * plane + ix;
  for (int m = s.nf; m >= 1; --m)
    acc = fma(s.cy[m], __ldg(pl + (long)wrap_near(iy - m, ny) * nx), acc);
  for (int m = 1; m <= s.nf; ++m)
    acc = fma(s.cy[m], __ldg(pl + (long)wrap_near(iy + m, ny) * nx), acc);
  for (int m = s.nf; m >= 1; --m)
    acc = fma(s.cz[m], __ldg(col + (long)wrap_near(iz - m, nz) * plane), acc);
  for (int m = 1; m <= s.nf; ++m)
    acc = fma(s.cz[m], __ldg(col + (long)wrap_near(iz + m, nz) * plane), acc);
  return acc;
}

template <class T>
StencilArgs<T> make_stencil_args(const rs_geom* g);
GradCoefs grad_coefs(int nf, double h);
HartreeCoefs hartree_coefs(int nfh, double ddx, double ddy, double ddz);

template <class T>
int launch_kslaplacian(const rs_geom* g, const T* psi, const T* veff, T* out, int nb,
                       cudaStream_t st);
template <class T>
int launch_precondition(const rs_geom* g, const T* in, T* out, int nb, cudaStream_t st);
int launch_hartree_lap(int nx, int ny, int nz, int nfh, const HartreeCoefs& c, const double* v,
                       double* av, cudaStream_t st);
template <class T>
int launch_gradient(const rs_geom* g, int axis, const T* psi, T* out, int nb, cudaStream_t st);

}  // namespace rs
