// potentials.cu -- the SCF potential and mixing steps around the band
// solver (scf_potentials, scf_chargemixing, scf_diffcharge) for periodic
// norm-conserving cells, one spin:
//
//  * rs_interp_d2c: the dense -> coarse transfer of trans_d2c_vh and
//    trans_d2c_vxc (trans8f.F90:93-152, 415-454): interpolation mode 2
//    (interpolation8f.F90:98-214), i.e. the transpose of the coarse -> dense
//    Lagrange interpolation, then v/8 and the periodic halo fold of
//    overlap_interpolation nflag=2 (overlap_interpolation8f.F90:492-892).
//    Three gather passes (z, y, x) each sum a target's contributions in the
//    reference's loop order, so the FP64 result is bit-exact;
//  * rs_vxc_pz: vxpot_lda_pz (vxpot8f.F90:126-155), pointwise;
//  * rs_veff_sum: veff = vx + (vloc + vh) (scf_potentials8f.F90:256-267);
//  * rs_diffcharge: the SCF charge difference (scf_diffcharge8f.F90,
//    kukan8f.F90:672-673), the sum in the fixed tree;
//  * rs_mixer_*: modified Broyden mixing of the grid density
//    (scf_chargemixing8f.F90:59-657) with its history on the device.
#include <math.h>

#include <algorithm>
#include <vector>

#include "reduce.cuh"
#include "rs_common.cuh"

namespace rs {

template <class T>
int tree_dot(long n, const T* a, const T* b, double* out, double* part, cudaStream_t st);

namespace {

struct D2cW {
  double w[2][16];  // w[parity][i + nf - 1], i = -nf+1..nf
};

// the interpolation weights aweight(i, k) for nmesh = 2
D2cW d2c_weights(int nf) {
  D2cW a;
  for (int k = 0; k < 2; ++k) {
    const double r = ((double)k + 0.5) * 0.5;
    for (int j = -nf + 1; j <= nf; ++j) {
      double w = 1.0;
      for (int i = -nf + 1; i <= nf; ++i)
        if (i != j) w = w * (r - (double)i) / ((double)j - (double)i);
      a.w[k][j + nf - 1] = w;
    }
  }
  return a;
}

// One pass of the transfer along one axis.  The input is indexed
// in[(c2*n1 + c1)*n0 + j] with j the dense coordinate along the pass axis
// (1-based j = idx+1); the output has the coarse halo'd coordinate (offset
// nf-1, extent nc + 2nf) in place of j.  Axis order of the three passes is
// handled by the caller's strides.
struct PassDims {
  int nd;        // dense points along the axis
  int hc;        // halo'd coarse extent along the axis
  long cnt;      // outputs
  long in_sa;    // input stride of the pass axis
  long out_sa;   // output stride of the pass axis
  int o0, o1;    // output extents of the two other axes (fastest first)
  long in_s0, in_s1, out_s0, out_s1;  // strides of the two other axes
  int axis_fast;  // threads walk the pass axis fastest (contiguous output)
};

__global__ void k_d2c_pass(PassDims p, int nf, D2cW aw, const double* __restrict__ in,
                           double* __restrict__ out, double scale) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.cnt) return;
  int a0, a1, hcz;  // hcz: halo'd coarse index along the pass axis
  if (p.axis_fast) {
    hcz = (int)(t % p.hc);
    const long r = t / p.hc;
    a0 = (int)(r % p.o0);
    a1 = (int)(r / p.o0);
  } else {
    a0 = (int)(t % p.o0);
    const long r = t / p.o0;
    a1 = (int)(r % p.o1);
    hcz = (int)(r / p.o1);
  }
  const int c = hcz - (nf - 1);        // 1-based coarse coordinate
  const long ib = a0 * p.in_s0 + a1 * p.in_s1;
  double acc = 0.0;
  for (int i = -nf + 1; i <= nf; ++i) {
    const int l = c - i;
    for (int j = 2 * l; j <= 2 * l + 1; ++j)
      if (j >= 1 && j <= p.nd) acc = fma(aw.w[j & 1][i + nf - 1], in[ib + (long)(j - 1) * p.in_sa], acc);
  }
  out[a0 * p.out_s0 + a1 * p.out_s1 + (long)hcz * p.out_sa] = scale == 1.0 ? acc : acc / scale;
}

// periodic fold of the halo onto the interior along one axis of the halo'd
// coarse array v (extents hx, hy, hz, x fastest): for o = 1..nf,
// v(o) += v(n+o) and v(n-nf+o) += v(-nf+o), over the full halo'd extent of
// the other two axes
__global__ void k_d2c_fold(int axis, int nx, int ny, int nz, int nf, double* __restrict__ v) {
  const int hx = nx + 2 * nf, hy = ny + 2 * nf, hz = nz + 2 * nf;
  const int ext[3] = {hx, hy, hz};
  const int n[3] = {nx, ny, nz};
  const long str[3] = {1, hx, (long)hx * hy};
  const int u = axis == 0 ? 1 : 0, w = axis == 2 ? 1 : 2;  // the other axes
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long total = (long)nf * ext[u] * ext[w];
  if (t >= total) return;
  const int o = (int)(t % nf) + 1;
  const long r = t / nf;
  const long base = (r % ext[u]) * str[u] + (r / ext[u]) * str[w];
  auto at = [&](int c) -> double& { return v[base + (long)(c + nf - 1) * str[axis]]; };
  at(o) = at(o) + at(n[axis] + o);
  at(n[axis] - nf + o) = at(n[axis] - nf + o) + at(-nf + o);
}

__global__ void k_d2c_extract(int nx, int ny, int nz, int nf, const double* __restrict__ v,
                              double* __restrict__ out) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long N = (long)nx * ny * nz;
  if (t >= N) return;
  const int ix = (int)(t % nx), iy = (int)((t / nx) % ny), iz = (int)(t / ((long)nx * ny));
  const int hx = nx + 2 * nf, hy = ny + 2 * nf;
  out[t] = v[((long)(iz + nf) * hy + (iy + nf)) * hx + (ix + nf)];
}

}  // namespace

int interp_d2c(int nx, int ny, int nz, int nf, const double* in, double* out, cudaStream_t st) {
  const int Nx = 2 * nx, Ny = 2 * ny, Nz = 2 * nz;
  const int hx = nx + 2 * nf, hy = ny + 2 * nf, hz = nz + 2 * nf;
  double *t2 = nullptr, *t1 = nullptr, *v = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&t2, sizeof(double) * (size_t)Nx * Ny * hz, st));
  cudaError_t e = cudaMallocAsync((void**)&t1, sizeof(double) * (size_t)Nx * hy * hz, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&v, sizeof(double) * (size_t)hx * hy * hz, st);
  if (e == cudaSuccess) {
    const D2cW aw = d2c_weights(nf);
    // z pass: in[(jz*Ny + jy)*Nx + jx] -> t2[(cz*Ny + jy)*Nx + jx]
    PassDims pz{Nz, hz, (long)Nx * Ny * hz, (long)Nx * Ny, (long)Nx * Ny, Nx, Ny, 1, Nx, 1, Nx, 0};
    k_d2c_pass<<<div_up(pz.cnt, 256), 256, 0, st>>>(pz, nf, aw, in, t2, 1.0);
    // y pass: t2[(cz*Ny + jy)*Nx + jx] -> t1[(cz*hy + cy)*Nx + jx]
    PassDims py{Ny, hy, (long)Nx * hy * hz, Nx, Nx, Nx, hz, 1, (long)Nx * Ny, 1, (long)Nx * hy, 0};
    k_d2c_pass<<<div_up(py.cnt, 256), 256, 0, st>>>(py, nf, aw, t2, t1, 1.0);
    // x pass: t1[(cz*hy + cy)*Nx + jx] -> v[(cz*hy + cy)*hx + cx], then / nmesh^3
    PassDims px{Nx, hx, (long)hx * hy * hz, 1, 1, hy, hz, Nx, (long)Nx * hy, hx, (long)hx * hy, 1};
    k_d2c_pass<<<div_up(px.cnt, 256), 256, 0, st>>>(px, nf, aw, t1, v, 8.0);
    for (int axis = 0; axis < 3; ++axis) {
      const long cnt = (long)nf * (axis == 0 ? (long)hy * hz : axis == 1 ? (long)hx * hz : (long)hx * hy);
      k_d2c_fold<<<div_up(cnt, 256), 256, 0, st>>>(axis, nx, ny, nz, nf, v);
    }
    k_d2c_extract<<<div_up((long)nx * ny * nz, 256), 256, 0, st>>>(nx, ny, nz, nf, v, out);
    e = cudaGetLastError();
  }
  if (t2) cudaFreeAsync(t2, st);
  if (t1) cudaFreeAsync(t1, st);
  if (v) cudaFreeAsync(v, st);
  if (e != cudaSuccess) return cuda_status(e, "rs_interp_d2c");
  return RS_OK;
}

namespace {

// vxpot_lda_pz per point, grouped as the Fortran source groups it
// (x**2.0d0 as x*x; pi as the double nearest pi)
__global__ void k_vxc_pz(long n, const double* __restrict__ rho, double* __restrict__ vx,
                         double* __restrict__ ex) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double pi = 3.141592653589793;
  const double third = 1.0 / 3.0;
  const double r = rho[i];
  if (r > 1.0e-15) {
    const double rs = pow(3.0 / (4.0 * pi * r), 1.0 / 3.0);
    double exc, v;
    if (rs >= 1.0) {
      const double den = 1.0 + 1.0529 * sqrt(rs) + 0.3334 * rs;
      exc = -0.1423 / den;
      v = exc - rs / 3.0 * (0.1423 * (0.3334 + 0.52645 / sqrt(rs)) / (den * den));
    } else {
      exc = -0.048 + 0.0311 * log(rs) - 0.0116 * rs + 0.002 * rs * log(rs);
      v = exc - rs / 3.0 * (0.0311 / rs - 0.0096 + 0.002 * log(rs));
    }
    const double cx = 0.75 * pow(2.25 / (pi * pi), third);
    exc = exc - cx / rs;
    ex[i] = exc;
    vx[i] = v - cx / rs - rs / 3.0 * (cx / (rs * rs));
  } else {
    vx[i] = 0.0;
    ex[i] = 0.0;
  }
}

__global__ void k_veff_sum(long n, const double* __restrict__ vx, const double* __restrict__ vloc,
                           const double* __restrict__ vh, double* __restrict__ veff,
                           float* __restrict__ veff32) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = vx[i] + (vloc[i] + vh[i]);
  if (veff) veff[i] = v;
  if (veff32) veff32[i] = (float)v;
}

// w = x1 - x0
__global__ void k_sub(long n, const double* __restrict__ x1, const double* __restrict__ x0,
                      double* __restrict__ w) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) w[i] = x1[i] - x0[i];
}

// All 2 mb - 1 products of one Broyden step in one pass (F_i = F + i n):
//   d < mb - 1:           (F_mb - F_mb-1) . (F_i - F_i-1), i = d + 2
//   mb - 1 <= d < 2mb-2:  (F_i - F_i-1) . F_mb,             i = d - mb + 3
//   d = 2 mb - 2:         (F_mb - F_mb-1) . (F_mb - F_mb-1)
// each over the fixed tree (a lane's 16 terms by fma from zero, then the
// block fold), with the differences formed as k_sub forms them, so every
// product has the bits of k_sub + tree_dot.  Block (chunk, group of
// kMixGroup products); part[d][chunk].
constexpr int kMixGroup = 8;
__device__ __forceinline__ void mix_operands(const double* F, long n, int mb, int d,
                                             const double*& x1, const double*& x0,
                                             const double*& y1, const double*& y0) {
  const double* Fm = F + (long)mb * n;
  if (d < mb - 1) {
    const int i = d + 2;
    x1 = Fm; x0 = Fm - n; y1 = F + (long)i * n; y0 = y1 - n;
  } else if (d < 2 * mb - 2) {
    const int i = d - mb + 3;
    x1 = F + (long)i * n; x0 = x1 - n; y1 = Fm; y0 = nullptr;
  } else {
    x1 = Fm; x0 = Fm - n; y1 = Fm; y0 = Fm - n;
  }
}
__global__ void __launch_bounds__(kTreeLanes) k_mix_partial(long n, const double* __restrict__ F,
                                                            int mb, int ndot, long nblk,
                                                            double* __restrict__ part) {
  __shared__ double ws[8];
  const int d0 = blockIdx.y * kMixGroup;
  const int nd = min(kMixGroup, ndot - d0);
  const long base = (long)blockIdx.x * kTreeChunk + threadIdx.x;
  double acc[kMixGroup];
#pragma unroll
  for (int j = 0; j < kMixGroup; ++j) acc[j] = 0.0;
#pragma unroll
  for (int j = 0; j < kMixGroup; ++j) {
    if (j < nd) {
      const double *x1, *x0, *y1, *y0;
      mix_operands(F, n, mb, d0 + j, x1, x0, y1, y0);
      for (int k = 0; k < kTreePerLane; ++k) {
        const long i = base + (long)k * kTreeLanes;
        if (i < n) {
          const double w1 = x1[i] - x0[i];
          const double w2 = y0 ? y1[i] - y0[i] : y1[i];
          acc[j] = fma(w1, w2, acc[j]);
        }
      }
    }
  }
#pragma unroll
  for (int j = 0; j < kMixGroup; ++j) {
    if (j < nd) {
      const double v = tree_fold256(acc[j], ws);
      if (threadIdx.x == 0) part[(long)(d0 + j) * nblk + blockIdx.x] = v;
    }
  }
}
// one block per product: the chunk sums folded as k_tree_final folds them
__global__ void __launch_bounds__(kTreeLanes) k_mix_final(long nblk, const double* __restrict__ part,
                                                          double* __restrict__ out) {
  __shared__ double ws[8];
  const double* p = part + (long)blockIdx.x * nblk;
  double acc = 0.0;
  for (long k = threadIdx.x; k < nblk; k += kTreeLanes) acc = acc + p[k];
  const double s = tree_fold256(acc, ws);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// f = o - i, g = (o - i) * eta (scf_chargemixing_broyden_vecs, one spin)
__global__ void k_fg(long n, const double* __restrict__ o, const double* __restrict__ in,
                     double eta, double* __restrict__ f, double* __restrict__ g) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  f[i] = o[i] - in[i];
  g[i] = (o[i] - in[i]) * eta;
}

__global__ void k_neg(long n, const double* __restrict__ x, double* __restrict__ y) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = -x[i];
}

// u = u + g + rho - prev, left to right
__global__ void k_u_new(long n, double* __restrict__ u, const double* __restrict__ g,
                        const double* __restrict__ rho, const double* __restrict__ prev) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) u[i] = u[i] + g[i] + rho[i] - prev[i];
}

// y = fma(-t, x, y)
__global__ void k_axmy(long n, double t, const double* __restrict__ x, double* __restrict__ y) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = fma(-t, x[i], y[i]);
}

// prev = rho; b = g
__global__ void k_keep(long n, const double* __restrict__ rho, const double* __restrict__ g,
                       double* __restrict__ prev, double* __restrict__ b) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  prev[i] = rho[i];
  b[i] = g[i];
}

__global__ void k_add(long n, const double* __restrict__ b, double* __restrict__ rho) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) rho[i] = rho[i] + b[i];
}

}  // namespace
}  // namespace rs

// Broyden history on the device; the (nbrydn x nbrydn) matrices on the host.
struct rs_mixer {
  long n;
  int nbrydn, lbrydn;
  double eta;
  double* f;     // [nbrydn+1][n]
  double* u;     // [nbrydn+1][n]
  double* g;
  double* prev;
  double* w1;
  double* w2;
  double* part;  // tree partials
  double* dsc;   // device scalar
  double* prod;  // the Broyden products of a step (up to 128)
  std::vector<double> amat1, amat3;
};

extern "C" int rs_interp_d2c(int nx, int ny, int nz, int nf, const double* in, double* out,
                             void* stream) {
  if (nx < 2 * nf || ny < 2 * nf || nz < 2 * nf || nf < 1 || nf > 8 || !in || !out)
    return rs::fail(RS_EINVAL, "rs_interp_d2c: needs nf in 1..8 and n >= 2 nf on each axis");
  return rs::interp_d2c(nx, ny, nz, nf, in, out, rs::as_stream(stream));
}

extern "C" int rs_vxc_pz(long n, const double* rho, double* vx, double* ex, void* stream) {
  if (n < 0 || (n > 0 && (!rho || !vx || !ex)))
    return rs::fail(RS_EINVAL, "rs_vxc_pz: null or negative argument");
  if (n == 0) return RS_OK;
  rs::k_vxc_pz<<<rs::div_up(n, 256), 256, 0, rs::as_stream(stream)>>>(n, rho, vx, ex);
  RS_LAUNCH_CHECK("k_vxc_pz");
  return RS_OK;
}

extern "C" int rs_veff_sum(long n, const double* vx, const double* vloc, const double* vh,
                           double* veff, float* veff32, void* stream) {
  if (n < 0 || (n > 0 && (!vx || !vloc || !vh || (!veff && !veff32))))
    return rs::fail(RS_EINVAL, "rs_veff_sum: null or negative argument");
  if (n == 0) return RS_OK;
  rs::k_veff_sum<<<rs::div_up(n, 256), 256, 0, rs::as_stream(stream)>>>(n, vx, vloc, vh, veff,
                                                                        veff32);
  RS_LAUNCH_CHECK("k_veff_sum");
  return RS_OK;
}

extern "C" int rs_diffcharge(long n, const double* rho_o, const double* rho_i, double dx,
                             double dy, double dz, double xmax, double ymax, double zmax,
                             double* diff, void* stream) {
  if (n <= 0 || !rho_o || !rho_i || !diff)
    return rs::fail(RS_EINVAL, "rs_diffcharge: null or empty argument");
  cudaStream_t st = rs::as_stream(stream);
  double *d = nullptr, *part = nullptr, *s = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&d, sizeof(double) * (n + rs::tree_chunks(n) + 1), st));
  part = d + n;
  s = part + rs::tree_chunks(n);
  rs::k_sub<<<rs::div_up(n, 256), 256, 0, st>>>(n, rho_i, rho_o, d);
  int rc = rs::tree_dot<double>(n, d, d, s, part, st);
  double h = 0.0;
  if (rc == RS_OK) {
    cudaError_t e = cudaMemcpyAsync(&h, s, sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = rs::cuda_status(e, "rs_diffcharge");
  }
  cudaFreeAsync(d, st);
  if (rc == RS_OK) *diff = sqrt(h * dx * dy * dz / (8.0 * xmax * ymax * zmax));
  return rc;
}

extern "C" int rs_mixer_destroy(rs_mixer* m) {
  if (!m) return RS_OK;
  cudaFree(m->f);
  delete m;
  return RS_OK;
}

extern "C" int rs_mixer_create(rs_mixer** out, long n, int nbrydn, double eta) {
  if (!out) return rs::fail(RS_EINVAL, "rs_mixer_create: null handle");
  *out = nullptr;
  if (n <= 0 || nbrydn < 2 || nbrydn > 63)
    return rs::fail(RS_EINVAL, "rs_mixer_create: needs n > 0 and nbrydn in 2..63");
  rs_mixer* m = new rs_mixer;
  m->n = n; m->nbrydn = nbrydn; m->lbrydn = 0; m->eta = eta;
  const long slots = nbrydn + 1;
  const long nc = rs::tree_chunks(n);
  const size_t words = (size_t)(2 * slots + 4) * n + nc + 1 + 128;
  double* base = nullptr;
  const cudaError_t e = cudaMalloc((void**)&base, words * sizeof(double));
  if (e != cudaSuccess) {
    delete m;
    return rs::cuda_status(e, "rs_mixer_create");
  }
  m->f = base;
  m->u = m->f + slots * n;
  m->g = m->u + slots * n;
  m->prev = m->g + n;
  m->w1 = m->prev + n;
  m->w2 = m->w1 + n;
  m->part = m->w2 + n;
  m->dsc = m->part + nc;
  m->prod = m->dsc + 1;
  m->amat1.assign(slots * slots, 0.0);
  m->amat3.assign(slots, 0.0);
  *out = m;
  return RS_OK;
}

namespace {

// the 2 mb - 1 products of a step (k_mix_partial), times dV, into prod
int mix_dots(rs_mixer* m, int mb, double dvol, cudaStream_t st, double* prod) {
  const long n = m->n;
  const long nblk = rs::tree_chunks(n);
  const int ndot = 2 * mb - 1;
  // part: ndot x nblk chunk sums in w1/w2 (2 n words >= ndot nblk: ndot < 128
  // and nblk = n / 4096 rounded up), then the products in prod
  double* part = m->w1;
  double* out = m->prod;
  if ((long)ndot * nblk > 2 * n || ndot > 128)
    return rs::fail(RS_EINVAL, "rs_mixer_step: Broyden products do not fit the work space");
  dim3 grid((unsigned)nblk, (unsigned)((ndot + rs::kMixGroup - 1) / rs::kMixGroup));
  rs::k_mix_partial<<<grid, rs::kTreeLanes, 0, st>>>(n, m->f, mb, ndot, nblk, part);
  rs::k_mix_final<<<ndot, rs::kTreeLanes, 0, st>>>(nblk, part, out);
  cudaError_t e = cudaMemcpyAsync(prod, out, sizeof(double) * ndot, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return rs::cuda_status(e, "rs_mixer_step");
  for (int d = 0; d < ndot; ++d) prod[d] *= dvol;
  return RS_OK;
}


}  // namespace

extern "C" int rs_mixer_step(rs_mixer* m, const double* rho_o, double* rho_i, double dvol,
                             void* stream) {
  if (!m || !rho_o || !rho_i) return rs::fail(RS_EINVAL, "rs_mixer_step: null argument");
  cudaStream_t st = rs::as_stream(stream);
  const long n = m->n;
  const int nb = m->nbrydn, M1 = nb + 1;
  const unsigned g = rs::div_up(n, 256);
  auto F = [&](int k) { return m->f + (long)k * n; };
  auto U = [&](int k) { return m->u + (long)k * n; };
  auto A1 = [&](int i, int j) -> double& { return m->amat1[(long)i * M1 + j]; };
  m->lbrydn += 1;
  if (m->lbrydn == 1) {
    RS_CUDA(cudaMemcpyAsync(rho_i, rho_o, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    return RS_OK;
  }
  if (m->lbrydn == 2) {
    std::fill(m->amat1.begin(), m->amat1.end(), 0.0);
    std::fill(m->amat3.begin(), m->amat3.end(), 0.0);
  }
  const int mb = std::min(m->lbrydn - 1, nb);
  double t1[64][64], t2[64];
  int rc = RS_OK;
  if (mb > 1) rs::k_neg<<<g, 256, 0, st>>>(n, m->g, U(mb));
  rs::k_fg<<<g, 256, 0, st>>>(n, rho_o, rho_i, m->eta, F(mb), m->g);
  if (mb > 1) {
    for (int i = 2; i <= nb; ++i)
      for (int j = 2; j <= nb; ++j) t1[i][j] = A1(i, j);
    // the step's 2 mb - 1 products, each equal bit for bit to its own
    // k_sub + tree_dot, in two launches and one read-back
    double prod[2 * 64];
    if ((rc = mix_dots(m, mb, dvol, st, prod))) return rc;
    for (int i = 2; i <= mb; ++i) {
      const double t = prod[i - 2];
      t1[mb][i] = t; t1[i][mb] = t;
      A1(mb, i) = t; A1(i, mb) = t;
    }
    for (int i = 2; i <= mb; ++i) t2[i] = prod[mb - 1 + i - 2];
    m->amat3[mb] = prod[2 * mb - 2];
    for (int j = 2; j <= mb; ++j) {
      for (int i = 2; i <= mb; ++i) t1[j][i] = t1[j][i] / m->amat3[j];
      t2[j] = t2[j] / m->amat3[j];
    }
    rs::k_u_new<<<g, 256, 0, st>>>(n, U(mb), m->g, rho_i, m->prev);
    for (int j = 2; j <= mb - 1; ++j) rs::k_axmy<<<g, 256, 0, st>>>(n, t1[j][mb], U(j), U(mb));
  }
  double* bv = m->w1;
  rs::k_keep<<<g, 256, 0, st>>>(n, rho_i, m->g, m->prev, bv);
  for (int j = 2; j <= mb; ++j) rs::k_axmy<<<g, 256, 0, st>>>(n, t2[j], U(j), bv);
  rs::k_add<<<g, 256, 0, st>>>(n, bv, rho_i);
  if (mb == nb) {
    t2[2] = 1.0;
    for (int i = 3; i <= mb; ++i) {
      t2[i] = 0.0;
      for (int j = 2; j <= i - 1; ++j) t2[i] = fma(-t1[j][i], t2[j], t2[i]);
      rs::k_axmy<<<g, 256, 0, st>>>(n, t2[i], U(2), U(i));
    }
    for (int i = 2; i <= mb; ++i) {
      RS_CUDA(cudaMemcpyAsync(F(i - 1), F(i), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
      if (i > 2)
        RS_CUDA(cudaMemcpyAsync(U(i - 1), U(i), sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    }
    for (int j = 2; j <= mb - 1; ++j) {
      for (int i = 2; i <= mb - 1; ++i) A1(i, j) = A1(i + 1, j + 1);
      m->amat3[j] = m->amat3[j + 1];
    }
  }
  RS_LAUNCH_CHECK("rs_mixer_step");
  return RS_OK;
}
