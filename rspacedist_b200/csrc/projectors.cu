// projectors.cu -- projector-table generation on the GPU: kukan's
// pseudocalc_07 (pseudocalc8f.F90:2515-3702) and the double-grid weights of
// pseudocalc_01a (pseudocalc8f.F90:343-629), for one species.
//
// For every atom the Fourier-filtered projectors
//     p_la(r) = sum_{iq=1..nqct} coef(iq, c) j_l(q r) q^2 * 4 pi dq / (2 pi)^3
//               * dp^3 * N_m * ylm_m(r) * fermidis(r)        (q = iq * pi / rcuts)
// are evaluated on the fine mesh (npmesh points per coarse spacing) inside
// r < rcut * psctoff, then contracted onto the coarse points with the
// separable double-grid weights (z, y, then x, each a 2 nfdg npmesh-tap sum in
// the order of the Fortran loops) and gathered at the sphere-list points.
//
// Device layout per batch of atoms: the fine arrays vnlspd
// [atom][la][kz][ky][kx] over (2 nxspd)(2 nyspd)(2 nzspd), then the two
// partial contractions and the coarse box [atom][la][iz][iy][ix].  Every value
// is FP64; the Bessel sums take about 60 sincos per fine point, so a batch is
// compute-bound on the FP64 pipe, and the contractions are small.
#include <math.h>

#include <algorithm>

#include "rs_common.cuh"

namespace rs {
namespace {

constexpr int kMaxPrj = 18;   // the largest projector set of pseudocalc_07 (s s' p p' d d')
constexpr int kMaxQ = 960;    // coefficients staged in shared memory (6 columns, < 48 KB)

struct ProjArgs {
  int nprj, nqct, q1, npmesh, used;  // used: bit c set when coefficient column c is read
  int npxd, npyd, npzd;              // fine evaluation box [-npxd+1, npxd] ...
  int nxs, nys, nzs;                 // fine array [-nxs+1, nxs] ...
  int nxmax, nymax, nzmax;
  double dx, dy, dz, dpx, dpy, dpz, dpxyz;
  double rcut, rlim, dqq, tq, eps, filpp;
  int nfiltyp;
  int col[kMaxPrj], ym[kMaxPrj];
  double nrm[kMaxPrj];
};

__device__ __forceinline__ double fermi_weight(double r, double t, double rc) {
  const double a = (r - rc) / t;
  if (fabs(a) < 1.0e2) return 1.0 / (exp(a) + 1.0);
  return a > 0.0 ? 0.0 : 1.0;
}

// one thread per fine point of one atom's evaluation box; blockIdx.y = atom
// of the batch (atom a0 + blockIdx.y)
__global__ void __launch_bounds__(256) k_proj_fine(ProjArgs a, int a0,
                                                   const double* __restrict__ atx,
                                                   const double* __restrict__ aty,
                                                   const double* __restrict__ atz,
                                                   const int* __restrict__ natx,
                                                   const int* __restrict__ naty,
                                                   const int* __restrict__ natz,
                                                   const double* __restrict__ coef,
                                                   double* __restrict__ spd) {
  __shared__ double cq[6][kMaxQ + 1];
  for (int c = 1; c <= 6; ++c)
    if (a.used & (1 << c))
      for (int iq = threadIdx.x; iq <= a.nqct; iq += blockDim.x) cq[c - 1][iq] = coef[c * a.q1 + iq];
  __syncthreads();
  const int bx = 2 * a.npxd, by = 2 * a.npyd, bz = 2 * a.npzd;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)bx * by * bz) return;
  const int ix = (int)(idx % bx) - a.npxd + 1;
  const int iy = (int)((idx / bx) % by) - a.npyd + 1;
  const int iz = (int)(idx / ((long)bx * by)) - a.npzd + 1;
  const int na = a0 + blockIdx.y;
  const double ax = atx[na], ay = aty[na], az = atz[na];
  const int npatx = (int)((ax + a.nxmax * a.dx + 0.5 * a.dpx) / a.dpx) - a.nxmax * a.npmesh;
  const int npaty = (int)((ay + a.nymax * a.dy + 0.5 * a.dpy) / a.dpy) - a.nymax * a.npmesh;
  const int npatz = (int)((az + a.nzmax * a.dz + 0.5 * a.dpz) / a.dpz) - a.nzmax * a.npmesh;
  const double x = ix * a.dpx - (ax - (npatx * a.dpx - 0.5 * a.dpx));
  const double y = iy * a.dpy - (ay - (npaty * a.dpy - 0.5 * a.dpy));
  const double z = iz * a.dpz - (az - (npatz * a.dpz - 0.5 * a.dpz));
  const double r = sqrt(x * x + y * y + z * z);
  if (!(r < a.rlim)) return;
  const int kx = ix + (npatx - a.npmesh * natx[na]);
  const int ky = iy + (npaty - a.npmesh * naty[na]);
  const int kz = iz + (npatz - a.npmesh * natz[na]);
  double s[7] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double ylm[10];
  double weight = 1.0;
  if (r > a.eps) {
    if (a.nfiltyp == 1) weight = fermi_weight(r, a.filpp, a.rcut);
    const double rin = 1.0 / r;
    ylm[1] = 1.0;
    ylm[2] = rin * x;
    ylm[3] = rin * y;
    ylm[4] = rin * z;
    ylm[5] = rin * rin * (x * x - y * y);
    ylm[6] = -rin * rin * z * x;
    ylm[7] = rin * rin * (3.0 * z * z - r * r);
    ylm[8] = -rin * rin * y * z;
    ylm[9] = rin * rin * x * y;
    for (int iq = 1; iq <= a.nqct; ++iq) {
      const double qqq = a.dqq * iq;
      const double qqq2 = qqq * qqq;
      const double qqqr = qqq * r;
      const double qqqr2 = qqqr * qqqr;
      const double qqqrin = rin / qqq;
      const double qqqr2in = qqqrin * qqqrin;
      const double qqqr3in = qqqr2in * qqqrin;
      double sn, cs;
      sincos(qqqr, &sn, &cs);
      const double j0 = sn * qqqrin;
      const double j1 = (sn - qqqr * cs) * qqqr2in;
      const double j2 = ((3.0 - qqqr2) * sn - 3.0 * qqqr * cs) * qqqr3in;
#pragma unroll
      for (int c = 1; c <= 6; ++c)
        if (a.used & (1 << c)) {
          const double jl = c <= 2 ? j0 : (c <= 4 ? j1 : j2);
          s[c] = s[c] + cq[c - 1][iq] * jl * qqq2;
        }
    }
  } else {
    ylm[1] = 1.0;
#pragma unroll
    for (int m = 2; m <= 9; ++m) ylm[m] = 0.0;
    for (int iq = 1; iq <= a.nqct; ++iq) {
      const double qqq = a.dqq * iq;
#pragma unroll
      for (int c = 1; c <= 2; ++c)
        if (a.used & (1 << c)) s[c] = s[c] + cq[c - 1][iq] * qqq * qqq;
    }
  }
  const long sx = 2L * a.nxs, sy = 2L * a.nys, sz = 2L * a.nzs;
  const long nspd = sx * sy * sz;
  double* o = spd + (long)blockIdx.y * a.nprj * nspd +
              ((long)(kz + a.nzs - 1) * sy + (ky + a.nys - 1)) * sx + (kx + a.nxs - 1);
  for (int la = 0; la < a.nprj; ++la) {
    int c = a.col[la], m = a.ym[la];
    double sc = 0.0, yv = 0.0;
#pragma unroll
    for (int k = 1; k <= 6; ++k) sc = c == k ? s[k] : sc;
#pragma unroll
    for (int k = 1; k <= 9; ++k) yv = m == k ? ylm[k] : yv;
    o[(long)la * nspd] = sc * a.tq * a.dpxyz * a.nrm[la] * yv * weight;
  }
}

// One contraction pass of the double grid along one axis (0 = x, the
// contiguous one; 1 = y; 2 = z).  Output element (c0, c1, c2) of plane p
// (atom x projector), coordinates from the output's lower bounds lo0..lo2, is
//     sum_{j = js..je} in[p][... c_axis -> t*npmesh - (npmesh-1)/2 + j ...] w(j)
// with t = c_axis; the two other coordinates index the input directly (their
// lower bounds equal the output's), the contracted one from the input's lower
// bound ilo.  The sum runs in the order of the Fortran loop over j.
struct DgPass {
  int n0, n1, n2;           // output extents (x, y, z order)
  int lo0, lo1, lo2;        // output lower bounds (-n/2 + 1)
  long is0, is1, is2, isp;  // input strides (x, y, z, per atom-projector plane)
  int ilo;                  // input lower bound on the contracted axis
  int axis, npmesh, js, je, nw;
};

__global__ void k_dg_pass(DgPass d, int planes, const double* __restrict__ w,
                          const double* __restrict__ in, double* __restrict__ out) {
  const long per = (long)d.n0 * d.n1 * d.n2;
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= per * planes) return;
  const long pl = idx / per;
  const long rem = idx - pl * per;
  const int i0 = (int)(rem % d.n0), i1 = (int)((rem / d.n0) % d.n1), i2 = (int)(rem / ((long)d.n0 * d.n1));
  int c[3] = {i0 + d.lo0, i1 + d.lo1, i2 + d.lo2};
  const int kk = c[d.axis] * d.npmesh - (d.npmesh - 1) / 2;
  // input offsets of the two fixed axes (their input lower bounds equal the
  // output ones, except the contracted axis)
  long base = pl * d.isp;
  const long st[3] = {d.is0, d.is1, d.is2};
  const int lo[3] = {d.lo0, d.lo1, d.lo2};
  for (int ax = 0; ax < 3; ++ax)
    if (ax != d.axis) base += (long)(c[ax] - lo[ax]) * st[ax];
  double acc = 0.0;
  for (int j = d.js; j <= d.je; ++j)
    acc = acc + in[base + (long)(kk + j - d.ilo) * st[d.axis]] * w[j + d.nw];
  out[idx] = acc;
}

// v[((a0 + b) * nprj + la) * num_list + i] from the coarse box at the list points
__global__ void k_dg_gather(int nb, int nprj, int num_list, int a0, int npxmax, int npymax,
                            int npzmax, const int* __restrict__ natinf,
                            const int* __restrict__ lstx, const int* __restrict__ lsty,
                            const int* __restrict__ lstz, const double* __restrict__ box,
                            double* __restrict__ v) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)nb * nprj * num_list) return;
  const int i = (int)(idx % num_list);
  const long bl = idx / num_list;
  const int b = (int)(bl / nprj);
  const int na = a0 + b;
  double val = 0.0;
  if (i < natinf[na]) {
    const long e = (long)na * num_list + i;
    const long n0 = 2L * npxmax, n1 = 2L * npymax, n2 = 2L * npzmax;
    val = box[bl * n0 * n1 * n2 + ((long)(lstz[e] + npzmax - 1) * n1 + (lsty[e] + npymax - 1)) * n0 +
              (lstx[e] + npxmax - 1)];
  }
  v[(long)a0 * nprj * num_list + idx] = val;
}

double ylm_norm(int m) {
  const double pi = acos(-1.0);
  if (m == 1) return sqrt(1.0 / 4.0 / pi);
  if (m <= 4) return sqrt(3.0 / 4.0 / pi);
  if (m == 5) return sqrt(15.0 / 16.0 / pi);
  if (m == 7) return sqrt(5.0 / 16.0 / pi);
  return sqrt(15.0 / 4.0 / pi);
}

}  // namespace
}  // namespace rs

// pseudocalc_01a: w[j + nfdg*npmesh], j = -nfdg*npmesh .. nfdg*npmesh-1: the
// Lagrange weight of the coarse node 0 at the fine offset r = |j + 1/2|/npmesh
// (even npmesh) or |j|/npmesh (odd), piecewise over the intervals (k-1, k]
// with the nodes k+nfdg-1 .. k-nfdg (0 excluded), multiplied from the largest
// node down and divided by the product of their negatives.
extern "C" int rs_double_grid_weights(int nfdg, int npmesh, double* w) {
  if (nfdg < 1 || nfdg > 8 || npmesh < 1 || !w)
    return rs::fail(RS_EINVAL, "rs_double_grid_weights: bad nfdg or npmesh");
  const int n = nfdg * npmesh;
  const bool odd = npmesh % 2 == 1;
  const int js = odd ? -n + 1 : -n, je = n - 1;
  const double tmp1 = odd ? 0.0 : 0.5, tmp = 1.0 / npmesh;
  const int ntmp1 = odd ? 0 : 1;
  for (int j = -n; j <= je; ++j) w[j + n] = 0.0;
  for (int j = js; j <= je; ++j) {
    const double r = fabs(j * tmp + tmp1 * tmp);
    int k = 1;
    while (k < nfdg && abs(2 * j + ntmp1) > 2 * k * npmesh) ++k;
    double p = 1.0, d = 1.0;
    for (int m = k + nfdg - 1; m >= 1; --m) {
      p = p * (r - m);
      d = d * (double)(-m);
    }
    for (int m = 1; m <= nfdg - k; ++m) {
      p = p * (r + m);
      d = d * (double)m;
    }
    w[j + n] = p / d;
  }
  return RS_OK;
}

extern "C" int rs_projector_tables(
    int natom, int nprj, int num_list, int nxmax, int nymax, int nzmax, double dx, double dy,
    double dz, int npxmax, int npymax, int npzmax, int nfdg, int npmesh, const double* atx,
    const double* aty, const double* atz, const int* natx, const int* naty, const int* natz,
    const int* natinf, const int* lstx, const int* lsty, const int* lstz, const int* prj_col,
    const int* prj_m, int nqct, int nqmx, const double* coef, double rcut, double psftrad,
    double psctoff, double eps, int nfiltyp, double filpp, const double* wxyz, double* vnlocp,
    void* stream) {
  using namespace rs;
  if (natom < 0 || nprj < 1 || nprj > kMaxPrj || num_list < 1 || nxmax < 1 || nymax < 1 ||
      nzmax < 1 || npxmax < 1 || npymax < 1 || npzmax < 1 || nfdg < 1 || npmesh < 1 ||
      nqct < 0 || nqct > nqmx || nqct > kMaxQ || !(rcut > 0.0) || !(psftrad > 0.0) ||
      !(filpp > 0.0))
    return fail(RS_EINVAL, "rs_projector_tables: bad sizes or parameters");
  for (int la = 0; la < nprj; ++la)
    if (prj_col[la] < 1 || prj_col[la] > 6 || prj_m[la] < 1 || prj_m[la] > 9)
      return fail(RS_EINVAL, "rs_projector_tables: projector column or harmonic out of range");
  if (natom == 0) return RS_OK;
  keep_pool_memory();
  cudaStream_t st = as_stream(stream);
  const double pi = acos(-1.0);
  ProjArgs a;
  a.nprj = nprj; a.nqct = nqct; a.q1 = nqmx + 1; a.npmesh = npmesh; a.used = 0;
  a.npxd = npxmax * npmesh; a.npyd = npymax * npmesh; a.npzd = npzmax * npmesh;
  a.nxs = npmesh * (npxmax + nfdg) - (npmesh + 1) / 2;
  a.nys = npmesh * (npymax + nfdg) - (npmesh + 1) / 2;
  a.nzs = npmesh * (npzmax + nfdg) - (npmesh + 1) / 2;
  a.nxmax = nxmax; a.nymax = nymax; a.nzmax = nzmax;
  a.dx = dx; a.dy = dy; a.dz = dz;
  a.dpx = dx / npmesh; a.dpy = dy / npmesh; a.dpz = dz / npmesh;
  a.dpxyz = a.dpx * a.dpy * a.dpz;
  a.rcut = rcut;
  a.rlim = rcut * psctoff;
  a.dqq = pi / (rcut * psftrad);
  a.tq = 4.0 * pi * a.dqq * (1.0 / ((2.0 * pi) * (2.0 * pi) * (2.0 * pi)));
  a.eps = eps; a.filpp = filpp; a.nfiltyp = nfiltyp;
  for (int la = 0; la < nprj; ++la) {
    a.col[la] = prj_col[la];
    a.ym[la] = prj_m[la];
    a.nrm[la] = ylm_norm(prj_m[la]);
    a.used |= 1 << prj_col[la];
  }
  const long sx = 2L * a.nxs, sy = 2L * a.nys, sz = 2L * a.nzs;
  const long nspd = sx * sy * sz;
  const long n1 = sx * sy * 2L * npzmax;          // after the z pass
  const long n2 = sx * 2L * npymax * 2L * npzmax;  // after the y pass
  const long n3 = 8L * npxmax * npymax * npzmax;   // coarse box
  const long per_atom = (long)nprj * (nspd + n1 + n2 + n3);
  const int B = (int)std::max<long>(1, std::min<long>(natom, (2L << 30) / (8 * per_atom)));
  const int nw = 2 * nfdg * npmesh;
  // device copies of the per-atom data, the lists, the coefficients and weights
  const size_t bytes_atoms = sizeof(double) * 3 * natom + sizeof(int) * 4 * natom;
  const size_t bytes_lists = sizeof(int) * 3 * (size_t)natom * num_list;
  const size_t bytes_c = sizeof(double) * (size_t)(nqmx + 1) * 8 + sizeof(double) * nw;
  // vnlocp in device memory is written in place, in stream order; host
  // memory gets a copy at the end
  cudaPointerAttributes pa;
  const bool dev_out = cudaPointerGetAttributes(&pa, vnlocp) == cudaSuccess &&
                       (pa.type == cudaMemoryTypeDevice || pa.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  const size_t bytes_v = dev_out ? 0 : sizeof(double) * (size_t)natom * nprj * num_list;
  const size_t bytes_w = sizeof(double) * (size_t)B * per_atom;
  char* buf = nullptr;
  const size_t total = bytes_atoms + bytes_lists + bytes_c + bytes_v + bytes_w + 5 * 256;
  RS_CUDA(cudaMallocAsync((void**)&buf, total, st));
  size_t off = 0;
  auto take = [&](size_t n) {
    char* p = buf + off;
    off += (n + 255) & ~(size_t)255;
    return p;
  };
  double* d_at = (double*)take(sizeof(double) * 3 * natom);
  int* d_nat = (int*)take(sizeof(int) * 4 * natom);
  int* d_lst = (int*)take(bytes_lists);
  double* d_coef = (double*)take(bytes_c);
  double* d_w = d_coef + (size_t)(nqmx + 1) * 8;
  double* d_v = dev_out ? vnlocp : (double*)take(bytes_v);
  double* d_work = (double*)take(bytes_w);
  int rc = RS_OK;
  cudaError_t e = cudaSuccess;
  auto h2d = [&](void* dst, const void* src, size_t n) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, src, n, cudaMemcpyHostToDevice, st);
  };
  h2d(d_at, atx, sizeof(double) * natom);
  h2d(d_at + natom, aty, sizeof(double) * natom);
  h2d(d_at + 2 * natom, atz, sizeof(double) * natom);
  h2d(d_nat, natx, sizeof(int) * natom);
  h2d(d_nat + natom, naty, sizeof(int) * natom);
  h2d(d_nat + 2 * natom, natz, sizeof(int) * natom);
  h2d(d_nat + 3 * natom, natinf, sizeof(int) * natom);
  h2d(d_lst, lstx, sizeof(int) * (size_t)natom * num_list);
  h2d(d_lst + (size_t)natom * num_list, lsty, sizeof(int) * (size_t)natom * num_list);
  h2d(d_lst + 2 * (size_t)natom * num_list, lstz, sizeof(int) * (size_t)natom * num_list);
  h2d(d_coef, coef, sizeof(double) * (size_t)(nqmx + 1) * 8);
  h2d(d_w, wxyz, sizeof(double) * nw);
  if (e != cudaSuccess) rc = cuda_status(e, "rs_projector_tables: upload");
  const int n = nfdg * npmesh;
  const int js = npmesh % 2 == 1 ? -n + 1 : -n, je = n - 1;
  for (int a0 = 0; a0 < natom && rc == RS_OK; a0 += B) {
    const int nb = std::min(B, natom - a0);
    double* spd = d_work;
    double* t1 = spd + (long)nb * nprj * nspd;
    double* t2 = t1 + (long)nb * nprj * n1;
    double* t0 = t2 + (long)nb * nprj * n2;
    e = cudaMemsetAsync(spd, 0, sizeof(double) * (size_t)nb * nprj * nspd, st);
    if (e != cudaSuccess) { rc = cuda_status(e, "rs_projector_tables: memset"); break; }
    const long box = 8L * a.npxd * a.npyd * a.npzd;
    k_proj_fine<<<dim3(div_up(box, 256), nb), 256, 0, st>>>(
        a, a0, d_at, d_at + natom, d_at + 2 * natom, d_nat, d_nat + natom, d_nat + 2 * natom,
        d_coef, spd);
    const int planes = nb * nprj;
    // z pass: (sx, sy, 2 npzmax) from the fine array
    DgPass pz{(int)sx, (int)sy, 2 * npzmax, -a.nxs + 1, -a.nys + 1, -npzmax + 1,
              1, sx, sx * sy, nspd, -a.nzs + 1, 2, npmesh, js, je, n};
    k_dg_pass<<<div_up((long)planes * n1, 256), 256, 0, st>>>(pz, planes, d_w, spd, t1);
    // y pass: (sx, 2 npymax, 2 npzmax) from t1
    DgPass py{(int)sx, 2 * npymax, 2 * npzmax, -a.nxs + 1, -npymax + 1, -npzmax + 1,
              1, sx, sx * sy, n1, -a.nys + 1, 1, npmesh, js, je, n};
    k_dg_pass<<<div_up((long)planes * n2, 256), 256, 0, st>>>(py, planes, d_w, t1, t2);
    // x pass: (2 npxmax, 2 npymax, 2 npzmax) from t2
    DgPass px{2 * npxmax, 2 * npymax, 2 * npzmax, -npxmax + 1, -npymax + 1, -npzmax + 1,
              1, sx, sx * 2L * npymax, n2, -a.nxs + 1, 0, npmesh, js, je, n};
    k_dg_pass<<<div_up((long)planes * n3, 256), 256, 0, st>>>(px, planes, d_w, t2, t0);
    k_dg_gather<<<div_up((long)planes * num_list, 256), 256, 0, st>>>(
        nb, nprj, num_list, a0, npxmax, npymax, npzmax, d_nat + 3 * natom, d_lst,
        d_lst + (size_t)natom * num_list, d_lst + 2 * (size_t)natom * num_list, t0, d_v);
    e = cudaGetLastError();
    if (e != cudaSuccess) rc = cuda_status(e, "rs_projector_tables: kernels");
  }
  if (rc == RS_OK && !dev_out) {
    e = cudaMemcpyAsync(vnlocp, d_v, sizeof(double) * (size_t)natom * nprj * num_list,
                        cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_status(e, "rs_projector_tables: download");
  }
  cudaFreeAsync(buf, st);
  return rc;
}
