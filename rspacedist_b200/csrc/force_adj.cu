// force_adj.cu -- atomic forces by one adjoint pass over the converged bands.
//
// The energy of a converged SCF depends on an atom position R_a through the
// local pseudopotential, the ion-ion energy and the projectors.  For the
// projector part, with rp_i = <p_i|psi_l> (vnlocp holds p times dV) and the
// S-orthonormality constraint of each band,
//
//   F_a = 2 sum_l f_l sum_ij (D_a - e_l S_a)_ij rp_i <grad p_j|psi_l>,
//
// the exact derivative of the discrete energy (grad p = -d p / d R_a).  The
// reference forms the same sum with the finite-difference derivative of the
// bands instead (force_eig_r, force8f.F90:9-195, with force_r_02..04).
//
// Nothing is stored per projector: every block recomputes, at each point of
// its atom's sphere list, the projector values p_j and their gradients from
// the radial tables (linear interpolation on a uniform radial grid, real
// harmonics in the order of pseudocalc8f.F90:2962-2970, zero outside r_cut),
// and contracts them with a block of 32 bands staged in shared memory.  One
// pass yields <p_j|psi_l> and <grad p_j|psi_l> of all bands; a second small
// kernel forms the forces per atom in FP64, band by band in order.
#include <math.h>

#include <vector>

#include "rs_common.cuh"

namespace rs {
namespace {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr int kBB = 32;     // bands per block
constexpr int kCH = 32;     // sphere points per staged chunk
constexpr int kMaxP = 18;   // projectors per atom (s*2 + p*6 + d*10)
constexpr int kRows = 4 * kMaxP;

struct AdjArgs {
  int natom, P, num_list, nb;
  long N;
  int nx, ny, nz;
  double dx, dy, dz, dvol, rcut, dr;
  int nr;
};

// value and gradient of projector j at separation (x, y, z) from its atom:
// P(r) Y(x, y, z) dV with P the linear interpolant of the channel table
__device__ void projector_vg(const AdjArgs& A, const double* tab, int l, int form, double x,
                             double y, double z, double* v, double* gx, double* gy, double* gz) {
  const double r = sqrt(x * x + y * y + z * z);
  if (!(r < A.rcut)) {
    *v = *gx = *gy = *gz = 0.0;
    return;
  }
  // np.interp on the grid i*dr: slope*(r - x_j) + p_j on the segment
  // x_j <= r < x_(j+1); the last value beyond the grid (zero slope)
  double pr, dpr;
  if (r >= (double)(A.nr - 1) * A.dr) {
    pr = tab[A.nr - 1];
    dpr = 0.0;
  } else {
    int j = (int)(r / A.dr);
    if (j > A.nr - 2) j = A.nr - 2;
    while (j > 0 && (double)j * A.dr > r) --j;
    while (j < A.nr - 2 && (double)(j + 1) * A.dr <= r) ++j;
    const double xj = (double)j * A.dr;
    dpr = (tab[j + 1] - tab[j]) / ((double)(j + 1) * A.dr - xj);
    pr = dpr * (r - xj) + tab[j];
  }
  const double rin = r > 1e-12 ? 1.0 / r : 0.0;
  double c, poly, px, py, pz;
  switch (form) {
    case 0: c = sqrt(1.0 / 4.0 / kPi); poly = 1.0; px = py = pz = 0.0; break;
    case 1: c = sqrt(3.0 / 4.0 / kPi); poly = x; px = 1.0; py = pz = 0.0; break;
    case 2: c = sqrt(3.0 / 4.0 / kPi); poly = y; py = 1.0; px = pz = 0.0; break;
    case 3: c = sqrt(3.0 / 4.0 / kPi); poly = z; pz = 1.0; px = py = 0.0; break;
    case 4: c = sqrt(15.0 / 16.0 / kPi); poly = x * x - y * y; px = 2 * x; py = -2 * y; pz = 0.0; break;
    case 5: c = sqrt(15.0 / 4.0 / kPi); poly = -z * x; px = -z; py = 0.0; pz = -x; break;
    case 6: c = sqrt(5.0 / 16.0 / kPi); poly = 3 * z * z - r * r; px = -2 * x; py = -2 * y; pz = 4 * z; break;
    case 7: c = sqrt(15.0 / 4.0 / kPi); poly = -y * z; px = 0.0; py = -z; pz = -y; break;
    default: c = sqrt(15.0 / 4.0 / kPi); poly = x * y; px = y; py = x; pz = 0.0; break;
  }
  // Y = c poly / r^l; dY/dx_k = c (dpoly_k / r^l - l poly x_k / r^(l+2))
  double rl = 1.0;
  for (int i = 0; i < l; ++i) rl *= rin;
  const double yv = c * poly * rl;
  const double t = (double)l * c * poly * rl * rin * rin;
  const double dyx = c * px * rl - t * x, dyy = c * py * rl - t * y, dyz = c * pz * rl - t * z;
  const double rad = dpr * rin;  // d P / d x_k = P'(r) x_k / r
  *v = pr * yv * A.dvol;
  *gx = (rad * x * yv + pr * dyx) * A.dvol;
  *gy = (rad * y * yv + pr * dyy) * A.dvol;
  *gz = (rad * z * yv + pr * dyz) * A.dvol;
}

// per (atom, band block): G[l][a][row], rows 0..P-1 = <p_j|psi_l>, then
// P..2P-1, 2P..3P-1, 3P..4P-1 = <d p_j / d x|psi_l>, y, z
template <class T>
__global__ void __launch_bounds__(256) k_force_adjoint(
    AdjArgs A, const double* __restrict__ xyz, const int* __restrict__ nat,
    const int* __restrict__ natinf, const int* __restrict__ lxyz, const int* __restrict__ lst,
    const double* __restrict__ tabs, const int* __restrict__ prj_tab,
    const int* __restrict__ prj_l, const int* __restrict__ prj_form, const T* __restrict__ psi,
    double* __restrict__ G) {
  __shared__ double sv[kRows][kCH];
  __shared__ double sp[kCH][kBB + 1];
  const int a = blockIdx.x;
  const int b0 = blockIdx.y * kBB;
  const int nbb = min(kBB, A.nb - b0);
  const int P = A.P, rows = 4 * P;
  const int tid = threadIdx.x;
  const int band = tid % kBB;
  const int rg = tid / kBB;  // 8 row groups
  double acc[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) acc[i] = 0.0;
  const int n = natinf[a];
  const double tx = xyz[3 * a] - (nat[3 * a] * A.dx - 0.5 * A.dx);
  const double ty = xyz[3 * a + 1] - (nat[3 * a + 1] * A.dy - 0.5 * A.dy);
  const double tz = xyz[3 * a + 2] - (nat[3 * a + 2] * A.dz - 0.5 * A.dz);
  for (int c0 = 0; c0 < n; c0 += kCH) {
    const int cn = min(kCH, n - c0);
    __syncthreads();
    // projector values and gradients of the chunk: (point, projector) pairs
    for (int w = tid; w < kCH * P; w += blockDim.x) {
      const int pt = w % kCH, j = w / kCH;
      double v = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
      if (pt < cn) {
        const long e = (long)a * A.num_list + c0 + pt;
        const double x = lxyz[3 * e] * A.dx - tx;
        const double y = lxyz[3 * e + 1] * A.dy - ty;
        const double z = lxyz[3 * e + 2] * A.dz - tz;
        projector_vg(A, tabs + (long)prj_tab[j] * A.nr, prj_l[j], prj_form[j], x, y, z, &v, &gx,
                     &gy, &gz);
      }
      sv[j][pt] = v;
      sv[P + j][pt] = gx;
      sv[2 * P + j][pt] = gy;
      sv[3 * P + j][pt] = gz;
    }
    // the bands of the block at the chunk's points
    for (int w = tid; w < kCH * kBB; w += blockDim.x) {
      const int pt = w / kBB, bb = w % kBB;
      double val = 0.0;
      if (pt < cn && bb < nbb)
        val = (double)psi[(long)(b0 + bb) * A.N + lst[(long)a * A.num_list + c0 + pt]];
      sp[pt][bb] = val;
    }
    __syncthreads();
    for (int pt = 0; pt < cn; ++pt) {
      const double s = sp[pt][band];
#pragma unroll
      for (int i = 0; i < 9; ++i) {
        const int row = rg + 8 * i;
        if (row < rows) acc[i] = fma(sv[row][pt], s, acc[i]);
      }
    }
  }
  if (band < nbb) {
    double* out = G + ((long)(b0 + band) * A.natom + a) * rows;
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      const int row = rg + 8 * i;
      if (row < rows) out[row] = acc[i];
    }
  }
}

// F_a = 2 sum_l f_l sum_ij (D - e_l S)_ij rp_i g_j, bands in order, and the
// recomputed <p|psi> copied out when asked
__global__ void k_force_adjoint_sum(int natom, int P, int nb, const double* __restrict__ G,
                                    const double* __restrict__ dij,
                                    const double* __restrict__ sss,
                                    const double* __restrict__ sval,
                                    const double* __restrict__ occ, double* __restrict__ f) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const double* D = dij + (long)a * P * P;
  const double* S = sss ? sss + (long)a * P * P : nullptr;
  double fx = 0.0, fy = 0.0, fz = 0.0;
  for (int l = 0; l < nb; ++l) {
    const double* g = G + ((long)l * natom + a) * 4 * P;
    const double w = 2.0 * occ[l];
    if (w == 0.0) continue;
    for (int i = 0; i < P; ++i)
      for (int j = 0; j < P; ++j) {
        double d = D[i * P + j];
        if (S) d -= sval[l] * S[i * P + j];
        const double t = w * d * g[i];
        fx += t * g[P + j];
        fy += t * g[2 * P + j];
        fz += t * g[3 * P + j];
      }
  }
  f[3 * a] = fx;
  f[3 * a + 1] = fy;
  f[3 * a + 2] = fz;
}

template <class T>
int force_adjoint(int natom, int P, int num_list, const double* atxyz, const int* natxyz,
                  const int* natinf, const int* lstxyz, const int* lst, int ntab, int nr,
                  double dr, const double* tabs, const int* prj_tab, const int* prj_l,
                  const int* prj_form, double rcut, int nx, int ny, int nz, double dx,
                  double dy, double dz, const double* dij, const double* sss, const T* psi,
                  const double* sval, const double* occ, int nb, double* force, double* rp_out,
                  cudaStream_t st) {
  if (natom <= 0 || P <= 0 || P > kMaxP || num_list <= 0 || nb <= 0 || ntab <= 0 || nr < 2 ||
      !atxyz || !natxyz || !natinf || !lstxyz || !lst || !tabs || !prj_tab || !prj_l ||
      !prj_form || !dij || !psi || !sval || !occ || !force)
    return fail(RS_EINVAL, "rs_force_adjoint: bad arguments");
  for (int j = 0; j < P; ++j)
    if (prj_tab[j] < 0 || prj_tab[j] >= ntab || prj_l[j] < 0 || prj_l[j] > 2 || prj_form[j] < 0 ||
        prj_form[j] > 8)
      return fail(RS_EINVAL, "rs_force_adjoint: bad projector layout");
  for (int a = 0; a < natom; ++a)
    if (natinf[a] < 0 || natinf[a] > num_list)
      return fail(RS_EINVAL, "rs_force_adjoint: natinf out of range");
  const long N = (long)nx * ny * nz;
  const long L = (long)natom * num_list;
  for (long e = 0; e < L; ++e)
    if (lst[e] < 0 || lst[e] >= N) return fail(RS_EINVAL, "rs_force_adjoint: list point out of range");
  // device copies of the inputs and the band sums G
  const size_t nG = (size_t)nb * natom * 4 * P;
  const size_t words_d = 3 * (size_t)natom + (size_t)ntab * nr + nG + 3 * (size_t)natom;
  const size_t words_i = 3 * (size_t)natom + natom + 3 * (size_t)L + L + 3 * (size_t)P;
  char* buf = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&buf, sizeof(double) * words_d + sizeof(int) * words_i + 64, st));
  double* d_xyz = (double*)buf;
  double* d_tabs = d_xyz + 3 * natom;
  double* d_G = d_tabs + (size_t)ntab * nr;
  double* d_f = d_G + nG;
  int* d_nat = (int*)(d_f + 3 * natom);
  int* d_natinf = d_nat + 3 * natom;
  int* d_lxyz = d_natinf + natom;
  int* d_lst = d_lxyz + 3 * L;
  int* d_pt = d_lst + L;
  int* d_pl = d_pt + P;
  int* d_pf = d_pl + P;
  std::vector<int> lx3(3 * L), nat3(3 * natom);
  for (long e = 0; e < L; ++e) {
    lx3[3 * e] = lstxyz[e];
    lx3[3 * e + 1] = lstxyz[L + e];
    lx3[3 * e + 2] = lstxyz[2 * L + e];
  }
  for (int a = 0; a < natom; ++a) {
    nat3[3 * a] = natxyz[a];
    nat3[3 * a + 1] = natxyz[natom + a];
    nat3[3 * a + 2] = natxyz[2 * natom + a];
  }
  cudaMemcpyAsync(d_xyz, atxyz, sizeof(double) * 3 * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_tabs, tabs, sizeof(double) * ntab * nr, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_nat, nat3.data(), sizeof(int) * 3 * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_natinf, natinf, sizeof(int) * natom, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_lxyz, lx3.data(), sizeof(int) * 3 * L, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_lst, lst, sizeof(int) * L, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_pt, prj_tab, sizeof(int) * P, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_pl, prj_l, sizeof(int) * P, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_pf, prj_form, sizeof(int) * P, cudaMemcpyHostToDevice, st);
  AdjArgs A{natom, P, num_list, nb, N, nx, ny, nz, dx, dy, dz, dx * dy * dz, rcut, dr, nr};
  const dim3 grid(natom, (nb + kBB - 1) / kBB);
  k_force_adjoint<T><<<grid, 256, 0, st>>>(A, d_xyz, d_nat, d_natinf, d_lxyz, d_lst, d_tabs,
                                           d_pt, d_pl, d_pf, psi, d_G);
  k_force_adjoint_sum<<<div_up(natom, 64), 64, 0, st>>>(natom, P, nb, d_G, dij, sss, sval, occ,
                                                        d_f);
  if (rp_out) {
    // rp[l][a][j] = G[l][a][j]
    cudaMemcpy2DAsync(rp_out, sizeof(double) * P, d_G, sizeof(double) * 4 * P,
                      sizeof(double) * P, (size_t)nb * natom, cudaMemcpyDeviceToDevice, st);
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(force, d_f, sizeof(double) * 3 * natom, cudaMemcpyDeviceToHost, st);
  cudaFreeAsync(buf, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(e, "rs_force_adjoint");
  return RS_OK;
}

}  // namespace
}  // namespace rs

#define RS_FORCE_ADJ_ARGS                                                                    \
  int natom, int nprj, int num_list, const double *atxyz, const int *natxyz,                 \
      const int *natinf, const int *lstxyz, const int *lst, int ntab, int nr, double dr,     \
      const double *tabs, const int *prj_tab, const int *prj_l, const int *prj_form,         \
      double rcut, int nx, int ny, int nz, double dx, double dy, double dz, const double *dij, \
      const double *sss
#define RS_FORCE_ADJ_PASS                                                                     \
  natom, nprj, num_list, atxyz, natxyz, natinf, lstxyz, lst, ntab, nr, dr, tabs, prj_tab,    \
      prj_l, prj_form, rcut, nx, ny, nz, dx, dy, dz, dij, sss

extern "C" int rs_force_adjoint_f64(RS_FORCE_ADJ_ARGS, const double* psi, const double* sval,
                                    const double* occ, int nb, double* force, double* rp,
                                    void* stream) {
  return rs::force_adjoint<double>(RS_FORCE_ADJ_PASS, psi, sval, occ, nb, force, rp,
                                   rs::as_stream(stream));
}

extern "C" int rs_force_adjoint_f32(RS_FORCE_ADJ_ARGS, const float* psi, const double* sval,
                                    const double* occ, int nb, double* force, double* rp,
                                    void* stream) {
  return rs::force_adjoint<float>(RS_FORCE_ADJ_PASS, psi, sval, occ, nb, force, rp,
                                  rs::as_stream(stream));
}
