// force.cu -- nonlocal pseudopotential force on the atoms (force_eig_r,
// kukan/force8f.F90:9-195):
//
//   F_a,x = - sum_l 2 f_l sum_j sum_i <p_i|psi_l> (D_a - eps_l S_a)_ij <p_j|d_x psi_l>
//
// with d_x psi the nf-order first derivative (force_r_02/03/04,
// force8f.F90:409-490) and S dropped when no S matrix is given (NC).
//
// The band-parallel work -- the projections <p|psi> of all bands, then per
// axis and band chunk the derivative and its projections -- runs as batched
// launches of the gradient and gather-dot kernels.  The contraction into the
// forces keeps the reference's accumulation order (axis, band, j, i) in one
// FMA chain per atom and axis: a thread per atom carries F across chunks, so
// the result is bit-for-bit that of the sequential loop.
#include <algorithm>

#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {

template <class T>
int launch_nl_dot(const rs_geom* g, const T* psi, int nb, double* rp, cudaStream_t st);

namespace {

// f[a] -= 2 f_l (r_i rd_j) (D_ji - eps_l S_ji), bands l of this chunk in order
__global__ void k_force_acc(int natom, int P, const int* __restrict__ nprj,
                            const double* __restrict__ dij, const double* __restrict__ sss,
                            const double* __restrict__ sval, const double* __restrict__ occ,
                            const double* __restrict__ rp, const double* __restrict__ rdp,
                            int nl, double* __restrict__ f) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= natom) return;
  const int n = nprj[a];
  const double* D = dij + (long)a * P * P;
  const double* Sm = sss ? sss + (long)a * P * P : nullptr;
  double acc = f[a];
  for (int l = 0; l < nl; ++l) {
    const double* r = rp + ((long)l * natom + a) * P;
    const double* rd = rdp + ((long)l * natom + a) * P;
    const double w = 2.0 * occ[l];
    const double e = -sval[l];
    for (int j = 0; j < n; ++j)
      for (int i = 0; i < n; ++i) {
        double d = D[j * P + i];
        if (Sm) d = fma(e, Sm[j * P + i], d);
        acc = fma(-(w * (r[i] * rd[j])), d, acc);
      }
  }
  f[a] = acc;
}

template <class T>
int force_nl(const rs_geom* g, const double* dij, const double* sss, const T* psi,
             const double* sval, const double* occ, int nb, double* fxyz, cudaStream_t st) {
  const int A = g->natom, P = g->nprjmx;
  RS_CUDA(cudaMemsetAsync(fxyz, 0, sizeof(double) * 3 * (size_t)(A > 0 ? A : 1), st));
  if (nb <= 0 || A == 0) return RS_OK;
  // bands per chunk: the derivative of a chunk takes at most 512 MB
  const long per = g->N * (long)sizeof(T);
  const int chunk = (int)std::max(1L, std::min((long)nb, (512L << 20) / per));
  double *rp = nullptr, *rdp = nullptr;
  T* grad = nullptr;
  RS_CUDA(cudaMallocAsync((void**)&rp, sizeof(double) * (size_t)nb * A * P, st));
  cudaError_t e = cudaMallocAsync((void**)&rdp, sizeof(double) * (size_t)chunk * A * P, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&grad, (size_t)per * chunk, st);
  int rc = e == cudaSuccess ? RS_OK : cuda_status(e, "force_nl: work arrays");
  if (rc == RS_OK) rc = launch_nl_dot<T>(g, psi, nb, rp, st);
  for (int axis = 0; axis < 3 && rc == RS_OK; ++axis) {
    for (int l0 = 0; l0 < nb && rc == RS_OK; l0 += chunk) {
      const int nl = std::min(chunk, nb - l0);
      rc = launch_gradient<T>(g, axis, psi + (long)l0 * g->N, grad, nl, st);
      if (rc == RS_OK) rc = launch_nl_dot<T>(g, grad, nl, rdp, st);
      if (rc == RS_OK) {
        k_force_acc<<<div_up(A, 128), 128, 0, st>>>(A, P, g->d_nprj, dij, sss, sval + l0,
                                                    occ + l0, rp + (long)l0 * A * P, rdp, nl,
                                                    fxyz + (long)axis * A);
        e = cudaGetLastError();
        if (e != cudaSuccess) rc = cuda_status(e, "k_force_acc");
      }
    }
  }
  if (rp) cudaFreeAsync(rp, st);
  if (rdp) cudaFreeAsync(rdp, st);
  if (grad) cudaFreeAsync(grad, st);
  return rc;
}

}  // namespace
}  // namespace rs

extern "C" int rs_force_nl_f64(const rs_geom* g, const double* dij, const double* sss,
                               const double* psi, const double* sval, const double* occ, int nb,
                               double* fxyz, void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_force_nl_f64: null geometry");
  if (nb < 0 || (nb > 0 && (!psi || !sval || !occ)) || !fxyz || (g->natom > 0 && !dij))
    return rs::fail(RS_EINVAL, "rs_force_nl_f64: null or negative argument");
  return rs::force_nl<double>(g, dij, sss, psi, sval, occ, nb, fxyz, rs::as_stream(stream));
}

extern "C" int rs_force_nl_f32(const rs_geom* g, const double* dij, const double* sss,
                               const float* psi, const double* sval, const double* occ, int nb,
                               double* fxyz, void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_force_nl_f32: null geometry");
  if (nb < 0 || (nb > 0 && (!psi || !sval || !occ)) || !fxyz || (g->natom > 0 && !dij))
    return rs::fail(RS_EINVAL, "rs_force_nl_f32: null or negative argument");
  return rs::force_nl<float>(g, dij, sss, psi, sval, occ, nb, fxyz, rs::as_stream(stream));
}
