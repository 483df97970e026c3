// state.cu -- a device-resident state handle over the C ABI: the band arrays
// (psi, S psi, H psi, <p|psi>), the geometry, veff, D and S of one cell stay on
// the GPU between calls, and host memory is touched only to upload inputs and
// to read results back (sval, residual_states, rho, psi for checkpoints), as
// the drop-in replacement of kukan's scf_diag / scf_charge call sites needs.
// Every entry point here is a thin composition of the functional entry points
// of include/rspace_b200.h on the state's stream.
#include <string.h>

#include <vector>

#include "rs_common.cuh"

struct rs_state {
  int prec = 64;  // 32 (mixed path) or 64 (plain FP64 path)
  int nx = 0, ny = 0, nz = 0, nf = 4;
  double dx = 0, dy = 0, dz = 0;
  long N = 0;
  int M = 0;
  cudaStream_t st = nullptr;
  rs_geom* g = nullptr;
  int natom = 0, nprjmx = 0;
  void* psi = nullptr;
  void* spsi = nullptr;
  void* hpsi = nullptr;
  double* rp = nullptr;
  void* veff = nullptr;
  double* dij = nullptr;
  double* sss = nullptr;  // nullptr: S = 1 (spsi is a copy of psi, kept equal)
  size_t esize() const { return prec == 32 ? sizeof(float) : sizeof(double); }
};

namespace {

__global__ void k_f64_to_f32(long n, const double* __restrict__ a, float* __restrict__ b) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) b[i] = (float)a[i];
}

void free_dev(void*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}
template <class T>
void free_dev(T*& p) {
  if (p) cudaFree(p);
  p = nullptr;
}

int need_geometry(const rs_state* s, const char* fn) {
  if (!s) return rs::fail(RS_EINVAL, std::string(fn) + ": null state");
  if (!s->g) return rs::fail(RS_EINVAL, std::string(fn) + ": no geometry uploaded");
  return RS_OK;
}

}  // namespace

extern "C" int rs_create(rs_state** out, int precision, int nx, int ny, int nz, int nf, double dx,
                         double dy, double dz, int nbands, void* stream) {
  if (!out) return rs::fail(RS_EINVAL, "rs_create: null handle");
  *out = nullptr;
  if (precision != 32 && precision != 64) return rs::fail(RS_EINVAL, "rs_create: precision 32 or 64");
  if (nx <= 0 || ny <= 0 || nz <= 0 || nbands <= 0 || !(dx > 0) || !(dy > 0) || !(dz > 0))
    return rs::fail(RS_EINVAL, "rs_create: bad grid or band count");
  rs_state* s = new rs_state;
  s->prec = precision;
  s->nx = nx; s->ny = ny; s->nz = nz; s->nf = nf;
  s->dx = dx; s->dy = dy; s->dz = dz;
  s->N = (long)nx * ny * nz;
  s->M = nbands;
  s->st = rs::as_stream(stream);
  const size_t bytes = s->esize() * (size_t)s->N * nbands;
  cudaError_t e = cudaMalloc(&s->psi, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->spsi, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->hpsi, bytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->veff, s->esize() * (size_t)s->N);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->hpsi, 0, bytes, s->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->veff, 0, s->esize() * (size_t)s->N, s->st);
  if (e != cudaSuccess) {
    rs_destroy(s);
    return rs::cuda_status(e, "rs_create: band arrays");
  }
  *out = s;
  return RS_OK;
}

extern "C" int rs_destroy(rs_state* s) {
  if (!s) return RS_OK;
  if (s->st) cudaStreamSynchronize(s->st);
  if (s->g) rs_geom_destroy(s->g);
  free_dev(s->psi); free_dev(s->spsi); free_dev(s->hpsi); free_dev(s->veff);
  free_dev(s->rp); free_dev(s->dij); free_dev(s->sss);
  delete s;
  return RS_OK;
}

extern "C" int rs_upload_geometry(rs_state* s, int natom, int nprjmx, int num_list,
                                  const int* nprj, const int* natinf, const int* lst,
                                  const double* vnlocp, const double* dij, const double* sss) {
  if (!s) return rs::fail(RS_EINVAL, "rs_upload_geometry: null state");
  if (natom > 0 && !dij) return rs::fail(RS_EINVAL, "rs_upload_geometry: D is required");
  rs_geom* g = nullptr;
  int rc = rs_geom_create(&g, s->nx, s->ny, s->nz, s->nf, s->dx, s->dy, s->dz, natom, nprjmx,
                          num_list, nprj, natinf, lst, vnlocp);
  if (rc) return rc;
  if (s->g) rs_geom_destroy(s->g);
  s->g = g;
  s->natom = natom;
  s->nprjmx = nprjmx;
  free_dev(s->rp); free_dev(s->dij); free_dev(s->sss);
  const size_t nrp = (size_t)natom * nprjmx, nm = nrp * nprjmx;
  cudaError_t e = cudaMalloc((void**)&s->rp, sizeof(double) * (nrp > 0 ? nrp : 1) * s->M);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->rp, 0, sizeof(double) * (nrp > 0 ? nrp : 1) * s->M, s->st);
  if (e == cudaSuccess && nm > 0) {
    e = cudaMalloc((void**)&s->dij, sizeof(double) * nm);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->dij, dij, sizeof(double) * nm, cudaMemcpyHostToDevice, s->st);
  }
  if (e == cudaSuccess && sss && nm > 0) {
    e = cudaMalloc((void**)&s->sss, sizeof(double) * nm);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(s->sss, sss, sizeof(double) * nm, cudaMemcpyHostToDevice, s->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  return e == cudaSuccess ? RS_OK : rs::cuda_status(e, "rs_upload_geometry");
}

extern "C" int rs_set_potential(rs_state* s, const double* veff) {
  if (!s || !veff) return rs::fail(RS_EINVAL, "rs_set_potential: null argument");
  cudaError_t e = cudaSuccess;
  if (s->prec == 64) {
    e = cudaMemcpyAsync(s->veff, veff, sizeof(double) * s->N, cudaMemcpyHostToDevice, s->st);
  } else {
    double* tmp = nullptr;
    e = cudaMallocAsync((void**)&tmp, sizeof(double) * s->N, s->st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(tmp, veff, sizeof(double) * s->N, cudaMemcpyHostToDevice, s->st);
    if (e == cudaSuccess) {
      k_f64_to_f32<<<rs::div_up(s->N, 256), 256, 0, s->st>>>(s->N, tmp, (float*)s->veff);
      e = cudaGetLastError();
    }
    if (tmp) cudaFreeAsync(tmp, s->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  return e == cudaSuccess ? RS_OK : rs::cuda_status(e, "rs_set_potential");
}

// psi (host, M x N in the state's precision); S psi starts as a copy, H psi and
// <p|psi> as zeros, as before kukan's first orthogonalisation
extern "C" int rs_upload_bands(rs_state* s, const void* psi) {
  int rc = need_geometry(s, "rs_upload_bands");
  if (rc) return rc;
  if (!psi) return rs::fail(RS_EINVAL, "rs_upload_bands: null psi");
  const size_t bytes = s->esize() * (size_t)s->N * s->M;
  const size_t nrp = (size_t)s->natom * s->nprjmx;
  cudaError_t e = cudaMemcpyAsync(s->psi, psi, bytes, cudaMemcpyHostToDevice, s->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s->spsi, s->psi, bytes, cudaMemcpyDeviceToDevice, s->st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s->hpsi, 0, bytes, s->st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(s->rp, 0, sizeof(double) * (nrp > 0 ? nrp : 1) * s->M, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  return e == cudaSuccess ? RS_OK : rs::cuda_status(e, "rs_upload_bands");
}

extern "C" int rs_download_bands(rs_state* s, void* psi) {
  if (!s || !psi) return rs::fail(RS_EINVAL, "rs_download_bands: null argument");
  const size_t bytes = s->esize() * (size_t)s->N * s->M;
  cudaError_t e = cudaMemcpyAsync(psi, s->psi, bytes, cudaMemcpyDeviceToHost, s->st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  return e == cudaSuccess ? RS_OK : rs::cuda_status(e, "rs_download_bands");
}

extern "C" int rs_state_arrays(rs_state* s, void** psi, void** spsi, void** hpsi, double** rp,
                               void** veff) {
  if (!s) return rs::fail(RS_EINVAL, "rs_state_arrays: null state");
  if (psi) *psi = s->psi;
  if (spsi) *spsi = s->sss ? s->spsi : s->psi;
  if (hpsi) *hpsi = s->hpsi;
  if (rp) *rp = s->rp;
  if (veff) *veff = s->veff;
  return RS_OK;
}

// orthogonalization_r_01 over all bands (kukan8f.F90:466-487)
extern "C" int rs_orthogonalize(rs_state* s, int cmpt) {
  int rc = need_geometry(s, "rs_orthogonalize");
  if (rc) return rc;
  void* sp = s->sss ? s->spsi : s->psi;
  if (s->prec == 64)
    return rs_orthogonalize_f64(s->g, s->sss, s->M, (double*)s->psi, (double*)sp, s->rp, cmpt,
                                s->st);
  return rs_orthogonalize_f32(s->g, s->sss, s->M, (float*)s->psi, (float*)sp, s->rp, cmpt,
                              s->st);
}

// H psi of every band from the state's psi and <p|psi>
extern "C" int rs_hpsi(rs_state* s) {
  int rc = need_geometry(s, "rs_hpsi");
  if (rc) return rc;
  if (s->prec == 64)
    return rs_hpsi_f64(s->g, (const double*)s->veff, s->dij, s->rp, (const double*)s->psi,
                       (double*)s->hpsi, s->M, s->st);
  return rs_hpsi_f32(s->g, (const float*)s->veff, s->dij, s->rp, (const float*)s->psi,
                     (float*)s->hpsi, s->M, s->st);
}

// scf_diag (scf_diag8f.F90:6-316) on the state: sval and resid are host arrays
// of M values (in/out, kukan's sval and residual_states)
extern "C" int rs_diag_step(rs_state* s, const rs_solver_prm* prm, int iscf, double* sval,
                            double* resid, int* ksconv, int* ksitmax) {
  int rc = need_geometry(s, "rs_diag_step");
  if (rc) return rc;
  if (!prm || !sval || !resid || !ksconv || !ksitmax)
    return rs::fail(RS_EINVAL, "rs_diag_step: null argument");
  void* sp = s->sss ? s->spsi : s->psi;
  if (s->prec == 64)
    return rs_scf_diag_f64(s->g, (const double*)s->veff, s->dij, s->sss, prm, iscf, s->M,
                           (double*)s->psi, (double*)sp, s->rp, (double*)s->hpsi, sval, resid,
                           ksconv, ksitmax, s->st);
  return rs_scf_diag_f32(s->g, (const float*)s->veff, s->dij, s->sss, prm, iscf, s->M,
                         (float*)s->psi, (float*)sp, s->rp, (float*)s->hpsi, sval, resid,
                         ksconv, ksitmax, s->st);
}

// scf_charge_smt_r (scf_charge8f.F90:290-321): rho (host, N) from the
// occupations occ (host, M)
extern "C" int rs_density(rs_state* s, const double* occ, double* rho) {
  if (!s || !occ || !rho) return rs::fail(RS_EINVAL, "rs_density: null argument");
  double *docc = nullptr, *drho = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&docc, sizeof(double) * (s->M + s->N), s->st);
  int rc = RS_OK;
  if (e == cudaSuccess) {
    drho = docc + s->M;
    e = cudaMemcpyAsync(docc, occ, sizeof(double) * s->M, cudaMemcpyHostToDevice, s->st);
  }
  if (e == cudaSuccess) {
    rc = s->prec == 64
             ? rs_density_f64(s->N, s->M, docc, (const double*)s->psi, drho, s->st)
             : rs_density_f32(s->N, s->M, docc, (const float*)s->psi, drho, s->st);
    if (!rc) e = cudaMemcpyAsync(rho, drho, sizeof(double) * s->N, cudaMemcpyDeviceToHost, s->st);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
  if (docc) cudaFreeAsync(docc, s->st);
  if (rc) return rc;
  return e == cudaSuccess ? RS_OK : rs::cuda_status(e, "rs_density");
}
