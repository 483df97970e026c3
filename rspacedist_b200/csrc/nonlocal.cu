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
// Thread (j, band) of block (atom, band group).  For T=double the chain is
// the reference's; for T=float the products and the sum are FP64.
template <class T>
__global__ void k_nl_dot(int natom, int nprjmx, int num_list, const int* __restrict__ nprj,
                         const int* __restrict__ natinf, const int* __restrict__ lst,
                         const T* __restrict__ vT, const T* __restrict__ psi, long N, int nb,
                         double* __restrict__ rp) {
  const int a = blockIdx.x;
  const int bpb = blockDim.x / nprjmx;
  const int j = threadIdx.x % nprjmx, bl = threadIdx.x / nprjmx;
  const int b = blockIdx.y * bpb + bl;
  if (bl >= bpb || b >= nb) return;
  double acc = 0.0;
  if (j < nprj[a]) {
    const int L = natinf[a];
    const int* l = lst + (long)a * num_list;
    const T* v = vT + (long)a * num_list * nprjmx + j;
    const T* x = psi + (long)b * N;
    for (int ii = 0; ii < L; ++ii)
      acc = fma((double)__ldg(v + (long)ii * nprjmx), (double)__ldg(x + __ldg(l + ii)), acc);
  }
  rp[((long)b * natom + a) * nprjmx + j] = acc;
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
  const int bpb = P > 128 ? 1 : 128 / P;
  const int threads = bpb * P;
  dim3 grid(g->natom, div_up(nb, bpb));
  const T* vT;
  if constexpr (sizeof(T) == 8) vT = (const T*)g->d_vT64; else vT = (const T*)g->d_vT32;
  k_nl_dot<T><<<grid, threads, 0, st>>>(g->natom, P, g->num_list, g->d_nprj, g->d_natinf,
                                        g->d_lst, vT, psi, g->N, nb, rp);
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

template <class T, int MODE>
int launch_gather(const rs_geom* g, const double* mat, const double* rp, const T* psi,
                  const T* veff, T* out, int nb, cudaStream_t st) {
  if (nb <= 0) return RS_OK;
  T* t = nullptr;
  int rc = make_tcoef<T>(g, mat, rp, nb, &t, st);
  if (rc) return rc;
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
extern "C" int rs_spsi_f32(const rs_geom* g, const double* sss, const double* rp,
                           const float* psi, float* spsi, int nb, void* stream) {
  RS_NEED_G("rs_spsi_f32");
  return rs::launch_gather<float, 2>(g, sss, rp, psi, nullptr, spsi, nb, rs::as_stream(stream));
}
