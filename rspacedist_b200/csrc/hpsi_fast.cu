// hpsi_fast.cu -- FP32 fused H*psi used by the mixed-precision path.
#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {
template <class T, int MODE>
int launch_gather(const rs_geom* g, const double* mat, const double* rp, const T* psi,
                  const T* veff, T* out, int nb, cudaStream_t st);

int launch_hpsi_f32_fast(const rs_geom* g, const float* veff, const double* dij,
                         const double* rp, const float* psi, float* hpsi, int nb,
                         cudaStream_t st) {
  return launch_gather<float, 1>(g, dij, rp, psi, veff, hpsi, nb, st);
}
}  // namespace rs
