// rs_common.cuh -- shared definitions of the B200 kernels behind the
// rspace_b200 C-ABI: status handling, the device-resident geometry (grid,
// sphere lists, projector tables, inverse lists) and small device helpers.
//
// Every FP64 kernel states its floating-point evaluation order explicitly:
// the library is compiled with --fmad=false and each fused multiply-add is an
// explicit fma(), so results reproduce the strict CPU restatement of kukan's
// loops bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/rspace_b200.h"

namespace rs {

// thread-local message for rs_last_error()
void set_error(const std::string& msg);
// sets the default memory pool of the current device to keep freed memory
void keep_pool_memory();
int fail(int code, const std::string& msg);
int cuda_status(cudaError_t e, const char* what);

#define RS_CUDA(call)                                          \
  do {                                                         \
    cudaError_t e__ = (call);                                  \
    if (e__ != cudaSuccess) return rs::cuda_status(e__, #call); \
  } while (0)

#define RS_LAUNCH_CHECK(what)                                      \
  do {                                                             \
    cudaError_t e__ = cudaGetLastError();                          \
    if (e__ != cudaSuccess) return rs::cuda_status(e__, what);     \
  } while (0)

}  // namespace rs

// Device-resident geometry: everything H*psi needs that does not change
// during an SCF iteration.  Layouts follow kukan's arrays (x fastest).
struct rs_geom {
  int nx, ny, nz, nf;
  double dx, dy, dz;
  long N;
  int natom, nprjmx, num_list;
  int max_prj;
  // atom-major sphere data (nonlocaloperation_*_01 side)
  int* d_nprj;      // [natom]
  int* d_natinf;    // [natom]
  int* d_lst;       // [natom*num_list] 0-based point index
  double* d_vT64;   // [(a*num_list+ii)*nprjmx + j]
  float* d_vT32;
  // point-major inverse lists (nonlocaloperation_*_02 scatter as a gather):
  // entries of point p are [inv_off[p], inv_off[p+1]) sorted by (atom, ii)
  long n_inv;
  int* d_inv_off;   // [N+1]
  int* d_inv_atom;  // [n_inv]
  double* d_inv_v64;  // [n_inv*nprjmx]
  float* d_inv_v32;
  int max_inv;      // longest inverse list
  // points with at least one entry (the projector support), ascending
  long n_cov;
  int* d_cov;       // [n_cov] point index
  int* d_cov_off;   // [n_cov+1] entry range of covered point c (== inv_off[cov[c]])
  // atom-major compact lists: the nonzero entries of each atom's sphere
  // (list positions whose projector values are not all zero), in list order
  int* d_nz_off;    // [natom+1]
  int* d_nz_pt;     // [nnz] grid point
  float* d_nz_v32;  // [nnz*nprjmx]
  double* d_nz_v64; // [nnz*nprjmx]
  // Laplacian coefficients, computed as acfd(m)/dx/dx*(-0.5d0)
  double cx[9], cy[9], cz[9];
  // staging of the host-buffer H psi (rs_hpsi_host_f32): two copy streams,
  // their completion events and one event on the caller's stream, created by
  // the first call; the device chunk buffers, grown on demand.  Released by
  // rs_geom_destroy.
  cudaStream_t host_cs[2];
  cudaEvent_t host_ev_done[2];
  cudaEvent_t host_ev_start;
  float* host_buf;
  size_t host_buf_bytes;
  // FP32 H psi: the nonlocal pass runs on nl_cs band chunk by band chunk
  // behind the stencil (nl_ev_in after a stencil chunk, nl_ev_out at its
  // end).  nl_chunk codes the chosen shape, 0 until the first large call has
  // timed the candidates: chunk * 64 + bands per nonlocal thread, or minus
  // the bands per thread for one stencil launch followed by one pass.
  cudaStream_t nl_cs;
  cudaEvent_t nl_ev_in, nl_ev_out;
  int nl_chunk;
  // FP32 stencil staging: 0 = tensor-map (TMA) loads where the grid allows
  // them, 1 = per-thread cp.async; st_err_h/_d: host-mapped flag that a
  // bounded wait of the TMA form raises (allocated by its first launch)
  int st_copy;
  int* st_err_h;
  int* st_err_d;
};

namespace rs {

__host__ __device__ inline long wrapi(long i, long n) {
  i %= n;
  return i < 0 ? i + n : i;
}

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

inline unsigned div_up(long a, long b) { return (unsigned)((a + b - 1) / b); }

// V consecutive values of T moved as one aligned vector access
template <class T, int V>
struct alignas(sizeof(T) * V) Pack {
  T v[V];
};
template <class T, int V>
__device__ __forceinline__ Pack<T, V> ldpk(const T* p) {
  return *reinterpret_cast<const Pack<T, V>*>(p);
}
template <class T, int V>
__device__ __forceinline__ void stpk(T* p, const Pack<T, V>& x) {
  *reinterpret_cast<Pack<T, V>*>(p) = x;
}

void fd_coefs(int nf, double a[9]);

}  // namespace rs
