// hpsi.cu -- mixed-precision (FP32 psi) H*psi entry points and the
// host-buffer variant that streams band chunks through the device.
#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {
template <class T, int MODE>
int launch_gather(const rs_geom* g, const double* mat, const double* rp, const T* psi,
                  const T* veff, T* out, int nb, cudaStream_t st);
int launch_hpsi_f32_fast(const rs_geom* g, const float* veff, const double* dij,
                         const double* rp, const float* psi, float* hpsi, int nb,
                         cudaStream_t st, bool local_only = false);
int hpsi_f32_nl_chunk(const rs_geom* g);
int hpsi_f32_staging(rs_geom* g, int mode, int nb, int* tma);
}  // namespace rs

extern "C" int rs_hpsi_f32_tuning(const rs_geom* g, int* nl_chunk, int* nl_bands) {
  if (!g || !nl_chunk || !nl_bands) return rs::fail(RS_EINVAL, "rs_hpsi_f32_tuning: null argument");
  const int code = rs::hpsi_f32_nl_chunk(g);
  *nl_chunk = code > 0 ? code / 64 : (code < 0 ? -1 : 0);
  *nl_bands = code > 0 ? code % 64 : (code < 0 ? -code : 0);
  return RS_OK;
}

extern "C" int rs_hpsi_f32_staging(rs_geom* g, int mode, int nb, int* tma) {
  if (!g || !tma) return rs::fail(RS_EINVAL, "rs_hpsi_f32_staging: null argument");
  return rs::hpsi_f32_staging(g, mode, nb, tma);
}

extern "C" int rs_hpsi_f32(const rs_geom* g, const float* veff, const double* dij,
                           const double* rp, const float* psi, float* hpsi, int nb,
                           void* stream) {
  if (!g) return rs::fail(RS_EINVAL, "rs_hpsi_f32: null geometry");
  return rs::launch_hpsi_f32_fast(g, veff, dij, rp, psi, hpsi, nb, rs::as_stream(stream));
}

// Host buffers in and out.  Band chunks alternate between two device
// buffers so that the upload of chunk k+1 and the download of chunk k-1
// overlap the H*psi of chunk k (copy engines vs SMs).  Host arrays should be
// pinned for the copies to run asynchronously.  The two copy streams, their
// events and the chunk buffers belong to the geometry: the first call
// creates them (and a later call with a larger chunk grows the buffers), so
// repeated calls allocate nothing.  Not reentrant per geometry.
extern "C" int rs_hpsi_host_f32(const rs_geom* gc, const float* veff_dev, const double* dij_dev,
                                const double* rp_dev, const float* psi_host, float* hpsi_host,
                                int nb, int chunk, void* stream) {
  if (!gc) return rs::fail(RS_EINVAL, "rs_hpsi_host_f32: null geometry");
  if (nb <= 0) return RS_OK;
  if (chunk <= 0) chunk = 64;
  if (chunk > nb) chunk = nb;
  rs_geom* g = const_cast<rs_geom*>(gc);
  cudaStream_t st = rs::as_stream(stream);
  const long N = g->N;
  const size_t cb = sizeof(float) * (size_t)N * chunk;
  if (!g->host_ev_start) {
    RS_CUDA(cudaEventCreateWithFlags(&g->host_ev_start, cudaEventDisableTiming));
    for (int i = 0; i < 2; ++i) {
      RS_CUDA(cudaStreamCreateWithFlags(&g->host_cs[i], cudaStreamNonBlocking));
      RS_CUDA(cudaEventCreateWithFlags(&g->host_ev_done[i], cudaEventDisableTiming));
    }
  }
  if (g->host_buf_bytes < 4 * cb) {
    // the old buffers may still be read by an earlier call's copies
    RS_CUDA(cudaDeviceSynchronize());
    if (g->host_buf) cudaFree(g->host_buf);
    g->host_buf = nullptr;
    g->host_buf_bytes = 0;
    RS_CUDA(cudaMalloc((void**)&g->host_buf, 4 * cb));
    g->host_buf_bytes = 4 * cb;
  }
  float* buf = g->host_buf;
  float* din[2] = {buf, buf + (size_t)N * chunk};
  float* dout[2] = {buf + 2 * (size_t)N * chunk, buf + 3 * (size_t)N * chunk};
  cudaStream_t* cs = g->host_cs;
  // the copy streams start after the work already queued on the caller's stream
  RS_CUDA(cudaEventRecord(g->host_ev_start, st));
  for (int i = 0; i < 2; ++i) RS_CUDA(cudaStreamWaitEvent(cs[i], g->host_ev_start, 0));
  int rc = RS_OK;
  int k = 0;
  for (int b0 = 0; b0 < nb && rc == RS_OK; b0 += chunk, ++k) {
    const int s = k & 1;
    const int n = (b0 + chunk <= nb) ? chunk : nb - b0;
    // the buffers of slot s are free once chunk k-2 has been downloaded (the
    // same stream orders them)
    cudaError_t e = cudaMemcpyAsync(din[s], psi_host + (size_t)b0 * N,
                                    sizeof(float) * (size_t)N * n, cudaMemcpyHostToDevice, cs[s]);
    if (e != cudaSuccess) { rc = rs::cuda_status(e, "rs_hpsi_host_f32: upload"); break; }
    // rp of this chunk starts at band b0
    rc = rs::launch_hpsi_f32_fast(g, veff_dev, dij_dev,
                                  rp_dev + (size_t)b0 * g->natom * g->nprjmx, din[s], dout[s],
                                  n, cs[s]);
    if (rc != RS_OK) break;
    e = cudaMemcpyAsync(hpsi_host + (size_t)b0 * N, dout[s], sizeof(float) * (size_t)N * n,
                        cudaMemcpyDeviceToHost, cs[s]);
    if (e != cudaSuccess) { rc = rs::cuda_status(e, "rs_hpsi_host_f32: download"); break; }
  }
  // the caller's stream waits for both copy streams (also after an error, so
  // that nothing of this call is left running when it returns)
  for (int i = 0; i < 2; ++i) {
    cudaEventRecord(g->host_ev_done[i], cs[i]);
    cudaStreamWaitEvent(st, g->host_ev_done[i], 0);
  }
  const cudaError_t e = cudaStreamSynchronize(st);
  if (rc != RS_OK) return rc;
  if (e != cudaSuccess) return rs::cuda_status(e, "rs_hpsi_host_f32");
  return RS_OK;
}
