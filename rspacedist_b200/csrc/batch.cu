// batch.cu -- H psi (FP32 bands) for many independent small cells in one
// persistent launch: kslaplacian_r + nonlocaloperation_r_02 of every cell
// (kslaplacian8f.F90:23-261, nonlocaloperation8f.F90:149-235), as kukan
// would run them cell after cell, for sets of small periodic cells of uneven
// grids (tens of cells of 20-40 points per axis and ~20 bands each), where a
// launch per cell and kernel would leave most SMs idle.
//
//  * A plan (rs_hpsi_batch) holds a device table of the cells: geometry
//    lists, stencil coefficients, the caller's veff / D / <p|psi> / psi /
//    H psi pointers and the first work item of each cell.
//  * k_batch_tcoef forms the D <p|psi> / dV coefficients of all cells in one
//    launch; k_batch_hpsi is persistent: CTAs stride over work items (cell,
//    block of BPB bands, block of points) and evaluate each point as the
//    per-cell gather kernel does (the nonlocal sum over the point's
//    inverse-list entries, then the stencil and veff), so every cell's
//    result equals its single-cell fused H psi bit for bit.
//  * An autotuner times the candidate shapes (threads per CTA, bands per
//    work item, CTAs per SM) on the first run and keeps the fastest.
//  * A run can be captured once into a CUDA graph and replayed.
#include <math.h>

#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "rs_common.cuh"
#include "stencil.cuh"

namespace rs {
namespace batch {

struct BatchCell {
  StencilArgs<float> s;
  long N;
  int nb, natom, nprjmx, nblk_pts;
  double dxyzin;
  const int* inv_off;
  const int* inv_atom;
  const float* inv_v;
  const int* nprj;
  const float* veff;
  const double* dij;
  const double* rp;
  const float* psi;
  float* out;
  float* t;        // [nb][natom][nprjmx]
  long t_off;      // first t element of this cell in the batch-wide t list
  long item0;      // first work item of this cell
};

struct Shape {
  int tpb, bpb, per_sm;
};

}  // namespace batch

namespace {
using batch::BatchCell;
using batch::Shape;

__device__ __forceinline__ int find_cell(const BatchCell* __restrict__ cells, int ncell,
                                         long key, bool by_t) {
  int lo = 0, hi = ncell - 1;
  while (lo < hi) {  // last cell whose start is <= key
    const int mid = (lo + hi + 1) >> 1;
    const long start = by_t ? cells[mid].t_off : cells[mid].item0;
    if (start <= key) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// t[b][a][i] = (sum_j rp[b][a][j] D_a[i][j]) / dV for all cells (k_tcoef's sum)
__global__ void k_batch_tcoef(const BatchCell* __restrict__ cells, int ncell, long total) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= total) return;
  const BatchCell& C = cells[find_cell(cells, ncell, idx, true)];
  const long k = idx - C.t_off;
  const int P = C.nprjmx;
  const int i = (int)(k % P);
  const long ba = k / P;
  const int a = (int)(ba % C.natom);
  const int np = C.nprj[a];
  double s = 0.0;
  if (i < np) {
    const double* r = C.rp + ba * P;
    const double* m = C.dij + ((long)a * P + i) * P;
    for (int j = 0; j < np; ++j) s = fma(r[j], m[j], s);
    s = s * C.dxyzin;
  }
  C.t[k] = (float)s;
}

template <int BPB>
__global__ void k_batch_hpsi(const BatchCell* __restrict__ cells, int ncell, long nitems) {
  for (long it = blockIdx.x; it < nitems; it += gridDim.x) {
    const BatchCell& C = cells[find_cell(cells, ncell, it, false)];
    const long local = it - C.item0;
    const long p = (local % C.nblk_pts) * blockDim.x + threadIdx.x;
    const int b0 = (int)(local / C.nblk_pts) * BPB;
    if (p >= C.N) continue;
    const int nx = C.s.nx, ny = C.s.ny;
    const int ix = (int)(p % nx), iy = (int)((p / nx) % ny), iz = (int)(p / ((long)nx * ny));
    const int e0 = __ldg(C.inv_off + p), e1 = __ldg(C.inv_off + p + 1);
    const float vloc = __ldg(C.veff + p);
    const int b1 = min(b0 + BPB, C.nb);
    for (int b = b0; b < b1; ++b) {
      float acc = 0.f;
      for (int e = e0; e < e1; ++e) {
        const int a = __ldg(C.inv_atom + e);
        const int P = __ldg(C.nprj + a);
        if (P <= 0) continue;
        const float* tv = C.t + ((long)b * C.natom + a) * C.nprjmx;
        const float* pv = C.inv_v + (long)e * C.nprjmx;
        float avr = tv[0] * __ldg(pv);
        for (int j = 1; j < P; ++j) avr = fmaf(tv[j], __ldg(pv + j), avr);
        acc = acc + avr;
      }
      acc = stencil_point<float>(C.s, C.psi + (long)b * C.N, ix, iy, iz, vloc, acc);
      C.out[(long)b * C.N + p] = acc;
    }
  }
}

}  // namespace
}  // namespace rs

struct rs_hpsi_batch {
  int ncell = 0;
  std::vector<const rs_geom*> g;
  std::vector<int> nb;
  std::vector<rs::batch::BatchCell> host;
  rs::batch::BatchCell* dev = nullptr;
  float* t = nullptr;
  long total_t = 0;
  int nsm = 148;
  bool ready = false;  // pointers set
  bool tuned = false;
  rs::batch::Shape shape{128, 4, 4};
  long nitems = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaStream_t graph_stream = nullptr;
};

namespace rs {
namespace {

void drop_graph(rs_hpsi_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// item layout for a shape, uploaded with the cell table
int layout(rs_hpsi_batch* b, const Shape& sh) {
  long item = 0;
  for (int c = 0; c < b->ncell; ++c) {
    BatchCell& C = b->host[c];
    C.nblk_pts = (int)div_up(C.N, sh.tpb);
    C.item0 = item;
    item += (long)C.nblk_pts * div_up(C.nb, sh.bpb);
  }
  b->nitems = item;
  RS_CUDA(cudaMemcpy(b->dev, b->host.data(), sizeof(BatchCell) * b->ncell,
                     cudaMemcpyHostToDevice));
  return RS_OK;
}

int launch(rs_hpsi_batch* b, const Shape& sh, cudaStream_t st) {
  if (b->total_t > 0)
    k_batch_tcoef<<<div_up(b->total_t, 256), 256, 0, st>>>(b->dev, b->ncell, b->total_t);
  const unsigned grid = (unsigned)std::max(1L, std::min(b->nitems, (long)b->nsm * sh.per_sm));
  switch (sh.bpb) {
    case 1: k_batch_hpsi<1><<<grid, sh.tpb, 0, st>>>(b->dev, b->ncell, b->nitems); break;
    case 2: k_batch_hpsi<2><<<grid, sh.tpb, 0, st>>>(b->dev, b->ncell, b->nitems); break;
    case 4: k_batch_hpsi<4><<<grid, sh.tpb, 0, st>>>(b->dev, b->ncell, b->nitems); break;
    default: k_batch_hpsi<8><<<grid, sh.tpb, 0, st>>>(b->dev, b->ncell, b->nitems); break;
  }
  RS_LAUNCH_CHECK("k_batch_hpsi");
  return RS_OK;
}

// time every candidate shape twice (after one untimed run) and keep the fastest
int autotune(rs_hpsi_batch* b, cudaStream_t st) {
  const Shape cands[] = {{128, 2, 8}, {128, 4, 8}, {128, 8, 8}, {256, 2, 4},
                         {256, 4, 4}, {256, 8, 4}, {64, 4, 16}, {128, 1, 8}};
  cudaEvent_t e0, e1;
  RS_CUDA(cudaEventCreate(&e0));
  RS_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  Shape pick = cands[0];
  int rc = RS_OK;
  for (const Shape& sh : cands) {
    if ((rc = layout(b, sh)) || (rc = launch(b, sh, st))) break;
    cudaEventRecord(e0, st);
    for (int r = 0; r < 2 && !rc; ++r) rc = launch(b, sh, st);
    cudaEventRecord(e1, st);
    if (cudaEventSynchronize(e1) != cudaSuccess) { rc = cuda_status(cudaGetLastError(), "autotune"); break; }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) { best = ms; pick = sh; }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (rc) return rc;
  b->shape = pick;
  b->tuned = true;
  return layout(b, pick);
}

}  // namespace
}  // namespace rs

extern "C" int rs_hpsi_batch_create(rs_hpsi_batch** out, int ncell, const rs_geom* const* geoms,
                                    const int* nb) {
  if (!out || ncell <= 0 || !geoms || !nb)
    return rs::fail(RS_EINVAL, "rs_hpsi_batch_create: bad arguments");
  *out = nullptr;
  rs::keep_pool_memory();
  auto* b = new rs_hpsi_batch;
  b->ncell = ncell;
  b->g.assign(geoms, geoms + ncell);
  b->nb.assign(nb, nb + ncell);
  b->host.resize(ncell);
  long toff = 0;
  for (int c = 0; c < ncell; ++c) {
    const rs_geom* g = geoms[c];
    if (!g || nb[c] <= 0 || g->nf > 8) {
      delete b;
      return rs::fail(RS_EINVAL, "rs_hpsi_batch_create: bad cell " + std::to_string(c));
    }
    rs::batch::BatchCell& C = b->host[c];
    memset(&C, 0, sizeof(C));
    C.s = rs::make_stencil_args<float>(g);
    C.N = g->N;
    C.nb = nb[c];
    C.natom = g->natom;
    C.nprjmx = g->nprjmx;
    C.dxyzin = 1.0 / (g->dx * g->dy * g->dz);
    C.inv_off = g->d_inv_off;
    C.inv_atom = g->d_inv_atom;
    C.inv_v = g->d_inv_v32;
    C.nprj = g->d_nprj;
    C.t_off = toff;
    toff += (long)nb[c] * g->natom * g->nprjmx;
  }
  b->total_t = toff;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaMalloc((void**)&b->dev, sizeof(rs::batch::BatchCell) * ncell) != cudaSuccess ||
      (toff > 0 && cudaMalloc((void**)&b->t, sizeof(float) * toff) != cudaSuccess)) {
    cudaGetLastError();
    if (b->dev) cudaFree(b->dev);
    delete b;
    return rs::fail(RS_ECUDA, "rs_hpsi_batch_create: device allocation failed");
  }
  for (int c = 0; c < ncell; ++c) b->host[c].t = b->t + b->host[c].t_off;
  *out = b;
  return RS_OK;
}

extern "C" int rs_hpsi_batch_set_f32(rs_hpsi_batch* b, const float* const* veff,
                                     const double* const* dij, const double* const* rp,
                                     const float* const* psi, float* const* hpsi) {
  if (!b || !veff || !dij || !rp || !psi || !hpsi)
    return rs::fail(RS_EINVAL, "rs_hpsi_batch_set_f32: null argument");
  for (int c = 0; c < b->ncell; ++c) {
    rs::batch::BatchCell& C = b->host[c];
    if (!veff[c] || !psi[c] || !hpsi[c] || (C.natom > 0 && (!dij[c] || !rp[c])))
      return rs::fail(RS_EINVAL, "rs_hpsi_batch_set_f32: null pointer for cell " +
                                     std::to_string(c));
    C.veff = veff[c];
    C.dij = dij[c];
    C.rp = rp[c];
    C.psi = psi[c];
    C.out = hpsi[c];
  }
  rs::drop_graph(b);
  b->ready = true;
  // the table is rewritten in place: no run of the plan may still read it
  RS_CUDA(cudaDeviceSynchronize());
  return rs::layout(b, b->shape);
}

extern "C" int rs_hpsi_batch_run_f32(rs_hpsi_batch* b, int use_graph, void* stream) {
  if (!b || !b->ready) return rs::fail(RS_EINVAL, "rs_hpsi_batch_run_f32: pointers not set");
  cudaStream_t st = rs::as_stream(stream);
  int rc;
  if (!b->tuned && (rc = rs::autotune(b, st))) return rc;
  if (!use_graph || st == nullptr) return rs::launch(b, b->shape, st);
  if (b->exec && b->graph_stream != st) rs::drop_graph(b);
  if (!b->exec) {
    RS_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    rc = rs::launch(b, b->shape, st);
    cudaGraph_t gph = nullptr;
    cudaError_t e = cudaStreamEndCapture(st, &gph);
    if (rc) {
      if (gph) cudaGraphDestroy(gph);
      return rc;
    }
    if (e != cudaSuccess) return rs::cuda_status(e, "rs_hpsi_batch: graph capture");
    b->graph = gph;
    e = cudaGraphInstantiate(&b->exec, gph, 0);
    if (e != cudaSuccess) {
      rs::drop_graph(b);
      return rs::cuda_status(e, "rs_hpsi_batch: graph instantiate");
    }
    b->graph_stream = st;
  }
  RS_CUDA(cudaGraphLaunch(b->exec, st));
  return RS_OK;
}

extern "C" int rs_hpsi_batch_info(const rs_hpsi_batch* b, int* tpb, int* bpb, int* ctas_per_sm) {
  if (!b) return rs::fail(RS_EINVAL, "rs_hpsi_batch_info: null plan");
  if (tpb) *tpb = b->shape.tpb;
  if (bpb) *bpb = b->shape.bpb;
  if (ctas_per_sm) *ctas_per_sm = b->shape.per_sm;
  return b->tuned ? RS_OK : 1;
}

extern "C" int rs_hpsi_batch_set_shape(rs_hpsi_batch* b, int tpb, int bpb, int ctas_per_sm) {
  if (!b) return rs::fail(RS_EINVAL, "rs_hpsi_batch_set_shape: null plan");
  if (tpb != 64 && tpb != 128 && tpb != 256)
    return rs::fail(RS_EINVAL, "rs_hpsi_batch_set_shape: threads per CTA must be 64, 128 or 256");
  if (bpb != 1 && bpb != 2 && bpb != 4 && bpb != 8)
    return rs::fail(RS_EINVAL, "rs_hpsi_batch_set_shape: bands per item must be 1, 2, 4 or 8");
  if (ctas_per_sm < 1 || ctas_per_sm > 16)
    return rs::fail(RS_EINVAL, "rs_hpsi_batch_set_shape: CTAs per SM must be 1..16");
  rs::drop_graph(b);
  b->shape = rs::batch::Shape{tpb, bpb, ctas_per_sm};
  b->tuned = true;
  RS_CUDA(cudaDeviceSynchronize());  // the table is rewritten in place
  return rs::layout(b, b->shape);
}

extern "C" int rs_hpsi_batch_destroy(rs_hpsi_batch* b) {
  if (!b) return RS_OK;
  rs::drop_graph(b);
  if (b->t) cudaFree(b->t);
  if (b->dev) cudaFree(b->dev);
  delete b;
  return RS_OK;
}
