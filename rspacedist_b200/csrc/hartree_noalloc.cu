// hartree_noalloc.cu -- the Hartree CG Poisson solve for callers that must
// not allocate device memory.
//
// Some callers cannot call cudaMalloc at solve time.  Examples: a Fortran
// code that carved all device memory into its own pool at start-up, a
// framework whose caching allocator owns the device, a solve issued from a
// path that must not take the driver's allocation lock.  For them this
// variant takes its work vectors from a fixed array compiled into the
// library instead of a stream-ordered allocation.  Every GPU that loads the
// library reserves the array (about 10.5 MB) until the process exits, so it is
// sized for dense grids of up to 64^3 points (the Hartree grid of a 32^3
// coarse cell with nmesh=2) and larger grids are rejected.
#include "reduce.cuh"
#include "rs_common.cuh"

namespace rs {
int hartree_cg(int nx, int ny, int nz, int nfh, double xmax, double ymax, double zmax,
               double epsvh, int ncgmin, int ncgmax, int ncgres, const double* rho, double* vh,
               double* work, int* iters, double* dp_out, cudaStream_t st, float* work32,
               bool allow_graph);
}

namespace {

constexpr long kNoAllocMaxPoints = 64L * 64L * 64L;
// b, r, p, A p, running A x (5 grid vectors), the chunk partial sums of the
// reduction tree, and the CG scalars
constexpr long kNoAllocWords = 5 * kNoAllocMaxPoints +
                               (kNoAllocMaxPoints + rs::kTreeChunk - 1) / rs::kTreeChunk + 1 +
                               16;
static __device__ __align__(256) double g_hartree_scratch[kNoAllocWords];

// Device address of the array in the current device's context.  Host code
// cannot use the symbol's name as a device address, so it is looked up on
// every call (a cheap query next to a CG solve); nothing is cached, which
// keeps the address right after a context is torn down and created again.
int scratch_address(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_hartree_scratch);
  if (e != cudaSuccess) return rs::cuda_status(e, "rs_hartree_cg_noalloc: cudaGetSymbolAddress");
  *out = static_cast<double*>(p);
  return RS_OK;
}

}  // namespace

// Same arguments and results as rs_hartree_cg.  No device memory is
// allocated or freed, and the iteration batches run as plain kernel launches
// on every stream (rs_hartree_cg instantiates a CUDA graph of them on a
// non-default stream, which this entry point never does).  Every word of the
// array is written before it is read within a call (the CG scalars are
// cleared at the start of each solve), so nothing needs clearing between
// calls; calls that overlap on the GPU (other streams, other host threads,
// same device) share the one array and race.
extern "C" int rs_hartree_cg_noalloc(int nx, int ny, int nz, int nfh, double xmax, double ymax,
                                     double zmax, double epsvh, int ncgmin, int ncgmax,
                                     int ncgres, const double* rho, double* vh, int* iters,
                                     double* dp, void* stream) {
  if (nfh < 1 || nfh > 6 || nx <= 2 * nfh || ny <= 2 * nfh || nz <= 2 * nfh)
    return rs::fail(RS_EINVAL, "rs_hartree_cg_noalloc: bad grid or nfh");
  if (ncgres <= 0 || ncgmax <= 0)
    return rs::fail(RS_EINVAL, "rs_hartree_cg_noalloc: bad iteration limits");
  const long N = (long)nx * ny * nz;
  if (N > kNoAllocMaxPoints)
    return rs::fail(RS_EINVAL,
                    "rs_hartree_cg_noalloc: grid exceeds the fixed work array (at most 262144 "
                    "points, e.g. 64^3); use rs_hartree_cg for larger grids");
  double* work = nullptr;
  int rc = scratch_address(&work);
  if (rc != RS_OK) return rc;
  // plain launches on every stream: no CUDA graph is captured or instantiated
  rc = rs::hartree_cg(nx, ny, nz, nfh, xmax, ymax, zmax, epsvh, ncgmin, ncgmax, ncgres, rho, vh,
                      work, iters, dp, rs::as_stream(stream), nullptr, false);
  // the same diagnostic as rs_hartree_cg when the iteration limit stops the solve
  if (rc == RS_OK && iters && *iters >= ncgmax && dp && *dp > epsvh)
    rs::set_error("rs_hartree_cg_noalloc: ncgmax reached");
  return rc;
}
