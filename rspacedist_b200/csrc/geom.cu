// geom.cu -- host side of the C-ABI: status/error plumbing, the sphere-list
// builder (pseudocalc_01b) and the device-resident geometry object.
#include <math.h>
#include <string.h>

#include <mutex>
#include <string>
#include <vector>

#include "rs_common.cuh"

namespace rs {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }

// The H*psi, band and subspace kernels take their per-call work arrays (up to
// tens of GB for a thousand bands) from the device's default stream-ordered
// pool.  Let the pool keep freed memory instead of unmapping it at every
// synchronisation, so repeated calls reuse it (as a caching allocator does).
void keep_pool_memory() {
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess &&
      cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  cudaGetLastError();
}

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_status(cudaError_t e, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? RS_ENOMEM : RS_ECUDA;
}

// tools_definefdcoef (tools8f.F90:144-237), exact rationals for nf <= 6
void fd_coefs(int nf, double a[9]) {
  for (int i = 0; i < 9; ++i) a[i] = 0.0;
  if (nf == 1) { a[0] = -2.0; a[1] = 1.0; }
  if (nf == 2) { a[0] = -5.0 / 2.0; a[1] = 4.0 / 3.0; a[2] = -1.0 / 12.0; }
  if (nf == 3) { a[0] = -49.0 / 18.0; a[1] = 3.0 / 2.0; a[2] = -3.0 / 20.0; a[3] = 1.0 / 90.0; }
  if (nf == 4) {
    a[0] = -205.0 / 72.0; a[1] = 8.0 / 5.0; a[2] = -1.0 / 5.0;
    a[3] = 8.0 / 315.0; a[4] = -1.0 / 560.0;
  }
  if (nf == 5) {
    a[0] = -36883.0 / 12600.0; a[1] = 5.0 / 3.0; a[2] = -5.0 / 21.0;
    a[3] = 5.0 / 126.0; a[4] = -5.0 / 1008.0; a[5] = 1.0 / 3150.0;
  }
  if (nf == 6) {
    a[0] = -5369.0 / 1800.0; a[1] = 12.0 / 7.0; a[2] = -15.0 / 56.0; a[3] = 10.0 / 189.0;
    a[4] = -1.0 / 112.0; a[5] = 2.0 / 1925.0; a[6] = -1.0 / 16632.0;
  }
}

}  // namespace rs

extern "C" int rs_last_error(char* buf, int len) {
  if (!buf || len <= 0) return RS_EINVAL;
  strncpy(buf, rs::g_last_error.c_str(), (size_t)len - 1);
  buf[len - 1] = 0;
  return RS_OK;
}

extern "C" const char* rs_version(void) { return "rspace_b200 0.1 sm_100a"; }

// Sphere lists for one rank and nperi=3 (pseudocalc8f.F90:691-693, 955-1033).
// A box point (ix,iy,iz) enters the list when some point of its
// (2nfdg+1)^3 neighbourhood lies within rcut.  The distance expression is
// monotone in each |coordinate|, so that test equals the test at the
// per-axis nearest neighbourhood point; this routine evaluates only that
// point, with the reference's arithmetic.
extern "C" int rs_sphere_lists(int natom, const double* atx, const double* aty,
                               const double* atz, const double* rcut, int nxmax, int nymax,
                               int nzmax, double dx, double dy, double dz, int npxmax,
                               int npymax, int npzmax, int nfdg, int num_list, int* natx,
                               int* naty, int* natz, int* natinf, int* lst, int* lstx,
                               int* lsty, int* lstz) {
  if (natom < 0 || nxmax <= 0 || nymax <= 0 || nzmax <= 0 || num_list <= 0 || nfdg < 0)
    return rs::fail(RS_EINVAL, "rs_sphere_lists: bad dimensions");
  const double xmax = nxmax * dx, ymax = nymax * dy, zmax = nzmax * dz;
  const int ncpx = 2 * nxmax, ncpy = 2 * nymax;
  int status = RS_OK;
  std::vector<double> sx, sy, sz;
  for (int a = 0; a < natom; ++a) {
    natx[a] = (int)((atx[a] + xmax + 0.5 * dx) / dx) - nxmax;
    naty[a] = (int)((aty[a] + ymax + 0.5 * dy) / dy) - nymax;
    natz[a] = (int)((atz[a] + zmax + 0.5 * dz) / dz) - nzmax;
    const double tx = atx[a] - (natx[a] * dx - 0.5 * dx);
    const double ty = aty[a] - (naty[a] * dy - 0.5 * dy);
    const double tz = atz[a] - (natz[a] * dz - 0.5 * dz);
    // nearest squared coordinate over the neighbourhood, per box index
    auto nearest = [&](int np, double h, double t, std::vector<double>& out) {
      out.assign(2 * np, 0.0);
      for (int i = -np + 1; i <= np; ++i) {
        double best = INFINITY;
        for (int j = -nfdg; j <= nfdg; ++j) {
          const double c = (i + j) * h - t;
          const double c2 = c * c;
          if (c2 < best) best = c2;
        }
        out[i + np - 1] = best;
      }
    };
    nearest(npxmax, dx, tx, sx);
    nearest(npymax, dy, ty, sy);
    nearest(npzmax, dz, tz, sz);
    int l0 = 0;
    for (int iz = -npzmax + 1; iz <= npzmax; ++iz)
      for (int iy = -npymax + 1; iy <= npymax; ++iy)
        for (int ix = -npxmax + 1; ix <= npxmax; ++ix) {
          const double r =
              sqrt(sx[ix + npxmax - 1] + sy[iy + npymax - 1] + sz[iz + npzmax - 1]);
          if (!(r < rcut[a])) continue;
          int i = ix + natx[a] + nxmax, j = iy + naty[a] + nymax, k = iz + natz[a] + nzmax;
          i = (int)rs::wrapi(i - 1, 2 * nxmax) + 1;
          j = (int)rs::wrapi(j - 1, 2 * nymax) + 1;
          k = (int)rs::wrapi(k - 1, 2 * nzmax) + 1;
          if (l0 >= num_list) {
            status = RS_EINVAL;
            continue;
          }
          const long o = (long)a * num_list + l0;
          lst[o] = ((k - 1) * ncpy + (j - 1)) * ncpx + (i - 1);
          if (lstx) lstx[o] = ix;
          if (lsty) lsty[o] = iy;
          if (lstz) lstz[o] = iz;
          ++l0;
        }
    natinf[a] = l0;
  }
  if (status != RS_OK) return rs::fail(status, "rs_sphere_lists: num_list is too small");
  return RS_OK;
}

template <class T>
static int upload(T** dst, const T* src, size_t n) {
  *dst = nullptr;
  if (n == 0) return RS_OK;
  RS_CUDA(cudaMalloc((void**)dst, n * sizeof(T)));
  RS_CUDA(cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice));
  return RS_OK;
}

extern "C" int rs_geom_destroy(rs_geom* g) {
  if (!g) return RS_OK;
  void* ptrs[] = {g->d_nprj, g->d_natinf, g->d_lst, g->d_vT64, g->d_vT32, g->d_inv_off,
                  g->d_inv_atom, g->d_inv_v64, g->d_inv_v32, g->d_cov,
                  g->d_cov_off, g->d_nz_off, g->d_nz_pt, g->d_nz_v32, g->d_nz_v64};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (g->host_buf) cudaFree(g->host_buf);
  for (int i = 0; i < 2; ++i) {
    if (g->host_cs[i]) cudaStreamDestroy(g->host_cs[i]);
    if (g->host_ev_done[i]) cudaEventDestroy(g->host_ev_done[i]);
  }
  if (g->host_ev_start) cudaEventDestroy(g->host_ev_start);
  if (g->nl_cs) cudaStreamDestroy(g->nl_cs);
  if (g->nl_ev_in) cudaEventDestroy(g->nl_ev_in);
  if (g->nl_ev_out) cudaEventDestroy(g->nl_ev_out);
  if (g->st_err_h) cudaFreeHost(g->st_err_h);
  delete g;
  return RS_OK;
}

extern "C" long rs_geom_entries(const rs_geom* g) { return g ? g->n_inv : -1; }

extern "C" int rs_geom_create(rs_geom** out, int nx, int ny, int nz, int nf, double dx,
                              double dy, double dz, int natom, int nprjmx, int num_list,
                              const int* nprj, const int* natinf, const int* lst,
                              const double* vnlocp) {
  if (!out) return rs::fail(RS_EINVAL, "rs_geom_create: null handle");
  *out = nullptr;
  if (nx <= 0 || ny <= 0 || nz <= 0) return rs::fail(RS_EINVAL, "rs_geom_create: bad grid");
  if (nf < 1 || nf > 6) return rs::fail(RS_EINVAL, "rs_geom_create: nf must be 1..6");
  if (natom < 0 || (natom > 0 && (nprjmx <= 0 || num_list <= 0)))
    return rs::fail(RS_EINVAL, "rs_geom_create: bad atom dimensions");
  if (2 * nf >= nx || 2 * nf >= ny || 2 * nf >= nz)
    return rs::fail(RS_EINVAL, "rs_geom_create: grid smaller than the stencil");
  const long N = (long)nx * ny * nz;
  if (N > (1L << 31) - 1) return rs::fail(RS_EINVAL, "rs_geom_create: grid too large");
  rs::keep_pool_memory();
  rs_geom* g = new rs_geom;
  memset(g, 0, sizeof(*g));
  g->nx = nx; g->ny = ny; g->nz = nz; g->nf = nf;
  g->dx = dx; g->dy = dy; g->dz = dz;
  g->N = N;
  g->natom = natom; g->nprjmx = nprjmx; g->num_list = num_list;
  double a[9];
  rs::fd_coefs(nf, a);
  for (int m = 0; m < 9; ++m) {
    g->cx[m] = a[m] / dx / dx * (-0.5);
    g->cy[m] = a[m] / dy / dy * (-0.5);
    g->cz[m] = a[m] / dz / dz * (-0.5);
  }
  int st = RS_OK;
  g->max_prj = 0;
  for (int i = 0; i < natom; ++i) {
    if (nprj[i] < 0 || nprj[i] > nprjmx || natinf[i] < 0 || natinf[i] > num_list) {
      rs_geom_destroy(g);
      return rs::fail(RS_EINVAL, "rs_geom_create: nprj/natinf out of range");
    }
    if (nprj[i] > g->max_prj) g->max_prj = nprj[i];
  }
  // inverse lists: entries of a point sorted by (atom, ii) -- the order in
  // which nonlocaloperation_r_02 scatters them.  An entry whose projector
  // values are all exactly zero adds exactly zero there and is left out.
  auto zero_entry = [&](int i, int ii) {
    for (int j = 0; j < nprj[i]; ++j)
      if (vnlocp[((long)i * nprjmx + j) * num_list + ii] != 0.0) return false;
    return true;
  };
  std::vector<int> off(N + 1, 0);
  long ne = 0;
  for (int i = 0; i < natom; ++i)
    for (int ii = 0; ii < natinf[i]; ++ii) {
      const int p = lst[(long)i * num_list + ii];
      if (p < 0 || p >= N) {
        rs_geom_destroy(g);
        return rs::fail(RS_EINVAL, "rs_geom_create: list entry outside the grid");
      }
      if (zero_entry(i, ii)) continue;
      off[p + 1]++;
      ++ne;
    }
  for (long p = 0; p < N; ++p) off[p + 1] += off[p];
  int maxinv = 0;
  for (long p = 0; p < N; ++p) maxinv = std::max(maxinv, off[p + 1] - off[p]);
  g->max_inv = maxinv;
  g->n_inv = ne;
  std::vector<int> cov;
  for (long p = 0; p < N; ++p)
    if (off[p + 1] > off[p]) cov.push_back((int)p);
  g->n_cov = (long)cov.size();
  std::vector<int> fillp(off.begin(), off.end() - 1);
  std::vector<int> inv_atom(ne > 0 ? ne : 1);
  std::vector<double> inv_v(ne > 0 ? (size_t)ne * nprjmx : 1, 0.0);
  std::vector<double> vT((size_t)natom * num_list * nprjmx + 1, 0.0);
  std::vector<float> vT32(vT.size()), inv_v32(inv_v.size());
  for (int i = 0; i < natom; ++i)
    for (int ii = 0; ii < natinf[i]; ++ii) {
      const int p = lst[(long)i * num_list + ii];
      for (int j = 0; j < nprjmx; ++j) {
        const double val = j < nprj[i] ? vnlocp[((long)i * nprjmx + j) * num_list + ii] : 0.0;
        vT[((size_t)i * num_list + ii) * nprjmx + j] = val;
      }
      if (zero_entry(i, ii)) continue;
      const int e = fillp[p]++;
      inv_atom[e] = i;
      for (int j = 0; j < nprjmx; ++j)
        inv_v[(size_t)e * nprjmx + j] = vT[((size_t)i * num_list + ii) * nprjmx + j];
    }
  for (size_t i = 0; i < vT.size(); ++i) vT32[i] = (float)vT[i];
  for (size_t i = 0; i < inv_v.size(); ++i) inv_v32[i] = (float)inv_v[i];
  std::vector<int> cov_off(cov.size() + 1, 0);
  for (size_t c = 0; c < cov.size(); ++c) {
    cov_off[c] = off[cov[c]];
    cov_off[c + 1] = off[cov[c] + 1];
  }
  // atom-major compact lists (skipping all-zero list positions leaves every
  // fma chain of the gather-dot unchanged: the skipped terms add zero)
  std::vector<int> nz_off(natom + 1, 0), nz_pt;
  std::vector<double> nz_v;
  for (int i = 0; i < natom; ++i) {
    for (int ii = 0; ii < natinf[i]; ++ii) {
      if (zero_entry(i, ii)) continue;
      nz_pt.push_back(lst[(long)i * num_list + ii]);
      for (int j = 0; j < nprjmx; ++j) nz_v.push_back(vT[((size_t)i * num_list + ii) * nprjmx + j]);
    }
    nz_off[i + 1] = (int)nz_pt.size();
  }
  if (nz_pt.empty()) {
    nz_pt.push_back(0);
    nz_v.assign(nprjmx > 0 ? nprjmx : 1, 0.0);
  }
  std::vector<float> nz_v32(nz_v.begin(), nz_v.end());
  if ((st = upload(&g->d_inv_off, off.data(), off.size())) ||
      (natom > 0 && (st = upload(&g->d_nprj, nprj, natom))) ||
      (natom > 0 && (st = upload(&g->d_natinf, natinf, natom))) ||
      (natom > 0 && (st = upload(&g->d_lst, lst, (size_t)natom * num_list))) ||
      (st = upload(&g->d_vT64, vT.data(), vT.size())) ||
      (st = upload(&g->d_vT32, vT32.data(), vT32.size())) ||
      (st = upload(&g->d_inv_atom, inv_atom.data(), inv_atom.size())) ||
      (st = upload(&g->d_inv_v64, inv_v.data(), inv_v.size())) ||
      (st = upload(&g->d_inv_v32, inv_v32.data(), inv_v32.size())) ||
      (st = upload(&g->d_cov, cov.data(), cov.size())) ||
      (st = upload(&g->d_cov_off, cov_off.data(), cov_off.size())) ||
      (st = upload(&g->d_nz_off, nz_off.data(), nz_off.size())) ||
      (st = upload(&g->d_nz_pt, nz_pt.data(), nz_pt.size())) ||
      (st = upload(&g->d_nz_v32, nz_v32.data(), nz_v32.size())) ||
      (st = upload(&g->d_nz_v64, nz_v.data(), nz_v.size()))) {
    rs_geom_destroy(g);
    return st;
  }
  *out = g;
  return RS_OK;
}
