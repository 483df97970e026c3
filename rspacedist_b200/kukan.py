"""Python mirror of kukan's hot-path subroutines, running on the B200 library.

Each function carries the name of the kukan subroutine it replaces and the
same argument meaning; arrays are torch CUDA tensors in kukan's layouts
(x-fastest grids, band-major band arrays, rspsep-layout <p|psi>).  The calls
go through the C ABI (rspacedist_b200.lib); torch provides device memory and
the current CUDA stream.  Errors raise ``RsError`` with the library's
message, the counterpart of kukan's ``stopp``.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import lib as L
from .system import Cell


def _ptr(t):
    return C.c_void_p(0 if t is None else t.data_ptr())


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _need(t, dtype, n=None, what="array"):
    if not (t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise L.RsError(f"{what}: expected a contiguous CUDA {dtype} tensor")
    if n is not None and t.numel() != n:
        raise L.RsError(f"{what}: expected {n} elements, got {t.numel()}")


class Geometry:
    """Device-resident grid + sphere lists + projector tables (rs_geom)."""

    def __init__(self, cell: Cell, nf: int = 4):
        L.load()
        self.cell = cell
        self.nf = nf
        h = C.c_void_p()
        ip = lambda a: np.ascontiguousarray(a, np.int32).ctypes.data_as(C.POINTER(C.c_int))
        self._keep = [np.ascontiguousarray(cell.nprj, np.int32),
                      np.ascontiguousarray(cell.natinf, np.int32),
                      np.ascontiguousarray(cell.lst, np.int32),
                      np.ascontiguousarray(cell.vnlocp, np.float64)]
        nprj, natinf, lst, v = self._keep
        L.call("rs_geom_create", C.byref(h), cell.shape[0], cell.shape[1], cell.shape[2], nf,
               cell.h[0], cell.h[1], cell.h[2], cell.natom, cell.nprjmx, cell.num_list,
               nprj.ctypes.data_as(C.POINTER(C.c_int)),
               natinf.ctypes.data_as(C.POINTER(C.c_int)),
               lst.ctypes.data_as(C.POINTER(C.c_int)),
               v.ctypes.data_as(C.POINTER(C.c_double)))
        self.handle = h
        self.N = cell.N
        self.natom = cell.natom
        self.nprjmx = cell.nprjmx

    @property
    def entries(self) -> int:
        return int(L.load().rs_geom_entries(self.handle))

    def close(self):
        if getattr(self, "handle", None) is not None and self.handle.value:
            L.load().rs_geom_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _nb(g: Geometry, psi):
    if psi.numel() % g.N:
        raise L.RsError("band array size is not a multiple of the grid size")
    return psi.numel() // g.N


def kslaplacian(g: Geometry, psi, veff, out):
    """out += (-1/2 lap + veff) psi  (kslaplacian_r)."""
    nb = _nb(g, psi)
    fn = "rs_kslaplacian_f64" if psi.dtype == torch.float64 else "rs_kslaplacian_f32"
    _need(veff, psi.dtype, g.N, "veff")
    _need(out, psi.dtype, psi.numel(), "out")
    L.call(fn, g.handle, _ptr(psi), _ptr(veff), _ptr(out), nb, _stream())
    return out


def nonlocaloperation_01(g: Geometry, psi):
    """<p|psi> for every band (nonlocaloperation_r_01), FP64 result."""
    nb = _nb(g, psi)
    rp = torch.empty((nb, g.natom, g.nprjmx), dtype=torch.float64, device=psi.device)
    fn = "rs_nonlocal_dot_f64" if psi.dtype == torch.float64 else "rs_nonlocal_dot_f32"
    L.call(fn, g.handle, _ptr(psi), nb, _ptr(rp), _stream())
    return rp


def nonlocaloperation_02(g: Geometry, mat, rp, out):
    """out += sum_a p_a (mat_a rp_a)/dV  (nonlocaloperation_r_02), FP64."""
    nb = _nb(g, out)
    _need(out, torch.float64, what="out")
    L.call("rs_nonlocal_apply_f64", g.handle, _ptr(mat), _ptr(rp), nb, _ptr(out), _stream())
    return out


def hpsi(g: Geometry, veff, dij, rp, psi, out=None):
    """Fused H psi (nonlocal D term + stencil + veff)."""
    nb = _nb(g, psi)
    out = torch.empty_like(psi) if out is None else out
    fn = "rs_hpsi_f64" if psi.dtype == torch.float64 else "rs_hpsi_f32"
    _need(veff, psi.dtype, g.N, "veff")
    L.call(fn, g.handle, _ptr(veff), _ptr(dij), _ptr(rp), _ptr(psi), _ptr(out), nb, _stream())
    return out


def spsi(g: Geometry, sss, rp, psi, out=None):
    """S psi = psi + nonlocal(sss) term (nhs=0)."""
    nb = _nb(g, psi)
    out = torch.empty_like(psi) if out is None else out
    fn = "rs_spsi_f64" if psi.dtype == torch.float64 else "rs_spsi_f32"
    L.call(fn, g.handle, _ptr(sss), _ptr(rp), _ptr(psi), _ptr(out), nb, _stream())
    return out


def hpsi_host(g: Geometry, veff, dij, rp, psi_host: torch.Tensor, out_host: torch.Tensor,
              chunk: int = 64):
    """H psi with host (pinned) psi/hpsi buffers, FP32."""
    nb = psi_host.numel() // g.N
    L.call("rs_hpsi_host_f32", g.handle, _ptr(veff), _ptr(dij), _ptr(rp), _ptr(psi_host),
           _ptr(out_host), nb, chunk, _stream())
    return out_host


def ksprecondition(g: Geometry, x, out=None):
    nb = _nb(g, x)
    out = torch.empty_like(x) if out is None else out
    fn = "rs_precondition_f64" if x.dtype == torch.float64 else "rs_precondition_f32"
    L.call(fn, g.handle, _ptr(x), _ptr(out), nb, _stream())
    return out


def scf_charge_smt(occ, psi, N: int):
    """rho = sum_b occ_b psi_b^2 (scf_charge_smt_r), FP64."""
    nb = psi.numel() // N
    rho = torch.empty(N, dtype=torch.float64, device=psi.device)
    fn = "rs_density_f64" if psi.dtype == torch.float64 else "rs_density_f32"
    L.call(fn, N, nb, _ptr(occ), _ptr(psi), _ptr(rho), _stream())
    return rho


def trans_c2d_smtcharge(shape, nf: int, rho):
    """Coarse -> dense (nmesh=2) Lagrange interpolation of order 2 nf."""
    nx, ny, nz = shape
    out = torch.empty(8 * nx * ny * nz, dtype=torch.float64, device=rho.device)
    L.call("rs_interp_c2d", nx, ny, nz, nf, _ptr(rho), _ptr(out), _stream())
    return out


def scf_hartee_laplacian(shape, nfh: int, h, v):
    nx, ny, nz = shape
    out = torch.empty_like(v)
    L.call("rs_hartree_laplacian", nx, ny, nz, nfh, h[0], h[1], h[2], _ptr(v), _ptr(out),
           _stream())
    return out


def scf_hartree(shape, nfh: int, xmax, rho, vh, epsvh=1e-12, ncgmin=1, ncgmax=800,
                ncgres=801, mixed: bool = False):
    """CG Poisson solve; vh (in/out) is the warm start.  Returns (iters, dp).
    mixed: FP32 CG vectors with FP64 vh, dots and norms (rs_hartree_cg_f32)."""
    nx, ny, nz = shape
    it = C.c_int(0)
    dp = C.c_double(0)
    L.call("rs_hartree_cg_f32" if mixed else "rs_hartree_cg", nx, ny, nz, nfh, xmax[0], xmax[1],
           xmax[2], epsvh, ncgmin, ncgmax, ncgres, _ptr(rho), _ptr(vh), C.byref(it),
           C.byref(dp), _stream())
    return it.value, dp.value


def trans_d2c(shape, nf: int, v_dense):
    """Dense -> coarse transfer (trans_d2c_vh / trans_d2c_vxc, periodic)."""
    nx, ny, nz = shape
    _need(v_dense, torch.float64, 8 * nx * ny * nz, "v_dense")
    out = torch.empty(nx * ny * nz, dtype=torch.float64, device=v_dense.device)
    L.call("rs_interp_d2c", nx, ny, nz, nf, _ptr(v_dense), _ptr(out), _stream())
    return out


def vxpot_lda_pz(rho):
    """Perdew-Zunger LDA: (vx, ex) per point of rho (FP64 device tensor)."""
    _need(rho, torch.float64, None, "rho")
    vx, ex = torch.empty_like(rho), torch.empty_like(rho)
    L.call("rs_vxc_pz", rho.numel(), _ptr(rho), _ptr(vx), _ptr(ex), _stream())
    return vx, ex


def veff_sum(vx, vloc, vh, veff=None, veff32=None):
    """veff = vx + (vloc + vh) into an FP64 and/or an FP32 tensor."""
    n = vx.numel()
    for t, what in ((vx, "vx"), (vloc, "vloc"), (vh, "vh")):
        _need(t, torch.float64, n, what)
    L.call("rs_veff_sum", n, _ptr(vx), _ptr(vloc), _ptr(vh), _ptr(veff), _ptr(veff32),
           _stream())
    return veff, veff32


def scf_diffcharge(rho_o, rho_i, h, xmax):
    """SCF charge difference sqrt(sum (rho_i - rho_o)^2 dV / V) (host float)."""
    out = C.c_double(0.0)
    L.call("rs_diffcharge", rho_o.numel(), _ptr(rho_o), _ptr(rho_i), h[0], h[1], h[2], xmax[0],
           xmax[1], xmax[2], C.byref(out), _stream())
    return out.value


class Mixer:
    """scf_chargemixing with modified Broyden history on the device."""

    def __init__(self, n: int, nbrydn: int = 20, eta: float = 0.02):
        L.load()
        self.h = C.c_void_p()
        L.call("rs_mixer_create", C.byref(self.h), n, nbrydn, eta)
        self.n = n

    def step(self, rho_o, rho_i, dvol: float):
        """rho_i (in/out): last input density -> next input density."""
        _need(rho_o, torch.float64, self.n, "rho_o")
        _need(rho_i, torch.float64, self.n, "rho_i")
        L.call("rs_mixer_step", self.h, _ptr(rho_o), _ptr(rho_i), dvol, _stream())
        return rho_i

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            L.load().rs_mixer_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def scf_charge_atomicocc(g: Geometry, rp, fnele):
    """Projector occupation matrices: [natom][nprjmx (nprjmx+1)/2] FP64, packed
    upper triangle with j outer (scf_charge_atomicocc)."""
    M = fnele.numel()
    _need(fnele, torch.float64, M, "fnele")
    _need(rp, torch.float64, M * g.natom * g.nprjmx, "rp")
    out = torch.empty((g.natom, g.nprjmx * (g.nprjmx + 1) // 2), dtype=torch.float64,
                      device=rp.device)
    L.call("rs_atomicocc", g.handle, _ptr(rp), _ptr(fnele), M, _ptr(out), _stream())
    return out


class HpsiBatch:
    """H psi of many small cells in one persistent launch (rs_hpsi_batch_*).

    geoms: Geometry per cell; bands: band count per cell.  set() takes per-cell
    torch CUDA tensors (veff FP32, dij FP64 per atom, rp FP64, psi and out
    FP32 [nb][N]); run() applies H to every cell, autotuning the launch on
    the first call and replaying a CUDA graph of it when graph=True."""

    def __init__(self, geoms, bands):
        L.load()
        self.geoms = list(geoms)
        self.bands = [int(b) for b in bands]
        n = len(self.geoms)
        garr = (C.c_void_p * n)(*[g.handle.value for g in self.geoms])
        barr = (C.c_int * n)(*self.bands)
        self.h = C.c_void_p()
        L.call("rs_hpsi_batch_create", C.byref(self.h), n, garr, barr)
        self._keep = []

    def set(self, veff, dij, rp, psi, out):
        n = len(self.geoms)
        arr = lambda ts: (C.c_void_p * n)(*[t.data_ptr() for t in ts])
        for g, nb, v, ps, o in zip(self.geoms, self.bands, veff, psi, out):
            _need(v, torch.float32, g.N, "veff")
            _need(ps, torch.float32, nb * g.N, "psi")
            _need(o, torch.float32, nb * g.N, "out")
        self._keep = [list(veff), list(dij), list(rp), list(psi), list(out)]
        L.call("rs_hpsi_batch_set_f32", self.h, arr(veff), arr(dij), arr(rp), arr(psi), arr(out))

    def run(self, graph: bool = False):
        L.call("rs_hpsi_batch_run_f32", self.h, 1 if graph else 0, _stream())

    def info(self):
        t, b, c = C.c_int(), C.c_int(), C.c_int()
        L.load().rs_hpsi_batch_info(self.h, C.byref(t), C.byref(b), C.byref(c))
        return {"threads_per_cta": t.value, "bands_per_item": b.value, "ctas_per_sm": c.value}

    def set_shape(self, threads_per_cta: int, bands_per_item: int, ctas_per_sm: int):
        """Fixes the launch shape (no autotuning); every shape gives the same bits."""
        L.call("rs_hpsi_batch_set_shape", self.h, threads_per_cta, bands_per_item, ctas_per_sm)

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            L.load().rs_hpsi_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def force_eig(g: Geometry, dij, sss, psi, sval, occ):
    """Nonlocal force on every atom (force_eig_r), as a (natom, 3) FP64 tensor.
    dij/sss are per-atom (natom, P, P) FP64 device tensors (sss None for NC),
    psi (nb, N) FP64 or FP32, sval/occ (nb,) FP64 device tensors."""
    nb = _nb(g, psi)
    f = torch.empty((3, max(g.natom, 1)), dtype=torch.float64, device=psi.device)
    for t, what in ((sval, "sval"), (occ, "occ")):
        _need(t, torch.float64, nb, what)
    fn = "rs_force_nl_f64" if psi.dtype == torch.float64 else "rs_force_nl_f32"
    L.call(fn, g.handle, _ptr(dij), None if sss is None else _ptr(sss), _ptr(psi), _ptr(sval),
           _ptr(occ), nb, _ptr(f), _stream())
    return f[:, : g.natom].T


def dot(a, b):
    out = torch.empty(1, dtype=torch.float64, device=a.device)
    fn = "rs_dot_f64" if a.dtype == torch.float64 else "rs_dot_f32"
    L.call(fn, a.numel(), _ptr(a), _ptr(b), _ptr(out), _stream())
    return out


# ----------------------------------------------------------------- band solvers
class Bands:
    """Band state of one k-point/spin: psi, S psi (aliases psi when S = 1),
    H psi, <p|psi> and the eigenvalue / residual arrays, on one device.
    dtype float64 is the plain FP64 path, float32 the mixed path."""

    def __init__(self, g: Geometry, psi: torch.Tensor, sss=None):
        self.g = g
        self.M = psi.shape[0]
        self.dtype = psi.dtype
        self.psi = psi.contiguous()
        self.sss = sss
        self.spsi = self.psi.clone() if sss is not None else self.psi
        self.hpsi = torch.zeros_like(self.psi)
        self.rp = torch.zeros((self.M, g.natom, g.nprjmx), dtype=torch.float64,
                              device=psi.device)
        self.sval = np.zeros(self.M)
        self.resid = np.zeros(self.M)

    @property
    def suffix(self):
        return "f64" if self.dtype == torch.float64 else "f32"

    def _dp(self, a):
        return a.ctypes.data_as(C.POINTER(C.c_double))


class State:
    """The device-resident state handle (rs_create ... rs_destroy): psi, S psi,
    H psi, <p|psi>, veff, D and S of one cell live in the library; numpy
    arrays go in and come out."""

    def __init__(self, cell: Cell, nbands: int, precision: int = 32, nf: int = 4):
        self.cell, self.M, self.prec = cell, nbands, precision
        self.dtype = np.float32 if precision == 32 else np.float64
        h = C.c_void_p()
        L.call("rs_create", C.byref(h), precision, cell.shape[0], cell.shape[1], cell.shape[2],
               nf, cell.h[0], cell.h[1], cell.h[2], nbands, _stream())
        self.handle = h
        self.sval = np.zeros(nbands)
        self.resid = np.zeros(nbands)
        ip = lambda a: np.ascontiguousarray(a, np.int32)
        dp = lambda a: np.ascontiguousarray(a, np.float64)
        self._keep = [ip(cell.nprj), ip(cell.natinf), ip(cell.lst), dp(cell.vnlocp),
                      dp(cell.dij), dp(cell.sss) if cell.sss is not None else None]
        nprj, natinf, lst, v, dij, sss = self._keep
        P = C.POINTER
        L.call("rs_upload_geometry", h, cell.natom, cell.nprjmx, cell.num_list,
               nprj.ctypes.data_as(P(C.c_int)), natinf.ctypes.data_as(P(C.c_int)),
               lst.ctypes.data_as(P(C.c_int)), v.ctypes.data_as(P(C.c_double)),
               dij.ctypes.data_as(P(C.c_double)),
               sss.ctypes.data_as(P(C.c_double)) if sss is not None else None)

    def _d(self, a):
        return a.ctypes.data_as(C.POINTER(C.c_double))

    def set_potential(self, veff):
        v = np.ascontiguousarray(veff, np.float64)
        L.call("rs_set_potential", self.handle, self._d(v))

    def upload_bands(self, psi):
        p = np.ascontiguousarray(psi, self.dtype)
        L.call("rs_upload_bands", self.handle, p.ctypes.data_as(C.c_void_p))

    def download_bands(self):
        out = np.empty((self.M, self.cell.N), self.dtype)
        L.call("rs_download_bands", self.handle, out.ctypes.data_as(C.c_void_p))
        return out

    def orthogonalize(self, cmpt: int = 1):
        L.call("rs_orthogonalize", self.handle, cmpt)

    def hpsi(self):
        L.call("rs_hpsi", self.handle)

    def diag_step(self, iscf: int, prm=None):
        prm = prm or L.solver_prm()
        conv, itm = C.c_int(0), C.c_int(0)
        L.call("rs_diag_step", self.handle, C.byref(prm), iscf, self._d(self.sval),
               self._d(self.resid), C.byref(conv), C.byref(itm))
        return bool(conv.value), itm.value

    def density(self, occ):
        o = np.ascontiguousarray(occ, np.float64)
        rho = np.empty(self.cell.N)
        L.call("rs_density", self.handle, self._d(o), self._d(rho))
        return rho

    def close(self):
        if self.handle:
            L.call("rs_destroy", self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def orthogonalization(b: Bands, cmpt: int = 1):
    """orthogonalization_r_01, all bands (Cholesky-QR in the S metric)."""
    L.call("rs_orthogonalize_" + b.suffix, b.g.handle, _ptr(b.sss), b.M, _ptr(b.psi),
           _ptr(b.spsi), _ptr(b.rp), cmpt, _stream())


def orthogonalization_band(b: Bands, l: int, cmpt: int = 0):
    L.call("rs_orthogonalize_band_" + b.suffix, b.g.handle, _ptr(b.sss), b.M, l, _ptr(b.psi),
           _ptr(b.spsi), _ptr(b.rp), cmpt, _stream())


def rayleighritz(b: Bands, veff, dij, l_rrb: int = 1):
    L.call("rs_rayleighritz_" + b.suffix, b.g.handle, _ptr(veff), _ptr(dij), _ptr(b.sss), b.M,
           _ptr(b.psi), _ptr(b.spsi), _ptr(b.rp), _ptr(b.hpsi), l_rrb, b._dp(b.sval), _stream())
    return b.sval


def kscg(b: Bands, veff, dij, prm=None):
    prm = prm or L.solver_prm()
    itm = C.c_int(0)
    L.call("rs_kscg_" + b.suffix, b.g.handle, _ptr(veff), _ptr(dij), _ptr(b.sss), C.byref(prm),
           b.M, _ptr(b.psi), _ptr(b.spsi), _ptr(b.rp), _ptr(b.hpsi), b._dp(b.sval),
           b._dp(b.resid), C.byref(itm), _stream())
    return itm.value


def ksdiis(b: Bands, veff, dij, prm=None, l_hsv: int = 1):
    prm = prm or L.solver_prm()
    conv = C.c_int(0)
    L.call("rs_ksdiis_" + b.suffix, b.g.handle, _ptr(veff), _ptr(dij), _ptr(b.sss), C.byref(prm),
           b.M, l_hsv, _ptr(b.psi), _ptr(b.spsi), _ptr(b.rp), _ptr(b.hpsi), b._dp(b.sval),
           b._dp(b.resid), C.byref(conv), _stream())
    return bool(conv.value)


def reorderstates(b: Bands):
    L.call("rs_reorder_" + b.suffix, b.g.handle, _ptr(b.sss), b.M, _ptr(b.psi), _ptr(b.spsi),
           _ptr(b.rp), b._dp(b.sval), b._dp(b.resid), _stream())


def scf_diag(b: Bands, veff, dij, iscf: int, prm=None):
    """scf_diag for one k-point/spin; returns (ksconv, ksitmax)."""
    prm = prm or L.solver_prm()
    conv, itm = C.c_int(0), C.c_int(0)
    L.call("rs_scf_diag_" + b.suffix, b.g.handle, _ptr(veff), _ptr(dij), _ptr(b.sss),
           C.byref(prm), iscf, b.M, _ptr(b.psi), _ptr(b.spsi), _ptr(b.rp), _ptr(b.hpsi),
           b._dp(b.sval), b._dp(b.resid), C.byref(conv), C.byref(itm), _stream())
    return bool(conv.value), itm.value


def syev(a: torch.Tensor):
    """FP64 symmetric eigen-decomposition on the GPU (ascending)."""
    n = a.shape[0]
    A = a.to(torch.float64).contiguous().clone()
    w = torch.empty(n, dtype=torch.float64, device=a.device)
    Z = torch.empty((n, n), dtype=torch.float64, device=a.device)
    sw = C.c_int(0)
    L.call("rs_syev_f64", n, _ptr(A), _ptr(w), _ptr(Z), C.byref(sw), _stream())
    return w, Z.T, sw.value   # Z stored column-major: columns are vectors
