"""kukan's local pseudopotential, ion-ion energy and initial bands of a
periodic cell, built on the GPU through the C ABI.

Host side (set-up scalars, as kukan computes them once per dataset):

* ``local_params`` -- cp1 (the valence charge rounded to 1e-4,
  read_ppfile8f.F90:122-125) and the soft part b cos(a r) + c inside r_c of
  tools_bisec (tools8f.F90:922-953), matched in value and slope to -cp1/r at
  r_c = radial(nradct);
* ``local_potc`` -- potc on the dataset's radial mesh, (vloc - vh)/2
  (read_ppfile8f.F90:158-167).  For PAW datasets kukan also subtracts the
  LDA potential of the dataset's density column (:168-186), which pairs with
  its one-centre and partial-core terms; the cells here carry neither, so
  that subtraction is off unless asked for (paw_xc=True, the LDA through
  rs_vxc_pz);
* ``local_coefs`` -- the Fourier-Bessel coefficients of the hard part
  potc - (b cos(a r) + c) summed over the radial mesh as
  filterpseudopotentials does (filterpseudopotentials8f.F90:62-69, 72-91,
  107-131; nfiltyp = 1 cut-off nqct = int(rcut psftrad / max(h))).

Device side:

* ``local_potential`` -- vloc_dense and vloc_coarse of pseudocalc
  (pseudocalc8f.F90:117-210): the soft part on the coarse grid
  (rs_vloc_soft), coarse -> dense (rs_interp_c2d), plus the hard part on the
  dense grid (rs_vloc_hard_add), dense -> coarse (rs_interp_d2c);
* ``ion_energy`` -- the Ewald energy eneat and the ion-ion forces (rs_ewald);
* ``initial_bands`` -- setup_initialwave's bands (rs_initial_wave_*).
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np
import torch

from . import lib as _lib
from .kukan import _stream
from .system import Cell, PSCTOFF

VETA = 0.2          # read_input_kukan8f.F90:273
NEW_PW = 11         # :274-276
NEW_RS = 11         # :277-279
ZS_PRE = 0.5        # :290
PSFTRAD = 10.0      # :266
FILPP = 0.02        # :269
NFILTYP = 1         # :262
EPS = 1.0e-16       # :245
NMESH = 2


def bisec(z: float, r: float, eps: float = 1.0e-12):
    """tools_bisec: (a, b, c) with b cos(a r) + c = -z/r and its slope equal to
    z/r^2 at r, a found by bisection of tan(a r)/a = -r/2 on (pi/2r, pi/r)."""
    a0 = math.pi * 0.5 / r + eps
    a2 = 2.0 * math.pi * 0.5 / r - eps
    fr = -r / 2.0
    l = 0
    while True:
        l += 1
        a = (a0 + a2) * 0.5
        f0 = math.tan(a0 * r) / a0 - fr
        f1 = math.tan(a * r) / a - fr
        if f0 * f1 < 0.0:
            a2 = a
        else:
            a0 = a
        if l > 1000000 or not (a2 - a0 > eps):
            break
    b = -z / r / r / a / math.sin(a * r)
    c = -z / r - b * math.cos(a * r)
    return a, b, c


def local_params(ds: dict):
    """(cp1, a, b, c, rcut) of the dataset's soft local part."""
    # i = nint(cp1 * 10000), cp1 = i / 10000 (Fortran nint: halves away from zero)
    cp1 = math.copysign(math.floor(abs(ds["zv"]) * 10000.0 + 0.5), ds["zv"]) / 10000.0
    rcut = float(ds["mesh_r"][ds["nradct"] - 1])
    a, b, c = bisec(cp1, rcut)
    return cp1, a, b, c, rcut


def local_potc(ds: dict, paw_xc: bool = False) -> np.ndarray:
    """potc on the radial mesh (Ha): (vloc - vh)/2, minus v_xc(PZ) of the
    mesh density for PAW datasets when paw_xc."""
    potc = np.asarray(ds["mesh_potc"], dtype=np.float64).copy()
    if paw_xc and ds["kind"] == "paw":
        rho = torch.tensor(np.asarray(ds["mesh_rho"], dtype=np.float64), device="cuda")
        vx, ex = torch.empty_like(rho), torch.empty_like(rho)
        _lib.call("rs_vxc_pz", rho.numel(), C.c_void_p(rho.data_ptr()),
                  C.c_void_p(vx.data_ptr()), C.c_void_p(ex.data_ptr()), _stream())
        potc = potc - vx.cpu().numpy()
    return potc


def local_coefs(ds: dict, h, potc=None, psftrad: float = PSFTRAD):
    """(coef[0..nqct], nqct, rcuts): coef(iq) = sum_{ir=2}^{nradps}
    4 pi r^2 j0(q r) vlocr(r) dr/di, q = iq pi / rcuts, with vlocr = potc -
    (b cos(a r) + c) up to nradct and 0 beyond (filterpseudopotentials)."""
    cp1, a, b, c, rcut = local_params(ds)
    potc = local_potc(ds) if potc is None else potc
    r = np.asarray(ds["mesh_r"], dtype=np.float64)
    dr = np.asarray(ds["mesh_drdi"], dtype=np.float64)
    nradps, nradct = ds["nradps"], ds["nradct"]
    rcuts = rcut * psftrad
    nqct = int(rcuts / max(h))
    vlocr = np.zeros(nradps)
    ir = np.arange(1, nradct)                     # Fortran ir = 2..nradct
    vlocr[ir] = potc[ir] - (b * np.cos(a * r[ir]) + c)
    rr, ddr, vv = r[1:nradps], dr[1:nradps], vlocr[1:nradps]
    coef = np.zeros(nqct + 1)
    for iq in range(nqct + 1):
        q = math.pi / rcuts * iq
        j0 = np.ones_like(rr) if iq == 0 else np.sin(q * rr) / (q * rr)
        terms = 4.0 * math.pi * rr * rr * j0 * vv * ddr
        coef[iq] = float(np.cumsum(terms)[-1])   # left to right, as the Fortran loop
    return coef, nqct, rcuts


def _atxyz(cell: Cell) -> np.ndarray:
    return np.ascontiguousarray(cell.atoms, dtype=np.float64).reshape(-1)


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def local_potential(cell: Cell, stream=None, npw: int = NEW_PW, veta: float = VETA):
    """(vloc_coarse, vloc_dense) of the cell as FP64 CUDA tensors (N and 8N)."""
    ds = cell.ds
    cp1, a, b, c, rcut = local_params(ds)
    coef, nqct, rcuts = local_coefs(ds, cell.h)
    nx, ny, nz = cell.shape
    dx, dy, dz = cell.h
    xm, ym, zm = cell.xmax
    N = cell.N
    atxyz = _atxyz(cell)
    prm = np.ascontiguousarray(np.tile([cp1, a, b, c, rcut], cell.natom), dtype=np.float64)
    st = _stream() if stream is None else C.c_void_p(stream)
    soft = torch.empty(N, dtype=torch.float64, device="cuda")
    sp = C.c_void_p(soft.data_ptr())
    _lib.call("rs_vloc_soft", cell.natom, _p(atxyz), _p(prm), nx, ny, nz, dx, dy, dz, xm, ym, zm,
              veta, npw, npw, npw, sp, st)
    dense = torch.empty(8 * N, dtype=torch.float64, device="cuda")
    dp = C.c_void_p(dense.data_ptr())
    _lib.call("rs_interp_c2d", nx, ny, nz, 4, sp, dp, st)
    spe = np.zeros(cell.natom, np.int32)
    sprm = np.array([rcut, rcuts, FILPP], dtype=np.float64)
    nq = np.array([nqct], np.int32)
    _lib.call("rs_vloc_hard_add", cell.natom, _p(atxyz), spe.ctypes.data_as(C.POINTER(C.c_int)),
              1, _p(sprm), nq.ctypes.data_as(C.POINTER(C.c_int)), nqct, _p(coef), nx, ny, nz,
              dx, dy, dz, xm, ym, zm, NMESH, cell.npmax[0], cell.npmax[1], cell.npmax[2],
              PSCTOFF, EPS, NFILTYP, dp, st)
    coarse = torch.empty(N, dtype=torch.float64, device="cuda")
    _lib.call("rs_interp_d2c", nx, ny, nz, 4, dp, C.c_void_p(coarse.data_ptr()), st)
    return coarse, dense


def ion_energy(cell: Cell, forces: bool = False, npw: int = NEW_PW, veta: float = VETA):
    """eneat (Ha) of the cell's ions, and their Ewald forces (natom x 3,
    Ha/bohr) when asked."""
    cp1 = local_params(cell.ds)[0]
    q = np.full(cell.natom, cp1)
    e = C.c_double(0.0)
    f = np.zeros(3 * cell.natom)
    _lib.call("rs_ewald", cell.natom, _p(_atxyz(cell)), _p(q), *cell.xmax, veta, npw, npw, npw,
              C.byref(e), _p(f) if forces else None, _stream())
    return (e.value, f.reshape(-1, 3)) if forces else e.value


def initial_bands(cell: Cell, M: int, dtype=torch.float64, zs_pre: float = ZS_PRE,
                  stream=None) -> torch.Tensor:
    """setup_initialwave's M bands (s, then p, then d forms per atom) as a
    CUDA tensor (M x N) of dtype."""
    cp1 = local_params(cell.ds)[0]
    zs = np.full(cell.natom, cp1 * zs_pre)
    psi = torch.empty((M, cell.N), dtype=dtype, device="cuda")
    fn = "rs_initial_wave_f64" if dtype == torch.float64 else "rs_initial_wave_f32"
    _lib.call(fn, cell.natom, _p(_atxyz(cell)), _p(zs), M, *cell.shape, *cell.h, *cell.xmax,
              C.c_void_p(psi.data_ptr()), _stream() if stream is None else C.c_void_p(stream))
    return psi
