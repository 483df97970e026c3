"""Projector tables on the GPU: the set-up path of kukan's nonlocal
pseudopotential (filterpseudopotentials, pseudocalc_01a, pseudocalc_07).

* ``bessel_coefs`` -- Fourier-Bessel coefficients of each projector channel,
  coef(iq, 1 + 2l + i) = sum_{ir >= 2} 4 pi r j_l(q r) (r p)(r) dr with
  q = iq pi / (rcut psftrad), iq = 0..nqct, nqct = int(rcut psftrad / max(h))
  (filterpseudopotentials8f.F90:72-91 for nfiltyp >= 1, :107-290 for the
  sums); the King-Smith correction of nfiltyp = 0 is not restated.
* ``channel_table`` -- per projector the coefficient column (tmpspd1..6) and
  the real harmonic (ylm01..ylm09) in the order of pseudocalc_07's cases.
* ``projector_tables`` -- vnlocp(num_list, nprj, natom) of a cell through
  ``rs_projector_tables`` (Bessel sums on the npmesh fine mesh, Fermi filter,
  double-grid contraction of pseudocalc_07), with the weights of
  ``rs_double_grid_weights`` (pseudocalc_01a).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import lib as _lib
from .system import Cell, projector_layout

PSFTRAD = 10.0   # read_input_kukan8f.F90:266
PSCTOFF = 1.05   # :264
FILPP = 0.02     # :269
NFILTYP = 1      # :262 (Fermi-distribution filter)
NPMESH = 2       # :287
EPS = 1.0e-16    # :245


def _spherical_jl(l: int, z: np.ndarray) -> np.ndarray:
    """j_l(z) for z > 0 in the closed forms of filterpseudopotentials."""
    s, c = np.sin(z), np.cos(z)
    if l == 0:
        return s / z
    if l == 1:
        return (s - z * c) / (z * z)
    return ((3.0 - z * z) * s - 3.0 * z * c) / (z * z * z)


def bessel_coefs(ds: dict, h, psftrad: float = PSFTRAD):
    """(coef, nqct, nqmx): coef is the (nqmx+1) x 8 column-major table
    coef(0:nqmx, 0:7) flattened, column 1 + 2l + i for the i-th radial
    projector of angular momentum l."""
    rcuts = ds["rcut"] * psftrad
    nqct = int(rcuts / max(h))
    nqmx = nqct
    coef = np.zeros((8, nqmx + 1))
    dr = ds["dr"]
    for ch in ds["channels"]:
        p = np.asarray(ch["p"], dtype=np.float64)
        r = np.arange(len(p)) * dr
        rp = r * p                       # (r p)(r), as stored in the dataset file
        col = 1 + 2 * ch["l"] + ch["i"]
        rr, rpp = r[1:], rp[1:]          # the radial sums start at ir = 2
        for iq in range(nqct + 1):
            q = np.pi / rcuts * iq
            if iq == 0:
                jl = np.ones_like(rr) if ch["l"] == 0 else np.zeros_like(rr)
            else:
                jl = _spherical_jl(ch["l"], q * rr)
            coef[col, iq] = np.sum(4.0 * np.pi * rr * jl * rpp * dr)
    return np.ascontiguousarray(coef.ravel()), nqct, nqmx


def channel_table(ds: dict):
    """(prj_col, prj_m) per projector in the order of projector_layout."""
    col, ym = [], []
    for ci, l, m in projector_layout(ds):
        ch = ds["channels"][ci]
        col.append(1 + 2 * l + ch["i"])
        ym.append(1 if l == 0 else (2 + m if l == 1 else 5 + m))
    return np.array(col, np.int32), np.array(ym, np.int32)


def double_grid_weights(nfdg: int, npmesh: int) -> np.ndarray:
    w = np.zeros(2 * nfdg * npmesh)
    _lib.call("rs_double_grid_weights", nfdg, npmesh, w.ctypes.data_as(C.POINTER(C.c_double)))
    return w


def projector_tables(cell: Cell, npmesh: int = NPMESH, nfdg: int = 4, psftrad: float = PSFTRAD,
                     psctoff: float = PSCTOFF, nfiltyp: int = NFILTYP, filpp: float = FILPP,
                     eps: float = EPS, stream=None, out=None):
    """vnlocp of the cell, shape (natom, nprj, num_list), from the GPU: a
    numpy array, or ``out`` (a contiguous FP64 CUDA tensor of that shape,
    written in stream order) when given."""
    ds = cell.ds
    coef, nqct, nqmx = bessel_coefs(ds, cell.h, psftrad)
    col, ym = channel_table(ds)
    w = double_grid_weights(nfdg, npmesh)
    A, L, P = cell.natom, cell.num_list, len(col)
    at = np.ascontiguousarray(cell.atoms, dtype=np.float64)
    ax, ay, az = (np.ascontiguousarray(at[:, k]) for k in range(3))
    lx, ly, lz = (np.ascontiguousarray(a, dtype=np.int32) for a in cell.lstxyz)
    nat = [np.ascontiguousarray(a, dtype=np.int32) for a in cell.natxyz]
    natinf = np.ascontiguousarray(cell.natinf, dtype=np.int32)
    v = np.zeros((A, P, L)) if out is None else out
    dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    vp = dp(v) if out is None else C.cast(C.c_void_p(out.data_ptr()), C.POINTER(C.c_double))
    ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))
    _lib.call("rs_projector_tables", A, P, L, cell.nmax[0], cell.nmax[1], cell.nmax[2],
              cell.h[0], cell.h[1], cell.h[2], cell.npmax[0], cell.npmax[1], cell.npmax[2], nfdg,
              npmesh, dp(ax), dp(ay), dp(az), ip(nat[0]), ip(nat[1]), ip(nat[2]), ip(natinf),
              ip(lx), ip(ly), ip(lz), ip(col), ip(ym), nqct, nqmx, dp(coef), ds["rcut"], psftrad,
              psctoff, eps, nfiltyp, filpp, dp(w), vp, stream)
    return v
