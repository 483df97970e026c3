"""Atomic forces of a converged SCF by one adjoint pass (kukan's force
routine, force8f.F90:1617-2013 with force_eig_r, :9-195, recast as the exact
derivative of the discrete total energy):

    F_a = F_local + F_projector + F_ion

* F_local (rs_force_local): dV sum rho_soft grad soft_a + dV/8 sum rho_dense
  grad hard_a, with rho_dense = c2d(rho) and rho_soft = d2c(rho_dense) -- the
  adjoint of vloc_coarse = d2c(c2d(soft) + hard);
* F_projector (rs_force_adjoint_*): 2 sum_l f_l (D - e_l S)_ij <p_i|psi_l>
  <grad p_j|psi_l>, the projector values and gradients recomputed from the
  radial tables at every sphere-list point;
* F_ion (rs_ewald): the Ewald forces of the ions.

The projector part follows the directly sampled tables of
system.build_projectors (radial function linearly interpolated, zero from
r_cut); it is the derivative of the energy whose H psi uses those tables.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import kukan as K
from . import lib as _lib
from . import pseudo as PP
from .system import Cell, PSCTOFF, projector_layout

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int)


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


def local_forces(cell: Cell, rho: torch.Tensor, npw: int = PP.NEW_PW,
                 veta: float = PP.VETA) -> np.ndarray:
    """(natom, 3) local-pseudopotential forces for the coarse density rho
    (FP64 CUDA tensor)."""
    ds = cell.ds
    cp1, a, b, c, rcut = PP.local_params(ds)
    coef, nqct, rcuts = PP.local_coefs(ds, cell.h)
    shape = cell.shape
    rho_d = K.trans_c2d_smtcharge(shape, 4, rho)
    rho_s = K.trans_d2c(shape, 4, rho_d)
    atxyz = np.ascontiguousarray(cell.atoms, dtype=np.float64).reshape(-1)
    prm = np.ascontiguousarray(np.tile([cp1, a, b, c, rcut], cell.natom), dtype=np.float64)
    spe = np.zeros(cell.natom, np.int32)
    sprm = np.array([rcut, rcuts, PP.FILPP])
    nq = np.array([nqct], np.int32)
    f = np.zeros(3 * cell.natom)
    _lib.call("rs_force_local", cell.natom, _d(atxyz), _d(prm), _i(spe), 1, _d(sprm), _i(nq),
              nqct, _d(coef), *shape, *cell.h, *cell.xmax, veta, npw, npw, npw, PP.NMESH,
              *cell.npmax, PSCTOFF, PP.EPS, PP.NFILTYP, C.c_void_p(rho_s.data_ptr()),
              C.c_void_p(rho_d.data_ptr()), _d(f), K._stream())
    return f.reshape(-1, 3)


def projector_forces(cell: Cell, psi: torch.Tensor, sval, occ, dij: torch.Tensor,
                     sss: torch.Tensor | None = None, rp_out: torch.Tensor | None = None):
    """(natom, 3) projector forces of the bands psi (FP64 or FP32 CUDA tensor,
    nb x N) with eigenvalues sval and occupations occ; rp_out (FP64 CUDA,
    nb x natom x nprj) receives the recomputed <p|psi> when given."""
    ds = cell.ds
    lay = projector_layout(ds)
    P = len(lay)
    tabs = np.ascontiguousarray(np.stack([np.asarray(ch["p"], np.float64)
                                          for ch in ds["channels"]]))
    ntab, nr = tabs.shape
    prj_tab = np.array([ci for ci, _, _ in lay], np.int32)
    prj_l = np.array([l for _, l, _ in lay], np.int32)
    prj_form = np.array([0 if l == 0 else (1 + m if l == 1 else 4 + m) for _, l, m in lay],
                        np.int32)
    atxyz = np.ascontiguousarray(cell.atoms, dtype=np.float64).reshape(-1)
    natxyz = np.ascontiguousarray(np.concatenate(cell.natxyz), dtype=np.int32)
    lstxyz = np.ascontiguousarray(np.concatenate(cell.lstxyz), dtype=np.int32)
    natinf = np.ascontiguousarray(cell.natinf, dtype=np.int32)
    lst = np.ascontiguousarray(cell.lst, dtype=np.int32)
    nb = psi.shape[0]
    sv = torch.as_tensor(np.ascontiguousarray(sval, dtype=np.float64), device=psi.device)
    oc = torch.as_tensor(np.ascontiguousarray(occ, dtype=np.float64), device=psi.device)
    f = np.zeros(3 * cell.natom)
    fn = "rs_force_adjoint_f64" if psi.dtype == torch.float64 else "rs_force_adjoint_f32"
    p = lambda t: C.c_void_p(0 if t is None else t.data_ptr())
    _lib.call(fn, cell.natom, P, cell.num_list, _d(atxyz), _i(natxyz), _i(natinf), _i(lstxyz),
              _i(lst), ntab, nr, float(ds["dr"]), _d(tabs), _i(prj_tab), _i(prj_l),
              _i(prj_form), float(ds["rcut"]), *cell.shape, *cell.h, p(dij), p(sss), p(psi),
              p(sv), p(oc), nb, _d(f), p(rp_out), K._stream())
    return f.reshape(-1, 3)


def atomic_forces(cell: Cell, res) -> dict:
    """Forces (natom x 3, Ha/bohr) of a converged scf.run_scf result (its
    bands, eigenvalues, occupations and output density): the local,
    projector and ion parts and their sum."""
    b = res.bands
    dij = torch.tensor(cell.dij, dtype=torch.float64, device="cuda")
    fl = local_forces(cell, res.rho_out)
    fp = projector_forces(cell, b.psi, res.sval, res.occ, dij, b.sss)
    _, fi = PP.ion_energy(cell, forces=True)
    return dict(local=fl, projector=fp, ion=fi, total=fl + fp + fi)
