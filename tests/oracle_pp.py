"""The local pseudopotential and ion-ion energy of a cell computed by the CPU
oracle (oracle/rs_oracle_vloc.c), with the set-up scalars of kukan
(tools_bisec, the potc of read_ppfile, the Fourier-Bessel coefficients of
filterpseudopotentials) also taken from the oracle.  Test infrastructure."""
import numpy as np

VETA, NPW, NRS = 0.2, 11, 11
PSFTRAD, FILPP, EPS, NFILTYP, PSCTOFF = 10.0, 0.02, 1.0e-16, 1, 1.05


def local_setup(O, ds, h, paw_xc=False):
    """(cp1, a, b, c, rcut, coef, nqct, rcuts) of the dataset by the oracle."""
    cp1 = np.floor(ds["zv"] * 10000.0 + 0.5) / 10000.0
    rcut = ds["mesh_r"][ds["nradct"] - 1]
    a, b, c = O.bisec(cp1, rcut)
    potc = np.asarray(ds["mesh_potc"], dtype=np.float64)
    if paw_xc and ds["kind"] == "paw":
        potc = potc - O.vxc_pz(np.asarray(ds["mesh_rho"]))[0]
    rcuts = rcut * PSFTRAD
    nqct = int(rcuts / max(h))
    coef = O.vloc_coef(ds["mesh_r"], ds["mesh_drdi"], potc, ds["nradct"], a, b, c, rcuts, nqct)
    return cp1, a, b, c, rcut, coef, nqct, rcuts


def local_potential(O, cell, veta=VETA):
    """(vloc_coarse, vloc_dense, soft) of pseudocalc for the cell."""
    cp1, a, b, c, rcut, coef, nqct, rcuts = local_setup(O, cell.ds, cell.h)
    soft = O.vloc_soft(cell.atoms, cp1, a, b, c, rcut, cell.shape, cell.h, cell.xmax, veta,
                       (NPW, NPW, NPW))
    dense = O.interp_c2d(cell.shape, 4, soft)
    O.vloc_hard(cell.atoms, cell.nmax, 2, cell.h, cell.xmax, cell.npmax, rcut, PSCTOFF, rcuts,
                nqct, coef, FILPP, EPS, NFILTYP, dense=dense)
    coarse = O.interp_d2c(cell.shape, 4, dense)
    return coarse, dense, soft


def ion_energy(O, cell, veta=VETA):
    cp1 = np.floor(cell.ds["zv"] * 10000.0 + 0.5) / 10000.0
    return O.ewald(cell.atoms, cp1, cell.xmax, veta, (NPW,) * 3, (NRS,) * 3)
