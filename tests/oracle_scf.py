"""The SCF loop of rspacedist_b200.scf restated on the CPU oracle (test
infrastructure), FP64 throughout, in kukan's order (kukan8f.F90:466-762):
the local pseudopotential of pseudocalc and the bands of setup_initialwave,
Gram-Schmidt, the start density with the occupations of equal eigenvalues;
per iteration Broyden mixing, c2d, Hartree CG, PZ LDA, d2c, veff sum, then
Rayleigh-Ritz + CG (iscf <= ncgscf) or Rayleigh-Ritz + DIIS, a stable
ascending reorder, the Fermi-Dirac occupations (the same host function as the
GPU driver), the density and the charge difference; at the end the terms of
output_energy on the last input density."""
import numpy as np

import oracle_pp as OP


def geo_dict(cell):
    return dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
                natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())


def oracle_scf(O, cell, M, nocc, eps_scf=1e-6, looplimit=100, nbrydn=20, eta=0.02,
               ncgscf=3, epsvh=1e-12, smearing=True, tf=3.0e-3):
    from rspacedist_b200 import scf as SCF
    geo = geo_dict(cell)
    N, shape = cell.N, cell.shape
    dshape = tuple(2 * s for s in shape)
    h, xmax = cell.h, cell.xmax
    dvol = h[0] * h[1] * h[2]
    vloc = OP.local_potential(O, cell)[0]
    cp1 = np.floor(cell.ds["zv"] * 10000.0 + 0.5) / 10000.0
    psi = O.initial_wave(cell.atoms, cp1, 0.5, M, shape, h, xmax)
    sysk = O.make_sys(geo, shape, 4, h, np.zeros(N), cell.dij, cell.sss)
    rp = O.nl_dot(geo, psi, N)
    sp = O.spsi(sysk, psi, rp) if cell.sss is not None else None
    psi, sp, rp = O.ortho(sysk, M, psi, sp, rp, 0, 1)
    if smearing:
        occ = SCF.scf_occupation(np.zeros(M), 2.0 * nocc, tf)[0]
    else:
        occ = np.zeros(M)
        occ[:nocc] = 2.0
    rho_o = O.density(occ, psi, N)
    mix = O.Broyden(N, nbrydn, eta)
    rho_i = np.zeros(N)
    vh_d = np.zeros(8 * N)
    diffs = []
    sval = rho_d = vx = ex_d = None
    for iscf in range(1, looplimit + 1):
        rho_i = mix.step(rho_o, rho_i, dvol)
        rho_d = O.interp_c2d(shape, 4, rho_i)
        vh_d, _, _ = O.hartree_cg(dshape, 4, xmax, epsvh, 1, 800, 801, rho_d, vh_d)
        vh = O.interp_d2c(shape, 4, vh_d)
        vx_d, ex_d = O.vxc_pz(rho_d)
        vx = O.interp_d2c(shape, 4, vx_d)
        veff = O.veff_sum(vx, vloc, vh)
        sysk = O.make_sys(geo, shape, 4, h, veff, cell.dij, cell.sss)
        _, psi, sp, rp, sval = O.rayleighritz(sysk, M, psi, sp, rp)
        if iscf <= ncgscf:
            _, psi, sp, rp, _, sval, _ = O.kscg(sysk, M, psi, sp, rp, nsdmax=4)
        else:
            _, psi, sp, rp, _, sval, _ = O.ksdiis(sysk, M, psi, sp, rp, l_hsv=1)
        order = np.argsort(sval, kind="stable")
        psi, rp, sval = psi[order], rp[order], sval[order]
        if sp is not None:
            sp = sp[order]
        if smearing:
            occ = SCF.scf_occupation(sval, 2.0 * nocc, tf)[0]
        rho_o = O.density(occ, psi, N)
        diffs.append(O.diffcharge(rho_o, rho_i, h, xmax))
        if diffs[-1] < eps_scf:
            break
    ddv = dvol / 8.0
    eband = float(np.cumsum(occ * sval)[-1])
    eneha = -0.5 * O.tree_dot(vh_d, rho_d) * ddv
    eneex = -O.tree_dot(rho_i, vx) * dvol + O.tree_dot(rho_d, ex_d) * ddv
    eneat = OP.ion_energy(O, cell)
    eneth = SCF.helmholtz_entropy(occ, tf) if smearing else 0.0
    etot = eband + eneex + eneha + eneat
    return dict(sval=np.asarray(sval), eband=eband, diff=diffs, converged=diffs[-1] < eps_scf,
                iterations=len(diffs), occ=occ, psi=psi, rho_out=rho_o,
                energy=dict(eneel=eband, eneex=eneex, eneha=eneha, eneat=eneat, eneth=eneth,
                            total=etot, free=etot + eneth))
