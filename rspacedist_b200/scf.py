"""The Kohn-Sham SCF loop of kukan (kukan8f.F90:466-762) driven through the
B200 library, one k-point and spin, periodic cell:

    set-up             vloc_coarse of pseudocalc                    (pseudo.local_potential)
                       bands of setup_initialwave, S-orthonormalised (rs_initial_wave_*,
                       and the start density scf_charge of them       rs_orthogonalize_*,
                       with the occupations of equal eigenvalues      rs_density_*)
    iscf = 1, 2, ...
      scf_chargemixing   rho_in  <- Broyden(rho_out, rho_in)      (rs_mixer_step)
      scf_potentials     rho_dense = c2d(rho_in)                   (rs_interp_c2d)
                         V_H dense by CG (warm start)              (rs_hartree_cg)
                         V_xc dense = PZ LDA(rho_dense)            (rs_vxc_pz)
                         veff = d2c(V_xc) + (vloc + d2c(V_H))     (rs_interp_d2c, rs_veff_sum)
      scf_diag           RR / CG / DIIS / reorder                  (rs_scf_diag_f64|f32)
      scf_occupation     Fermi-Dirac, kT = tf                      (host bisection)
      scf_charge         rho_out = sum_l f_l psi_l^2               (rs_density_*)
      scf_diffcharge     stop when sqrt(sum (rho_in-rho_out)^2 dV/V) < eps_scf
    totalenergy_space / totalenergy_eig / output_energy (kukan8f.F90:722-762,
    totalenergy8f.F90:8-199, output8f.F90:240-242) on the last input density:
      E = sum f e - 1/2 sum V_H rho_d dV_d - sum rho vx dV + sum rho_d e_xc dV_d + E_ewald
    with the dot products in FP64 on the device (rs_dot_f64) and the ion-ion
    energy from rs_ewald.

`dtype=torch.float64` is the plain FP64 path, `torch.float32` the mixed path
(FP32 bands, FP64 potentials, densities, subspace eigensolve and sums).

For PAW datasets D and S stay at the dataset's values and the density is the
smooth part only: the one-centre terms of scf_dij, scf_charge_onecenter and
scf_augcharge are not part of this loop.  `potential="model"` replaces the
local potential and start density by Gaussians per atom (a depth-1.5 Ha well
and the valence charge), as an analytic test input."""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import checkpoint as CK
from . import kukan as K
from . import lib as L
from .system import Cell


def gaussian_sum(cell: Cell, amp: float, sigma: float) -> np.ndarray:
    """sum_a amp * exp(-|r - R_a|^2 / (2 sigma^2)) on the coarse grid, with
    the minimum periodic image (grid point x = (ix + 1/2) dx - xmax)."""
    nx, ny, nz = cell.shape
    out = np.zeros((nz, ny, nx))
    reach = [int(np.ceil(5.0 * sigma / h)) for h in cell.h]
    n = (nx, ny, nz)
    for at in cell.atoms:
        idx = []
        for ax in range(3):
            c = int(np.floor((at[ax] + cell.xmax[ax]) / cell.h[ax] - 0.5))
            i = np.arange(c - reach[ax], c + reach[ax] + 2)
            x = (i + 0.5) * cell.h[ax] - cell.xmax[ax] - at[ax]
            L2 = 2.0 * cell.xmax[ax]
            x = x - L2 * np.round(x / L2)
            idx.append((np.mod(i, n[ax]), x))
        (ix, x), (iy, y), (iz, z) = idx
        r2 = z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2
        np.add.at(out, (iz[:, None, None], iy[None, :, None], ix[None, None, :]),
                  amp * np.exp(-r2 / (2.0 * sigma * sigma)))
    return out.ravel()


def model_local_potential(cell: Cell, depth: float = 1.5, width: float = 1.2) -> np.ndarray:
    return gaussian_sum(cell, -depth, width)


def atomic_density(cell: Cell, zval: float, sigma: float = 1.0) -> np.ndarray:
    amp = zval / (2.0 * np.pi * sigma * sigma) ** 1.5
    return gaussian_sum(cell, amp, sigma)


def smooth_start_bands(shape, M: int, seed: int) -> np.ndarray:
    """Seeded random bands low-pass filtered on the grid (a smooth start)."""
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((M, nz, ny, nx))
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(nz), np.fft.fftfreq(ny), np.fft.fftfreq(nx),
                             indexing="ij")
    filt = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / 0.005)
    x = np.real(np.fft.ifftn(np.fft.fftn(x, axes=(1, 2, 3)) * filt, axes=(1, 2, 3)))
    return x.reshape(M, -1)


def fermidis(fwght: float, r: float, t: float, rc: float) -> float:
    """mathfunctions8f.F90:21-36: fwght / (exp((r - rc)/t) + 1), clipped."""
    acoef = (r - rc) / t
    if abs(acoef) < 1.0e2:
        fdis = 1.0 / (np.exp(acoef) + 1.0)
    else:
        fdis = 0.0 if acoef > 0.0 else 1.0
    return fdis * fwght


def scf_occupation(sval, tnumele: float, tf: float = 3.0e-3, tfmin: float = -3.0e2,
                   tfmax: float = 3.0e2):
    """scf_occupation_fnele (scf_occupation8f.F90:227-388), mpre = 0, one
    k-point and spin: Fermi-Dirac occupations (weight 2) with the Fermi level
    found by bisection between tfmin and tfmax (at most 100 halvings, stop
    when the electron count is within 1e-12).  Returns (fnele, ferm)."""
    fwght = 2.0
    sval = np.asarray(sval, dtype=np.float64)

    def count(ferm):
        # fermidis of every band at once (the same formula and clipping), and
        # the electron count summed left to right as the Fortran loop does
        acoef = (sval - ferm) / tf
        inside = np.abs(acoef) < 1.0e2
        f = np.where(inside, 1.0 / (np.exp(np.where(inside, acoef, 0.0)) + 1.0),
                     np.where(acoef > 0.0, 0.0, 1.0)) * fwght
        return f, float(np.cumsum(f)[-1]) if f.size else 0.0

    ferm1, ferm3 = tfmax, tfmin
    _, n1 = count(ferm1)
    bisec1 = n1 - tnumele
    _, n3 = count(ferm3)
    bisec3 = n3 - tnumele
    lbisec = 0
    f, ferm = None, ferm1
    while lbisec < 100:
        lbisec += 1
        ferm = (ferm1 + ferm3) * 0.5
        f, n0 = count(ferm)
        bisec = n0 - tnumele
        if abs(bisec) < 1.0e-12:
            lbisec = 100
        if bisec1 * bisec > 0.0:
            ferm1, bisec1 = ferm, bisec
        if bisec * bisec3 > 0.0:
            ferm3, bisec3 = ferm, bisec
    return f, ferm


def smooth_start_bands_device(shape, M: int, seed: int, dtype=torch.float64):
    """The same kind of start as smooth_start_bands, generated on the device
    (seeded normal bands, the same Gaussian low-pass filter), for large cells."""
    nx, ny, nz = shape
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    kz, ky, kx = torch.meshgrid(torch.fft.fftfreq(nz, device="cuda"),
                                torch.fft.fftfreq(ny, device="cuda"),
                                torch.fft.fftfreq(nx, device="cuda"), indexing="ij")
    filt = torch.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / 0.005)
    out = torch.empty((M, nx * ny * nz), dtype=dtype, device="cuda")
    for b0 in range(0, M, 64):
        x = torch.randn((min(64, M - b0), nz, ny, nx), generator=gen, device="cuda",
                        dtype=torch.float64)
        x = torch.fft.ifftn(torch.fft.fftn(x, dim=(1, 2, 3)) * filt, dim=(1, 2, 3)).real
        out[b0:b0 + x.shape[0]] = x.reshape(x.shape[0], -1).to(dtype)
    return out


@dataclass
class ScfResult:
    converged: bool
    iterations: int
    seconds: float
    diff: list = field(default_factory=list)      # diff_charge per iteration
    seconds_per_iter: list = field(default_factory=list)
    sval: np.ndarray | None = None                 # eigenvalues (Ha), ascending
    eband: float = 0.0                             # sum_l f_l e_l (Ha)
    fermi: float = 0.0                             # Fermi level (Ha), smearing only
    hartree_iters: list = field(default_factory=list)
    phase_seconds: dict = field(default_factory=dict)  # with profile=True only
    energy: dict = field(default_factory=dict)    # output_energy's terms (Ha)
    energies: list = field(default_factory=list)  # free energy per iteration (when tracked)
    occ: np.ndarray | None = None                  # final occupations


def helmholtz_entropy(occ, tf: float) -> float:
    """eneth of totalenergy_eig (totalenergy8f.F90:166-196), one k-point and
    spin (tmpfac = 1/2): tf sum_l (f ln f + (1-f) ln(1-f)) / tmpfac, with
    f = occ/2 and the logarithms dropped below 1e-8."""
    tmpfac = 0.5
    e = 0.0
    for o in np.asarray(occ, dtype=np.float64):
        t = o * tmpfac
        t1 = np.log(t) if t > 1.0e-8 else 0.0
        t2 = np.log(1.0 - t) if 1.0 - t > 1.0e-8 else 0.0
        e = e + (t * t1 + (1.0 - t) * t2) / tmpfac
    return float(e * tf)


def run_scf(cell: Cell, M: int, nocc: int, dtype=torch.float64, eps_scf: float = 1e-6,
            looplimit: int = 200, prm=None, nbrydn: int = 20, eta: float = 0.02,
            seed: int = 0, zval: float = 4.0, epsvh: float = 1e-12, vloc=None, rho0=None,
            psi0=None, log=None, profile: bool = False, smearing: bool = True,
            tf: float = 3.0e-3, restart_dir: str | None = None,
            save_dir: str | None = None, potential: str = "kukan",
            polish: bool = True, start: str = "kukan",
            eps_energy: float | None = None) -> ScfResult:
    """kukan's SCF loop (kukan8f.F90:466-762) over the C ABI.

    potential: "kukan" (the dataset's local pseudopotential, setup_initialwave
    start) or "model" (Gaussian wells and charges per atom, smooth random
    start bands); vloc / rho0 / psi0 override the local potential, the start
    density and the start bands.
    restart_dir: start from kukan restart files there (wfc.00000.000 for the
    bands, rho.00000 for the start density, vht.00000 for the Hartree warm
    start).
    save_dir: write the same files after the last iteration (the last input
    density as rho.*, the output density as r_o.*), as write_wf and
    write_rhovht do.
    polish: on the mixed path, finish with one FP64 orthonormalisation and
    Rayleigh-Ritz step of the converged bands (its time is part of the
    loop's), so that eigenvalues and energies are FP64 quantities.
    eps_energy: when given (Ha/atom), the loop also waits until the free
    energy changed by less than eps_energy per atom over the last iteration
    (kukan stops on diff_charge alone).
    start: "kukan" (setup_initialwave's s and p orbitals) or "random" (seeded
    smooth random bands, `seed`); the start density is the density of the
    start bands either way.  RR + DIIS from the first iteration needs a start
    whose span reaches the lowest states: with fewer bands than four per atom
    kukan's orbitals leave out the p orbitals of the later atoms, and DIIS
    then settles on high states (measured on Si512, 1100 bands)."""
    dev = torch.device("cuda")
    # the loop runs on a stream of its own (launches are stream-ordered there
    # and the Hartree solve can replay its iteration batches as CUDA graphs)
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    with torch.cuda.stream(side):
        res = _run_scf(cell, M, nocc, dtype, eps_scf, looplimit, prm, nbrydn, eta, seed, zval,
                       epsvh, vloc, rho0, psi0, log, profile, smearing, tf, restart_dir,
                       save_dir, dev, potential, polish, start, eps_energy)
    side.synchronize()
    return res


def _run_scf(cell, M, nocc, dtype, eps_scf, looplimit, prm, nbrydn, eta, seed, zval, epsvh,
             vloc, rho0, psi0, log, profile, smearing, tf, restart_dir, save_dir, dev,
             potential, polish, start, eps_energy):
    from . import pseudo as PP
    if potential not in ("kukan", "model"):
        raise ValueError(f"potential must be 'kukan' or 'model', not {potential!r}")
    g = K.Geometry(cell)
    N, shape = cell.N, cell.shape
    dshape = tuple(2 * s for s in shape)
    h, xmax = cell.h, cell.xmax
    dvol = h[0] * h[1] * h[2]
    f64 = torch.float64
    rho_start = vh_start = None
    if restart_dir is not None:
        psi = torch.empty((M, N), dtype=dtype, device=dev)
        CK.read_wf(restart_dir, M, shape, out=psi)
        got = CK.read_rho(restart_dir, shape)
        rho_start = None if got is None else got[0]
        vh_start = CK.read_vht(restart_dir, shape)
    elif psi0 is not None:
        if torch.is_tensor(psi0):
            psi = psi0.to(device=dev, dtype=dtype).contiguous()
        else:
            psi = torch.as_tensor(np.ascontiguousarray(psi0), device=dev).to(dtype)
    elif potential == "kukan" and start == "kukan":
        psi = PP.initial_bands(cell, M, dtype)
    else:
        psi = smooth_start_bands_device(shape, M, seed, dtype)
    sss = None if cell.sss is None else torch.tensor(cell.sss, dtype=f64, device=dev)
    b = K.Bands(g, psi, sss)
    K.orthogonalization(b, 1)
    # kukan's first occupations: scf_occupation of the initial all-zero
    # eigenvalues (equal occupations) with smearing, the lowest nocc bands
    # otherwise
    occ = torch.zeros(M, dtype=f64, device=dev)
    if smearing:
        occ.copy_(torch.from_numpy(scf_occupation(np.zeros(M), 2.0 * nocc, tf)[0]))
    else:
        occ[:nocc] = 2.0
    if vloc is not None:
        vloc_t = torch.as_tensor(np.ascontiguousarray(vloc), dtype=f64, device=dev)
    elif potential == "kukan":
        vloc_t = PP.local_potential(cell)[0]
    else:
        vloc_t = torch.tensor(model_local_potential(cell), dtype=f64, device=dev)
    if rho_start is not None:
        rho0 = rho_start
    if rho0 is not None:
        rho_o = torch.as_tensor(np.ascontiguousarray(rho0), dtype=f64, device=dev)
    elif potential == "kukan":
        rho_o = K.scf_charge_smt(occ, b.psi, N)
    else:
        rho_o = torch.tensor(atomic_density(cell, zval), dtype=f64, device=dev)
    rho_i = torch.zeros(N, dtype=f64, device=dev)
    vh_d = torch.zeros(8 * N, dtype=f64, device=dev)
    if vh_start is not None:
        vh_d.copy_(torch.from_numpy(vh_start))
    veff64 = torch.empty(N, dtype=f64, device=dev)
    veff32 = torch.empty(N, dtype=torch.float32, device=dev) if dtype == torch.float32 else None
    veff = veff64 if veff32 is None else veff32
    dij = torch.tensor(cell.dij, dtype=f64, device=dev)
    prm = prm or L.solver_prm()
    mixer = K.Mixer(N, nbrydn, eta)
    res = ScfResult(False, 0, 0.0)

    def mark(name, t):
        # per-phase wall time (synchronising), only when profiling
        if not profile:
            return t
        torch.cuda.synchronize()
        now = time.perf_counter()
        res.phase_seconds[name] = res.phase_seconds.get(name, 0.0) + now - t
        return now

    eneat = PP.ion_energy(cell) if potential == "kukan" else 0.0
    ddv = dvol / 8.0

    def energy(occ_h, sval, rho_i, rho_d, vh_d, vx, ex_d):
        # totalenergy_space / totalenergy_eig on an input density and its
        # potentials (output8f.F90:240-242)
        eneel = float(np.cumsum(occ_h * sval)[-1])
        eneha = -0.5 * float(K.dot(vh_d, rho_d).item()) * ddv
        eneex = -float(K.dot(rho_i, vx).item()) * dvol + float(K.dot(rho_d, ex_d).item()) * ddv
        eneth = helmholtz_entropy(occ_h, tf) if smearing else 0.0
        etot = eneel + eneex + eneha + eneat
        return dict(eneel=eneel, eneex=eneex, eneha=eneha, eneat=eneat, eneth=eneth,
                    total=etot, free=etot + eneth)

    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rho_d = vx = ex_d = None
    e_prev = None
    for iscf in range(1, looplimit + 1):
        ti = time.perf_counter()
        tp = ti
        mixer.step(rho_o, rho_i, dvol)
        tp = mark("mixing", tp)
        rho_d = K.trans_c2d_smtcharge(shape, 4, rho_i)
        it, _ = K.scf_hartree(dshape, 4, xmax, rho_d, vh_d, epsvh,
                              mixed=dtype == torch.float32)
        tp = mark("hartree", tp)
        vh = K.trans_d2c(shape, 4, vh_d)
        vx_d, ex_d = K.vxpot_lda_pz(rho_d)
        vx = K.trans_d2c(shape, 4, vx_d)
        K.veff_sum(vx, vloc_t, vh, veff64, veff32)
        tp = mark("xc+transfer", tp)
        K.scf_diag(b, veff, dij, iscf, prm)
        tp = mark("scf_diag", tp)
        if smearing:
            fn, res.fermi = scf_occupation(b.sval, 2.0 * nocc, tf)
            occ.copy_(torch.from_numpy(fn))
        rho_o = K.scf_charge_smt(occ, b.psi, N)
        diff = K.scf_diffcharge(rho_o, rho_i, h, xmax)
        tp = mark("charge", tp)
        res.diff.append(diff)
        res.hartree_iters.append(it)
        res.seconds_per_iter.append(time.perf_counter() - ti)
        res.iterations = iscf
        e_now = None
        if log or eps_energy is not None:
            e_now = energy(occ.cpu().numpy(), np.asarray(b.sval), rho_i, rho_d, vh_d, vx,
                           ex_d)["free"]
            res.energies.append(e_now)
        if log:
            log(f"iscf {iscf:3d}  diff_charge {diff:.3e}  hartree_cg {it}  free energy "
                f"{e_now:.8f}  {res.seconds_per_iter[-1]:.3f} s")
        e_ok = eps_energy is None or (e_prev is not None and
                                      abs(e_now - e_prev) < eps_energy * cell.natom)
        e_prev = e_now
        if diff < eps_scf and e_ok:
            res.converged = True
            break
    if polish and dtype == torch.float32:
        # FP64 polish of the mixed path: the converged FP32 bands in FP64,
        # S-orthonormalised and rotated by one FP64 Rayleigh-Ritz step with
        # the last effective potential, so that the eigenvalue sums carry no
        # FP32 rounding of H psi or of the tensor-core Gram products
        b64 = K.Bands(g, b.psi.double(), sss)
        K.orthogonalization(b64, 1)
        K.rayleighritz(b64, veff64, dij, 1)
        K.reorderstates(b64)
        b = b64
        if smearing:
            fn, res.fermi = scf_occupation(b.sval, 2.0 * nocc, tf)
            occ.copy_(torch.from_numpy(fn))
        rho_o = K.scf_charge_smt(occ, b.psi, N)
        tp = mark("fp64_polish", tp)
    torch.cuda.synchronize()
    res.seconds = time.perf_counter() - t0
    res.sval = np.array(b.sval)
    occ_h = occ.cpu().numpy()
    res.occ = occ_h
    res.eband = float(np.cumsum(occ_h * res.sval)[-1])
    res.energy = energy(occ_h, res.sval, rho_i, rho_d, vh_d, vx, ex_d)
    if save_dir is not None:
        CK.write_wf(save_dir, b.psi, res.sval, shape)
        CK.write_rho(save_dir, rho_i, shape)
        CK.write_rho(save_dir, rho_o, shape, name="r_o")
        CK.write_vht(save_dir, vh_d, shape)
    res.bands = b
    res.rho_out = rho_o
    mixer.close()
    return res
