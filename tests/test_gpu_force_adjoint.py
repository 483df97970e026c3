"""Atomic forces by the adjoint pass (rspacedist_b200.forces).

* The local part equals the oracle's sums of the same gradients (C8 with the
  NC carbon dataset, 20^3).
* Si8 with the PAW dataset (S != 1), atoms displaced by sigma = 0.10 bohr
  (seed 3), 32^3 (h = 0.32 bohr, the spacing of the Si64 and Si512 cells),
  after an FP64 SCF to diff_charge < 1e-8:
  - the total force equals minus the central difference of the SCF free
    energy over +-1e-3 bohr on three atom-axis components within 3e-4
    Ha/bohr.  The discrete energy is not smooth below that: kukan's hard
    local part ends at 1.05 r_c where its filter still weighs about 0.5 %,
    the projector tables end at r_c, and both tables are piecewise-linear in
    r, so grid points crossing these edges add steps to E(R).  Measured:
    0.9e-4 to 1.8e-4;
  - the projector part and force_eig_r (finite-difference derivatives of
    the bands, rs_force_nl_f64) approach each other as the grid is refined,
    as the discretisation error of force_eig_r shrinks (about h^4: 1.0e-2 at
    32^3, 2.1e-3 at 48^3);
  - the mixed path (FP32 bands, SCF to 1e-7) gives the FP64 forces within
    1e-4 Ha/bohr."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

STEP = 1e-3


def _si8(n, atoms=None):
    from rspacedist_b200 import system as S
    pos = S.diamond_positions(1, 10.26, 0.10, 3) if atoms is None else atoms
    return S.make_cell(10.26, n, pos, S.load_dataset("si_paw"))


def _scf(cell, dtype=torch.float64, eps=1e-8):
    from rspacedist_b200 import lib, scf
    r = scf.run_scf(cell, 20, 16, dtype=dtype, prm=lib.solver_prm(ncgscf=200), eta=0.1,
                    eps_scf=eps, looplimit=300)
    assert r.converged, r.diff[-5:]
    return r


@pytest.fixture(scope="module")
def si8(built_lib, cuda):
    from rspacedist_b200 import forces
    cell = _si8(32)
    r = _scf(cell)
    return cell, r, forces.atomic_forces(cell, r)


def test_local_forces_match_oracle(oracle, built_lib, cuda):
    import oracle_pp as OP
    from rspacedist_b200 import forces, system as S
    cell = S.make_cell(6.74, 20, S.diamond_positions(1, 6.74, 0.10, 3), S.load_dataset("c_ncps"))
    rng = np.random.default_rng(4)
    rho = np.abs(rng.standard_normal(cell.N)) * 0.05
    fl = forces.local_forces(cell, torch.tensor(rho, device="cuda"))
    rho_d = oracle.interp_c2d(cell.shape, 4, rho)
    rho_s = oracle.interp_d2c(cell.shape, 4, rho_d)
    cp1, a, b, c, rcut, coef, nqct, rcuts = OP.local_setup(oracle, cell.ds, cell.h)
    _, g = oracle.vloc_soft(cell.atoms, cp1, a, b, c, rcut, cell.shape, cell.h, cell.xmax,
                            OP.VETA, (OP.NPW,) * 3, grad=True)
    f_soft = np.einsum("kap,p->ak", g, rho_s) * cell.dvol
    f_hard = oracle.vloc_hard(cell.atoms, cell.nmax, 2, cell.h, cell.xmax, cell.npmax, rcut,
                              OP.PSCTOFF, rcuts, nqct, coef, OP.FILPP, OP.EPS, OP.NFILTYP,
                              rho_dense=rho_d)
    ref = f_soft + f_hard
    assert np.abs(fl - ref).max() <= 1e-9 * max(1.0, np.abs(ref).max())


def test_forces_match_energy_differences(si8):
    cell, r, f = si8
    for a, ax in ((0, 0), (2, 1), (5, 2)):
        es = []
        for s in (1, -1):
            at = cell.atoms.copy()
            at[a, ax] += s * STEP
            es.append(_scf(_si8(32, at)).energy["free"])
        fd = -(es[0] - es[1]) / (2 * STEP)
        assert abs(f["total"][a, ax] - fd) <= 3e-4, (a, ax, f["total"][a, ax], fd)


def test_projector_forces_converge_to_force_eig(si8):
    from rspacedist_b200 import forces, kukan as K

    def gap(cell, r, fp):
        g = K.Geometry(cell)
        dij = torch.tensor(cell.dij, dtype=torch.float64, device="cuda")
        sss = torch.tensor(cell.sss, dtype=torch.float64, device="cuda")
        fe = K.force_eig(g, dij, sss, r.bands.psi, torch.tensor(r.sval, device="cuda"),
                         torch.tensor(r.occ, device="cuda")).cpu().numpy()
        return float(np.abs(fp - fe).max())

    cell, r, f = si8
    g32 = gap(cell, r, f["projector"])
    cell48 = _si8(48)
    r48 = _scf(cell48)
    g48 = gap(cell48, r48, forces.atomic_forces(cell48, r48)["projector"])
    assert g48 < 0.35 * g32 and g48 < 5e-3, (g32, g48)


def test_mixed_path_forces(si8):
    from rspacedist_b200 import forces
    cell, r, f = si8
    r32 = _scf(cell, torch.float32, 1e-7)
    f32 = forces.atomic_forces(cell, r32)
    assert np.abs(f32["total"] - f["total"]).max() <= 1e-4
