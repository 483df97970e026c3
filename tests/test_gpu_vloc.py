"""kukan's local pseudopotential, ion-ion energy and initial bands on the GPU
(rspacedist_b200.pseudo over rs_vloc_soft / rs_vloc_hard_add / rs_ewald /
rs_initial_wave_*) against the CPU oracle's restatement of pseudocalc_02-04,
totalenergy_space_03 and setup_initialwave, on a C8 cell (NC dataset) and
an Si8 cell (PAW dataset)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", params=["c8", "si8"])
def cell(request, built_lib, cuda):
    import conftest
    return conftest.make_c8(20) if request.param == "c8" else conftest.make_si8(24, 0.05, 4)


def test_local_potential_matches_oracle(cell, oracle):
    import oracle_pp as OP
    from rspacedist_b200 import pseudo as P
    coarse, dense = P.local_potential(cell)
    ref_c, ref_d, _ = OP.local_potential(oracle, cell)
    scale = np.abs(ref_d).max()
    assert np.abs(dense.cpu().numpy() - ref_d).max() <= 1e-11 * scale
    assert np.abs(coarse.cpu().numpy() - ref_c).max() <= 1e-11 * scale


def test_ewald_energy_and_forces(cell, oracle):
    import oracle_pp as OP
    from rspacedist_b200 import pseudo as P
    e, f = P.ion_energy(cell, forces=True)
    ref = OP.ion_energy(oracle, cell)
    assert abs(e - ref) <= 1e-11 * abs(ref)
    # forces are minus the energy gradient: central differences, 1e-4 bohr
    import copy
    for a, ax in ((0, 0), (3, 1), (5, 2)):
        c2 = copy.copy(cell)
        step = 1e-4
        es = []
        for s in (1, -1):
            at = cell.atoms.copy()
            at[a, ax] += s * step
            c2.atoms = at
            es.append(P.ion_energy(c2))
        fd = -(es[0] - es[1]) / (2 * step)
        assert abs(f[a, ax] - fd) <= 1e-6, (a, ax, f[a, ax], fd)
    # the ions of a cell sum to zero force
    assert np.abs(f.sum(axis=0)).max() <= 1e-10 * max(1.0, np.abs(f).max())


def test_initial_bands_match_oracle(cell, oracle):
    from rspacedist_b200 import pseudo as P
    M = 5 * cell.natom  # s and p of every atom, then d forms of the first ones
    cp1 = P.local_params(cell.ds)[0]
    ref = oracle.initial_wave(cell.atoms, cp1, P.ZS_PRE, M, cell.shape, cell.h, cell.xmax)
    got = P.initial_bands(cell, M, torch.float64).cpu().numpy()
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    g32 = P.initial_bands(cell, M, torch.float32).cpu().numpy()
    np.testing.assert_allclose(g32, ref, rtol=0, atol=1e-6 * np.abs(ref).max())
