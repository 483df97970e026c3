"""kukan's SCF on the GPU (rspacedist_b200.scf: the dataset's local
pseudopotential, setup_initialwave start, Broyden mixing, Hartree CG, PZ LDA,
scf_diag, Fermi-Dirac occupations) against the same loop on the CPU oracle
(tests/oracle_scf.py), C8 diamond with the NC carbon dataset, 20 bands, 16
occupied, kukan's all-CG band solver, Broyden mixing with eta 0.1.  The plain
FP64 path and the mixed path (FP32 bands) both converge
to diff_charge < 1e-6; their total energy is within 1e-6 Ha/atom of the
oracle's and their occupied eigenvalues within 1e-5 Ha (the bounds the
mixed path is built to)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref(built_lib, oracle, cuda):
    import conftest
    import oracle_scf
    cell = conftest.make_c8(20)
    return cell, oracle_scf.oracle_scf(oracle, cell, 20, 16, eta=0.1, ncgscf=200)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_scf_matches_oracle(ref, dtype):
    from rspacedist_b200 import lib, scf
    cell, r = ref
    assert r["converged"]
    res = scf.run_scf(cell, 20, 16, dtype=dtype, prm=lib.solver_prm(ncgscf=200), looplimit=100,
                      eta=0.1)
    assert res.converged, res.diff[-5:]
    np.testing.assert_allclose(np.sort(res.sval)[:16], r["sval"][:16], atol=1e-5)
    for key in ("total", "free", "eneel", "eneha", "eneex"):
        assert abs(res.energy[key] - r["energy"][key]) / cell.natom < 1e-6, key
    assert abs(res.energy["eneat"] - r["energy"]["eneat"]) < 1e-9 * abs(r["energy"]["eneat"])


def test_scf_restart_files(ref, tmp_path):
    """A converged run writes kukan's restart files (wfc, rho, r_o, vht); a
    run restarted from them starts converged: its first charge difference is
    already below the stopping rule, and its eigenvalues match."""
    from rspacedist_b200 import checkpoint as CK, lib, scf
    cell, r = ref
    prm = lib.solver_prm(ncgscf=200)
    a = scf.run_scf(cell, 20, 16, dtype=torch.float64, prm=prm, looplimit=100, eta=0.1,
                    save_dir=str(tmp_path))
    assert a.converged
    for name in ("wfc.00000.000", "rho.00000", "r_o.00000", "vht.00000"):
        assert (tmp_path / name).exists(), name
    sv, _ = CK.read_wf(str(tmp_path), 20, cell.shape)
    assert np.array_equal(sv, a.sval)
    b = scf.run_scf(cell, 20, 16, dtype=torch.float64, prm=lib.solver_prm(ncgscf=0),
                    looplimit=3, restart_dir=str(tmp_path))
    assert b.diff[0] < 1e-5, b.diff
    np.testing.assert_allclose(np.sort(b.sval)[:16], np.sort(a.sval)[:16], atol=1e-6)
