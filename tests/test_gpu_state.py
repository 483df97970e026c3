"""The device-resident state handle (rs_create ... rs_destroy) against the
functional entry points it composes: the same orthogonalisation, two
scf_diag steps and the density give the same bits on both paths."""
import numpy as np
import pytest
import torch

from conftest import make_si8

pytestmark = pytest.mark.gpu


def T(a, d=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=d, device="cuda")


@pytest.mark.parametrize("precision", [32, 64])
def test_state_handle_matches_functional_calls(cuda, built_lib, precision):
    from rspacedist_b200 import kukan as K, lib, system as S
    cell = make_si8(sigma=0.02, seed=5)
    M = 10
    dtype = torch.float32 if precision == 32 else torch.float64
    veff = S.smooth_veff(cell, 2)
    psi = S.random_bands(cell, M, 4).astype(np.float32 if precision == 32 else np.float64)
    prm = lib.solver_prm()
    occ = np.array([2.0] * 6 + [1.0, 0.5, 0.0, 0.0])

    st = K.State(cell, M, precision)
    st.set_potential(veff)
    st.upload_bands(psi)
    st.orthogonalize(1)
    for iscf in (1, 2):
        st.diag_step(iscf, prm)
    psi_s, sval_s, rho_s = st.download_bands(), st.sval.copy(), st.density(occ)
    st.close()

    g = K.Geometry(cell)
    b = K.Bands(g, T(psi, dtype), T(cell.sss))
    K.orthogonalization(b, 1)
    v = T(veff, dtype)
    for iscf in (1, 2):
        K.scf_diag(b, v, T(cell.dij), iscf, prm)
    rho_f = K.scf_charge_smt(T(occ), b.psi, cell.N).cpu().numpy()
    assert np.array_equal(psi_s, b.psi.cpu().numpy())
    assert np.array_equal(sval_s, b.sval)
    assert np.array_equal(rho_s, rho_f)
    g.close()
