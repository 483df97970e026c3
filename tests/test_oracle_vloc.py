"""The oracle's local pseudopotential and Ewald energy against known
answers (no GPU): the soft part of tools_bisec matches -Z/r in value and
slope at r_c; the Ewald energy of one ion per simple-cubic cell on a uniform
background is the Madelung energy -1.4186487397 Z^2/a for every splitting
parameter; the soft local potential does not depend on the splitting
parameter; the package's host-side set-up scalars equal the oracle's."""
import numpy as np
import pytest


def test_bisec_matches_coulomb_tail(oracle):
    for z, rc in ((4.0, 1.19444052466403), (4.0, 2.14043960083515), (1.0, 0.7)):
        a, b, c = oracle.bisec(z, rc)
        assert abs(b * np.cos(a * rc) + c + z / rc) < 1e-12 * z / rc
        assert abs(-b * a * np.sin(a * rc) - z / rc ** 2) < 1e-9 * z / rc ** 2


@pytest.mark.parametrize("veta", [0.2, 0.35, 0.6])
def test_ewald_madelung_simple_cubic(oracle, veta):
    a = 5.0
    e = oracle.ewald(np.zeros((1, 3)), 1.0, (a / 2,) * 3, veta, (11,) * 3, (11,) * 3)
    assert abs(e * a + 1.4186487397403) < 1e-11


def test_ewald_extensive(oracle):
    from rspacedist_b200 import system as S
    a = 6.74
    e8 = oracle.ewald(S.diamond_positions(1, a), 4.0, (a / 2,) * 3, 0.2, (11,) * 3, (11,) * 3)
    e64 = oracle.ewald(S.diamond_positions(2, a), 4.0, (a,) * 3, 0.2, (11,) * 3, (11,) * 3)
    assert abs(e64 / 8 - e8) < 1e-10 * abs(e8)


def test_soft_local_part_independent_of_splitting(oracle):
    from rspacedist_b200 import system as S
    ds = S.load_dataset("c_ncps")
    n, a0 = 12, 6.74
    h = (a0 / n,) * 3
    atoms = S.diamond_positions(1, a0, 0.03, 2)
    rc = ds["mesh_r"][ds["nradct"] - 1]
    a, b, c = oracle.bisec(4.0, rc)
    v1 = oracle.vloc_soft(atoms, 4.0, a, b, c, rc, (n,) * 3, h, (a0 / 2,) * 3, 0.2, (11,) * 3)
    v2 = oracle.vloc_soft(atoms, 4.0, a, b, c, rc, (n,) * 3, h, (a0 / 2,) * 3, 0.3, (11,) * 3)
    assert np.abs(v1 - v2).max() < 1e-12 * np.abs(v1).max()


def test_host_setup_equals_oracle(oracle):
    import oracle_pp as OP
    from rspacedist_b200 import pseudo as P, system as S
    ds = S.load_dataset("c_ncps")
    h = (6.74 / 20,) * 3
    cp1, a, b, c, rcut = P.local_params(ds)
    ref = OP.local_setup(oracle, ds, h)
    assert (cp1, a, b, c, rcut) == tuple(ref[:5])
    coef, nqct, rcuts = P.local_coefs(ds, h, potc=np.asarray(ds["mesh_potc"]))
    assert nqct == ref[6] and rcuts == ref[7]
    np.testing.assert_allclose(coef, ref[5], rtol=0, atol=1e-12 * np.abs(ref[5]).max())
