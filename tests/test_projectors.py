"""Projector-table generation (pseudocalc_01a double-grid weights and
pseudocalc_07 Fourier-filtered projectors with the double-grid contraction).

CPU: the oracle is pinned by known answers -- the weights reproduce
polynomials of degree < 2 nfdg, and the Bessel sums of analytic Fourier-Bessel
coefficients give back r^l exp(-r^2/2s^2) Y_lm dV -- and the library's host
weights equal the oracle's.  GPU: rs_projector_tables against the oracle on
Si8 and C8 cells with npmesh 1, 2 and 3.
"""
import numpy as np
import pytest

from conftest import make_c8, make_si8

LM = [(0, 0), (1, 0), (1, 1), (1, 2), (2, 0), (2, 1), (2, 2), (2, 3), (2, 4)]
COL = [1, 3, 3, 3, 5, 5, 5, 5, 5]
YM = [1, 2, 3, 4, 5, 6, 7, 8, 9]


def _gauss_case(oracle, npmesh, sig=0.6):
    """One atom off the grid points, analytic coefficients of r^l exp(-r^2/2s^2):
    4 pi int r^(l+2) exp(-r^2/2s^2) j_l(qr) dr = (2 pi)^(3/2) s^(2l+3) q^l exp(-q^2 s^2/2)."""
    h, nmax = (0.25, 0.25, 0.25), (12, 12, 12)
    atoms = np.array([[0.113, -0.071, 0.052]])
    rcut, psctoff, psftrad = 2.6, 1.05, 20.0
    npx = int(rcut * psctoff / h[0]) + 1 + 4
    npmax = (npx,) * 3
    num_list = (2 * npx) ** 3
    st, L = oracle.sphere_lists(atoms, rcut * psctoff, nmax, h, npmax, 4, num_list)
    assert st == 0
    nqct = 200
    q = np.pi / (rcut * psftrad) * np.arange(nqct + 1)
    coef = np.zeros((8, nqct + 1))
    for l, col in ((0, 1), (1, 3), (2, 5)):
        coef[col] = (2 * np.pi) ** 1.5 * sig ** (2 * l + 3) * q ** l * np.exp(-q * q * sig * sig / 2)
    w = oracle.dg_weights(4, npmesh)
    v = oracle.projector_tables(atoms, L, nmax, h, npmax, 4, npmesh, num_list, COL, YM,
                                coef.ravel(), nqct, nqct, rcut, psftrad, psctoff, 1e-16, 2, 0.02, w)
    n = int(L["natinf"][0])
    x = L["lstx"][:n] * h[0] - (atoms[0, 0] - (L["natx"][0] * h[0] - 0.5 * h[0]))
    y = L["lsty"][:n] * h[1] - (atoms[0, 1] - (L["naty"][0] * h[1] - 0.5 * h[1]))
    z = L["lstz"][:n] * h[2] - (atoms[0, 2] - (L["natz"][0] * h[2] - 0.5 * h[2]))
    r = np.sqrt(x * x + y * y + z * z)
    return v[0, :, :n], x, y, z, r, r < rcut * psctoff, np.prod(h), sig


def test_dg_weights_reproduce_polynomials(oracle, built_lib):
    from rspacedist_b200 import projectors as PR
    for nfdg in (1, 2, 3, 4):
        for npm in (1, 2, 3, 4):
            w = oracle.dg_weights(nfdg, npm)
            assert np.array_equal(w, PR.double_grid_weights(nfdg, npm))
            n = nfdg * npm
            odd = npm % 2 == 1
            js, t1 = (-n + 1, 0.0) if odd else (-n, 0.5)
            for j0 in range(npm):
                u = (j0 + t1) / npm  # fine point, in coarse spacings from node 0
                for k in range(2 * nfdg):
                    acc = sum(w[j0 - c * npm + n] * float(c) ** k
                              for c in range(-3 * nfdg, 3 * nfdg) if js <= j0 - c * npm <= n - 1)
                    assert abs(acc - u ** k) <= 1e-13 * max(1.0, u ** k)


def test_bessel_sums_give_back_the_radial_function(oracle):
    from rspacedist_b200 import system as S
    v, x, y, z, r, inside, dv, sig = _gauss_case(oracle, 1)
    for la, (l, m) in enumerate(LM):
        ref = np.where(inside, r ** l * np.exp(-r * r / (2 * sig * sig)) *
                       S._real_ylm(l, x, y, z, r)[m] * dv, 0.0)
        np.testing.assert_allclose(v[la], ref, atol=1e-9 * np.abs(ref).max())


@pytest.mark.parametrize("npmesh", [2, 3])
def test_double_grid_contraction_is_close_to_point_values(oracle, npmesh):
    """With a fine mesh the contracted value of a smooth projector stays
    within the interpolation error (~1e-4 relative) of its point value."""
    from rspacedist_b200 import system as S
    v, x, y, z, r, inside, dv, sig = _gauss_case(oracle, npmesh)
    for la in (0, 1, 6):
        l, m = LM[la]
        ref = np.where(inside, r ** l * np.exp(-r * r / (2 * sig * sig)) *
                       S._real_ylm(l, x, y, z, r)[m] * dv, 0.0)
        np.testing.assert_allclose(v[la], ref, atol=1e-3 * np.abs(ref).max())


def test_channel_table_and_coefficients(built_lib):
    from rspacedist_b200 import projectors as PR, system as S
    ds = S.load_dataset("si_paw")
    col, ym = PR.channel_table(ds)
    # the nprj = 12 case of pseudocalc_07: s, p, p', d
    assert col.tolist() == [1, 3, 3, 3, 4, 4, 4, 5, 5, 5, 5, 5]
    assert ym.tolist() == [1, 2, 3, 4, 2, 3, 4, 5, 6, 7, 8, 9]
    coef, nqct, nqmx = PR.bessel_coefs(ds, (0.32, 0.32, 0.32))
    assert nqct == int(ds["rcut"] * PR.PSFTRAD / 0.32)
    c = coef.reshape(8, nqmx + 1)
    assert np.all(c[[0, 2, 6, 7]] == 0.0)
    assert np.all(c[[3, 4, 5], 0] == 0.0)  # j_l(0) = 0 for l > 0


def test_channel_table_of_the_nc_carbon_dataset(built_lib):
    """The 4-projector case of pseudocalc_07 (s, p): columns 1, 3, 3, 3."""
    from rspacedist_b200 import projectors as PR, system as S
    col, ym = PR.channel_table(S.load_dataset("c_ncps"))
    assert col.tolist() == [1, 3, 3, 3]
    assert ym.tolist() == [1, 2, 3, 4]


def test_dg_weights_higher_orders_match_the_library(oracle, built_lib):
    from rspacedist_b200 import projectors as PR
    for nfdg in (5, 6):
        for npm in (1, 2, 3):
            assert np.array_equal(oracle.dg_weights(nfdg, npm), PR.double_grid_weights(nfdg, npm))


def _tables_case(cell, oracle, npmesh):
    from rspacedist_b200 import projectors as PR
    ds = cell.ds
    coef, nqct, nqmx = PR.bessel_coefs(ds, cell.h)
    col, ym = PR.channel_table(ds)
    lists = dict(natx=cell.natxyz[0], naty=cell.natxyz[1], natz=cell.natxyz[2],
                 natinf=cell.natinf, lstx=cell.lstxyz[0], lsty=cell.lstxyz[1],
                 lstz=cell.lstxyz[2])
    ref = oracle.projector_tables(cell.atoms, lists, cell.nmax, cell.h, cell.npmax, 4, npmesh,
                                  cell.num_list, col, ym, coef, nqct, nqmx, ds["rcut"], PR.PSFTRAD,
                                  PR.PSCTOFF, PR.EPS, PR.NFILTYP, PR.FILPP,
                                  oracle.dg_weights(4, npmesh))
    return ref


def test_filtered_tables_track_the_sampled_projectors(oracle, built_lib):
    """The Fermi-filtered projectors of the Si dataset, cut at the grid's
    Nyquist wave number, stay close to the radial functions sampled directly
    at the coarse points (a check of the coefficient transform and of the
    table layout, not of parity)."""
    cell = make_si8()
    ref = _tables_case(cell, oracle, 1)
    got = cell.vnlocp
    for la in range(ref.shape[1]):
        a, b = ref[:, la].ravel(), got[:, la].ravel()
        assert np.linalg.norm(a - b) < 0.1 * np.linalg.norm(b)
        assert a @ b > 0.99 * np.linalg.norm(a) * np.linalg.norm(b)


@pytest.mark.gpu
@pytest.mark.parametrize("which,npmesh", [("si8", 2), ("si8", 3), ("c8", 1), ("c8", 2)])
def test_projector_tables_gpu_match_oracle(oracle, cuda, which, npmesh):
    from rspacedist_b200 import projectors as PR
    cell = make_si8(sigma=0.02, seed=3) if which == "si8" else make_c8()
    ref = _tables_case(cell, oracle, npmesh)
    got = PR.projector_tables(cell, npmesh=npmesh)
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * np.abs(ref).max())
    assert np.abs(ref).max() > 0
    import torch
    dev = torch.full(got.shape, np.nan, dtype=torch.float64, device="cuda")
    PR.projector_tables(cell, npmesh=npmesh, out=dev)
    torch.cuda.synchronize()
    assert np.array_equal(dev.cpu().numpy(), got)


@pytest.mark.gpu
def test_filtered_tables_drive_the_fp64_hpsi(oracle, cuda):
    """A cell built with the filtered tables (make_cell(filtered=True)) runs the
    hot path like any other: FP64 H psi on the GPU equals the oracle's bits."""
    import torch
    from rspacedist_b200 import kukan as K, system as S
    ds = S.load_dataset("si_paw")
    cell = S.make_cell(10.26, 32, S.diamond_positions(1, 10.26, 0.02, 6), ds, filtered=True)
    g = K.Geometry(cell)
    veff = S.smooth_veff(cell, 3)
    psi = S.random_bands(cell, 3, 8)
    geo = dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
               natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())
    sysk = oracle.make_sys(geo, cell.shape, 4, cell.h, veff, cell.dij, cell.sss)
    rp = oracle.nl_dot(geo, psi, cell.N)
    ref = oracle.hpsi(sysk, psi, rp)
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device="cuda")
    out = K.hpsi(g, t(veff), t(cell.dij), K.nonlocaloperation_01(g, t(psi)), t(psi))
    assert np.array_equal(out.cpu().numpy(), ref)
    g.close()
