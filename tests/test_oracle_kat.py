"""Pins the CPU oracle against analytic known answers (the reference ships no
tests or outputs): exact FD rationals, plane-wave symbols, the FFT-exact
discrete Poisson solution, interpolation error bounds, dense
diagonalisation, and the band solvers' converged eigenvalues."""
import json
import os
from fractions import Fraction

import numpy as np
import pytest

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_fd_coefficients_are_the_exact_rationals(oracle):
    d = json.load(open(os.path.join(GOLD, "fd_coefs.json")))
    for nf in range(1, 7):
        a = oracle.fdcoef(nf)
        exact = [float(Fraction(x)) for x in d["fd"][str(nf)]]
        assert np.array_equal(a[: nf + 1], np.array(exact))
        # and they are the Fornberg central weights of order 2nf
        fb = [float(Fraction(x)) for x in d["fornberg"][str(nf)]]
        np.testing.assert_allclose(a[: nf + 1], fb, rtol=1e-15, atol=1e-17)


@pytest.mark.parametrize("k", [(0, 0, 0), (1, 0, 0), (3, 2, 1), (5, 4, 6)])
def test_stencil_plane_wave_symbol(oracle, k):
    nx, ny, nz = 16, 12, 14
    h = (0.31, 0.29, 0.33)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    psi = np.cos(2 * np.pi * (k[0] * x / nx + k[1] * y / ny + k[2] * z / nz)).ravel()
    a = oracle.fdcoef(4)
    lam = lambda kk, n, hh: -0.5 / hh ** 2 * (a[0] + 2 * sum(a[m] * np.cos(2 * np.pi * kk * m / n)
                                                           for m in range(1, 5)))
    ev = lam(k[0], nx, h[0]) + lam(k[1], ny, h[1]) + lam(k[2], nz, h[2])
    veff = np.full(nx * ny * nz, 0.25)
    out = oracle.kslaplacian((nx, ny, nz), 4, h, psi, veff)
    np.testing.assert_allclose(out, (ev + 0.25) * psi, atol=1e-12 * max(1, abs(ev)))


def test_hartree_cg_matches_fft_solution(oracle):
    g = np.load(os.path.join(GOLD, "poisson_fft.npz"))
    nx, ny, nz = (int(v) for v in g["shape"])
    h = g["h"]
    xmax = (nx * h[0] / 2, ny * h[1] / 2, nz * h[2] / 2)
    vh, it, dp = oracle.hartree_cg((nx, ny, nz), 4, xmax, 1e-12, 1, 800, 801, g["rho"],
                                   np.zeros(nx * ny * nz))
    assert dp <= 1e-12 and it < 800
    v = vh - vh.mean()
    np.testing.assert_allclose(v, g["v"], atol=1e-10 * np.abs(g["v"]).max())


def test_interpolation_order(oracle):
    g = np.load(os.path.join(GOLD, "interp_trig.npz"))
    shape = tuple(int(v) for v in g["shape"])
    out = oracle.interp_c2d(shape, 4, g["coarse"])
    err = np.abs(out - g["dense"]).max()
    assert err < 5e-3
    # constant and order: weights sum to one
    one = oracle.interp_c2d(shape, 4, np.ones(np.prod(shape)))
    np.testing.assert_allclose(one, 1.0, atol=1e-14)


def test_jacobi_matches_lapack(oracle):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((40, 40))
    a = a + a.T
    st, w, z = oracle.jacobi_eig(a)
    assert st > 0
    np.testing.assert_allclose(w, np.linalg.eigvalsh(a), atol=1e-12)
    np.testing.assert_allclose(z.T @ a @ z, np.diag(w), atol=1e-11)


def test_eig2(oracle):
    rng = np.random.default_rng(4)
    for _ in range(50):
        a = rng.standard_normal((2, 2))
        a = a + a.T
        w, z = oracle.eig2(a)
        np.testing.assert_allclose(w, np.linalg.eigvalsh(a), atol=1e-14)
        np.testing.assert_allclose(a @ z, z * w, atol=1e-13)


def test_reorder_rank_is_stable_sort(oracle):
    s = np.array([0.3, -1.0, 0.3, 2.0, -1.0, 0.0])
    r = oracle.reorder_rank(s)
    assert list(r) == list(np.argsort(np.argsort(s, kind="stable"), kind="stable"))


def test_tree_dot_is_a_dot(oracle):
    rng = np.random.default_rng(5)
    for n in (0, 1, 4095, 4096, 4097, 1 << 20):
        a, b = rng.standard_normal(n), rng.standard_normal(n)
        assert abs(oracle.tree_dot(a, b) - float(a @ b)) <= 1e-12 * (1 + np.abs(a) @ np.abs(b))


def smooth_random(shape, M, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((M, nz, ny, nx))
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(nz), np.fft.fftfreq(ny), np.fft.fftfreq(nx),
                             indexing="ij")
    filt = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / 0.02)
    x = np.real(np.fft.ifftn(np.fft.fftn(x, axes=(1, 2, 3)) * filt, axes=(1, 2, 3)))
    return x.reshape(M, -1)


def _tiny_system(oracle, paw):
    """A 12^3 cell with one or two synthetic projector atoms: small enough to
    build H and S densely from unit vectors."""
    nx = ny = nz = 12
    h = (0.5, 0.5, 0.5)
    N = nx * ny * nz
    st, lists = oracle.sphere_lists(np.array([[0.1, -0.2, 0.3], [-2.0, 1.5, 1.0]]), 1.2,
                                    (6, 6, 6), h, (3, 3, 3), 1, 6 * 6 * 6)
    assert st == 0
    A, P, Lm = 2, 2, 216
    v = np.zeros((A, P, Lm))
    rng = np.random.default_rng(11)
    atoms = np.array([[0.1, -0.2, 0.3], [-2.0, 1.5, 1.0]])
    for a in range(A):
        n = lists["natinf"][a]
        # smooth s- and p_x-like projectors on the list points
        tx = [atoms[a, k] - (lists["nat" + "xyz"[k]][a] * h[k] - 0.5 * h[k]) for k in range(3)]
        x = lists["lstx"][a * Lm:a * Lm + n] * h[0] - tx[0]
        y = lists["lsty"][a * Lm:a * Lm + n] * h[1] - tx[1]
        z = lists["lstz"][a * Lm:a * Lm + n] * h[2] - tx[2]
        g = np.exp(-(x * x + y * y + z * z) / 0.9)
        v[a, 0, :n] = g * 0.125
        v[a, 1, :n] = g * x * 0.125
    geo = dict(natom=A, nprjmx=P, num_list=Lm, nprj=np.full(A, P, np.int32),
               natinf=lists["natinf"], lst=lists["lst"], v=v.ravel())
    D = np.zeros((A, P, P))
    Sm = np.zeros((A, P, P))
    for a in range(A):
        m = rng.standard_normal((P, P))
        D[a] = (m + m.T) * 0.5
        m = rng.standard_normal((P, P)) * 0.2
        Sm[a] = (m + m.T) * 0.5 + 0.3 * np.eye(P)
    veff = rng.standard_normal(N) * 0.3
    sysk = oracle.make_sys(geo, (nx, ny, nz), 4, h, veff, D, Sm if paw else None)
    return sysk, geo, N, h


@pytest.mark.parametrize("paw", [False, True])
def test_band_solvers_reach_dense_eigenvalues(oracle, paw):
    sysk, geo, N, h = _tiny_system(oracle, paw)
    dv = h[0] * h[1] * h[2]
    eye = np.eye(N)
    rp = oracle.nl_dot(geo, eye, N)
    H = oracle.hpsi(sysk, eye, rp).reshape(N, N).T
    S = oracle.spsi(sysk, eye, rp).reshape(N, N).T if paw else np.eye(N)
    import scipy.linalg as sl
    ref = sl.eigh(0.5 * (H + H.T), 0.5 * (S + S.T), eigvals_only=True)[:6]
    M = 8
    # smooth start: the preconditioner (1/2 + 1/12 sum of 6 neighbours) is
    # blind to the (pi,pi,pi) mode, so a white-noise start would keep that
    # component for ever; kukan starts from smooth atomic orbitals
    psi = smooth_random((12, 12, 12), M, 1)
    rp = oracle.nl_dot(geo, psi, N)
    sp = oracle.spsi(sysk, psi, rp) if paw else None
    psi, sp, rp = oracle.ortho(sysk, M, psi, sp, rp, 0, 1)
    start = (psi.copy(), None if sp is None else sp.copy(), rp.copy())
    # without the smoother: converges to rounding
    for it in range(60):
        st, psi, sp, rp, sval = oracle.rayleighritz(sysk, M, psi, sp, rp)
        st, psi, sp, rp, hh, sval, resid = oracle.kscg(sysk, M, psi, sp, rp, nsdmax=4, nprecon=0)
    st, psi, sp, rp, sval = oracle.rayleighritz(sysk, M, psi, sp, rp)
    np.testing.assert_allclose(sval[:6], ref, atol=1e-9)
    # DIIS keeps the converged subspace
    conv, psi2, sp2, rp2, h2, sval2, res2 = oracle.ksdiis(sysk, M, psi, sp, rp, nprecon=0)
    st, psi2, sp2, rp2, sval3 = oracle.rayleighritz(sysk, M, psi2, sp2, rp2)
    np.testing.assert_allclose(sval3[:6], ref, atol=1e-9)
    # with kukan's smoother: the (pi,pi,pi) mode it cannot reach bounds the error
    psi3, sp3, rp3 = start
    for it in range(40):
        st, psi3, sp3, rp3, sval = oracle.rayleighritz(sysk, M, psi3, sp3, rp3)
        st, psi3, sp3, rp3, hh, sval, resid = oracle.kscg(sysk, M, psi3, sp3, rp3, nsdmax=4)
        conv, psi3, sp3, rp3, hh, sval, resid = oracle.ksdiis(sysk, M, psi3, sp3, rp3)
    st, psi3, sp3, rp3, sval = oracle.rayleighritz(sysk, M, psi3, sp3, rp3)
    np.testing.assert_allclose(sval[:6], ref, atol=2e-5)
    # S-orthonormality of the Ritz vectors
    spn = oracle.spsi(sysk, psi2, oracle.nl_dot(geo, psi2, N)) if paw else psi2
    np.testing.assert_allclose(psi2 @ spn.T * dv, np.eye(M), atol=1e-9)


def _smooth_bands(shape, M, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((M, nz, ny, nx))
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(nz), np.fft.fftfreq(ny), np.fft.fftfreq(nx),
                             indexing="ij")
    filt = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / 0.01)
    x = np.real(np.fft.ifftn(np.fft.fftn(x, axes=(1, 2, 3)) * filt, axes=(1, 2, 3)))
    return x.reshape(M, -1)


def _geo(cell):
    return dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
                natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())


@pytest.mark.parametrize("kind,n,tol", [("si_paw", 32, 0.015), ("c_ncps", 24, 0.025)])
def test_force_nl_is_minus_energy_gradient(oracle, kind, n, tol):
    """force_eig's nonlocal force equals -dE/dR of E = sum_l f_l <psi_l|p> (D - e_l S) <p|psi_l>
    with psi held fixed: central differences over atom displacements of 1e-3 bohr, the
    projector tables re-sampled at the moved atoms.  The two differ only by the grid's
    summation by parts (the oracle differentiates psi with the 8th-order FD, the energy
    moves the sampled projectors), measured at 0.7 % (Si, 32^3) and 1.1 % (C, 24^3)."""
    from rspacedist_b200 import system as S
    ds = S.load_dataset(kind)
    a0, sig, seed = (10.26, 0.05, 4) if kind == "si_paw" else (6.74, 0.03, 2)
    pos = S.diamond_positions(1, a0, sig, seed)
    cell = S.make_cell(a0, n, pos, ds)
    M = 2
    psi = _smooth_bands(cell.shape, M, 3)
    sval, occ = np.array([-0.3, -0.1]), np.array([2.0, 1.0])
    sysk = oracle.make_sys(_geo(cell), cell.shape, 4, cell.h, S.smooth_veff(cell, 1), cell.dij,
                           cell.sss)
    F = oracle.force_nl(sysk, M, psi, sval, occ)

    def energy(c):
        rp = oracle.nl_dot(_geo(c), psi, c.N)
        e = 0.0
        for l in range(M):
            for a in range(c.natom):
                D = c.dij[a] - (sval[l] * c.sss[a] if c.sss is not None else 0.0)
                e += occ[l] * rp[l, a] @ D @ rp[l, a]
        return e

    d = 1e-3
    for a in (0, 3):
        for ax in range(3):
            p = pos.copy()
            p[a, ax] += d
            ep = energy(S.make_cell(a0, n, p, ds))
            p[a, ax] -= 2 * d
            em = energy(S.make_cell(a0, n, p, ds))
            assert abs(F[a, ax] + (ep - em) / (2 * d)) < tol * np.abs(F).max(), (a, ax)


def test_d2c_is_the_scaled_transpose_of_c2d(oracle):
    """trans_d2c (interpolation mode 2 + periodic fold + 1/nmesh^3) is the exact
    transpose of the periodic coarse->dense interpolation divided by 8:
    <c2d(u), w>_dense = 8 <u, d2c(w)>_coarse for any u, w."""
    rng = np.random.default_rng(5)
    for shape in ((8, 10, 12), (16, 16, 16)):
        nx, ny, nz = shape
        u = rng.standard_normal(nx * ny * nz)
        w = rng.standard_normal(8 * nx * ny * nz)
        lhs = oracle.interp_c2d(shape, 4, u) @ w
        rhs = 8.0 * (u @ oracle.interp_d2c(shape, 4, w))
        assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
        # a constant field maps to the same constant (weights sum to one)
        c = oracle.interp_d2c(shape, 4, np.full(8 * nx * ny * nz, 0.7))
        np.testing.assert_allclose(c, 0.7, rtol=1e-14)


def test_pz_lda_known_values_and_derivative(oracle):
    """Exchange part -0.458165.../rs; v = d(rho eps)/drho (central differences)
    on both sides of rs = 1; eps continuous at rs = 1 to the fit's accuracy."""
    pi = np.pi
    rs = np.array([0.3, 0.7, 0.999, 1.0, 1.5, 3.0, 8.0])
    rho = 3.0 / (4.0 * pi * rs ** 3)
    vx, ex = oracle.vxc_pz(rho)
    cx = 0.75 * (2.25 / pi ** 2) ** (1 / 3)
    assert abs(cx - 0.4581652932831429) < 1e-15
    ec = np.where(rs >= 1.0, -0.1423 / (1 + 1.0529 * np.sqrt(rs) + 0.3334 * rs),
                  -0.048 + 0.0311 * np.log(rs) - 0.0116 * rs + 0.002 * rs * np.log(rs))
    np.testing.assert_allclose(ex, ec - cx / rs, rtol=1e-14)
    for r in rho[np.abs(rs - 1.0) > 1e-2]:  # the fit switches branch at rs = 1
        d = 1e-6 * r
        ep, em = oracle.vxc_pz([r + d])[1][0], oracle.vxc_pz([r - d])[1][0]
        fd = ((r + d) * ep - (r - d) * em) / (2 * d)
        assert abs(fd - oracle.vxc_pz([r])[0][0]) < 1e-8
    lo, hi = oracle.vxc_pz([3.0 / (4.0 * pi * (1 - 1e-12)), 3.0 / (4.0 * pi)])[1]
    assert abs(lo - hi) < 1e-4
    vx0, ex0 = oracle.vxc_pz([0.0, 1e-16])
    assert not vx0.any() and not ex0.any()


def test_diffcharge(oracle):
    rng = np.random.default_rng(2)
    a, b = rng.random(5000), rng.random(5000)
    h, xmax = (0.3, 0.31, 0.29), (3.0, 3.1, 2.9)
    ref = np.sqrt(np.sum((b - a) ** 2) * h[0] * h[1] * h[2] / (8 * xmax[0] * xmax[1] * xmax[2]))
    assert abs(oracle.diffcharge(a, b, h, xmax) - ref) < 1e-14 * ref


def test_broyden_first_step_is_linear_and_it_solves_a_fixed_point(oracle):
    """scf_chargemixing: the first call copies rho_out, the second is linear
    mixing with eta; on rho_out = A rho_in + c (A symmetric, eigenvalues in
    [-0.9, 0.95]) the Broyden iteration reaches the fixed point far faster
    than linear mixing."""
    rng = np.random.default_rng(3)
    n = 300
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = Q @ np.diag(np.linspace(-0.9, 0.95, n)) @ Q.T
    c = rng.standard_normal(n)
    fix = np.linalg.solve(np.eye(n) - A, c)
    mix = oracle.Broyden(n, nbrydn=8, eta=0.3)
    r0 = rng.standard_normal(n)
    ri = mix.step(r0, np.zeros(n), 0.01)
    assert np.array_equal(ri, r0)
    ro = A @ ri + c
    r2 = mix.step(ro, ri, 0.01)
    np.testing.assert_array_equal(r2, ri + (ro - ri) * 0.3)
    ri = r2
    for _ in range(100):
        ro = A @ ri + c
        ri = mix.step(ro, ri, 0.01)
    assert np.linalg.norm(ri - fix) < 1e-7 * np.linalg.norm(fix)
    lin = r0.copy()
    for _ in range(101):
        lin = lin + 0.3 * (A @ lin + c - lin)
    assert np.linalg.norm(lin - fix) > 1e-3 * np.linalg.norm(fix)


def test_atomicocc_known_answer(oracle):
    """scf_charge_atomicocc restated: packed upper triangle (j outer, i <= j),
    off-diagonal entries doubled, equal to sum_l f_l r_i r_j from numpy."""
    rng = np.random.default_rng(3)
    M, natom, P = 7, 3, 4
    rp = rng.standard_normal((M, natom, P))
    f = rng.uniform(0, 2, M)
    got = oracle.atomicocc(np.array([4, 4, 2]), P, rp, f)
    full = np.einsum("l,lai,laj->aij", f, rp, rp)
    for a, npa in enumerate((4, 4, 2)):
        ij = 0
        for j in range(P):
            for i in range(j + 1):
                want = 0.0 if j >= npa else full[a, i, j] * (1.0 if i == j else 2.0)
                assert abs(got[a, ij] - want) <= 1e-13 * max(1.0, abs(want))
                ij += 1
