"""GPU parity of the hot-path kernels against the CPU oracle.

FP64 kernels must match the strict oracle bit for bit (same evaluation
order); FP32 (mixed-precision) kernels must match within the stated relative
tolerance.  All calls go through the C ABI."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

F32_RTOL = 2e-5   # FP32 psi vs FP64 oracle, relative to the max |value|


def T(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def geo_dict(cell):
    return dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
                natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())


@pytest.fixture(scope="module")
def setup(si8, cuda):
    from rspacedist_b200 import kukan as K, system as S
    g = K.Geometry(si8)
    veff = S.smooth_veff(si8, 1)
    psi = S.random_bands(si8, 5, 2)
    return si8, g, veff, psi


def test_kslaplacian_f64_bit_exact(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    base = np.random.default_rng(3).standard_normal(psi.shape)
    ref = oracle.kslaplacian(cell.shape, 4, cell.h, psi, veff, base)
    out = T(base)
    K.kslaplacian(g, T(psi), T(veff), out)
    assert np.array_equal(out.cpu().numpy(), ref)


def test_kslaplacian_f32(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    ref = oracle.kslaplacian(cell.shape, 4, cell.h, psi.astype(np.float32), veff.astype(np.float32))
    out = torch.zeros(psi.shape, dtype=torch.float32, device="cuda")
    K.kslaplacian(g, T(psi, torch.float32), T(veff, torch.float32), out)
    np.testing.assert_allclose(out.cpu().numpy(), ref, atol=F32_RTOL * np.abs(ref).max())


def test_nonlocal_dot_f64_bit_exact(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    ref = oracle.nl_dot(geo_dict(cell), psi, cell.N)
    rp = K.nonlocaloperation_01(g, T(psi))
    assert np.array_equal(rp.cpu().numpy(), ref)


def test_nonlocal_dot_f32(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    p32 = psi.astype(np.float32)
    ref = oracle.nl_dot(geo_dict(cell), p32.astype(np.float64), cell.N)
    rp = K.nonlocaloperation_01(g, T(p32, torch.float32)).cpu().numpy()
    np.testing.assert_allclose(rp, ref, atol=1e-6 * np.abs(ref).max())


@pytest.mark.parametrize("which", ["dij", "sss"])
def test_nonlocal_apply_f64_bit_exact(setup, oracle, which):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    mat = cell.dij if which == "dij" else cell.sss
    rp = oracle.nl_dot(geo_dict(cell), psi, cell.N)
    base = np.random.default_rng(4).standard_normal(psi.shape)
    ref = oracle.nl_apply(geo_dict(cell), mat, cell.dvol, rp, cell.N, base)
    out = T(base)
    K.nonlocaloperation_02(g, T(mat), T(rp), out)
    assert np.array_equal(out.cpu().numpy(), ref)


def test_hpsi_f64_bit_exact(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    sysk = oracle.make_sys(geo_dict(cell), cell.shape, 4, cell.h, veff, cell.dij, cell.sss)
    rp = oracle.nl_dot(geo_dict(cell), psi, cell.N)
    ref = oracle.hpsi(sysk, psi, rp)
    out = K.hpsi(g, T(veff), T(cell.dij), T(rp), T(psi))
    assert np.array_equal(out.cpu().numpy(), ref)
    sref = oracle.spsi(sysk, psi, rp)
    sout = K.spsi(g, T(cell.sss), T(rp), T(psi))
    assert np.array_equal(sout.cpu().numpy(), sref)


@pytest.mark.parametrize("nb", [1, 5, 13])
def test_hpsi_f32(setup, oracle, nb):
    from rspacedist_b200 import kukan as K, system as S
    cell, g, veff, _ = setup
    psi = S.random_bands(cell, nb, 7 + nb).astype(np.float32)
    v32 = veff.astype(np.float32)
    sysk = oracle.make_sys(geo_dict(cell), cell.shape, 4, cell.h, v32, cell.dij, cell.sss)
    rp = oracle.nl_dot(geo_dict(cell), psi, cell.N)
    ref = oracle.hpsi(sysk, psi, rp)
    out = K.hpsi(g, T(v32, torch.float32), T(cell.dij), T(rp), T(psi, torch.float32))
    np.testing.assert_allclose(out.cpu().numpy(), ref, atol=F32_RTOL * np.abs(ref).max())
    sref = oracle.spsi(sysk, psi, rp)
    sout = K.spsi(g, T(cell.sss), T(rp), T(psi, torch.float32))
    np.testing.assert_allclose(sout.cpu().numpy(), sref, atol=F32_RTOL * np.abs(sref).max())


@pytest.mark.parametrize("nb", [1, 8, 13])
def test_spsi_f32_vector_path_matches_rmw_path(setup, nb):
    """The FP32 S psi of aligned bands (per-entry sums, then one 16-byte
    vector pass over the grid) and the copy + covered-point pass used for
    unaligned bands give the same bits, also in place."""
    from rspacedist_b200 import kukan as K, system as S
    cell, g, veff, _ = setup
    psi = torch.tensor(S.random_bands(cell, nb, 7), dtype=torch.float32, device="cuda")
    rp = K.nonlocaloperation_01(g, psi)
    sss = T(cell.sss)
    fused = K.spsi(g, sss, rp, psi)
    big = torch.zeros(nb * cell.N + 1, dtype=torch.float32, device="cuda")
    shifted = big[1:].view(nb, cell.N)  # 4 bytes off a 16-byte boundary
    shifted.copy_(psi)
    two_pass = K.spsi(g, sss, rp, shifted)
    assert torch.equal(fused, two_pass)
    inplace = psi.clone()
    K.spsi(g, sss, rp, inplace, out=inplace)
    assert torch.equal(fused, inplace)


def test_hpsi_host_matches_device(setup):
    from rspacedist_b200 import kukan as K, system as S
    cell, g, veff, _ = setup
    psi = S.random_bands(cell, 11, 5).astype(np.float32)
    rp = K.nonlocaloperation_01(g, T(psi, torch.float32))
    v32 = T(veff, torch.float32)
    dev = K.hpsi(g, v32, T(cell.dij), rp, T(psi, torch.float32)).cpu()
    hin = torch.tensor(psi).pin_memory()
    hout = torch.empty_like(hin).pin_memory()
    K.hpsi_host(g, v32, T(cell.dij), rp, hin, hout, chunk=4)
    assert torch.equal(hout, dev)


def test_precondition(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    ref = oracle.precondition(cell.shape, psi)
    out = K.ksprecondition(g, T(psi))
    assert np.array_equal(out.cpu().numpy(), ref)
    o32 = K.ksprecondition(g, T(psi, torch.float32)).cpu().numpy()
    np.testing.assert_allclose(o32, ref, atol=1e-6 * np.abs(ref).max())


def _grid_only_geometry(shape, h=0.3):
    """A geometry without atoms, for the grid kernels on arbitrary shapes."""
    import types
    from rspacedist_b200 import kukan as K
    N = int(np.prod(shape))
    e = types.SimpleNamespace(shape=tuple(shape), h=(h, h, h), natom=0, nprjmx=4, num_list=1,
                              nprj=np.zeros(1, np.int32), natinf=np.zeros(1, np.int32),
                              lst=np.zeros(1, np.int32), vnlocp=np.zeros(1), N=N)
    return K.Geometry(e)


@pytest.mark.parametrize("shape", [(12, 10, 10), (20, 9, 11), (18, 10, 9), (16, 16, 40),
                                   (10, 12, 64)])
def test_precondition_shapes(cuda, oracle, shape):
    """The plane-marching preconditioner (rows in 16-byte vectors, partial y
    tiles and z runs) and the row-wise form it falls back to give the
    oracle's bits in FP64 on grids of every parity."""
    from rspacedist_b200 import kukan as K
    g = _grid_only_geometry(shape)
    nx, ny, nz = shape
    psi = np.random.default_rng(nx * ny + nz).standard_normal((3, nx * ny * nz))
    ref = oracle.precondition(shape, psi)
    out = K.ksprecondition(g, T(psi))
    assert np.array_equal(out.cpu().numpy(), ref)
    o32 = K.ksprecondition(g, T(psi, torch.float32)).cpu().numpy()
    np.testing.assert_allclose(o32, ref, atol=1e-6 * np.abs(ref).max())


def test_density(setup, oracle):
    from rspacedist_b200 import kukan as K
    cell, g, veff, psi = setup
    occ = np.array([2.0, 2.0, 1.5, 0.5, 0.0])
    ref = oracle.density(occ, psi, cell.N)
    rho = K.scf_charge_smt(T(occ), T(psi), cell.N)
    assert np.array_equal(rho.cpu().numpy(), ref)
    r32 = K.scf_charge_smt(T(occ), T(psi, torch.float32), cell.N).cpu().numpy()
    ref32 = oracle.density(occ, psi.astype(np.float32).astype(np.float64), cell.N)
    assert np.array_equal(r32, ref32)


def test_interp_c2d_bit_exact(oracle, cuda, built_lib):
    from rspacedist_b200 import kukan as K
    shape = (12, 10, 14)
    x = np.random.default_rng(8).standard_normal(np.prod(shape))
    ref = oracle.interp_c2d(shape, 4, x)
    out = K.trans_c2d_smtcharge(shape, 4, T(x))
    assert np.array_equal(out.cpu().numpy(), ref)


def test_hartree_bit_exact(oracle, cuda, built_lib):
    from rspacedist_b200 import kukan as K
    shape = (24, 20, 16)
    h = (0.31, 0.33, 0.29)
    xmax = tuple(n * hh / 2 for n, hh in zip(shape, h))
    rng = np.random.default_rng(9)
    rho = rng.standard_normal(np.prod(shape))
    v = rng.standard_normal(np.prod(shape))
    ref = oracle.hartree_laplacian(shape, 4, h, v)
    out = K.scf_hartee_laplacian(shape, 4, h, T(v))
    assert np.array_equal(out.cpu().numpy(), ref)
    vh0 = rng.standard_normal(np.prod(shape)) * 0.01
    vref, itref, dpref = oracle.hartree_cg(shape, 4, xmax, 1e-12, 1, 800, 801, rho, vh0)
    vh = T(vh0)
    it, dp = K.scf_hartree(shape, 4, xmax, T(rho), vh)
    assert it == itref and dp == dpref
    assert np.array_equal(vh.cpu().numpy(), vref)
    # on a stream of its own the solve replays its iteration batches as a graph
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        vh2 = T(vh0)
        it2, dp2 = K.scf_hartree(shape, 4, xmax, T(rho), vh2)
    st.synchronize()
    assert it2 == itref and dp2 == dpref
    assert np.array_equal(vh2.cpu().numpy(), vref)


@pytest.mark.parametrize("n", [1, 4095, 4096, 4097, 300000])
def test_tree_dot_bit_exact(oracle, cuda, built_lib, n):
    from rspacedist_b200 import kukan as K
    rng = np.random.default_rng(n)
    a, b = rng.standard_normal(n), rng.standard_normal(n)
    assert K.dot(T(a), T(b)).item() == oracle.tree_dot(a, b)
    a32, b32 = a.astype(np.float32), b.astype(np.float32)
    assert K.dot(T(a32, torch.float32), T(b32, torch.float32)).item() == oracle.tree_dot(a32, b32)


def test_c8_norm_conserving_hpsi(c8, oracle, cuda):
    from rspacedist_b200 import kukan as K, system as S
    g = K.Geometry(c8)
    veff = S.smooth_veff(c8, 3)
    psi = S.random_bands(c8, 3, 4)
    sysk = oracle.make_sys(geo_dict(c8), c8.shape, 4, c8.h, veff, c8.dij, None)
    rp = oracle.nl_dot(geo_dict(c8), psi, c8.N)
    ref = oracle.hpsi(sysk, psi, rp)
    out = K.hpsi(g, T(veff), T(c8.dij), T(rp), T(psi))
    assert np.array_equal(out.cpu().numpy(), ref)


@pytest.mark.parametrize("n", [(24, 24, 24), (40, 36, 28), (128, 40, 16)])
def test_hpsi_f32_ragged_tiles(oracle, cuda, built_lib, n):
    """Grids whose x/y sizes are not multiples of the CTA tile (64 x 32)."""
    from rspacedist_b200 import kukan as K, system as S
    ds = S.load_dataset("c_ncps")
    A = np.array(n) * 0.28
    pos = S.diamond_positions(1, 1.0, 0.0)[:4] * A - A / 2 + 0.37
    pos = (pos + A / 2) % A - A / 2
    cell = S.make_cell(A, n, pos, ds)
    g = K.Geometry(cell)
    veff = S.smooth_veff(cell, 5).astype(np.float32)
    psi = S.random_bands(cell, 3, 6).astype(np.float32)
    sysk = oracle.make_sys(geo_dict(cell), cell.shape, 4, cell.h, veff, cell.dij, None)
    rp = oracle.nl_dot(geo_dict(cell), psi, cell.N)
    ref = oracle.hpsi(sysk, psi, rp)
    out = K.hpsi(g, T(veff, torch.float32), T(cell.dij), T(rp), T(psi, torch.float32))
    np.testing.assert_allclose(out.cpu().numpy(), ref, atol=F32_RTOL * np.abs(ref).max())


def test_atomicocc_bit_exact(oracle, cuda, built_lib, si8):
    """scf_charge_atomicocc: GPU occupation matrices equal the oracle's bit for
    bit, and their diagonal is sum_l f_l <p_i|psi_l>^2."""
    from rspacedist_b200 import kukan as K
    g = K.Geometry(si8)
    rng = np.random.default_rng(5)
    M = 20
    rp = rng.standard_normal((M, si8.natom, si8.nprjmx))
    f = rng.uniform(0.0, 2.0, M)
    got = K.scf_charge_atomicocc(g, T(rp), T(f)).cpu().numpy()
    ref = oracle.atomicocc(si8.nprj, si8.nprjmx, rp, f)
    assert np.array_equal(got, ref)
    diag = [j * (j + 1) // 2 + j for j in range(si8.nprjmx)]
    np.testing.assert_allclose(ref[:, diag], np.einsum("l,lai->ai", f, rp ** 2), rtol=1e-13)


@pytest.mark.parametrize("shape", [(40, 48, 56), (42, 44, 40)])
def test_hartree_mixed_anisotropic(cuda, built_lib, shape):
    """Mixed Hartree CG on box grids: (40, 48, 56) takes the 4 x 2-point A p
    z-march with a partial z run, (42, 44, 40) the paired Hartree z-march."""
    from rspacedist_b200 import kukan as K
    nx, ny, nz = shape
    hh = 0.22
    axes = [(np.arange(n) + 0.5) * hh - n * hh / 2 for n in (nx, ny, nz)]
    rho = np.zeros((nz, ny, nx))
    rng = np.random.default_rng(nx)
    for c in rng.uniform(-1.5, 1.5, (3, 3)):
        d = [axes[k] - c[k] for k in range(3)]
        r2 = d[2][:, None, None] ** 2 + d[1][None, :, None] ** 2 + d[0][None, None, :] ** 2
        rho += np.exp(-r2 / 1.5)
    rho -= rho.mean()
    xm = tuple(n * hh / 2 for n in (nx, ny, nz))
    v64 = torch.zeros(rho.size, dtype=torch.float64, device="cuda")
    v32 = torch.zeros_like(v64)
    K.scf_hartree(shape, 4, xm, T(rho.ravel()), v64, 1e-12)
    it, dp = K.scf_hartree(shape, 4, xm, T(rho.ravel()), v32, 1e-12, mixed=True)
    err = float((v32 - v64).abs().max() / v64.abs().max())
    assert err < 2e-6, (err, it, dp)


def test_hartree_mixed_matches_fp64(cuda, built_lib):
    """The mixed Hartree CG (FP32 vectors, FP64 dots and vh) solves the same
    problem: its potential agrees with the FP64 solve to FP32 accuracy."""
    from rspacedist_b200 import kukan as K
    n = 48
    a = 10.26
    x = (np.arange(n) + 0.5) * (a / n) - a / 2
    rng = np.random.default_rng(0)
    rho = np.zeros((n, n, n))
    for c in rng.uniform(-a / 2, a / 2, (4, 3)):
        d = [x - c[k] for k in range(3)]
        d = [di - a * np.round(di / a) for di in d]
        r2 = d[2][:, None, None] ** 2 + d[1][None, :, None] ** 2 + d[0][None, None, :] ** 2
        rho += np.exp(-r2 / 2.0) / (2 * np.pi) ** 1.5
    rho -= rho.mean()
    xm = (a / 2,) * 3
    v64 = torch.zeros(n ** 3, dtype=torch.float64, device="cuda")
    v32 = torch.zeros_like(v64)
    K.scf_hartree((n, n, n), 4, xm, T(rho.ravel()), v64, 1e-12)
    it, dp = K.scf_hartree((n, n, n), 4, xm, T(rho.ravel()), v32, 1e-12, mixed=True)
    err = float((v32 - v64).abs().max() / v64.abs().max())
    assert err < 2e-6, (err, it, dp)
