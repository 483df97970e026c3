"""Nonlocal forces (force_eig_r) on the GPU against the CPU oracle: the FP64
path must match bit for bit (same projections, same FD derivative, same
accumulation order per atom); the FP32-band path within 2e-5 of the largest
force component."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def T(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def geo_dict(cell):
    return dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
                natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())


def smooth_bands(shape, M, seed):
    nx, ny, nz = shape
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((M, nz, ny, nx))
    kz, ky, kx = np.meshgrid(np.fft.fftfreq(nz), np.fft.fftfreq(ny), np.fft.fftfreq(nx),
                             indexing="ij")
    filt = np.exp(-(kx ** 2 + ky ** 2 + kz ** 2) / 0.01)
    x = np.real(np.fft.ifftn(np.fft.fftn(x, axes=(1, 2, 3)) * filt, axes=(1, 2, 3)))
    return x.reshape(M, -1)


@pytest.fixture(scope="module", params=["si_paw", "c_nc"])
def system(request, built_lib, oracle, cuda):
    import conftest
    from rspacedist_b200 import kukan as K, system as S
    cell = conftest.make_si8(24, 0.05, 4) if request.param == "si_paw" else conftest.make_c8(24)
    g = K.Geometry(cell)
    sysk = oracle.make_sys(geo_dict(cell), cell.shape, 4, cell.h, S.smooth_veff(cell, 1),
                           cell.dij, cell.sss)
    M = 6
    psi = smooth_bands(cell.shape, M, 5)
    sval = np.linspace(-0.4, 0.2, M)
    occ = np.array([2.0, 2.0, 2.0, 1.5, 0.5, 0.0])
    ref = oracle.force_nl(sysk, M, psi, sval, occ)
    return dict(cell=cell, g=g, psi=psi, sval=sval, occ=occ, ref=ref)


def run(sy, dtype):
    from rspacedist_b200 import kukan as K
    cell = sy["cell"]
    sss = None if cell.sss is None else T(cell.sss)
    f = K.force_eig(sy["g"], T(cell.dij), sss, T(sy["psi"], dtype), T(sy["sval"]),
                    T(sy["occ"]))
    return f.cpu().numpy()


def test_force_nl_f64_bit_exact(system):
    f = run(system, torch.float64)
    assert np.abs(system["ref"]).max() > 1e-3  # a non-trivial force
    assert np.array_equal(f, system["ref"])


def test_force_nl_f32_close(system):
    f = run(system, torch.float32)
    ref = system["ref"]
    assert np.abs(f - ref).max() <= 2e-5 * np.abs(ref).max()


def test_force_nl_zero_bands_and_bad_args(system):
    from rspacedist_b200 import kukan as K, lib
    cell = system["cell"]
    f = K.force_eig(system["g"], T(cell.dij), None, T(np.zeros((0, cell.N))), T(np.zeros(0)),
                    T(np.zeros(0)))
    assert f.shape == (cell.natom, 3) and not f.abs().any()
    with pytest.raises(lib.RsError):
        lib.call("rs_force_nl_f64", None, None, None, None, None, None, 1, None, None)
