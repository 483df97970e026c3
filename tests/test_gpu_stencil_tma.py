"""The FP32 stencil's two staging forms: tensor-map (TMA) loads of whole rows
(k_stencil_f32_tma, mode 0) and per-thread cp.async (k_stencil_f32_zmarch,
mode 1).

* On every grid the TMA form takes (nx = 64, 128 or 256, ny a multiple of
  2048 / nx) the TMA form gives the same bits as the cp.async form, with and without
  atoms, over tiles at both y edges, one-tile grids and z runs shorter and
  longer than the shared-memory ring;
* both are within the FP32 tolerance of the oracle's FP64 kslaplacian_r
  (kslaplacian8f.F90:207-261);
* rs_hpsi_f32_staging reports which form a call takes, and grids outside the
  TMA shapes keep the cp.async form."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

F32_TOL = 2e-5


def T(a, dtype=torch.float32):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _staging(g, mode, nb):
    from rspacedist_b200 import lib
    tma = C.c_int(-1)
    lib.call("rs_hpsi_f32_staging", g.handle, mode, nb, C.byref(tma))
    return tma.value


def _grid_only(shape, h=0.31):
    import types
    from rspacedist_b200 import kukan as K
    N = int(np.prod(shape))
    e = types.SimpleNamespace(shape=tuple(shape), h=(h, 0.9 * h, 1.1 * h), natom=0, nprjmx=4,
                              num_list=1, nprj=np.zeros(1, np.int32), natinf=np.zeros(1, np.int32),
                              lst=np.zeros(1, np.int32), vnlocp=np.zeros(1), N=N)
    return K.Geometry(e)


@pytest.mark.parametrize("shape,nb", [((64, 64, 64), 5), ((128, 32, 24), 3), ((256, 16, 10), 2),
                                      ((64, 96, 40), 4), ((128, 16, 12), 3), ((256, 16, 9), 2)])
def test_tma_staging_matches_cp_async(cuda, built_lib, oracle, shape, nb):
    from rspacedist_b200 import kukan as K
    g = _grid_only(shape)
    nx, ny, nz = shape
    rng = np.random.default_rng(nx + 7 * ny + 13 * nz)
    psi = rng.standard_normal((nb, nx * ny * nz)).astype(np.float32)
    veff = rng.standard_normal(nx * ny * nz).astype(np.float32)
    assert _staging(g, 0, nb) == 1
    out_tma = K.hpsi(g, T(veff), None, None, T(psi)).cpu().numpy()
    assert _staging(g, 1, nb) == 0
    out_cp = K.hpsi(g, T(veff), None, None, T(psi)).cpu().numpy()
    assert np.array_equal(out_tma, out_cp)
    ref = oracle.kslaplacian(shape, 4, g.cell.h, psi, veff)
    assert np.abs(out_tma - ref).max() <= F32_TOL * np.abs(ref).max()


@pytest.mark.parametrize("shape", [(96, 32, 16), (128, 40, 16), (32, 32, 32), (64, 48, 12)])
def test_other_grids_keep_cp_async(cuda, built_lib, shape):
    g = _grid_only(shape)
    assert _staging(g, 0, 4) == 0


def test_tma_staging_with_atoms(cuda, built_lib, oracle):
    """A carbon cell on a 64 x 64 x 32 grid: the full H psi (stencil, then
    the nonlocal pass) is the same with either staging and within the FP32
    tolerance of the oracle."""
    from rspacedist_b200 import kukan as K, system as S
    ds = S.load_dataset("c_ncps")
    n = (64, 64, 32)
    A = np.array(n) * 0.21
    pos = S.diamond_positions(1, 1.0, 0.0) * A - A / 2 + 0.29
    pos = (pos + A / 2) % A - A / 2
    cell = S.make_cell(A, n, pos, ds)
    g = K.Geometry(cell)
    nb = 7
    veff = S.smooth_veff(cell, 3).astype(np.float32)
    psi = S.random_bands(cell, nb, 4).astype(np.float32)
    geo = dict(natom=cell.natom, nprjmx=cell.nprjmx, num_list=cell.num_list, nprj=cell.nprj,
               natinf=cell.natinf, lst=cell.lst, v=cell.vnlocp.ravel())
    sysk = oracle.make_sys(geo, cell.shape, 4, cell.h, veff, cell.dij, None)
    rp = oracle.nl_dot(geo, psi, cell.N)
    ref = oracle.hpsi(sysk, psi, rp)
    args = (g, T(veff), T(cell.dij, torch.float64), T(rp, torch.float64), T(psi))
    assert _staging(g, 0, nb) == 1
    out_tma = K.hpsi(*args).cpu().numpy()
    _staging(g, 1, nb)
    out_cp = K.hpsi(*args).cpu().numpy()
    assert np.array_equal(out_tma, out_cp)
    assert np.abs(out_tma - ref).max() <= F32_TOL * np.abs(ref).max()


def test_staging_mode_checked(cuda, built_lib):
    from rspacedist_b200 import lib
    g = _grid_only((64, 64, 16))
    with pytest.raises(lib.RsError):
        _staging(g, 2, 4)
    assert _staging(g, -1, 4) == 1
