"""Subspace contractions on the GPU against FP64 numpy: tcgen05 3xTF32 Gram
and rotation kernels (FP32 operands) and the FP64 kernels."""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr())


def _s():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


@pytest.mark.parametrize("m,n,K,sym", [(20, 20, 32768, 1), (160, 160, 20004, 1),
                                       (200, 72, 50000, 0), (130, 257, 4096, 0)])
def test_gram_f32_tensor_cores(built_lib, cuda, m, n, K, sym):
    from rspacedist_b200 import lib
    rng = np.random.default_rng(m + n)
    A = rng.standard_normal((m, K)).astype(np.float32)
    B = A if sym else rng.standard_normal((n, K)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T * 0.5
    dA = torch.tensor(A, device="cuda")
    dB = dA if sym else torch.tensor(B, device="cuda")
    Cm = torch.zeros((n, m), dtype=torch.float64, device="cuda")  # column-major m x n
    lib.call("rs_gram_f32", m, n, K, _p(dA), K, _p(dB), K, 0.5, _p(Cm), m, sym, _s())
    got = Cm.cpu().numpy().T
    # 3xTF32 products, FP32 accumulation over 64 terms, FP64 beyond
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err


@pytest.mark.parametrize("m,K", [(20, 32768), (257, 20004), (300, 50000)])
def test_gram_f32_lower_triangle(built_lib, cuda, m, K):
    """sym=2: the lower triangle of A B^T for distinct A, B (a product known to
    be symmetric), mirrored into the upper one.  The K splits follow the
    number of tile pairs, so the lower triangle agrees with the full product
    to rounding, not bit for bit."""
    from rspacedist_b200 import lib
    rng = np.random.default_rng(m + K)
    A = rng.standard_normal((m, K)).astype(np.float32)
    B = rng.standard_normal((m, K)).astype(np.float32)
    ref = A.astype(np.float64) @ B.astype(np.float64).T
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    full = torch.zeros((m, m), dtype=torch.float64, device="cuda")
    low = torch.zeros_like(full)
    lib.call("rs_gram_f32", m, m, K, _p(dA), K, _p(dB), K, 1.0, _p(full), m, 0, _s())
    lib.call("rs_gram_f32", m, m, K, _p(dA), K, _p(dB), K, 1.0, _p(low), m, 2, _s())
    f, lo = full.cpu().numpy().T, low.cpu().numpy().T  # C(i, j) at [i, j]
    il = np.tril_indices(m)
    assert np.array_equal(lo, lo.T)
    scale = np.abs(ref).max()
    assert np.abs(lo[il] - ref[il]).max() < 2e-6 * scale
    assert np.abs(lo[il] - f[il]).max() < 2e-6 * scale


@pytest.mark.parametrize("npts,kin,nout", [(4096, 20, 20), (65536, 160, 160),
                                           (12288, 300, 270), (8192, 70, 513),
                                           (4100, 33, 129)])
def test_rotate_f32_tensor_cores(built_lib, cuda, npts, kin, nout):
    from rspacedist_b200 import lib
    rng = np.random.default_rng(npts + kin)
    X = rng.standard_normal((kin, npts)).astype(np.float32)
    Z = rng.standard_normal((kin, nout)) / np.sqrt(kin)
    ref = (X.astype(np.float64).T @ Z).T  # (nout, npts)
    dX = torch.tensor(X, device="cuda")
    dZ = torch.tensor(Z.T.copy(), device="cuda")  # column-major kin x nout
    dY = torch.zeros((nout, npts), dtype=torch.float32, device="cuda")
    lib.call("rs_rotate_f32", npts, kin, nout, _p(dX), npts, _p(dZ), kin, _p(dY), npts, _s())
    got = dY.cpu().numpy()
    err = np.abs(got - ref).max() / np.abs(ref).max()
    assert err < 2e-6, err
    if nout <= kin:  # in place over X gives the same bits
        lib.call("rs_rotate_f32", npts, kin, nout, _p(dX), npts, _p(dZ), kin, _p(dX), npts, _s())
        assert torch.equal(dX[:nout], dY)


def test_gram_and_rotate_f64(built_lib, cuda):
    from rspacedist_b200 import lib
    rng = np.random.default_rng(1)
    m, n, K = 70, 45, 30001
    A = rng.standard_normal((m, K))
    B = rng.standard_normal((n, K))
    dA, dB = torch.tensor(A, device="cuda"), torch.tensor(B, device="cuda")
    Cm = torch.zeros((n, m), dtype=torch.float64, device="cuda")
    lib.call("rs_gram_f64", m, n, K, _p(dA), K, _p(dB), K, 2.0, _p(Cm), m, _s())
    np.testing.assert_allclose(Cm.cpu().numpy().T, 2.0 * A @ B.T, rtol=1e-12, atol=1e-10)
    Z = rng.standard_normal((m, 33))
    dZ = torch.tensor(Z.T.copy(), device="cuda")
    dY = torch.zeros((33, K), dtype=torch.float64, device="cuda")
    lib.call("rs_rotate_f64", K, m, 33, _p(dA), K, _p(dZ), m, _p(dY), K, _s())
    np.testing.assert_allclose(dY.cpu().numpy(), (A.T @ Z).T, rtol=1e-12, atol=1e-11)
