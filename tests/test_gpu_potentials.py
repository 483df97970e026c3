"""SCF potential and mixing steps on the GPU against the CPU oracle: the
dense -> coarse transfer, the veff sum, the charge difference and the Broyden
mixer bit for bit; the PZ LDA potential within 1e-14 relative (CUDA's pow and
log may round the last bit differently from the host library, and vx ends in
a subtraction that can cancel a few bits)."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def T(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


@pytest.mark.parametrize("shape", [(8, 10, 12), (24, 24, 24), (16, 12, 8)])
def test_d2c_bit_exact(built_lib, oracle, cuda, shape):
    from rspacedist_b200 import kukan as K
    rng = np.random.default_rng(1)
    w = rng.standard_normal(8 * int(np.prod(shape)))
    out = K.trans_d2c(shape, 4, T(w)).cpu().numpy()
    assert np.array_equal(out, oracle.interp_d2c(shape, 4, w))


def test_d2c_rejects_small_grids(built_lib, cuda):
    from rspacedist_b200 import kukan as K, lib
    with pytest.raises(lib.RsError):
        K.trans_d2c((6, 8, 8), 4, T(np.zeros(8 * 6 * 8 * 8)))


def test_vxc_pz_close(built_lib, oracle, cuda):
    from rspacedist_b200 import kukan as K
    rng = np.random.default_rng(2)
    rho = np.concatenate([10.0 ** rng.uniform(-8, 1.5, 20000), [0.0, 1e-16, 1e-15, 2e-15],
                          3.0 / (4 * np.pi * np.array([1.0, 0.999999, 1.000001]))])
    vx, ex = (t.cpu().numpy() for t in K.vxpot_lda_pz(T(rho)))
    rvx, rex = oracle.vxc_pz(rho)
    for a, b in ((vx, rvx), (ex, rex)):
        assert np.array_equal(a == 0, b == 0)
        np.testing.assert_allclose(a, b, rtol=1e-14, atol=0)


def test_veff_sum_and_diffcharge_bit_exact(built_lib, oracle, cuda):
    from rspacedist_b200 import kukan as K
    rng = np.random.default_rng(3)
    n = 24 ** 3
    vx, vl, vh = rng.standard_normal((3, n))
    veff = torch.empty(n, dtype=torch.float64, device="cuda")
    v32 = torch.empty(n, dtype=torch.float32, device="cuda")
    K.veff_sum(T(vx), T(vl), T(vh), veff, v32)
    ref = oracle.veff_sum(vx, vl, vh)
    assert np.array_equal(veff.cpu().numpy(), ref)
    assert np.array_equal(v32.cpu().numpy(), ref.astype(np.float32))
    a, b = rng.random((2, n))
    h, xm = (0.28, 0.28, 0.28), (3.37, 3.37, 3.37)
    assert K.scf_diffcharge(T(a), T(b), h, xm) == oracle.diffcharge(a, b, h, xm)


def test_broyden_mixer_bit_exact_through_history_shifts(built_lib, oracle, cuda):
    """The same SCF-like sequence (a linear response rho_out = A rho_in + c on
    a grid-sized vector) mixed on the GPU and by the oracle gives the same
    densities bit for bit at every step, through the history shift that
    starts once nbrydn steps are stored."""
    from rspacedist_b200 import kukan as K
    rng = np.random.default_rng(4)
    n = 13824
    k = np.fft.fftfreq(n)
    resp = 0.9 * np.cos(2 * np.pi * k * 7)  # a diagonal response in Fourier space

    def respond(r):
        return np.real(np.fft.ifft(np.fft.fft(r) * resp)) + 1.0

    nb, eta, dv = 5, 0.2, 0.02
    mix_g, mix_o = K.Mixer(n, nb, eta), oracle.Broyden(n, nb, eta)
    r0 = 1.0 + 0.1 * rng.standard_normal(n)
    ri_o = mix_o.step(r0, np.zeros(n), dv)
    ri_g = T(np.zeros(n))
    mix_g.step(T(r0), ri_g, dv)
    assert np.array_equal(ri_g.cpu().numpy(), ri_o)
    for _ in range(3 * nb):
        ro = respond(ri_o)
        ri_o = mix_o.step(ro, ri_o, dv)
        mix_g.step(T(ro), ri_g, dv)
        assert np.array_equal(ri_g.cpu().numpy(), ri_o)
