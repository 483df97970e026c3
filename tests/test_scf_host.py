"""Host logic of the SCF driver (no GPU): kukan's Fermi-Dirac occupations."""
import numpy as np


def test_scf_occupation_counts_and_orders():
    from rspacedist_b200 import scf
    rng = np.random.default_rng(0)
    sval = np.sort(rng.uniform(-0.5, 0.2, 60))
    for nel in (20.0, 37.0, 64.0):
        f, ef = scf.scf_occupation(sval, nel)
        assert abs(f.sum() - nel) < 1e-9
        assert np.all(np.diff(f) <= 0) and f.min() >= 0 and f.max() <= 2
        assert abs(f[np.argmin(np.abs(sval - ef))] - 1.0) < 1.0
    # an insulator: a 1 Ha gap after 10 bands gives integer occupations
    gap = np.concatenate([np.linspace(-2, -1.5, 10), np.linspace(-0.5, 0, 10)])
    f, ef = scf.scf_occupation(gap, 20.0)
    assert np.array_equal(f, np.r_[np.full(10, 2.0), np.zeros(10)])
    assert -1.5 < ef < -0.5


def test_fermidis_clips_far_tails():
    from rspacedist_b200 import scf
    assert scf.fermidis(2.0, 1.0, 1e-3, 0.0) == 0.0
    assert scf.fermidis(2.0, -1.0, 1e-3, 0.0) == 2.0
    assert scf.fermidis(2.0, 0.0, 1e-3, 0.0) == 1.0
