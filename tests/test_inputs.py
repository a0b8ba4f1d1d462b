"""CPU tests of the seeded synthetic inputs."""
import numpy as np

from dhara_b200 import inputs


def test_deterministic_for_a_seed():
    a = inputs.make_domain(20, 18, 6, seed=4)
    b = inputs.make_domain(20, 18, 6, seed=4)
    for k in a.fields:
        assert np.array_equal(a.fields[k], b.fields[k]), k
    c = inputs.make_domain(20, 18, 6, seed=5)
    assert not np.array_equal(a.fields["ksat"], c.fields["ksat"])


def test_grf_moments_and_correlation():
    rng = np.random.default_rng(0)
    f = inputs.gaussian_random_field(256, 256, 1.0, 1.0, 0.05, 3.0, rng)
    assert abs(f.std() - 0.05) < 1e-12
    lag = 3
    rho = np.mean(f[:, :-lag] * f[:, lag:]) / f.var()
    assert 0.2 < rho < 0.55   # Gaussian covariance: exp(-1) at one correlation length


def test_hydrostatic_head_and_conductivity():
    d = inputs.make_domain(16, 16, 20, seed=1, water_table=0.8, ks_median=1e-5, ks_sigma_ln=0.5)
    psi = d.fields["psi"].reshape(20, 16 * 16)
    np.testing.assert_allclose(psi[:, 0], (np.arange(20) + 0.5) * 0.05 - 0.8)
    assert np.all(psi == psi[:, :1])
    lk = np.log(d.fields["ksat"])
    assert abs(np.median(lk) - np.log(1e-5)) < 0.05
    assert abs(lk.std() - 0.5) < 0.02


def test_rain_schedules():
    d = inputs.mixed_512x512x40(nx=8, ny=8)
    assert len(d.rain_mm) == 240
    assert abs(d.rain_mm[:120].sum() - 40.0) < 1e-9 and d.rain_mm[120:].sum() == 0
    storm = inputs.triangular_storm(720, 120.0)
    assert abs(storm.sum() - 120.0) < 0.5
    assert abs(storm.max() / (120.0 / 3600.0) - 50.0) < 1.0


def test_ensemble_sizes():
    doms = inputs.ensemble(ndomains=32, nsteps=2)
    assert len(doms) == 32
    for d in doms:
        p = d.params
        assert 16 <= p.nx <= 128 and 16 <= p.ny <= 128 and 20 <= p.nz <= 40
        assert 1.0 <= p.alpha <= 5.0 and 1.3 <= p.n <= 2.2
