"""The seeded synthetic inputs (fmmgpu/workloads.py) have the distributions
the benchmark configurations name: the bench and the parity tests measure
on these, so their shapes, masses and radial profiles are checked here."""
import numpy as np
import pytest

from fmmgpu import workloads


@pytest.mark.parametrize("name", sorted(workloads.WORKLOADS))
def test_seeded_and_normalised(name):
    gen = workloads.WORKLOADS[name]
    p1, m1 = gen(5000, seed=11)
    p2, m2 = gen(5000, seed=11)
    p3, _ = gen(5000, seed=12)
    np.testing.assert_array_equal(p1, p2)
    np.testing.assert_array_equal(m1, m2)
    assert not np.array_equal(p1, p3)
    assert p1.shape == (5000, 2 if name.endswith("2d") else 3) and m1.shape == (5000,)
    assert p1.dtype == np.float64 and m1.dtype == np.float64
    assert np.all(np.isfinite(p1)) and np.all(m1 > 0)
    assert m1.sum() == pytest.approx(1.0, rel=1e-12)


def plummer_enclosed(r, a=1.0, rmax=20.0):
    """Mass fraction within r of a Plummer sphere cut at rmax."""
    f = lambda x: x ** 3 / (x * x + a * a) ** 1.5
    return f(r) / f(rmax)


def test_plummer_profile_and_isotropy():
    n = 200_000
    pos, m = workloads.plummer(n, seed=2)
    r = np.linalg.norm(pos, axis=1)
    assert r.max() <= 20.0
    for x in (0.25, 0.5, 1.0, 2.0, 5.0):
        # binomial standard deviation <= 0.0012 at this n
        assert np.mean(r <= x) == pytest.approx(plummer_enclosed(x), abs=0.006), x
    u = pos / r[:, None]
    assert np.all(np.abs(u.mean(axis=0)) < 0.01)                    # isotropic directions
    assert np.all(np.abs((u * u).mean(axis=0) - 1.0 / 3.0) < 0.01)
    np.testing.assert_array_equal(m, np.full(n, 1.0 / n))


def test_uniform_cube_and_disk():
    pos, m = workloads.uniform_cube(50_000, seed=1)
    assert pos.min() >= 0.0 and pos.max() < 1.0
    assert np.all(np.abs(pos.mean(axis=0) - 0.5) < 0.01)
    d, _ = workloads.uniform_disk_2d(50_000, seed=3)
    rad = np.linalg.norm(d, axis=1)
    assert rad.max() <= 1.0
    assert np.mean(rad <= 0.5) == pytest.approx(0.25, abs=0.01)    # uniform in area


def test_disk_clumps_2d():
    n = 100_000
    pos, m = workloads.disk_clumps_2d(n, seed=3)
    half = n // 2
    rad = np.linalg.norm(pos[:half], axis=1)
    assert rad.max() <= 1.0 and np.mean(rad <= 0.5) == pytest.approx(0.25, abs=0.01)
    # the other half sits in 64 clumps of width 0.005: nearly all of it within 4 sigma of one of few centres
    b = pos[half:]
    keys = np.unique(np.round(b / 0.05).astype(np.int64), axis=0)
    assert len(keys) < 64 * 8
    # log-normal(0, 0.5) masses before normalisation
    assert np.std(np.log(m)) == pytest.approx(0.5, rel=0.02)


def test_plummer_mixture():
    n = 64_000
    pos, m = workloads.plummer_mixture(n, seed=5)
    per = n // 32
    # 32 equal-count spheres of equal mass, stored one after another
    np.testing.assert_allclose(m.reshape(32, per).sum(axis=1), 1.0 / 32, rtol=1e-12)
    centres = np.median(pos.reshape(32, per, 3), axis=1)
    assert np.all((centres > -0.05) & (centres < 1.05))
    # each sphere's half-mass radius is that of a Plummer sphere (1.305 a), a in [0.01, 0.1]
    r = np.linalg.norm(pos.reshape(32, per, 3) - centres[:, None, :], axis=2)
    half = np.median(r, axis=1) / 1.305
    assert half.min() > 0.008 and half.max() < 0.12


def test_ensemble_sizes():
    s = workloads.ensemble_sizes()
    assert s.shape == (256,) and s.min() >= 1024 and s.max() <= 65536
    assert np.median(np.log(s)) == pytest.approx(0.5 * (np.log(1024) + np.log(65536)), rel=0.05)
