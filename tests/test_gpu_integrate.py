"""Integrators on the GPU (fmm_integrate) against CPU restatements driven by
FP64 oracle forces.  The force error of the FMM (relative ~1e-4 at p = 6)
enters positions only through dt^2 terms, so positions agree to ~1e-8."""
import numpy as np
import pytest

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu


def cpu_se(force, x, v, dt, steps):
    """SyplecticEuler::integrate (symplectic_euler.cpp:8-15)."""
    x, v = x.copy(), v.copy()
    for _ in range(steps):
        a = force(x)
        v = v + dt * a
        x = x + dt * v
    return x, v


def cpu_rk4(oracle, x, v, m, dt, eps2):
    f = lambda y: oracle.direct(y, m, eps2=eps2)
    a1 = f(x)
    v2 = v + dt / 2 * a1; x2 = x + dt / 2 * v
    a2 = f(x2)
    v3 = v + dt / 2 * a2; x3 = x + dt / 2 * v2
    a3 = f(x3)
    v4 = v + dt * a3; x4 = x + dt * v3
    a4 = f(x4)
    return x + dt / 6 * (v + 2 * v2 + 2 * v3 + v4), v + dt / 6 * (a1 + 2 * a2 + 2 * a3 + a4)


def test_symplectic_euler_c1(oracle):
    """3D, N=500 uniform in [0,1]^3, masses 1/N, G=1, softening 1e-3, p=6,
    leaf capacity 16, SyplecticEuler dt=1e-3 for 10 steps."""
    x, m = workloads.uniform_cube(500, seed=1)
    v = np.zeros_like(x)
    eps2 = 1e-6
    with fmmgpu.Context(dim=3, p=6, leaf_cap=16, G=1.0, eps2=eps2, direct_max=0) as c:
        xg, vg, _ = c.integrate(fmmgpu.FMM_INT_SYMPLECTIC_EULER, 1e-3, 10, x, v, m)
    # the same FMM (p, leaf capacity, softening) in FP64 on the CPU
    xc, vc = cpu_se(lambda y: oracle.fmm(y, m, 6, 16, eps2=eps2), x, v, 1e-3, 10)
    assert np.abs(xg - xc).max() < 1e-9
    assert np.abs(vg - vc).max() < 1e-6 * np.abs(vc).max()
    # and within the FMM's truncation error of the exact dynamics
    xd, vd = cpu_se(lambda y: oracle.direct(y, m, eps2=eps2), x, v, 1e-3, 10)
    assert np.abs(xg - xd).max() < 1e-6


def test_rk4_plummer(oracle):
    """One classical RK4 step on a Plummer sphere (the reference's
    RungeKutta4 aborts, runge_kutta_4.cpp:12-29, so the CPU side is the
    textbook scheme)."""
    x, m = workloads.plummer(4000, seed=2)
    v = np.random.default_rng(3).normal(size=x.shape) * 0.1
    with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0) as c:
        xg, vg, _ = c.integrate(fmmgpu.FMM_INT_RK4, 1e-4, 1, x, v, m)
    xc, vc = cpu_rk4(oracle, x, v, m, 1e-4, 0.0)
    assert np.abs(xg - xc).max() < 1e-10
    dv = np.linalg.norm(vg - vc) / np.linalg.norm(vc - v)
    assert dv < 1e-3


def test_two_bodies_approach():
    """tests/test_naive_update.cpp:13-55 of the reference, with the FMM."""
    x = np.array([[-10.0, 0, 0], [10.0, 0, 0]])
    v = np.zeros_like(x)
    m = np.array([1e9, 1e9])
    prev = 20.0
    with fmmgpu.Context(dim=3, p=4, leaf_cap=20, G=6.6743e-11) as c:
        for _ in range(20):
            x, v, _ = c.integrate(fmmgpu.FMM_INT_SYMPLECTIC_EULER, 0.5, 1, x, v, m)
            d = np.linalg.norm(x[1] - x[0])
            assert d < prev
            assert x[0, 0] > -10.0 and x[1, 0] < 10.0
            prev = d


def test_se_naive_matches_reference_trajectory():
    """The reference's own SyplecticEuler with NaiveUpdate (ref_naive.npz, 300
    particles, masses 1/300, 10 steps of 1e-3) and with heavy particles whose
    forces move the state (ref_se.npz, masses 1e8), replayed with the GPU's
    FP64 direct sum in NaiveUpdate's form (FMM_SOFT_NAIVE_REF) as the update
    method (symplectic_euler.cpp:8-15: v += dt a, then x += dt v)."""
    from conftest import golden

    for fx, pre, sfx in ((golden("ref_naive.npz"), "d3/", ("se_x", "se_v")),
                         (golden("ref_se.npz"), "naive3/", ("x", "v"))):
        G = float(fx["G"])
        x, v, m = fx[pre + "pos"].copy(), fx[pre + "vel"].copy(), fx[pre + "mass"]
        with fmmgpu.Context(dim=3, G=G) as c:
            for _ in range(10):
                v = v + 1e-3 * c.direct(x, m, soft_mode=fmmgpu.FMM_SOFT_NAIVE_REF)
                x = x + 1e-3 * v
        xr, vr = fx[pre + sfx[0]], fx[pre + sfx[1]]
        v0 = fx[pre + "vel"]
        np.testing.assert_allclose(x, xr, rtol=0, atol=1e-13)
        # the velocity change is the forces' doing: compared relative to itself
        dv, dvr = v - v0, vr - v0
        if pre == "naive3/":
            assert np.linalg.norm(dvr) > 1e-3 * np.linalg.norm(v0)  # the forces do move the state
            assert np.linalg.norm(dv - dvr) / np.linalg.norm(dvr) < 1e-10


def test_se_fmm_2d_matches_reference_trajectory():
    """fmm_integrate (SyplecticEuler, 2D FMM at p = 12, threshold 16) against
    the reference's SyplecticEuler driving its own 2D FMM::update on a
    uniform disk (ref_se.npz), where the reference's 2D FMM is accurate: the
    velocity changes agree within 1e-6 relative, the FP32 force bar."""
    from conftest import golden

    fx = golden("ref_se.npz")
    x0, v0, m = fx["fmm2/pos"], fx["fmm2/vel"], fx["fmm2/mass"]
    with fmmgpu.Context(dim=2, p=int(fx["fmm2/p"]), leaf_cap=int(fx["fmm2/T"]), G=float(fx["G"]), direct_max=0) as c:
        x, v, _ = c.integrate(fmmgpu.FMM_INT_SYMPLECTIC_EULER, 1e-3, 10, x0, v0, m)
    dv, dvr = v - v0, fx["fmm2/v"] - v0
    assert np.linalg.norm(dvr) > 1e-3 * np.linalg.norm(v0)
    assert np.linalg.norm(dv - dvr) / np.linalg.norm(dvr) < 1e-6
    dx, dxr = x - x0, fx["fmm2/x"] - x0
    assert np.linalg.norm(dx - dxr) / np.linalg.norm(dxr) < 1e-6
