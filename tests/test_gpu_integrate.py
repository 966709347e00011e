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
