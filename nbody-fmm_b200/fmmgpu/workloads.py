"""Seeded synthetic particle sets for the FMM force pass.

The reference draws its inputs with glibc rand() inside its tests and in
src/main.cpp:36-96; it ships no dataset.  These generators produce the
distributions the benchmark configurations name, from numpy's PCG64 with a
fixed seed, as row-major (n, dim) FP64 positions and (n,) FP64 masses.
"""
import numpy as np


def uniform_cube(n, seed=1, dim=3):
    """Positions uniform in [0,1]^dim, masses 1/n."""
    rng = np.random.default_rng(seed)
    return rng.random((n, dim)), np.full(n, 1.0 / n)


def plummer(n, seed=2, a=1.0, rmax=20.0, centre=(0.0, 0.0, 0.0), total_mass=1.0):
    """Plummer sphere: r = a (U^(-2/3) - 1)^(-1/2), rejected above rmax,
    isotropic direction; equal masses summing to total_mass."""
    rng = np.random.default_rng(seed)
    r = np.empty(0)
    while r.size < n:
        u = rng.random(2 * (n - r.size) + 16)
        u = u[u > 0]
        rr = a / np.sqrt(u ** (-2.0 / 3.0) - 1.0)
        r = np.concatenate([r, rr[rr <= rmax]])
    r = r[:n]
    cz = rng.uniform(-1.0, 1.0, n)
    ph = rng.uniform(0.0, 2.0 * np.pi, n)
    sz = np.sqrt(1.0 - cz * cz)
    pos = np.stack([r * sz * np.cos(ph), r * sz * np.sin(ph), r * cz], axis=1) + np.asarray(centre)
    return pos, np.full(n, total_mass / n)


def disk_clumps_2d(n, seed=3, nclumps=64, sigma=0.005):
    """2D: half uniform in the unit disk, half in Gaussian clumps (sigma)
    whose centres are uniform in the disk; log-normal(0, 0.5) masses
    normalised to 1."""
    rng = np.random.default_rng(seed)
    nu = n // 2
    rad = np.sqrt(rng.random(nu))
    th = rng.uniform(0, 2 * np.pi, nu)
    a = np.stack([rad * np.cos(th), rad * np.sin(th)], axis=1)
    crad = np.sqrt(rng.random(nclumps))
    cth = rng.uniform(0, 2 * np.pi, nclumps)
    cc = np.stack([crad * np.cos(cth), crad * np.sin(cth)], axis=1)
    which = rng.integers(0, nclumps, n - nu)
    b = cc[which] + rng.normal(0.0, sigma, (n - nu, 2))
    pos = np.concatenate([a, b])
    m = rng.lognormal(0.0, 0.5, n)
    return pos, m / m.sum()


def uniform_disk_2d(n, seed=3):
    rng = np.random.default_rng(seed)
    rad = np.sqrt(rng.random(n))
    th = rng.uniform(0, 2 * np.pi, n)
    return np.stack([rad * np.cos(th), rad * np.sin(th)], axis=1), np.full(n, 1.0 / n)


def plummer_mixture(n, seed=5, nspheres=32, amin=0.01, amax=0.1):
    """32 Plummer spheres, scale radii log-uniform in [amin, amax], centres
    uniform in [0,1]^3, equal total mass per sphere (sum 1)."""
    rng = np.random.default_rng(seed)
    counts = np.full(nspheres, n // nspheres)
    counts[: n - counts.sum()] += 1
    parts = []
    for s in range(nspheres):
        a = float(np.exp(rng.uniform(np.log(amin), np.log(amax))))
        c = rng.random(3)
        p, _ = plummer(int(counts[s]), seed=int(rng.integers(1 << 31)), a=a, rmax=20.0 * a, centre=c)
        parts.append(p)
    pos = np.concatenate(parts)
    mass = np.concatenate([np.full(k, 1.0 / nspheres / k) for k in counts])
    return pos, mass


def ensemble_sizes(nsys=256, lo=1024, hi=65536, seed=4):
    """Per-system sizes floor(exp(U[ln lo, ln hi]))."""
    rng = np.random.default_rng(seed)
    return np.floor(np.exp(rng.uniform(np.log(lo), np.log(hi), nsys))).astype(np.int64)


WORKLOADS = {
    "uniform3d": uniform_cube,
    "plummer": plummer,
    "disk_clumps2d": disk_clumps_2d,
    "disk2d": uniform_disk_2d,
    "plummer_mixture": plummer_mixture,
}
