"""Pins the CPU oracle (oracle/fmm_oracle.c) to the reference: its own
test_tree golden, fixtures generated from the reference built from source,
and, where that build is present, live comparisons."""
import json
import os
import subprocess

import numpy as np
import pytest
from conftest import GOLDEN, golden, rel_l2, tree_pairs_set

from fmmgpu import workloads


def test_tree_golden_15(oracle):
    """tests/test_tree.cpp:42-100 of the reference."""
    g = json.load(open(os.path.join(GOLDEN, "tree15.json")))
    pos = np.array([[float.fromhex(v) for v in row] for row in g["positions_hex"]])
    t = oracle.tree(pos, g["threshold"])
    assert t["depth"] == g["depth"] == 1
    got = {str(int(k)): t["perm"][s:e].tolist() for k, s, e in zip(t["leaf_keys"], t["leaf_start"][:-1], t["leaf_start"][1:])}
    assert got == g["leaves"]


def _cases():
    z = golden("ref_trees.npz")
    names = sorted({k.split("/")[0] for k in z.files})
    return z, names


@pytest.mark.parametrize("name", _cases()[1])
def test_tree_matches_reference_fixture(oracle, name):
    z = golden("ref_trees.npz")
    pos = z[f"{name}/pos"]
    t = oracle.tree(pos, int(z[f"{name}/T"]))
    D = int(z[f"{name}/depth"])
    assert t["depth"] == D
    np.testing.assert_array_equal(t["leaf_keys"], z[f"{name}/leaf_keys"])
    np.testing.assert_array_equal(t["leaf_start"], z[f"{name}/leaf_start"])
    np.testing.assert_array_equal(t["perm"], z[f"{name}/perm"])
    for d in range(D + 1):
        np.testing.assert_array_equal(t["level_keys"][d], z[f"{name}/level{d}"])
        for kind in (0, 1):
            key = f"{name}/pairs{d}_{kind}"
            if key not in z.files:
                continue
            want = set(zip(z[key][0].tolist(), z[key][1].tolist()))
            assert tree_pairs_set(t, d, kind) == want, (d, kind)


def test_morton_roundtrip(oracle):
    rng = np.random.default_rng(0)
    for dim, bits in ((3, 16), (2, 32)):
        for _ in range(200):
            c = rng.integers(0, 1 << bits, dim, dtype=np.uint64).astype(np.uint32)
            code = oracle.morton_encode(c)
            np.testing.assert_array_equal(oracle.morton_decode(code, dim), c)
    # bit b of coordinate i at bit i + b*dim (morton_code.cpp:13-20)
    assert oracle.morton_encode([1, 0, 0]) == 1
    assert oracle.morton_encode([0, 1, 0]) == 2
    assert oracle.morton_encode([0, 0, 1]) == 4
    assert oracle.morton_encode([2, 0, 0]) == 8
    assert oracle.morton_encode([0, 0, 1 << 15]) == 1 << 47


def test_harmonics_match_reference(oracle):
    z = golden("ref_harm.npz")
    p = int(z["p"])
    for v, r, i in zip(z["vecs"], z["regular"], z["irregular"]):
        np.testing.assert_allclose(oracle.regular_racah(p, v), r, rtol=1e-12, atol=1e-12 * np.abs(r).max())
        np.testing.assert_allclose(oracle.irregular_racah(p, v), i, rtol=1e-12, atol=1e-12 * np.abs(i).max())


def test_p2m_matches_reference(oracle):
    """MultipoleSet<3> += PowerSet<3> (multipole_set3D.cpp:31-43) stores
    sum q R_n^{-m}(x - c) = (-1)^m sqrt((n-m)!(n+m)!) M_n^m in the project's
    scaled convention."""
    from math import factorial, sqrt

    z = golden("ref_harm.npz")
    p = 8
    M = oracle.p2m_3d(p, z["p2m_pos"], z["p2m_mass"], z["p2m_centre"])
    ref = z["p2m"]
    for n in range(p + 1):
        for m in range(-n, n + 1):
            am = abs(m)
            v = M[n * (n + 1) // 2 + am]
            if m < 0:
                v = (-1) ** am * np.conj(v)
            want = (-1) ** m * sqrt(factorial(n - m) * factorial(n + m)) * v
            if n == 0:
                assert abs(ref[0] - want.real) < 1e-12
                continue
            idx = 2 * n * n + 2 * n + 2 * m - 1
            assert abs(ref[idx] - want.real) < 1e-11 * max(1, abs(want))
            assert abs(ref[idx + 1] - want.imag) < 1e-11 * max(1, abs(want))


def test_near_field_matches_reference(oracle):
    z = golden("ref_near3d.npz")
    g = oracle.fmm(z["pos"], z["mass"], 0, int(z["T"]))
    np.testing.assert_allclose(g, z["grad"], rtol=1e-10, atol=1e-10 * np.abs(z["grad"]).max())


@pytest.mark.parametrize("p", [2, 8, 15])
def test_fmm2d_matches_reference(oracle, p):
    """2D with the reference's mass centres reproduces FMM::update."""
    z = golden("ref_fmm2d.npz")
    g = oracle.fmm(z["pos"], z["mass"], p, 16, centre_mode=1)
    assert rel_l2(g, z[f"p{p}"]) < 1e-12


def test_naive_matches_reference(oracle):
    z = golden("ref_naive.npz")
    for dim in (2, 3):
        g = oracle.naive_ref(z[f"d{dim}/pos"], z[f"d{dim}/mass"])
        np.testing.assert_allclose(g, z[f"d{dim}/grad"], rtol=1e-12, atol=1e-14)


def test_fmm3d_converges_to_direct(oracle):
    """The project's 3D operators converge with p (the reference's stay near 1e-1)."""
    pos, m = workloads.uniform_cube(1500, seed=5)
    gd = oracle.direct(pos, m)
    errs = [rel_l2(oracle.fmm(pos, m, p, 16), gd) for p in (2, 4, 6, 8)]
    assert all(b < a / 3 for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 5e-5


def test_fmm_potential_converges(oracle):
    pos, m = workloads.plummer(1500, seed=6)
    gd, pd = oracle.direct(pos, m, want_pot=True)
    g, pt = oracle.fmm(pos, m, 10, 16, want_pot=True)
    assert rel_l2(g, gd) < 3e-5
    assert rel_l2(pt, pd) < 3e-6


def test_fmm2d_geometric_centres_converge(oracle):
    pos, m = workloads.uniform_disk_2d(2000, seed=8)
    gd, pd = oracle.direct(pos, m, want_pot=True)
    g, pt = oracle.fmm(pos, m, 15, 16, centre_mode=0, want_pot=True)
    assert rel_l2(g, gd) < 1e-7
    assert rel_l2(pt, pd) < 1e-7


def test_reference_zero_extent_axis(oracle):
    """All particles on a plane: the reference divides 0/0 on that axis
    (tree.cpp:49,58) which its x86 build turns into coordinate 0."""
    pos, _ = workloads.uniform_cube(200, seed=9)
    pos[:, 2] = 0.25
    t = oracle.tree(pos, 8)
    assert all(int(k) & 4 == 0 for k in t["leaf_keys"])  # z bit 0 never set


def test_reference_live(oracle, reflib):
    """Live comparison against the reference build on fresh inputs."""
    rng = np.random.default_rng(99)
    for dim, n, T in ((3, 1200, 12), (2, 1500, 10)):
        pos = rng.random((n, dim)) * 3 - 1
        a, b = oracle.tree(pos, T), reflib.tree(pos, T)
        assert a["depth"] == b["depth"]
        np.testing.assert_array_equal(a["perm"], b["perm"])
        np.testing.assert_array_equal(a["leaf_keys"], b["leaf_keys"])
        for d in range(a["depth"] + 1):
            for kind in (0, 1):
                assert tree_pairs_set(a, d, kind) == tree_pairs_set(b, d, kind)
    pos = rng.random((800, 2))
    m = rng.random(800)
    assert rel_l2(oracle.fmm(pos, m, 10, 16, centre_mode=1), reflib.fmm(pos, m, 10, 16)) < 1e-12


def test_reference_own_tests_pass():
    """The reference's five gtest files, built against the project's gtest
    stand-in, pass on the reference built from source."""
    d = os.path.join(os.path.dirname(GOLDEN), "..", "oracle", "_ref")
    bins = ["test_tensor", "test_naive_update", "test_tree", "test_fmm_vs_naive_2d", "test_fmm_vs_naive_3d"]
    if not all(os.path.exists(os.path.join(d, b)) for b in bins):
        pytest.skip("reference tests not built")
    for b in bins:
        r = subprocess.run([os.path.join(d, b)], capture_output=True, timeout=120)
        assert r.returncode == 0, (b, r.stderr[-500:])


def test_oracle_converges_on_an_elongated_box(oracle):
    """Interaction pairs that are not well separated for the box's aspect
    ratio are summed directly, so the FMM error falls as p rises even when
    the bounding box is far from cubic."""
    from fmmgpu import workloads

    pos, m = workloads.plummer(1457, seed=1138)
    ext = pos.max(0) - pos.min(0)
    assert ext.max() / ext.min() > 1.5
    ref = oracle.direct(pos, m)
    errs = [rel_l2(oracle.fmm(pos, m, p, 64), ref) for p in (4, 8, 12)]
    assert errs[0] > errs[1] > errs[2] and errs[2] < 2e-6, errs


@pytest.mark.parametrize("gen,n,T", [("plummer", 3000, 16), ("plummer_mixture", 4000, 16), ("uniform3d", 2000, 8),
                                     ("disk_clumps2d", 3000, 16), ("disk2d", 2000, 8)])
def test_adaptive_targets_partition_the_pairs_exactly(oracle, gen, n, T):
    """orc_fmm_adaptive with every interaction-list pair and every W-list
    child summed directly is the direct sum: the adaptive leaves' lists and
    colleague sums cover every pair exactly once."""
    pos, m = workloads.WORKLOADS[gen](n, seed=3)
    d, pd = oracle.direct(pos, m, want_pot=True)
    big = 10 ** 18
    g, pg = oracle.fmm_adaptive(pos, m, 4, T, direct_max=big, w_direct_max=big, want_pot=True)
    assert rel_l2(g, d) < 1e-12 and rel_l2(pg, pd) < 1e-12


@pytest.mark.parametrize("gen,n,T", [("plummer", 3000, 16), ("plummer_mixture", 4000, 16), ("disk_clumps2d", 4000, 16)])
def test_adaptive_targets_converge_like_the_uniform_fmm(oracle, gen, n, T):
    """Adaptive targets (multipoles of far W-list children included) converge
    with p, as accurately as the uniform-depth FMM with the same
    direct-pair rule."""
    pos, m = workloads.WORKLOADS[gen](n, seed=3)
    d = oracle.direct(pos, m)
    errs = []
    for p in (4, 8, 12):
        ga = oracle.fmm_adaptive(pos, m, p, T, direct_max=256, w_direct_max=256)
        gu = oracle.fmm(pos, m, p, T, direct_max=256)
        errs.append(rel_l2(ga, d))
        assert errs[-1] < 1.5 * rel_l2(gu, d) + 1e-7, (p, errs[-1], rel_l2(gu, d))
    assert errs[0] > errs[1] > errs[2]


@pytest.mark.parametrize("gen", ["plummer", "disk_clumps2d"])
def test_adaptive_w_list_multipoles_converge(oracle, gen):
    """Every far W-list child evaluated through its multipole (M2P,
    w_direct_max = 0) converges with p and stays within a few times the
    error with every W-list child summed directly."""
    pos, m = workloads.WORKLOADS[gen](4000, seed=3)
    d = oracle.direct(pos, m)
    errs = []
    for p in (4, 8, 16):
        gw = oracle.fmm_adaptive(pos, m, p, 16, direct_max=256, w_direct_max=0)
        gd = oracle.fmm_adaptive(pos, m, p, 16, direct_max=256, w_direct_max=10 ** 18)
        errs.append(rel_l2(gw, d))
        assert rel_l2(gw, gd) > 0  # the multipoles were used
        assert errs[-1] < 5 * rel_l2(gd, d) + 1e-9, (p, errs[-1], rel_l2(gd, d))
    assert errs[0] > 10 * errs[1] > 100 * errs[2]


@pytest.mark.parametrize("gen,n,T,A", [("plummer_mixture", 20000, 16, 32), ("plummer", 20000, 32, 64),
                                       ("uniform3d", 5000, 8, 8), ("disk_clumps2d", 20000, 16, 32)])
def test_adaptive_flags_have_a_closed_form(oracle, gen, n, T, A):
    """The adaptive targets' top-down rule (orc_fmm_adaptive) equals a rule
    a GPU can apply to every cell at once: a cell is an active target iff it
    is the root or its parent holds more than A particles; an adaptive leaf
    iff it is active and holds at most A particles or is at the leaf level.
    (A cell's particles are a subset of its parent's.)  The adaptive leaves
    partition the particles."""
    pos, m = workloads.WORKLOADS[gen](n, seed=3)
    dim = pos.shape[1]
    t = oracle.tree(pos, T)
    D, keys = t["depth"], t["level_keys"]
    flags = oracle.adaptive_flags(pos, T, A)
    leaf_cnt = np.diff(t["leaf_start"])
    cnt = [np.bincount(np.searchsorted(keys[d], t["leaf_keys"] >> np.uint64(dim * (D - d))), weights=leaf_cnt,
                       minlength=len(keys[d])).astype(np.int64) for d in range(D + 1)]
    covered = 0
    for d in range(D + 1):
        if d == 0:
            act = np.ones(len(keys[0]), bool)
        else:
            parent = np.searchsorted(keys[d - 1], keys[d] >> np.uint64(dim))
            act = cnt[d - 1][parent] > A
        leaf = act & ((cnt[d] <= A) | (d == D))
        np.testing.assert_array_equal(flags[d] & 1, act.astype(np.uint8))
        np.testing.assert_array_equal((flags[d] >> 1) & 1, leaf.astype(np.uint8))
        covered += int(cnt[d][leaf].sum())
    assert covered == n


def test_oracle_se_matches_reference_trajectories(oracle):
    """The oracle's NaiveUpdate and 2D FMM (mass centres, as the reference
    forms them) driving SyplecticEuler (symplectic_euler.cpp:8-15) reproduce
    the reference's own trajectories in ref_se.npz."""
    z = golden("ref_se.npz")
    G = float(z["G"])

    def se(force, x, v):
        for _ in range(10):
            v = v + 1e-3 * G * force(x)
            x = x + 1e-3 * v
        return x, v

    m = z["naive3/mass"]
    x, v = se(lambda y: oracle.naive_ref(y, m), z["naive3/pos"], z["naive3/vel"])
    assert rel_l2(v - z["naive3/vel"], z["naive3/v"] - z["naive3/vel"]) < 1e-12
    assert np.abs(x - z["naive3/x"]).max() < 1e-13
    m = z["fmm2/mass"]
    p, T = int(z["fmm2/p"]), int(z["fmm2/T"])
    x, v = se(lambda y: oracle.fmm(y, m, p, T, centre_mode=1), z["fmm2/pos"], z["fmm2/vel"])
    assert rel_l2(v - z["fmm2/vel"], z["fmm2/v"] - z["fmm2/vel"]) < 1e-10
    assert rel_l2(x - z["fmm2/pos"], z["fmm2/x"] - z["fmm2/pos"]) < 1e-10


def test_oracle_tree_matches_reference_at_2p20(oracle):
    """The oracle's tree of the 2^20 Plummer sphere (seed 2, threshold 64,
    depth 10) has the reference's depth, level sizes and leaf arrays
    (SHA-256 digests in ref_tree_c2.json, from the compiled reference)."""
    import hashlib
    import json

    from fmmgpu import workloads

    g = json.load(open(os.path.join(GOLDEN, "ref_tree_c2.json")))
    pos, _ = workloads.plummer(1 << 20, seed=2)
    t = oracle.tree(pos, g["threshold"], with_pairs=False)
    assert t["depth"] == g["depth"]
    assert [len(k) for k in t["level_keys"]] == g["level_sizes"]
    got = {"leaf_keys": hashlib.sha256(np.asarray(t["leaf_keys"], "<u8").tobytes()).hexdigest(),
           "leaf_start": hashlib.sha256(np.asarray(t["leaf_start"], "<i8").tobytes()).hexdigest(),
           "perm": hashlib.sha256(np.asarray(t["perm"], "<i8").tobytes()).hexdigest()}
    assert got == g["sha256"]
