"""Parity of the CUDA path (through the C ABI) with the oracle and the
reference fixtures.  Tolerances:
  - tree build: bit-exact (depth, leaf keys, membership order, lists);
  - FP64 direct sum: 1e-12 relative to the CPU FP64 sum;
  - FMM in FP32 mode vs the FP64 oracle FMM with the same p, leaf capacity
    and direct-pair rule: relative L2 force error <= 1e-6 (the bar for the
    FP32 mode); largest per-particle error <= 2e-5 of the RMS acceleration;
  - FMM vs FP64 direct sum: within 1.5x the oracle's own truncation error
    plus 1e-6.
"""
import json
import os

import numpy as np
import pytest
from conftest import GOLDEN, golden, rel_l2, tree_pairs_set

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx3():
    c = fmmgpu.Context(dim=3, p=8, leaf_cap=64)
    yield c
    c.close()


def _assert_same_tree(got, want_depth, want_keys, want_start, want_perm):
    assert got["depth"] == want_depth
    np.testing.assert_array_equal(got["leaf_keys"], want_keys)
    np.testing.assert_array_equal(got["leaf_start"], want_start)
    np.testing.assert_array_equal(got["perm"], want_perm)


def test_tree_golden_15():
    """The reference's tests/test_tree.cpp:42-100."""
    g = json.load(open(os.path.join(GOLDEN, "tree15.json")))
    pos = np.array([[float.fromhex(v) for v in row] for row in g["positions_hex"]])
    with fmmgpu.Context(dim=3, leaf_cap=g["threshold"]) as c:
        t = c.tree(pos)
    assert t["depth"] == 1
    got = {str(int(k)): t["perm"][s:e].tolist() for k, s, e in zip(t["leaf_keys"], t["leaf_start"][:-1], t["leaf_start"][1:])}
    assert got == g["leaves"]


def _tree_cases():
    z = golden("ref_trees.npz")
    return sorted({k.split("/")[0] for k in z.files})


@pytest.mark.parametrize("name", _tree_cases())
def test_tree_matches_reference_fixture(name):
    z = golden("ref_trees.npz")
    pos = z[f"{name}/pos"]
    dim = pos.shape[1]
    with fmmgpu.Context(dim=dim, leaf_cap=int(z[f"{name}/T"])) as c:
        t = c.tree(pos)
    D = int(z[f"{name}/depth"])
    _assert_same_tree(t, D, z[f"{name}/leaf_keys"], z[f"{name}/leaf_start"], z[f"{name}/perm"])
    for d in range(D + 1):
        np.testing.assert_array_equal(t["level_keys"][d], z[f"{name}/level{d}"])
        for kind in (0, 1):
            key = f"{name}/pairs{d}_{kind}"
            if key in z.files:
                assert tree_pairs_set(t, d, kind) == set(zip(z[key][0].tolist(), z[key][1].tolist())), (d, kind)


def test_tree_matches_reference_at_2p20():
    """The tree of the 2^20 Plummer sphere at threshold 64 (seed 2), depth
    10, where the reference's 32-bit list keys (node_i.cpp:31,63) are at
    their limit: depth, level sizes and the SHA-256 of the leaf keys, leaf
    starts and membership equal the reference's Tree::init_tree
    (ref_tree_c2.json, generated from the compiled reference)."""
    import hashlib

    g = json.load(open(os.path.join(GOLDEN, "ref_tree_c2.json")))
    pos, _ = workloads.plummer(1 << 20, seed=2)
    with fmmgpu.Context(dim=3, leaf_cap=g["threshold"]) as c:
        t = c.tree(pos, with_pairs=False)
    assert t["depth"] == g["depth"] == 10
    assert [len(k) for k in t["level_keys"]] == g["level_sizes"]
    got = {"leaf_keys": hashlib.sha256(np.asarray(t["leaf_keys"], "<u8").tobytes()).hexdigest(),
           "leaf_start": hashlib.sha256(np.asarray(t["leaf_start"], "<i8").tobytes()).hexdigest(),
           "perm": hashlib.sha256(np.asarray(t["perm"], "<i8").tobytes()).hexdigest()}
    assert got == g["sha256"]


@pytest.mark.parametrize("gen,n,T", [("uniform3d", 30000, 16), ("plummer", 50000, 64), ("plummer", 20000, 4)])
def test_tree_matches_oracle(oracle, gen, n, T):
    pos, _ = workloads.WORKLOADS[gen](n, seed=3)
    with fmmgpu.Context(dim=3, leaf_cap=T) as c:
        t = c.tree(pos)
    o = oracle.tree(pos, T)
    _assert_same_tree(t, o["depth"], o["leaf_keys"], o["leaf_start"], o["perm"])
    for d in range(o["depth"] + 1):
        np.testing.assert_array_equal(t["level_keys"][d], o["level_keys"][d])
        for kind in (0, 1):
            assert tree_pairs_set(t, d, kind) == tree_pairs_set(o, d, kind), (d, kind)


@pytest.mark.parametrize("nclump", [400, 700])
def test_tree_dense_clump_matches_oracle(oracle, nclump):
    """A clump of nclump particles inside one cell of the maximum depth: the
    depth loop runs to depth 16 and that leaf holds all of them.  Up to 512
    particles per leaf the Dmax order is put back in input order inside each
    leaf; above that the leaf keys are sorted afresh from input order.  Both
    paths must give the oracle's tree bit for bit."""
    rng = np.random.default_rng(11)
    pos = rng.random((3000, 3))
    clump = 0.4 + 1e-7 * rng.random((nclump, 3))
    pos = np.concatenate([pos, clump])[rng.permutation(3000 + nclump)]  # the clump spread over the input order
    with fmmgpu.Context(dim=3, leaf_cap=16) as c:
        t = c.tree(pos)
    o = oracle.tree(pos, 16)
    assert o["depth"] == 16 and int(np.diff(o["leaf_start"]).max()) == nclump
    _assert_same_tree(t, o["depth"], o["leaf_keys"], o["leaf_start"], o["perm"])
    for d in range(o["depth"] + 1):
        np.testing.assert_array_equal(t["level_keys"][d], o["level_keys"][d])


def test_direct_matches_oracle(oracle):
    pos, m = workloads.plummer(3000, seed=4)
    with fmmgpu.Context(dim=3, G=1.0) as c:
        a, ph = c.direct(pos, m, want_pot=True)
        tg = np.array([0, 17, 2999, 1500])
        at = c.direct(pos, m, targets=tg)
    g, po = oracle.direct(pos, m, want_pot=True)
    assert rel_l2(a, g) < 1e-12
    assert rel_l2(ph, po) < 1e-12
    assert rel_l2(at, g[tg]) < 1e-12


def test_direct_naive_softening_matches_reference():
    """FMM_SOFT_NAIVE_REF reproduces NaiveUpdate::update (naive_update.cpp:19-30)."""
    z = golden("ref_naive.npz")
    pos, m = z["d3/pos"], z["d3/mass"]
    with fmmgpu.Context(dim=3, G=1.0) as c:
        a = c.direct(pos, m, soft_mode=fmmgpu.FMM_SOFT_NAIVE_REF)
    np.testing.assert_allclose(a, z["d3/grad"], rtol=1e-11, atol=1e-13)


def _check_parity(a, ph, g, po):
    e = rel_l2(a, g)
    assert e < 1e-6, e
    rms = np.sqrt((g * g).sum(axis=1).mean())
    worst = np.linalg.norm(a - g, axis=1).max() / rms
    assert worst < 2e-5, worst
    assert rel_l2(ph, po) < 1e-6


@pytest.mark.parametrize("gen,n,p,T", [("uniform3d", 4000, 4, 16), ("uniform3d", 6000, 8, 16), ("plummer", 8000, 8, 32),
                                       ("plummer", 5000, 6, 64), ("uniform3d", 3000, 10, 20)])
def test_fmm_matches_oracle(oracle, gen, n, p, T):
    """Every interaction-list pair through M2L, as the reference does."""
    pos, m = workloads.WORKLOADS[gen](n, seed=5)
    with fmmgpu.Context(dim=3, p=p, leaf_cap=T, G=1.0, direct_max=0) as c:
        a, ph = c.evaluate(pos, m, want_pot=True)
    g, po = oracle.fmm(pos, m, p, T, want_pot=True)
    _check_parity(a, ph, g, po)


@pytest.mark.parametrize("gen,n,p,T,dm", [("plummer", 8000, 8, 64, 256), ("uniform3d", 6000, 6, 16, 64),
                                          ("plummer", 20000, 8, 64, 4096)])
def test_fmm_hybrid_matches_oracle(oracle, gen, n, p, T, dm):
    """Small interaction pairs summed directly: same rule in the oracle."""
    pos, m = workloads.WORKLOADS[gen](n, seed=11)
    with fmmgpu.Context(dim=3, p=p, leaf_cap=T, G=1.0, direct_max=dm) as c:
        a, ph = c.evaluate(pos, m, want_pot=True)
        s = c.stats()
    g, po = oracle.fmm(pos, m, p, T, want_pot=True, direct_max=dm)
    _check_parity(a, ph, g, po)
    with fmmgpu.Context(dim=3, p=p, leaf_cap=T, G=1.0, direct_max=0) as c:
        c.evaluate(pos, m)
        s0 = c.stats()
    assert s["m2l_pairs"] < s0["m2l_pairs"] and s["p2p_pairs"] > s0["p2p_pairs"]


@pytest.mark.parametrize("n,p,T,mode", [(30000, 8, 256, fmmgpu.FMM_M2L_FP32), (20000, 12, 128, fmmgpu.FMM_M2L_TC)])
def test_fmm_large_leaves_match_oracle(oracle, n, p, T, mode):
    """Leaf capacities the autotuner may choose (128, 256) on a clustered
    input: leaves of up to 130 particles take their multipoles in several
    32-particle chunks, and the few M2L batches of a small tree are split
    into runs of slots on the tensor cores."""
    pos, m = workloads.plummer_mixture(n, seed=13)
    with fmmgpu.Context(dim=3, p=p, leaf_cap=T, G=1.0, direct_max=256, m2l_mode=mode) as c:
        a, ph = c.evaluate(pos, m, want_pot=True)
    g, po = oracle.fmm(pos, m, p, T, want_pot=True, direct_max=256)
    _check_parity(a, ph, g, po)


def test_fmm_near_field_matches_reference():
    """p = 0: the far field's gradient vanishes and what remains is the
    reference's near-field sum (leaf.cpp:118-142), checked on its fixture."""
    z = golden("ref_near3d.npz")
    with fmmgpu.Context(dim=3, p=0, leaf_cap=int(z["T"]), G=1.0, direct_max=0) as c:
        a = c.evaluate(z["pos"], z["mass"])
    assert rel_l2(a, z["grad"]) < 1e-6


@pytest.mark.parametrize("p", [4, 8, 12])
def test_fmm_error_vs_direct(oracle, p):
    """Default settings (automatic direct-pair rule) against the FP64 sum."""
    pos, m = workloads.plummer(20000, seed=6)
    with fmmgpu.Context(dim=3, p=p, leaf_cap=64, G=1.0) as c:
        a = c.evaluate(pos, m)
        tg = np.arange(0, 20000, 7)
        d = c.direct(pos, m, targets=tg)
    og = oracle.fmm(pos, m, p, 64)  # every pair by M2L: the hybrid must do no worse
    e_orc = rel_l2(og[tg], d)
    e_gpu = rel_l2(a[tg], d)
    assert e_gpu < 1.5 * e_orc + 1e-6, (e_gpu, e_orc)


def test_gravitational_constant_scales():
    pos, m = workloads.uniform_cube(2000, seed=7)
    with fmmgpu.Context(dim=3, p=6, leaf_cap=16, G=1.0) as c:
        a1 = c.evaluate(pos, m)
    with fmmgpu.Context(dim=3, p=6, leaf_cap=16, G=6.6743e-11) as c:
        a2 = c.evaluate(pos, m)
    np.testing.assert_allclose(a2, a1 * 6.6743e-11, rtol=1e-12)


def test_repeatable_and_reusable(ctx3):
    pos, m = workloads.plummer(30000, seed=8)
    a = ctx3.evaluate(pos, m)
    b = ctx3.evaluate(pos, m)
    # P2M sums a leaf that straddles two warps with FP32 atomics, so repeats
    # agree to rounding, not bit for bit
    assert rel_l2(b, a) < 1e-7
    small = ctx3.evaluate(pos[:100], m[:100])
    assert small.shape == (100, 3)
    c = ctx3.evaluate(pos, m)
    assert rel_l2(c, a) < 1e-7


def test_edge_cases():
    with fmmgpu.Context(dim=3, p=4, leaf_cap=8) as c:
        assert c.evaluate(np.zeros((0, 3)), np.zeros(0)).shape == (0, 3)
        np.testing.assert_array_equal(c.evaluate(np.array([[0.3, 0.1, 0.2]]), np.array([1.0])), 0.0)
        a = c.evaluate(np.array([[0.0, 0, 0], [1.0, 0, 0]]), np.array([1.0, 2.0]))
        np.testing.assert_allclose(a, [[2.0, 0, 0], [-1.0, 0, 0]], rtol=1e-6)
        # every particle on one plane (zero-extent axis, tree.cpp:49)
        pos, m = workloads.uniform_cube(3000, seed=9)
        pos[:, 2] = 0.5
        a = c.evaluate(pos, m)
        d = c.direct(pos, m)
        assert rel_l2(a, d) < 1e-3
        # coincident particles: the reference divides by zero; reported
        with pytest.raises(fmmgpu.FmmError) as e:
            c.evaluate(np.array([[0.1, 0.1, 0.1], [0.1, 0.1, 0.1], [0.5, 0.5, 0.5]]), np.ones(3))
        assert e.value.code == fmmgpu.FMM_ERR_NONFINITE_OUTPUT
        bad = np.array([[0.1, np.nan, 0.1], [0.2, 0.2, 0.2]])
        with pytest.raises(fmmgpu.FmmError) as e:
            c.evaluate(bad, np.ones(2))
        assert e.value.code == fmmgpu.FMM_ERR_NONFINITE_INPUT
        # still usable after the errors
        a = c.evaluate(np.array([[0.0, 0, 0], [1.0, 0, 0]]), np.array([1.0, 2.0]))
        np.testing.assert_allclose(a[0], [2.0, 0, 0], rtol=1e-6)


def test_reference_fmm_vs_naive_3d_case():
    """The reference's tests/test_fmm_vs_naive_3d.cpp setting (100 particles
    in [-50,50]^3, mass 1e9, p = 2, threshold 20) with its 1e-2 tolerance
    against NaiveUpdate."""
    from oracle import RAND_MAX, glibc_rand_sequence

    r = glibc_rand_sequence(42, 600)
    pos = np.zeros((100, 3))
    for i in range(100):
        pos[i] = (r[6 * i: 6 * i + 3] * 2.0 * 50.0) / RAND_MAX - 50.0
    m = np.full(100, 1e9)
    with fmmgpu.Context(dim=3, p=2, leaf_cap=20, G=6.6743e-11) as c:
        a = c.evaluate(pos, m)
        d = c.direct(pos, m, soft_mode=fmmgpu.FMM_SOFT_NAIVE_REF)
    assert np.abs(a - d).max() < 1e-2


def test_stats_and_launches(ctx3):
    pos, m = workloads.plummer(20000, seed=10)
    n0 = ctx3.launch_count()
    ctx3.evaluate(pos, m)
    s = ctx3.stats()
    assert s["depth"] >= 2 and s["n_leaves"] > 0 and s["ms_total"] > 0
    assert ctx3.launch_count() > n0


def test_elongated_box_converges_and_matches_oracle(oracle):
    """A small Plummer sample whose bounding box is far from cubic: the
    offsets that are not well separated for that aspect go to the direct far
    field on the GPU and in the oracle alike."""
    pos, m = workloads.plummer(1457, seed=1138)
    ref = oracle.direct(pos, m)
    errs = []
    for p in (8, 12):
        for mode in (fmmgpu.FMM_M2L_FP32, fmmgpu.FMM_M2L_TC):
            with fmmgpu.Context(dim=3, p=p, leaf_cap=64, G=1.0, direct_max=0, m2l_mode=mode) as c:
                a = c.evaluate(pos, m)
            assert rel_l2(a, oracle.fmm(pos, m, p, 64)) < 1e-6
        errs.append(rel_l2(a, ref))
    assert errs[1] < errs[0] < 2e-5
