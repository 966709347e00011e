"""Adaptive targets on the GPU (fmm_config.adaptive_leaf = A), through the
C ABI, against the oracle's orc_fmm_adaptive with every W-list child summed
directly (the GPU sums every colleague of an adaptive leaf particle by
particle).

Tolerances, as for the uniform FMM in FP32 mode:
  - per-cell flags: bit-exact against orc_adaptive_flags;
  - forces and potentials: relative L2 <= 1e-6 against the FP64 oracle at
    the same p, leaf capacity, A and direct-pair rule; largest per-particle
    force error <= 2e-5 of the larger of the particle's own acceleration and
    the RMS acceleration (an adaptive leaf in a dense clump sums thousands of
    colleague pairs in FP32, so its particles' rounding error scales with
    their own, far above average, accelerations);
  - every output element written (outputs filled with NaN beforehand);
  - A >= n (the root is the only adaptive leaf: all pairs direct) within
    2e-5 of the FP64 direct sum: each particle's sum then runs over all
    n - 1 others in FP32 (chunks of 256 sources added into FP32
    accumulators), and that accumulation alone rounds at about
    sqrt(n) * 2^-24 on this clustered input.

The reference has no adaptive mode: its targets are every cell of its
uniform-depth tree (src/system_updaters/tree_components/tree.cpp:43-69,
node_i.cpp:105-120); this mode keeps that tree and stops the targets early.
"""
import numpy as np
import pytest
from conftest import rel_l2

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu

W_ALL_DIRECT = 10 ** 18


@pytest.mark.parametrize("gen,n,T,A", [("plummer", 20000, 16, 16), ("plummer_mixture", 30000, 32, 32),
                                       ("uniform3d", 8000, 8, 64), ("plummer_mixture", 40000, 128, 256)])
def test_flags_match_oracle(oracle, gen, n, T, A):
    pos, _ = workloads.WORKLOADS[gen](n, seed=11)
    with fmmgpu.Context(dim=3, leaf_cap=T) as c:
        t = c.tree(pos, with_pairs=False)
        got = c.adaptive_flags(A)
    want = oracle.adaptive_flags(pos, T, A)
    assert len(got) == len(want) == t["depth"] + 1
    for d in range(len(want)):
        np.testing.assert_array_equal(got[d], want[d], err_msg=f"level {d}")
    # the adaptive leaves partition the particles: each particle lies in
    # exactly one of them
    D = t["depth"]
    pkey = np.repeat(t["leaf_keys"], np.diff(t["leaf_start"]))  # leaf key of each particle, leaf order
    hits = np.zeros(n, np.int64)
    for d in range(D + 1):
        leaves = t["level_keys"][d][(got[d] & 2) != 0]
        hits += np.isin(pkey >> np.uint64(3 * (D - d)), leaves)
    assert (hits == 1).all()


def _check(a, ph, g, po):
    e = rel_l2(a, g)
    assert e < 1e-6, e
    rms = np.sqrt((g * g).sum(axis=1).mean())
    worst = (np.linalg.norm(a - g, axis=1) / np.maximum(np.linalg.norm(g, axis=1), rms)).max()
    assert worst < 2e-5, worst
    assert rel_l2(ph, po) < 1e-6


CASES = [("plummer", 8000, 8, 16, 16, 256), ("plummer_mixture", 20000, 10, 32, 32, 512),
         ("uniform3d", 6000, 8, 8, 32, 0), ("plummer_mixture", 40000, 8, 128, 64, 1142),
         ("plummer_mixture", 40000, 12, 256, 128, 1142)]


@pytest.mark.parametrize("m2l", [fmmgpu.FMM_M2L_FP32, fmmgpu.FMM_M2L_TC])
@pytest.mark.parametrize("gen,n,p,T,A,dm", CASES)
def test_adaptive_matches_oracle(oracle, m2l, gen, n, p, T, A, dm):
    pos, m = workloads.WORKLOADS[gen](n, seed=12)
    with fmmgpu.Context(dim=3, p=p, leaf_cap=T, G=1.0, direct_max=dm, m2l_mode=m2l, adaptive_leaf=A) as c:
        a, ph = c.evaluate(pos, m, want_pot=True)
        st = c.stats()
    assert st["depth"] >= 3  # the adaptive path runs on trees of depth >= 3
    g, po = oracle.fmm_adaptive(pos, m, p, T, aleaf=A, want_pot=True, direct_max=dm, w_direct_max=W_ALL_DIRECT)
    _check(a, ph, g, po)


def test_adaptive_writes_every_output_and_root_leaf(oracle):
    """Outputs pre-filled with NaN are all finite after the pass; with A >= n
    the root is the only adaptive leaf and the pass is the direct sum."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n = 12000
    pos, m = workloads.plummer_mixture(n, seed=13)
    d_pos, d_m = torch.from_numpy(pos).to(dev), torch.from_numpy(m).to(dev)
    direct, dpot = oracle.direct(pos, m, want_pot=True)
    for A, T in ((16, 16), (64, 32), (n, 16)):
        d_acc = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
        d_pot = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
        with fmmgpu.Context(dim=3, p=10, leaf_cap=T, G=1.0, direct_max=512, m2l_mode=fmmgpu.FMM_M2L_TC,
                            adaptive_leaf=A) as c:
            c.evaluate_device(n, d_pos.data_ptr(), d_m.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr())
            c.synchronize()
            assert c.stats()["depth"] >= 3
        a, ph = d_acc.cpu().numpy(), d_pot.cpu().numpy()
        assert np.isfinite(a).all() and np.isfinite(ph).all(), A
        if A >= n:
            assert rel_l2(a, direct) < 2e-5
            assert rel_l2(ph, dpot) < 2e-5
        else:
            assert rel_l2(a, direct) < 1e-4  # p = 10 truncation


def test_adaptive_converges_to_direct(oracle):
    """With adaptive targets the error against the FP64 direct sum falls with
    p as the uniform FMM's does (within 1.5x of the oracle's own truncation
    error plus 1e-6)."""
    pos, m = workloads.plummer_mixture(30000, seed=14)
    direct = oracle.direct(pos, m)
    for p in (6, 10, 12):
        with fmmgpu.Context(dim=3, p=p, leaf_cap=32, G=1.0, direct_max=512, m2l_mode=fmmgpu.FMM_M2L_TC,
                            adaptive_leaf=32) as c:
            a = c.evaluate(pos, m)
        g = oracle.fmm_adaptive(pos, m, p, 32, aleaf=32, direct_max=512, w_direct_max=W_ALL_DIRECT)
        assert rel_l2(a, direct) <= 1.5 * rel_l2(g, direct) + 1e-6, p
