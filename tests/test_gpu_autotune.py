"""The autotuner (fmm_autotune): it times every candidate direct-pair
threshold (and, when asked, leaf capacity) on the caller's system, keeps the
fastest in the context, and the tuned context still evaluates within the
accuracy of the untuned one (the threshold only moves pairs between M2L and
the exact direct sum)."""
import numpy as np
import pytest
from conftest import rel_l2

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu


def test_autotune_picks_the_fastest_candidate_and_keeps_accuracy():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    n = 1 << 17
    pos, m = workloads.plummer(n, seed=41)
    idx = np.sort(np.random.default_rng(2).choice(n, 2048, replace=False)).astype(np.int64)
    with fmmgpu.Context(dim=3, G=1.0) as c:
        ref = c.direct(pos, m, targets=idx)
    d_pos, d_m = torch.from_numpy(pos).to(dev), torch.from_numpy(m).to(dev)
    torch.cuda.synchronize()
    with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0, m2l_mode=fmmgpu.FMM_M2L_TC) as c:
        a0 = c.evaluate(pos, m)
        cands, best = c.autotune(n, d_pos.data_ptr(), d_m.data_ptr())
        assert len(cands) == 5 and all(x["ms"] > 0 for x in cands)
        assert best["ms"] == min(x["ms"] for x in cands)
        assert len({x["direct_max"] for x in cands}) == 5
        a1 = c.evaluate(pos, m)
        assert c.stats()["direct_max"] == best["direct_max"]
    assert rel_l2(a1[idx], ref) < 1.5 * rel_l2(a0[idx], ref) + 1e-7


def test_autotune_with_leaf_capacities():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    n = 1 << 16
    pos, m = workloads.uniform_cube(n, seed=42)
    d_pos, d_m = torch.from_numpy(pos).to(dev), torch.from_numpy(m).to(dev)
    torch.cuda.synchronize()
    with fmmgpu.Context(dim=3, p=6, leaf_cap=64, G=1.0, m2l_mode=fmmgpu.FMM_M2L_TC) as c:
        cands, best = c.autotune(n, d_pos.data_ptr(), d_m.data_ptr(), tune_leaf=True)
        # coordinate search: four capacities at one threshold, then three
        # more thresholds at the best capacity
        assert len(cands) == 7 and [x["leaf_cap"] for x in cands[:4]] == [32, 64, 128, 256]
        assert len({x["direct_max"] for x in cands[:4]}) == 1
        assert {x["leaf_cap"] for x in cands[4:]} == {cands[int(np.argmin([x["ms"] for x in cands[:4]]))]["leaf_cap"]}
        assert best["ms"] == min(x["ms"] for x in cands)
        a = c.evaluate(pos, m)
        assert np.all(np.isfinite(a))


def test_autotune_adaptive_and_kernel_shapes():
    """With FMM_TUNE_ADAPTIVE and FMM_TUNE_KERNELS the tuner also tries the
    adaptive-target thresholds (0 = uniform targets among them), then the
    colleague-sum chunk and the tensor-core M2L work-item length; the kept
    setting evaluates within the accuracy of the untuned one, and each
    kernel shape alone gives the same forces to FP32 rounding."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    n = 1 << 17
    pos, m = workloads.plummer_mixture(n, seed=43)
    idx = np.sort(np.random.default_rng(3).choice(n, 2048, replace=False)).astype(np.int64)
    with fmmgpu.Context(dim=3, G=1.0) as c:
        ref = c.direct(pos, m, targets=idx)
    d_pos, d_m = torch.from_numpy(pos).to(dev), torch.from_numpy(m).to(dev)
    torch.cuda.synchronize()
    with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0, m2l_mode=fmmgpu.FMM_M2L_TC, adaptive_leaf=32) as c:
        a0 = c.evaluate(pos, m)
        cands, best = c.autotune(n, d_pos.data_ptr(), d_m.data_ptr(), tune_adaptive=True, tune_kernels=True)
        assert {0, 16, 64} <= {x["adaptive_leaf"] for x in cands}
        # five thresholds, three more adaptive thresholds, then the best
        # threshold of those times 1/sqrt(2) and sqrt(2)
        b8 = cands[int(np.argmin([x["ms"] for x in cands[:8]]))]
        assert [x["direct_max"] for x in cands[8:10]] == [
            max(8, int(b8["direct_max"] * f)) for f in (0.70710678118654752, 1.41421356237309505)]
        assert all(x["adaptive_leaf"] == b8["adaptive_leaf"] for x in cands[8:10])
        assert {128, 512} <= {x["p2p_chunk"] for x in cands} or best["adaptive_leaf"] == 0
        assert {24, 189} <= {x["m2l_run"] for x in cands}
        assert best["ms"] == min(x["ms"] for x in cands)
        a1 = c.evaluate(pos, m)
    assert rel_l2(a1[idx], ref) < 1.5 * rel_l2(a0[idx], ref) + 1e-7
    outs = []
    for pc, mr in ((0, 0), (64, 8), (1024, 189)):
        with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0, m2l_mode=fmmgpu.FMM_M2L_TC, adaptive_leaf=32,
                            p2p_chunk=pc, m2l_run=mr) as c:
            outs.append(c.evaluate(pos, m))
    for o in outs[1:]:
        assert rel_l2(o, outs[0]) < 1e-6


def test_kernel_shape_settings_are_checked():
    for bad in (dict(p2p_chunk=16), dict(p2p_chunk=100), dict(p2p_chunk=8192), dict(m2l_run=4), dict(m2l_run=200)):
        with pytest.raises(fmmgpu.FmmError) as e:
            fmmgpu.Context(dim=3, **bad)
        assert e.value.code == fmmgpu.FMM_ERR_INVALID_ARGUMENT
