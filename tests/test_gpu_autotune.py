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
