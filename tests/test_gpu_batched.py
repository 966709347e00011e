"""Batched ensemble (fmm_evaluate_batched): independent systems stored one
after another, evaluated concurrently on worker streams, give every system
the forces a single evaluation of that system gives (to the FP32 round-off
of the pass), including empty and one-particle systems."""
import numpy as np
import pytest
from conftest import rel_l2

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu


def _ensemble(sizes, seed):
    pos, mass = [], []
    for k, n in enumerate(sizes):
        if n == 0:
            continue
        p, m = workloads.plummer(int(n), seed=seed + k)
        pos.append(p + 100.0 * k)  # far apart, so a mix-up would show
        mass.append(m)
    return np.concatenate(pos), np.concatenate(mass)


@pytest.mark.parametrize("workers", [0, 1, 3])
def test_batched_matches_single_evaluations(workers):
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    sizes = [1500, 0, 7000, 1, 2048, 20000, 333, 4096, 12000, 2]
    pos, mass = _ensemble(sizes, 50)
    off = np.r_[0, np.cumsum(sizes)].astype(np.int64)
    d_pos, d_m = torch.from_numpy(pos).to(dev), torch.from_numpy(mass).to(dev)
    d_acc = torch.full((len(pos), 3), float("nan"), dtype=torch.float64, device=dev)
    d_pot = torch.full((len(pos),), float("nan"), dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    with fmmgpu.Context(dim=3, p=8, leaf_cap=64, G=1.0, m2l_mode=fmmgpu.FMM_M2L_TC) as c:
        c.evaluate_batched(off, d_pos.data_ptr(), d_m.data_ptr(), d_acc.data_ptr(), d_pot.data_ptr(), workers)
        st = c.stats()
        acc, pot = d_acc.cpu().numpy(), d_pot.cpu().numpy()
        assert st["ms_total"] > 0
        for s in range(len(sizes)):
            a, b = off[s], off[s + 1]
            if b == a:
                continue
            if b - a == 1:
                assert np.all(acc[a] == 0.0)
                continue
            a1, p1 = c.evaluate(pos[a:b], mass[a:b], want_pot=True)
            assert rel_l2(acc[a:b], a1) < 1e-6
            assert rel_l2(pot[a:b], p1) < 1e-6
    assert np.all(np.isfinite(acc)) and np.all(np.isfinite(pot))


def test_batched_rejects_bad_offsets():
    with fmmgpu.Context(dim=3, p=4, G=1.0) as c:
        with pytest.raises(fmmgpu.FmmError) as e:
            c.evaluate_batched(np.array([0, 5, 3], np.int64), None, None, None)
        assert e.value.code == fmmgpu.FMM_ERR_INVALID_ARGUMENT
