"""fmm_direct_noalloc: the FP64 direct sum for callers that cannot allocate
device memory when they need forces (a code whose own pool owns the GPU's
memory, or one that must not block on cudaMalloc).  It takes the caller's
device buffers, needs no context, and keeps its partial sums in the
library's fixed scratch array.  Checked through the C ABI against the
existing entry point fmm_direct on two calls in a row, with the 1e-12
relative tolerance the other direct-sum tests use.

This file is collected last on purpose: a failure here leaves every other
test already run."""
import numpy as np
import pytest
from conftest import rel_l2

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu


def _ptr(t):
    return t.data_ptr()


def test_direct_noalloc_matches_direct():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n = 30000
    pos, m = workloads.plummer(n, seed=21)
    targets = np.sort(np.random.default_rng(3).choice(n, 5000, replace=False)).astype(np.int64)
    with fmmgpu.Context(dim=3, G=1.0) as c:
        ref_all, ref_pot = c.direct(pos, m, want_pot=True)
        ref_sub = c.direct(pos, m, targets=targets)

    d_pos = torch.from_numpy(pos).to(dev)
    d_mass = torch.from_numpy(m).to(dev)
    d_tg = torch.from_numpy(targets).to(dev)
    d_acc = torch.full((n, 3), float("nan"), dtype=torch.float64, device=dev)
    d_pot = torch.full((n,), float("nan"), dtype=torch.float64, device=dev)
    d_acc2 = torch.full((len(targets), 3), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)

    # call 1: every particle is a target
    fmmgpu.direct_noalloc(3, n, _ptr(d_pos), _ptr(d_mass), _ptr(d_acc), _ptr(d_pot), stream=stream.cuda_stream)
    stream.synchronize()
    assert rel_l2(d_acc.cpu().numpy(), ref_all) < 1e-12
    assert rel_l2(d_pot.cpu().numpy(), ref_pot) < 1e-12

    # call 2, right after: a subset of targets, while the scratch still holds
    # call 1's partial sums; no device memory may be taken
    free_before = torch.cuda.mem_get_info(dev)[0]
    fmmgpu.direct_noalloc(3, n, _ptr(d_pos), _ptr(d_mass), _ptr(d_acc2), None, ntargets=len(targets),
                          targets_ptr=_ptr(d_tg), stream=stream.cuda_stream)
    stream.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free_before
    assert rel_l2(d_acc2.cpu().numpy(), ref_sub) < 1e-12


def test_direct_noalloc_rejects_oversize():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    d = torch.zeros(16, dtype=torch.float64, device=dev)
    with pytest.raises(fmmgpu.FmmError) as e:
        fmmgpu.direct_noalloc(3, 4, _ptr(d), _ptr(d), _ptr(d), None, ntargets=fmmgpu.FMM_NOALLOC_MAX_TARGETS + 1,
                              targets_ptr=_ptr(d))
    assert e.value.code == fmmgpu.FMM_ERR_TOO_LARGE


def test_direct_noalloc_full_scratch_and_two_d():
    """A call with the largest target count the scratch holds (one source
    chunk per target) and a 2D call with NaiveUpdate's softening, each
    against fmm_direct."""
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    nmax = fmmgpu.FMM_NOALLOC_MAX_TARGETS
    n = 20000
    pos, m = workloads.plummer(n, seed=22)
    targets = np.random.default_rng(4).integers(0, n, nmax).astype(np.int64)  # repeats allowed
    pos2 = np.random.default_rng(5).random((n, 2))
    m2 = np.full(n, 1.0 / n)
    with fmmgpu.Context(dim=3, G=1.0) as c:
        ref_full = c.direct(pos, m, targets=targets)
    with fmmgpu.Context(dim=2, G=1.0) as c:
        ref_2d = c.direct(pos2, m2, soft_mode=fmmgpu.FMM_SOFT_NAIVE_REF)
    d_pos, d_mass = torch.from_numpy(pos).to(dev), torch.from_numpy(m).to(dev)
    d_tg = torch.from_numpy(targets).to(dev)
    d_acc = torch.full((nmax, 3), float("nan"), dtype=torch.float64, device=dev)
    d_pos2, d_m2 = torch.from_numpy(pos2).to(dev), torch.from_numpy(m2).to(dev)
    d_acc2 = torch.full((n, 2), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream(dev)
    torch.cuda.synchronize(dev)
    fmmgpu.direct_noalloc(3, n, _ptr(d_pos), _ptr(d_mass), _ptr(d_acc), None, ntargets=nmax, targets_ptr=_ptr(d_tg),
                          stream=stream.cuda_stream)
    stream.synchronize()
    assert rel_l2(d_acc.cpu().numpy(), ref_full) < 1e-12
    fmmgpu.direct_noalloc(2, n, _ptr(d_pos2), _ptr(d_m2), _ptr(d_acc2), None, soft_mode=fmmgpu.FMM_SOFT_NAIVE_REF,
                          stream=stream.cuda_stream)
    stream.synchronize()
    assert rel_l2(d_acc2.cpu().numpy(), ref_2d) < 1e-12
