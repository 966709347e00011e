"""Tensor-core translations (FMM_M2L_TC: M2L, M2M and L2L on tcgen05, BF16
three-way split operands, FP32 accumulation) against the SIMT FP32
contraction and the FP64 oracle.  Tolerance: relative L2 <= 1e-6, the same
bar as FP32 mode."""
import numpy as np
import pytest
from conftest import rel_l2

import fmmgpu
from fmmgpu import workloads

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gen,n,p,T,dm", [("plummer", 20000, 8, 64, 0), ("uniform3d", 12000, 4, 16, 0),
                                          ("plummer", 30000, 8, 64, 256), ("uniform3d", 8000, 10, 20, 0),
                                          ("uniform3d", 6000, 11, 32, 0), ("uniform3d", 6000, 12, 32, 0),
                                          ("plummer", 12000, 12, 32, 64)])
def test_tc_matches_fp32_and_oracle(oracle, gen, n, p, T, dm):
    pos, m = workloads.WORKLOADS[gen](n, seed=13)
    res = {}
    for mode in (fmmgpu.FMM_M2L_FP32, fmmgpu.FMM_M2L_TC):
        with fmmgpu.Context(dim=3, p=p, leaf_cap=T, G=1.0, direct_max=dm, m2l_mode=mode) as c:
            a, ph = c.evaluate(pos, m, want_pot=True)
            res[mode] = (a, ph, c.stats())
    a32, p32, s32 = res[fmmgpu.FMM_M2L_FP32]
    atc, ptc, stc = res[fmmgpu.FMM_M2L_TC]
    assert stc["m2l_pairs"] == s32["m2l_pairs"] > 0
    assert rel_l2(atc, a32) < 1e-6
    g, po = oracle.fmm(pos, m, p, T, want_pot=True, direct_max=dm)
    assert rel_l2(atc, g) < 1e-6
    assert rel_l2(ptc, po) < 1e-6


def test_tc_two_d(oracle):
    pos, m = workloads.disk_clumps_2d(30000, seed=14)
    with fmmgpu.Context(dim=2, p=16, leaf_cap=32, G=1.0, direct_max=0, m2l_mode=fmmgpu.FMM_M2L_TC) as c:
        a, ph = c.evaluate(pos, m, want_pot=True)
    g, po = oracle.fmm(pos, m, 16, 32, want_pot=True)
    assert rel_l2(a, g) < 1e-6
    assert rel_l2(ph, po) < 1e-6


def test_tc_counts_tiles():
    pos, m = workloads.uniform_cube(20000, seed=3)
    with fmmgpu.Context(dim=3, p=6, leaf_cap=16, G=1.0, direct_max=0, m2l_mode=fmmgpu.FMM_M2L_TC) as c:
        c.evaluate(pos, m)
        s = c.stats()
    # every tile holds at most 128 pairs, and a uniform cube fills them well
    assert s["m2l_pairs"] <= 128 * s["m2l_tiles"] < 4 * s["m2l_pairs"]


def test_tc_rejects_orders_beyond_tile():
    with pytest.raises(fmmgpu.FmmError) as e:
        fmmgpu.Context(dim=3, p=13, m2l_mode=fmmgpu.FMM_M2L_TC)
    assert e.value.code == fmmgpu.FMM_ERR_UNSUPPORTED
