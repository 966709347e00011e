"""Learned pair orders: the MLP's CPU oracle against finite differences (CPU),
the GPU forward/backward kernels against the oracle (GPU), and the
configuration checks of FMM_ORDER_LEARNED (CPU, no device calls)."""
import numpy as np
import pytest

import fmmgpu
import order_mlp as om


def _data(n, seed):
    rng = np.random.default_rng(seed)
    feat = rng.normal(0.0, 0.7, (n, om.NF)).astype(np.float32)
    feat[:, 22:] = 0.0
    labels = rng.uniform(-12.0, -2.0, (n, om.NQ)).astype(np.float32)
    labels[::7, 3] = -30.0  # below the clamp
    return feat, labels


def test_oracle_layout_matches_library():
    assert om.NPARAM == fmmgpu.FMM_ORDER_NPARAM
    assert om.NF == fmmgpu.FMM_ORDER_NFEAT and om.NQ == fmmgpu.FMM_ORDER_NOUT
    p = fmmgpu.order_init_params(1)
    assert p.shape == (om.NPARAM,) and np.all(p[om.W3 + om.NQ * om.NH:om.B3] == 0.0)


def test_bf16_rounding_is_nearest_even():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.0e-5, 65504.0], np.float32)
    r = om.bf16(x)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # halfway between 1 and 1 + 2^-7: ties to even
    assert r[2] == np.float32(1.0078125)    # above halfway: up
    assert r[3] == np.float32(1.0078125)
    assert abs(r[4] - x[4]) <= abs(x[4]) * 2.0 ** -8
    assert abs(r[5] - x[5]) <= abs(x[5]) * 2.0 ** -8


def test_oracle_gradient_matches_finite_differences():
    feat, labels = _data(40, 3)
    p = fmmgpu.order_init_params(5).astype(np.float64)
    loss, g, _ = om.loss_grad(p, feat, labels, bf16_round=False)
    rng = np.random.default_rng(0)
    live = np.r_[np.arange(om.W1, om.B3 - 16 * om.NH + om.NQ * om.NH), np.arange(om.B3, om.B3 + om.NQ)]
    for i in rng.choice(live, 60, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fd = (om.loss_grad(pp, feat, labels, False)[0] - om.loss_grad(pm, feat, labels, False)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * (abs(g[i]) + 1e-3), (i, fd, g[i])


@pytest.mark.gpu
def test_gpu_forward_and_gradient_match_oracle():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    n = 300  # not a multiple of the 128-row blocks
    feat, labels = _data(n, 11)
    p = fmmgpu.order_init_params(7)
    d_feat = torch.from_numpy(feat).to(dev)
    d_lab = torch.from_numpy(labels).to(dev)
    d_par = torch.from_numpy(p).to(dev)
    d_pred = torch.zeros((n, om.NQ), dtype=torch.float32, device=dev)
    d_grad = torch.zeros(om.NPARAM, dtype=torch.float32, device=dev)
    d_loss = torch.zeros(1, dtype=torch.float32, device=dev)
    torch.cuda.synchronize()
    fmmgpu.order_forward_grad(d_feat.data_ptr(), d_lab.data_ptr(), n, d_par.data_ptr(), d_pred.data_ptr(),
                              d_grad.data_ptr(), d_loss.data_ptr())
    loss, g, y = om.loss_grad(p, feat, labels, bf16_round=True)
    pred = d_pred.cpu().numpy()
    # FP32 accumulation on the GPU against FP64 in the oracle, same BF16
    # operands: an activation whose accumulated value lies within the
    # accumulation error of a BF16 rounding boundary may round the other way
    # (one BF16 ulp, 2^-8 relative), so the bound is on almost all outputs
    scale = np.abs(y).max() + 1.0
    d = np.abs(pred - y)
    assert np.mean(d <= 1e-4 * scale) >= 0.99 and d.max() <= 1e-2 * scale
    assert abs(float(d_loss.item()) - loss) <= 1e-3 * loss
    gg = d_grad.cpu().numpy()
    assert np.linalg.norm(gg - g) <= 1e-3 * np.linalg.norm(g)
    assert np.all(gg[om.W3 + om.NQ * om.NH:om.B3] == 0.0)


@pytest.mark.gpu
def test_gpu_training_reduces_the_loss():
    torch = pytest.importorskip("torch")
    dev = torch.device("cuda", 0)
    rng = np.random.default_rng(2)
    n = 8192
    feat = rng.normal(0.0, 0.5, (n, om.NF)).astype(np.float32)
    feat[:, 22:] = 0.0
    # a smooth target the network can learn: decreasing in the order index
    base = -2.0 - 3.0 * np.tanh(feat[:, :4].sum(1))
    labels = (base[:, None] - 0.8 * np.arange(om.NQ)[None, :]).astype(np.float32)
    with fmmgpu.Context(dim=3, p=12, m2l_mode=fmmgpu.FMM_M2L_TC) as c:
        c.set_order_model(fmmgpu.order_init_params(3))
        d_feat = torch.from_numpy(feat).to(dev)
        d_lab = torch.from_numpy(labels).to(dev)
        torch.cuda.synchronize()
        loss = c.order_train(d_feat.data_ptr(), d_lab.data_ptr(), n, epochs=40, batch=1024, lr=3e-3)
    assert loss[-1] < 0.05 * loss[0], loss


def test_learned_mode_configuration_checks():
    with pytest.raises(fmmgpu.FmmError) as e:
        fmmgpu.Context(dim=3, p=12, m2l_mode=fmmgpu.FMM_M2L_FP32, order_mode=fmmgpu.FMM_ORDER_LEARNED)
    assert e.value.code == fmmgpu.FMM_ERR_UNSUPPORTED
    with pytest.raises(fmmgpu.FmmError) as e:
        fmmgpu.Context(dim=2, p=12, m2l_mode=fmmgpu.FMM_M2L_TC, order_mode=fmmgpu.FMM_ORDER_LEARNED)
    assert e.value.code == fmmgpu.FMM_ERR_UNSUPPORTED
