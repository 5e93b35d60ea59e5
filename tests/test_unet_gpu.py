"""The warm-start U-Net on the GPU (tcgen05 BF16 convolutions) against the NumPy FP64 oracle, and the warm start
it gives the corrector solve."""
import numpy as np
import pytest

from oracle import density_ref as OD
from oracle import unet_ref as U

pytestmark = pytest.mark.gpu

W = (16, 32, 32)


@pytest.fixture(scope="module")
def learned():
    import torch  # noqa: F401
    from nlfiber_b200 import learned
    return learned


def rel_l2(a, b):
    return float(np.linalg.norm(np.ravel(a) - np.ravel(b)) / np.linalg.norm(np.ravel(b)))


def _case(n=8, nb=2, seed=0):
    rng = np.random.default_rng(seed)
    rho = rng.random((nb, n, n, n))
    t = rng.standard_normal((nb, n, n, n, 18)) * 0.05
    w = rng.random((nb, n, n, n))
    return rho, t, w / w.sum()


def _cuda(a):
    import torch
    return torch.tensor(np.asarray(a), dtype=torch.float32, device="cuda")


@pytest.mark.parametrize("n", [8, 16])
def test_forward_and_gradients_match_oracle(learned, n):
    """BF16 operands with FP32 accumulation against FP64: 3% on the output, the loss and every layer's gradient."""
    net = learned.UNet(W, seed=3)
    p = U.init_params(W, seed=5)
    p[-U.OUT - W[0] * U.OUT:-U.OUT] *= 100.0  # an output layer of the size of the hidden ones
    net.set_params(p)
    rho, t, w = _case(n)
    y = net.forward(_cuda(rho)).cpu().numpy()
    yr, _ = U.forward(p, rho[..., None], W)
    assert rel_l2(y, yr) < 3e-2, rel_l2(y, yr)
    loss, g = net.loss_grad(_cuda(rho), _cuda(t), _cuda(w), want_grad=True)
    lr_, gr = U.backward(p, rho[..., None], t, w, W)
    assert abs(loss - lr_) < 3e-2 * lr_, (loss, lr_)
    o = 0
    for k, (ci, co, nt, _) in enumerate(U.layers(*W)):
        for size in (nt * co * ci, co):
            err = rel_l2(g[o:o + size], gr[o:o + size])
            assert err < 6e-2, (k, size, err)
            o += size


def test_adam_step_matches_oracle_and_training_fits(learned):
    net = learned.UNet(W, seed=4)
    p = U.init_params(W, seed=6)
    net.set_params(p)
    rho, t, w = _case(8, nb=2, seed=1)
    _, g = net.loss_grad(_cuda(rho), _cuda(t), _cuda(w), want_grad=True)
    net.adam_step(1e-3)
    p1 = net.get_params()
    pr, _, _ = U.adam(p.astype(np.float64), g.astype(np.float64), 0.0, 0.0, 1, 1e-3)
    assert np.allclose(p1, pr, rtol=1e-5, atol=1e-7)
    # a learnable target: the network fits a smooth function of the density
    rng = np.random.default_rng(2)
    rho = rng.random((4, 8, 8, 8))
    t = np.repeat((rho - 0.5)[..., None], 18, axis=-1) * np.linspace(-0.2, 0.2, 18)
    w = np.ones((4, 8, 8, 8))
    net.set_params(U.init_params(W, seed=7))
    losses = learned.train(net, _cuda(rho), _cuda(t), _cuda(w), steps=80, batch=2, lr=3e-3)
    assert np.mean(losses[-5:]) < 0.2 * np.mean(losses[:5]), (losses[:5], losses[-5:])
