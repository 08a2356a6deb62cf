"""Warm-start network: tensor-core forward and backward passes against the
FP64 numpy restatement (oracle/cnn_oracle.py) with BF16 operand rounding.

Tolerances: the restatement rounds to BF16 at the same points, so what is left
is FP32 accumulation against FP64 and the BF16 roundings that this flips (an
activation one BF16 step apart): outputs within 5e-3 relative L2, every
layer's weight and bias gradients within 5e-3, the loss within 1e-3 (measured on
B200: outputs 5.9e-4, gradients at most 2.5e-3, loss 4.4e-6).
"""
import numpy as np
import pytest

import cnn_oracle as O

DIMS = (21, 14, 9)  # ni, nj, nk


def _case(seed):
    rng = np.random.default_rng(seed)
    ni, nj, nk = DIMS
    n = ni * nj * nk
    feat = rng.normal(size=(n, O.NFEAT)).astype(np.float32)
    target = (0.3 * feat[:, :2] + 0.1 * rng.normal(size=(n, 2))).astype(np.float32)
    return feat, target


def test_oracle_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -3.14159], dtype=np.float32)
    r = O.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1.0 + 2 ** -6 and abs(r[3] + 3.140625) < 1e-12


def test_oracle_gradient_matches_finite_differences():
    """The restatement's backward pass is the derivative of its forward pass
    (checked without BF16 rounding, by central differences)."""
    rng = np.random.default_rng(3)
    dims = (7, 6, 5)
    n = int(np.prod(dims))
    feat = rng.normal(size=(n, O.NFEAT))
    target = rng.normal(size=(n, 2))
    params = rng.normal(size=O.param_count()) * 0.1
    saved = O.bf16
    O.bf16 = lambda a: np.asarray(a, dtype=np.float64)
    try:
        y, acts = O.forward(params, feat, dims)
        loss, g = O.backward(params, acts, y, target, dims)
        def loss_at(p):
            yp, ap = O.forward(p, feat, dims)
            return O.backward(p, ap, yp, target, dims)[0]

        for q in rng.choice(O.param_count(), size=12, replace=False):
            e = 1e-5
            p1, p2 = params.copy(), params.copy()
            p1[q] += e
            p2[q] -= e
            fd = (loss_at(p1) - loss_at(p2)) / (2 * e)
            assert abs(fd - g[q]) <= 1e-5 * max(1.0, abs(fd)), (q, fd, g[q])
    finally:
        O.bf16 = saved


@pytest.mark.gpu
def test_forward_and_gradients_match_oracle():
    import torch
    import amcfd
    feat, target = _case(1)
    net = amcfd.Net(seed=7)
    params = net.params().astype(np.float64)
    ft = torch.from_numpy(feat).cuda()
    tt = torch.from_numpy(target).cuda()
    y = torch.zeros((feat.shape[0], 2), dtype=torch.float32, device="cuda")
    net.forward(ft.data_ptr(), DIMS, y.data_ptr())
    loss = net.backward(tt.data_ptr())
    g = net.grads().astype(np.float64)
    yo, acts = O.forward(params, feat.astype(np.float64), DIMS)
    lo, go = O.backward(params, acts, yo, target.astype(np.float64), DIMS)
    yg = y.cpu().numpy().astype(np.float64)
    ey = np.linalg.norm(yg - yo) / np.linalg.norm(yo)
    eg = [[float(np.linalg.norm(g[sl] - go[sl]) / max(np.linalg.norm(go[sl]), 1e-300)) for sl in ls]
          for ls in O.layer_slices()]
    print(f"outputs {ey:.2e}, loss {abs(loss - lo) / abs(lo):.2e}, "
          "gradients (W, b) per layer " + " ".join(f"({a:.2e}, {b:.2e})" for a, b in eg))
    assert ey <= 5e-3, ey
    assert abs(loss - lo) <= 1e-3 * abs(lo), (loss, lo)
    for l, (a, b) in enumerate(eg):
        assert a <= 5e-3 and b <= 5e-3, (l, a, b)
    net.close()


@pytest.mark.gpu
def test_training_reduces_loss():
    import torch
    import amcfd
    feat, target = _case(2)
    net = amcfd.Net(seed=11)
    ft = torch.from_numpy(feat).cuda()
    tt = torch.from_numpy(target).cuda()
    losses = []
    for _ in range(60):
        net.forward(ft.data_ptr(), DIMS)
        losses.append(net.backward(tt.data_ptr()))
        net.adam(3e-3)
    assert losses[-1] < 0.5 * losses[0], (losses[0], losses[-1])
    net.close()
