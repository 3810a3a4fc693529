"""The float64 numpy oracle of the learned smoother: analytic gradients
against central finite differences (no GPU)."""
import numpy as np

import oracle.cnn_oracle as CO


def test_oracle_gradients_finite_differences():
    rng = np.random.default_rng(0)
    w = CO.init_weights(C=4, seed=1)
    x = rng.standard_normal((2, 5, 6))
    t = rng.standard_normal((2, 5, 6))
    _, g = CO.loss_and_grads(w, x, t)
    for li in range(6):
        for _ in range(3):
            idx = tuple(int(rng.integers(0, s)) for s in w[li].shape)
            e = 1e-6
            wp = [a.copy() for a in w]
            wp[li][idx] += e
            wm = [a.copy() for a in w]
            wm[li][idx] -= e
            fd = (CO.loss_and_grads(wp, x, t)[0] - CO.loss_and_grads(wm, x, t)[0]) / (2 * e)
            assert abs(fd - g[li][idx]) <= 1e-6 * max(1.0, abs(fd)), (li, idx)


def test_conv_adjoint():
    """<conv(x, w), g> = <x, conv_grad_input(g, w)>."""
    rng = np.random.default_rng(2)
    x = rng.standard_normal((2, 7, 5, 3))
    w = rng.standard_normal((4, 3, 3, 3))
    g = rng.standard_normal((2, 7, 5, 4))
    lhs = np.sum(CO.conv(x, w) * g)
    rhs = np.sum(x * CO.conv_grad_input(g, w))
    assert abs(lhs - rhs) <= 1e-10 * abs(lhs)


def test_bf16_rounding_and_emulated_network():
    """bf16() rounds like torch's FP32 -> BF16 conversion (nearest, ties to
    even), and the network with BF16 storage roundings stays within BF16
    accuracy of the exact one (forward and gradients)."""
    import torch
    rng = np.random.default_rng(0)
    a = rng.standard_normal(50000) * np.exp(rng.standard_normal(50000) * 4)
    t = torch.from_numpy(a.astype(np.float32)).to(torch.bfloat16).to(torch.float32).numpy().astype(np.float64)
    assert np.array_equal(CO.bf16(a), t)
    w = CO.init_weights(8, seed=1)
    x = rng.standard_normal((2, 9, 11))
    tt = rng.standard_normal((2, 9, 11))
    y, _ = CO.forward(w, x)
    yb, _ = CO.forward_bf16(w, x)
    assert np.linalg.norm(yb - y) / np.linalg.norm(y) < 3e-2
    L, g = CO.loss_and_grads(w, x, tt)
    Lb, gb = CO.loss_and_grads_bf16(w, x, tt)
    assert abs(Lb - L) / L < 3e-2
    for a_, b_ in zip(g, gb):
        assert np.linalg.norm(a_ - b_) / np.linalg.norm(a_) < 6e-2
