"""The learned smoother network: GPU forward and backward kernels against the
float64 numpy oracle (oracle/cnn_oracle.py), and GPU training."""
import numpy as np
import pytest
import torch

import oracle.cnn_oracle as CO
from jfem_b200.cnn import LearnedSmoother, he_init, num_params, unpack

pytestmark = pytest.mark.gpu


def bf16_round(a):
    t = torch.from_numpy(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).to(torch.float32)
    return t.numpy().astype(np.float64)


@pytest.mark.parametrize("shape", [(1, 16, 16), (2, 19, 37), (3, 33, 8)])
def test_forward_matches_oracle(ctx, shape):
    rng = np.random.default_rng(1)
    w = he_init(seed=2, gain_last=1.0)
    x = rng.standard_normal(shape).astype(np.float32)
    net = LearnedSmoother(ctx, w)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    # the GPU rounds weights and activations to BF16: compare with the oracle on
    # BF16-rounded weights, tolerance of a few BF16 ulps accumulated over 6 layers
    yr, _ = CO.forward([bf16_round(a) for a in unpack(w)], x.astype(np.float64))
    err = np.linalg.norm(y - yr) / np.linalg.norm(yr)
    assert err < 3e-2, err


@pytest.mark.parametrize("shape", [(2, 16, 16), (1, 21, 18)])
def test_gradient_matches_oracle(ctx, shape):
    rng = np.random.default_rng(3)
    w = he_init(seed=4, gain_last=1.0)
    x = rng.standard_normal(shape).astype(np.float32)
    t = rng.standard_normal(shape).astype(np.float32)
    net = LearnedSmoother(ctx, w)
    loss, g = net.loss_and_grad(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    L, gr = CO.loss_and_grads([bf16_round(a) for a in unpack(w)], x.astype(np.float64), t.astype(np.float64))
    assert abs(loss - L) / L < 2e-2
    for l, (gg, rr) in enumerate(zip(unpack(g), gr)):
        err = np.linalg.norm(gg - rr) / np.linalg.norm(rr)
        assert err < 6e-2, (l, err)


@pytest.mark.parametrize("shape", [(1, 16, 16), (2, 19, 37), (3, 33, 8), (1, 130, 257)])
def test_forward_matches_bf16_oracle(ctx, shape):
    """The forward against the oracle that rounds where the GPU stores BF16
    (weights of the 32 -> 32 layers, every stored activation): what is left
    is FP32 summation order and the BF16 rounding flips it causes (measured
    up to 5e-4 on these shapes, against 3e-2 for the unrounded oracle)."""
    rng = np.random.default_rng(1)
    w = he_init(seed=2, gain_last=1.0)
    x = rng.standard_normal(shape).astype(np.float32)
    net = LearnedSmoother(ctx, w)
    y = net.forward(torch.from_numpy(x).cuda()).cpu().numpy()
    yr, _ = CO.forward_bf16(unpack(w), x.astype(np.float64))
    err = np.linalg.norm(y - yr) / np.linalg.norm(yr)
    print(f"forward {shape}: rel err {err:.3e}")
    assert err < 2e-3, err


@pytest.mark.parametrize("shape", [(2, 16, 16), (1, 21, 18), (1, 67, 45)])
def test_gradient_matches_bf16_oracle(ctx, shape):
    """Loss and all six weight gradients against the oracle with the
    backward's BF16 roundings (gradient images entering the 32 -> 32
    products, BF16 weights and activations)."""
    rng = np.random.default_rng(3)
    w = he_init(seed=4, gain_last=1.0)
    x = rng.standard_normal(shape).astype(np.float32)
    t = rng.standard_normal(shape).astype(np.float32)
    net = LearnedSmoother(ctx, w)
    loss, g = net.loss_and_grad(torch.from_numpy(x).cuda(), torch.from_numpy(t).cuda())
    L, gr = CO.loss_and_grads_bf16(unpack(w), x.astype(np.float64), t.astype(np.float64))
    errs = [np.linalg.norm(gg - rr) / np.linalg.norm(rr) for gg, rr in zip(unpack(g), gr)]
    print(f"gradients {shape}: loss rel err {abs(loss - L) / L:.3e}, " + " ".join(f"{e:.3e}" for e in errs))
    assert abs(loss - L) / L < 1e-3
    for l, err in enumerate(errs):
        assert err < 3e-3, (l, err)


def test_training_reduces_loss(ctx):
    """A few hundred Adam steps fit a fixed linear target operator (a 3x3
    smoothing stencil) on random inputs."""
    rng = np.random.default_rng(5)
    net = LearnedSmoother(ctx, he_init(seed=6))
    k = np.array([[1, 2, 1], [2, 4, 2], [1, 2, 1]], dtype=np.float64) / 16.0

    def target(x):
        xp = np.pad(x, ((0, 0), (1, 1), (1, 1)))
        out = np.zeros_like(x)
        for dy in range(3):
            for dx in range(3):
                out += k[dy, dx] * xp[:, dy:dy + x.shape[1], dx:dx + x.shape[2]]
        return out

    losses = []
    for it in range(300):
        x = rng.standard_normal((8, 32, 32))
        t = target(x)
        losses.append(net.train_step(torch.from_numpy(x.astype(np.float32)).cuda(),
                                     torch.from_numpy(t.astype(np.float32)).cuda(), lr=2e-3))
    assert np.mean(losses[-20:]) < 0.2 * np.mean(losses[:5])
    w = net.get_weights()
    assert w.size == num_params() == 37440 and np.all(np.isfinite(w))


@pytest.mark.parametrize("shape", [(2, 45, 27), (1, 257, 131)])
def test_tcgen05_forward_matches_mma_sync(ctx, shape, monkeypatch):
    """The tcgen05 forward (TMEM accumulators) and the mma.sync forward agree
    to BF16 rounding of the activations (partial tiles and a batch included)."""
    rng = np.random.default_rng(11)
    w = he_init(seed=5, gain_last=1.0)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    net = LearnedSmoother(ctx, w)
    monkeypatch.setenv("JFEM_CNN_TC", "1")
    y_tc = net.forward(x).cpu().numpy()
    monkeypatch.setenv("JFEM_CNN_TC", "0")
    y_ms = net.forward(x).cpu().numpy()
    assert np.all(np.isfinite(y_tc))
    err = np.linalg.norm(y_tc - y_ms) / np.linalg.norm(y_ms)
    assert err < 1e-2, err


@pytest.mark.parametrize("shape", [(2, 45, 27), (1, 131, 66)])
def test_tcgen05_backward_matches_mma_sync(ctx, shape, monkeypatch):
    """The input gradients of the backward pass on tcgen05 (flipped,
    channel-transposed weights, FP32 epilogues with the ReLU masks and the
    skip path) and on mma.sync read the same BF16-rounded gradient images:
    the weight gradients agree to FP32 accumulation-order rounding."""
    rng = np.random.default_rng(12)
    w = he_init(seed=7, gain_last=1.0)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    net = LearnedSmoother(ctx, w)
    monkeypatch.setenv("JFEM_CNN_TC", "1")
    l_tc, g_tc = net.loss_and_grad(x, t)
    monkeypatch.setenv("JFEM_CNN_TC", "0")
    l_ms, g_ms = net.loss_and_grad(x, t)
    assert np.all(np.isfinite(g_tc))
    for l, (a, b) in enumerate(zip(unpack(g_tc), unpack(g_ms))):
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < 1e-2, (l, err)


@pytest.mark.parametrize("shape", [(2, 45, 27), (1, 1025, 1025)])
def test_warp_specialised_conv_equals_single_role(ctx, shape, monkeypatch):
    """The warp-specialised tcgen05 pipeline (TMA, MMA and epilogue warps,
    four halo stages, two TMEM accumulators) issues the same MMAs per tile as
    the single-role kernel: forward outputs and gradients are bit-identical."""
    rng = np.random.default_rng(13)
    w = he_init(seed=8, gain_last=1.0)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    net = LearnedSmoother(ctx, w)
    monkeypatch.setenv("JFEM_CNN_TC", "1")
    monkeypatch.setenv("JFEM_CNN_PROJ", "0")          # the separate output layer in both
    outs = []
    for ws in ("1", "0"):
        monkeypatch.setenv("JFEM_CNN_WS", ws)
        y = net.forward(x).cpu().numpy()
        _, g = net.loss_and_grad(x, t)
        outs.append((y, g))
    assert np.all(np.isfinite(outs[0][0]))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][1], outs[1][1])


@pytest.mark.parametrize("shape", [(2, 45, 27), (1, 1025, 1025)])
def test_fused_output_projection(ctx, shape, monkeypatch):
    """Inference forwards fuse the 32 -> 1 output layer into the last tcgen05
    layer's epilogue (nine per-pixel tap sums of the BF16 activations, then a
    nine-tap gather): the same activations, FP32 sums in another order, so the
    output equals the separate output layer's to FP32 rounding."""
    rng = np.random.default_rng(14)
    w = he_init(seed=9, gain_last=1.0)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    net = LearnedSmoother(ctx, w)
    monkeypatch.setenv("JFEM_CNN_TC", "1")
    y_f = net.forward(x).cpu().numpy()
    monkeypatch.setenv("JFEM_CNN_PROJ", "0")
    y_s = net.forward(x).cpu().numpy()
    assert np.all(np.isfinite(y_f))
    err = np.abs(y_f - y_s).max() / np.abs(y_s).max()
    assert err < 1e-5, err


@pytest.mark.parametrize("shape", [(2, 45, 27), (3, 130, 257), (1, 1025, 1025)])
def test_strip_conv_equals_tiled(ctx, shape, monkeypatch):
    """The strip convolution (activations copied into TMEM three times
    shifted, the MMA's A operand from TMEM, weights from shared memory) issues
    every output pixel's MMAs in the tiled kernels' order: forward outputs
    (with and without the fused output projection) and gradients equal the
    warp-specialised tiled kernel's bit for bit, strips of 128 pixels with
    ragged last strips and row segments included."""
    rng = np.random.default_rng(15)
    w = he_init(seed=10, gain_last=1.0)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    net = LearnedSmoother(ctx, w)
    monkeypatch.setenv("JFEM_CNN_TC", "1")
    outs = []
    for strip in ("1", "0"):
        monkeypatch.setenv("JFEM_CNN_STRIP", strip)
        monkeypatch.setenv("JFEM_CNN_PROJ", "1")
        y_p = net.forward(x).cpu().numpy()
        monkeypatch.setenv("JFEM_CNN_PROJ", "0")
        y_s = net.forward(x).cpu().numpy()
        _, g = net.loss_and_grad(x, t)
        outs.append((y_p, y_s, g))
    assert np.all(np.isfinite(outs[0][0]))
    for a, b in zip(outs[0], outs[1]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("shape", [(2, 45, 27), (1, 257, 131), (3, 64, 64)])
def test_tcgen05_weight_gradients_match_mma_sync(ctx, shape, monkeypatch):
    """Weight gradients of the 32 -> 32 layers on the tensor cores (k_wgrad_tc:
    G^T and the tap-shifted X as K-major channel-planar tiles, the pixels as
    the contraction, nine TMEM accumulators per CTA) against the mma.sync
    kernel on the same BF16 gradient images and activations: the same
    products summed in another order, so they agree to FP32 rounding of the
    sums."""
    rng = np.random.default_rng(16)
    w = he_init(seed=11, gain_last=1.0)
    x = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    t = torch.from_numpy(rng.standard_normal(shape).astype(np.float32)).cuda()
    net = LearnedSmoother(ctx, w)
    monkeypatch.setenv("JFEM_CNN_TC", "1")
    l_tc, g_tc = net.loss_and_grad(x, t)
    monkeypatch.setenv("JFEM_CNN_WGRAD_TC", "0")
    l_ms, g_ms = net.loss_and_grad(x, t)
    assert l_tc == l_ms
    parts_tc, parts_ms = unpack(g_tc), unpack(g_ms)
    for l in (1, 2, 3, 4):                       # the 32 -> 32 layers
        a, b = parts_tc[l], parts_ms[l]
        assert np.all(np.isfinite(a))
        err = np.linalg.norm(a - b) / np.linalg.norm(b)
        assert err < 1e-4, (l, err)
    for l in (0, 5):                             # the edge layers are unchanged
        assert np.array_equal(parts_tc[l], parts_ms[l])
