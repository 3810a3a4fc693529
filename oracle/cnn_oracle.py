"""float64 numpy restatement of the learned smoother network (test infrastructure).

The network has no counterpart in the reference; this module is the CPU
oracle its GPU forward and backward kernels are checked against.  Layout:
images (B, H, W) for the scalar input/output, (B, H, W, C) activations,
weights W[l] of shape (Cout, Cin, 3, 3), zero padding, no biases:

    h1 = relu(conv1(x))            1 -> C
    a2 = relu(conv2(h1))           C -> C
    h3 = relu(h1 + conv3(a2))      C -> C   (residual block)
    a4 = relu(conv4(h3))           C -> C
    h5 = relu(h3 + conv5(a4))      C -> C   (residual block)
    y  = conv6(h5)                 C -> 1

Loss: L = mean over pixels of (y - t)^2.
"""
import numpy as np

SHAPES = lambda C: [(C, 1, 3, 3), (C, C, 3, 3), (C, C, 3, 3), (C, C, 3, 3), (C, C, 3, 3), (1, C, 3, 3)]


def conv(x, w):
    """x: (B, H, W, Cin); w: (Cout, Cin, 3, 3) -> (B, H, W, Cout); 3x3, zero pad."""
    B, H, Wd, Ci = x.shape
    xp = np.zeros((B, H + 2, Wd + 2, Ci))
    xp[:, 1:-1, 1:-1, :] = x
    out = np.zeros((B, H, Wd, w.shape[0]))
    for dy in range(3):
        for dx in range(3):
            out += xp[:, dy:dy + H, dx:dx + Wd, :] @ w[:, :, dy, dx].T
    return out


def conv_grad_input(g, w):
    """d(conv(x, w))/dx applied to g: (B, H, W, Cout) -> (B, H, W, Cin)."""
    B, H, Wd, Co = g.shape
    gp = np.zeros((B, H + 2, Wd + 2, Co))
    gp[:, 1:-1, 1:-1, :] = g
    out = np.zeros((B, H, Wd, w.shape[1]))
    for dy in range(3):
        for dx in range(3):
            # out[p] += sum_co w[co, ci, dy, dx] g[p - (dy-1, dx-1)]
            out += gp[:, 2 - dy:2 - dy + H, 2 - dx:2 - dx + Wd, :] @ w[:, :, dy, dx]
    return out


def conv_grad_weight(g, x):
    """dL/dw for out = conv(x, w) with upstream g: (Cout, Cin, 3, 3)."""
    B, H, Wd, Ci = x.shape
    xp = np.zeros((B, H + 2, Wd + 2, Ci))
    xp[:, 1:-1, 1:-1, :] = x
    Co = g.shape[-1]
    dw = np.zeros((Co, Ci, 3, 3))
    g2 = g.reshape(-1, Co)
    for dy in range(3):
        for dx in range(3):
            dw[:, :, dy, dx] = g2.T @ xp[:, dy:dy + H, dx:dx + Wd, :].reshape(-1, Ci)
    return dw


def relu(v):
    return np.maximum(v, 0.0)


def forward(weights, x):
    """x: (B, H, W) -> y (B, H, W) and the cache of activations."""
    w1, w2, w3, w4, w5, w6 = weights
    h1 = relu(conv(x[..., None], w1))
    a2 = relu(conv(h1, w2))
    h3 = relu(h1 + conv(a2, w3))
    a4 = relu(conv(h3, w4))
    h5 = relu(h3 + conv(a4, w5))
    y = conv(h5, w6)[..., 0]
    return y, (x, h1, a2, h3, a4, h5)


def loss_and_grads(weights, x, t):
    w1, w2, w3, w4, w5, w6 = weights
    y, (x, h1, a2, h3, a4, h5) = forward(weights, x)
    npx = y.size
    L = float(np.mean((y - t) ** 2))
    dy = (2.0 / npx) * (y - t)
    g6 = dy[..., None]
    dw6 = conv_grad_weight(g6, h5)
    dh5 = conv_grad_input(g6, w6)
    g5 = dh5 * (h5 > 0)
    dw5 = conv_grad_weight(g5, a4)
    g4 = conv_grad_input(g5, w5) * (a4 > 0)
    dw4 = conv_grad_weight(g4, h3)
    dh3 = g5 + conv_grad_input(g4, w4)
    g3 = dh3 * (h3 > 0)
    dw3 = conv_grad_weight(g3, a2)
    g2 = conv_grad_input(g3, w3) * (a2 > 0)
    dw2 = conv_grad_weight(g2, h1)
    dh1 = g3 + conv_grad_input(g2, w2)
    g1 = dh1 * (h1 > 0)
    dw1 = conv_grad_weight(g1, x[..., None])
    return L, [dw1, dw2, dw3, dw4, dw5, dw6]


def bf16(a):
    """Round to the nearest BF16 value, ties to even (via FP32), as the GPU's
    __float2bfloat16_rn does; returned as float64."""
    f = np.ascontiguousarray(np.asarray(a, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def forward_bf16(weights, x):
    """The forward with the GPU's storage roundings (float64 arithmetic
    otherwise): the 32 -> 32 layers read BF16 weights and BF16 input and skip
    activations, every stored activation (h1, a2, h3, a4, h5) is BF16, the
    1 -> 32 and 32 -> 1 layers use the FP32 master weights on the FP32 input
    image and the BF16 h5."""
    w1, w2, w3, w4, w5, w6 = weights
    m2, m3, m4, m5 = (bf16(w) for w in (w2, w3, w4, w5))
    h1 = bf16(relu(conv(x[..., None], w1)))
    a2 = bf16(relu(conv(h1, m2)))
    h3 = bf16(relu(h1 + conv(a2, m3)))
    a4 = bf16(relu(conv(h3, m4)))
    h5 = bf16(relu(h3 + conv(a4, m5)))
    y = conv(h5, w6)[..., 0]
    return y, (x, h1, a2, h3, a4, h5)


def loss_and_grads_bf16(weights, x, t):
    """loss_and_grads with the GPU backward's roundings: the gradient images
    that enter a 32 -> 32 product (input gradient or weight gradient) are
    rounded to BF16 (g5, g4, g3, g2), the products read the BF16 weights
    (flipped for the input gradients) and the BF16 activations; the skip
    gradients, the ReLU masks and the edge layers stay FP32."""
    w1, w2, w3, w4, w5, w6 = weights
    m2, m3, m4, m5 = (bf16(w) for w in (w2, w3, w4, w5))
    y, (x, h1, a2, h3, a4, h5) = forward_bf16(weights, x)
    npx = y.size
    L = float(np.mean((y - t) ** 2))
    dy = (2.0 / npx) * (y - t)
    g6 = dy[..., None]
    dw6 = conv_grad_weight(g6, h5)
    g5 = conv_grad_input(g6, w6) * (h5 > 0)
    b5 = bf16(g5)
    dw5 = conv_grad_weight(b5, a4)
    b4 = bf16(conv_grad_input(b5, m5) * (a4 > 0))
    dw4 = conv_grad_weight(b4, h3)
    g3 = (g5 + conv_grad_input(b4, m4)) * (h3 > 0)
    b3 = bf16(g3)
    dw3 = conv_grad_weight(b3, a2)
    b2 = bf16(conv_grad_input(b3, m3) * (a2 > 0))
    dw2 = conv_grad_weight(b2, h1)
    g1 = (g3 + conv_grad_input(b2, m2)) * (h1 > 0)
    dw1 = conv_grad_weight(g1, x[..., None])
    return L, [dw1, dw2, dw3, dw4, dw5, dw6]


def init_weights(C=32, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for s in SHAPES(C):
        fan_in = s[1] * 9
        out.append(rng.standard_normal(s) * np.sqrt(2.0 / fan_in))
    return out
