"""The learned smoother network (no counterpart in the reference).

A 6-layer 3x3 convolutional residual network on the node grid (32 channels,
no biases, ReLU), run and trained on the GPU by libjfem_gpu.so's own BF16
tensor-core kernels with FP32 accumulation and FP32 Adam master weights.
Weights are packed layer by layer in (Cout, Cin, 3, 3) order:
conv1 (32,1), conv2..conv5 (32,32), conv6 (1,32); 37,440 parameters.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import _native as N

CHANNELS = 32
SHAPES = [(32, 1, 3, 3), (32, 32, 3, 3), (32, 32, 3, 3), (32, 32, 3, 3), (32, 32, 3, 3), (1, 32, 3, 3)]


def num_params() -> int:
    c = C.c_int()
    N.load().jfg_cnn_num_params(C.byref(c))
    return c.value


def he_init(seed: int = 0, gain_last: float = 0.1) -> np.ndarray:
    """He-normal weights (numpy Philox stream); the last layer is scaled by gain_last."""
    rng = np.random.Generator(np.random.Philox(seed))
    parts = []
    for i, s in enumerate(SHAPES):
        w = rng.standard_normal(s) * np.sqrt(2.0 / (s[1] * 9))
        if i == len(SHAPES) - 1:
            w *= gain_last
        parts.append(w.reshape(-1))
    return np.concatenate(parts).astype(np.float32)


def unpack(flat) -> list:
    out, o = [], 0
    for s in SHAPES:
        n = int(np.prod(s))
        out.append(np.asarray(flat[o:o + n], dtype=np.float64).reshape(s))
        o += n
    return out


class LearnedSmoother:
    def __init__(self, ctx: N.Context, weights=None, seed: int = 0):
        self.ctx = ctx
        h = C.c_void_p()
        ctx.check(N.load().jfg_cnn_create(ctx.handle, C.byref(h)))
        self._h = h
        self.set_weights(he_init(seed) if weights is None else weights)

    @property
    def handle(self):
        return self._h

    def set_weights(self, w):
        w = np.ascontiguousarray(w, dtype=np.float32)
        if w.size != num_params():
            raise ValueError("wrong number of weights")
        self.ctx.check(N.load().jfg_cnn_set_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_float))))

    def get_weights(self) -> np.ndarray:
        w = np.empty(num_params(), dtype=np.float32)
        self.ctx.check(N.load().jfg_cnn_get_weights(self._h, w.ctypes.data_as(C.POINTER(C.c_float))))
        return w

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x: (B, H, W) float32 CUDA tensor -> (B, H, W)."""
        x = x.contiguous()
        B, H, W = x.shape
        y = torch.empty_like(x)
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_cnn_forward_dev(self._h, B, H, W, C.c_void_p(x.data_ptr()),
                                                    C.c_void_p(y.data_ptr())))
        return y

    def loss_and_grad(self, x: torch.Tensor, t: torch.Tensor):
        """Mean squared error and its gradient (numpy float32) w.r.t. the weights."""
        x, t = x.contiguous(), t.contiguous()
        B, H, W = x.shape
        loss = C.c_double()
        g = np.empty(num_params(), dtype=np.float32)
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_cnn_loss_grad_dev(self._h, B, H, W, C.c_void_p(x.data_ptr()),
                                                      C.c_void_p(t.data_ptr()), C.byref(loss),
                                                      g.ctypes.data_as(C.POINTER(C.c_float))))
        return loss.value, g

    def train_step(self, x: torch.Tensor, t: torch.Tensor, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8) -> float:
        x, t = x.contiguous(), t.contiguous()
        B, H, W = x.shape
        loss = C.c_double()
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_cnn_loss_grad_dev(self._h, B, H, W, C.c_void_p(x.data_ptr()),
                                                      C.c_void_p(t.data_ptr()), C.byref(loss), None))
        self.ctx.check(N.load().jfg_cnn_adam_step(self._h, lr, beta1, beta2, eps))
        return loss.value

    def time_forward(self, B, H, W, iters=20):
        tot, mid = C.c_double(), C.c_double()
        self.ctx.check(N.load().jfg_cnn_time_forward(self._h, B, H, W, iters, C.byref(tot), C.byref(mid)))
        return tot.value, mid.value

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_cnn_free(self._h)
        except Exception:
            pass


class MGCNNPreconditioner:
    """The nonlinear preconditioner "FP32 V-cycle of `mg`, then the learned
    smoother" for FGMRES (libjfem_gpu.so's jfg_mgcnn):

        z = V(v);  r' = v - A z;  q = D^-1 r';  s = rms(q);  z += out_scale * s * net(q / s)

    on the H x W node grid (``dof_of_pixel[i]`` is the unknown at row-major
    pixel i), with the correction zeroed on the Dirichlet nodes ``boundary``.
    ``use_net=False`` keeps only the V-cycle (the same preconditioner without
    the network, for comparisons)."""

    def __init__(self, mg, net: LearnedSmoother, A, H: int, W: int, dof_of_pixel, boundary, out_scale: float = 1.0,
                 use_net: bool = True):
        from .linalg import _as_device
        self.mg, self.net = mg, net
        self.A = _as_device(A)
        self.ctx = self.A.ctx
        self.n = self.A.rows
        dof = np.ascontiguousarray(dof_of_pixel, dtype=np.int32)
        bd = np.ascontiguousarray(boundary, dtype=np.int32)
        h = C.c_void_p()
        self.ctx.check(N.load().jfg_mgcnn_create(
            self.ctx.handle, mg.handle, net.handle, self.A.handle, H, W, dof.ctypes.data_as(C.POINTER(C.c_int)),
            bd.ctypes.data_as(C.POINTER(C.c_int)), int(bd.size), float(out_scale), 1 if use_net else 0,
            C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    def set(self, out_scale: float, use_net: bool = True):
        self.ctx.check(N.load().jfg_mgcnn_set(self._h, float(out_scale), 1 if use_net else 0))

    def apply_dev(self, v: torch.Tensor) -> torch.Tensor:
        """z = M(v) for an FP64 CUDA vector."""
        v = v.contiguous()
        z = torch.empty_like(v)
        torch.cuda.synchronize()
        self.ctx.check(N.load().jfg_mgcnn_apply_dev(self._h, C.c_void_p(v.data_ptr()), C.c_void_p(z.data_ptr())))
        return z

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                N.load().jfg_mgcnn_free(self._h)
        except Exception:
            pass


def pixel_map(space):
    """(H, W, dof_of_pixel) of a Q_p space's node grid: pixel (gx, gy) at
    row-major index gx * W + gy holds unknown node_of_grid[gx * W + gy]."""
    return space.nx, space.ny, np.ascontiguousarray(space.node_of_grid, dtype=np.int32)


def main(argv=None):
    """python -m jfem_b200.cnn B H W [iters]: times the forward pass on random
    input (CUDA events inside the library) and prints ms and TFLOP/s."""
    import json
    import sys
    a = [int(v) for v in (argv if argv is not None else sys.argv[1:])]
    B, H, W = a[:3]
    iters = a[3] if len(a) > 3 else 20
    net = LearnedSmoother(N.default_context(), weights=he_init(0))
    tot, mid = net.time_forward(B, H, W, iters)
    flops = 2.0 * sum(int(np.prod(s)) for s in SHAPES) * B * H * W
    mid_flops = 2.0 * 9 * 32 * 32 * B * H * W
    print(json.dumps({"pixels": B * H * W, "forward_ms": tot, "forward_tflops": flops / (tot * 1e-3) / 1e12,
                      "mid_layer_ms": mid, "mid_layer_tflops": mid_flops / (mid * 1e-3) / 1e12}))


if __name__ == "__main__":
    main()
