"""CPU oracle for the learned Poisson start's network (test infrastructure only).

The network has no counterpart in the reference, so this oracle is a plain PyTorch (CPU,
FP32) statement of the same architecture and parameter layout, with autograd for the
gradients.  It rounds weights and stored activations to BF16 where the device kernels do,
so the device forward pass and gradients can be compared with it at BF16 tolerance.

Layout shared with the device code (dft_b200/csrc/neural.cu):
* activations NDHWC, point index (z*ny + y)*nx + x, channels innermost;
* weights [tap][cin][cout] followed by bias[cout], each layer's block padded to 8 floats;
  3x3x3 taps t = (dz*3 + dy)*3 + dx (offsets -1..1), 2x2x2 taps t = tx | ty<<1 | tz<<2.
Only tests/ use this module.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.nn.functional as F

# (type, cin, cout): conv3 / down / up / head, in network order
LAYERS = [("conv3", 2, 16), ("conv3", 16, 16), ("down", 16, 32), ("conv3", 32, 32), ("down", 32, 32),
          ("conv3", 32, 32), ("conv3", 32, 32), ("up", 32, 32), ("conv3", 32, 32), ("up", 32, 16),
          ("conv3", 16, 16), ("head", 16, 1)]
TAPS = {"conv3": 27, "down": 8, "up": 8, "head": 1}


def offsets():
    """(w offset, b offset) per layer and the total parameter count."""
    off, out = 0, []
    for typ, cin, cout in LAYERS:
        w = off
        off += TAPS[typ] * cin * cout
        b = off
        off += cout
        off = (off + 7) // 8 * 8
        out.append((w, b))
    return out, off


def _bf16(t: torch.Tensor) -> torch.Tensor:
    """Round to BF16 in the forward pass, identity in the backward pass."""
    return t + (t.to(torch.bfloat16).to(torch.float32) - t).detach()


def _torch_weight(typ, w_flat, cin, cout):
    """Our [tap][ci][co] block as the weight tensor torch's op expects."""
    if typ == "conv3":
        w = w_flat.reshape(3, 3, 3, cin, cout)           # [dz][dy][dx][ci][co]
        return w.permute(4, 3, 0, 1, 2)                  # (co, ci, dz, dy, dx)
    if typ in ("down", "up"):
        w = w_flat.reshape(2, 2, 2, cin, cout)           # [tz][ty][tx][ci][co]
        w = w.permute(3, 4, 0, 1, 2) if typ == "up" else w.permute(4, 3, 0, 1, 2)
        return w                                         # up: (ci, co, ...); down: (co, ci, ...)
    return w_flat.reshape(cin, cout).t().reshape(cout, cin, 1, 1, 1)


def forward(params: torch.Tensor, x: torch.Tensor, shape):
    """params: flat FP32 tensor (requires_grad allowed); x: (N, 2) input; shape (nx, ny, nz).
    Returns y (N,) in FP32."""
    nx, ny, nz = shape
    offs, _ = offsets()
    a = _bf16(x.reshape(nz, ny, nx, -1).permute(3, 0, 1, 2).unsqueeze(0))
    acts = []
    for i, ((typ, cin, cout), (wo, bo)) in enumerate(zip(LAYERS, offs)):
        wf = _bf16(params[wo:wo + TAPS[typ] * cin * cout])
        b = params[bo:bo + cout]
        w = _torch_weight(typ, wf, cin, cout)
        if typ == "conv3":
            z = F.conv3d(a, w, b, padding=1)
        elif typ == "down":
            d, h, wd = a.shape[2:]
            z = F.conv3d(F.pad(a, (0, wd % 2, 0, h % 2, 0, d % 2)), w, b, stride=2)
        elif typ == "up":
            skip = acts[3] if cout == 32 else acts[1]
            z = F.conv_transpose3d(a, w, b, stride=2)[:, :, :skip.shape[2], :skip.shape[3], :skip.shape[4]] + skip
        else:
            y = F.conv3d(a, w, b)
            return y[0, 0].reshape(-1)
        a = _bf16(F.silu(z))
        acts.append(a)
    raise AssertionError("unreachable")


def loss_grad(params: np.ndarray, x: np.ndarray, t: np.ndarray, shape):
    """Loss = mean over interior points of (y - t)^2, its gradient (flat, our layout) and y."""
    nx, ny, nz = shape
    p = torch.tensor(params, dtype=torch.float32, requires_grad=True)
    y = forward(p, torch.tensor(x, dtype=torch.float32), shape)
    tt = torch.tensor(t, dtype=torch.float32)
    mask = torch.zeros(nz, ny, nx, dtype=torch.bool)
    mask[1:-1, 1:-1, 1:-1] = True
    mask = mask.reshape(-1)
    d = (y - tt)[mask]
    loss = (d * d).mean()
    loss.backward()
    return float(loss), p.grad.numpy().copy(), y.detach().numpy()


def direct_conv3(x: np.ndarray, w: np.ndarray, b: np.ndarray, shape) -> np.ndarray:
    """Plain loop 3x3x3 convolution in our layout (pins the layout convention of forward())."""
    nx, ny, nz = shape
    cin, cout = x.shape[1], b.size
    xv = x.reshape(nz, ny, nx, cin)
    wv = w.reshape(27, cin, cout)
    out = np.tile(b, (nz, ny, nx, 1)).astype(np.float64)
    for dz in range(3):
        for dy in range(3):
            for dx in range(3):
                tap = (dz * 3 + dy) * 3 + dx
                src = np.zeros_like(xv)
                zs, ys, xs = slice(max(0, dz - 1), nz + min(0, dz - 1)), slice(max(0, dy - 1), ny + min(0, dy - 1)), \
                    slice(max(0, dx - 1), nx + min(0, dx - 1))
                zd, yd, xd = slice(max(0, 1 - dz), nz - max(0, dz - 1)), slice(max(0, 1 - dy), ny - max(0, dy - 1)), \
                    slice(max(0, 1 - dx), nx - max(0, dx - 1))
                src[zd, yd, xd] = xv[zs, ys, xs]
                out += src @ wv[tap]
    return out.reshape(-1, cout)
