"""PyTorch reference of the radiance-cache network (test infrastructure): the same
encoding, a float64 forward pass with BF16 rounding where the kernels round
(encoded input, weights, post-ReLU activations, backpropagated gradients), and the
relative-L2 loss gradient, so the fused tensor-core kernels can be compared with it."""
import math

import torch

LAYERS = ((96, 64), (64, 64), (64, 64), (64, 64), (64, 16))
LOSS_EPS = 0.01


def bf16(x: torch.Tensor) -> torch.Tensor:
    return x.to(torch.bfloat16).to(x.dtype)


def sh16(d: torch.Tensor) -> torch.Tensor:
    x, y, z = d[:, 0], d[:, 1], d[:, 2]
    xx, yy, zz = x * x, y * y, z * z
    return torch.stack([
        torch.full_like(x, 0.28209479177387814),
        0.4886025119029199 * y, 0.4886025119029199 * z, 0.4886025119029199 * x,
        1.0925484305920792 * x * y, 1.0925484305920792 * y * z, 0.31539156525252005 * (3 * zz - 1),
        1.0925484305920792 * x * z, 0.5462742152960396 * (xx - yy),
        0.5900435899266435 * y * (3 * xx - yy), 2.890611442640554 * x * y * z,
        0.4570457994644658 * y * (5 * zz - 1), 0.3731763325901154 * z * (5 * zz - 3),
        0.4570457994644658 * x * (5 * zz - 1), 1.445305721320277 * z * (xx - yy),
        0.5900435899266435 * x * (xx - 3 * yy)], 1)


def encode(samples: torch.Tensor, box) -> torch.Tensor:
    """(n, 16) float32 samples -> (n, 96) float64 encoding (before BF16 rounding)."""
    s = samples.to(torch.float32)
    bmin = torch.tensor(box[:3], dtype=torch.float32)
    ext = torch.tensor(box[3:], dtype=torch.float32) - bmin
    binv = torch.where(ext > 0, 1.0 / ext, torch.zeros_like(ext))
    p = ((s[:, 0:3] - bmin) * binv).to(torch.float64)                      # float32 ops, as the kernel
    freqs = torch.tensor([2.0 ** k for k in range(12)], dtype=torch.float64)
    arg = math.pi * p[:, :, None] * freqs                                  # exact p * 2^k, then pi
    pos = torch.stack([torch.sin(arg), torch.cos(arg)], -1).reshape(len(s), 72)
    d = s[:, 4:7].to(torch.float32)
    sh = sh16(d).to(torch.float64)
    n = s[:, 8:11].to(torch.float64)
    a = s[:, 12:15].to(torch.float64)
    one = torch.ones(len(s), 1, dtype=torch.float64)
    zero = torch.zeros(len(s), 1, dtype=torch.float64)
    return torch.cat([pos, sh, n, a, one, zero], 1)


def forward(weights, samples, box):
    """Returns (y (n, 16) float64, [x, a0, a1, a2, a3]) with BF16-rounded activations."""
    x = bf16(encode(samples, box))
    ws = [bf16(torch.as_tensor(w, dtype=torch.float64)) for w in weights]
    acts = [x]
    h = x
    for w in ws[:-1]:
        h = bf16(torch.relu(h @ w))
        acts.append(h)
    return h @ ws[-1], acts


def gradients(weights, samples, box):
    """Weight gradients of the mean relative-L2 loss, with the kernels' rounding:
    the output gradient and every backpropagated gradient are rounded to BF16."""
    y, acts = forward(weights, samples, box)
    ws = [bf16(torch.as_tensor(w, dtype=torch.float64)) for w in weights]
    t = samples[:, [3, 7, 11]].to(torch.float64)
    n = len(samples)
    yc = y[:, :3]
    den = yc * yc + LOSS_EPS
    dy = torch.zeros_like(y)
    dy[:, :3] = 2.0 * (yc - t) / den / n
    loss = ((yc - t) ** 2 / den).mean().item()
    dz = bf16(dy)
    grads = [None] * len(ws)
    for l in range(len(ws) - 1, -1, -1):
        grads[l] = acts[l].T @ dz
        if l > 0:
            dz = bf16((dz @ ws[l].T) * (acts[l] > 0))
    return grads, loss
