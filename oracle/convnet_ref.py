"""CPU oracle of the learned force-correction network -- TEST INFRASTRUCTURE.

torch-CPU restatement of the three-layer 3x3x3 periodic conv net that
csrc/convnet.cu runs on the GPU (no reference counterpart: the learned
correction is new).  Parameters are the library's flat float32 vector:
per layer W[tap][ci][cout] (27 x 16 x 16, tap = 9 (dx+1) + 3 (dy+1) + (dz+1))
then 16 biases.  The GPU stores inputs, weights and hidden activations in
bfloat16 and accumulates in float32; the oracle rounds at the same points
and computes in float64.
"""
import numpy as np
import torch
import torch.nn.functional as F

C = 16
WSZ = 27 * C * C
LAYER = WSZ + C
NPARAMS = 3 * LAYER


def bf16(x):
    """Round to bfloat16 (nearest even) and back, as the device does."""
    t = torch.as_tensor(x)
    return t.to(torch.bfloat16).to(t.dtype if t.dtype != torch.bfloat16 else torch.float32)


class _RoundBF16(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x):
        return x.to(torch.bfloat16).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        return g


def layer_weights(params, l, dtype=torch.float64, rounding=True):
    p = torch.as_tensor(np.asarray(params, dtype=np.float32 if rounding else np.float64))
    w = p[l * LAYER: l * LAYER + WSZ].reshape(3, 3, 3, C, C)      # [dx][dy][dz][ci][co]
    b = p[l * LAYER + WSZ: (l + 1) * LAYER]
    w = w.to(torch.bfloat16).to(dtype) if rounding else w.to(dtype)   # bf16 weights
    # torch conv3d weight [co][ci][kx][ky][kz] (cross-correlation, offset k-1)
    return w.permute(4, 3, 0, 1, 2).contiguous(), b.to(dtype)


def forward(in2, params, dtype=torch.float64, requires_grad=False, rounding=True):
    """in2: (N,N,N,2) features -> (N,N,N,3) network output.  rounding=False
    skips every bf16 rounding (exact float64 network, for derivative checks)."""
    rnd = _RoundBF16.apply if rounding else (lambda t: t)
    x = torch.as_tensor(np.asarray(in2, dtype=np.float32)).to(dtype)
    x = rnd(x)
    N = x.shape[0]
    h = torch.zeros((1, C, N, N, N), dtype=dtype)
    h[0, :2] = x.permute(3, 0, 1, 2)
    ws = []
    for l in range(3):
        w, b = layer_weights(params, l, dtype, rounding)
        if requires_grad:
            w.requires_grad_(True)
            b.requires_grad_(True)
        ws.append((w, b))
        hp = F.pad(h, (1, 1, 1, 1, 1, 1), mode="circular")
        h = F.conv3d(hp, w, b)
        if l < 2:
            h = F.leaky_relu(h, 0.1)
            h = rnd(h)
    out = h[0, :3].permute(1, 2, 3, 0)
    return out, ws


def grads(in2, params, grad3, rounding=True):
    """Flat parameter gradient of sum(grad3 * out); bf16 roundings are
    passed straight through in the backward pass, as on the device."""
    out, ws = forward(in2, params, torch.float64, requires_grad=True, rounding=rounding)
    g = torch.as_tensor(np.asarray(grad3, dtype=np.float64))
    (out * g).sum().backward()
    flat = np.zeros(NPARAMS)
    for l, (w, b) in enumerate(ws):
        gw = w.grad.permute(2, 3, 4, 1, 0).reshape(-1).numpy()     # back to [t][ci][co]
        flat[l * LAYER: l * LAYER + WSZ] = gw
        flat[l * LAYER + WSZ: (l + 1) * LAYER] = b.grad.numpy()
    return flat
