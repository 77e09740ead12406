"""The torch-CPU oracle of the conv net: its autograd gradient of the exact
(unrounded, float64) network agrees with central finite differences on a
tiny mesh; with bf16 rounding on, the gradient is the straight-through
gradient the device computes and stays close to the exact one."""
import numpy as np
import torch

from oracle import convnet_ref as CR


def test_oracle_gradient_finite_differences():
    n = 6
    rng = np.random.default_rng(0)
    x = rng.normal(0, 1, (n, n, n, 2)).astype(np.float32)
    p = rng.normal(0, 0.2, CR.NPARAMS)
    g3 = rng.normal(0, 1, (n, n, n, 3))
    exact = CR.grads(x, p, g3, rounding=False)

    def f(pp):
        out, _ = CR.forward(x, pp, torch.float64, rounding=False)
        return float((out.detach().numpy() * g3).sum())
    for idx in (5, 300, CR.LAYER + 17, 2 * CR.LAYER + CR.WSZ + 1):
        h = 1e-5
        up, dn = p.copy(), p.copy()
        up[idx] += h
        dn[idx] -= h
        fd = (f(up) - f(dn)) / (2 * h)
        assert abs(fd - exact[idx]) <= 1e-5 * max(1.0, abs(exact[idx])), (idx, fd, exact[idx])
    rounded = CR.grads(x, p.astype(np.float32), g3)
    live = exact != 0
    cos = np.dot(rounded[live], exact[live]) / np.linalg.norm(rounded[live]) / np.linalg.norm(exact[live])
    assert cos > 0.999
