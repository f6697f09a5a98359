"""Inverse rendering driver: recover scene parameters (shader colours,
specular weights, fBm amplitude and base colour, light powers) from target
images with Adam, through yr_backward_batch (all scenes' forward + adjoint
as one CUDA graph per step) or through yr_render + yr_backward per scene.

The optimiser state is a few floats per scene and lives on the host; each
step uploads the parameters (yr_params_set), runs the device step, and
reads the gradients back."""
from __future__ import annotations

import time
from typing import List, Optional

import numpy as np

from . import api


class Adam:
    """Adam (Kingma & Ba, 2015) with bias correction, in float64."""

    def __init__(self, x0: np.ndarray, lr: float = 1e-2, b1: float = 0.9, b2: float = 0.999, eps: float = 1e-8):
        self.x = np.asarray(x0, np.float64).copy()
        self.m = np.zeros_like(self.x)
        self.v = np.zeros_like(self.x)
        self.t = 0
        self.lr, self.b1, self.b2, self.eps = lr, b1, b2, eps

    def step(self, g: np.ndarray) -> np.ndarray:
        self.t += 1
        g = np.asarray(g, np.float64)
        self.m = self.b1 * self.m + (1 - self.b1) * g
        self.v = self.b2 * self.v + (1 - self.b2) * g * g
        mh = self.m / (1 - self.b1 ** self.t)
        vh = self.v / (1 - self.b2 ** self.t)
        self.x -= self.lr * mh / (np.sqrt(vh) + self.eps)
        return self.x


def fit(dss: List[api.DeviceScene], targets, steps: int = 200, lr: float = 1e-2, batched: bool = True,
        streams: int = 0, lower: float = 0.0, loss_scale: Optional[List[float]] = None, masks=None):
    """Run `steps` Adam steps on every scene (each its own problem).
    targets: device RGBA float tensors (torch), one per scene.  masks: per
    scene a boolean array over the parameter vector, True = optimised (None:
    all).  Parameters are kept >= `lower` (colours and powers are
    non-negative).  Gradients are scaled per scene by 1 / (initial loss) so
    that one learning rate suits problems of any image size.  Returns
    (params per scene, loss history [steps, scenes], seconds of the device
    loop)."""
    import torch
    n = len(dss)
    imgs = [torch.empty_like(t) for t in targets]
    grads = [torch.zeros(max(1, d.param_count()), dtype=torch.float32, device="cuda") for d in dss]
    opts = [Adam(d.params_get(), lr) for d in dss]
    hist = np.zeros((steps, n))
    scale = np.ones(n) if loss_scale is None else np.asarray(loss_scale, np.float64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for it in range(steps):
        if batched:
            losses = api.backward_batch(dss, [t.data_ptr() for t in imgs], [t.data_ptr() for t in targets],
                                        [g.data_ptr() for g in grads], 1.0, streams)
        else:
            losses = np.zeros(n, np.float32)
            for i, d in enumerate(dss):
                d.render_into(imgs[i].data_ptr())
                losses[i] = d.backward(imgs[i].data_ptr(), targets[i].data_ptr(), grads[i].data_ptr(), 1.0)
        g_host = torch.cat(grads).cpu().numpy()
        hist[it] = losses
        if it == 0 and loss_scale is None:
            scale = 1.0 / np.maximum(losses.astype(np.float64), 1e-30)
        off = 0
        for i, d in enumerate(dss):
            k = d.param_count()
            g = g_host[off:off + k] * scale[i]
            if masks is not None:
                g = np.where(masks[i], g, 0.0)
            x = opts[i].step(g)
            np.maximum(x, lower, out=x)
            d.params_set(x.astype(np.float32))
            off += max(1, k)
    torch.cuda.synchronize()
    return [o.x.copy() for o in opts], hist, time.perf_counter() - t0
