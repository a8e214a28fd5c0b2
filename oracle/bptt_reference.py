"""FP64 dense PyTorch autograd reference of the recurrent LIF layer (the BPTT workload) -- test
infrastructure only: the tests compare the library's forward and adjoint kernels (naer2_b200/csrc/bptt.cu)
with it; nothing in the product imports it.

naer2 has no differentiable path, so there is no reference code to restate: this is the model as the layer
states it (include/naer2b.h), written with dense matrices and torch.autograd in float64:
  U = x @ w_in;   R[t] = sum_d s[t - d] @ W_d   (W_d[pre, post] = w of the links of delay d)
  Vpre = alpha V + U[t] + R[t];   s = spike(Vpre - theta);   V = Vpre - theta s
  O[t] = beta O[t-1] + s @ w_out;  m = O[t*] with t* the first argmax over t
spike(): Heaviside forward with the fast-sigmoid surrogate 1 / (1 + slope |x|)^2 as its derivative, or, with
smooth=True, the smooth f(x) = x / (1 + slope |x|) (whose true derivative is that surrogate), for finite
differences. `forced` replaces the Heaviside decisions by given spikes (the kernels' raster), so that a run
in float64 takes the same spike path as the float32 kernels; `forced_tstar` does the same for t*.
"""

from __future__ import annotations

import torch


class _Spike(torch.autograd.Function):
    @staticmethod
    def forward(ctx, x, slope, forced):
        ctx.save_for_backward(x)
        ctx.slope = slope
        return forced.to(x.dtype) if forced is not None else (x >= 0).to(x.dtype)

    @staticmethod
    def backward(ctx, g):
        (x,) = ctx.saved_tensors
        return g / (1.0 + ctx.slope * x.abs()) ** 2, None, None


def dense_delays(w_rec, pre, post, delay, hidden: int, max_delay: int = 5):
    """[W_1 .. W_max_delay], W_d [H, H] (pre, post): differentiable in w_rec."""
    out = []
    for d in range(1, max_delay + 1):
        mask = delay == d
        W = torch.zeros(hidden, hidden, dtype=w_rec.dtype, device=w_rec.device)
        out.append(W.index_put((pre[mask], post[mask]), w_rec[mask], accumulate=True))
    return out


def run(x, w_in, w_rec, w_out, pre, post, delay, alpha, beta, theta, slope, smooth=False, forced=None,
        forced_tstar=None):
    """m [B, R] (differentiable), t* [B, R], the decisions' margins (Vpre - theta) [T, B, H] (detached) and the
    spikes [T, B, H] (detached). x [T, B, C]; every tensor argument on one device, float64 for the weights."""
    T, B, C = x.shape
    H = w_in.shape[1]
    Ws = dense_delays(w_rec, pre, post, delay, H)
    U = torch.matmul(x.to(w_in.dtype), w_in)
    V = torch.zeros(B, H, dtype=w_in.dtype, device=w_in.device)
    O = torch.zeros(B, w_out.shape[1], dtype=w_in.dtype, device=w_in.device)
    hist, Os, margins = [], [], []
    for t in range(T):
        vp = alpha * V + U[t]
        for d in range(1, len(Ws) + 1):
            if t - d >= 0:
                vp = vp + hist[t - d] @ Ws[d - 1]
        xm = vp - theta
        if smooth:
            s = xm / (1.0 + slope * xm.abs())
        else:
            s = _Spike.apply(xm, slope, None if forced is None else forced[t])
        V = vp - theta * s
        O = beta * O + s @ w_out
        hist.append(s)
        Os.append(O)
        margins.append(xm.detach())
    Ost = torch.stack(Os)
    ts = Ost.detach().argmax(dim=0) if forced_tstar is None else forced_tstar.to(torch.int64)
    m = Ost.gather(0, ts.unsqueeze(0)).squeeze(0)
    return m, ts, torch.stack(margins), torch.stack([h.detach() for h in hist])


def loss(m, y):
    return torch.nn.functional.cross_entropy(m, y)
