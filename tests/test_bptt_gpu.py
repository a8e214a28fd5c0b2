"""The BPTT kernels (n2b_bptt_forward / n2b_bptt_backward through the layer's autograd.Function) against the
FP64 dense autograd reference (oracle/bptt_reference.py) and finite differences.

Tolerances: gradients within 1e-4 relative (norm of the difference over the norm of the reference) of the
float64 reference; readout maxima within 1e-5 relative. In the spiking model the float64 run is
teacher-forced with the kernels' spikes and t* (a float32 and a float64 run take different spike paths
wherever a membrane lands within rounding of the threshold); the test checks that the reference's own
decisions agree with the forced ones except within 1e-4 of the threshold."""

import pytest
import torch

from naer2_b200.bptt import RecurrentLIF
from naer2_b200.networks import bptt_task
from oracle import bptt_reference as ref

pytestmark = pytest.mark.gpu


def make(cuda, B=8, T=60, C=32, H=64, R=5, K=9, smooth=False, seed=0, density=0.2, w_scale=(4.0, 0.5, 1.0)):
    layer = RecurrentLIF(n_in=C, hidden=H, readouts=R, density=density, checkpoint=K, seed=seed, device=cuda,
                         smooth=smooth, w_scale=w_scale)
    rates = bptt_task.templates(classes=R, channels=C, steps=T, seed=seed)
    x, y = bptt_task.sample(rates, B, seed=seed + 1, device=cuda)
    return layer, x, y


def kernel_grads(layer, x, y):
    layer.zero_grad(set_to_none=True)
    m = layer(x)
    loss = torch.nn.functional.cross_entropy(m, y)
    loss.backward()
    torch.cuda.synchronize()
    return m.detach(), loss.item(), [p.grad.detach().clone() for p in (layer.w_in, layer.w_rec, layer.w_out)]


def reference(layer, x, y, forced=None, forced_tstar=None):
    w = layer.wiring
    dev = x.device
    params = [p.detach().double().clone().requires_grad_() for p in (layer.w_in, layer.w_rec, layer.w_out)]
    pre, post, delay = (torch.from_numpy(a).to(dev) for a in (w.pre, w.post, w.delay))
    m, ts, margins, spikes = ref.run(x.double(), *params, pre, post, delay, layer.alpha, layer.beta, layer.theta,
                                     layer.slope, smooth=layer.smooth, forced=forced, forced_tstar=forced_tstar)
    loss = ref.loss(m, y)
    grads = torch.autograd.grad(loss, params)
    return m.detach(), ts, margins, spikes, loss.item(), grads, params


def rel(a, b):
    return ((a.double() - b.double()).norm() / b.double().norm()).item()


def test_smooth_kernels_match_fp64_autograd_and_finite_differences(cuda):
    layer, x, y = make(cuda, smooth=True, T=50, K=7)
    m, loss, grads = kernel_grads(layer, x, y)
    assert layer.status(8, 50) == [0, 0, 0, 0]
    m64, _, _, _, loss64, g64, params = reference(layer, x, y)
    assert rel(m, m64) < 1e-5
    for g, r in zip(grads, g64):
        assert r.abs().max() > 0 and rel(g, r) < 1e-4
    # central differences of the float64 smooth model, a few entries of every weight array
    w = layer.wiring
    pre, post, delay = (torch.from_numpy(a).to(cuda) for a in (w.pre, w.post, w.delay))

    def L(ps):
        mm, *_ = ref.run(x.double(), *ps, pre, post, delay, layer.alpha, layer.beta, layer.theta, layer.slope,
                         smooth=True)
        return ref.loss(mm, y).item()

    gen = torch.Generator().manual_seed(0)
    eps = 1e-6
    for i, g in enumerate(grads):
        scale = g.abs().max().item()
        for k in torch.randperm(g.numel(), generator=gen)[:6].tolist():
            hi = [p.detach().clone() for p in params]
            lo = [p.detach().clone() for p in params]
            hi[i].view(-1)[k] += eps
            lo[i].view(-1)[k] -= eps
            fd = (L(hi) - L(lo)) / (2 * eps)
            assert abs(fd - g.view(-1)[k].item()) <= 1e-4 * scale, (i, k, fd, g.view(-1)[k].item())


@pytest.mark.parametrize("K", [13, 80])
def test_spiking_kernels_match_the_teacher_forced_fp64_reference(cuda, K):
    B, T, H = 16, 80, 64
    layer, x, y = make(cuda, B=B, T=T, H=H, K=K, seed=2)
    m, loss, grads = kernel_grads(layer, x, y)
    assert layer.status(B, T) == [0, 0, 0, 0]
    spikes = layer.spikes(B, T)
    rate = spikes.float().mean().item()
    assert 0.005 < rate < 0.5, rate
    _, ts = layer.infer(x)
    m64, _, margins, _, _, g64, _ = reference(layer, x, y, forced=spikes, forced_tstar=ts)
    own = margins >= 0
    assert ((own != spikes) <= (margins.abs() < 1e-4)).all()
    assert rel(m, m64) < 1e-5
    for g, r in zip(grads, g64):
        assert rel(g, r) < 1e-4


def test_checkpoint_interval_changes_nothing(cuda):
    """The kernels' outputs (dU, dw_rec, dw_out) are bit-identical for any checkpoint interval: the recomputed
    segments reproduce the forward exactly. (w_in's gradient, x^T dU, does not depend on them: its kernels
    are tested on their own.)"""
    out = []
    for K in (1, 7, 60):
        layer, x, y = make(cuda, B=16, T=60, K=K, seed=4)
        with torch.no_grad():
            U = layer.current(x).contiguous()
            m, ts = layer.run_forward(U, tape=True)
            dm = torch.softmax(m, 1) - torch.nn.functional.one_hot(y, m.shape[1]).float()
            out.append((m, ts) + layer.run_backward(U, dm, ts))
        assert layer.status(16, 60) == [0, 0, 0, 0]
    for o in out[1:]:
        for a, b in zip(o, out[0]):
            assert torch.equal(a, b)


def test_plain_forward_equals_the_taped_one_and_the_tape_is_guarded(cuda):
    layer, x, y = make(cuda, B=8, T=40, seed=5)
    m_plain, ts_plain = layer.infer(x)
    m = layer(x)
    _, ts = layer.infer(x)
    assert torch.equal(m.detach(), m_plain) and torch.equal(ts, ts_plain)
    m1 = layer(x)
    layer(x)  # a later taped forward overwrites the tape
    with pytest.raises(RuntimeError, match="later forward"):
        torch.nn.functional.cross_entropy(m1, y).backward()


def test_workload_gradients_match_the_fp64_reference(cuda):
    """The BPTT workload at full size: B 128, T 500, 700 channels, 1024 hidden, 10% density, 20 readouts,
    checkpoints every 50 steps."""
    layer, x, y = bptt_task.build(seed=1, device=cuda)
    B, T = x.shape[1], x.shape[0]
    m, loss, grads = kernel_grads(layer, x, y)
    assert layer.status(B, T) == [0, 0, 0, 0]
    spikes = layer.spikes(B, T)
    rate = spikes.float().mean().item()
    assert 0.002 < rate < 0.3, rate
    _, ts = layer.infer(x)
    m64, _, margins, _, _, g64, _ = reference(layer, x, y, forced=spikes, forced_tstar=ts)
    assert ((margins >= 0) != spikes).float().mean() < 1e-5  # the float64 decisions agree but near threshold
    assert rel(m, m64) < 1e-5
    for g, r in zip(grads, g64):
        assert rel(g, r) < 1e-4


def test_projection_kernels_match_the_dense_product_and_repeat(cuda):
    """n2b_project_forward / n2b_project_backward against x @ w_in and x^T dU in float64 (1e-6 and 1e-5
    relative), on the BPTT workload's input statistics (some channels with far more events than others, so that
    channels span several chunks), bit-identical on a second call; empty rows and channels included."""
    from naer2_b200.bptt import SpikeEvents, project, project_grad

    T, B, C, H = 120, 64, 700, 1024
    rates = bptt_task.templates(classes=20, channels=C, steps=T, seed=5)
    x, _ = bptt_task.sample(rates, B, seed=6, device=cuda)
    x = x.clone()
    x[:, :, 3] = 0  # a channel without events
    x[7] = 0  # a step without events
    g = torch.Generator(device="cpu").manual_seed(7)
    w = torch.randn(C, H, generator=g).to(cuda)
    du = torch.randn(T, B, H, generator=g).to(cuda)
    ev = SpikeEvents.from_dense(x)
    assert ev.n_chunks > C // 2 and int((ev.channel_chunk[1:] - ev.channel_chunk[:-1]).max()) > 1
    xd = x.reshape(T * B, C).double()
    u, u2 = project(ev, w), project(ev, w)
    ref_u = (xd @ w.double()).reshape(T, B, H)
    assert torch.equal(u, u2)
    assert float((u.double() - ref_u).abs().max() / ref_u.abs().max()) < 1e-6
    dw, dw2 = project_grad(ev, du), project_grad(ev, du)
    ref_dw = xd.t() @ du.reshape(T * B, H).double()
    assert torch.equal(dw, dw2)
    assert float((dw.double() - ref_dw).abs().max() / ref_dw.abs().max()) < 1e-5
    assert float(dw[3].abs().max()) == 0.0


def test_groups_beyond_one_cooperative_launch(cuda):
    """B = 152 at H = 1024: 19 groups of 8 samples, more than one cooperative adjoint launch holds at one CTA per
    SM on 148 SMs (18 groups), so the last group runs in a second launch of each segment. Groups are
    independent: its samples' m, t* and dU equal those of the same 8 samples run alone, bit for bit."""
    T, B, C = 30, 152, 40
    layer = RecurrentLIF(n_in=C, hidden=1024, readouts=5, density=0.1, checkpoint=11, seed=9, device=cuda)
    rates = bptt_task.templates(classes=5, channels=C, steps=T, seed=9)
    x, y = bptt_task.sample(rates, B, seed=10, device=cuda)
    out = []
    for xb, yb in ((x, y), (x[:, B - 8:].contiguous(), y[B - 8:])):
        nb = xb.shape[1]
        with torch.no_grad():
            U = layer.current(xb).contiguous()
            m, ts = layer.run_forward(U, tape=True)
            dm = torch.softmax(m, 1) - torch.nn.functional.one_hot(yb, m.shape[1]).float()
            du, _, _ = layer.run_backward(U, dm, ts)
        torch.cuda.synchronize()
        assert layer.status(nb, T) == [0, 0, 0, 0]
        out.append((m[-8:], ts[-8:], du[:, -8:]))
    for a, b in zip(*out):
        assert torch.equal(a, b)
