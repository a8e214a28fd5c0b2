"""The BPTT workload on CPU: the FP64 reference's autograd against central finite differences in its smooth
model, the surrogate's spiking backward, the wiring the kernels read, and the synthetic task."""

import numpy as np
import pytest
import torch

from naer2_b200.bptt import MAX_DELAY, Wiring, draw_links
from naer2_b200.networks import bptt_task
from oracle import bptt_reference as ref


def small_problem(seed=0, T=25, B=3, C=10, H=16, R=4, density=0.3):
    g = torch.Generator().manual_seed(seed)
    pre, post, delay = draw_links(H, density, seed=seed)
    x = (torch.rand(T, B, C, generator=g) < 0.2).double()
    w_in = (torch.randn(C, H, generator=g, dtype=torch.float64) * 1.2).requires_grad_()
    w_rec = (torch.randn(len(pre), generator=g, dtype=torch.float64) * 0.4).requires_grad_()
    w_out = (torch.randn(H, R, generator=g, dtype=torch.float64) * 0.5).requires_grad_()
    y = torch.randint(0, R, (B,), generator=g)
    links = tuple(torch.from_numpy(a) for a in (pre, post, delay))
    return x, y, (w_in, w_rec, w_out), links


def test_reference_autograd_matches_finite_differences_in_the_smooth_model():
    """d loss / d(every weight) by autograd through the smooth model = central differences (float64)."""
    x, y, params, (pre, post, delay) = small_problem()
    consts = dict(alpha=float(np.exp(-1 / 20)), beta=float(np.exp(-1 / 20)), theta=1.0, slope=10.0, smooth=True)

    def L(*ps):
        m, *_ = ref.run(x, *ps, pre, post, delay, **consts)
        return ref.loss(m, y)

    grads = torch.autograd.grad(L(*params), params)
    g = torch.Generator().manual_seed(3)
    eps = 1e-6
    for i, (p, gp) in enumerate(zip(params, grads)):
        assert gp.abs().max() > 0
        for k in torch.randperm(p.numel(), generator=g)[:12].tolist():
            hi = [q.detach().clone() for q in params]
            lo = [q.detach().clone() for q in params]
            hi[i].view(-1)[k] += eps
            lo[i].view(-1)[k] -= eps
            fd = (L(*hi) - L(*lo)).item() / (2 * eps)
            got = gp.reshape(-1)[k].item()
            assert abs(fd - got) <= 1e-6 * max(1.0, abs(fd)), (i, k, fd, got)


def test_spiking_backward_uses_the_surrogate_and_forced_spikes():
    x, y, params, (pre, post, delay) = small_problem(seed=1)
    consts = dict(alpha=0.95, beta=0.95, theta=1.0, slope=10.0)
    m, ts, margins, spikes = ref.run(x, *params, pre, post, delay, **consts)
    assert torch.equal(spikes, (margins >= 0).double())  # Heaviside forward
    m2, ts2, _, spikes2 = ref.run(x, *params, pre, post, delay, forced=spikes.bool(), forced_tstar=ts, **consts)
    assert torch.equal(m, m2) and torch.equal(spikes, spikes2)
    grads = torch.autograd.grad(ref.loss(m, y), params)
    assert all(torch.isfinite(gr).all() and gr.abs().max() > 0 for gr in grads)


def test_wiring_rows_and_permutation():
    H = 64
    pre, post, delay = draw_links(H, 0.1, seed=5)
    assert len(pre) == round(0.1 * H * H) and len(set(zip(pre.tolist(), post.tolist()))) == len(pre)
    assert delay.min() >= 1 and delay.max() <= MAX_DELAY
    w = Wiring(pre, post, delay, H, "cpu")
    in_ptr = w.in_ptr.numpy()
    code = w.in_code.numpy().astype(np.int64)
    assert np.array_equal(code & 0x7FF, pre) and np.array_equal(code >> 11, delay)
    assert np.array_equal(np.repeat(np.arange(H), np.diff(in_ptr)), post)
    grp = w.out_grp.numpy().reshape(H, MAX_DELAY + 1)
    oc = w.out_code.numpy().astype(np.int64)
    perm = w.out_perm.numpy()
    for i in range(H):
        for d in range(1, MAX_DELAY + 1):
            seg = slice(grp[i, d - 1], grp[i, d])
            assert (oc[seg] >> 11 == d).all() and (pre[perm[seg]] == i).all()
            assert np.array_equal(oc[seg] & 0x7FF, post[perm[seg]])
    assert grp[-1, -1] == len(pre) and np.array_equal(np.sort(perm), np.arange(len(pre)))
    hc = H // 8
    assert w.in_cta_max == max(in_ptr[(r + 1) * hc] - in_ptr[r * hc] for r in range(8))
    with pytest.raises(ValueError):
        Wiring(pre[::-1].copy(), post[::-1].copy(), delay, H, "cpu")  # not in canonical order


def test_bank_order_spreads_the_gather_over_the_banks():
    """The outgoing order keeps every (pre, delay) group and lowers the passes of the adjoint's quarter-warp
    loads (8 threads of two neurons at the same chunk k; a pass per repeat of post mod 8)."""
    H = 1024
    pre, post, delay = draw_links(H, 0.1, seed=3)
    w = Wiring(pre, post, delay, H, "cpu")
    grp = w.out_grp.numpy().reshape(H, MAX_DELAY + 1)
    oc = w.out_code.numpy().astype(np.int64)
    sorted_post = post[np.lexsort((post, delay, pre))]

    def passes(targets):
        n = 0
        for i in range(0, H, 2):
            for d in range(MAX_DELAY):
                a, b = (targets[grp[j, d]:grp[j, d + 1]] % 8 for j in (i, i + 1))
                for k in range(0, max(len(a), len(b)), 4):
                    n += np.bincount(np.concatenate([a[k:k + 4], b[k:k + 4]]), minlength=8).max()
        return n

    for i in range(0, H, 97):
        for d in range(MAX_DELAY):
            seg = slice(grp[i, d], grp[i, d + 1])
            assert np.array_equal(np.sort(oc[seg] & 0x7FF), np.sort(sorted_post[seg]))
    assert passes(oc & 0x7FF) < 0.8 * passes(sorted_post)


def test_spike_events_by_row_and_by_channel_chunks():
    """SpikeEvents (CPU tensors here): the row lists reproduce x; the chunks cover each channel's rows in
    ascending order, at most CHUNK rows each, never two channels in one chunk; dense and sparse inputs agree."""
    from naer2_b200.bptt import SpikeEvents

    g = torch.Generator().manual_seed(3)
    T, B, C = 30, 8, 40
    x = (torch.rand(T, B, C, generator=g) < torch.linspace(0.0, 0.9, C)).float()  # channel 0 silent
    ev = SpikeEvents.from_dense(x)
    dense = torch.zeros(T * B, C)
    rows = torch.repeat_interleave(torch.arange(T * B), (ev.row_ptr[1:] - ev.row_ptr[:-1]).long())
    dense[rows, ev.channel.long()] = 1.0
    assert torch.equal(dense, x.reshape(T * B, C))
    for r in range(0, T * B, 17):
        ch = ev.channel[ev.row_ptr[r]:ev.row_ptr[r + 1]]
        assert torch.equal(ch, torch.sort(ch).values)
    cp, cc = ev.chunk_ptr.long(), ev.channel_chunk.long()
    assert int(cp[-1]) == ev.nnz == int(x.sum())
    for c in range(C):
        got = ev.row_idx[cp[cc[c]]:cp[cc[c + 1]]].long()
        assert torch.equal(got, torch.nonzero(x.reshape(T * B, C)[:, c]).reshape(-1))
        assert all(0 < int(cp[k + 1] - cp[k]) <= SpikeEvents.CHUNK for k in range(int(cc[c]), int(cc[c + 1])))
    assert int(cc[1]) == 0 and int((cc[1:] - cc[:-1]).max()) > 1
    sp = SpikeEvents.from_sparse(x.reshape(T * B, C).to_sparse(), T)
    for name in ("row_ptr", "channel", "row_idx", "chunk_ptr", "channel_chunk"):
        assert torch.equal(getattr(sp, name), getattr(ev, name))
    with pytest.raises(ValueError):
        SpikeEvents.from_dense(x * 2)


def test_task_templates_and_samples():
    rates = bptt_task.templates(classes=5, channels=50, steps=60, seed=2)
    assert rates.shape == (5, 60, 50) and rates.min() >= 0 and rates.max() <= 50
    x, y = bptt_task.sample(rates, 16, seed=3, device="cpu")
    assert x.shape == (60, 16, 50) and x.dtype == torch.bool and y.shape == (16,)
    x2, y2 = bptt_task.sample(rates, 16, seed=3, device="cpu")
    assert torch.equal(x, x2) and torch.equal(y, y2)  # seeded
    assert 0.001 < x.float().mean() < 0.05
