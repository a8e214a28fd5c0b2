"""A recurrent LIF layer trained by surrogate-gradient BPTT, on the library's forward and adjoint kernels.

The layer: input spikes x [T, B, C] -> input current U = x @ w_in (`n2b_project_forward` over the input's
spike events, `SpikeEvents`; its gradient to w_in by `n2b_project_backward`) -> H recurrent LIF neurons with
sparse delayed recurrence (w_rec, delays 1..5 steps) -> R leaky non-spiking readouts; the output is the max
over time of each readout, m [B, R], for a cross-entropy loss.
The recurrence and its adjoint run in `n2b_bptt_forward` / `n2b_bptt_backward` (naer2_b200/csrc/bptt.cu)
behind `torch.autograd.Function`: the forward keeps the spikes of every step (one bit per neuron, sample and
step) and the membrane every `checkpoint` steps; the backward recomputes each segment from its checkpoint and
runs it backwards over the transposed (outgoing) rows. The model equations are stated in include/naer2b.h.

naer2 itself has no differentiable path; this layer follows the BPTT workload's description (700 input
channels, 1024 hidden neurons at 10% recurrent density, delays of 1-5 steps, 20 readouts, fast-sigmoid
surrogate of slope 10, checkpoints every 50 steps).
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib

MAX_DELAY = 5


def draw_links(hidden: int, density: float, max_delay: int = MAX_DELAY, seed: int = 0):
    """round(density * H^2) distinct (pre, post) pairs (self-links allowed), delays uniform in 1..max_delay:
    (pre, post, delay) int64 arrays in the canonical (incoming) order, sorted by (post, pre)."""
    n = int(round(density * hidden * hidden))
    rng = np.random.Generator(np.random.Philox(seed))
    flat = np.sort(rng.choice(hidden * hidden, size=n, replace=False))
    post, pre = np.divmod(flat, hidden)  # flat = post * H + pre: sorted by (post, pre)
    delay = rng.integers(1, max_delay + 1, size=n)
    return pre.astype(np.int64), post.astype(np.int64), delay.astype(np.int64)


def bank_order(post: np.ndarray, grp: np.ndarray) -> np.ndarray:
    """An order of the outgoing links within each (pre, delay) group for the adjoint's shared-memory gather.

    The adjoint gives each neuron four threads; the thread `sub` of a neuron takes the links 4k + sub of each
    of its delay groups (k = 0, 1, ...), and one 128-bit load of a quarter warp serves the 8 threads of two
    neurons 2i, 2i + 1 at the same k. Each thread reads the q row of its link's target, rows 48 bytes apart,
    so the load touches the 16-byte bank group (3 post + half) mod 8: targets with distinct post mod 8 are
    served in one pass, equal ones in several. Greedily, each chunk k of the two neurons' groups takes links
    with distinct residues mod 8, the most frequent remaining residues first. Returns positions into `post`
    (a permutation within each group); the sums are the same up to their order."""
    hidden = grp.shape[0]
    perm = np.arange(len(post))
    res = post % 8
    for i in range(0, hidden, 2):
        for d in range(MAX_DELAY):
            spans = [(grp[j, d], grp[j, d + 1]) for j in (i, i + 1) if j < hidden]
            pools = []
            for s, e in spans:
                pool = [[] for _ in range(8)]
                for j in range(s, e):
                    pool[res[j]].append(j)
                pools.append(pool)
            outs = [[] for _ in spans]
            while any(len(o) < e - s for o, (s, e) in zip(outs, spans)):
                used = set()
                for pool, out, (s, e) in zip(pools, outs, spans):
                    take, got = min(4, e - s - len(out)), 0
                    for r in sorted(range(8), key=lambda r: -len(pool[r])):
                        if got == take:
                            break
                        if pool[r] and r not in used:
                            out.append(pool[r].pop())
                            used.add(r)
                            got += 1
                    while got < take:  # no distinct residue left: the fullest one
                        out.append(pool[max(range(8), key=lambda r: len(pool[r]))].pop())
                        got += 1
            for out, (s, e) in zip(outs, spans):
                perm[s:e] = out
    return perm


class Wiring:
    """The recurrent links as the kernels read them: incoming rows (the weights' order) and outgoing rows
    sorted by delay (each delay group in `bank_order`), with the permutation between the two."""

    def __init__(self, pre, post, delay, hidden: int, device):
        pre, post, delay = (np.asarray(a, dtype=np.int64) for a in (pre, post, delay))
        if hidden > 2048 or (len(pre) and (pre.max() >= hidden or post.max() >= hidden)):
            raise ValueError("neuron index out of range (at most 2048 hidden neurons)")
        if len(delay) and (delay.min() < 1 or delay.max() > MAX_DELAY):
            raise ValueError(f"delays must be 1..{MAX_DELAY} steps")
        order = np.lexsort((pre, post))
        if not np.array_equal(order, np.arange(len(pre))):
            raise ValueError("links must be sorted by (post, pre)")
        self.hidden, self.nnz = hidden, len(pre)
        self.pre, self.post, self.delay = pre, post, delay
        in_ptr = np.zeros(hidden + 1, dtype=np.int64)
        np.add.at(in_ptr, post + 1, 1)
        in_ptr = np.cumsum(in_ptr)
        out_order = np.lexsort((post, delay, pre))  # by pre, then delay, then post
        out_pre, out_post, out_delay = pre[out_order], post[out_order], delay[out_order]
        grp = np.zeros((hidden, MAX_DELAY + 1), dtype=np.int64)
        counts = np.zeros((hidden, MAX_DELAY), dtype=np.int64)
        np.add.at(counts, (out_pre, out_delay - 1), 1)
        row_start = np.concatenate([[0], np.cumsum(counts.sum(1))[:-1]])
        grp[:, 0] = row_start
        grp[:, 1:] = row_start[:, None] + np.cumsum(counts, axis=1)
        out_order = out_order[bank_order(out_post, grp)]
        out_post, out_delay = post[out_order], delay[out_order]
        hc = hidden // 8
        self.in_cta_max = int(max((in_ptr[(r + 1) * hc] - in_ptr[r * hc] for r in range(8)), default=0))
        self.out_cta_max = int(max((grp[(r + 1) * hc - 1, -1] - grp[r * hc, 0] for r in range(8)), default=0))
        dev = torch.device(device)
        self.in_ptr = torch.from_numpy(in_ptr.astype(np.int32)).to(dev)
        self.in_code = torch.from_numpy((pre | (delay << 11)).astype(np.int16)).to(dev)
        self.out_grp = torch.from_numpy(grp.astype(np.int32).reshape(-1)).to(dev)
        self.out_code = torch.from_numpy((out_post | (out_delay << 11)).astype(np.int16)).to(dev)
        self.out_perm = torch.from_numpy(out_order.astype(np.int32)).to(dev)
        self.out_degree = torch.from_numpy(np.bincount(pre, minlength=hidden)).to(dev)


class SpikeEvents:
    """Binary input spikes x [T, B, C] as the projection kernels read them, built once per input (like a data
    loader's output): by input row r = t * B + b (`row_ptr` [T*B + 1], `channel`: its spiking channels,
    ascending) and by channel in chunks of at most CHUNK rows (`row_idx`: rows ascending per channel,
    `chunk_ptr` [n_chunks + 1], `channel_chunk` [C + 1]: each channel's first chunk)."""

    CHUNK = 128

    def __init__(self, rows: torch.Tensor, chans: torch.Tensor, steps: int, batch: int, channels: int):
        n_rows = steps * batch
        rows, chans = rows.long().reshape(-1), chans.long().reshape(-1)
        if rows.numel() and (int(rows.min()) < 0 or int(rows.max()) >= n_rows or int(chans.min()) < 0
                             or int(chans.max()) >= channels):
            raise ValueError("spike event out of range")
        dev = rows.device
        key = torch.unique(rows * channels + chans)  # sorted by (row, channel), duplicates merged
        r, c = key // channels, key % channels
        self.steps, self.batch, self.channels, self.nnz = steps, batch, channels, int(key.numel())
        self.row_ptr = torch.zeros(n_rows + 1, dtype=torch.int32, device=dev)
        self.row_ptr[1:] = torch.cumsum(torch.bincount(r, minlength=n_rows), 0)
        self.channel = c.int()
        key2 = torch.sort(c * n_rows + r).values  # by (channel, row)
        c2 = key2 // n_rows
        self.row_idx = (key2 % n_rows).int()
        counts = torch.bincount(c2, minlength=channels)
        col_start = torch.zeros(channels + 1, dtype=torch.long, device=dev)
        col_start[1:] = torch.cumsum(counts, 0)
        chunks = (counts + self.CHUNK - 1) // self.CHUNK
        self.channel_chunk = torch.zeros(channels + 1, dtype=torch.int32, device=dev)
        self.channel_chunk[1:] = torch.cumsum(chunks, 0)
        self.n_chunks = int(self.channel_chunk[-1])
        owner = torch.repeat_interleave(torch.arange(channels, device=dev), chunks)
        j = torch.arange(self.n_chunks, device=dev) - self.channel_chunk[owner].long()
        start = col_start[owner] + j * self.CHUNK
        self.chunk_ptr = torch.cat([start, torch.tensor([self.nnz], device=dev)]).int()

    @classmethod
    def from_dense(cls, x: torch.Tensor) -> "SpikeEvents":
        T, B, C = x.shape
        if bool(((x != 0) & (x != 1)).any()):
            raise ValueError("the input must be binary spikes")
        idx = torch.nonzero(x.reshape(T * B, C))
        return cls(idx[:, 0], idx[:, 1], T, B, C)

    @classmethod
    def from_sparse(cls, x: torch.Tensor, steps: int) -> "SpikeEvents":
        x = x.coalesce()
        if bool((x.values() != 1).any()):
            raise ValueError("the input must be binary spikes")
        n_rows, C = x.shape
        if n_rows % steps:
            raise ValueError("rows of the sparse input must be steps x batch")
        return cls(x.indices()[0], x.indices()[1], steps, n_rows // steps, C)


def project(events: SpikeEvents, w_in: torch.Tensor) -> torch.Tensor:
    """U [T, B, H] = x @ w_in through n2b_project_forward (channel order per row)."""
    C, H = w_in.shape
    if C != events.channels or not w_in.is_cuda or w_in.dtype != torch.float32:
        raise RuntimeError("w_in must be a CUDA fp32 [channels, hidden] tensor (no CPU fallback)")
    w = w_in.detach().contiguous()
    u = torch.empty(events.steps, events.batch, H, dtype=torch.float32, device=w.device)
    s = ctypes.c_void_p(torch.cuda.current_stream(w.device).cuda_stream)
    _lib.check(_lib.load().n2b_project_forward(events.row_ptr.data_ptr(), events.channel.data_ptr(),
                                               events.steps * events.batch, C, H, w.data_ptr(), u.data_ptr(), s),
               "n2b_project_forward")
    return u


def project_grad(events: SpikeEvents, du: torch.Tensor) -> torch.Tensor:
    """dw_in [C, H] = x^T du through n2b_project_backward (per channel: chunks of rows, then the chunks in order)."""
    du = du.contiguous()
    H = du.shape[-1]
    partials = torch.empty(max(events.n_chunks, 1), H, dtype=torch.float32, device=du.device)
    dw = torch.empty(events.channels, H, dtype=torch.float32, device=du.device)
    s = ctypes.c_void_p(torch.cuda.current_stream(du.device).cuda_stream)
    _lib.check(_lib.load().n2b_project_backward(events.chunk_ptr.data_ptr(), events.n_chunks,
                                                events.row_idx.data_ptr(), events.channel_chunk.data_ptr(),
                                                events.channels, events.steps * events.batch, H, du.data_ptr(),
                                                partials.data_ptr(), dw.data_ptr(), s), "n2b_project_backward")
    return dw


class _ProjectFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, w_in, events):
        ctx.events = events
        return project(events, w_in)

    @staticmethod
    def backward(ctx, du):
        return (project_grad(ctx.events, du) if ctx.needs_input_grad[0] else None), None


class RecurrentLIF(torch.nn.Module):
    """The BPTT workload's layer. Parameters: w_in [C, H], w_rec [nnz] (canonical order: by post, then pre),
    w_out [H, R]. `forward(x)` returns m [B, R]; `infer(x)` is the plain forward (no tape, no autograd)."""

    def __init__(self, n_in: int = 700, hidden: int = 1024, readouts: int = 20, density: float = 0.1,
                 tau_mem: float = 20.0, tau_out: float = 20.0, dt: float = 1.0, theta: float = 1.0,
                 slope: float = 10.0, checkpoint: int = 50, seed: int = 0, device="cuda", smooth: bool = False,
                 links=None, w_scale: tuple = (4.0, 0.5, 1.0)):
        super().__init__()
        if hidden % 32 or hidden > 1024:
            raise ValueError("hidden must be a multiple of 32, at most 1024")
        self.n_in, self.hidden, self.readouts = n_in, hidden, readouts
        self.alpha = float(np.float32(math.exp(-dt / tau_mem)))
        self.beta = float(np.float32(math.exp(-dt / tau_out)))
        self.theta, self.slope, self.checkpoint, self.smooth = float(theta), float(slope), int(checkpoint), smooth
        dev = torch.device(device)
        pre, post, delay = links if links is not None else draw_links(hidden, density, seed=seed)
        self.wiring = Wiring(pre, post, delay, hidden, dev)
        gen = torch.Generator(device="cpu").manual_seed(seed + 1)
        fan_rec = max(1.0, self.wiring.nnz / hidden)
        s_in, s_rec, s_out = w_scale
        self.w_in = torch.nn.Parameter((torch.randn(n_in, hidden, generator=gen) * s_in / math.sqrt(n_in)).to(dev))
        self.w_rec = torch.nn.Parameter(
            (torch.randn(self.wiring.nnz, generator=gen) * s_rec / math.sqrt(fan_rec)).to(dev))
        self.w_out = torch.nn.Parameter(
            (torch.randn(hidden, readouts, generator=gen) * s_out / math.sqrt(hidden)).to(dev))
        self._ws = None
        self._ws_key = None
        self.tape_id = 0
        # polls before a wait of the backward's per-step exchange gives up (0: the library's default, about a
        # second); tests set a few to make the wait give up without a hang
        self.wait_polls = 0

    # ------------------------------------------------------------------ the kernels' view

    def desc(self, batch: int, steps: int) -> _lib.BpttDesc:
        w = self.wiring
        d = _lib.BpttDesc()
        d.batch, d.steps, d.hidden, d.readouts = batch, steps, self.hidden, self.readouts
        d.checkpoint, d.smooth, d.nnz = self.checkpoint, int(self.smooth), w.nnz
        d.in_cta_max, d.out_cta_max = w.in_cta_max, w.out_cta_max
        d.alpha, d.beta, d.theta, d.slope = self.alpha, self.beta, self.theta, self.slope
        d.in_ptr, d.in_code, d.out_grp = w.in_ptr.data_ptr(), w.in_code.data_ptr(), w.out_grp.data_ptr()
        d.out_code, d.out_perm = w.out_code.data_ptr(), w.out_perm.data_ptr()
        d.wait_polls = int(self.wait_polls)
        return d

    def workspace(self, d: _lib.BpttDesc) -> torch.Tensor:
        key = (d.batch, d.steps, d.checkpoint, d.smooth)
        if self._ws_key != key:
            n = ctypes.c_size_t()
            lib = _lib.load()
            _lib.check(lib.n2b_bptt_workspace_bytes(ctypes.byref(d), ctypes.byref(n)), "n2b_bptt_workspace_bytes")
            self._ws = torch.empty(n.value, dtype=torch.uint8, device=self.w_in.device)
            self._ws_key = key
        return self._ws

    def current(self, x, steps: int | None = None) -> torch.Tensor:
        """U [T, B, H] = x @ w_in (autograd to w_in). x: SpikeEvents, binary [T, B, C] (dense), or a sparse COO
        matrix [T * B, C] (row t * B + b) with `steps` = T; the last two are turned into SpikeEvents on every
        call, so a caller that reuses an input builds its SpikeEvents once."""
        if not isinstance(x, SpikeEvents):
            if x.is_sparse:
                if steps is None:
                    raise ValueError("a sparse input needs steps=T")
                x = SpikeEvents.from_sparse(x, steps)
            else:
                x = SpikeEvents.from_dense(x)
        return _ProjectFn.apply(self.w_in, x)

    def forward(self, x: torch.Tensor, steps: int | None = None) -> torch.Tensor:
        U = self.current(x, steps)
        return _BpttFn.apply(U.contiguous(), self.w_rec, self.w_out, self)

    @torch.no_grad()
    def infer(self, x: torch.Tensor, steps: int | None = None):
        """The plain forward: (m [B, R], t* [B, R]) with no tape."""
        U = self.current(x, steps).contiguous()
        return self.run_forward(U, tape=False)

    def run_forward(self, U: torch.Tensor, tape: bool):
        T, B, H = U.shape
        if U.dtype != torch.float32 or not U.is_cuda:
            raise RuntimeError("the layer runs on a CUDA device with fp32 currents (no CPU fallback)")
        d = self.desc(B, T)
        ws = self.workspace(d)
        m = torch.empty(B, self.readouts, dtype=torch.float32, device=U.device)
        ts = torch.empty(B, self.readouts, dtype=torch.int32, device=U.device)
        s = ctypes.c_void_p(torch.cuda.current_stream(U.device).cuda_stream)
        _lib.check(_lib.load().n2b_bptt_forward(ctypes.byref(d), U.data_ptr(), self.w_rec.data_ptr(),
                                                self.w_out.data_ptr(), int(tape), m.data_ptr(), ts.data_ptr(),
                                                ws.data_ptr(), ws.numel(), s), "n2b_bptt_forward")
        if tape:
            self.tape_id += 1
        return m, ts

    def run_backward(self, U, dm, ts):
        T, B, H = U.shape
        d = self.desc(B, T)
        ws = self.workspace(d)
        du = torch.empty_like(U)
        dw_rec = torch.empty_like(self.w_rec)
        dw_out = torch.empty_like(self.w_out)
        dm = dm.contiguous()
        s = ctypes.c_void_p(torch.cuda.current_stream(U.device).cuda_stream)
        _lib.check(_lib.load().n2b_bptt_backward(ctypes.byref(d), U.data_ptr(), self.w_rec.data_ptr(),
                                                 self.w_out.data_ptr(), dm.data_ptr(), ts.data_ptr(),
                                                 du.data_ptr(), dw_rec.data_ptr(), dw_out.data_ptr(),
                                                 ws.data_ptr(), ws.numel(), s), "n2b_bptt_backward")
        return du, dw_rec, dw_out

    def status(self, batch: int, steps: int) -> list:
        d = self.desc(batch, steps)
        ws = self.workspace(d)
        words = (ctypes.c_int32 * _lib.BPTT_ERR_WORDS)()
        s = ctypes.c_void_p(torch.cuda.current_stream(ws.device).cuda_stream)
        _lib.check(_lib.load().n2b_bptt_status(ctypes.byref(d), ws.data_ptr(), ws.numel(), words, s),
                   "n2b_bptt_status")
        return list(words)

    def spikes(self, batch: int, steps: int) -> torch.Tensor:
        """The last taped forward's spikes as [T, B, H] (bool; float in the smooth model)."""
        d = self.desc(batch, steps)
        ws = self.workspace(d)
        NC, H = batch // 8, self.hidden
        s = ctypes.c_void_p(torch.cuda.current_stream(ws.device).cuda_stream)
        if self.smooth:
            out = torch.empty(steps, NC, H, 8, dtype=torch.float32, device=ws.device)
            _lib.check(_lib.load().n2b_bptt_spikes(ctypes.byref(d), ws.data_ptr(), ws.numel(), out.data_ptr(), s),
                       "n2b_bptt_spikes")
            return out.permute(0, 1, 3, 2).reshape(steps, batch, H)
        raw = torch.empty(steps, NC, H, dtype=torch.uint8, device=ws.device)
        _lib.check(_lib.load().n2b_bptt_spikes(ctypes.byref(d), ws.data_ptr(), ws.numel(), raw.data_ptr(), s),
                   "n2b_bptt_spikes")
        bits = (raw.unsqueeze(-1) >> torch.arange(8, device=ws.device, dtype=torch.uint8)) & 1
        return bits.permute(0, 1, 3, 2).reshape(steps, batch, H).bool()


class _BpttFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, U, w_rec, w_out, layer):
        m, ts = layer.run_forward(U, tape=True)
        ctx.layer, ctx.tape_id = layer, layer.tape_id
        ctx.save_for_backward(U, ts)
        ctx.mark_non_differentiable(ts)
        return m

    @staticmethod
    def backward(ctx, dm):
        U, ts = ctx.saved_tensors
        layer = ctx.layer
        if layer.tape_id != ctx.tape_id:
            raise RuntimeError("the layer's tape belongs to a later forward: run backward before the next forward")
        du, dw_rec, dw_out = layer.run_backward(U, dm, ts)
        return du, dw_rec, dw_out, None
