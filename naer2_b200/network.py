"""Network: the populations and connections one DSL chain joined (reference
naer2/network.py:16-79), stepped at a fixed dt (`resolution`, ms).

Network.step(t) advances round(t / dt) steps on the GPU: whole windows of
`window` steps replay one captured CUDA graph, the remainder launches step
by step (reference naer2/network.py:80-152, 264-321: the host scheduler's
rounds and captured windows become one graph of fixed-dt steps). The first
step builds the runtime (naer2_b200/runtime.py); the network's structure is
fixed from then on.
"""

from __future__ import annotations

import math

import torch


class Network:
    def __init__(self, population):
        self.populations: list = [population]
        self.connections: list = []
        self.t: float = 0.0
        self.step_count: int = 0
        self.resolution: float = 0.1  # the step dt (ms)
        self.window: int = 100  # steps per captured graph
        self.block: int | None = None  # neurons per block (None: the smallest population group_size)
        self.grid: int | None = None  # blocks per launch (None: two per SM)
        # a window of steps as one persistent cooperative launch (steps separated by a grid barrier), or one
        # launch per step
        self.persistent: bool = True
        # persistent windows: how long a block may wait at a grid barrier before the window stops with an error
        # word (0: the library's 2 s); tests set a few ns to make the wait give up without a hang
        self.barrier_limit_ns: int = 0
        self.device = torch.device("cuda", torch.cuda.current_device()) if torch.cuda.is_available() else None
        self.record_steps: int = 0  # raster rows kept per population (Network.record)
        self.tuned: dict = {}  # per connection id: the push/pull choice the tuner measured (naer2_b200.tune)
        # event-driven intake at exact spike times (the transpiled path; naer2_b200.transpiler.template)
        self.exact: bool = False
        self.tune_report: dict | None = None
        self._runtime = None

    # ------------------------------------------------------------------ structure

    def merge(self, other: "Network") -> "Network":
        if other is self:
            return self
        if self._runtime is not None or other._runtime is not None:
            raise RuntimeError("a network's structure is fixed once it has run")
        for pop in other.populations:
            object.__setattr__(pop, "network", self)
            if pop not in self.populations:
                self.populations.append(pop)
        for conn in other.connections:
            if conn not in self.connections:
                self.connections.append(conn)
        self.populations.sort(key=lambda p: p._order)  # creation order, whatever the merges' order
        self.connections.sort(key=lambda c: c._order)
        return self

    def __add__(self, other):
        return self.merge(other)

    def __iadd__(self, other):
        return self.merge(other)

    # ------------------------------------------------------------------ running

    @property
    def runtime(self):
        """The GPU runtime, built on first use (no CPU fallback: raises without CUDA)."""
        if self._runtime is None:
            if self.device is None or self.device.type != "cuda":
                raise RuntimeError("naer2_b200 steps networks on a CUDA device only (no CPU fallback)")
            from .models import BUILTIN
            from .runtime import NetworkRuntime

            if not self.exact and all(type(p.instance) in BUILTIN for p in self.populations):
                self._runtime = NetworkRuntime(self)
            else:  # a model without a built-in kernel: every population's hooks transpiled, compiled at run time
                from .transpiler import JitRuntime

                self._runtime = JitRuntime(self)
        return self._runtime

    def steps_for(self, t_step: float) -> int:
        n = t_step / self.resolution
        k = int(round(n))
        if abs(n - k) > 1e-6 * max(1.0, abs(n)):
            raise ValueError(f"t_step={t_step} is not a whole number of steps of dt={self.resolution}")
        return k

    def step(self, t_step: float) -> None:
        """Advance by t_step ms (a whole number of steps)."""
        self.run_steps(self.steps_for(t_step))

    def run_steps(self, n_steps: int) -> None:
        if n_steps < 0:
            raise ValueError("n_steps < 0")
        self.runtime.advance(n_steps)
        self.step_count += n_steps
        self.t = self.step_count * self.resolution

    def record(self, steps: int) -> None:
        """Keep the spike raster of the next `steps` steps of every population (Population.spikes)."""
        if self._runtime is not None:
            self._runtime.start_recording(steps)
        self.record_steps = int(steps)

    def check(self) -> None:
        """Raise on links the kernels found out of range (error words; a synchronisation)."""
        if self._runtime is not None:
            self._runtime.check()

    def counters(self) -> dict:
        """Synaptic events and spikes so far (a synchronisation)."""
        return self.runtime.counters()

    def synapses(self) -> int:
        return sum(len(c.fabric.topology) for c in self.connections)

    def close(self) -> None:
        """Release the runtime (its graph and device buffers)."""
        if self._runtime is not None:
            self._runtime.close()
            self._runtime = None

    @staticmethod
    def next_pow2(x: int) -> int:
        return 1 << max(0, math.ceil(math.log2(max(x, 1))))
