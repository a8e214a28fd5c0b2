"""Built-in neuron models: node classes whose hooks the CUDA step kernel
implements by hand (csrc/n2b_device.cuh), as the reference pairs PD14's
hooks with its hand-written kernel (test/fused_reference.py:35-114,
pd14_neuron_reference). Each class is an ordinary @n2.node with Python
hooks stating its semantics at a fixed step dt; `kernel_params(pop, dt)`
gives what the kernel needs.

Every model sums its synaptic input of a step exactly (int64 fixed point,
the population's `shift`) and converts it to float once; its external
Poisson drive (if any) joins that sum as events of weight ext_weight.
"""

from __future__ import annotations

import math
import random

import numpy as np

from . import receives as _r
from ._lib import MODEL_LIF_DELTA, MODEL_PD14, MODEL_POISSON_SOURCE
from .decorators import node
from .poisson import cdf_table
from .sends import spike


def _f32(x: float) -> float:
    return float(np.float32(x))


class KernelParams(dict):
    """model, p (8 floats), ref_steps, ext_lambda, ext_weight, fire_threshold, state {kernel slot: attr},
    port (the attr receive accumulates into: the arrival ring, no tensor)."""


@node
class LIF:
    """Brunel's LIF with delta synapses, time-driven (the reference's tools/brunel_reference.py:34-48):
    every step the arriving input I (recurrent links + ext_weight x Poisson(ext_rate dt) external events)
    is summed; a refractory neuron keeps V and drops it; otherwise V = V exp(-dt/tau) + I, and at
    V >= theta it spikes, resets to V_r and stays refractory for round(t_ref / dt) steps (the reference's
    `t > ref_until` test at dt = 0.1: exactly 20 steps for t_ref = 2 ms).

    Units ms / mV. ext_rate: external events per ms (C_E nu_ext for Brunel's model A)."""

    def __init__(self, tau: float = 20.0, theta: float = 20.0, V_r: float = 10.0, t_ref: float = 2.0,
                 ext_rate: float = 0.0, ext_weight: float = 0.0):
        self.tau = tau
        self.theta = theta
        self.V_r = V_r
        self.t_ref = t_ref
        self.ext_rate = ext_rate
        self.ext_weight = ext_weight
        self.decay = 1.0  # exp(-dt / tau) once the network's dt is known (kernel_params)
        self.ref_steps = 0
        self.V: float = 0.0
        self.ref: int = 0
        self.I: float = 0.0  # the step's summed input: the population's arrival ring, not a state tensor

    def receive(self, time: _r.time, edge: _r.edge, source: _r.source):
        self.I += edge.weight

    def update(self, time: _r.time):
        if self.ref > 0:
            self.ref -= 1
        else:
            self.V = self.V * self.decay + self.I
        self.I = 0.0

    def send(self, time: _r.time):
        if self.ref == 0 and self.V >= self.theta:
            spike()
            self.V = self.V_r
            self.ref = self.ref_steps

    @staticmethod
    def kernel_params(inst, dt: float) -> KernelParams:
        return KernelParams(
            model=MODEL_LIF_DELTA,
            p=[_f32(math.exp(-dt / inst.tau)), _f32(inst.theta), _f32(inst.V_r)],
            ref_steps=int(round(inst.t_ref / dt)),
            ext_lambda=inst.ext_rate * dt, ext_weight=float(inst.ext_weight),
            state={"v": "V", "ref": "ref"}, port="I")


@node
class PD14_neuron:
    """PD14's LIF with exponential current synapses (the reference's test/networks/PD14/neuron.py:143-189,
    same parameters) at a fixed step dt: receive adds the step's input (recurrent links + J_ext x
    Poisson(nu_ext K_cortical dt) background events) to `current`; update integrates with the exact
    propagators P_V = exp(-dt/t_mem), P_I = exp(-dt/t_syn), P_VI = R t_syn/(t_mem - t_syn) (P_V - P_I)
    (fp64 on the host, rounded to fp32) -- V clamped at V_reset while refractory; send spikes at
    V > V_thresh, resets, and clamps the next round(t_ref/dt) - 1 steps (the hook's `time < t_ref_end`).

    background: "poisson" (explicit background events; V_rest = E_leak) or "dc" (the reference's DC
    approximation, V_rest = E_leak + R_mem K nu_ext J_ext t_syn, no events). Units ms / mV / nA / MOhm."""

    def __init__(self, K_cortical: int, t_mem: float = 10.0, t_syn: float = 0.5, t_ref: float = 2.0,
                 R_mem: float = 40.0, E_leak: float = -65.0, V_thresh: float = -50.0, V_reset: float = -65.0,
                 nu_ext: float = 8e-3, J_ext: float = 0.08781, background: str = "poisson"):
        if background not in ("poisson", "dc"):
            raise ValueError("background is 'poisson' or 'dc'")
        self.K_cortical = K_cortical
        self.t_mem = t_mem
        self.t_syn = t_syn
        self.t_ref = t_ref
        self.R_mem = R_mem
        self.V_thresh = V_thresh
        self.V_reset = V_reset
        self.nu_ext = nu_ext
        self.J_ext = J_ext
        self.background = background
        self.V_rest = E_leak if background == "poisson" else E_leak + R_mem * K_cortical * nu_ext * J_ext * t_syn
        self.P_V = self.P_I = self.P_VI = 0.0  # the propagators once dt is known (kernel_params)
        self.ref_steps = 0
        self.potential: float = V_reset
        self.current: float = 0.0
        self.ref: int = 0
        self.I: float = 0.0  # the step's summed input: the arrival ring

    def receive(self, time: _r.time, edge: _r.edge, source: _r.source):
        self.I += edge.weight

    def update(self, time: _r.time):
        self.current += self.I
        self.I = 0.0
        if self.ref > 0:
            self.ref -= 1
            self.potential = self.V_reset
        else:
            self.potential = self.V_rest + self.P_V * (self.potential - self.V_rest) + self.P_VI * self.current
        self.current = self.P_I * self.current

    def send(self, time: _r.time):
        if self.potential > self.V_thresh:
            spike()
            self.potential = self.V_reset
            self.ref = self.ref_steps

    @staticmethod
    def kernel_params(inst, dt: float) -> KernelParams:
        P_V = math.exp(-dt / inst.t_mem)
        P_I = math.exp(-dt / inst.t_syn)
        P_VI = inst.R_mem * inst.t_syn / (inst.t_mem - inst.t_syn) * (P_V - P_I)
        poisson = inst.background == "poisson"
        return KernelParams(
            model=MODEL_PD14,
            p=[_f32(P_V), _f32(P_I), _f32(P_VI), _f32(inst.V_rest), _f32(inst.V_thresh), _f32(inst.V_reset)],
            ref_steps=max(int(round(inst.t_ref / dt)) - 1, 0),
            ext_lambda=inst.nu_ext * inst.K_cortical * dt if poisson else 0.0,
            ext_weight=float(inst.J_ext) if poisson else 0.0,
            state={"v": "potential", "i": "current", "ref": "ref"}, port="I")


@node(receive=None)
class Poisson_source:
    """Independent Poisson spike trains on the step grid: each neuron spikes in a step with probability
    1 - exp(-rate dt) (rate in spikes / ms), one uniform draw per neuron and step."""

    def __init__(self, rate: float):
        self.rate = rate
        self.p_fire = 0.0  # once dt is known

    def update(self, time: _r.time):
        pass

    def send(self, time: _r.time):
        if random.random() < self.p_fire:
            spike()

    @staticmethod
    def kernel_params(inst, dt: float) -> KernelParams:
        p = 1.0 - math.exp(-inst.rate * dt)
        return KernelParams(model=MODEL_POISSON_SOURCE, p=[], ref_steps=0, ext_lambda=0.0, ext_weight=0.0,
                            fire_threshold=min(int(math.floor(p * 4294967296.0)), 0xFFFFFFFF), state={},
                            port=None)


BUILTIN = (LIF, PD14_neuron, Poisson_source)


def params_of(pop, dt: float) -> KernelParams:
    """The kernel parameters of a population's built-in model (its instance's values at step dt); the
    inverse-CDF table of its external drive as `ext_table`."""
    cls = type(pop.instance)
    if cls not in BUILTIN:
        raise NotImplementedError(f"{cls.__name__} is not a built-in CUDA model ({', '.join(c.__name__ for c in BUILTIN)}): "
                                  f"a network with it runs on the transpiled path (naer2_b200.transpiler)")
    kp = cls.kernel_params(pop.instance, dt)
    kp.setdefault("fire_threshold", 0)
    kp["ext_table"] = cdf_table(kp["ext_lambda"]) if kp["ext_lambda"] > 0 and kp["ext_weight"] != 0 else \
        np.zeros(0, dtype=np.uint32)
    kp["p"] = list(kp["p"]) + [0.0] * (8 - len(kp["p"]))
    return kp


__all__ = ["LIF", "PD14_neuron", "Poisson_source", "params_of", "BUILTIN"]
