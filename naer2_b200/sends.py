"""n2.spike() (reference naer2/sends.py:4-20): marks a spike emission inside a
node's send hook. The built-in CUDA models implement their hooks' spike sites
directly; the call itself does nothing when a hook runs as Python."""

from .receives import time


def spike(time: float = None):
    """Emit a spike of this neuron at this step (time: recorded as given; default the step)."""


__all__ = ["time", "spike"]
