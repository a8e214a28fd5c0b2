"""naer2_b200: the per-timestep hot path of the naer2 spiking-network
simulator, rebuilt for NVIDIA B200 (sm_100a).

The DSL is the reference's (MatteoSchmider/naer2): @node / @edge / @pattern
classes, `Node(...) * n` populations, `pop_a >> edge @ pattern >> pop_b`
connections with per-link `weight` and `delay`, `Network.step(t)`. Networks
step at a fixed dt on the GPU: one fused CUDA kernel per step (membrane
update, spike-bit ring, push/pull delivery), windows of steps replayed from
one CUDA graph, through the C ABI of libnaer2b.so (include/naer2b.h).
"""

from . import models, patterns, receives, sends
from .connection import Connection, ConnectionBuilder
from .decorators import edge, node, pattern
from .network import Network
from .population import Population
from .receives import time
from .sends import spike
from .topology import Topology
from .types import Points, Position, Region

__all__ = ["edge", "node", "pattern", "Population", "Network", "Connection", "ConnectionBuilder", "Topology",
           "receives", "sends", "time", "spike", "Region", "Points", "Position", "models", "patterns"]
