"""What the decorators register (reference naer2/nodes.py, edges.py, patterns.py)."""

from dataclasses import dataclass

from .hook import Hook


@dataclass
class Node:
    send: Hook
    update: Hook
    receive: dict  # port -> Hook


node_types: dict = {}
edge_types: dict = {}
pattern_types: dict = {}
