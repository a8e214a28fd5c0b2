"""Hooks: a node's or edge's method parsed once into its AST, with the
members it assigns and a check of its annotated parameters (reference
naer2/types/hook.py:10-77, naer2/transpiler/analyzers/assigned_members.py)."""

from __future__ import annotations

import ast
import inspect
from inspect import Parameter, signature
from textwrap import dedent
from typing import Callable


def assigned_members(fn: ast.FunctionDef, root: str = "self") -> set[str]:
    """Names X of every `root.X = ...`, `root.X += ...` and `root.X: T = ...` in the function."""
    out: set[str] = set()
    for node in ast.walk(fn):
        targets = []
        if isinstance(node, ast.Assign):
            targets = node.targets
        elif isinstance(node, (ast.AugAssign, ast.AnnAssign)):
            targets = [node.target]
        for t in targets:
            for sub in ast.walk(t):
                if isinstance(sub, ast.Attribute) and isinstance(sub.value, ast.Name) and sub.value.id == root:
                    out.add(sub.attr)
    return out


def used_members(fn: ast.FunctionDef, root: str) -> set[str]:
    """Names X of every `root.X` the function mentions (read or written)."""
    return {n.attr for n in ast.walk(fn)
            if isinstance(n, ast.Attribute) and isinstance(n.value, ast.Name) and n.value.id == root}


class Hook:
    def __init__(self, name: str, function: Callable):
        if not isinstance(name, str):
            raise ValueError("Hook name must be a string")
        if not callable(function):
            raise ValueError("Hook function must be a Callable")
        self.name = name
        self.function = function
        tree = ast.parse(dedent(inspect.getsource(function)))
        if len(tree.body) != 1 or not isinstance(tree.body[0], ast.FunctionDef):
            raise ValueError(f"Can't parse {function!r}: its source is not one function")
        self.ast: ast.FunctionDef = tree.body[0]
        self.assigned_members: set[str] = assigned_members(self.ast)
        self.parameter_type_to_name: dict = {}

    def verify(self, allowed_types: set) -> "Hook":
        """Every annotated parameter's type in allowed_types, each at most once; every required parameter
        annotated (optional ones may stay bare)."""
        try:  # (string annotations, from `from __future__ import annotations`, evaluated)
            sig = signature(self.function, eval_str=True)
        except NameError:
            sig = signature(self.function)
        params = list(sig.parameters.values())
        skip = 0
        for index, p in enumerate(params):
            if p.name == "self":
                if index != 0:
                    raise TypeError(f"{self.name} must have 'self' as the first parameter.")
                skip = 1
        rest = params[skip:]
        annotated = [p for p in rest if p.annotation is not Parameter.empty]
        type_to_name = {p.annotation: p.name for p in annotated}
        if set(type_to_name) - set(allowed_types):
            raise TypeError(f"{self.name} arguments can only use types inside the allowed set.")
        for p in rest:
            if p.annotation is Parameter.empty and p.default is Parameter.empty:
                raise TypeError(f"Required parameter '{p.name}' of '{self.name}' must be annotated with an "
                                f"allowed type.")
        if len(type_to_name) != len(annotated):
            raise TypeError(f"Annotated parameters of '{self.name}' must each use a unique type "
                            f"(found duplicate annotations).")
        self.parameter_type_to_name = type_to_name
        return self
