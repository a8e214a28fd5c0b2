"""Python hook AST -> CUDA C++ statements (the transpiler's lowering; reference naer2/transpiler/
hook_transpiler.py:17-120 and its transformers, which lower the same hooks to Triton/Gluon block code).

Here a hook body becomes scalar CUDA code run by one thread per neuron (and, for receive, once per arrived
link). Names are resolved as follows:
  self.<x>   a dynamic attribute -> the thread's register copy s_<x>; a static one -> its literal value
  edge.<x>   a per-link attribute -> e_<x> (loaded per link); a scalar one -> its literal value
  time       (the parameter annotated n2.time) -> t, the step's time
  locals     -> float l_<name>, declared at the top of the hook (Python locals are function-scoped)
  n2.spike(t) -> the neuron fires at time t (default: the hook's time); the first spike of a step counts
  math.<f>   -> the CUDA single-precision function; abs/min/max/float/int builtins; random.random() ->
             a Philox-based uniform draw keyed by (population, neuron, step, call site, link)
  return     -> leaves the hook (each hook body is wrapped in do { ... } while (0))
Supported statements: assignments (=, +=, -=, *=, /=, annotated), if/elif/else, pass, return, expression
calls of n2.spike. Loops and anything else raise NotImplementedError naming the construct.
"""

from __future__ import annotations

import ast
import math

_MATH = {"exp": "expf", "log": "logf", "sqrt": "sqrtf", "sin": "sinf", "cos": "cosf", "tan": "tanf",
         "tanh": "tanhf", "sinh": "sinhf", "cosh": "coshf", "atan": "atanf", "asin": "asinf", "acos": "acosf",
         "floor": "floorf", "ceil": "ceilf", "fabs": "fabsf", "log1p": "log1pf", "expm1": "expm1f",
         "log10": "log10f", "log2": "log2f", "pow": "powf", "atan2": "atan2f", "trunc": "truncf"}
_BIN = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*"}
_CMP = {ast.Lt: "<", ast.LtE: "<=", ast.Gt: ">", ast.GtE: ">=", ast.Eq: "==", ast.NotEq: "!="}
_CTYPE = {float: "float", int: "int", bool: "bool"}


def flit(v) -> str:
    """A float literal (single precision)."""
    v = float(v)
    if math.isnan(v):
        return "__int_as_float(0x7fc00000)"
    if math.isinf(v):
        return "__int_as_float(0x7f800000)" if v > 0 else "__int_as_float(0xff800000)"
    r = repr(v)
    if "e" not in r and "." not in r:
        r += ".0"
    return r + "f"


def literal(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, float)):
        return flit(v)
    raise NotImplementedError(f"a constant of type {type(v).__name__} cannot be lowered")


class Root:
    """An object a hook reads attributes of: `prefix` + name for its register copies of dynamic attributes
    (python type per name), literals for its static ones, and whether the hook may assign it."""

    def __init__(self, prefix: str, dynamic: dict, static: dict, writable: bool, what: str):
        self.prefix, self.dynamic, self.static, self.writable, self.what = prefix, dynamic, static, writable, what


class HookContext:
    """What a hook's names refer to. A node hook: self_attrs (dynamic attr -> python type) and self_static
    (static attr -> value) of its neuron; for receive, edge_dynamic (per-link edge attrs, hook-facing names)
    and edge_static (hook-facing name -> value). An edge hook (forward/backward) passes `roots` instead:
    self = the link's edge state, the destination = the neuron's state. `refused`: parameter names whose
    attributes may not be used (the sending neuron), `random`: whether random.random() may be called."""

    def __init__(self, self_attrs: dict | None = None, self_static: dict | None = None,
                 time_name: str | None = None, edge_name: str | None = None, source_name: str | None = None,
                 edge_dynamic: set | None = None, edge_static: dict | None = None, site_base: int = 0,
                 roots: dict | None = None, random: bool = True):
        self.self_attrs = self_attrs or {}
        self.time_name = time_name
        self.site = site_base  # random call sites numbered from here
        self.random = random
        self.roots = dict(roots) if roots is not None else {
            "self": Root("s_", self.self_attrs, dict(self_static or {}), True, "the neuron")}
        if edge_name is not None and roots is None:
            self.roots[edge_name] = Root("e_", {n: float for n in (edge_dynamic or ())}, dict(edge_static or {}),
                                         False, "the link")
        self.refused = {source_name} if source_name is not None else set()


class CudaLowering:
    def __init__(self, ctx: HookContext, where: str):
        self.ctx = ctx
        self.where = where  # for messages
        self.locals: list[str] = []

    # ------------------------------------------------------------------ entry

    def lower(self, fn: ast.FunctionDef) -> str:
        for node in ast.walk(fn):
            if isinstance(node, (ast.Assign, ast.AugAssign, ast.AnnAssign)):
                targets = node.targets if isinstance(node, ast.Assign) else [node.target]
                for t in targets:
                    if isinstance(t, ast.Name) and t.id not in self.locals:
                        self.locals.append(t.id)
        body = self.block(fn.body, 1)
        decl = "".join(f"    float l_{n} = 0.f;\n" for n in self.locals)
        return "do {\n" + decl + body + "} while (0);\n"

    def fail(self, node, what: str):
        raise NotImplementedError(f"{self.where}: {what} (line {getattr(node, 'lineno', '?')}) is not supported "
                                  f"by the CUDA transpiler")

    # ------------------------------------------------------------------ statements

    def block(self, stmts, depth: int) -> str:
        return "".join(self.stmt(s, depth) for s in stmts)

    def stmt(self, s, depth: int) -> str:
        pad = "    " * depth
        if isinstance(s, ast.Pass):
            return ""
        if isinstance(s, ast.Expr):
            if isinstance(s.value, ast.Constant) and isinstance(s.value.value, str):
                return ""  # a docstring
            if self.is_spike(s.value):
                when = self.expr(s.value.args[0]) if s.value.args else "t"
                return pad + f"if (!fired) {{ fired = true; spike_t = (float)({when}); }}\n"
            self.fail(s, "an expression statement other than n2.spike()")
        if isinstance(s, ast.Return):
            if s.value is not None:
                self.fail(s, "returning a value")
            return pad + "break;\n"
        if isinstance(s, (ast.Assign, ast.AnnAssign)):
            targets = s.targets if isinstance(s, ast.Assign) else [s.target]
            if s.value is None:
                return ""
            if len(targets) != 1:
                self.fail(s, "chained assignment")
            return pad + f"{self.target(targets[0])} = {self.cast_for(targets[0], self.expr(s.value))};\n"
        if isinstance(s, ast.AugAssign):
            op = s.op
            t = self.target(s.target)
            rhs = self.binop(op, t, self.expr(s.value), s)
            return pad + f"{t} = {self.cast_for(s.target, rhs)};\n"
        if isinstance(s, ast.If):
            out = pad + f"if ({self.expr(s.test)}) {{\n" + self.block(s.body, depth + 1) + pad + "}"
            if s.orelse:
                out += " else {\n" + self.block(s.orelse, depth + 1) + pad + "}"
            return out + "\n"
        self.fail(s, type(s).__name__)

    def target(self, t) -> str:
        if isinstance(t, ast.Name):
            return f"l_{t.id}"
        if isinstance(t, ast.Attribute) and isinstance(t.value, ast.Name):
            if t.value.id in self.ctx.refused:
                self.fail(t, f"{t.value.id}.<attr> (the sending neuron's state)")
            root = self.ctx.roots.get(t.value.id)
            if root is not None:
                if not root.writable:
                    self.fail(t, f"assigning {t.value.id}.{t.attr} ({root.what} is read-only here)")
                if t.attr not in root.dynamic:
                    self.fail(t, f"assigning {t.value.id}.{t.attr}, which is not a dynamic attribute")
                return f"{root.prefix}{t.attr}"
        self.fail(t, "this assignment target")

    def cast_for(self, t, expr: str) -> str:
        if isinstance(t, ast.Attribute):
            root = self.ctx.roots.get(t.value.id) if isinstance(t.value, ast.Name) else None
            ty = root.dynamic.get(t.attr, float) if root is not None else float
            if ty is bool:
                return f"(({expr}) != 0)"
            return f"({_CTYPE.get(ty, 'float')})({expr})"
        return f"(float)({expr})"

    def is_spike(self, e) -> bool:
        return (isinstance(e, ast.Call) and isinstance(e.func, ast.Attribute) and e.func.attr == "spike"
                and isinstance(e.func.value, ast.Name)) or (isinstance(e, ast.Call) and isinstance(e.func, ast.Name)
                                                          and e.func.id == "spike")

    # ------------------------------------------------------------------ expressions

    def binop(self, op, a: str, b: str, node) -> str:
        if type(op) in _BIN:
            return f"({a} {_BIN[type(op)]} {b})"
        if isinstance(op, ast.Div):
            return f"((float)({a}) / (float)({b}))"
        if isinstance(op, ast.FloorDiv):
            return f"floorf((float)({a}) / (float)({b}))"
        if isinstance(op, ast.Mod):
            return f"n2_pymod((float)({a}), (float)({b}))"
        if isinstance(op, ast.Pow):
            return f"powf((float)({a}), (float)({b}))"
        self.fail(node, f"the operator {type(op).__name__}")

    def expr(self, e) -> str:
        c = self.ctx
        if isinstance(e, ast.Constant):
            return literal(e.value)
        if isinstance(e, ast.Name):
            if e.id == c.time_name:
                return "t"
            if e.id in self.locals:
                return f"l_{e.id}"
            if e.id in ("True", "False"):
                return "true" if e.id == "True" else "false"
            self.fail(e, f"the name '{e.id}'")
        if isinstance(e, ast.Attribute):
            if isinstance(e.value, ast.Name):
                base = e.value.id
                root = c.roots.get(base)
                if root is not None:
                    if e.attr in root.dynamic:
                        return f"{root.prefix}{e.attr}"
                    if e.attr in root.static:
                        return literal(root.static[e.attr])
                    self.fail(e, f"{base}.{e.attr} ({root.what} has no such attribute)")
                if base in c.refused:
                    self.fail(e, f"{base}.<attr> (reading the sending neuron's state)")
                if base == "math" and e.attr in ("pi", "e", "inf", "tau"):
                    return flit(getattr(math, e.attr))
            self.fail(e, "this attribute")
        if isinstance(e, ast.BinOp):
            if isinstance(e.op, ast.Pow) and isinstance(e.right, ast.Constant) and e.right.value == 2:
                a = self.expr(e.left)
                return f"((float)({a}) * (float)({a}))"
            return self.binop(e.op, self.expr(e.left), self.expr(e.right), e)
        if isinstance(e, ast.UnaryOp):
            v = self.expr(e.operand)
            if isinstance(e.op, ast.USub):
                return f"(-({v}))"
            if isinstance(e.op, ast.UAdd):
                return f"(+({v}))"
            if isinstance(e.op, ast.Not):
                return f"(!({v}))"
            self.fail(e, f"the operator {type(e.op).__name__}")
        if isinstance(e, ast.BoolOp):
            op = " && " if isinstance(e.op, ast.And) else " || "
            return "(" + op.join(f"({self.expr(v)})" for v in e.values) + ")"
        if isinstance(e, ast.Compare):
            parts, left = [], self.expr(e.left)
            for op, right in zip(e.ops, e.comparators):
                if type(op) not in _CMP:
                    self.fail(e, f"the comparison {type(op).__name__}")
                r = self.expr(right)
                parts.append(f"({left} {_CMP[type(op)]} {r})")
                left = r
            return "(" + " && ".join(parts) + ")"
        if isinstance(e, ast.IfExp):
            return f"(({self.expr(e.test)}) ? ({self.expr(e.body)}) : ({self.expr(e.orelse)}))"
        if isinstance(e, ast.Call):
            return self.call(e)
        self.fail(e, type(e).__name__)

    def call(self, e: ast.Call) -> str:
        if e.keywords:
            self.fail(e, "keyword arguments")
        args = [self.expr(a) for a in e.args]
        f = e.func
        if isinstance(f, ast.Attribute) and isinstance(f.value, ast.Name):
            mod, name = f.value.id, f.attr
            if mod == "math" and name in _MATH:
                return f"{_MATH[name]}(" + ", ".join(f"(float)({a})" for a in args) + ")"
            if mod == "random" and name == "random" and not args:
                if not self.ctx.random:
                    self.fail(e, "random.random() in an edge hook")
                site = self.ctx.site
                self.ctx.site += 1
                return f"n2_uniform(p, j, n, {site}u, link_k)"
        if isinstance(f, ast.Name):
            if f.id == "abs" and len(args) == 1:
                return f"fabsf((float)({args[0]}))"
            if f.id in ("min", "max") and len(args) == 2:
                return f"{'fminf' if f.id == 'min' else 'fmaxf'}((float)({args[0]}), (float)({args[1]}))"
            if f.id == "float" and len(args) == 1:
                return f"(float)({args[0]})"
            if f.id == "int" and len(args) == 1:
                return f"truncf((float)({args[0]}))"
        self.fail(e, f"the call {ast.unparse(e.func)}()")


def lower_hook(fn: ast.FunctionDef, ctx: HookContext, where: str) -> str:
    """The hook body as a CUDA block: do { ... } while (0);"""
    return CudaLowering(ctx, where).lower(fn)
