"""The transpiler: a population's Python hooks lowered to CUDA device code in a step-kernel template,
compiled at run time with NVRTC (naer2_b200/csrc/jit.cu) -- the path of models without a built-in kernel."""

from .cuda import HookContext, lower_hook
from .runtime import JitRuntime, PlannedNetwork, load_plan, plan_of, save_plan
from .template import build_source

__all__ = ["HookContext", "lower_hook", "build_source", "JitRuntime", "PlannedNetwork", "plan_of", "save_plan",
           "load_plan"]
