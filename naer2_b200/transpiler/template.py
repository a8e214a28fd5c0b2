"""The step-kernel template of a transpiled population (reference naer2/transpiler/templates/fused_template.py:
85-371, the Gluon kernel it fills: pull -> deliver -> update/send -> emit).

One launch per population per step n (time t = (n + 1) dt, the end of the step); clocked intake: 32 neurons
per block, scan(n) threads per neuron (the neuron's first thread runs its hooks); exact-time intake: one thread
per neuron.
  1. intake and receive: for each incoming connection (in the network's order), the neuron's pull row (its
     incoming links, canonical order within the row); a link whose source spiked at step n - d (the source
     population's spike-bit ring) runs the connection's receive hook once, with its per-link edge values
     (clocked: the SCAN threads list the arrivals of their row segments first, the hooks then run over the
     lists in link order);
  2. update, then send (n2.spike() anywhere marks the neuron as firing at step n);
  3. the spike-bit word of 32 neurons (clocked: one per block; exact-time: a ballot per warp) into the
     population's spike-bit ring slot n mod depth (and the raster), the state back to memory, and the spike /
     arrival counters.
The source is self-contained (NVRTC compiles it with no includes); its one parameter is the `Params` block,
mirrored field by field by the ctypes structure `params_type` builds, so that the host fills it directly.
"""

from __future__ import annotations

import ctypes

from .cuda import HookContext, lower_hook

_PRELUDE = r'''
typedef unsigned int u32;
typedef unsigned long long u64;

// Philox4x32-10 (Salmon et al., SC 2011): the first output word of counter (c0..c3) under key (k0, k1).
__device__ __forceinline__ u32 n2_philox_w0(u32 c0, u32 c1, u32 c2, u32 c3, u32 k0, u32 k1) {
    #pragma unroll
    for (int r = 0; r < 10; ++r) {
        const u32 h0 = __umulhi(0xD2511F53u, c0), l0 = 0xD2511F53u * c0;
        const u32 h1 = __umulhi(0xCD9E8D57u, c2), l1 = 0xCD9E8D57u * c2;
        const u32 n0 = h1 ^ c1 ^ k0, n2 = h0 ^ c3 ^ k1;
        c0 = n0; c1 = l1; c2 = n2; c3 = l0;
        k0 += 0x9E3779B9u; k1 += 0xBB67AE85u;
    }
    return c0;
}

// Python's % on floats: the result takes the sign of the divisor.
__device__ __forceinline__ float n2_pymod(float a, float b) {
    float r = fmodf(a, b);
    if (r != 0.f && ((r < 0.f) != (b < 0.f))) r += b;
    return r;
}
'''


def ctype_of(py) -> tuple[str, object, object]:
    """(C type, ctypes type, torch dtype) of a dynamic attribute's Python type."""
    import torch

    if py is bool:
        return "bool", ctypes.c_bool, torch.bool
    if py is int:
        return "int", ctypes.c_int32, torch.int32
    return "float", ctypes.c_float, torch.float32


MAX_ARRIVALS = 64  # exact-time intake: arrivals a neuron can hold in one step (more are counted, dropped)


def _arrival_body(pop_name: str, c: int, inc: dict) -> str:
    """One arrival of connection c: the link's edge values, edge forward, receive, edge values stored."""
    body = ""
    if inc.get("forward") is not None:
        fn, ctx = inc["forward"]
        body += lower_hook(fn, ctx, f"{pop_name} edge forward (connection {c})")
    body += "".join(f"const float e_{h} = e_{real};\n" for h, real in inc.get("alias", {}).items())
    if inc["receive"] is not None:
        fn, ctx = inc["receive"]
        body += lower_hook(fn, ctx, f"{pop_name} receive (connection {c})")
    body += "".join(f"p.c{c}_e_{e}[l] = e_{e};\n" for e in inc.get("edge_written", ()))
    return body


NPB_C = 32  # clocked intake: neurons per block (one spike-bit word), scan(n) * NPB_C threads
LIST_WORDS = 4096  # clocked intake: the block's arrival lists (u32), SCAN * CAP per neuron


def scan(n: int) -> int:
    """Clocked intake: threads scanning one neuron's incoming row, for a population of n neurons (more for small
    populations, so that their blocks still fill the GPU)."""
    return 32 if n <= 4096 else 8


def _clocked_kernel(pop_name: str, attrs: dict, hooks: dict, incoming: list, n: int) -> str:
    """The clocked step kernel: SCAN threads per neuron split each incoming row into SCAN contiguous segments
    and list the arrivals of their segment in shared memory (link words and spike bits of many links in
    flight); the neuron's first thread (the owner) then runs the hooks over the lists in segment order, i.e.
    in link order, with the same arrival numbers and draws as one link at a time. A segment with more than CAP
    arrivals is walked again by the owner, link by link. SCAN = scan(n), CAP = LIST_WORDS / (NPB_C * SCAN)."""
    SCAN = scan(n)
    CAP = LIST_WORDS // (NPB_C * SCAN)
    src = [f"constexpr int SCAN = {SCAN}, NPB_C = {NPB_C}, CAP = {CAP};\n\n"]
    src.append(f'// population {pop_name}\nextern "C" __global__ void __launch_bounds__({SCAN * NPB_C}) '
               "n2b_user_step(const __grid_constant__ Params p) {\n")
    src.append("""    __shared__ u32 s_list[NPB_C * SCAN * CAP];
    __shared__ int s_cnt[NPB_C * SCAN];
    __shared__ u32 s_word, s_arrivals;
    const int jl = threadIdx.x / SCAN, sc = threadIdx.x % SCAN;
    const int j = blockIdx.x * NPB_C + jl;
    const bool live = j < p.n, own = sc == 0;
    const long long n = p.step;
    const float t = p.t;
    bool fired = false;
    float spike_t = t;
    u32 arrived = 0;
    u32 link_k = 0xFFFFFFu;
    if (threadIdx.x == 0) { s_word = 0u; s_arrivals = 0u; }
""")
    for a, py in attrs.items():
        ct, _, _ = ctype_of(py)
        src.append(f"    {ct} s_{a} = (live && own) ? p.s_{a}[j] : ({ct})0;\n")
    src.append("    __syncthreads();\n")
    for c, inc in enumerate(incoming):
        if inc["receive"] is None and inc.get("forward") is None:
            continue
        body = ""
        if inc.get("forward") is not None:
            fn, ctx = inc["forward"]
            body += lower_hook(fn, ctx, f"{pop_name} edge forward (connection {c})")
        body += "".join(f"const float e_{h} = e_{real};\n" for h, real in inc.get("alias", {}).items())
        if inc["receive"] is not None:
            fn, ctx = inc["receive"]
            body += lower_hook(fn, ctx, f"{pop_name} receive (connection {c})")
        body += "".join(f"p.c{c}_e_{e}[l] = e_{e};\n" for e in inc.get("edge_written", ()))
        body = "{\n" + body + "}\n"
        loads = "".join(f"float e_{e} = p.c{c}_e_{e}[l];\n" for e in inc["edge_dynamic"])
        arrival = loads + "link_k = arrived++;\n" + body
        hit = (f"(p.c{c}_src_bits[(size_t)(m & p.c{c}_src_mask) * p.c{c}_src_words + (src >> 5)] >> (src & 31)) & 1u")
        src.append(f"""    {{  // connection {c}: scan
        const int r0 = live ? p.c{c}_ptr[j] : 0, r1 = live ? p.c{c}_ptr[j + 1] : 0;
        const int seg = (r1 - r0 + SCAN - 1) / SCAN;
        const int a = min(r1, r0 + sc * seg), b = min(r1, a + seg);
        int cnt = 0;
        for (int l = a; l < b; ++l) {{
            const u32 w = p.c{c}_link[l];
            const int src = (int)(w & 0xFFFFFFu), d = (int)(w >> 24);
            if (d < 1 || d > p.c{c}_src_mask) {{ atomicAdd(p.err, 1); continue; }}
            const long long m = n - d;
            if (m < 0 || !({hit})) continue;
            if (cnt < CAP) s_list[(jl * SCAN + sc) * CAP + cnt] = (u32)l;
            ++cnt;
        }}
        s_cnt[jl * SCAN + sc] = cnt;
        __syncthreads();
        if (live && own) {{  // the hooks, in link order
            for (int s = 0; s < SCAN; ++s) {{
                const int cs = s_cnt[jl * SCAN + s];
                if (cs <= CAP) {{
                    for (int i = 0; i < cs; ++i) {{
                        const int l = (int)s_list[(jl * SCAN + s) * CAP + i];
""")
        src.append("                        " + arrival.replace("\n", "\n                        ").rstrip() + "\n")
        src.append(f"""                    }}
                }} else {{  // the segment again, one link at a time
                    const int as = min(r1, r0 + s * seg), bs = min(r1, as + seg);
                    for (int l = as; l < bs; ++l) {{
                        const u32 w = p.c{c}_link[l];
                        const int src = (int)(w & 0xFFFFFFu), d = (int)(w >> 24);
                        if (d < 1 || d > p.c{c}_src_mask) continue;
                        const long long m = n - d;
                        if (m < 0 || !({hit})) continue;
""")
        src.append("                        " + arrival.replace("\n", "\n                        ").rstrip() + "\n")
        src.append("""                    }
                }
            }
        }
        link_k = 0xFFFFFFu;
        __syncthreads();  // the lists are rewritten by the next connection
    }
""")
    src.append("    if (live && own) {\n")
    for name in ("update", "send"):
        fn, ctx = hooks[name]
        body = lower_hook(fn, ctx, f"{pop_name} {name}")
        src.append("        " + body.replace("\n", "\n        ").rstrip() + "\n")
    backward = [(c, inc) for c, inc in enumerate(incoming) if inc.get("backward") is not None]
    if backward:  # the neuron fired: every incoming link's edge backward hook at its spike's time
        src.append("        if (fired) {\n            const float t = spike_t;\n")
        for c, inc in backward:
            fn, ctx = inc["backward"]
            body = lower_hook(fn, ctx, f"{pop_name} edge backward (connection {c})")
            body += "".join(f"p.c{c}_e_{e}[l] = e_{e};\n" for e in inc.get("edge_written", ()))
            loads = "".join(f"                float e_{e} = p.c{c}_e_{e}[l];\n" for e in inc["edge_dynamic"])
            src.append(f"            for (int l = p.c{c}_ptr[j]; l < p.c{c}_ptr[j + 1]; ++l) {{\n{loads}")
            src.append("                " + body.replace("\n", "\n                ").rstrip() + "\n")
            src.append("            }\n")
        src.append("        }\n")
    src.append("""        if (fired) {
            const float o = spike_t - p.t0;  // the spike's time within its step
            p.off[(size_t)(n & p.bit_mask) * p.n + j] = o;
            const long long r = n - p.rec0;
            if (p.raster_off && r >= 0 && r < p.raster_steps) p.raster_off[(size_t)r * p.n + j] = o;
            atomicOr(&s_word, 1u << jl);
        }
        if (arrived) atomicAdd(&s_arrivals, arrived);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // the block's 32 neurons: one spike-bit word
        const u32 b = s_word;
        const int word = blockIdx.x;
        if (word < p.words) {
            p.bits[(size_t)(n & p.bit_mask) * p.words + word] = b;
            const long long r = n - p.rec0;
            if (p.raster && r >= 0 && r < p.raster_steps) p.raster[(size_t)r * p.words + word] = b;
        }
        if (b) atomicAdd(p.counters + 1, (u64)__popc(b));
        if (s_arrivals) atomicAdd(p.counters, (u64)s_arrivals);
    }
""")
    for a in attrs:
        src.append(f"    if (live && own) p.s_{a}[j] = s_{a};\n")
    src.append("}\n")
    return "".join(src)


def build_source(pop_name: str, attrs: dict, hooks: dict, incoming: list, exact: bool = False,
                 n: int = 1 << 30) -> tuple[str, list]:
    """(CUDA source, params fields [(name, C type, ctypes type)]) of one population.

    attrs: dynamic attr -> python type; hooks: {"update": (fn_ast, ctx), "send": (fn_ast, ctx)};
    incoming: one dict per incoming connection: "receive": (fn_ast, ctx) or None; "edge_dynamic": the per-link
    arrays by the edge's own attribute names; "edge_written": those the edge hooks assign (stored back);
    "alias": {receive-facing name: edge name} where they differ; "forward" / "backward": (fn_ast, ctx) of the
    edge hooks or None.

    n: the population's size (the clocked intake's threads per neuron, `scan(n)`).

    exact: event-driven intake at exact times. Every spike carries its time (its offset in its step, in the
    population's offset ring); a link of delay d delivers it at that time plus d steps. A neuron collects its
    arrivals of the step, sorts them by time (stable: connection order, then link order, among equal times),
    runs receive (and edge forward) for each at its own time and send after each group of equal times; then
    update and send at the end of the step, as in the clocked intake."""
    fields = [("step", "long long", ctypes.c_int64), ("rec0", "long long", ctypes.c_int64),
              ("raster_steps", "long long", ctypes.c_int64), ("t", "float", ctypes.c_float),
              ("t0", "float", ctypes.c_float),
              ("n", "int", ctypes.c_int32), ("words", "int", ctypes.c_int32), ("bit_mask", "int", ctypes.c_int32),
              ("seed_lo", "u32", ctypes.c_uint32), ("seed_hi", "u32", ctypes.c_uint32)]
    for a, py in attrs.items():
        ct, cty, _ = ctype_of(py)
        fields.append((f"s_{a}", f"{ct} *", ctypes.c_void_p))
    fields += [("bits", "u32 *", ctypes.c_void_p), ("off", "float *", ctypes.c_void_p),
               ("raster", "u32 *", ctypes.c_void_p), ("raster_off", "float *", ctypes.c_void_p),
               ("err", "int *", ctypes.c_void_p),
               ("counters", "u64 *", ctypes.c_void_p)]
    for c, inc in enumerate(incoming):
        fields += [(f"c{c}_ptr", "const int *", ctypes.c_void_p), (f"c{c}_link", "const u32 *", ctypes.c_void_p),
                   (f"c{c}_src_bits", "const u32 *", ctypes.c_void_p), (f"c{c}_src_off", "const float *", ctypes.c_void_p),
                   (f"c{c}_src_words", "int", ctypes.c_int32), (f"c{c}_src_mask", "int", ctypes.c_int32),
                   (f"c{c}_src_n", "int", ctypes.c_int32)]
        for e in inc["edge_dynamic"]:
            fields.append((f"c{c}_e_{e}", "float *" if e in inc.get("edge_written", ()) else "const float *",
                           ctypes.c_void_p))

    src = [_PRELUDE, "struct Params {\n"]
    src += [f"    {ct} {name};\n" for name, ct, _ in fields]
    src.append("};\n\n")
    src.append(r'''// uniform in [0, 1): 24 bits of the draw for (neuron j, step n, call site, link k)
__device__ __forceinline__ float n2_uniform(const Params &p, int j, long long n, u32 site, u32 k) {
    const u32 w = n2_philox_w0((u32)j, (u32)n, (u32)((u64)n >> 32), (site << 24) | (k & 0xFFFFFFu), p.seed_lo,
                               p.seed_hi);
    return (float)(w >> 8) * 5.9604644775390625e-08f;
}

''')
    if not exact:
        src.append(_clocked_kernel(pop_name, attrs, hooks, incoming, n))
        return "".join(src), fields
    src.append(f'// population {pop_name}\nextern "C" __global__ void __launch_bounds__(128) n2b_user_step('
               "const __grid_constant__ Params p) {\n")
    src.append("    const int j = blockIdx.x * blockDim.x + threadIdx.x;\n")
    src.append("    const bool live = j < p.n;\n    const long long n = p.step;\n    const float t = p.t;\n")
    src.append("    bool fired = false;\n    float spike_t = t;\n    u32 arrived = 0;\n    u32 link_k = 0xFFFFFFu;\n")
    for a, py in attrs.items():
        ct, _, _ = ctype_of(py)
        src.append(f"    {ct} s_{a} = live ? p.s_{a}[j] : ({ct})0;\n")
    src.append("    if (live) {\n")
    if exact:
        src.append(_exact_intake(pop_name, incoming, hooks))
    for c, inc in enumerate(incoming):
        if exact:
            break
        if inc["receive"] is None and inc.get("forward") is None:
            continue
        body = ""
        if inc.get("forward") is not None:
            fn, ctx = inc["forward"]
            body += lower_hook(fn, ctx, f"{pop_name} edge forward (connection {c})")
        body += "".join(f"const float e_{h} = e_{real};\n" for h, real in inc.get("alias", {}).items())
        if inc["receive"] is not None:
            fn, ctx = inc["receive"]
            body += lower_hook(fn, ctx, f"{pop_name} receive (connection {c})")
        body += "".join(f"p.c{c}_e_{e}[l] = e_{e};\n" for e in inc.get("edge_written", ()))
        if inc.get("alias"):
            body = "{\n" + body + "}\n"
        loads = "".join(f"            float e_{e} = p.c{c}_e_{e}[l];\n" for e in inc["edge_dynamic"])
        src.append(f"""        for (int l = p.c{c}_ptr[j]; l < p.c{c}_ptr[j + 1]; ++l) {{
            const u32 w = p.c{c}_link[l];
            const int src = (int)(w & 0xFFFFFFu), d = (int)(w >> 24);
            if (d < 1 || d > p.c{c}_src_mask) {{ atomicAdd(p.err, 1); continue; }}
            const long long m = n - d;
            if (m < 0) continue;
            if (!((p.c{c}_src_bits[(size_t)(m & p.c{c}_src_mask) * p.c{c}_src_words + (src >> 5)] >> (src & 31)) & 1u))
                continue;
{loads}            link_k = arrived++;
""")
        src.append("            " + body.replace("\n", "\n            ").rstrip() + "\n")
        src.append("        }\n        link_k = 0xFFFFFFu;\n")
    for name in ("update", "send"):
        fn, ctx = hooks[name]
        body = lower_hook(fn, ctx, f"{pop_name} {name}")
        src.append("        " + body.replace("\n", "\n        ").rstrip() + "\n")
    backward = [(c, inc) for c, inc in enumerate(incoming) if inc.get("backward") is not None]
    if backward:  # the neuron fired: every incoming link's edge backward hook at its spike's time
        src.append("        if (fired) {\n            const float t = spike_t;\n")
        for c, inc in backward:
            fn, ctx = inc["backward"]
            body = lower_hook(fn, ctx, f"{pop_name} edge backward (connection {c})")
            body += "".join(f"p.c{c}_e_{e}[l] = e_{e};\n" for e in inc.get("edge_written", ()))
            loads = "".join(f"                float e_{e} = p.c{c}_e_{e}[l];\n" for e in inc["edge_dynamic"])
            src.append(f"            for (int l = p.c{c}_ptr[j]; l < p.c{c}_ptr[j + 1]; ++l) {{\n{loads}")
            src.append("                " + body.replace("\n", "\n                ").rstrip() + "\n")
            src.append("            }\n")
        src.append("        }\n")
    src.append("    }\n")
    src.append("""    if (live && fired) {
        const float o = spike_t - p.t0;  // the spike's time within its step
        p.off[(size_t)(n & p.bit_mask) * p.n + j] = o;
        const long long r = n - p.rec0;
        if (p.raster_off && r >= 0 && r < p.raster_steps) p.raster_off[(size_t)r * p.n + j] = o;
    }
""")
    src.append(r'''    const u32 b = __ballot_sync(0xffffffffu, live && fired);
    const u32 arrivals = __reduce_add_sync(0xffffffffu, arrived);
    if ((threadIdx.x & 31) == 0) {
        const int word = j >> 5;
        if (word < p.words) {
            p.bits[(size_t)(n & p.bit_mask) * p.words + word] = b;
            const long long r = n - p.rec0;
            if (p.raster && r >= 0 && r < p.raster_steps) p.raster[(size_t)r * p.words + word] = b;
        }
        if (b) atomicAdd(p.counters + 1, (u64)__popc(b));
        if (arrivals) atomicAdd(p.counters, (u64)arrivals);
    }
''')
    for a in attrs:
        src.append(f"    if (live) p.s_{a}[j] = s_{a};\n")
    src.append("}\n")
    return "".join(src), fields


def _exact_intake(pop_name: str, incoming: list, hooks: dict) -> str:
    """The event-driven intake: collect the step's arrivals with their times, sort, deliver in time order."""
    out = [f"""        float a_t[{MAX_ARRIVALS}];
        int a_c[{MAX_ARRIVALS}], a_l[{MAX_ARRIVALS}];
        int na = 0;
"""]
    for c, inc in enumerate(incoming):
        if inc["receive"] is None and inc.get("forward") is None:
            continue
        out.append(f"""        for (int l = p.c{c}_ptr[j]; l < p.c{c}_ptr[j + 1]; ++l) {{
            const u32 w = p.c{c}_link[l];
            const int src = (int)(w & 0xFFFFFFu), d = (int)(w >> 24);
            if (d < 1 || d > p.c{c}_src_mask) {{ atomicAdd(p.err, 1); continue; }}
            const long long m = n - d;
            if (m < 0) continue;
            const size_t slot = (size_t)(m & p.c{c}_src_mask);
            if (!((p.c{c}_src_bits[slot * p.c{c}_src_words + (src >> 5)] >> (src & 31)) & 1u)) continue;
            const float tau = p.t0 + p.c{c}_src_off[slot * p.c{c}_src_n + src];
            if (na == {MAX_ARRIVALS}) {{ atomicAdd(p.err, 1); continue; }}
            int k = na++;
            while (k > 0 && a_t[k - 1] > tau) {{ a_t[k] = a_t[k - 1]; a_c[k] = a_c[k - 1]; a_l[k] = a_l[k - 1]; --k; }}
            a_t[k] = tau; a_c[k] = {c}; a_l[k] = l;
        }}
""")
    out.append("""        for (int i = 0; i < na;) {
            const float tau = a_t[i];
            int e = i;
            while (e < na && a_t[e] == tau) ++e;
            for (int k = i; k < e; ++k) {
                const int l = a_l[k];
                const float t = tau;
                link_k = arrived++;
                switch (a_c[k]) {
""")
    for c, inc in enumerate(incoming):
        if inc["receive"] is None and inc.get("forward") is None:
            continue
        loads = "".join(f"float e_{x} = p.c{c}_e_{x}[l];\n" for x in inc["edge_dynamic"])
        body = loads + _arrival_body(pop_name, c, inc)
        out.append(f"                case {c}: {{\n                    " +
                   body.replace("\n", "\n                    ").rstrip() + "\n                } break;\n")
    fn, ctx = hooks["send"]
    send = lower_hook(fn, ctx, f"{pop_name} send")
    out.append("""                default: break;
                }
            }
            {
                const float t = tau;
                """ + send.replace("\n", "\n                ").rstrip() + """
            }
            i = e;
        }
        link_k = 0xFFFFFFu;
""")
    return "".join(out)


def params_type(fields: list):
    """The ctypes structure of a Params block."""
    return type("Params", (ctypes.Structure,), {"_fields_": [(name, cty) for name, _, cty in fields]})


def edge_hook_context(pop, hook, per_link: list, edge_static: dict) -> HookContext:
    """An edge hook's names: self = the link (per-link arrays, the edge's static values), the destination =
    the target neuron's state; the source's state and random draws are refused."""
    from .. import receives
    from .cuda import Root

    names = {ty: nm for ty, nm in hook.parameter_type_to_name.items()}
    static = {k: v for k, v in pop.instance.__dict__.items()
              if k not in pop.dynamic_attrs and isinstance(v, (int, float, bool))}
    roots = {"self": Root("e_", {n: float for n in per_link}, dict(edge_static), True, "the link")}
    if receives.destination in names:
        roots[names[receives.destination]] = Root("s_", dict(pop.dynamic_attrs), static, True,
                                                  "the destination neuron")
    return HookContext(time_name=names.get(receives.time), source_name=names.get(receives.source), roots=roots,
                       random=False)


def hook_context(pop, hook, edge_dynamic=(), edge_static=None, site_base: int = 0) -> HookContext:
    """The names a hook's body may use, from its signature and the population's attributes."""
    from .. import receives

    names = {ty: nm for ty, nm in hook.parameter_type_to_name.items()}
    static = {k: v for k, v in pop.instance.__dict__.items()
              if k not in pop.dynamic_attrs and isinstance(v, (int, float, bool))}
    return HookContext(self_attrs=dict(pop.dynamic_attrs), self_static=static,
                       time_name=names.get(receives.time), edge_name=names.get(receives.edge),
                       source_name=names.get(receives.source), edge_dynamic=set(edge_dynamic),
                       edge_static=dict(edge_static or {}), site_base=site_base)
