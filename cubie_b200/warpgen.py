"""Code generation for the warp-per-system path (large systems).

For a system with many states, one warp integrates one run: lane ``l``
holds components ``l, l + 32, l + 64, ...`` of every state-sized vector, and
the right-hand side and the Jacobian-vector product are evaluated by all 32
lanes together from a copy of the state in shared memory.

A straight-line, component-by-component translation would make every lane
execute different code.  Instead the expressions are grouped into
*classes*: two components belong to the same class when their expressions
are the same up to which states, parameters and drivers they read (the
interior compartments of a cable, every gate of the same kind, ...).  A
class is emitted once as a function of its slot values; lane ``l`` then
evaluates members ``l, l + 32, ...`` of the class, gathering each member's
slots from shared memory through index tables (or through an affine formula
``index = a * member + b`` when the indices follow one, which is the common
case and needs no table).  All lanes run the same instructions; only the
member count of a class decides how many lanes are busy.

The Jacobian-vector product ``(J v)_i = sum_k df_i/dy_k v_k`` is generated
the same way, with the components of ``v`` as a fourth kind of slot.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import sympy as sp

from .codegen import FlopCount, _CudaPrinter, count_ops
from .symbolic import TIME, SymbolicODE

KINDS = ("y", "v", "p", "d")


@dataclass
class ExprClass:
    """One group of isomorphic component expressions."""

    template: sp.Expr                    # expression in slot placeholders
    slots: List[Tuple[str, int]]         # (kind, slot number) in placeholder order
    members: List[int] = field(default_factory=list)          # output component of each member
    indices: List[List[int]] = field(default_factory=list)    # per member, the index of each slot


def _placeholder(kind: str, k: int) -> sp.Symbol:
    return sp.Symbol(f"_{kind}{k}", real=True)


def _canonical(expr: sp.Expr, kind_of: Dict[sp.Symbol, Tuple[str, int]]) -> Tuple[sp.Expr, List[Tuple[str, int]]]:
    """Replace the states, v components, parameters and drivers in ``expr``
    by placeholders numbered per kind in order of first appearance (a
    preorder walk; repeated twice so the ordering no longer depends on the
    original names).  Returns the template and, per placeholder, the
    original (kind, index)."""
    cur = expr
    binding: Dict[sp.Symbol, Tuple[str, int]] = {}
    for _ in range(2):
        order: List[sp.Symbol] = []
        for node in sp.preorder_traversal(cur):
            if isinstance(node, sp.Symbol) and node not in order and (node in kind_of or node in binding):
                order.append(node)
        counters = {k: 0 for k in KINDS}
        new_binding = {}
        rename = {}
        for s in order:
            kind, idx = binding[s] if s in binding else kind_of[s]
            ph = _placeholder(kind, counters[kind])
            counters[kind] += 1
            rename[s] = ph
            new_binding[ph] = (kind, idx)
        cur = cur.xreplace(rename)
        binding = new_binding
    slots = [binding[ph] for ph in sorted(binding, key=lambda s: (KINDS.index(s.name[1]), int(s.name[2:])))]
    return cur, slots


def group_classes(exprs: Sequence[sp.Expr], kind_of: Dict[sp.Symbol, Tuple[str, int]]) -> List[ExprClass]:
    classes: Dict[str, ExprClass] = {}
    order: List[str] = []
    for i, e in enumerate(exprs):
        tmpl, slots = _canonical(sp.sympify(e), kind_of)
        key = sp.srepr(tmpl)
        if key not in classes:
            ph = sorted(tmpl.free_symbols & {_placeholder(k, j) for k in KINDS for j in range(len(slots) + 1)},
                        key=lambda s: (KINDS.index(s.name[1]), int(s.name[2:])))
            classes[key] = ExprClass(template=tmpl, slots=[(s.name[1], int(s.name[2:])) for s in ph])
            order.append(key)
        c = classes[key]
        c.members.append(i)
        c.indices.append([idx for (_, idx) in slots])
    return [classes[k] for k in order]


def _times(fc: FlopCount, k: int) -> FlopCount:
    """The operation count of ``k`` evaluations of one class body."""
    return FlopCount(fc.add * k, fc.mul * k, fc.div * k, fc.special * k)


def _affine(values: List[int]):
    """(a, b) with values[m] == a * m + b for every m, or None."""
    if len(values) == 1:
        return 0, values[0]
    a = values[1] - values[0]
    b = values[0]
    if all(v == a * m + b for m, v in enumerate(values)):
        return a, b
    return None


@dataclass
class WarpSystemCode:
    source: str
    n_classes_f: int
    n_classes_jv: int
    flops: Dict[str, FlopCount]
    nnz: int = 0                 # cached Jacobian coefficients per run (0: J v stays matrix-free)
    n_classes_fj: int = 0


# Largest cached Jacobian (coefficients per run) the generator emits: one
# warp keeps them in shared memory, 4 bytes each in FP32.
CACHED_JAC_MAX = 2048


def _emit_classes(name: str, classes: List[ExprClass], with_v: bool, tables: List[str]) -> Tuple[str, FlopCount]:
    """A device function evaluating every class for the calling lane."""
    lines = []
    fc = FlopCount()
    sig = (f"    template <class R> static __device__ CBX_NOINLINE void {name}(const R* __restrict__ ys, "
           + ("const R* __restrict__ vs, " if with_v else "")
           + "const R* __restrict__ ps, const R* __restrict__ ds, R t, R* __restrict__ out, int lane)")
    lines.append(sig)
    lines.append("    {")
    lines.append("        (void)ys; (void)ps; (void)ds; (void)t;" + (" (void)vs;" if with_v else ""))
    for ci, c in enumerate(classes):
        nm = len(c.members)
        slot_syms = [_placeholder(k, j) for (k, j) in c.slots]
        sym_map = {TIME: "t"}
        for s in slot_syms:
            sym_map[s] = f"s_{s.name[1:]}"
        lines.append(f"        // class {ci}: {nm} member(s)")
        # kept as a loop: unrolled over a lane's members the class code
        # grew the kernel until instruction fetch bounded it
        lines.append("        #pragma unroll 1")
        lines.append(f"        for (int m = lane; m < {nm}; m += 32) {{")
        # output index
        aff = _affine(c.members)
        if aff is not None:
            lines.append(f"            const int o = {aff[0]} * m + {aff[1]};")
        else:
            tname = f"{name}_c{ci}_out"
            tables.append(f"    static __device__ const unsigned short {tname}[{nm}] = "
                          f"{{{', '.join(str(v) for v in c.members)}}};")
            lines.append(f"            const int o = {tname}[m];")
        for q, (kind, j) in enumerate(c.slots):
            col = [row[q] for row in c.indices]
            src = {"y": "ys", "v": "vs", "p": "ps", "d": "ds"}[kind]
            aff = _affine(col)
            if aff is not None:
                idx = f"{aff[0]} * m + {aff[1]}" if aff[0] != 0 else f"{aff[1]}"
            else:
                tname = f"{name}_c{ci}_s{q}"
                tables.append(f"    static __device__ const unsigned short {tname}[{nm}] = "
                              f"{{{', '.join(str(v) for v in col)}}};")
                idx = f"{tname}[m]"
            lines.append(f"            const R s_{kind}{j} = {src}[{idx}];")
        printer = _CudaPrinter(sym_map)
        reps, reduced = sp.cse([c.template], symbols=sp.numbered_symbols("_t"), optimizations="basic")
        for s, e in reps:
            lines.append(f"            const R {s} = {printer.doprint(e)};")
            fc = fc + _times(count_ops(e), nm)
        lines.append(f"            out[o] = {printer.doprint(reduced[0])};")
        fc = fc + _times(count_ops(reduced[0]), nm)
        lines.append("        }")
    lines.append("    }")
    return "\n".join(lines), fc


def _index_expr(name: str, ci: int, q: int, values: List[int], tables: List[str]) -> str:
    aff = _affine(values)
    if aff is not None:
        return f"{aff[0]} * m + {aff[1]}" if aff[0] != 0 else f"{aff[1]}"
    tname = f"{name}_c{ci}_s{q}"
    tables.append(f"    static __device__ const unsigned short {tname}[{len(values)}] = "
                  f"{{{', '.join(str(v) for v in values)}}};")
    return f"{tname}[m]"


def _emit_cached_jacobian(classes: List[ExprClass], tables: List[str]):
    """``fj_lanes`` (f and the Jacobian's nonzero coefficients at one state,
    in one pass that shares the subexpressions of both) and ``jmv_cached``
    (J v from those coefficients) for classes of the joint expression
    (f_i, (J v)_i).  A class of M members whose (J v) template reads r
    components of v stores its coefficients at
    ``jac[base + j * M + m]`` (slot j, member m), so the lanes of a warp
    read and write consecutive words."""
    fj = ["    template <class R> static __device__ CBX_NOINLINE void fj_lanes(const R* __restrict__ ys, "
          "const R* __restrict__ ps, const R* __restrict__ ds, R t, R* __restrict__ out, R* __restrict__ jac, "
          "int lane)", "    {", "        (void)ys; (void)ps; (void)ds; (void)t; (void)jac;"]
    jm = ["    template <class R> static __device__ CBX_NOINLINE void jmv_cached(const R* __restrict__ vs, "
          "const R* __restrict__ jac, R* __restrict__ out, int lane)", "    {", "        (void)jac; (void)vs;"]
    fl_fj, fl_jm = FlopCount(), FlopCount()
    base = 0
    for ci, c in enumerate(classes):
        f_t, jv_t = c.template.args
        nm = len(c.members)
        slot_syms = [_placeholder(k, j) for (k, j) in c.slots]
        v_syms = [ph for ph in slot_syms if ph.name[1] == "v"]
        coefs = [sp.diff(jv_t, v) for v in v_syms]
        if any(v in cf.free_symbols for cf in coefs for v in v_syms):
            raise ValueError("Jacobian-vector template is not linear in v")
        sym_map = {TIME: "t"}
        for sy in slot_syms:
            sym_map[sy] = f"s_{sy.name[1:]}"
        printer = _CudaPrinter(sym_map)
        out_idx = _index_expr("fj", ci, 99, c.members, tables)
        head = [f"        // class {ci}: {nm} member(s), {len(v_syms)} coefficient(s) each",
                "        #pragma unroll 1",
                f"        for (int m = lane; m < {nm}; m += 32) {{", f"            const int o = {out_idx};"]
        fj += head
        jm += head
        for q, (kind, j) in enumerate(c.slots):
            col = [row[q] for row in c.indices]
            idx = _index_expr("cj", ci, q, col, tables)
            src = {"y": "ys", "v": "vs", "p": "ps", "d": "ds"}[kind]
            if kind == "v":
                jm.append(f"            const R s_{kind}{j} = {src}[{idx}];")
            else:
                fj.append(f"            const R s_{kind}{j} = {src}[{idx}];")
        reps, reduced = sp.cse([f_t, *coefs], symbols=sp.numbered_symbols("_t"), optimizations="basic")
        for sy, e in reps:
            fj.append(f"            const R {sy} = {printer.doprint(e)};")
            fl_fj = fl_fj + _times(count_ops(e), nm)
        fj.append(f"            out[o] = {printer.doprint(reduced[0])};")
        for k, e in enumerate(reduced):
            fl_fj = fl_fj + _times(count_ops(e), nm)
        for j, e in enumerate(reduced[1:]):
            fj.append(f"            jac[{base + j * nm} + m] = {printer.doprint(e)};")
        terms = [f"jac[{base + j * nm} + m] * {printer.doprint(v)}" for j, v in enumerate(v_syms)]
        jm.append(f"            out[o] = {' + '.join(terms) if terms else 'R(0)'};")
        fl_jm = fl_jm + FlopCount(add=max(len(terms) - 1, 0) * nm, mul=len(terms) * nm)
        fj.append("        }")
        jm.append("        }")
        base += nm * len(v_syms)
    fj.append("    }")
    jm.append("    }")
    return "\n".join(fj), "\n".join(jm), base, fl_fj, fl_jm


def generate_warp_system(system: SymbolicODE, struct_name: str = "WarpSystem") -> WarpSystemCode:
    """Class-grouped right-hand side and Jacobian-vector product."""
    n = system.num_states
    ys = list(system.state_symbols)
    kind_of: Dict[sp.Symbol, Tuple[str, int]] = {}
    for i, s in enumerate(ys):
        kind_of[s] = ("y", i)
    for i, s in enumerate(system.parameter_symbols):
        kind_of[s] = ("p", i)
    for i, s in enumerate(system.driver_symbols):
        kind_of[s] = ("d", i)
    vs = [sp.Symbol(f"_vcomp{i:06d}", real=True) for i in range(n)]  # padded: name order = index order
    kind_v = dict(kind_of)
    for i, s in enumerate(vs):
        kind_v[s] = ("v", i)
    f = system.rhs_expressions()
    J = system.jacobian()
    jv = []
    for i in range(n):
        terms = [J[i, k] * vs[k] for k in range(n) if J[i, k] != 0]
        jv.append(sp.Add(*terms) if terms else sp.Integer(0))
    cf = group_classes(f, kind_of)
    cj = group_classes(jv, kind_v)
    tables: List[str] = []
    body_f, fl_f = _emit_classes("dxdt_lanes", cf, False, tables)
    body_j, fl_j = _emit_classes("jmv_lanes", cj, True, tables)
    flops = {"dxdt": fl_f, "jmv": fl_j}
    # J cached at each linearisation: its nonzero coefficients evaluated
    # together with f, then every J v is a short sum over shared memory
    nnz = sum(1 for i in range(n) for k in range(n) if J[i, k] != 0)
    cached, n_fj = [], 0
    if 0 < nnz <= CACHED_JAC_MAX:
        cfj = group_classes([sp.Tuple(f[i], jv[i]) for i in range(n)], kind_v)
        body_fj, body_jc, stored, fl_fj, fl_jc = _emit_cached_jacobian(cfj, tables)
        cached = [body_fj, body_jc]
        n_fj = len(cfj)
        nnz = stored
        flops.update({"fj": fl_fj, "jmv_cached": fl_jc})
    else:
        nnz = 0
    src = [*(t.strip() for t in tables),
           f"struct {struct_name} {{",
           f"    static constexpr int N = {n};",
           f"    static constexpr int NP = {system.num_parameters};",
           f"    static constexpr int ND = {system.num_drivers};",
           f"    static constexpr int NNZ = {nnz};",
           body_f,
           body_j,
           *cached,
           "};"]
    return WarpSystemCode(source="\n".join(src), n_classes_f=len(cf), n_classes_jv=len(cj),
                          flops=flops, nnz=nnz, n_classes_fj=n_fj)
