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
            fc = fc + count_ops(e)
        lines.append(f"            out[o] = {printer.doprint(reduced[0])};")
        fc = fc + count_ops(reduced[0])
        lines.append("        }")
    lines.append("    }")
    return "\n".join(lines), fc


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
    src = [*(t.strip() for t in tables),
           f"struct {struct_name} {{",
           f"    static constexpr int N = {n};",
           f"    static constexpr int NP = {system.num_parameters};",
           f"    static constexpr int ND = {system.num_drivers};",
           body_f,
           body_j,
           "};"]
    return WarpSystemCode(source="\n".join(src), n_classes_f=len(cf), n_classes_jv=len(cj),
                          flops={"dxdt": fl_f, "jmv": fl_j})
