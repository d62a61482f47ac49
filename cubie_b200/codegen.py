"""Emit a system's device functions as CUDA C++ from SymPy.

The reference prints Numba-Python device functions from its own IR
(``src/cubie/odesystems/symbolic/engine/printer.py:33-72,429`` and the
templates in ``codegen/dxdt.py:50-93``, ``codegen/linear_operators.py``,
``codegen/time_derivative.py``).  Here one SymPy system becomes one C++
``struct`` of ``template <class R>`` device functions, compiled by NVRTC
together with the hand-written integrator headers:

* ``dxdt``        f(t, y, p, d)
* ``observables`` observable values
* ``jac``         the structurally non-zero Jacobian entries df/dy
* ``jmv``         J v from those entries (compile-time sparsity)
* ``jtmv``        J^T v from the same entries (adjoint sweeps)
* ``dfdt``        df/dt + sum_k df/dd_k * dd_k  (Rosenbrock time term)
* ``pjac``        df/dp non-zeros and ``ptmv`` (df/dp)^T v (adjoint)

Constants are baked in as literals, as the reference bakes constants into
its closures.  Each function reports its flop count (adds, multiplies,
divisions and special-function calls counted from the common-subexpression
DAG) so throughput can be stated against a roofline.
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field
from typing import Dict, List, Sequence, Tuple

import sympy as sp
from sympy.printing.c import C99CodePrinter

from .symbolic import TIME, SymbolicODE


@dataclass
class FlopCount:
    add: int = 0
    mul: int = 0
    div: int = 0
    special: int = 0

    @property
    def flops(self) -> int:
        """Arithmetic operations: add, mul, div and special calls count 1."""
        return self.add + self.mul + self.div + self.special

    def __add__(self, other: "FlopCount") -> "FlopCount":
        return FlopCount(self.add + other.add, self.mul + other.mul,
                         self.div + other.div, self.special + other.special)

    def as_dict(self) -> dict:
        return dict(add=self.add, mul=self.mul, div=self.div, special=self.special, flops=self.flops)


def count_ops(expr: sp.Expr) -> FlopCount:
    """Count arithmetic operations of one (already CSE-reduced) expression."""
    c = FlopCount()

    def walk(e):
        if e.is_Atom:
            return
        if isinstance(e, sp.Add):
            c.add += len(e.args) - 1
        elif isinstance(e, sp.Mul):
            args = [a for a in e.args if not (a.is_Number and abs(a) == 1)]
            c.mul += max(len(args) - 1, 0)
        elif isinstance(e, sp.Pow):
            b, x = e.args
            if x.is_Integer:
                k = abs(int(x))
                c.mul += max(k - 1, 0)
                if int(x) < 0:
                    c.div += 1
            elif x == sp.Rational(1, 2) or x == sp.Rational(-1, 2):
                c.special += 1
                if x < 0:
                    c.div += 1
            else:
                c.special += 1
        elif isinstance(e, sp.Piecewise):
            c.add += len(e.args) - 1  # one select per branch
        elif isinstance(e, (sp.Function, sp.Min, sp.Max, sp.Abs)):
            c.special += 1
        for a in e.args:
            walk(a)

    walk(expr)
    return c


class _CudaPrinter(C99CodePrinter):
    """Print SymPy as templated CUDA C++ (all literals typed as ``R``)."""

    def __init__(self, symbol_map: Dict[sp.Symbol, str]):
        super().__init__()
        self.symbol_map = symbol_map

    def _print_Symbol(self, expr):
        if expr in self.symbol_map:
            return self.symbol_map[expr]
        return super()._print_Symbol(expr)

    def _print_Float(self, expr):
        return f"R({float(expr)!r})"

    def _print_Integer(self, expr):
        return f"R({int(expr)})"

    def _print_Rational(self, expr):
        return f"R({float(expr)!r})"

    def _print_NumberSymbol(self, expr):
        return f"R({float(expr)!r})"

    _print_Pi = _print_NumberSymbol
    _print_Exp1 = _print_NumberSymbol

    def _print_BooleanTrue(self, expr):
        return "true"

    def _print_BooleanFalse(self, expr):
        return "false"

    def _print_Pow(self, expr):
        b, e = expr.args
        bs = self.parenthesize(b, 100)
        if e.is_Integer:
            k = int(e)
            if k == 0:
                return "R(1)"
            mag = abs(k)
            if mag <= 8:
                prod = "*".join([bs] * mag)
                prod = f"({prod})" if mag > 1 else prod
            else:
                prod = f"pow({self._print(b)}, R({mag}))"
            return prod if k > 0 else f"(R(1)/{prod})"
        if e == sp.Rational(1, 2):
            return f"sqrt({self._print(b)})"
        if e == sp.Rational(-1, 2):
            return f"(R(1)/sqrt({self._print(b)}))"
        return f"pow({self._print(b)}, {self._print(e)})"

    def _print_Mul(self, expr):
        # avoid the C printer's "1.0/x" literal forms: print factors explicitly
        coeff, rest = expr.as_coeff_Mul()
        if coeff == -1:
            return "-" + self.parenthesize(rest, 50)
        num, den = [], []
        for a in sp.Mul.make_args(expr):
            if isinstance(a, sp.Pow) and a.args[1].is_Integer and int(a.args[1]) < 0:
                den.append(sp.Pow(a.args[0], -a.args[1]))
            elif a.is_Rational and not a.is_Integer and a.p == 1:
                den.append(sp.Integer(a.q))
            else:
                num.append(a)
        ns = "*".join(self.parenthesize(a, 50) for a in num) if num else "R(1)"
        if not den:
            return ns
        ds = "*".join(self.parenthesize(a, 50) for a in den)
        if len(den) > 1:
            ds = f"({ds})"
        return f"{ns}/{ds}"

    def _print_Piecewise(self, expr):
        parts = []
        for e, c in expr.args[:-1]:
            parts.append(f"({self._print(c)}) ? ({self._print(e)}) : ")
        last_e, last_c = expr.args[-1]
        tail = f"({self._print(last_e)})"
        if last_c is not sp.true and last_c != True:  # noqa: E712
            tail = f"(({self._print(last_c)}) ? ({self._print(last_e)}) : R(0))"
        return "(" + "".join(parts) + tail + ")"

    def _print_Min(self, expr):
        args = [self._print(a) for a in expr.args]
        out = args[0]
        for a in args[1:]:
            out = f"fmin({out}, {a})"
        return out

    def _print_Max(self, expr):
        args = [self._print(a) for a in expr.args]
        out = args[0]
        for a in args[1:]:
            out = f"fmax({out}, {a})"
        return out

    def _print_Abs(self, expr):
        return f"fabs({self._print(expr.args[0])})"

    def _print_sign(self, expr):
        a = self._print(expr.args[0])
        return f"(R(({a}) > R(0)) - R(({a}) < R(0)))"

    def _print_And(self, expr):
        return " && ".join(f"({self._print(a)})" for a in expr.args)

    def _print_Or(self, expr):
        return " || ".join(f"({self._print(a)})" for a in expr.args)

    def _print_Not(self, expr):
        return f"!({self._print(expr.args[0])})"

    def _print_Relational(self, expr):
        return f"({self._print(expr.lhs)} {expr.rel_op} {self._print(expr.rhs)})"

    def _print_ceiling(self, expr):
        return f"ceil({self._print(expr.args[0])})"

    def _print_floor(self, expr):
        return f"floor({self._print(expr.args[0])})"


def _emit_block(outputs: Sequence[Tuple[str, sp.Expr]], symbol_map, indent="        ",
                prefix="cse") -> Tuple[str, FlopCount]:
    """CSE a list of (target, expr) pairs and print C++ statements."""
    exprs = [e for _, e in outputs]
    if not exprs:
        return "", FlopCount()
    syms = sp.numbered_symbols(f"_{prefix}")
    reps, reduced = sp.cse(exprs, symbols=syms, optimizations="basic")
    printer = _CudaPrinter(symbol_map)
    lines = []
    fc = FlopCount()
    for s, e in reps:
        lines.append(f"{indent}const R {s} = {printer.doprint(e)};")
        fc = fc + count_ops(e)
    for (target, _), e in zip(outputs, reduced):
        lines.append(f"{indent}{target} = {printer.doprint(e)};")
        fc = fc + count_ops(e)
    return "\n".join(lines), fc


@dataclass
class GeneratedSystem:
    """CUDA source of a system plus its structural facts."""

    name: str
    source: str
    n: int
    n_params: int
    n_drivers: int
    n_observables: int
    jac_pattern: List[Tuple[int, int]]
    pjac_pattern: List[Tuple[int, int]]
    flops: Dict[str, FlopCount] = field(default_factory=dict)

    @property
    def hash(self) -> str:
        return hashlib.sha256(self.source.encode()).hexdigest()[:16]


def generate_system(system: SymbolicODE, struct_name: str = "System", second_order: bool = False) -> GeneratedSystem:
    """Return the CUDA C++ ``struct`` implementing ``system``.

    With ``second_order`` the struct also carries the contractions the
    Rosenbrock adjoint needs, ``hvpy``: out_i = d/dy_i (v^T J(y) w) and
    ``hvpp``: out_m = d/dp_m (v^T J(y) w), generated from the symbolic
    second derivatives."""
    n = system.num_states
    y_map = {s: f"y[{i}]" for i, s in enumerate(system.state_symbols)}
    p_map = {s: f"p[{i}]" for i, s in enumerate(system.parameter_symbols)}
    d_map = {s: f"d[{i}]" for i, s in enumerate(system.driver_symbols)}
    # Constants stay symbols through CSE and differentiation and print as
    # literals, so ``sigma*(y - x)`` keeps its factored form (substituting
    # the number first would let SymPy distribute it) and rounds exactly as
    # the reference's closure-bound constants do (symbolicODE.py constants,
    # codegen/dxdt.py constant assignments).
    c_map = {s: f"R({float(system.constants[nm])!r})"
             for s, nm in zip(system.constant_symbols, system.constant_names)}
    base_map = {TIME: "t", **y_map, **p_map, **d_map, **c_map}

    f = system.rhs_expressions(substitute_constants=False)
    obs = system.observable_expressions(substitute_constants=False)
    J = sp.Matrix(f).jacobian(sp.Matrix(system.state_symbols)) if n else sp.zeros(0, 0)
    jac_pattern = [(i, j) for i in range(n) for j in range(n) if J[i, j] != 0]
    # parameter Jacobian
    P = sp.Matrix(f).jacobian(sp.Matrix(system.parameter_symbols)) if system.parameter_symbols else sp.zeros(n, 0)
    pjac_pattern = [(i, j) for i in range(n) for j in range(P.shape[1]) if P[i, j] != 0]
    # time derivative (explicit t plus driver chain rule)
    dfdt = []
    for i in range(n):
        e = sp.diff(f[i], TIME)
        for k, ds in enumerate(system.driver_symbols):
            e = e + sp.diff(f[i], ds) * sp.Symbol(f"_dd{k}", real=True)
        dfdt.append(e)
    dd_map = {sp.Symbol(f"_dd{k}", real=True): f"dd[{k}]" for k in range(system.num_drivers)}

    flops: Dict[str, FlopCount] = {}
    body_f, flops["dxdt"] = _emit_block([(f"f[{i}]", e) for i, e in enumerate(f)], base_map)
    body_o, flops["observables"] = _emit_block([(f"o[{i}]", e) for i, e in enumerate(obs)], base_map)
    body_j, flops["jac"] = _emit_block([(f"J[{k}]", J[i, j]) for k, (i, j) in enumerate(jac_pattern)], base_map)
    body_p, flops["pjac"] = _emit_block([(f"P[{k}]", P[i, j]) for k, (i, j) in enumerate(pjac_pattern)], base_map)
    body_t, flops["dfdt"] = _emit_block([(f"out[{i}]", e) for i, e in enumerate(dfdt)], {**base_map, **dd_map})

    # sparse products
    rows: Dict[int, List[Tuple[int, int]]] = {}
    cols: Dict[int, List[Tuple[int, int]]] = {}
    for k, (i, j) in enumerate(jac_pattern):
        rows.setdefault(i, []).append((k, j))
        cols.setdefault(j, []).append((k, i))
    jmv_lines, jtmv_lines = [], []
    for i in range(n):
        terms = " + ".join(f"J[{k}]*v[{j}]" for k, j in rows.get(i, [])) or "R(0)"
        jmv_lines.append(f"        out[{i}] = {terms};")
        terms_t = " + ".join(f"J[{k}]*v[{r}]" for k, r in cols.get(i, [])) or "R(0)"
        jtmv_lines.append(f"        out[{i}] = {terms_t};")
    nnz = len(jac_pattern)
    flops["jmv"] = FlopCount(add=max(nnz - n, 0), mul=nnz)
    pcols: Dict[int, List[Tuple[int, int]]] = {}
    for k, (i, j) in enumerate(pjac_pattern):
        pcols.setdefault(j, []).append((k, i))
    ptmv_lines = []
    for j in range(system.num_parameters):
        terms = " + ".join(f"P[{k}]*v[{i}]" for k, i in pcols.get(j, [])) or "R(0)"
        ptmv_lines.append(f"        out[{j}] = {terms};")

    second = []
    if second_order:
        w_syms = [sp.Symbol(f"_w{i}", real=True) for i in range(n)]
        v_syms = [sp.Symbol(f"_v{i}", real=True) for i in range(n)]
        wv_map = {**{w_syms[i]: f"w[{i}]" for i in range(n)}, **{v_syms[i]: f"v[{i}]" for i in range(n)}}
        contraction = sum(v_syms[i] * J[i, j] * w_syms[j] for (i, j) in jac_pattern) if jac_pattern else sp.Integer(0)
        gy = [sp.diff(contraction, ys) for ys in system.state_symbols]
        gp = [sp.diff(contraction, ps) for ps in system.parameter_symbols]
        body_hy, flops["hvpy"] = _emit_block([(f"out[{i}]", e) for i, e in enumerate(gy)], {**base_map, **wv_map})
        body_hp, flops["hvpp"] = _emit_block([(f"out[{i}]", e) for i, e in enumerate(gp)], {**base_map, **wv_map})
        second = [("hvpy(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, R t, "
                   "const R* __restrict__ w, const R* __restrict__ v, R* __restrict__ out)", body_hy),
                  ("hvpp(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, R t, "
                   "const R* __restrict__ w, const R* __restrict__ v, R* __restrict__ out)", body_hp)]

    def fn(sig, body):
        body = body if body.strip() else "        (void)0;"
        return f"    template <class R>\n    static __device__ __forceinline__ void {sig}\n    {{\n{body}\n    }}\n"

    # M v for a constant mass matrix, row by row in column order, zero entries
    # skipped (the reference's operator and residual generators,
    # linear_operators.py:708-735, nonlinear_residuals.py:324-345)
    mass_lines = []
    if system.mass is not None:
        for i in range(n):
            terms = [("v[%d]" % j) if system.mass[i, j] == 1.0 else f"R({_lit_f(system.mass[i, j])})*v[{j}]"
                     for j in range(n) if system.mass[i, j] != 0.0]
            mass_lines.append(f"        out[{i}] = {' + '.join(terms) if terms else 'R(0)'};")

    unused = "(void)y; (void)p; (void)d; (void)t;"
    src = [f"struct {struct_name} {{",
           f"    static constexpr int N = {n};",
           f"    static constexpr int NP = {system.num_parameters};",
           f"    static constexpr int ND = {system.num_drivers};",
           f"    static constexpr int NO = {system.num_observables};",
           f"    static constexpr int NJ = {max(nnz, 1)};",
           f"    static constexpr bool HAS_DFDT = {str(any(e != 0 for e in dfdt)).lower()};",
           f"    static constexpr int NPJ = {max(len(pjac_pattern), 1)};",
           f"    static constexpr bool HAS_MASS = {str(system.mass is not None).lower()};",
           fn("mass_mv(const R* __restrict__ v, R* __restrict__ out)",
              "        (void)v; (void)out;\n" + "\n".join(mass_lines)),
           fn("dxdt(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, R t, R* __restrict__ f)",
              f"        {unused}\n" + body_f),
           fn("observables(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, R t, R* __restrict__ o)",
              f"        {unused} (void)o;\n" + body_o),
           fn("jac(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, R t, R* __restrict__ J)",
              f"        {unused} (void)J;\n" + body_j),
           fn("jmv(const R* __restrict__ J, const R* __restrict__ v, R* __restrict__ out)",
              "        (void)J; (void)v;\n" + "\n".join(jmv_lines)),
           fn("jtmv(const R* __restrict__ J, const R* __restrict__ v, R* __restrict__ out)",
              "        (void)J; (void)v;\n" + "\n".join(jtmv_lines)),
           fn("dfdt(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, const R* __restrict__ dd, R t, R* __restrict__ out)",
              f"        {unused} (void)dd;\n" + body_t),
           fn("pjac(const R* __restrict__ y, const R* __restrict__ p, const R* __restrict__ d, R t, R* __restrict__ P)",
              f"        {unused} (void)P;\n" + body_p),
           fn("ptmv(const R* __restrict__ P, const R* __restrict__ v, R* __restrict__ out)",
              "        (void)P; (void)v; (void)out;\n" + "\n".join(ptmv_lines)),
           *[fn(sig, f"        {unused} (void)w; (void)v; (void)out;\n" + body) for sig, body in second],
           "};"]
    source = "\n".join(src)
    return GeneratedSystem(name=system.name, source=source, n=n,
                           n_params=system.num_parameters, n_drivers=system.num_drivers,
                           n_observables=system.num_observables,
                           jac_pattern=jac_pattern, pjac_pattern=pjac_pattern, flops=flops)


def _lit_f(x: float) -> str:
    return repr(float(x))


def system_stub(system: SymbolicODE, struct_name: str = "System") -> GeneratedSystem:
    """The size constants of ``system`` without any functions: the
    warp-per-system layout evaluates the system through its class-grouped
    code (cubie_b200/warpgen.py) and needs nothing else from the
    straight-line struct."""
    n = system.num_states
    src = "\n".join([f"struct {struct_name} {{",
                     f"    static constexpr int N = {n};",
                     f"    static constexpr int NP = {system.num_parameters};",
                     f"    static constexpr int ND = {system.num_drivers};",
                     f"    static constexpr int NO = {system.num_observables};",
                     "    static constexpr int NJ = 1;",
                     "    static constexpr bool HAS_DFDT = true;",
                     "    static constexpr int NPJ = 1;",
                     f"    static constexpr bool HAS_MASS = {str(system.mass is not None).lower()};",
                     "};"])
    return GeneratedSystem(name=system.name, source=src, n=n, n_params=system.num_parameters,
                           n_drivers=system.num_drivers, n_observables=system.num_observables,
                           jac_pattern=[], pjac_pattern=[], flops={})
