"""Symbolic ODE systems built from equation strings.

A system is a list of ``lhs = rhs`` assignments.  ``dX = ...`` defines the
derivative of state ``X``; any other left-hand side is an auxiliary
(an *observable* when it is listed in ``observables``).  This mirrors the
string front end of ``create_ODE_system``
(``src/cubie/odesystems/symbolic/symbolicODE.py:102-211``) and the
symbol categories of ``parsing/parser.py:627-800`` in the reference:
states, parameters (per-run values), constants (baked into the compiled
code), drivers (time series sampled by an interpolator) and observables.

Expressions are parsed with Python's own ``ast`` module (so conditional
expressions ``a if cond else b``, comparisons and ``**`` read as in
Python) and turned into SymPy expressions.
"""

from __future__ import annotations

import ast
import re
import hashlib
from typing import Callable, Dict, Iterable, List, Mapping, Optional, Sequence, Tuple, Union

import numpy as np
import sympy as sp

TIME = sp.Symbol("t", real=True)

_FUNCTIONS: Dict[str, Callable] = {
    "exp": sp.exp, "log": sp.log, "ln": sp.log, "sqrt": sp.sqrt,
    "sin": sp.sin, "cos": sp.cos, "tan": sp.tan,
    "asin": sp.asin, "acos": sp.acos, "atan": sp.atan, "atan2": sp.atan2,
    "sinh": sp.sinh, "cosh": sp.cosh, "tanh": sp.tanh,
    "abs": sp.Abs, "Abs": sp.Abs, "fabs": sp.Abs,
    "min": sp.Min, "Min": sp.Min, "max": sp.Max, "Max": sp.Max,
    "pow": sp.Pow, "floor": sp.floor, "ceil": sp.ceiling,
    "sign": sp.sign, "erf": sp.erf,
}

_CMP = {ast.Lt: sp.Lt, ast.LtE: sp.Le, ast.Gt: sp.Gt, ast.GtE: sp.Ge,
        ast.Eq: sp.Eq, ast.NotEq: sp.Ne}


class _ToSympy(ast.NodeVisitor):
    """Convert a Python expression AST into a SymPy expression."""

    def __init__(self, symbols: Dict[str, sp.Symbol]):
        self.symbols = symbols

    def sym(self, name: str) -> sp.Symbol:
        if name not in self.symbols:
            self.symbols[name] = sp.Symbol(name, real=True)
        return self.symbols[name]

    def visit_Expression(self, node):
        return self.visit(node.body)

    def visit_Constant(self, node):
        if isinstance(node.value, bool):
            return sp.true if node.value else sp.false
        if isinstance(node.value, int):
            return sp.Integer(node.value)
        if isinstance(node.value, float):
            return sp.Float(node.value, 17)
        raise ValueError(f"unsupported literal {node.value!r}")

    def visit_Name(self, node):
        if node.id == "t":
            return TIME
        if node.id in ("pi",):
            return sp.pi
        if node.id in ("E", "e") and node.id not in self.symbols:
            return sp.E
        return self.sym(node.id)

    def visit_UnaryOp(self, node):
        v = self.visit(node.operand)
        if isinstance(node.op, ast.USub):
            return -v
        if isinstance(node.op, ast.UAdd):
            return v
        if isinstance(node.op, ast.Not):
            return sp.Not(v)
        raise ValueError("unsupported unary operator")

    def visit_BinOp(self, node):
        a, b = self.visit(node.left), self.visit(node.right)
        op = node.op
        if isinstance(op, ast.Add):
            return a + b
        if isinstance(op, ast.Sub):
            return a - b
        if isinstance(op, ast.Mult):
            return a * b
        if isinstance(op, ast.Div):
            return a / b
        if isinstance(op, ast.Pow):
            return a ** b
        raise ValueError("unsupported binary operator")

    def visit_BoolOp(self, node):
        vals = [self.visit(v) for v in node.values]
        return sp.And(*vals) if isinstance(node.op, ast.And) else sp.Or(*vals)

    def visit_Compare(self, node):
        left = self.visit(node.left)
        parts = []
        for op, comp in zip(node.ops, node.comparators):
            right = self.visit(comp)
            parts.append(_CMP[type(op)](left, right))
            left = right
        return parts[0] if len(parts) == 1 else sp.And(*parts)

    def visit_IfExp(self, node):
        cond = self.visit(node.test)
        return sp.Piecewise((self.visit(node.body), cond),
                            (self.visit(node.orelse), True))

    def visit_Call(self, node):
        if not isinstance(node.func, ast.Name) or node.func.id not in _FUNCTIONS:
            name = getattr(node.func, "id", "?")
            raise ValueError(f"unsupported function '{name}'")
        args = [self.visit(a) for a in node.args]
        return _FUNCTIONS[node.func.id](*args)

    def generic_visit(self, node):
        raise ValueError(f"unsupported syntax: {ast.dump(node)}")


def parse_expression(text: str, symbols: Dict[str, sp.Symbol]) -> sp.Expr:
    """Parse one right-hand side into SymPy using ``symbols`` for names."""
    tree = ast.parse(text.strip().replace("^", "**"), mode="eval")
    return _ToSympy(symbols).visit(tree)


def _split_equations(dxdt: Union[str, Iterable[str]]) -> List[Tuple[str, str]]:
    if isinstance(dxdt, str):
        lines = [ln for ln in dxdt.replace(";", "\n").splitlines()]
    else:
        lines = list(dxdt)
    eqs = []
    for ln in lines:
        ln = ln.split("#", 1)[0].strip()
        if not ln:
            continue
        if "=" not in ln:
            raise ValueError(f"equation '{ln}' has no '='")
        # split on the first bare '=' (not part of ==, <=, >=, !=)
        idx = None
        for i, ch in enumerate(ln):
            if ch == "=" and (i + 1 >= len(ln) or ln[i + 1] != "=") and (i == 0 or ln[i - 1] not in "=<>!"):
                idx = i
                break
        if idx is None:
            raise ValueError(f"equation '{ln}' has no assignment")
        eqs.append((ln[:idx].strip(), ln[idx + 1:].strip()))
    return eqs


def _as_defaults(spec, kind: str) -> Dict[str, float]:
    if spec is None:
        return {}
    if isinstance(spec, Mapping):
        return {str(k): float(np.asarray(v).flat[0]) if v is not None else 0.0 for k, v in spec.items()}
    return {str(k): 0.0 for k in spec}


class SymbolicODE:
    """An ODE system ``dy/dt = f(t, y, p, d)`` with optional observables.

    Attributes mirror the reference ``SymbolicODE`` bookkeeping
    (``symbolicODE.py:213-1059``): ordered state, parameter, constant,
    driver and observable names with default values, the precision the
    system compiles at, and a stable hash of the definition used to key
    compiled modules.
    """

    def __init__(self, *, states: Dict[str, float], parameters: Dict[str, float],
                 constants: Dict[str, float], drivers: List[str],
                 observables: List[str], assignments: List[Tuple[sp.Symbol, sp.Expr]],
                 derivatives: Dict[str, sp.Expr], precision=np.float32,
                 name: Optional[str] = None, driver_settings: Optional[dict] = None,
                 source: str = "", mass=None):
        self.state_names = list(states)
        self.initial_values = dict(states)
        self.parameter_names = list(parameters)
        self.parameters = dict(parameters)
        self.constant_names = list(constants)
        self.constants = dict(constants)
        self.driver_names = list(drivers)
        self.observable_names = list(observables)
        self.assignments = list(assignments)
        self.derivatives = derivatives
        self.precision = np.dtype(precision).type
        self.driver_settings = driver_settings
        # constant mass matrix M of M y' = f(t, y) (None: identity), paired
        # row for row with the state order (symbolicODE.py ``mass``)
        n = len(self.state_names)
        if mass is not None:
            m = np.asarray(mass, dtype=np.float64)
            if m.shape != (n, n):
                raise ValueError(f"mass matrix has shape {m.shape}; expected ({n}, {n})")
            if not np.all(np.isfinite(m)):
                raise ValueError("mass matrix entries must be finite")
            mass = None if np.array_equal(m, np.eye(n)) else m
        self.mass = mass
        if mass is not None:
            source = source + "|M" + ",".join(repr(float(v)) for v in mass.ravel())
        self._source = source
        self.fn_hash = hashlib.sha256(
            (source + repr(sorted(self.constants.items())) + str(np.dtype(self.precision))).encode()
        ).hexdigest()[:16]
        self.name = name or f"system_{self.fn_hash}"
        self.state_symbols = [sp.Symbol(n, real=True) for n in self.state_names]
        self.parameter_symbols = [sp.Symbol(n, real=True) for n in self.parameter_names]
        self.constant_symbols = [sp.Symbol(n, real=True) for n in self.constant_names]
        self.driver_symbols = [sp.Symbol(n, real=True) for n in self.driver_names]
        self.observable_symbols = [sp.Symbol(n, real=True) for n in self.observable_names]
        self._jac = None

    def with_precision(self, precision) -> "SymbolicODE":
        """The same system compiled at another precision."""
        return SymbolicODE(states=self.initial_values, parameters=self.parameters, constants=self.constants,
                           drivers=self.driver_names, observables=self.observable_names,
                           assignments=self.assignments, derivatives=self.derivatives, precision=precision,
                           name=self.name, driver_settings=self.driver_settings,
                           source=self._source.split("|M")[0], mass=self.mass)

    # -- sizes ---------------------------------------------------------
    @property
    def num_states(self) -> int:
        return len(self.state_names)

    @property
    def num_parameters(self) -> int:
        return len(self.parameter_names)

    @property
    def num_drivers(self) -> int:
        return len(self.driver_names)

    @property
    def num_observables(self) -> int:
        return len(self.observable_names)

    @property
    def sizes(self) -> dict:
        return dict(states=self.num_states, parameters=self.num_parameters,
                    drivers=self.num_drivers, observables=self.num_observables,
                    constants=len(self.constant_names))

    # -- expressions ---------------------------------------------------
    def _substitution_chain(self) -> Dict[sp.Symbol, sp.Expr]:
        """Fully substituted expressions for every auxiliary symbol."""
        subs: Dict[sp.Symbol, sp.Expr] = {}
        for lhs, rhs in self.assignments:
            subs[lhs] = rhs.xreplace(subs)
        return subs

    def rhs_expressions(self, substitute_constants: bool = True) -> List[sp.Expr]:
        """Return ``f_i`` for each state with auxiliaries substituted."""
        chain = self._substitution_chain()
        out = []
        for name in self.state_names:
            e = self.derivatives[name].xreplace(chain)
            if substitute_constants:
                e = e.xreplace(self.constant_map())
            out.append(e)
        return out

    def observable_expressions(self, substitute_constants: bool = True) -> List[sp.Expr]:
        chain = self._substitution_chain()
        out = []
        for sym in self.observable_symbols:
            e = chain.get(sym, sym)
            if substitute_constants:
                e = e.xreplace(self.constant_map())
            out.append(e)
        return out

    def constant_map(self) -> Dict[sp.Symbol, sp.Expr]:
        return {s: sp.Float(self.constants[n], 17) for s, n in zip(self.constant_symbols, self.constant_names)}

    def jacobian(self) -> sp.Matrix:
        """Dense symbolic Jacobian ``df/dy`` (constants substituted)."""
        if self._jac is None:
            f = sp.Matrix(self.rhs_expressions())
            self._jac = f.jacobian(sp.Matrix(self.state_symbols))
        return self._jac

    # -- default arrays -----------------------------------------------
    def default_initial_values(self) -> np.ndarray:
        return np.array([self.initial_values[n] for n in self.state_names], dtype=self.precision)

    def default_parameters(self) -> np.ndarray:
        return np.array([self.parameters[n] for n in self.parameter_names], dtype=self.precision)

    def state_index(self, name: str) -> int:
        return self.state_names.index(name)

    def observable_index(self, name: str) -> int:
        return self.observable_names.index(name)

    def __repr__(self) -> str:
        return (f"SymbolicODE(name={self.name!r}, states={self.state_names}, "
                f"parameters={self.parameter_names}, drivers={self.driver_names}, "
                f"observables={self.observable_names})")


def create_ODE_system(
    dxdt: Union[str, Iterable[str]],
    precision=np.float32,
    states: Optional[Union[Mapping[str, float], Iterable[str]]] = None,
    observables: Optional[Iterable[str]] = None,
    parameters: Optional[Union[Mapping[str, float], Iterable[str]]] = None,
    constants: Optional[Union[Mapping[str, float], Iterable[str]]] = None,
    drivers: Optional[Union[Iterable[str], Mapping[str, object]]] = None,
    name: Optional[str] = None,
    strict: bool = False,
    mass=None,
    simplify: Optional[bool] = None,
    state_priority: Optional[Mapping[str, float]] = None,
    irreducible: Optional[Iterable[str]] = None,
    **unsupported,
) -> SymbolicODE:
    """Build a :class:`SymbolicODE` from ``lhs = rhs`` equation strings.

    Mirrors ``create_ODE_system`` (``symbolicODE.py:102-211``) for the
    string front end.  ``dX`` on the left declares the derivative of state
    ``X``.  With ``strict=False`` undeclared states are inferred from
    ``dX`` left-hand sides and undeclared right-hand-side names become
    parameters (default 0), as the reference's inference does
    (``parsing/parser.py:715-800``); ``strict=True`` raises instead.
    ``mass`` is a constant mass matrix M (``M y' = f``, states in declared
    order; ``None`` is the identity), as the reference's ``mass`` argument:
    a singular M makes a semi-explicit DAE and needs an implicit
    algorithm.

    DAE input (an implicit equation ``0 = g`` or ``expr = expr``, a
    declared state without a derivative equation or defined explicitly,
    a second derivative ``d(d(x, t), t) = f``), or ``simplify=True``, goes
    through :func:`cubie_b200.structural.structural_simplify` first, as
    the reference's ``simplify`` path does (``symbolicODE.py:380-470``):
    aliases and solvable algebraic unknowns become observables, the
    remaining algebraic unknowns stay as states with their residuals, and
    the system carries the mass matrix diag(1, ..., 1, 0, ..., 0), which a
    caller's ``mass`` cannot override.  ``state_priority`` and
    ``irreducible`` steer which unknowns survive.
    """
    for key, value in unsupported.items():
        if value not in (None, False, {}):
            raise NotImplementedError(f"create_ODE_system option '{key}' is not supported")
    eqs = _split_equations(dxdt)
    state_defaults = _as_defaults(states, "states")
    param_defaults = _as_defaults(parameters, "parameters")
    const_defaults = _as_defaults(constants, "constants")
    driver_settings = None
    if isinstance(drivers, Mapping):
        driver_settings = dict(drivers)
        driver_names = [k for k in drivers.keys() if k not in ("time", "driver_sample_period", "wrap", "order", "boundary_condition", "t0")]
    else:
        driver_names = list(drivers) if drivers is not None else []
    obs_names = list(observables) if observables is not None else []
    if simplify is not False and (simplify or _is_dae_input(eqs, state_defaults)):
        if mass is not None:
            raise ValueError("the system's mass matrix is derived by structural simplification and pairs with "
                             "the simplified state order; 'mass' cannot override it")
        return _create_dae_system(eqs, precision, state_defaults, obs_names, param_defaults, const_defaults,
                                  driver_names, driver_settings, name, strict, state_priority or {},
                                  list(irreducible or ()))

    lhs_names = [lhs for lhs, _ in eqs]
    # derivative targets
    deriv_targets = {}
    for lhs in lhs_names:
        if lhs.startswith("d") and len(lhs) > 1:
            target = lhs[1:]
            if target in state_defaults or (not strict and target not in lhs_names and target not in param_defaults
                                             and target not in const_defaults and target not in driver_names
                                             and target not in obs_names):
                deriv_targets[lhs] = target
    if states is None:
        if strict:
            raise ValueError("strict=True requires states to be declared")
        for lhs, tgt in deriv_targets.items():
            state_defaults.setdefault(tgt, 0.0)
    else:
        for lhs, tgt in list(deriv_targets.items()):
            if tgt not in state_defaults:
                if strict:
                    raise ValueError(f"'{lhs}' refers to undeclared state '{tgt}'")
                state_defaults[tgt] = 0.0

    symbols: Dict[str, sp.Symbol] = {}
    known = set(state_defaults) | set(param_defaults) | set(const_defaults) | set(driver_names)
    assignments: List[Tuple[sp.Symbol, sp.Expr]] = []
    derivatives: Dict[str, sp.Expr] = {}
    defined: set = set()
    for lhs, rhs in eqs:
        expr = parse_expression(rhs, symbols)
        if lhs in deriv_targets and deriv_targets[lhs] in state_defaults:
            tgt = deriv_targets[lhs]
            if tgt in derivatives:
                raise ValueError(f"state '{tgt}' has two derivative equations")
            derivatives[tgt] = expr
            sym = sp.Symbol(lhs, real=True)
            symbols.setdefault(lhs, sym)
            assignments.append((sym, expr))
            defined.add(lhs)
        else:
            if lhs in known:
                raise ValueError(f"'{lhs}' is declared as an input and cannot be assigned")
            sym = symbols.setdefault(lhs, sp.Symbol(lhs, real=True))
            assignments.append((sym, expr))
            defined.add(lhs)
    missing = [s for s in state_defaults if s not in derivatives]
    if missing:
        raise ValueError(f"states without derivative equations: {missing}")
    # undeclared inputs
    used = set()
    for _, e in assignments:
        used |= {s.name for s in e.free_symbols}
    used.discard("t")
    undeclared = sorted(used - known - defined)
    if undeclared:
        if strict:
            raise ValueError(f"undeclared symbols with strict=True: {undeclared}")
        for u in undeclared:
            param_defaults[u] = 0.0
    for o in obs_names:
        if o not in defined:
            raise ValueError(f"observable '{o}' has no defining equation")
    # dependency order check (auxiliaries must be defined before use)
    seen = set(state_defaults) | set(param_defaults) | set(const_defaults) | set(driver_names) | {"t"}
    for lhs, rhs in assignments:
        deps = {s.name for s in rhs.free_symbols}
        if not deps <= seen | defined:
            raise ValueError(f"'{lhs}' uses undefined names {sorted(deps - seen - defined)}")
    assignments = _topological(assignments, seen)
    source = "\n".join(f"{l} = {r}" for l, r in eqs)
    source += "|S" + ",".join(state_defaults) + "|P" + ",".join(param_defaults)
    source += "|D" + ",".join(driver_names) + "|O" + ",".join(obs_names)
    return SymbolicODE(states=state_defaults, parameters=param_defaults,
                       constants=const_defaults, drivers=driver_names,
                       observables=obs_names, assignments=assignments,
                       derivatives=derivatives, precision=precision, name=name,
                       driver_settings=driver_settings, source=source, mass=mass)


_SECOND = re.compile(r"^d\(\s*d\(\s*([A-Za-z_]\w*)\s*,\s*t\s*\)\s*,\s*t\s*\)$")
_FIRST = re.compile(r"^d\(\s*([A-Za-z_]\w*)\s*,\s*t\s*\)$")


def _is_dae_input(eqs, state_defaults) -> bool:
    """Whether the equations need structural simplification: an implicit
    or higher-order left-hand side, an explicit definition of a declared
    state, or a declared state without a derivative equation."""
    have_deriv = set()
    for lhs, _ in eqs:
        if _SECOND.match(lhs) or _FIRST.match(lhs):
            return True
        if not lhs.isidentifier():
            return True
        if lhs in state_defaults:
            return True
        if lhs.startswith("d") and lhs[1:] in state_defaults:
            have_deriv.add(lhs[1:])
    return bool(state_defaults) and any(s not in have_deriv for s in state_defaults)


def _create_dae_system(eqs, precision, state_defaults, obs_names, param_defaults, const_defaults, driver_names,
                       driver_settings, name, strict, state_priority, irreducible) -> "SymbolicODE":
    """The DAE front end of :func:`create_ODE_system` (structural
    simplification, then an implicit system with a singular mass matrix)."""
    from .structural import structural_simplify
    if not state_defaults:
        raise ValueError("DAE input needs its unknowns declared as states")
    symbols: Dict[str, sp.Symbol] = {}
    unknowns = {n: symbols.setdefault(n, sp.Symbol(n, real=True)) for n in state_defaults}
    inputs = set(param_defaults) | set(const_defaults) | set(driver_names)
    derivs: Dict[sp.Symbol, sp.Expr] = {}
    explicit: List[Tuple[sp.Symbol, sp.Expr]] = []
    implicit: List[sp.Expr] = []
    aux: List[Tuple[sp.Symbol, sp.Expr]] = []
    order = list(state_defaults)
    defaults = dict(state_defaults)

    def set_derivative(target: str, expr: sp.Expr) -> None:
        sym = unknowns[target]
        if sym in derivs:
            raise ValueError(f"state '{target}' has two derivative equations")
        derivs[sym] = expr

    for lhs, rhs in eqs:
        expr = parse_expression(rhs, symbols)
        m2, m1 = _SECOND.match(lhs), _FIRST.match(lhs)
        target = m2.group(1) if m2 else (m1.group(1) if m1 else None)
        if target is None and lhs.startswith("d") and lhs[1:] in unknowns:
            target = lhs[1:]
        if target is not None:
            if target not in unknowns:
                raise ValueError(f"'{lhs}' differentiates '{target}', which is not a declared state")
            if m2:
                # companion state for the first derivative: x_t (a declared
                # state of that name is used as it, with its initial value)
                comp = f"{target}_t"
                if comp not in unknowns:
                    while comp in inputs or comp in symbols:
                        comp += "_"
                    unknowns[comp] = symbols.setdefault(comp, sp.Symbol(comp, real=True))
                    order.insert(order.index(target) + 1, comp)
                    defaults.setdefault(comp, 0.0)
                set_derivative(target, unknowns[comp])
                set_derivative(comp, expr)
            else:
                set_derivative(target, expr)
        elif lhs.isidentifier() and lhs in unknowns:
            explicit.append((unknowns[lhs], expr))
        elif lhs.isidentifier() and lhs not in inputs:
            aux.append((symbols.setdefault(lhs, sp.Symbol(lhs, real=True)), expr))
        elif lhs.isidentifier():
            raise ValueError(f"'{lhs}' is declared as an input and is immutable")
        else:
            # ``lhs = rhs`` constrains rhs - lhs to zero (``0 = g`` gives g)
            implicit.append(expr - parse_expression(lhs, symbols))
    # auxiliary definitions (and references to a state's derivative) are
    # substituted so that the structure is seen in the unknowns
    dsyms = {symbols[f"d{n}"]: derivs[unknowns[n]] for n in unknowns
             if f"d{n}" in symbols and unknowns[n] in derivs}
    rule = {**{a: e for a, e in aux}, **dsyms}
    for _ in range(len(rule) + 1):
        new_rule = {k: v.xreplace(rule) for k, v in rule.items()}
        if new_rule == rule:
            break
        rule = new_rule

    def expand(e: sp.Expr) -> sp.Expr:
        return e.xreplace(rule)

    derivs = {k: expand(v) for k, v in derivs.items()}
    explicit = [(u, expand(e)) for u, e in explicit]
    implicit = [expand(g) for g in implicit]
    # the derivative of an unknown with no derivative equation inside an
    # expression makes a higher-index system
    hidden = sorted(n for n in unknowns if unknowns[n] not in derivs and f"d{n}" in symbols
                    and any(symbols[f"d{n}"] in e.free_symbols
                            for e in list(derivs.values()) + [e for _, e in explicit] + implicit))
    if hidden:
        from .structural import InvalidSystemError
        raise InvalidSystemError(f"derivatives of algebraic unknowns {hidden} appear in the equations (a "
                                 "higher-index system); index reduction is not built")
    known_names = set(unknowns) | inputs | {a.name for a, _ in aux} | {"t"}
    used = set()
    for e in list(derivs.values()) + [e for _, e in explicit] + implicit:
        used |= {s.name for s in e.free_symbols}
    undeclared = sorted(used - known_names)
    if undeclared:
        if strict:
            raise ValueError(f"undefined symbols with strict=True: {undeclared}")
        for u in undeclared:
            param_defaults[u] = 0.0
    for o in obs_names:
        if o not in {a.name for a, _ in aux} and o not in unknowns:
            raise ValueError(f"observable '{o}' has no defining equation")
    res = structural_simplify([unknowns[n] for n in order], derivs, implicit, explicit,
                              {unknowns[k]: float(v) for k, v in state_priority.items() if k in unknowns},
                              [unknowns[k] for k in irreducible if k in unknowns])
    states_out = {s.name: defaults[s.name] for s in res.states}
    derivatives: Dict[str, sp.Expr] = {}
    assignments: List[Tuple[sp.Symbol, sp.Expr]] = []
    for s_ in res.differential_states:
        derivatives[s_.name] = res.dxdt[s_]
    for s_, g in zip(res.algebraic_states, res.residuals):
        derivatives[s_.name] = g
    observed_names = [u.name for u, _ in res.observed]
    for u, e in res.observed:
        assignments.append((u, e))
    # the caller's auxiliaries, in terms of the surviving states
    obs_rule = {u: e for u, e in res.observed}
    for a, e in aux:
        assignments.append((a, expand(e).xreplace(obs_rule)))
    for n, e in derivatives.items():
        assignments.append((sp.Symbol(f"d{n}", real=True), e))
    seen = set(states_out) | set(param_defaults) | set(const_defaults) | set(driver_names) | {"t"}
    assignments = _topological(assignments, seen)
    observables_out = list(obs_names) + [n for n in observed_names if n not in obs_names]
    source = "DAE|" + "\n".join(f"{l} = {r}" for l, r in eqs)
    source += "|S" + ",".join(states_out) + "|P" + ",".join(param_defaults)
    source += "|D" + ",".join(driver_names) + "|O" + ",".join(observables_out)
    return SymbolicODE(states=states_out, parameters=param_defaults, constants=const_defaults,
                       drivers=driver_names, observables=observables_out, assignments=assignments,
                       derivatives=derivatives, precision=precision, name=name,
                       driver_settings=driver_settings, source=source, mass=res.mass_matrix)


def _topological(assignments, base_names):
    """Order auxiliary assignments so every use follows its definition."""
    remaining = list(assignments)
    done = set(base_names)
    ordered = []
    while remaining:
        progressed = False
        for item in list(remaining):
            lhs, rhs = item
            if {s.name for s in rhs.free_symbols} <= done:
                ordered.append(item)
                done.add(lhs.name)
                remaining.remove(item)
                progressed = True
        if not progressed:
            raise ValueError(f"circular definitions among {[l.name for l, _ in remaining]}")
    return ordered
