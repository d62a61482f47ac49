"""Structural simplification of differential-algebraic input (host side).

The reference turns DAE input into a system its implicit steppers can
integrate (``src/cubie/odesystems/symbolic/structural/``: the pipeline in
``simplify.py:271-420``, alias elimination ``alias_elimination.py``, the
equation/unknown matching ``bipartite.py`` and ``consistency.py``, tearing
``tearing.py``, the mass matrix of the torn system
``singularity_removal.py``).  This module does the same for index-1
systems, in SymPy on the host, before code generation:

* unknowns are the declared states; an unknown with a derivative equation
  is differential, the others are algebraic;
* a second derivative ``d(d(x, t), t) = f`` is lowered with a companion
  state ``x_t`` (``dx = x_t``, ``dx_t = f``);
* an implicit equation ``0 = a - b`` or ``0 = a + b`` between two
  unknowns is a perfect alias: one unknown is replaced by the other (the
  one with the higher ``state_priority`` survives, then a differential
  over an algebraic one, then the earlier declared), and becomes an
  observed output; aliasing two differential states drops the eliminated
  state's derivative equation when it coincides with the survivor's;
* an unknown defined explicitly (``y = expr``) becomes observed unless it
  is listed as ``irreducible`` (irreducible unknowns take no part in alias
  elimination or tearing and stay as states);
* the remaining implicit equations are matched to the remaining algebraic
  unknowns (every equation to a distinct unknown it contains); more
  equations than unknowns, or fewer, raise;
* a set of constraints that cannot be matched (a higher-index system, such
  as the pendulum in Cartesian coordinates) is differentiated along the
  differential equations until its highest derivatives match
  (Pantelides' criterion); the lower derivatives stay as invariants, and
  each demotes one differential state it contains to an algebraic unknown
  (the lowest ``state_priority`` first), as the dummy-derivative method
  selects states (see ``_reduce_index``);
* the matched blocks are visited in dependency order (strongly connected
  components of the equation graph): a single equation affine in its
  unknown, or a block linear in its unknowns with a nonsingular matrix, is
  solved and its unknowns become observed; any other block is torn: its
  unknowns stay as algebraic states and its equations as residuals.

The result carries the differential states, the algebraic states with one
residual each, and the observed definitions.  The system it becomes has
the states in that order and the mass matrix diag(1, ..., 1, 0, ..., 0):
``M y' = F(y)`` with F the derivatives of the differential states followed
by the residuals.  The state selection of the index reduction is static,
as the reference's priorities make it: it holds while the invariants stay
regular in the demoted states along the solution (the pendulum with y and
vy kept needs x away from 0).  Constraints whose derivatives involve the
derivatives of algebraic unknowns are not reduced (they raise).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, Iterable, List, Mapping, Optional, Sequence, Set, Tuple

import sympy as sp


class InvalidSystemError(ValueError):
    """The equations do not determine the unknowns."""


class ExtraEquationsSystemError(InvalidSystemError):
    """More independent equations than unknowns."""


class ExtraVariablesSystemError(InvalidSystemError):
    """More unknowns than equations."""


@dataclass
class SimplifiedSystem:
    differential_states: List[sp.Symbol]
    algebraic_states: List[sp.Symbol]
    dxdt: Dict[sp.Symbol, sp.Expr]
    residuals: List[sp.Expr]
    observed: List[Tuple[sp.Symbol, sp.Expr]] = field(default_factory=list)

    @property
    def states(self) -> List[sp.Symbol]:
        return list(self.differential_states) + list(self.algebraic_states)

    @property
    def mass_matrix(self) -> Optional[List[List[float]]]:
        """diag(1 per differential state, 0 per algebraic state), or None
        for an ODE."""
        if not self.algebraic_states:
            return None
        n = len(self.states)
        nd = len(self.differential_states)
        return [[1.0 if (i == j and i < nd) else 0.0 for j in range(n)] for i in range(n)]


def _alias(g: sp.Expr, unknowns: Set[sp.Symbol]) -> Optional[Tuple[sp.Symbol, sp.Symbol, int]]:
    """(a, b, s) when g = c (a - s b) with a, b unknowns and s = +-1."""
    terms = sp.Add.make_args(sp.expand(g))
    if len(terms) != 2:
        return None
    parts = []
    for term in terms:
        coeff, rest = term.as_coeff_Mul()
        if rest not in unknowns or coeff not in (1, -1):
            return None
        parts.append((rest, int(coeff)))
    (a, ca), (b, cb) = parts
    return a, b, -ca * cb


def _match(equations: Sequence[Set[sp.Symbol]], unknowns: Sequence[sp.Symbol]) -> Optional[List[int]]:
    """A complete matching of equations to distinct unknowns they contain
    (augmenting paths), as ``unknown index per equation``; None when there
    is none."""
    owner: Dict[int, int] = {}
    index = {u: k for k, u in enumerate(unknowns)}
    adj = [sorted(index[u] for u in inc if u in index) for inc in equations]

    def augment(e: int, seen: Set[int]) -> bool:
        for v in adj[e]:
            if v in seen:
                continue
            seen.add(v)
            if v not in owner or augment(owner[v], seen):
                owner[v] = e
                return True
        return False

    for e in range(len(equations)):
        if not augment(e, set()):
            return None
    out = [0] * len(equations)
    for v, e in owner.items():
        out[e] = v
    return out


def _components(n: int, edges: Sequence[Sequence[int]]) -> List[List[int]]:
    """Strongly connected components of a directed graph (Tarjan), each
    after every component it has an edge into (dependencies first)."""
    index: Dict[int, int] = {}
    low: Dict[int, int] = {}
    stack: List[int] = []
    on: Set[int] = set()
    out: List[List[int]] = []
    counter = [0]

    def visit(v: int) -> None:
        index[v] = low[v] = counter[0]
        counter[0] += 1
        stack.append(v)
        on.add(v)
        for w in edges[v]:
            if w not in index:
                visit(w)
                low[v] = min(low[v], low[w])
            elif w in on:
                low[v] = min(low[v], index[w])
        if low[v] == index[v]:
            comp = []
            while True:
                w = stack.pop()
                on.discard(w)
                comp.append(w)
                if w == v:
                    break
            out.append(sorted(comp))

    for v in range(n):
        if v not in index:
            visit(v)
    return out


def _solve_single(g: sp.Expr, z: sp.Symbol) -> Optional[sp.Expr]:
    """z from g(z) = 0 when g is affine in z (a unique, branch-free
    solution); None otherwise, and the equation is torn."""
    try:
        poly = sp.Poly(sp.expand(g), z)
    except sp.PolynomialError:
        return None
    if poly.degree() != 1:
        return None
    c1, c0 = poly.all_coeffs()
    if z in c1.free_symbols or z in c0.free_symbols or c1 == 0:
        return None
    return sp.simplify(-c0 / c1)


def _solve_linear(gs: Sequence[sp.Expr], zs: Sequence[sp.Symbol]) -> Optional[Dict[sp.Symbol, sp.Expr]]:
    try:
        A, b = sp.linear_eq_to_matrix([sp.expand(g) for g in gs], list(zs))
    except (sp.PolynomialError, ValueError, TypeError):
        return None
    if any(z in A.free_symbols or z in b.free_symbols for z in zs):
        return None
    if A.shape[0] != A.shape[1] or sp.simplify(A.det()) == 0:
        return None
    sol = A.LUsolve(b)
    return {z: sp.simplify(sol[k]) for k, z in enumerate(zs)}


def _time_derivative(g: sp.Expr, derivs: Mapping[sp.Symbol, sp.Expr], algebraic: Set[sp.Symbol],
                     time: sp.Symbol) -> sp.Expr:
    """dg/dt along the solution: the explicit time dependence plus
    sum_u dg/du f_u over the differential unknowns.  A constraint whose
    derivative would need an algebraic unknown's derivative is outside this
    scheme (None)."""
    out = sp.diff(g, time)
    for u in g.free_symbols:
        if u in derivs:
            out += sp.diff(g, u) * derivs[u]
        elif u in algebraic and sp.diff(g, u) != 0:
            return None
    return out


def _reduce_index(residuals: List[sp.Expr], derivs: Dict[sp.Symbol, sp.Expr], algebraic: List[sp.Symbol],
                  prio: Mapping[sp.Symbol, float], order: Mapping[sp.Symbol, int], keep_always: Set[sp.Symbol],
                  time: sp.Symbol):
    """Index reduction of a semi-explicit DAE whose constraints do not
    determine its algebraic unknowns (Pantelides' criterion on the
    equation/unknown graph, Pantelides 1988, with the constraint chains of
    Mattsson and Soederlind's dummy-derivative method, 1993).

    Every implicit equation in a set that an augmenting path cannot match
    to distinct algebraic unknowns is replaced by its time derivative along
    the differential equations, until the highest derivatives match; the
    lower members of each chain stay as invariants.  Each invariant then
    demotes one differential state that it contains to an algebraic
    unknown, dropping that state's differential equation (its derivative
    is implied by the chain), with the lowest ``state_priority`` demoted
    first and irreducible states kept.  The selection is static: it holds
    while the invariants' Jacobian in the demoted states stays regular
    along the solution, as with the reference's priorities.  Returns the
    residuals (highest derivatives, then invariants) and the algebraic
    unknowns (the originals, then the demoted states)."""
    chains = [[g] for g in residuals]
    alg_set = set(algebraic)
    for _ in range(8):
        top = [c[-1] for c in chains]
        inc = [set(g.free_symbols) & alg_set for g in top]
        owner: Dict[sp.Symbol, int] = {}
        failed = None
        for e in range(len(top)):
            seen_v: Set[sp.Symbol] = set()
            seen_e: Set[int] = set()

            def augment(i):
                seen_e.add(i)
                for v in sorted(inc[i], key=lambda z: order[z]):
                    if v in seen_v:
                        continue
                    seen_v.add(v)
                    if v not in owner or augment(owner[v]):
                        owner[v] = i
                        return True
                return False

            if not augment(e):
                failed = seen_e
                break
        if failed is None:
            break
        for e in failed:
            d = _time_derivative(chains[e][-1], derivs, alg_set, time)
            if d is None:
                raise InvalidSystemError("a constraint's derivative needs the derivative of an algebraic unknown; "
                                         "this index reduction differentiates constraints on the differential "
                                         "states only")
            if d == 0:
                raise InvalidSystemError("a constraint's time derivative vanishes identically (a redundant "
                                         "or inconsistent system)")
            chains[e].append(d)
    else:
        raise InvalidSystemError("index reduction did not reach an index-1 system in 8 differentiations")
    invariants = [g for c in chains for g in c[:-1]]
    diff_states = [u for u in order if u in derivs]
    # demote the least preferred states first: lowest priority, then the
    # later declared
    ranked = sorted((u for u in diff_states if u not in keep_always), key=lambda u: (prio.get(u, 0.0), -order[u]))
    inc = [[u for u in ranked if u in g.free_symbols] for g in invariants]
    owner2: Dict[sp.Symbol, int] = {}

    def augment2(i, seen):
        for v in inc[i]:
            if v in seen:
                continue
            seen.add(v)
            if v not in owner2 or augment2(owner2[v], seen):
                owner2[v] = i
                return True
        return False

    for i in range(len(invariants)):
        if not augment2(i, set()):
            raise InvalidSystemError("no state selection satisfies the invariants of the reduced system")
    demoted = sorted(owner2, key=lambda u: order[u])
    for u in demoted:
        derivs.pop(u)
    by_state = {u: invariants[i] for u, i in owner2.items()}
    new_res = [c[-1] for c in chains] + [by_state[u] for u in demoted]
    return new_res, list(algebraic) + demoted


def structural_simplify(unknowns: Sequence[sp.Symbol], derivatives: Mapping[sp.Symbol, sp.Expr],
                        implicit: Sequence[sp.Expr], explicit: Sequence[Tuple[sp.Symbol, sp.Expr]] = (),
                        state_priority: Optional[Mapping[sp.Symbol, float]] = None,
                        irreducible: Iterable[sp.Symbol] = (), inline_linear_sccs: bool = True,
                        time: Optional[sp.Symbol] = None) -> SimplifiedSystem:
    """Index-1 structural simplification (see the module docstring).

    ``unknowns``: the declared states, in order; ``derivatives``: the
    derivative equation of each differential unknown; ``implicit``:
    residuals g of ``0 = g``; ``explicit``: definitions ``u = expr`` of
    algebraic unknowns.  Expressions may use the unknowns and any known
    symbol (parameters, constants, drivers, t)."""
    order = {u: k for k, u in enumerate(unknowns)}
    prio = dict(state_priority or {})
    time = time if time is not None else sp.Symbol("t", real=True)
    keep_always = set(irreducible)
    derivs: Dict[sp.Symbol, sp.Expr] = dict(derivatives)
    residuals: List[sp.Expr] = list(implicit)
    observed: Dict[sp.Symbol, sp.Expr] = {}
    for u, e in explicit:
        if u in derivs:
            raise InvalidSystemError(f"'{u}' has a derivative equation and an explicit definition")
        if u in keep_always or u in e.free_symbols:
            residuals.append(u - e)
        else:
            observed[u] = e

    def substitute(rule: Dict[sp.Symbol, sp.Expr]) -> None:
        for k in list(derivs):
            derivs[k] = derivs[k].xreplace(rule)
        for k in range(len(residuals)):
            residuals[k] = residuals[k].xreplace(rule)
        for k in list(observed):
            observed[k] = observed[k].xreplace(rule)

    # observed definitions may use one another: resolve them into the
    # equations so that the structure is seen in terms of unknowns
    def resolve_observed() -> None:
        for _ in range(len(observed) + 1):
            rule = dict(observed)
            changed = False
            for k in list(observed):
                new = observed[k].xreplace(rule)
                if new != observed[k]:
                    observed[k] = new
                    changed = True
            if not changed:
                break
        for k, e in observed.items():
            if k in e.free_symbols:
                raise InvalidSystemError(f"observed definition of '{k}' depends on itself")
        substitute(dict(observed))

    resolve_observed()

    # perfect aliases
    while True:
        # irreducible unknowns take no part in alias elimination
        live = {u for u in unknowns if u not in observed and u not in keep_always}
        found = None
        for k, g in enumerate(residuals):
            al = _alias(g, live)
            if al is not None:
                found = (k, al)
                break
        if found is None:
            break
        k, (a, b, s) = found

        def rank(u: sp.Symbol) -> tuple:
            return (prio.get(u, 0.0), u in derivs, -order[u])

        keep, elim = (a, b) if rank(a) >= rank(b) else (b, a)
        value = s * keep
        residuals.pop(k)
        if elim in derivs:
            f_elim = derivs.pop(elim).xreplace({elim: value})
            moved = s * f_elim   # d(keep) = s d(elim)
            if keep in derivs:
                if sp.simplify(derivs[keep].xreplace({elim: value}) - moved) != 0:
                    raise NotImplementedError(
                        f"aliased differential states '{keep}' and '{elim}' with different dynamics need "
                        "index reduction, which is not built")
            else:
                derivs[keep] = moved
        observed[elim] = value
        substitute({elim: value})

    # matching of the implicit equations to the algebraic unknowns
    algebraic = [u for u in unknowns if u not in derivs and u not in observed]
    if len(residuals) > len(algebraic):
        raise ExtraEquationsSystemError(
            f"{len(residuals)} implicit equations for {len(algebraic)} algebraic unknowns {algebraic}")
    if len(residuals) < len(algebraic):
        raise ExtraVariablesSystemError(
            f"{len(algebraic)} algebraic unknowns {algebraic} for {len(residuals)} implicit equations")
    incidence = [set(g.free_symbols) & set(algebraic) for g in residuals]
    matched = _match(incidence, algebraic)
    if matched is None:
        residuals, algebraic = _reduce_index(residuals, derivs, algebraic, prio, order, keep_always, time)
        incidence = [set(g.free_symbols) & set(algebraic) for g in residuals]
        matched = _match(incidence, algebraic)
        if matched is None:
            raise InvalidSystemError("the implicit equations stay structurally singular after index reduction")
    var_of = {e: algebraic[v] for e, v in enumerate(matched)}
    eq_of = {z: e for e, z in var_of.items()}
    # equation e depends on equation f when e contains f's unknown
    edges = [[eq_of[z] for z in incidence[e] if eq_of[z] != e] for e in range(len(residuals))]
    torn_vars: List[sp.Symbol] = []
    torn_res: List[sp.Expr] = []
    for comp in _components(len(residuals), edges):
        gs = [residuals[e] for e in comp]
        zs = [var_of[e] for e in comp]
        solved = None
        if any(z in keep_always for z in zs):
            pass   # an irreducible unknown stays a solver state
        elif len(comp) == 1:
            sol = _solve_single(gs[0], zs[0])
            solved = {zs[0]: sol} if sol is not None else None
        elif inline_linear_sccs:
            solved = _solve_linear(gs, zs)
        if solved is None:
            torn_vars.extend(zs)
            torn_res.extend(gs)
            continue
        observed.update(solved)
        for k in range(len(residuals)):
            residuals[k] = residuals[k].xreplace(solved)
        torn_res[:] = [g.xreplace(solved) for g in torn_res]
        for k in list(derivs):
            derivs[k] = derivs[k].xreplace(solved)
        for k in list(observed):
            observed[k] = observed[k].xreplace(solved)
    resolve_observed()
    torn_res = [g.xreplace(dict(observed)) for g in torn_res]
    # torn unknowns in declaration order, each with the residual it was
    # matched to
    pairs = sorted(zip(torn_vars, torn_res), key=lambda p: order[p[0]])
    diff_states = [u for u in unknowns if u in derivs]
    obs_list = [(u, observed[u]) for u in unknowns if u in observed]
    return SimplifiedSystem(differential_states=diff_states, algebraic_states=[p[0] for p in pairs],
                            dxdt={u: derivs[u] for u in diff_states}, residuals=[p[1] for p in pairs],
                            observed=obs_list)
