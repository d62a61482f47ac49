"""CellML models as :class:`~cubie_b200.symbolic.SymbolicODE` systems.

Mirrors the reference's ``load_cellml_model``
(``src/cubie/odesystems/symbolic/parsing/cellml.py:184``), which reads a
model through a vendored copy of cellmlmanip (lxml, pint, rdflib).  Those
libraries are not part of this engine; this loader reads the XML with the
standard library and converts the MathML itself:

* CellML 1.0, 1.1 and 2.0 documents (namespace picked from the root);
* components, their variables and ``initial_value`` attributes (a number,
  or in CellML 2.0 the name of a variable of the same component);
* connections (``map_components`` / ``map_variables``): connected
  variables are one model variable, named after the occurrence that
  defines it (the one with an initial value or an equation);
* MathML content markup: ``eq`` equations whose left side is a variable
  (algebraic) or ``diff`` of a variable with respect to the time variable
  (differential); ``plus minus times divide power root exp ln log abs
  floor ceiling min max rem``, the trigonometric and hyperbolic functions
  and their inverses, ``piecewise``/``piece``/``otherwise``, relations
  (``eq neq lt gt leq geq``) and ``and or xor not``; ``cn`` in plain,
  ``e-notation`` and ``integer`` forms; ``pi``, ``exponentiale``, ``true``,
  ``false``, ``infinity``, ``notanumber``.

Units: every unit resolves to a factor times a product of base units
(the SI base and derived units, prefixes, exponents, multipliers,
component-level and user-defined base units).  A model variable is held in
the units of its defining occurrence; an occurrence in another component
with compatible but different units reads it scaled by the ratio of the
factors, and equations defining it there are scaled back (the reference
converts through pint, cellmlmanip's units handling).  Units with an
offset (celsius, or a CellML 1.x unit with an ``offset`` attribute) convert
affinely, x_occ = k x_src + b; in products of units an offset describes a
difference and drops out.  Incompatible units across a connection raise
``ValueError``.

Imports (CellML 1.1 and 2.0): components and units of other documents,
found relative to the importing file; an imported component brings the
components it encapsulates (named ``<local name>__<name>``) and the
connections among them; imports may nest.  Both documents use the same
CellML version.

Removable Goldman-Hodgkin-Katz singularities (``N / (exp(U) - 1)`` with U
affine in the membrane voltage and N vanishing at U = 0) are rewritten as
(N / U) times U / (exp(U) - 1), the latter from its Taylor series near
U = 0, when ``fix_singularities`` is set (the reference's default, which
bridges the singular point by linear interpolation instead).

Not done here: ``reset`` elements (rejected with ``NotImplementedError``).

States are the variables that have a ``diff`` equation; variables with an
initial value and no equation are constants unless named in
``parameters``; algebraic equations become auxiliaries, observables when
named in ``observables``.  Names are the variables' own names, prefixed by
their component (``component__name``) only where two model variables
share a name.
"""

from __future__ import annotations

import hashlib
import warnings
import re
import xml.etree.ElementTree as ET
from pathlib import Path
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import sympy as sp

from .symbolic import TIME, SymbolicODE, _topological

MATHML = "http://www.w3.org/1998/Math/MathML"
CELLML_NS = ("http://www.cellml.org/cellml/1.0#", "http://www.cellml.org/cellml/1.1#",
             "http://www.cellml.org/cellml/2.0#")

_UNARY = {
    "exp": sp.exp, "ln": sp.log, "abs": sp.Abs, "floor": sp.floor, "ceiling": sp.ceiling,
    "sin": sp.sin, "cos": sp.cos, "tan": sp.tan, "sec": sp.sec, "csc": sp.csc, "cot": sp.cot,
    "sinh": sp.sinh, "cosh": sp.cosh, "tanh": sp.tanh, "sech": sp.sech, "csch": sp.csch, "coth": sp.coth,
    "arcsin": sp.asin, "arccos": sp.acos, "arctan": sp.atan, "arcsec": sp.asec, "arccsc": sp.acsc,
    "arccot": sp.acot, "arcsinh": sp.asinh, "arccosh": sp.acosh, "arctanh": sp.atanh,
    "arcsech": sp.asech, "arccsch": sp.acsch, "arccoth": sp.acoth, "not": sp.Not,
}
_RELATIONS = {"eq": sp.Eq, "neq": sp.Ne, "lt": sp.Lt, "gt": sp.Gt, "leq": sp.Le, "geq": sp.Ge}
_CONSTANTS = {"pi": sp.pi, "exponentiale": sp.E, "true": sp.true, "false": sp.false,
              "infinity": sp.oo, "notanumber": sp.nan}


def _local(tag: str) -> str:
    return tag.rsplit("}", 1)[-1]


def _sanitize(name: str) -> str:
    s = re.sub(r"\W", "_", name)
    return s if not s[0].isdigit() else "_" + s


class _UnionFind:
    def __init__(self):
        self.parent: Dict[Tuple[str, str], Tuple[str, str]] = {}

    def find(self, x):
        self.parent.setdefault(x, x)
        while self.parent[x] != x:
            self.parent[x] = self.parent[self.parent[x]]
            x = self.parent[x]
        return x

    def union(self, a, b):
        ra, rb = self.find(a), self.find(b)
        if ra != rb:
            self.parent[rb] = ra


class _MathML:
    """MathML content markup of one component into SymPy."""

    def __init__(self, resolve):
        self.resolve = resolve  # local variable name -> SymPy symbol

    def convert(self, el) -> sp.Expr:
        tag = _local(el.tag)
        if tag == "ci":
            return self.resolve((el.text or "").strip())
        if tag == "cn":
            return self._number(el)
        if tag in _CONSTANTS:
            return _CONSTANTS[tag]
        if tag == "apply":
            return self._apply(list(el))
        if tag == "piecewise":
            pieces = []
            otherwise = None
            for child in el:
                kind = _local(child.tag)
                if kind == "piece":
                    value, cond = list(child)
                    pieces.append((self.convert(value), self.convert(cond)))
                elif kind == "otherwise":
                    otherwise = self.convert(list(child)[0])
            pieces.append((otherwise if otherwise is not None else sp.nan, sp.true))
            return sp.Piecewise(*pieces)
        raise ValueError(f"unsupported MathML element <{tag}>")

    @staticmethod
    def _number(el) -> sp.Expr:
        kind = el.get("type", "real")
        parts = [el.text or ""] + [(c.tail or "") for c in el]
        if kind == "e-notation":
            mant, expo = (p.strip() for p in parts[:2])
            return sp.Float(f"{mant}e{expo}", 17)
        text = "".join(parts).strip()
        if kind == "integer":
            return sp.Integer(int(text))
        if kind == "rational":
            num, den = (p.strip() for p in parts[:2])
            return sp.Rational(int(num), int(den))
        value = float(text)
        return sp.Integer(int(value)) if value.is_integer() and abs(value) < 2 ** 53 else sp.Float(text, 17)

    def _apply(self, children) -> sp.Expr:
        op = _local(children[0].tag)
        qualifiers = {_local(c.tag): c for c in children[1:] if _local(c.tag) in ("degree", "logbase", "bvar")}
        args = [self.convert(c) for c in children[1:] if _local(c.tag) not in ("degree", "logbase", "bvar")]
        if op == "plus":
            return sp.Add(*args)
        if op == "minus":
            return -args[0] if len(args) == 1 else args[0] - args[1]
        if op == "times":
            return sp.Mul(*args)
        if op == "divide":
            return args[0] / args[1]
        if op == "power":
            return args[0] ** args[1]
        if op == "root":
            degree = self.convert(list(qualifiers["degree"])[0]) if "degree" in qualifiers else sp.Integer(2)
            return sp.sqrt(args[0]) if degree == 2 else args[0] ** (1 / degree)
        if op == "log":
            base = self.convert(list(qualifiers["logbase"])[0]) if "logbase" in qualifiers else sp.Integer(10)
            return sp.log(args[0]) / sp.log(base)
        if op == "rem":
            return sp.Mod(args[0], args[1])
        if op == "min":
            return sp.Min(*args)
        if op == "max":
            return sp.Max(*args)
        if op in _RELATIONS:
            rel = [_RELATIONS[op](a, b) for a, b in zip(args[:-1], args[1:])]
            return rel[0] if len(rel) == 1 else sp.And(*rel)
        if op == "and":
            return sp.And(*args)
        if op == "or":
            return sp.Or(*args)
        if op == "xor":
            return sp.Xor(*args)
        if op in _UNARY:
            return _UNARY[op](args[0])
        raise ValueError(f"unsupported MathML operator <{op}>")


# --------------------------------------------------------------------------
# units (CellML 1.0 section 5, CellML 2.0 section 9): a unit is a factor
# times a product of base units; converting between compatible units of
# connected variables scales by the ratio of their factors
# --------------------------------------------------------------------------
_PREFIX = {"yotta": 24, "zetta": 21, "exa": 18, "peta": 15, "tera": 12, "giga": 9, "mega": 6, "kilo": 3,
           "hecto": 2, "deka": 1, "deca": 1, "deci": -1, "centi": -2, "milli": -3, "micro": -6, "nano": -9,
           "pico": -12, "femto": -15, "atto": -18, "zepto": -21, "yocto": -24}


def _u(factor=1.0, **dims):
    return float(factor), {k: v for k, v in dims.items() if v}


_BUILTIN_UNITS = {
    "ampere": _u(A=1), "candela": _u(cd=1), "kelvin": _u(K=1), "kilogram": _u(kg=1), "metre": _u(m=1),
    "meter": _u(m=1), "mole": _u(mol=1), "second": _u(s=1), "gram": _u(1e-3, kg=1), "dimensionless": _u(),
    "radian": _u(), "steradian": _u(), "becquerel": _u(s=-1), "hertz": _u(s=-1), "coulomb": _u(s=1, A=1),
    "farad": _u(m=-2, kg=-1, s=4, A=2), "gray": _u(m=2, s=-2), "sievert": _u(m=2, s=-2),
    "henry": _u(m=2, kg=1, s=-2, A=-2), "joule": _u(m=2, kg=1, s=-2), "katal": _u(s=-1, mol=1),
    "liter": _u(1e-3, m=3), "litre": _u(1e-3, m=3), "lumen": _u(cd=1), "lux": _u(m=-2, cd=1),
    "newton": _u(m=1, kg=1, s=-2), "ohm": _u(m=2, kg=1, s=-3, A=-2), "pascal": _u(m=-1, kg=1, s=-2),
    "siemens": _u(m=-2, kg=-1, s=3, A=2), "tesla": _u(kg=1, s=-2, A=-1), "volt": _u(m=2, kg=1, s=-3, A=-1),
    "watt": _u(m=2, kg=1, s=-3), "weber": _u(m=2, kg=1, s=-2, A=-1), "celsius": _u(K=1),
}
# additive offsets to the base units (value_base = factor * value + offset)
_BUILTIN_OFFSET = {"celsius": 273.15}


class _Units:
    """Unit definitions in scope for one component: its own, its model's,
    and the built-in units."""

    def __init__(self, defs: Dict[str, ET.Element], cml: str, parent: Optional["_Units"] = None):
        self.defs, self.cml, self.parent = defs, cml, parent
        self._cache: Dict[str, Tuple[float, Dict[str, float]]] = {}

    def _find(self, name):
        scope = self
        while scope is not None:
            if name in scope.defs:
                return scope
            scope = scope.parent
        return None

    def resolve(self, name: str, _depth: int = 0) -> Tuple[float, Dict[str, float]]:
        if name in self._cache:
            return self._cache[name]
        scope = self._find(name)
        if scope is None:
            if name not in _BUILTIN_UNITS:
                raise ValueError(f"unknown units '{name}'")
            return _BUILTIN_UNITS[name]
        if _depth > 64:
            raise ValueError(f"units '{name}' are defined in terms of themselves")
        el = scope.defs[name]
        if el.get("base_units") == "yes":
            out = (1.0, {name: 1.0})
        else:
            factor, dims = 1.0, {}
            children = el.findall(scope.cml + "unit")
            for un in children:
                if float(un.get("offset", "0") or 0) != 0.0 and (
                        len(children) != 1 or float(un.get("exponent", "1")) != 1.0):
                    # CellML 1.x allows an offset only on a sole unit of
                    # exponent 1
                    raise ValueError(f"units '{name}': an offset needs a single unit of exponent 1")
                f, d = scope.resolve(un.get("units"), _depth + 1)
                pre = un.get("prefix", "0")
                pexp = _PREFIX[pre] if pre in _PREFIX else int(pre)
                e = float(un.get("exponent", "1"))
                m = float(un.get("multiplier", "1"))
                factor *= m * (10.0 ** pexp * f) ** e
                for k, v in d.items():
                    dims[k] = dims.get(k, 0.0) + v * e
            out = (factor, {k: v for k, v in dims.items() if abs(v) > 1e-12})
        self._cache[name] = out
        return out

    def offset(self, name: str, _depth: int = 0) -> float:
        """The additive offset of ``name`` to its base units
        (value_base = factor * value + offset): 273.15 for celsius; for a
        unit defined as one unit of exponent 1 with multiplier m, prefix p
        and offset o over a unit of factor f_r and offset o_r,
        f_r * o + o_r (CellML 1.1 section 5.2.2: the offset is added after
        the multiplier and prefix); zero for products of units, whose
        offsets describe differences."""
        scope = self._find(name)
        if scope is None:
            return _BUILTIN_OFFSET.get(name, 0.0)
        if _depth > 64:
            raise ValueError(f"units '{name}' are defined in terms of themselves")
        el = scope.defs[name]
        if el.get("base_units") == "yes":
            return 0.0
        children = el.findall(scope.cml + "unit")
        if len(children) != 1 or float(children[0].get("exponent", "1")) != 1.0:
            return 0.0
        un = children[0]
        f_r, _ = scope.resolve(un.get("units"), _depth + 1)
        o_r = scope.offset(un.get("units"), _depth + 1)
        return f_r * float(un.get("offset", "0") or 0) + o_r


def _scale(factor: float) -> sp.Expr:
    """A unit-conversion factor as a SymPy number (exact for powers of ten
    and other short decimals)."""
    r = sp.nsimplify(repr(factor), rational=True)
    return r if abs(float(r) - factor) <= 1e-15 * abs(factor) else sp.Float(repr(factor), 17)


# --------------------------------------------------------------------------
# imports (CellML 1.1 section 3, CellML 2.0 section 5): components and units
# of other documents, with the components they encapsulate
# --------------------------------------------------------------------------
XLINK = "{http://www.w3.org/1999/xlink}href"


def _encapsulation(root, cml: str) -> Dict[str, List[str]]:
    """Parent -> children of the encapsulation hierarchy."""
    children: Dict[str, List[str]] = {}

    def walk(ref):
        name = ref.get("component")
        for sub in ref.findall(cml + "component_ref"):
            children.setdefault(name, []).append(sub.get("component"))
            walk(sub)

    for grp in list(root.iter(cml + "group")) + list(root.iter(cml + "encapsulation")):
        if grp.tag == cml + "group":
            rels = [r.get("relationship") for r in grp.findall(cml + "relationship_ref")]
            if "encapsulation" not in rels:
                continue
        for ref in grp.findall(cml + "component_ref"):
            walk(ref)
    return children


def _flatten(path: Path, _seen: Tuple[str, ...] = ()):
    """The model at ``path`` with its imports resolved: ``(cml namespace,
    components {name: (element, units scope)}, connections [(c1, c2,
    [(v1, v2), ...])], resets present)``.  Imported components keep the
    local name the import gives them; the components they encapsulate are
    brought along as ``<local name>__<their name>``."""
    key = str(path.resolve())
    if key in _seen:
        raise ValueError(f"CellML import cycle through {path.name}")
    doc = ET.parse(path).getroot()
    ns = doc.tag[1:].split("}", 1)[0] if doc.tag.startswith("{") else ""
    if ns not in CELLML_NS:
        raise ValueError(f"not a CellML 1.0/1.1/2.0 model (root namespace '{ns}')")
    cml = "{" + ns + "}"
    v2 = ns.endswith("2.0#")
    model_units = _Units({u.get("name"): u for u in doc.findall(cml + "units")}, cml)
    comps: Dict[str, Tuple[ET.Element, _Units]] = {}
    conns: List[Tuple[str, str, List[Tuple[str, str]]]] = []
    resets = any(True for _ in doc.iter(cml + "reset"))
    for imp in doc.findall(cml + "import"):
        href = imp.get(XLINK)
        if not href:
            raise ValueError("CellML import without an xlink:href")
        sub_ns, sub_comps, sub_conns, sub_resets = _flatten(path.parent / href, _seen + (key,))
        resets = resets or sub_resets
        sub_doc = ET.parse(path.parent / href).getroot()
        sub_cml = "{" + sub_ns + "}"
        tree = _encapsulation(sub_doc, sub_cml)
        for iu in imp.findall(cml + ("import_units" if v2 else "units")):
            ref = iu.get("units_ref")
            defs = {u.get("name"): u for u in sub_doc.findall(sub_cml + "units")}
            if ref not in defs:
                raise ValueError(f"import of units '{ref}' from {href}: not defined there")
            model_units.defs[iu.get("name")] = defs[ref]
            # the imported definition's own references resolve among the
            # imported document's units
            model_units.defs.update({k: v for k, v in defs.items() if k not in model_units.defs})
        for ic in imp.findall(cml + ("import_component" if v2 else "component")):
            local, ref = ic.get("name"), ic.get("component_ref")
            if ref not in sub_comps:
                raise ValueError(f"import of component '{ref}' from {href}: not defined there")
            names = {ref: local}
            stack = [ref]
            while stack:
                parent = stack.pop()
                for child in tree.get(parent, []):
                    names[child] = f"{local}__{child}"
                    stack.append(child)
            for old, new in names.items():
                comps[new] = sub_comps[old]
            for c1, c2, pairs in sub_conns:
                if c1 in names and c2 in names:
                    conns.append((names[c1], names[c2], pairs))
    for comp in doc.findall(cml + "component"):
        local_units = {u.get("name"): u for u in comp.findall(cml + "units")}
        comps[comp.get("name")] = (comp, _Units(local_units, cml, model_units) if local_units else model_units)
    for conn in doc.findall(cml + "connection"):
        if v2:
            c1, c2 = conn.get("component_1"), conn.get("component_2")
        else:
            mc = conn.find(cml + "map_components")
            c1, c2 = mc.get("component_1"), mc.get("component_2")
        pairs = [(mv.get("variable_1"), mv.get("variable_2")) for mv in conn.findall(cml + "map_variables")]
        conns.append((c1, c2, pairs))
    return ns, comps, conns, resets


def load_cellml_model(path, precision=np.float32, name: Optional[str] = None,
                      parameters: Optional[Sequence[str]] = None, observables: Optional[Sequence[str]] = None,
                      fix_singularities: bool = True, voltage_variable: Optional[str] = None,
                      show_gui: bool = False) -> SymbolicODE:
    """Read a CellML file into a :class:`SymbolicODE` (arguments as the
    reference's ``load_cellml_model``).  ``parameters`` and ``observables``
    name model variables (by their model name, or ``component__name``).
    With ``fix_singularities`` (the default) removable
    Goldman-Hodgkin-Katz singularities in the membrane voltage
    (``voltage_variable``, or the state auto-detected as the reference
    detects it: a V or voltage variable of a membrane component, with a
    warning and no rewrite when none is found) are rewritten to a form that
    is finite at the singular point.  The constants editor GUI
    (``show_gui``) is not part of this engine."""
    if not isinstance(path, (str, Path)):
        raise TypeError("path must be a string or a Path")
    path = Path(path)
    if not path.exists():
        raise FileNotFoundError(str(path))
    if path.suffix != ".cellml":
        raise ValueError(f"expected a .cellml file, got '{path.name}'")
    if show_gui:
        raise NotImplementedError("the constants editor GUI is not part of cubie_b200")
    ns, comp_els, connections, resets = _flatten(path)
    cml = "{" + ns + "}"
    if resets:
        raise NotImplementedError("CellML reset rules are not supported")

    # variables per component
    comps: Dict[str, Dict[str, dict]] = {}
    uf = _UnionFind()
    for cname, (comp, units) in comp_els.items():
        vars_ = {}
        for var in comp.findall(cml + "variable"):
            vars_[var.get("name")] = {"initial": var.get("initial_value"), "units": var.get("units")}
            uf.find((cname, var.get("name")))
        comps[cname] = vars_
    for c1, c2, pairs in connections:
        for v1, v2_ in pairs:
            uf.union((c1, v1), (c2, v2_))

    # equations per component, before naming (definitions decide names)
    equations = []  # (component, kind, target local name, rhs element, time local name)
    for cname in comps:
        comp = comp_els[cname][0]
        for math in comp.findall("{%s}math" % MATHML):
            for ap in math:
                kids = list(ap)
                if _local(ap.tag) != "apply" or _local(kids[0].tag) != "eq":
                    raise ValueError(f"component '{cname}': only <apply><eq/> equations are supported")
                lhs, rhs = kids[1], kids[2]
                if _local(lhs.tag) == "ci":
                    equations.append((cname, "alg", lhs.text.strip(), rhs, None))
                elif _local(lhs.tag) == "apply" and _local(list(lhs)[0].tag) == "diff":
                    dk = list(lhs)
                    bvar = next(c for c in dk if _local(c.tag) == "bvar")
                    tname = list(bvar)[0].text.strip()
                    target = next(c for c in dk[1:] if _local(c.tag) == "ci").text.strip()
                    equations.append((cname, "ode", target, rhs, tname))
                else:
                    raise ValueError(f"component '{cname}': unsupported equation left-hand side")

    # one model variable per connected class; its defining occurrence names it
    classes: Dict[Tuple[str, str], List[Tuple[str, str]]] = {}
    for cname, vars_ in comps.items():
        for vname in vars_:
            classes.setdefault(uf.find((cname, vname)), []).append((cname, vname))
    defined = {uf.find((c, v)) for c, _, v, _, _ in equations}
    time_classes = {uf.find((c, tname)) for c, kind, _, _, tname in equations if kind == "ode"}
    if len(time_classes) > 1:
        raise ValueError("differential equations use more than one time variable")

    def source_of(members):
        for c, v in members:
            if comps[c][v]["initial"] is not None:
                return c, v
        for c, v in members:
            if uf.find((c, v)) in defined:
                for cc, _, vv, _, _ in equations:
                    if (cc, vv) == (c, v):
                        return c, v
        return members[0]

    sources = {root_: source_of(members) for root_, members in classes.items()}
    counts: Dict[str, int] = {}
    for root_, (c, v) in sources.items():
        counts[v] = counts.get(v, 0) + 1
    names = {root_: (_sanitize(v) if counts[v] == 1 else _sanitize(f"{c}__{v}")) for root_, (c, v) in sources.items()}
    for root_ in time_classes:
        names[root_] = "t"
    reserved = {"t"}
    for root_, nm in list(names.items()):
        if root_ not in time_classes and nm in reserved | {"pi", "E", "e"}:
            names[root_] = _sanitize(f"{sources[root_][0]}__{nm}")
    symbols = {root_: (TIME if root_ in time_classes else sp.Symbol(nm, real=True)) for root_, nm in names.items()}

    def initial(root_):
        c, v = sources[root_]
        val = comps[c][v]["initial"]
        if val is None:
            return None
        try:
            return float(val)
        except ValueError:  # CellML 2.0: a variable of the same component
            return initial(uf.find((c, val)))

    # unit conversion: a model variable is held in the units of its
    # defining occurrence; an occurrence in another component with other
    # (compatible) units reads it scaled by k = f_source / f_occurrence
    def unit_of(c, v):
        return comp_els[c][1].resolve(comps[c][v]["units"] or "dimensionless")

    def k(c, v):
        root_ = uf.find((c, v))
        sc, sv = sources[root_]
        if (sc, sv) == (c, v) or (comps[sc][sv]["units"] == comps[c][v]["units"]
                                  and comp_els[sc][1] is comp_els[c][1]):
            return 1.0      # the same units in the same scope: nothing to convert (or resolve)
        f_src, d_src = unit_of(*sources[root_])
        f_occ, d_occ = unit_of(c, v)
        if set(d_src) != set(d_occ) or any(abs(d_src[q] - d_occ[q]) > 1e-12 for q in d_src):
            raise ValueError(f"variable '{v}' of component '{c}' is connected to '{sources[root_][1]}' of "
                             f"'{sources[root_][0]}' with incompatible units")
        return f_src / f_occ

    def b(c, v):
        """Additive part of the conversion from the source's units to this
        occurrence's: x_occ = k x_src + (o_src - o_occ) / f_occ."""
        root_ = uf.find((c, v))
        sc, sv = sources[root_]
        if (sc, sv) == (c, v):
            return 0.0
        o_src = comp_els[sc][1].offset(comps[sc][sv]["units"] or "dimensionless")
        o_occ = comp_els[c][1].offset(comps[c][v]["units"] or "dimensionless")
        if o_src == o_occ:
            return 0.0
        f_occ, _ = unit_of(c, v)
        return (o_src - o_occ) / f_occ

    def read(c, local):
        kk, bb = k(c, local), b(c, local)
        sym = symbols[uf.find((c, local))]
        out = sym if kk == 1.0 else _scale(kk) * sym
        return out if bb == 0.0 else out + _scale(bb)

    derivatives: Dict[str, sp.Expr] = {}
    assignments: List[Tuple[sp.Symbol, sp.Expr]] = []
    states: Dict[str, float] = {}
    algebraic = set()
    for cname, kind, target, rhs, tname in equations:
        conv = _MathML(lambda local, c=cname: read(c, local))
        expr = conv.convert(rhs)
        root_ = uf.find((cname, target))
        # d(k_x x + b_x)/d(k_t t) = rhs  ->  dx/dt = (k_t / k_x) rhs;
        # k_x x + b_x = rhs  ->  x = (rhs - b_x) / k_x
        kx = k(cname, target)
        kt = k(cname, tname) if kind == "ode" else 1.0
        if kind != "ode":
            bx = b(cname, target)
            if bx != 0.0:
                expr = expr - _scale(bx)
        if kt / kx != 1.0:
            expr = _scale(kt / kx) * expr
        if kind == "ode":
            sname = names[root_]
            if sname in derivatives:
                raise ValueError(f"state '{sname}' has two differential equations")
            derivatives[sname] = expr
            states[sname] = initial(root_) if initial(root_) is not None else 0.0
            assignments.append((sp.Symbol("d" + sname, real=True), expr))
        else:
            algebraic.add(root_)
            assignments.append((symbols[root_], expr))
    param_set = set(parameters or [])
    obs_list = list(observables or [])
    params: Dict[str, float] = {}
    consts: Dict[str, float] = {}
    state_roots = {uf.find((c, t)) for c, kind, t, _, _ in equations if kind == "ode"}
    used = set()
    for _, e in assignments:
        used |= e.free_symbols
    for root_, nm in names.items():
        if root_ in time_classes or root_ in state_roots or root_ in algebraic:
            continue
        val = initial(root_)
        if val is None and symbols[root_] not in used:
            continue
        if val is None:
            raise ValueError(f"variable '{nm}' has neither a value nor an equation")
        (params if nm in param_set else consts)[nm] = val
    unknown = param_set - set(params)
    if unknown:
        raise ValueError(f"parameters {sorted(unknown)} are not constants of the model")
    params = {nm: params[nm] for nm in (parameters or [])}   # the caller's order: the rows of a parameter array
    alg_names = {names[r] for r in algebraic}
    for o in obs_list:
        if o not in alg_names:
            raise ValueError(f"observable '{o}' is not defined by an algebraic equation")
    if fix_singularities:
        vname = voltage_variable
        if vname is None:
            # a state of a component named like "membrane" whose variable
            # is V or a voltage (as the reference detects it)
            for root_ in state_roots:
                comp_name, var_name = sources[root_]
                low = var_name.lower()
                if "membrane" in comp_name.lower() and (low == "v" or "voltage" in low):
                    vname = names[root_]
                    break
            if vname is None:
                warnings.warn("fix_singularities is enabled but no membrane voltage state could be "
                              "auto-detected; skipping singularity removal. Pass voltage_variable to apply it.",
                              UserWarning, stacklevel=2)
        elif vname not in states and vname not in {a.name for a, _ in assignments}:
            raise ValueError(f"Could not resolve membrane voltage variable {vname!r} for singularity removal.")
        if vname is not None:
            Vsym = sp.Symbol(vname, real=True)
            derivatives = {k: _remove_ghk_singularities(e, Vsym) for k, e in derivatives.items()}
            assignments = [(a, _remove_ghk_singularities(e, Vsym)) for a, e in assignments]
    base = set(states) | set(params) | set(consts) | {"t"}
    assignments = _topological(assignments, base)
    # derivative assignments go last, in state order, as the string front end builds them
    aux = [(s, e) for s, e in assignments if not (s.name.startswith("d") and s.name[1:] in states)]
    ders = [(sp.Symbol("d" + s, real=True), derivatives[s]) for s in states]
    return SymbolicODE(states=states, parameters=params, constants=consts, drivers=[], observables=obs_list,
                       assignments=aux + ders, derivatives=derivatives, precision=precision,
                       name=name or path.stem,
                       source="cellml:" + hashlib.sha256(_model_bytes(path)).hexdigest() + "|P" + ",".join(params)
                       + "|O" + ",".join(obs_list))


# --------------------------------------------------------------------------
# removable Goldman-Hodgkin-Katz singularities: N(V) / (exp(U(V)) - 1) with
# U affine in the membrane voltage V and N vanishing where U does is finite
# at U = 0 but evaluates to 0 / 0 there.  It is rewritten as
# (N / U) * B(U), B(U) = U / (exp(U) - 1), with B taken from its Taylor
# series 1 - U/2 + U^2/12 - U^4/720 for |U| < 1e-2 (truncation error below
# 1e-14 relative; the direct form loses about eps / |U| there to the
# cancellation in exp(U) - 1).
# --------------------------------------------------------------------------
_GHK_SERIES_BOUND = 1e-2


def _bernoulli_factor(U: sp.Expr) -> sp.Expr:
    series = 1 - U / 2 + U ** 2 / 12 - U ** 4 / 720
    return sp.Piecewise((series, sp.Abs(U) < _GHK_SERIES_BOUND), (U / (sp.exp(U) - 1), True))


def _exp_minus_one(D: sp.Expr):
    """(c, U) with D = c (exp(U) - 1), or None."""
    D = sp.expand(D, power_exp=False, power_base=False, log=False)
    terms = sp.Add.make_args(D)
    if len(terms) != 2:
        return None
    exps = [t for t in terms if t.func is sp.exp or (t.is_Mul and any(f.func is sp.exp for f in t.args))]
    rest = [t for t in terms if t not in exps]
    if len(exps) != 1 or len(rest) != 1 or not rest[0].is_number:
        return None
    coeff, ex = exps[0].as_coeff_Mul()
    if ex.func is not sp.exp or rest[0] != -coeff:
        return None
    return coeff, ex.args[0]


def _remove_ghk_singularities(expr: sp.Expr, V: sp.Symbol) -> sp.Expr:
    def visit(e):
        if not e.args:
            return e
        e = e.func(*[visit(a) for a in e.args])
        if not e.is_Mul:
            return e
        for k, factor in enumerate(e.args):
            if not (factor.is_Pow and factor.exp == -1):
                continue
            found = _exp_minus_one(factor.base)
            if found is None:
                continue
            c, U = found
            try:
                poly = sp.Poly(U, V)
            except sp.PolynomialError:
                continue
            if poly.degree() != 1:
                continue
            V0 = sp.solve(U, V)
            if len(V0) != 1:
                continue
            num = sp.Mul(*[f for j, f in enumerate(e.args) if j != k])
            if sp.simplify(num.subs(V, V0[0])) != 0:
                continue
            return sp.cancel(num / U) / c * _bernoulli_factor(U)
        return e
    return visit(expr)


def _model_bytes(path: Path) -> bytes:
    """The document and every document it imports (the system's identity)."""
    out = path.read_bytes()
    root = ET.parse(path).getroot()
    for imp in root.iter():
        if _local(imp.tag) == "import" and imp.get(XLINK):
            out += _model_bytes(path.parent / imp.get(XLINK))
    return out
