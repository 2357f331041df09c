"""Model equations: parsing, preparation and the exact linear propagator.

Follows Brian 1.4.4's Equations (equations.py:82-986):

* line forms ``dx/dt = expr : unit`` (differential equation),
  ``x = expr : unit`` (static equation), ``x = y`` (alias) and ``x : unit``
  (parameter, a differential equation with zero derivative),
  parse_string_equations (equations.py:222-263);
* ``prepare`` moves the membrane potential (v, V, vm or Vm) to the first
  row by a swap (equations.py:352-399) and substitutes static equations;
* ``get_linear_equations`` (stateupdater.py:253-282) evaluates the right
  hand sides at 0 and at the unit vectors in double precision, and
  ``LinearStateUpdater`` (stateupdater.py:351-392) forms
  ``A = expm(M dt)`` and ``C = -A.B + B`` on the host.
"""
import ast
import inspect
import math
import re

import numpy as np

from . import units as _units

__all__ = ["Equations", "linear_propagator"]

_diffeq_re = re.compile(r"^\s*d(\w+)\s*/\s*dt\s*=\s*(.+?)\s*:\s*(.*?)\s*$")
_eq_re = re.compile(r"^\s*(\w+)\s*=\s*(.+?)\s*:\s*(.*?)\s*$")
_alias_re = re.compile(r"^\s*(\w+)\s*=\s*(\w+)\s*$")
_param_re = re.compile(r"^\s*(\w+)\s*:\s*(.*?)\s*$")

_MATH = {"exp": math.exp, "log": math.log, "sqrt": math.sqrt, "sin": math.sin, "cos": math.cos,
         "tan": math.tan, "tanh": math.tanh, "sinh": math.sinh, "cosh": math.cosh, "abs": abs,
         "arctan": math.atan, "pi": math.pi, "e": math.e, "Inf": float("inf"), "inf": float("inf")}


def _identifiers(expr):
    try:
        tree = ast.parse(expr, mode="eval")
    except SyntaxError:
        return set(re.findall(r"\b[A-Za-z_]\w*\b", expr))
    return {n.id for n in ast.walk(tree) if isinstance(n, ast.Name)}


def _picklable_namespace(ns):
    """The entries of a captured namespace that model code can use and that
    pickle: numbers, arrays and strings (a caller's modules and functions
    are left out)."""
    keep = (int, float, complex, bool, str, np.number, np.ndarray)
    return {k: v for k, v in ns.items() if isinstance(v, keep) and not k.startswith("__")}


def _caller_namespace(level):
    frame = inspect.currentframe()
    for _ in range(level + 1):
        frame = frame.f_back if frame is not None else None
    ns = {}
    if frame is not None:
        ns.update(frame.f_globals)
        ns.update(frame.f_locals)
    return ns


class Equations(object):
    """Set of model equations (equations.py:82).

    ``Equations(expr, level=0, **kwds)``: names in ``expr`` that are not
    variables are looked up in ``kwds`` if given, else in the caller's
    namespace (``level`` frames up), as in the reference."""

    def __getstate__(self):
        return dict(self.__dict__, _namespace=_picklable_namespace(self._namespace))

    def __init__(self, expr="", level=0, **kwds):
        self._diffeq_names = []
        self._diffeq_names_nonzero = []
        self._eq_names = []
        self._alias = {}
        self._string = {}
        self._units = {}
        self._Vm = None
        self._prepared = False
        if kwds:
            self._namespace = dict(kwds)
        else:
            self._namespace = _caller_namespace(level + 1)
        if expr:
            self._parse(expr)

    # ------------------------------------------------------------------ parse
    def _parse(self, expr):
        for raw in expr.split("\n"):
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            m = _diffeq_re.match(line)
            if m:
                self._add_diffeq(m.group(1), m.group(2), m.group(3))
                continue
            m = _alias_re.match(line)
            if m:
                self._alias[m.group(1)] = m.group(2)
                self._eq_names.append(m.group(1))
                self._string[m.group(1)] = m.group(2)
                self._units[m.group(1)] = ""
                continue
            m = _eq_re.match(line)
            if m:
                self._eq_names.append(m.group(1))
                self._string[m.group(1)] = m.group(2)
                self._units[m.group(1)] = m.group(3)
                continue
            m = _param_re.match(line)
            if m:
                self.add_param(m.group(1), m.group(2))
                continue
            raise ValueError("Cannot parse equation line: %r" % raw)

    def _add_diffeq(self, name, expr, unit, nonzero=True):
        if name in self._string:
            raise ValueError("Variable %s defined twice" % name)
        self._diffeq_names.append(name)
        if nonzero:
            self._diffeq_names_nonzero.append(name)
        self._string[name] = expr
        self._units[name] = unit

    def add_param(self, name, unit=""):
        """Parameter: a state variable with zero derivative (equations.py:334)."""
        self._add_diffeq(name, "0", unit, nonzero=False)

    def __add__(self, other):
        res = Equations.__new__(Equations)
        res.__dict__ = {k: (list(v) if isinstance(v, list) else dict(v) if isinstance(v, dict) else v)
                        for k, v in self.__dict__.items()}
        for n in other._diffeq_names:
            res._add_diffeq(n, other._string[n], other._units[n], n in other._diffeq_names_nonzero)
        for n in other._eq_names:
            res._eq_names.append(n)
            res._string[n] = other._string[n]
            res._units[n] = other._units[n]
        res._alias.update(other._alias)
        ns = dict(other._namespace)
        ns.update(self._namespace)
        res._namespace = ns
        res._prepared = False
        return res

    # ----------------------------------------------------------------- access
    def __len__(self):
        return len(self._diffeq_names)

    def get_Vm(self):
        if self._Vm:
            return self._Vm
        guesses = [v for v in self._diffeq_names if v in ("v", "V", "vm", "Vm")]
        return guesses[0] if len(guesses) == 1 else None

    def prepare(self):
        """Vm first (swap), static equations substituted (equations.py:352-385)."""
        if self._prepared:
            return
        vm = self.get_Vm()
        if vm:
            i = self._diffeq_names.index(vm)
            self._diffeq_names[0], self._diffeq_names[i] = self._diffeq_names[i], self._diffeq_names[0]
        # substitute static equations (dependencies first) into the diffeqs
        order = self._static_order()
        for name in order:
            pat = re.compile(r"\b" + re.escape(name) + r"\b")
            for other in order[order.index(name) + 1:] + self._diffeq_names:
                self._string[other] = pat.sub("(" + self._string[name] + ")", self._string[other])
        self._prepared = True

    def _static_order(self):
        deps = {n: _identifiers(self._string[n]) & set(self._eq_names) for n in self._eq_names}
        order, seen = [], set()

        def visit(n, stack=()):
            if n in seen:
                return
            if n in stack:
                raise ValueError("Cyclic static equations")
            for d in deps[n]:
                visit(d, stack + (n,))
            seen.add(n)
            order.append(n)

        for n in self._eq_names:
            visit(n)
        return order

    @property
    def namespace(self):
        ns = dict(_MATH)
        for k in _units.__all__:
            ns.setdefault(k, getattr(_units, k))
        for k, v in self._namespace.items():
            if isinstance(v, (int, float, np.floating, np.integer)) and not isinstance(v, bool):
                ns[k] = float(v)
            elif callable(v) and k in _MATH:
                pass
            elif k not in ns:
                ns[k] = v
        return ns

    def free_identifiers(self, name):
        return _identifiers(self._string[name])

    def is_time_dependent(self):
        return any("t" in _identifiers(self._string[n]) for n in self._diffeq_names_nonzero)

    def is_linear(self):
        """All right-hand sides affine in the state variables, no time
        dependence, no external functions (equations.py:620-632)."""
        self.prepare()
        if self.is_time_dependent():
            return False
        import sympy
        syms = {n: sympy.Symbol("s_" + n) for n in self._diffeq_names}
        ns = self.namespace
        for name in self._diffeq_names_nonzero:
            expr = self._string[name]
            ids = _identifiers(expr)
            for i in ids:
                if i not in syms and i in ns and callable(ns[i]) and i not in ("exp", "log", "sqrt"):
                    return False
            local = {}
            for i in ids:
                if i in syms:
                    local[i] = syms[i]
                elif i in ns and isinstance(ns[i], float):
                    local[i] = sympy.Float(ns[i], 17)
                elif i in ("exp", "log", "sqrt", "sin", "cos", "tanh"):
                    local[i] = getattr(sympy, i)
                else:
                    return False
            try:
                f = sympy.sympify(expr, locals=local)
            except Exception:
                return False
            for s in syms.values():
                d = sympy.diff(f, s)
                if d.free_symbols & set(syms.values()):
                    return False
        return True

    def _compile(self, name):
        return compile(self._string[name], "<eq %s>" % name, "eval")

    def apply(self, name, values):
        """Right-hand side of `name` evaluated in double precision."""
        ns = self.namespace
        ns.update(values)
        return float(eval(self._compile(name), ns))

    def get_linear_equations(self):
        """M, B with dX/dt = M(X - B) (stateupdater.py:253-282)."""
        self.prepare()
        names = self._diffeq_names
        n = len(names)
        AB = np.zeros((n, 1))
        d = dict.fromkeys(names, 0.0)
        for i, var in enumerate(names):
            AB[i] = -self.apply(var, d)
        M = np.zeros((n, n))
        for i in range(n):
            for j in range(n):
                d[names[j]] = 0.0
            d[names[i]] = 1.0
            for j, var in enumerate(names):
                M[j, i] = self.apply(var, d) + AB[j, 0]
        B = np.linalg.solve(M, AB)
        return M, B


def linear_propagator(eqs, dt):
    """A = expm(M dt), C = -A.B + B (stateupdater.py:351-392); falls back to
    the 100-step Euler product when M is singular (stateupdater.py:284-314)."""
    import scipy.linalg
    try:
        M, B = eqs.get_linear_equations()
        A = scipy.linalg.expm(M * dt)
        C = -np.dot(A, B) + B
    except np.linalg.LinAlgError:
        names = eqs._diffeq_names
        n = len(names)
        AB = np.zeros((n, 1))
        dd = dict.fromkeys(names, 0.0)
        for i, var in enumerate(names):
            AB[i] = -eqs.apply(var, dd)
        M = np.zeros((n, n))
        for i in range(n):
            for j in range(n):
                dd[names[j]] = 0.0
            dd[names[i]] = 1.0
            for j, var in enumerate(names):
                M[j, i] = eqs.apply(var, dd) + AB[j, 0]
        steps = 100
        deltat = dt / steps
        E = np.eye(n) + deltat * M
        A = np.eye(n)
        C = np.zeros((n, 1))
        for _ in range(steps):
            A, C = np.dot(E, A), np.dot(E, C) - AB * deltat
    return np.ascontiguousarray(A, dtype=np.float64), np.ascontiguousarray(C.reshape(-1), dtype=np.float64)
