"""Model code generation for the batched fitting kernel.

Turns a model (``Equations``, threshold, reset) into the three C snippets the
fitting kernel template needs: the state update of one step, the threshold
condition and the reset statements.  It plays the part of the reference's
``generate_modelfitting_kernel_src`` (library/modelfitting/gpu_modelfitting.py:
158-199) and of its integration schemes (experimental/codegen/
integration_schemes.py:3-43: euler, rk2, exp_euler), but works on Python's
``ast`` of each expression instead of sympy, so the generated arithmetic keeps
the expression's own evaluation order (the order the reference's numpy CPU
path evaluates it in):

* every binary operation is emitted fully parenthesised, left to right;
* every named constant and literal is rounded to the kernel's scalar type on
  its own (``float`` literals carry an ``f`` suffix and are written in hex, so
  the value is exact); nothing is folded in a wider type;
* ``x**2`` is ``x*x``, ``x**0.5`` is ``sqrt(x)``, ``x**-1`` is ``1/x`` (the
  cases numpy's power special-cases), any other power calls ``pow``.
"""
import ast
import math

import numpy as np

__all__ = ["ModelCode", "SCHEMES", "generate_model_code"]

SCHEMES = ("Euler", "RK", "exponential_Euler")

_FUNCS1 = {"exp": "exp", "log": "log", "sqrt": "sqrt", "sin": "sin", "cos": "cos", "tan": "tan",
           "tanh": "tanh", "sinh": "sinh", "cosh": "cosh", "arctan": "atan", "abs": "fabs",
           "log10": "log10", "floor": "floor", "ceil": "ceil"}
_BINOPS = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*", ast.Div: "/"}
_CMPOPS = {ast.Gt: ">", ast.Lt: "<", ast.GtE: ">=", ast.LtE: "<=", ast.Eq: "==", ast.NotEq: "!="}


class CodegenError(ValueError):
    pass


class _Emitter(object):
    """AST to C for one scalar type.  ``names`` maps identifiers to C
    expressions (state registers, the input, ``t``); other identifiers are
    looked up in ``namespace`` and must be numbers."""

    def __init__(self, scalar, names, namespace, fast=None):
        self.scalar = scalar
        self.names = names
        self.namespace = namespace
        self.fast = fast

    def copy(self):
        return _Emitter(self.scalar, dict(self.names), self.namespace, self.fast)

    def literal(self, value):
        value = float(value)
        if self.scalar == "float":
            f = float(np.float32(value))
            if math.isinf(f):
                return "(__int_as_float(0x7f800000))" if f > 0 else "(-__int_as_float(0x7f800000))"
            if math.isnan(f):
                return "(__int_as_float(0x7fffffff))"
            return "(%sf)" % f.hex() if f >= 0 else "(-%sf)" % (-f).hex()
        if math.isinf(value):
            return "(__longlong_as_double(0x7ff0000000000000LL))" if value > 0 else \
                "(-__longlong_as_double(0x7ff0000000000000LL))"
        if math.isnan(value):
            return "(__longlong_as_double(0x7ff8000000000000LL))"
        return "(%s)" % value.hex() if value >= 0 else "(-%s)" % (-value).hex()

    def func(self, name):
        c = _FUNCS1[name]
        if self.scalar == "float" and c != "fabs":
            return c + "f"
        if self.scalar == "float":
            return "fabsf"
        return c

    def expr(self, node):
        if isinstance(node, ast.Expression):
            return self.expr(node.body)
        if isinstance(node, ast.Constant):
            if isinstance(node.value, bool) or not isinstance(node.value, (int, float)):
                raise CodegenError("unsupported constant %r" % (node.value,))
            return self.literal(node.value)
        if isinstance(node, ast.Name):
            if node.id in self.names:
                return self.names[node.id]
            if node.id in self.namespace:
                v = self.namespace[node.id]
                if isinstance(v, (int, float, np.integer, np.floating)) and not isinstance(v, bool):
                    return self.literal(v)
            raise CodegenError("unknown identifier %r" % node.id)
        if isinstance(node, ast.UnaryOp):
            if isinstance(node.op, ast.USub):
                return "(-%s)" % self.expr(node.operand)
            if isinstance(node.op, ast.UAdd):
                return self.expr(node.operand)
            if isinstance(node.op, ast.Not):
                return "(!%s)" % self.expr(node.operand)
            raise CodegenError("unsupported unary operator")
        if isinstance(node, ast.BinOp):
            if isinstance(node.op, ast.Pow):
                return self.power(node)
            op = _BINOPS.get(type(node.op))
            if op is None:
                raise CodegenError("unsupported operator %s" % type(node.op).__name__)
            if op == "/" and self.fast is not None:
                k = self.fast.slot(node.right)
                if k is not None:
                    return "bg_div_fast(%s, %s, bg_y%d, bg_t%d, suspect)" % (
                        self.expr(node.left), self.expr(node.right), k, k)
            return "(%s %s %s)" % (self.expr(node.left), op, self.expr(node.right))
        if isinstance(node, ast.Call):
            if not isinstance(node.func, ast.Name) or node.func.id not in _FUNCS1 or len(node.args) != 1 \
                    or node.keywords:
                raise CodegenError("unsupported function call")
            return "%s(%s)" % (self.func(node.func.id), self.expr(node.args[0]))
        if isinstance(node, ast.Compare):
            parts = []
            left = node.left
            for op, right in zip(node.ops, node.comparators):
                c = _CMPOPS.get(type(op))
                if c is None:
                    raise CodegenError("unsupported comparison")
                parts.append("(%s %s %s)" % (self.expr(left), c, self.expr(right)))
                left = right
            return "(" + " && ".join(parts) + ")"
        if isinstance(node, ast.BoolOp):
            j = " && " if isinstance(node.op, ast.And) else " || "
            return "(" + j.join(self.expr(v) for v in node.values) + ")"
        if isinstance(node, ast.IfExp):
            return "(%s ? %s : %s)" % (self.expr(node.test), self.expr(node.body), self.expr(node.orelse))
        raise CodegenError("unsupported expression element %s" % type(node).__name__)

    def power(self, node):
        base = self.expr(node.left)
        e = node.right
        neg = isinstance(e, ast.UnaryOp) and isinstance(e.op, ast.USub) and isinstance(e.operand, ast.Constant)
        if isinstance(e, ast.Constant) or neg:
            val = float(e.operand.value if neg else e.value)
            val = -val if neg else val
            if val == 2.0:
                return "(%s * %s)" % (base, base)
            if val == 1.0:
                return base
            if val == 0.5:
                return "%s(%s)" % ("sqrtf" if self.scalar == "float" else "sqrt", base)
            if val == -1.0:
                return "(%s / %s)" % (self.literal(1.0), base)
        return "%s(%s, %s)" % ("powf" if self.scalar == "float" else "pow", base, self.expr(node.right))


def _parse(expr):
    try:
        return ast.parse(expr.strip(), mode="eval")
    except SyntaxError as e:
        raise CodegenError("cannot parse %r: %s" % (expr, e))


def _cname(name):
    return "s_" + name


class _FastDivisions(object):
    """Divisions whose divisor depends only on parameters the reset never
    assigns (and on constants) divide by a per-simulation reciprocal fixed at
    load time.  Each gets members bg_y<k> (the reciprocal, double) and
    bg_t<k> (the dividend magnitude below which the fast form may round
    differently, or a guard exponent for double).  The kernel checks those
    conditions branch-free and redoes a block with IEEE division when any
    dividend falls outside them, so results equal plain division."""

    def __init__(self, base, invariant):
        self.base = base            # emitter over the load-time names
        self.invariant = invariant
        self.keys = []

    def slot(self, node):
        for n in ast.walk(node):
            if isinstance(n, ast.Name):
                if n.id in self.invariant:
                    continue
                if n.id in self.base.names:          # state, input or time
                    return None
                if n.id not in self.base.namespace:
                    return None
            elif isinstance(n, ast.Call):
                if not isinstance(n.func, ast.Name) or n.func.id not in _FUNCS1:
                    return None
        key = self.base.expr(node)
        if key not in self.keys:
            self.keys.append(key)
        return self.keys.index(key)

    def declarations(self):
        sc = self.base.scalar
        return "".join("    double bg_y%d;\n    %s bg_t%d;\n" % (k, sc, k) for k in range(len(self.keys)))

    def setup(self):
        """Reciprocal and dividend bound of each divisor; a divisor outside
        the range where the fast forms are exact (zero, subnormal, huge,
        infinite, NaN) sends the whole simulation down the IEEE path
        (bg_exact)."""
        out = []
        for k, key in enumerate(self.keys):
            if self.base.scalar == "float":
                out.append("{ const float b = %s; bg_y%d = 1.0 / (double)b; "
                           "if (!(fabsf(b) >= 0x1p-126f && fabsf(b) <= 0x1p+126f)) bg_exact = true; "
                           "bg_t%d = (float)(0x1p-126 * fmax(1.0, fabs((double)b)) * (1.0 + 0x1p-20)); }"
                           % (key, k, k))
            else:
                out.append("{ const double b = %s; bg_y%d = 1.0 / b; "
                           "if (!(fabs(b) >= 0x1p-100 && fabs(b) <= 0x1p+100)) bg_exact = true; "
                           "bg_t%d = 0x1p-900; }" % (key, k, k))
        return "\n".join(out)


class ModelCode(object):
    """Generated snippets of one model for one scalar type.

    ``state`` lists the state variables the kernel keeps per simulation in
    their storage order (the prepared equations' differential equations,
    parameters included, without the input variable); ``update``,
    ``threshold`` and ``reset`` are C code over the registers ``s_<name>``,
    the input ``I_in`` and the time ``t``; the reset statements are selects
    on the kernel's flag ``reset_on``.  ``update_fast`` is the same step with
    divisions by invariant divisors in reciprocal form (empty when there are
    none); ``aux_decl`` and ``setup`` declare and initialise the
    reciprocals."""

    def __init__(self, state, dynamic, update, threshold, reset, scalar, scheme, uses_t, update_fast="",
                 aux_decl="", setup=""):
        self.state = list(state)
        self.dynamic = list(dynamic)
        self.update = update
        self.threshold = threshold
        self.reset = reset
        self.scalar = scalar
        self.scheme = scheme
        self.uses_t = uses_t
        self.update_fast = update_fast
        self.aux_decl = aux_decl
        self.setup = setup

    def index(self, name):
        return self.state.index(name)


def _scheme_code(eqs, em, dynamic, state, scheme):
    """Statements of one step, following integration_schemes.py:3-43."""
    sc = em.scalar
    dt = em.literal(em.namespace["dt"])
    trees = {v: _parse(eqs._string[v]).body for v in state}
    lines = []
    if scheme == "Euler":
        for v in dynamic:
            lines.append("const %s %s__tmp = %s;" % (sc, v, em.expr(trees[v])))
        for v in dynamic:
            lines.append("%s = (%s + (%s__tmp * %s));" % (_cname(v), _cname(v), v, dt))
    elif scheme == "RK":
        half = "(%s * %s)" % (em.literal(0.5), dt)
        for v in state:
            lines.append("%s %s__buf = %s;" % (sc, v, em.expr(trees[v])))
            lines.append("%s %s__half = (%s * %s__buf);" % (sc, v, half, v))
            lines.append("%s__half = (%s__half + %s);" % (v, v, _cname(v)))
        sub = em.copy()
        for v in state:
            sub.names[v] = v + "__half"
        for v in dynamic:
            lines.append("%s__buf = %s;" % (v, sub.expr(trees[v])))
            lines.append("%s = (%s + (%s * %s__buf));" % (_cname(v), _cname(v), dt, v))
    elif scheme == "exponential_Euler":
        for v in dynamic:
            z = em.copy()
            z.names[v] = em.literal(0.0)
            o = em.copy()
            o.names[v] = em.literal(1.0)
            lines.append("%s %s__B = %s;" % (sc, v, z.expr(trees[v])))
            lines.append("%s %s__A = %s;" % (sc, v, o.expr(trees[v])))
            lines.append("%s__A = (%s__A - %s__B);" % (v, v, v))
            lines.append("%s__B = (%s__B / %s__A);" % (v, v, v))
            lines.append("%s__A = (%s__A * %s);" % (v, v, dt))
        for v in dynamic:
            lines.append("%s = (%s + %s__B);" % (_cname(v), _cname(v), v))
            lines.append("%s = (%s * %s(%s__A));" % (_cname(v), _cname(v), em.func("exp"), v))
            lines.append("%s = (%s - %s__B);" % (_cname(v), _cname(v), v))
    else:
        raise CodegenError("scheme must be one of %s" % (SCHEMES,))
    return "\n".join(lines)


def _statements(text, em, state):
    """Reset statements ``x = expr`` / ``x += expr`` (one per line or ';')."""
    out = []
    for raw in text.replace(";", "\n").split("\n"):
        line = raw.split("#", 1)[0].strip()
        if not line:
            continue
        try:
            tree = ast.parse(line, mode="exec").body
        except SyntaxError as e:
            raise CodegenError("cannot parse reset %r: %s" % (line, e))
        if len(tree) != 1:
            raise CodegenError("one statement per line: %r" % line)
        st = tree[0]
        if isinstance(st, ast.Assign) and len(st.targets) == 1 and isinstance(st.targets[0], ast.Name):
            tgt, value = st.targets[0].id, em.expr(st.value)
        elif isinstance(st, ast.AugAssign) and isinstance(st.target, ast.Name):
            op = _BINOPS.get(type(st.op))
            if op is None:
                raise CodegenError("unsupported reset operator in %r" % line)
            tgt = st.target.id
            value = "(%s %s %s)" % (_cname(tgt), op, em.expr(st.value))
        else:
            raise CodegenError("unsupported reset statement %r" % line)
        if tgt not in state:
            raise CodegenError("reset assigns %r, which is not a state variable" % tgt)
        out.append(_masked(tgt, value))
    return "\n".join(out)


def _masked(tgt, value):
    """The reset runs every step as selects on `reset_on` (the kernel's
    spiking-or-refractory flag), so no branch breaks the step's chain."""
    return "%s = (reset_on ? %s : %s);" % (_cname(tgt), value, _cname(tgt))


def generate_model_code(eqs, threshold, reset, dt, input_var="I", scalar="double", scheme="Euler",
                        namespace=None):
    """Snippets for ``eqs`` with the given threshold and reset.

    ``threshold`` is a number (``Vm > value``), a string condition, or a
    ``Threshold``/``VariableThreshold``/``StringThreshold`` object; ``reset``
    a number (``Vm = value``), a string of statements, or a ``Reset``/
    ``VariableReset``/``StringReset`` object, as ``GPUModelFitting.__init__``
    accepts them (gpu_modelfitting.py:281-325)."""
    from . import groups as _g
    eqs.prepare()
    ns = dict(eqs.namespace)
    if namespace:
        ns.update(namespace)
    ns["dt"] = float(dt)
    state = [v for v in eqs._diffeq_names if v != input_var]
    dynamic = [v for v in eqs._diffeq_names_nonzero if v != input_var]
    if input_var in eqs._diffeq_names_nonzero:
        raise CodegenError("the input variable %r must be a parameter" % input_var)
    names = {v: _cname(v) for v in state}
    names[input_var] = "I_in"
    names["t"] = "t"
    em = _Emitter(scalar, names, ns)
    vm = state[0]

    def var_name(x):
        return x if isinstance(x, str) else state[x]

    if isinstance(threshold, _g.VariableThreshold):
        thr = "(%s > %s)" % (_cname(var_name(threshold.state)), _cname(var_name(threshold.threshold_state)))
    elif isinstance(threshold, _g.StringThreshold):
        thr = em.expr(_parse(threshold.expr))
    elif isinstance(threshold, _g.Threshold):
        thr = "(%s > %s)" % (_cname(var_name(threshold.state)), em.literal(threshold.threshold))
    elif isinstance(threshold, str):
        thr = em.expr(_parse(threshold))
    else:
        thr = "(%s > %s)" % (_cname(vm), em.literal(threshold))

    if reset is None:
        rst = ""
    elif isinstance(reset, _g.VariableReset):
        rst = _masked(var_name(reset.state), _cname(var_name(reset.resetvaluestate)))
    elif isinstance(reset, _g.StringReset):
        rst = _statements(reset.expr, em, state)
    elif isinstance(reset, _g.Reset):
        rst = _masked(var_name(reset.state), em.literal(reset.resetvalue))
    elif isinstance(reset, str):
        rst = _statements(reset, em, state)
    else:
        rst = _masked(vm, em.literal(reset))

    upd = _scheme_code(eqs, em, dynamic, state, scheme)
    uses_t = any("t" == n.id for v in dynamic for n in ast.walk(_parse(eqs._string[v]))
                 if isinstance(n, ast.Name))
    # parameters the reset leaves alone are fixed for a whole run
    assigned = set()
    for raw in rst.split("\n"):
        if raw.strip():
            assigned.add(raw.split("=", 1)[0].strip()[2:])
    invariant = {v for v in state if v not in dynamic and v not in assigned}
    fast = _FastDivisions(_Emitter(scalar, names, ns), invariant)
    upd_fast = _scheme_code(eqs, _Emitter(scalar, names, ns, fast), dynamic, state, scheme)
    if not fast.keys:
        upd_fast = ""
    return ModelCode(state, dynamic, upd, thr, rst, scalar, scheme, uses_t, upd_fast, fast.declarations(),
                     fast.setup())
