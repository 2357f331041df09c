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

    def __init__(self, scalar, names, namespace):
        self.scalar = scalar
        self.names = names
        self.namespace = namespace

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


class ModelCode(object):
    """Generated snippets of one model for one scalar type.

    ``state`` lists the state variables the kernel keeps per simulation in
    their storage order (the prepared equations' differential equations,
    parameters included, without the input variable); ``update``,
    ``threshold`` and ``reset`` are C code over the registers ``s_<name>``,
    the input ``I_in`` and the time ``t``."""

    def __init__(self, state, dynamic, update, threshold, reset, scalar, scheme, uses_t):
        self.state = list(state)
        self.dynamic = list(dynamic)
        self.update = update
        self.threshold = threshold
        self.reset = reset
        self.scalar = scalar
        self.scheme = scheme
        self.uses_t = uses_t

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
        sub = _Emitter(sc, dict(em.names), em.namespace)
        for v in state:
            sub.names[v] = v + "__half"
        for v in dynamic:
            lines.append("%s__buf = %s;" % (v, sub.expr(trees[v])))
            lines.append("%s = (%s + (%s * %s__buf));" % (_cname(v), _cname(v), dt, v))
    elif scheme == "exponential_Euler":
        for v in dynamic:
            z = _Emitter(sc, dict(em.names), em.namespace)
            z.names[v] = em.literal(0.0)
            o = _Emitter(sc, dict(em.names), em.namespace)
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
        out.append("%s = %s;" % (_cname(tgt), value))
    return "\n".join(out)


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
        rst = "%s = %s;" % (_cname(var_name(reset.state)), _cname(var_name(reset.resetvaluestate)))
    elif isinstance(reset, _g.StringReset):
        rst = _statements(reset.expr, em, state)
    elif isinstance(reset, _g.Reset):
        rst = "%s = %s;" % (_cname(var_name(reset.state)), em.literal(reset.resetvalue))
    elif isinstance(reset, str):
        rst = _statements(reset, em, state)
    else:
        rst = "%s = %s;" % (_cname(vm), em.literal(reset))

    upd = _scheme_code(eqs, em, dynamic, state, scheme)
    uses_t = any("t" == n.id for v in dynamic for n in ast.walk(_parse(eqs._string[v]))
                 if isinstance(n, ast.Name))
    return ModelCode(state, dynamic, upd, thr, rst, scalar, scheme, uses_t)
