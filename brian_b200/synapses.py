"""Synapses (synapses/synapses.py:43-1058 of Brian 1.4.4).

What runs on the engine:

* ``model``: static synaptic variables (``w : 1``, ``w : volt``) and
  event-driven linear equations (``dApre/dt = -Apre/taupre : 1
  (event-driven)``, any ``a*x + b`` with constant a, b), whose exact
  solution is applied at each event before the code, with ``lastupdate``
  set to t after it (synapses.py:179-187, 257-296).  Clock-driven synaptic
  equations raise NotImplementedError.
* ``pre``: one code string.  Lines ``x += e`` / ``x -= e`` adding a
  synaptic variable, a constant or their product to a postsynaptic
  variable run on the engine's static kernels; anything else (assignments
  and ``+= -= *= /=`` of synaptic or postsynaptic variables, expressions
  with ``clip``, ``exp``, ``abs``, ``sqrt``, ``t``, ``x_pre`` reads) is
  compiled into a generated kernel, which runs the whole code for each
  event of a target in queue order.
* ``post``: one code string changing synaptic variables, run for every
  synapse of a target that spiked in the step, after the presynaptic
  events (the post queue, delay 0).  Lists of several codes raise
  NotImplementedError, as do postsynaptic codes that change neuron
  variables.
* Synapse creation as the reference's ``S[i, j] = True | int | float |
  'condition'`` (synapses.py:583-723), ``connect_random`` and
  ``connect_one_to_one``; synapse indices are allocated in the same order
  (row by row).
* Presynaptic delays: ``S.delay[...] = seconds`` is stored in bins as
  ``int(value / dt)`` (synapticvariable.py:161).

Event timing follows the SpikeQueue (spikequeue.py:69-330) and the
schedule (network.py:365-380, 472-483): the queue is filled in the
connections slot with the spikes of step s, at the row due d steps later,
and read in the 'synapses' slot (after the connections, before the resets)
before ``next()`` advances it, so an event of delay d bins is applied at
step s + d.  Events reaching one target in one step are applied in queue
order: insertion step, then source index, then synapse index.  A target
variable that a DelayConnection also feeds on the same neurons is refused
by the engine (it adds the connection's due row after the Synapses, the
reference before).  The reference applies repeated targets
in rounds over numpy's default (unstable) argsort (synapses.py:502-516),
which orders ties by numpy's sort implementation; queue order is the order
a stable sort gives.  ``exp`` in generated synaptic code is the engine's
own ``bg_exp`` (csrc/bg_expfn.h), the same operations on the GPU and in
the CPU restatement, within one ulp of the C library's exp.
"""
import ast
import re
import sys

import numpy as np

from ._lib import EngineBound
from .groups import NeuronGroup, Subgroup

__all__ = ["Synapses"]


def _split(code):
    """Statements of a code string, one per line or ';'."""
    out = []
    for ln in code.replace(";", "\n").split("\n"):
        ln = ln.split("#", 1)[0].strip()
        if ln:
            out.append(ln)
    return out


def _flat(code):
    if "\n" in code:
        return [ln.strip() for ln in code.split("\n") if ln.strip()]
    return [ln.strip() for ln in code.split(";") if ln.strip()]


def _caller_namespace(level):
    """Globals and locals of the first frame outside this module, `level`
    frames further out (the namespace the reference's code strings see)."""
    frame = sys._getframe(1)
    while frame is not None and frame.f_globals is globals():
        frame = frame.f_back
    for _ in range(level):
        frame = frame.f_back
    ns = dict(frame.f_globals)
    ns.update(frame.f_locals)
    return ns


def _group_range(x, G):
    """Indices (relative to the group G) of an int, slice, array or subgroup
    (synapses.py:1100-1111 neuron_indexes)."""
    if isinstance(x, (NeuronGroup, Subgroup)):
        owner = x._owner
        if owner is not G._owner:
            raise ValueError("subgroup of another group")
        lo = x._origin - G._origin
        if lo < 0 or lo + len(x) > len(G):
            raise ValueError("subgroup outside the group")
        return np.arange(lo, lo + len(x), dtype=np.int64)
    if isinstance(x, slice):
        return np.arange(len(G), dtype=np.int64)[x]
    if np.isscalar(x):
        return np.array([int(x)], dtype=np.int64)
    return np.asarray(x, dtype=np.int64).ravel()


class _SynapticVariable(object):
    """``S.w[...]`` (synapticvariable.py): synapse indices, (i, j) pairs of
    neuron indices, or a string of i, j (and rand()) as the index of a
    write."""

    def __init__(self, S, name):
        self._S, self._name = S, name

    def _get(self):
        S = self._S
        b = S.__dict__.get("_binding")
        if b is not None and S._coded:
            # a variable the synaptic code changes lives on the engine
            S._vars[self._name] = b.read_synapse_var(S, S._names.index(self._name))
        return S._vars[self._name]

    def __array__(self, dtype=None, copy=None):
        a = self._get()
        return a.astype(dtype) if dtype is not None else a.copy()

    def __len__(self):
        return len(self._S)

    def __getitem__(self, key):
        return self._get()[self._S._synapse_index(key)]

    def __setitem__(self, key, value):
        S = self._S
        idx = S._synapse_index(key)
        if isinstance(value, str):
            value = S._eval_string(value, idx)
        self._get()
        S._vars[self._name][idx] = np.asarray(value, dtype=np.float64)
        S._changed(var=self._name)


class _SynapticDelay(_SynapticVariable):
    """Presynaptic delays, stored in bins as int(value / dt)
    (synapticvariable.py:143-161); read back in seconds."""

    def _get(self):
        return self._S._delay * self._S.clock.dt

    def __setitem__(self, key, value):
        S = self._S
        idx = S._synapse_index(key)
        if isinstance(value, str):
            value = S._eval_string(value, idx)
        steps = np.array(np.asarray(value, dtype=np.float64) / S.clock.dt, dtype=np.int16)
        S._delay[idx] = steps
        S._changed(delays=True)


class Synapses(EngineBound):
    def __init__(self, source, target=None, model=None, pre=None, post=None, max_delay=0.0, level=0, clock=None,
                 code_namespace=None, **kwds):
        target = target or source
        if source.clock is not target.clock:
            raise ValueError("Source and target groups must have the same clock")
        if isinstance(post, (list, tuple)):
            if len(post) != 1:
                raise NotImplementedError("several postsynaptic codes are not run by the engine")
            post = post[0]
        if isinstance(pre, (list, tuple)):
            if len(pre) != 1:
                raise NotImplementedError("several presynaptic codes are not run by the engine")
            pre = pre[0]
        if kwds.get("method") is not None or kwds.get("implicit") or kwds.get("order", 1) != 1:
            raise NotImplementedError("synaptic differential equations are not run by the engine")
        object.__setattr__(self, "_vars", {})
        self.source, self.target = source, target
        self.clock = clock or source.clock
        self.max_delay = float(max_delay)
        ns = _caller_namespace(level)
        if code_namespace:
            ns.update(code_namespace)
        self._names, self._ed = self._parse_model(model or "", ns)
        # lastupdate (synapses.py:179-187): with event-driven variables or
        # when a code names it; set to t after each pre and post code
        uses_lu = re.search(r"\blastupdate\b", (pre or "") + "\n" + (post or "")) is not None
        if self._ed or uses_lu:
            self._names.append("lastupdate")
        for n in self._names:
            self._vars[n] = np.zeros(0)
        self.presynaptic = np.zeros(0, dtype=np.int64)
        self.postsynaptic = np.zeros(0, dtype=np.int64)
        self._delay = np.zeros(0, dtype=np.int16)
        self._coded = bool(post) or bool(self._ed) or uses_lu
        self._ops = []
        if not self._coded:
            try:
                self._ops = self._parse_pre(pre or "", ns)
            except NotImplementedError:
                self._coded = True
        self._code = self._generate(pre or "", post or "", ns) if self._coded else None
        self._binding = None
        self._iscompressed = False

    # ---------------------------------------------------------------- model
    def _parse_model(self, model, ns):
        """Static variables ('w : unit') and event-driven linear equations
        ('dx/dt = a*x + b : unit (event-driven)', a and b constants), whose
        exact solution is applied at each event (synapses.py:257-296):
        x = -b/a + exp(a (t - lastupdate)) (x + b/a), or x + b (t -
        lastupdate) for a = 0.  Returns the names and [(name, a, b)]."""
        names, ed = [], []
        for line in _flat(model):
            line = line.split("#")[0].strip()
            if not line:
                continue
            m = re.match(r"^d(\w+)\s*/\s*dt\s*=\s*(.+?)\s*:\s*([^()]*?)\s*\(\s*event-driven\s*\)\s*$", line)
            if m:
                var, rhs = m.group(1), m.group(2)
                ed.append((var,) + self._affine(var, rhs, ns, line))
                names.append(var)
                continue
            m = re.match(r"^(\w+)\s*:\s*[\w\s\*/\.]+$", line)
            if not m or "=" in line:
                raise NotImplementedError("synaptic equations other than static variables and event-driven "
                                          "linear equations are not run by the engine: %r" % line)
            names.append(m.group(1))
        for n in names:
            if n in ("delay", "delay_pre", "delay_post", "lastupdate"):
                raise NotImplementedError("synaptic variable %r" % n)
        return names, ed

    @staticmethod
    def _affine(var, rhs, ns, line):
        """(a, b) of rhs = a*var + b, from rhs at var = 0 and var = 1 (the
        reference's AffineFunction test, synapses.py:262-273)."""
        tree = ast.parse(rhs, mode="eval")
        env = {}
        for node in ast.walk(tree):
            if isinstance(node, ast.Name) and node.id != var:
                v = ns.get(node.id)
                if not (np.isscalar(v) and isinstance(v, (int, float, np.integer, np.floating))):
                    raise TypeError("Cannot turn equation for %s into event-driven code: %r" % (var, line))
                env[node.id] = float(v)
        code = compile(tree, "<event-driven>", "eval")
        f = lambda x: float(eval(code, {"__builtins__": {}}, dict(env, **{var: x})))
        b = f(0.0)
        a = f(1.0) - b
        if abs(f(2.0) - (2.0 * a + b)) > 1e-9 * max(1.0, abs(a), abs(b)):
            raise TypeError("Cannot turn equation for %s into event-driven code: %r" % (var, line))
        return a, b

    def _generate(self, pre, post, ns):
        """C bodies of the pre and post codes for the engine (over X(slot),
        SV(var), PRE(k), T): the event-driven updates, the code's
        statements in order, then lastupdate = t.  Returns (pre, post,
        target variables of the slots, the written ones, source
        variables)."""
        from .codegen import _Emitter, CodegenError
        tvars = self.target._owner.var_index
        svars = self.source._owner.var_index
        slots, writes, pres = [], [], []

        def slot(var):
            if var not in slots:
                if len(slots) == 4:
                    raise NotImplementedError("synaptic code using more than four postsynaptic variables")
                slots.append(var)
            return "X(%d)" % slots.index(var)

        def pre_slot(var):
            if var not in pres:
                if len(pres) == 4:
                    raise NotImplementedError("synaptic code reading more than four presynaptic variables")
                pres.append(var)
            return "PRE(%d)" % pres.index(var)

        def resolve(name):
            if name in self._names:
                return "SV(%d)" % self._names.index(name)
            if name == "t":
                return "T"
            if name.endswith("_post") and name[:-5] in tvars and isinstance(name[:-5], str):
                return slot(name[:-5])
            if name.endswith("_pre") and name[:-4] in svars and isinstance(name[:-4], str):
                return pre_slot(name[:-4])
            if name in tvars and isinstance(name, str):
                return slot(name)
            return None

        class _SynEmitter(_Emitter):
            def expr(self, node):
                if isinstance(node, ast.Call) and isinstance(node.func, ast.Name) and not node.keywords:
                    f, args = node.func.id, node.args
                    if f == "clip" and len(args) == 3:
                        return "bg_clip(%s, %s, %s)" % tuple(self.expr(x) for x in args)
                    if f == "exp" and len(args) == 1:
                        return "bg_exp(%s)" % self.expr(args[0])
                    if f in ("abs", "fabs") and len(args) == 1:
                        return "fabs(%s)" % self.expr(args[0])
                    if f == "sqrt" and len(args) == 1:
                        return "sqrt(%s)" % self.expr(args[0])
                    raise CodegenError("function %r in synaptic code" % f)
                return _Emitter.expr(self, node)

            def power(self, node):
                out = _Emitter.power(self, node)
                if out.startswith("pow("):
                    raise CodegenError("powers other than 2, 1, 0.5 and -1 in synaptic code")
                return out

        def emitter(code):
            names = {}
            for line in _split(code):
                for node in ast.walk(ast.parse(line, mode="exec")):
                    if isinstance(node, ast.Name):
                        c = resolve(node.id)
                        if c is not None:
                            names[node.id] = c
            return _SynEmitter("double", names, ns)

        def body(code, is_post):
            em = emitter(code)
            out = []
            lu = self._names.index("lastupdate") if "lastupdate" in self._names else None
            for var, a, b in self._ed:
                v = "SV(%d)" % self._names.index(var)
                dt_ = "(T - SV(%d))" % lu
                if a == 0.0:
                    out.append("%s = (%s + (%s * %s));" % (v, v, em.literal(b), dt_))
                elif b == 0.0:
                    out.append("%s = (%s * bg_exp((%s * %s)));" % (v, v, em.literal(a), dt_))
                else:
                    out.append("%s = (%s + (bg_exp((%s * %s)) * (%s + %s)));"
                               % (v, em.literal(-b / a), em.literal(a), dt_, v, em.literal(b / a)))
            for line in _split(code):
                st = ast.parse(line, mode="exec").body
                if len(st) != 1:
                    raise NotImplementedError("synaptic statement %r" % line)
                st = st[0]
                if isinstance(st, ast.Assign) and len(st.targets) == 1 and isinstance(st.targets[0], ast.Name):
                    name, value = st.targets[0].id, None
                elif isinstance(st, ast.AugAssign) and isinstance(st.target, ast.Name):
                    name, value = st.target.id, st.op
                else:
                    raise NotImplementedError("synaptic statement %r" % line)
                if name.endswith("_pre") and name[:-4] in svars:
                    raise ValueError('The synaptic code "%s" changes the value of a pre-synaptic variable.' % line)
                lhs = resolve(name)
                if lhs is None or lhs == "T" or lhs.startswith("PRE"):
                    raise NotImplementedError("synaptic code assigns %r: %r" % (name, line))
                if lhs.startswith("X("):
                    if is_post:
                        raise NotImplementedError("postsynaptic code that changes a neuron variable: %r" % line)
                    var = tvars[name[:-5] if name.endswith("_post") else name]
                    if var not in writes:
                        writes.append(var)
                try:
                    rhs = em.expr(st.value)
                except CodegenError as e:
                    raise NotImplementedError("synaptic code %r: %s" % (line, e))
                if value is None:
                    out.append("%s = %s;" % (lhs, rhs))
                else:
                    ops = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*", ast.Div: "/"}
                    if type(value) not in ops:
                        raise NotImplementedError("synaptic statement %r" % line)
                    out.append("%s = (%s %s %s);" % (lhs, lhs, ops[type(value)], rhs))
            if lu is not None:
                out.append("SV(%d) = T;" % lu)
            return "\n".join("        " + x for x in out)

        pre_c = body(pre, False)
        post_c = body(post, True) if post.strip() else ""
        return pre_c, post_c, [int(tvars[v]) for v in slots], [int(w) for w in writes], [int(svars[v]) for v in pres]

    def _parse_pre(self, pre, ns):
        """Lines 'x += e' / 'x -= e' -> (target var index, subtract, synaptic
        variable name or None, constant factor)."""
        ops = []
        tvars = self.target._owner.var_index
        for line in _flat(pre):
            if re.search(r"\b\w+_pre\s*[-+*/]?=", line):
                raise ValueError('The synaptic code "%s" changes the value of a pre-synaptic variable.' % line)
            m = re.match(r"^(\w+)\s*(\+=|-=)\s*(.+)$", line)
            if not m:
                raise NotImplementedError("presynaptic code other than 'x += e' / 'x -= e': %r" % line)
            lhs, op, rhs = m.groups()
            name = lhs[:-5] if lhs.endswith("_post") and lhs[:-5] in tvars else lhs
            if name in self._names or name not in tvars or not isinstance(name, str):
                raise NotImplementedError("presynaptic code must modify a postsynaptic variable: %r" % line)
            var, c = self._term(ast.parse(rhs.strip(), mode="eval").body, ns, line)
            ops.append((int(tvars[name]), op == "-=", var, c))
        if len(ops) > 4:
            raise NotImplementedError("more than four presynaptic statements")
        return ops

    def _term(self, node, ns, line):
        """(synaptic variable or None, constant) of e = c, w, c*w, w*c, -e."""
        if isinstance(node, ast.UnaryOp) and isinstance(node.op, ast.USub):
            var, c = self._term(node.operand, ns, line)
            return var, -c
        if isinstance(node, ast.Constant) and isinstance(node.value, (int, float)):
            return None, float(node.value)
        if isinstance(node, ast.Name):
            if node.id in self._names:
                return node.id, 1.0
            if node.id in ns and np.isscalar(ns[node.id]):
                return None, float(ns[node.id])
        if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Mult):
            a = self._term(node.left, ns, line)
            b = self._term(node.right, ns, line)
            if (a[0] is None) != (b[0] is None):
                var = a[0] if a[0] is not None else b[0]
                c = b[1] if a[0] is not None else a[1]
                if (a[0] is not None and a[1] != 1.0) or (b[0] is not None and b[1] != 1.0):
                    raise NotImplementedError("presynaptic expression: %r" % line)
                return var, c
        raise NotImplementedError("presynaptic expression other than c, w, c*w: %r" % line)

    # ------------------------------------------------------------ creation
    def __len__(self):
        return len(self.presynaptic)

    def _check_open(self):
        if self._iscompressed:
            raise AttributeError("Synapses cannot be added after they have been run")

    def __setitem__(self, key, value):
        """Create synapses (synapses.py:583-723).  Synapses are added, never
        replaced: S[1,2]=True twice makes two."""
        self._check_open()
        if not isinstance(key, tuple):
            raise AttributeError("Synapses behave as 2-D objects")
        pre, post = key
        pre_idx = _group_range(pre, self.source)
        post_idx = _group_range(post, self.target)
        if len(pre_idx) and pre_idx[-1] >= len(self.source):
            raise ValueError("Presynaptic index %d greater than number of presynaptic neurons (%d)"
                             % (pre_idx[-1], len(self.source)))
        if len(post_idx) and post_idx[-1] >= len(self.target):
            raise ValueError("Postsynaptic index %d greater than number of postsynaptic neurons (%d)"
                             % (post_idx[-1], len(self.target)))
        if isinstance(value, float):
            self.connect_random(pre, post, value)
            return
        if isinstance(value, (bool, int, np.integer)) and not isinstance(value, str):
            if value is False:
                raise ValueError("Synapses cannot be deleted")
            k = 1 if value is True else int(value)
            # row-major over (pre, post), the whole block repeated k times
            P, Q = np.meshgrid(pre_idx, post_idx, indexing="ij")
            pres = np.tile(P.ravel(), k)
            posts = np.tile(Q.ravel(), k)
            self._create(pres, posts)
            return
        if isinstance(value, str):
            # the condition is evaluated row by row with i a scalar and j the
            # post indices; subgroup indices are relative to the subgroup
            pre_shift = pre_idx[0] if isinstance(pre, (NeuronGroup, Subgroup)) and len(pre_idx) else 0
            post_shift = post_idx[0] if isinstance(post, (NeuronGroup, Subgroup)) and len(post_idx) else 0
            code = re.sub(r"\brand\(\)", "rand(n)", value)
            code = re.sub(r"\brandn\(\)", "randn(n)", code)
            ns = _caller_namespace(0)
            ns.update({"j": post_idx - post_shift, "n": len(post_idx), "rand": np.random.rand,
                       "randn": np.random.randn})
            pres, posts = [], []
            for i in pre_idx:
                ns["i"] = int(i) - pre_shift
                res = np.asarray(eval(code, ns))
                if res.dtype.kind == "f":
                    res = np.random.rand(len(post_idx)) < res
                res = np.broadcast_to(res, (len(post_idx),))
                sel = np.nonzero(res)[0]
                pres.append(np.full(len(sel), i, dtype=np.int64))
                posts.append(post_idx[sel])
            self._create(np.concatenate(pres) if pres else np.zeros(0, np.int64),
                         np.concatenate(posts) if posts else np.zeros(0, np.int64))
            return
        raise NotImplementedError("synapse creation from %r" % type(value))

    def connect_random(self, pre=None, post=None, sparseness=None):
        """Each presynaptic neuron gets Binomial(m, p) distinct targets drawn
        uniformly (synapses.py:845-885)."""
        self._check_open()
        if sparseness is None or not 0.0 <= float(sparseness) <= 1.0:
            raise ValueError("connection probability must lie in [0, 1], not %r" % (sparseness,))
        pre_idx = _group_range(self.source if pre is None else pre, self.source)
        post_idx = _group_range(self.target if post is None else post, self.target)
        m = len(post_idx)
        ks = np.random.binomial(m, sparseness, size=len(pre_idx)).astype(np.int64)
        # rows holding more than a quarter of the targets take a random
        # permutation's prefix (redrawing repeats would take ~m log m rounds)
        dense = ks > m // 4 if m else np.zeros(len(ks), dtype=bool)
        kd = np.where(dense, 0, ks)
        rows = np.repeat(np.arange(len(pre_idx)), kd)
        # k distinct targets per sparse row: draw with replacement for all rows
        # at once, then redraw the repeats within a row until none is left
        sel = np.random.randint(0, max(m, 1), size=len(rows)).astype(np.int64) if m else np.zeros(0, np.int64)
        while len(sel):
            key = rows * max(m, 1) + sel
            order = np.argsort(key, kind="stable")
            dup = np.zeros(len(sel), dtype=bool)
            dup[order[1:]] = key[order[1:]] == key[order[:-1]]
            nd = int(dup.sum())
            if nd == 0:
                break
            sel[dup] = np.random.randint(0, m, size=nd)
        if dense.any():
            parts_r, parts_s = [rows], [sel]
            for r in np.nonzero(dense)[0]:
                parts_r.append(np.full(ks[r], r, dtype=np.int64))
                parts_s.append(np.argsort(np.random.random(m), kind="stable")[:ks[r]].astype(np.int64))
            rows, sel = np.concatenate(parts_r), np.concatenate(parts_s)
            order = np.argsort(rows, kind="stable")        # synapses created row by row
            rows, sel = rows[order], sel[order]
        self._create(pre_idx[rows], post_idx[sel])

    def connect_one_to_one(self, pre=None, post=None):
        self._check_open()

        def size(x, G):
            if x is None:
                return len(G)
            if isinstance(x, (NeuronGroup, Subgroup)):
                return len(x)
            return len(_group_range(x, G))

        # the sizes are compared first, as in synapses.py:829-843
        if size(pre, self.source) != size(post, self.target):
            raise TypeError("Source and target groups do not have the same size")
        pre_idx = _group_range(self.source if pre is None else pre, self.source)
        post_idx = _group_range(self.target if post is None else post, self.target)
        self._create(pre_idx, post_idx)

    def create_synapses(self, presynaptic, postsynaptic, synapses_pre=None, synapses_post=None):
        """New synapses from arrays of pre- and postsynaptic indices, taking
        the next synapse indices in array order (synapses.py:725-763)."""
        self._check_open()
        if synapses_pre is not None or synapses_post is not None:
            raise NotImplementedError("explicit synapse index maps")
        pres = np.asarray(presynaptic, dtype=np.int64)
        posts = np.asarray(postsynaptic, dtype=np.int64)
        if pres.shape != posts.shape:
            raise ValueError("presynaptic and postsynaptic arrays differ in length")
        if len(pres) and (pres.min() < 0 or pres.max() >= len(self.source) or posts.min() < 0
                          or posts.max() >= len(self.target)):
            raise ValueError("neuron index out of range")
        self._create(pres, posts)

    def _create(self, pres, posts):
        """create_synapses (synapses.py:725-763): new synapses take the next
        indices in the given order."""
        n = len(pres)
        self.presynaptic = np.concatenate([self.presynaptic, np.asarray(pres, dtype=np.int64)])
        self.postsynaptic = np.concatenate([self.postsynaptic, np.asarray(posts, dtype=np.int64)])
        self._delay = np.concatenate([self._delay, np.zeros(n, dtype=np.int16)])
        for name in self._names:
            self._vars[name] = np.concatenate([self._vars[name], np.zeros(n)])
        self._changed(delays=True)

    def save_connectivity(self, fn):
        """Save the synapses' neuron indices and delays (bins) with
        numpy.savez under the reference's keys (synapses.py:1003-1038):
        presynaptic, postsynaptic, _delay_pre (one row per pre code),
        _delay_post."""
        np.savez(fn, presynaptic=self.presynaptic, postsynaptic=self.postsynaptic,
                 _delay_pre=self._delay.reshape(1, -1), _delay_post=np.zeros(len(self), dtype=np.int16))
        return 1

    def load_connectivity(self, fn):
        """Create the saved synapses (appended after any existing ones) with
        their delays (synapses.py:1040-1054)."""
        data = np.load(fn)
        n0 = len(self)
        self.create_synapses(data["presynaptic"], data["postsynaptic"])
        d = np.asarray(data["_delay_pre"])
        self._delay[n0:] = (d[0] if d.ndim == 2 else d).astype(np.int16)

    # ------------------------------------------------------------- indexing
    def synapse_index(self, key):
        return self._synapse_index(key)

    def _synapse_index(self, key):
        """Synapse indices of a slice / int / array, or of (i, j) neuron
        indices (synapses.py:946-1001)."""
        if isinstance(key, tuple):
            # (i, j): every synapse between the neurons; (i, j, k): the k-th
            # synapse of each pair, in creation order
            i, j = key[0], key[1]
            pi = _group_range(i, self.source)
            qj = _group_range(j, self.target)
            sel = np.nonzero(np.isin(self.presynaptic, pi) & np.isin(self.postsynaptic, qj))[0]
            if len(key) == 3:
                pair = self.presynaptic[sel] * max(1, len(self.target)) + self.postsynaptic[sel]
                rank = np.zeros(len(sel), dtype=np.int64)
                seen = {}
                for n_, p_ in enumerate(pair.tolist()):
                    rank[n_] = seen.get(p_, 0)
                    seen[p_] = rank[n_] + 1
                k = key[2]
                if isinstance(k, slice):
                    want = np.arange(int(rank.max()) + 1 if len(rank) else 0)[k]
                elif np.isscalar(k):
                    want = [int(k)]
                else:
                    want = np.asarray(k, dtype=np.int64).ravel()
                sel = sel[np.isin(rank, want)]
            return sel
        if isinstance(key, slice):
            return np.arange(len(self))[key]
        return np.asarray(key, dtype=np.int64)

    def _eval_string(self, code, idx):
        ns = _caller_namespace(0)
        n = len(idx)
        code = re.sub(r"\brand\(\)", "rand(n)", code)
        code = re.sub(r"\brandn\(\)", "randn(n)", code)
        ns.update({"i": self.presynaptic[idx], "j": self.postsynaptic[idx], "n": n,
                   "rand": np.random.rand, "randn": np.random.randn})
        for name in self._names:
            ns[name] = self._vars[name][idx]
        return np.broadcast_to(np.asarray(eval(code, ns), dtype=np.float64), (n,))

    def __getattr__(self, name):
        if name.startswith("_"):
            raise AttributeError(name)
        if name in ("delay", "delay_pre"):
            return _SynapticDelay(self, name)
        if name in self.__dict__.get("_vars", {}):
            return _SynapticVariable(self, name)
        raise AttributeError(name)

    def __setattr__(self, name, value):
        if name in ("delay", "delay_pre"):
            _SynapticDelay(self, name)[:] = value
        elif name in self.__dict__.get("_vars", {}):
            _SynapticVariable(self, name)[:] = value
        else:
            object.__setattr__(self, name, value)

    # ------------------------------------------------------------- lowering
    def _changed(self, delays=False, var=None):
        b = self.__dict__.get("_binding")
        if b is None:
            return
        if delays:
            raise NotImplementedError("changing synapses or delays after the first run is not supported")
        if self._coded:
            if var is not None:
                b.write_synapse_var(self, self._names.index(var), self._vars[var])
            return
        b.write_synapse_terms(self, self._terms())

    def _sync_vars(self):
        """Synaptic variables the engine holds, into the host copies."""
        b = self.__dict__.get("_binding")
        if b is not None and self._coded:
            for k, n in enumerate(self._names):
                self._vars[n] = b.read_synapse_var(self, k)

    def _host_state(self, d):
        if self._coded:
            self._sync_vars()
            d["_vars"] = {n: v.copy() for n, v in self._vars.items()}

    def _terms(self):
        """Per statement and synapse, the value added or subtracted:
        c*w evaluated as numpy does it (one rounding), w itself for c = 1."""
        out = np.empty((len(self._ops), len(self)))
        for k, (_, _, name, c) in enumerate(self._ops):
            if name is None:
                out[k] = c
            else:
                v = self._vars[name]
                out[k] = v if c == 1.0 else c * v
        return out

    def _queue_check(self):
        """SpikeQueue.compress (spikequeue.py:172-208): with max_delay > 0
        the queue has int(floor(max_delay/dt)) + 1 rows and longer delays
        are refused."""
        if len(self) == 0:
            return
        dmax = int(self._delay.max())
        if int(self._delay.min()) < 0:
            raise ValueError("negative synaptic delay")
        if self.max_delay > 0 and dmax + 1 > int(np.floor(self.max_delay / self.clock.dt)) + 1:
            raise ValueError("Synaptic delays exceed maximum delay")
        if dmax > 253:
            raise NotImplementedError("synaptic delays of more than 253 bins are not supported")

    def _lower(self, rt, gids):
        self._queue_check()
        src, tgt = self.source._owner, self.target._owner
        ops = self._ops
        if self._coded:
            sid = rt.synapses_add(gids[src], self.source._origin, len(self.source), gids[tgt], self.target._origin,
                                  len(self.target), self.presynaptic, self.postsynaptic, self._delay, [], [],
                                  np.zeros((0, len(self))))
            pre_c, post_c, slots, writes, pres = self._code
            sv = np.array([self._vars[n] for n in self._names], dtype=np.float64).reshape(len(self._names), len(self))
            rt.synapses_set_code(sid, sv, pre_c, post_c, slots, writes, pres)
            self._iscompressed = True
            return sid
        sid = rt.synapses_add(gids[src], self.source._origin, len(self.source), gids[tgt], self.target._origin,
                              len(self.target), self.presynaptic, self.postsynaptic, self._delay,
                              [o[0] for o in ops], [1 if o[1] else 0 for o in ops], self._terms())
        self._iscompressed = True
        return sid

    def __repr__(self):
        return "Synapses(%r -> %r, %d synapses)" % (self.source, self.target, len(self))
