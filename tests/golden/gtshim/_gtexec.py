"""A small GT4Py-cartesian executor on numpy, for generating golden fixtures.

TEST INFRASTRUCTURE ONLY: ``tests/golden/make_golden.py`` puts this directory
on ``sys.path`` so that the reference's own stencil source (pySHiELD's
``microphysics.py``, ``microphysics_funcs.py``, ``physics.py``,
``update_atmos_state.py``, ``fv_update_phys.py``) can be imported and run in a
container where gt4py and NDSL are not installed.

It interprets a stencil definition's AST with the documented GT4Py semantics
that the numpy backend implements:

* ``computation(PARALLEL)``: every statement runs over its whole interval
  before the next statement runs;
* ``computation(FORWARD)`` / ``computation(BACKWARD)``: levels run in
  increasing / decreasing order, all statements of a level in order, so offset
  reads ``[0, 0, -1]`` / ``[0, 0, +1]`` see values updated earlier in the sweep;
* ``interval(a, b)`` with negative bounds counted from the top of the domain;
* ``if`` / ``elif`` / ``else`` become masks; an assignment under a mask keeps
  the previous value elsewhere; temporaries start as NaN so that a read of an
  unassigned value shows up in the outputs;
* ``gtscript.function`` calls are inlined with fresh locals; ``from
  __externals__ import`` names resolve to the stencil's externals.

Horizontal dimensions are always vectorised; arithmetic is evaluated in the
order the source's expression tree gives. A stencil that reads horizontal
offsets runs on its domain widened by the largest offset, so that its
temporaries hold values wherever their readers look; it writes the caller's
fields on the domain only.
"""

import ast
import inspect
import textwrap

import numpy as np

PARALLEL = "PARALLEL"
FORWARD = "FORWARD"
BACKWARD = "BACKWARD"


class _Builtin:
    def __init__(self, name):
        self.name = name

    def __repr__(self):
        return f"<gtscript builtin {self.name}>"


sqrt = _Builtin("sqrt")
exp = _Builtin("exp")
log = _Builtin("log")
computation = _Builtin("computation")
interval = _Builtin("interval")

_NP_BUILTINS = {"sqrt": np.sqrt, "exp": np.exp, "log": np.log}


def function(func):
    func._gtscript_function = True
    return func


class _Ctx:
    """Vertical context: a k-range [k0, k1) of the compute domain."""

    def __init__(self, k0, k1):
        self.k0 = k0
        self.k1 = k1


class _Field:
    """A 3-D (or 2-D) view of caller storage restricted to the stencil's
    horizontal domain. In k the view runs from the origin to the end of the
    storage: GT4Py lets a stencil read levels above its domain (``[0, 0, 1]``
    on the last level) when the storage has them; writes stay inside the
    computation's interval."""

    def __init__(self, arr, origin, domain, is2d=False):
        self.is2d = is2d
        if is2d:
            self.a = arr[origin[0] : origin[0] + domain[0], origin[1] : origin[1] + domain[1]]
        else:
            self.a = arr[
                origin[0] : origin[0] + domain[0],
                origin[1] : origin[1] + domain[1],
                origin[2] :,
            ]

    def read(self, ctx, dk=0):
        if self.is2d:
            return self.a[:, :, None]
        return self.a[:, :, ctx.k0 + dk : ctx.k1 + dk]

    def write(self, ctx, value, mask):
        if self.is2d:
            # GT4Py allows a 2-D field to be written from a single-level context
            if ctx.k1 - ctx.k0 != 1:
                raise RuntimeError("write to a 2-D field over more than one level")
            v = np.broadcast_to(value, self.a.shape + (1,))[..., 0]
            if mask is None:
                self.a[...] = v
            else:
                self.a[...] = np.where(mask[..., 0], v, self.a)
            return
        cur = self.a[:, :, ctx.k0 : ctx.k1]
        if mask is None:
            cur[...] = np.broadcast_to(value, cur.shape)
        else:
            cur[...] = np.where(mask, value, cur)


class _Local:
    """A function-local (context-shaped) variable."""

    def __init__(self, shape):
        self.a = np.full(shape, np.nan)

    def read(self, ctx, dk=0):
        if dk != 0:
            raise RuntimeError("offset read of a function local")
        return self.a

    def write(self, ctx, value, mask):
        if mask is None:
            self.a = np.array(np.broadcast_to(value, self.a.shape), dtype=np.float64)
        else:
            self.a = np.where(mask, value, self.a)


class _HField:
    """A field of a stencil that reads horizontal offsets. Such a stencil runs
    on its domain widened by ``ext`` = (ex, ey) points on each side, so that
    a temporary read at an offset holds values there (GT4Py computes a
    temporary on the extent its readers need); fields of the caller are
    written on the domain only. ``kind``: "3d", "ij" (FloatFieldIJ), "i"
    (FloatFieldI) or "temp"."""

    def __init__(self, arr, origin, domain, ext, kind):
        self.ext, self.dom, self.kind = ext, domain, kind
        ex, ey = ext
        ni, nj, nk = domain
        if kind == "temp":
            self.a = np.full((ni + 4 * ex, nj + 4 * ey, nk), np.nan)
            return
        self.arr = arr
        self.origin = origin

    def _padded(self):
        """The caller's array on [-2ex, n + 2ex) around the domain (NaN where
        the storage has no point), as of now."""
        ex, ey = self.ext
        ni, nj, nk = self.dom
        o = self.origin
        if self.kind == "i":
            out = np.full((ni + 4 * ex,), np.nan)
            lo = o[0] - 2 * ex
            for e in range(ni + 4 * ex):
                if 0 <= lo + e < self.arr.shape[0]:
                    out[e] = self.arr[lo + e]
            return out
        shape = (ni + 4 * ex, nj + 4 * ey) + (() if self.kind == "ij" else (self.arr.shape[2] - o[2],))
        out = np.full(shape, np.nan)
        i_lo, j_lo = o[0] - 2 * ex, o[1] - 2 * ey
        a0, a1 = max(0, i_lo), min(self.arr.shape[0], i_lo + shape[0])
        b0, b1 = max(0, j_lo), min(self.arr.shape[1], j_lo + shape[1])
        if self.kind == "ij":
            out[a0 - i_lo : a1 - i_lo, b0 - j_lo : b1 - j_lo] = self.arr[a0:a1, b0:b1]
        else:
            out[a0 - i_lo : a1 - i_lo, b0 - j_lo : b1 - j_lo] = self.arr[a0:a1, b0:b1, o[2]:]
        return out

    def read(self, ctx, dk=0, di=0, dj=0):
        ex, ey = self.ext
        ni, nj, _ = self.dom
        si = slice(ex + di, ex + di + ni + 2 * ex)
        sj = slice(ey + dj, ey + dj + nj + 2 * ey)
        a = self.a if self.kind == "temp" else self._padded()
        if self.kind == "i":
            return a[si][:, None, None]
        if self.kind == "ij":
            return a[si, sj][:, :, None]
        return a[si, sj, ctx.k0 + dk : ctx.k1 + dk]

    def write(self, ctx, value, mask):
        ex, ey = self.ext
        ni, nj, _ = self.dom
        eshape = (ni + 2 * ex, nj + 2 * ey, ctx.k1 - ctx.k0)
        v = np.broadcast_to(value, eshape)
        m = None if mask is None else np.broadcast_to(mask, eshape)
        if self.kind == "temp":
            cur = self.a[ex : ex + ni + 2 * ex, ey : ey + nj + 2 * ey, ctx.k0 : ctx.k1]
            cur[...] = v if m is None else np.where(m, v, cur)
            return
        if self.kind != "3d":
            raise RuntimeError("write to a 2-D or 1-D field of a stencil with horizontal offsets")
        o = self.origin
        cur = self.arr[o[0] : o[0] + ni, o[1] : o[1] + nj, o[2] + ctx.k0 : o[2] + ctx.k1]
        vi = v[ex : ex + ni, ey : ey + nj]
        cur[...] = vi if m is None else np.where(m[ex : ex + ni, ey : ey + nj], vi, cur)


class _Frame:
    def __init__(self, names, globs, externals, shape, temps=None, fields=None):
        self.names = names  # name -> _Field/_Local/scalar
        self.globs = globs
        self.externals = externals
        self.shape = shape
        self.temps = temps  # stencil-level temporaries (None inside functions)
        self.fields = fields


class Stencil:
    def __init__(self, func, externals=None, origin=None, domain=None):
        self.func = func
        self.externals = dict(externals or {})
        self.origin = tuple(origin)
        self.domain = tuple(domain)
        src = textwrap.dedent(inspect.getsource(func))
        tree = ast.parse(src)
        self.fdef = tree.body[0]
        self.params = [a.arg for a in self.fdef.args.args]
        self.annotations = {}
        for a in self.fdef.args.args:
            self.annotations[a.arg] = ast.unparse(a.annotation) if a.annotation else ""
        self.globs = func.__globals__
        ex = ey = 0
        for node in ast.walk(self.fdef):
            if isinstance(node, ast.Subscript) and isinstance(node.value, ast.Name):
                try:
                    off = ast.literal_eval(node.slice)
                except ValueError:
                    continue
                if isinstance(off, tuple) and len(off) == 3:
                    ex, ey = max(ex, abs(off[0])), max(ey, abs(off[1]))
        self.ext = (ex, ey)

    # ------------------------------------------------------------------ call
    def __call__(self, *args, **kwargs):
        bound = dict(zip(self.params, args))
        bound.update(kwargs)
        ni, nj, nk = self.domain
        names = {}
        ext = self.ext
        horizontal = ext != (0, 0)
        for p in self.params:
            v = bound[p]
            ann = self.annotations[p]
            if horizontal and ann in ("FloatField", "FloatFieldIJ", "FloatFieldI"):
                kind = {"FloatField": "3d", "FloatFieldIJ": "ij", "FloatFieldI": "i"}[ann]
                names[p] = _HField(np.asarray(getattr(v, "data", v)), self.origin, self.domain, ext, kind)
            elif ann in ("FloatField", "FloatFieldIJ"):
                arr = getattr(v, "data", v)
                names[p] = _Field(np.asarray(arr), self.origin, self.domain, is2d=(ann == "FloatFieldIJ"))
            else:
                names[p] = v
        shape = (ni + 2 * ext[0], nj + 2 * ext[1], nk)
        frame = _Frame(names, self.globs, self.externals, shape, temps={}, fields=names)
        frame.ext = ext
        frame.domain = self.domain
        with np.errstate(all="ignore"):
            for stmt in self.fdef.body:
                self._top_stmt(stmt, frame)

    def _interval(self, node):
        nk = self.domain[2]
        if len(node.args) == 1 and isinstance(node.args[0], ast.Constant) and node.args[0].value is Ellipsis:
            return 0, nk
        a = ast.literal_eval(node.args[0])
        b = ast.literal_eval(node.args[1])
        start = a if a >= 0 else nk + a
        end = nk if b is None else (b if b >= 0 else nk + b)
        return start, end

    def _top_stmt(self, stmt, frame):
        if isinstance(stmt, ast.ImportFrom) and stmt.module == "__externals__":
            return
        if isinstance(stmt, ast.Expr) and isinstance(stmt.value, ast.Constant):
            return
        if not isinstance(stmt, ast.With):
            raise NotImplementedError(ast.dump(stmt))
        order = None
        iv = None
        for item in stmt.items:
            call = item.context_expr
            fname = call.func.id
            if fname == "computation":
                order = call.args[0].id
            elif fname == "interval":
                iv = self._interval(call)
        if iv is not None:
            blocks = [(iv, stmt.body)]
        else:
            blocks = []
            for sub in stmt.body:
                if isinstance(sub, ast.Expr) and isinstance(sub.value, ast.Constant):
                    continue
                assert isinstance(sub, ast.With)
                blocks.append((self._interval(sub.items[0].context_expr), sub.body))
        if order == PARALLEL:
            for (k0, k1), body in blocks:
                if k1 <= k0:
                    continue
                ctx = _Ctx(k0, k1)
                for s in body:
                    self._stmt(s, frame, ctx, None)
        elif order == FORWARD:
            for (k0, k1), body in sorted(blocks, key=lambda b: b[0][0]):
                for k in range(k0, k1):
                    ctx = _Ctx(k, k + 1)
                    for s in body:
                        self._stmt(s, frame, ctx, None)
        elif order == BACKWARD:
            for (k0, k1), body in sorted(blocks, key=lambda b: -b[0][0]):
                for k in range(k1 - 1, k0 - 1, -1):
                    ctx = _Ctx(k, k + 1)
                    for s in body:
                        self._stmt(s, frame, ctx, None)
        else:
            raise NotImplementedError(order)

    # ------------------------------------------------------------ statements
    def _ctx_shape(self, frame, ctx):
        return (frame.shape[0], frame.shape[1], ctx.k1 - ctx.k0)

    def _lookup_var(self, name, frame):
        if name in frame.names:
            return frame.names[name]
        if frame.temps is not None and name in frame.temps:
            return frame.temps[name]
        return None

    def _assign(self, name, value, frame, ctx, mask):
        var = self._lookup_var(name, frame)
        if var is None:
            if frame.temps is not None:
                ni, nj, nk = frame.shape
                if getattr(frame, "ext", (0, 0)) != (0, 0):
                    var = _HField(None, None, frame.domain, frame.ext, "temp")
                else:
                    var = _Field(np.full((ni, nj, nk), np.nan), (0, 0, 0), (ni, nj, nk))
                frame.temps[name] = var
            else:
                var = _Local(self._ctx_shape(frame, ctx))
                frame.names[name] = var
        if not isinstance(var, (_Field, _Local, _HField)):
            # function parameter passed by value: rebind as a local
            var = _Local(self._ctx_shape(frame, ctx))
            old = frame.names[name]
            var.a = np.array(np.broadcast_to(old, var.a.shape), dtype=np.float64)
            frame.names[name] = var
        var.write(ctx, value, mask)

    def _stmt(self, s, frame, ctx, mask):
        if isinstance(s, ast.ImportFrom):
            return
        if isinstance(s, ast.Expr) and isinstance(s.value, ast.Constant):
            return
        if isinstance(s, ast.Pass):
            return
        if isinstance(s, ast.Assign):
            assert len(s.targets) == 1
            tgt = s.targets[0]
            val = self._expr(s.value, frame, ctx)
            if isinstance(tgt, ast.Tuple):
                for t, v in zip(tgt.elts, val):
                    self._assign(self._target_name(t), v, frame, ctx, mask)
            else:
                self._assign(self._target_name(tgt), val, frame, ctx, mask)
            return
        if isinstance(s, ast.AugAssign):
            name = self._target_name(s.target)
            cur = self._expr(ast.Name(id=name, ctx=ast.Load()), frame, ctx)
            rhs = self._expr(s.value, frame, ctx)
            self._assign(name, self._binop(s.op, cur, rhs), frame, ctx, mask)
            return
        if isinstance(s, ast.If):
            cond = self._expr(s.test, frame, ctx)
            cond = np.broadcast_to(np.asarray(cond, dtype=bool), self._ctx_shape(frame, ctx))
            m_if = cond if mask is None else (mask & cond)
            m_else = ~cond if mask is None else (mask & ~cond)
            for b in s.body:
                self._stmt(b, frame, ctx, m_if)
            for b in s.orelse:
                self._stmt(b, frame, ctx, m_else)
            return
        if isinstance(s, ast.Return):
            raise RuntimeError("return outside a function")
        raise NotImplementedError(ast.dump(s))

    @staticmethod
    def _target_name(t):
        if isinstance(t, ast.Name):
            return t.id
        if isinstance(t, ast.Subscript):
            off = ast.literal_eval(t.slice)
            assert tuple(off) == (0, 0, 0), off
            return t.value.id
        raise NotImplementedError(ast.dump(t))

    # ----------------------------------------------------------- expressions
    @staticmethod
    def _binop(op, a, b):
        if isinstance(op, ast.Add):
            return a + b
        if isinstance(op, ast.Sub):
            return a - b
        if isinstance(op, ast.Mult):
            return a * b
        if isinstance(op, ast.Div):
            return a / b
        if isinstance(op, ast.Pow):
            return np.power(a, b)
        raise NotImplementedError(op)

    def _resolve_global(self, node, frame):
        if isinstance(node, ast.Name):
            if node.id in frame.externals:
                return frame.externals[node.id]
            if node.id in frame.globs:
                return frame.globs[node.id]
            import builtins

            return getattr(builtins, node.id)
        if isinstance(node, ast.Attribute):
            base = self._resolve_global(node.value, frame)
            return getattr(base, node.attr)
        raise NotImplementedError(ast.dump(node))

    def _expr(self, e, frame, ctx):
        if isinstance(e, ast.Constant):
            return e.value
        if isinstance(e, ast.Name):
            var = self._lookup_var(e.id, frame)
            if var is not None:
                if isinstance(var, (_Field, _Local, _HField)):
                    return var.read(ctx)
                return var
            return self._resolve_global(e, frame)
        if isinstance(e, ast.Attribute):
            return self._resolve_global(e, frame)
        if isinstance(e, ast.Subscript):
            off = ast.literal_eval(e.slice)
            var = self._lookup_var(e.value.id, frame)
            if isinstance(var, _HField):
                return var.read(ctx, off[2], off[0], off[1])
            assert off[0] == 0 and off[1] == 0
            return var.read(ctx, off[2])
        if isinstance(e, ast.BinOp):
            return self._binop(e.op, self._expr(e.left, frame, ctx), self._expr(e.right, frame, ctx))
        if isinstance(e, ast.UnaryOp):
            v = self._expr(e.operand, frame, ctx)
            if isinstance(e.op, ast.USub):
                return -v
            if isinstance(e.op, ast.UAdd):
                return +v
            if isinstance(e.op, ast.Not):
                return np.logical_not(v)
            raise NotImplementedError(e.op)
        if isinstance(e, ast.BoolOp):
            vals = [np.asarray(self._expr(v, frame, ctx), dtype=bool) for v in e.values]
            out = vals[0]
            for v in vals[1:]:
                out = (out & v) if isinstance(e.op, ast.And) else (out | v)
            return out
        if isinstance(e, ast.Compare):
            assert len(e.ops) == 1
            a = self._expr(e.left, frame, ctx)
            b = self._expr(e.comparators[0], frame, ctx)
            op = e.ops[0]
            if isinstance(op, ast.Lt):
                return np.less(a, b)
            if isinstance(op, ast.LtE):
                return np.less_equal(a, b)
            if isinstance(op, ast.Gt):
                return np.greater(a, b)
            if isinstance(op, ast.GtE):
                return np.greater_equal(a, b)
            if isinstance(op, ast.Eq):
                return np.equal(a, b)
            if isinstance(op, ast.NotEq):
                return np.not_equal(a, b)
            raise NotImplementedError(op)
        if isinstance(e, ast.IfExp):
            c = self._expr(e.test, frame, ctx)
            return np.where(c, self._expr(e.body, frame, ctx), self._expr(e.orelse, frame, ctx))
        if isinstance(e, ast.Tuple):
            return tuple(self._expr(x, frame, ctx) for x in e.elts)
        if isinstance(e, ast.Call):
            return self._call(e, frame, ctx)
        raise NotImplementedError(ast.dump(e))

    def _call(self, e, frame, ctx):
        args = [self._expr(a, frame, ctx) for a in e.args]
        fn = self._resolve_global(e.func, frame)
        if isinstance(fn, _Builtin):
            return _NP_BUILTINS[fn.name](*args)
        if fn is min:
            return np.minimum(*args)
        if fn is max:
            return np.maximum(*args)
        if fn is abs:
            return np.abs(*args)
        if getattr(fn, "_gtscript_function", False):
            return self._inline(fn, args, frame, ctx)
        raise NotImplementedError(f"call to {fn}")

    def _inline(self, fn, args, frame, ctx):
        src = textwrap.dedent(inspect.getsource(fn))
        fdef = ast.parse(src).body[0]
        names = {}
        for a, v in zip(fdef.args.args, args):
            names[a.arg] = v
        sub = _Frame(names, fn.__globals__, frame.externals, frame.shape)
        ret = None
        for s in fdef.body:
            if isinstance(s, ast.Return):
                ret = self._expr(s.value, sub, ctx)
                break
            self._stmt(s, sub, ctx, None)
        return ret
