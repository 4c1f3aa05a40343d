"""The reference's Lua setup interface: ``initialise(x, y, z, xs, ys, zs)``.

A run without an initial-conditions file takes its initial state from a Lua
setup script (``config/torch-setup.lua`` by default, ``src/main.cpp:29``):
the script runs once, then ``Torch::setUpLua`` (``src/Torch/Torch.cpp:196-228``)
calls its global function ``initialise`` once per cell with the cell's and
the star's positions in cgs, and takes nine results: density, pressure,
ionisation fraction, three velocity components and three gravity
components.

No Lua interpreter is shipped with this library, so this module evaluates
the subset of Lua 5.2 that setup scripts are written in: numbers (IEEE
doubles, as in Lua 5.2), booleans, nil, strings, local and global variables,
``function`` definitions (global and local, closures, multiple results),
``if``/``elseif``/``else``, ``while``, numeric ``for``, ``do`` blocks,
``return``, ``break``, arithmetic ``+ - * / % ^`` and unary minus,
comparisons, ``and``/``or``/``not``, ``..`` and the ``math`` library
functions.  Arithmetic follows Lua 5.2's C implementation: ``+ - * /`` are
single IEEE operations, ``a % b`` is ``a - floor(a/b)*b``, and ``^``,
``math.pow``, ``math.exp``, ``math.log`` etc. call the C math library (the
same libm the reference's Lua calls), so the results are bitwise those of the
reference's own Lua evaluation.  Anything outside the subset (tables other
than ``math``, metatables, goto, varargs, the standard library beyond
``math``) raises ``LuaError``.

The tests pin this evaluator bit for bit against the reference's own Lua
evaluation of the same scripts (``tests/golden``).
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
import re
from typing import Dict, List, Optional

import numpy as np


class LuaError(RuntimeError):
    pass


# ----------------------------------------------------------------- C libm
_libm = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
for _name in ("pow", "exp", "log", "log10", "sqrt", "floor", "ceil", "fabs", "sin", "cos", "tan", "asin",
              "acos", "atan", "atan2", "sinh", "cosh", "tanh", "fmod"):
    _f = getattr(_libm, _name)
    _f.restype = ctypes.c_double
    _f.argtypes = [ctypes.c_double, ctypes.c_double] if _name in ("pow", "atan2", "fmod") else [ctypes.c_double]


def _num(v, what="arithmetic"):
    if isinstance(v, bool) or v is None:
        raise LuaError(f"attempt to perform {what} on a {'boolean' if isinstance(v, bool) else 'nil'} value")
    if isinstance(v, float):
        return v
    if isinstance(v, str):  # Lua coerces numeric strings
        try:
            return float(v)
        except ValueError:
            pass
    raise LuaError(f"attempt to perform {what} on a {type(v).__name__} value")


def _div(a: float, b: float) -> float:
    try:
        return a / b
    except ZeroDivisionError:
        if a != a or a == 0.0:
            return math.nan
        return math.copysign(math.inf, a) * math.copysign(1.0, b)


def _mod(a: float, b: float) -> float:
    # luai_nummod (Lua 5.2, luaconf.h): a - floor(a/b)*b
    return a - _libm.floor(_div(a, b)) * b


def _math_log(x, base=None):
    # math_log (Lua 5.2.3, lmathlib.c): log10 for base 10, else log(x)/log(base)
    x = _num(x)
    if base is None:
        return _libm.log(x)
    base = _num(base)
    if base == 10.0:
        return _libm.log10(x)
    return _div(_libm.log(x), _libm.log(base))


def _math_min(*a):
    if not a:
        raise LuaError("bad argument #1 to 'min' (number expected, got no value)")
    r = _num(a[0])
    for v in a[1:]:
        v = _num(v)
        if v < r:
            r = v
    return r


def _math_max(*a):
    if not a:
        raise LuaError("bad argument #1 to 'max' (number expected, got no value)")
    r = _num(a[0])
    for v in a[1:]:
        v = _num(v)
        if v > r:
            r = v
    return r


def _math_modf(x):
    x = _num(x)
    ip = _libm.floor(x) if x >= 0 else _libm.ceil(x)
    return [ip, x - ip if not math.isinf(x) else 0.0]


def _math_table() -> Dict[str, object]:
    one = lambda f: (lambda x: getattr(_libm, f)(_num(x)))  # noqa: E731
    t = {name: one(name) for name in ("exp", "log10", "sqrt", "floor", "ceil", "sin", "cos", "tan", "asin",
                                      "acos", "atan", "sinh", "cosh", "tanh")}
    t.update({
        "abs": one("fabs"),
        "pow": lambda x, y: _libm.pow(_num(x), _num(y)),
        "atan2": lambda y, x: _libm.atan2(_num(y), _num(x)),
        "fmod": lambda x, y: _libm.fmod(_num(x), _num(y)),
        "log": _math_log,
        "min": _math_min,
        "max": _math_max,
        "modf": _math_modf,
        "pi": math.pi,
        "huge": math.inf,
    })
    return t


# ----------------------------------------------------------------- lexer
_TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<comment>--\[(?P<eq>=*)\[.*?\](?P=eq)\]|--[^\n]*)
  | (?P<num>0[xX][0-9a-fA-F]*(?:\.[0-9a-fA-F]*)?(?:[pP][+-]?\d+)?|(?:\d+\.?\d*|\.\d+)(?:[eE][+-]?\d+)?)
  | (?P<name>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<str>"(?:[^"\\\n]|\\.)*"|'(?:[^'\\\n]|\\.)*')
  | (?P<op>\.\.\.|\.\.|==|~=|<=|>=|::|[-+*/%^\#<>=(){}\[\];:,.])
""", re.S | re.X)

_KEYWORDS = {"and", "break", "do", "else", "elseif", "end", "false", "for", "function", "goto", "if", "in",
             "local", "nil", "not", "or", "repeat", "return", "then", "true", "until", "while"}


def _lua_number(text: str) -> float:
    if text[:2].lower() == "0x":
        if "." in text or "p" in text.lower():
            return float.fromhex(text)
        return float(int(text, 16))
    return float(text)  # strtod: correctly rounded, as lua_str2number


def _tokens(src: str):
    out = []
    pos, line = 0, 1
    if src.startswith("#"):  # shebang line
        pos = src.find("\n") if "\n" in src else len(src)
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise LuaError(f"line {line}: unexpected symbol near {src[pos:pos + 10]!r}")
        kind = m.lastgroup if m.lastgroup != "eq" else "comment"
        text = m.group(0)
        if kind == "num":
            out.append(("num", _lua_number(text), line))
        elif kind == "name":
            out.append(("kw" if text in _KEYWORDS else "name", text, line))
        elif kind == "str":
            out.append(("str", bytes(text[1:-1], "utf-8").decode("unicode_escape"), line))
        elif kind == "op":
            out.append(("op", text, line))
        line += text.count("\n")
        pos = m.end()
    out.append(("eof", None, line))
    return out


# ----------------------------------------------------------------- parser
_BINPRI = {"or": (1, 1), "and": (2, 2), "<": (3, 3), ">": (3, 3), "<=": (3, 3), ">=": (3, 3), "~=": (3, 3),
           "==": (3, 3), "..": (9, 8), "+": (10, 10), "-": (10, 10), "*": (11, 11), "/": (11, 11),
           "%": (11, 11), "^": (14, 13)}
_UNARY_PRI = 12


class _Parser:
    def __init__(self, src: str):
        self.t = _tokens(src)
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def check(self, kind, value=None):
        tok = self.peek()
        return tok[0] == kind and (value is None or tok[1] == value)

    def accept(self, kind, value=None):
        if self.check(kind, value):
            return self.next()
        return None

    def expect(self, kind, value=None):
        tok = self.next()
        if tok[0] != kind or (value is not None and tok[1] != value):
            raise LuaError(f"line {tok[2]}: '{value or kind}' expected near {tok[1]!r}")
        return tok

    def chunk(self):
        body = self.block()
        self.expect("eof")
        return body

    def block(self):
        stmts = []
        while True:
            tok = self.peek()
            if tok[0] == "eof" or (tok[0] == "kw" and tok[1] in ("end", "else", "elseif", "until")):
                return stmts
            if tok[0] == "kw" and tok[1] == "return":
                self.next()
                exprs = []
                if not (self.check("eof") or self.check("op", ";") or
                        (self.peek()[0] == "kw" and self.peek()[1] in ("end", "else", "elseif", "until"))):
                    exprs = self.exprlist()
                self.accept("op", ";")
                stmts.append(("return", exprs, tok[2]))
                return stmts
            st = self.statement()
            if st is not None:
                stmts.append(st)

    def statement(self):
        tok = self.peek()
        line = tok[2]
        if tok[0] == "op" and tok[1] == ";":
            self.next()
            return None
        if tok[0] == "kw":
            kw = tok[1]
            if kw == "local":
                self.next()
                if self.accept("kw", "function"):
                    name = self.expect("name")[1]
                    return ("localfunc", name, self.funcbody(), line)
                names = [self.expect("name")[1]]
                while self.accept("op", ","):
                    names.append(self.expect("name")[1])
                exprs = self.exprlist() if self.accept("op", "=") else []
                return ("local", names, exprs, line)
            if kw == "function":
                self.next()
                name = self.expect("name")[1]
                if self.check("op", ".") or self.check("op", ":"):
                    raise LuaError(f"line {line}: method/field functions are outside the supported subset")
                return ("assign", [("name", name, line)], [("function", self.funcbody(), line)], line)
            if kw == "if":
                self.next()
                clauses = []
                cond = self.expr()
                self.expect("kw", "then")
                clauses.append((cond, self.block()))
                orelse = None
                while True:
                    if self.accept("kw", "elseif"):
                        cond = self.expr()
                        self.expect("kw", "then")
                        clauses.append((cond, self.block()))
                    elif self.accept("kw", "else"):
                        orelse = self.block()
                        self.expect("kw", "end")
                        break
                    else:
                        self.expect("kw", "end")
                        break
                return ("if", clauses, orelse, line)
            if kw == "while":
                self.next()
                cond = self.expr()
                self.expect("kw", "do")
                body = self.block()
                self.expect("kw", "end")
                return ("while", cond, body, line)
            if kw == "do":
                self.next()
                body = self.block()
                self.expect("kw", "end")
                return ("do", body, line)
            if kw == "for":
                self.next()
                var = self.expect("name")[1]
                if not self.accept("op", "="):
                    raise LuaError(f"line {line}: generic 'for' is outside the supported subset")
                start = self.expr()
                self.expect("op", ",")
                stop = self.expr()
                step = self.expr() if self.accept("op", ",") else None
                self.expect("kw", "do")
                body = self.block()
                self.expect("kw", "end")
                return ("fornum", var, start, stop, step, body, line)
            if kw == "break":
                self.next()
                return ("break", line)
            raise LuaError(f"line {line}: '{kw}' is outside the supported subset")
        # assignment or call statement
        target = self.suffixedexp()
        if self.check("op", "=") or self.check("op", ","):
            targets = [target]
            while self.accept("op", ","):
                targets.append(self.suffixedexp())
            self.expect("op", "=")
            for t in targets:
                if t[0] not in ("name", "index"):
                    raise LuaError(f"line {line}: cannot assign to this expression")
            return ("assign", targets, self.exprlist(), line)
        if target[0] != "call":
            raise LuaError(f"line {line}: syntax error near {self.peek()[1]!r}")
        return ("callstat", target, line)

    def funcbody(self):
        self.expect("op", "(")
        params = []
        if not self.check("op", ")"):
            while True:
                if self.check("op", "..."):
                    raise LuaError("varargs are outside the supported subset")
                params.append(self.expect("name")[1])
                if not self.accept("op", ","):
                    break
        self.expect("op", ")")
        body = self.block()
        self.expect("kw", "end")
        return (params, body)

    def exprlist(self):
        exprs = [self.expr()]
        while self.accept("op", ","):
            exprs.append(self.expr())
        return exprs

    def expr(self, limit=0):
        tok = self.peek()
        if (tok[0] == "kw" and tok[1] == "not") or (tok[0] == "op" and tok[1] in ("-", "#")):
            self.next()
            left = ("unop", tok[1], self.expr(_UNARY_PRI), tok[2])
        else:
            left = self.simpleexp()
        while True:
            tok = self.peek()
            op = tok[1] if tok[0] in ("op", "kw") else None
            if op not in _BINPRI or _BINPRI[op][0] <= limit:
                return left
            self.next()
            right = self.expr(_BINPRI[op][1])
            left = ("binop", op, left, right, tok[2])

    def simpleexp(self):
        tok = self.peek()
        if tok[0] == "num":
            self.next()
            return ("const", tok[1])
        if tok[0] == "str":
            self.next()
            return ("const", tok[1])
        if tok[0] == "kw" and tok[1] in ("nil", "true", "false"):
            self.next()
            return ("const", {"nil": None, "true": True, "false": False}[tok[1]])
        if tok[0] == "kw" and tok[1] == "function":
            self.next()
            return ("function", self.funcbody(), tok[2])
        if tok[0] == "op" and tok[1] == "{":
            raise LuaError(f"line {tok[2]}: table constructors are outside the supported subset")
        return self.suffixedexp()

    def suffixedexp(self):
        tok = self.next()
        if tok[0] == "name":
            e = ("name", tok[1], tok[2])
        elif tok[0] == "op" and tok[1] == "(":
            e = ("paren", self.expr(), tok[2])
            self.expect("op", ")")
        else:
            raise LuaError(f"line {tok[2]}: unexpected symbol near {tok[1]!r}")
        while True:
            if self.accept("op", "."):
                e = ("index", e, ("const", self.expect("name")[1]), tok[2])
            elif self.check("op", "["):
                self.next()
                key = self.expr()
                self.expect("op", "]")
                e = ("index", e, key, tok[2])
            elif self.check("op", "("):
                self.next()
                args = [] if self.check("op", ")") else self.exprlist()
                self.expect("op", ")")
                e = ("call", e, args, tok[2])
            elif self.check("str"):
                e = ("call", e, [("const", self.next()[1])], tok[2])
            elif self.check("op", ":"):
                raise LuaError(f"line {tok[2]}: method calls are outside the supported subset")
            else:
                return e


# ----------------------------------------------------------------- evaluator
class _Return(Exception):
    def __init__(self, values):
        self.values = values


class _Break(Exception):
    pass


class _Function:
    def __init__(self, params, body, scope, interp):
        self.params, self.body, self.scope, self.interp = params, body, scope, interp

    def __call__(self, *args):
        frame = dict(zip(self.params, list(args) + [None] * (len(self.params) - len(args))))
        try:
            self.interp.exec_block(self.body, self.scope + [frame])
        except _Return as r:
            return r.values
        return []


def _truthy(v) -> bool:
    return not (v is None or v is False)


class LuaScript:
    """A Lua setup script: run once on construction, then its global
    functions can be called (``call``)."""

    def __init__(self, source: str):
        self.globals: Dict[str, object] = {"math": _math_table()}
        self.exec_block(_Parser(source).chunk(), [])

    @classmethod
    def from_file(cls, path: str) -> "LuaScript":
        with open(path) as f:
            return cls(f.read())

    # scope: list of local frames (innermost last); globals in self.globals
    def _lookup(self, name, scope):
        for frame in reversed(scope):
            if name in frame:
                return frame[name]
        return self.globals.get(name)

    def _store(self, name, value, scope):
        for frame in reversed(scope):
            if name in frame:
                frame[name] = value
                return
        self.globals[name] = value

    def exec_block(self, stmts, scope):
        scope = scope + [{}]
        for st in stmts:
            self.exec_stmt(st, scope)

    def exec_stmt(self, st, scope):
        kind = st[0]
        if kind == "local":
            vals = self.eval_list(st[2], scope, len(st[1]))
            for n, v in zip(st[1], vals):
                scope[-1][n] = v
        elif kind == "localfunc":
            scope[-1][st[1]] = None
            scope[-1][st[1]] = _Function(st[2][0], st[2][1], list(scope), self)
        elif kind == "assign":
            vals = self.eval_list(st[2], scope, len(st[1]))
            for target, v in zip(st[1], vals):
                if target[0] == "name":
                    self._store(target[1], v, scope)
                else:
                    tbl = self.eval(target[1], scope)
                    if not isinstance(tbl, dict):
                        raise LuaError(f"line {st[3]}: attempt to index a non-table value")
                    tbl[self.eval(target[2], scope)] = v
        elif kind == "callstat":
            self.call(st[1], scope)
        elif kind == "if":
            for cond, body in st[1]:
                if _truthy(self.eval(cond, scope)):
                    self.exec_block(body, scope)
                    return
            if st[2] is not None:
                self.exec_block(st[2], scope)
        elif kind == "while":
            try:
                while _truthy(self.eval(st[1], scope)):
                    self.exec_block(st[2], scope)
            except _Break:
                pass
        elif kind == "do":
            self.exec_block(st[1], scope)
        elif kind == "fornum":
            _, var, e0, e1, e2, body, line = st
            v0, v1 = _num(self.eval(e0, scope), "'for' initial value"), _num(self.eval(e1, scope), "'for' limit")
            step = 1.0 if e2 is None else _num(self.eval(e2, scope), "'for' step")
            if step == 0:
                raise LuaError(f"line {line}: 'for' step is zero")
            v = v0
            try:
                while (v <= v1) if step > 0 else (v >= v1):
                    self.exec_block(body, scope + [{var: v}])
                    v += step
            except _Break:
                pass
        elif kind == "return":
            raise _Return(self.eval_list(st[1], scope, None))
        elif kind == "break":
            raise _Break()
        else:
            raise LuaError(f"unsupported statement {kind}")

    def eval_list(self, exprs, scope, want: Optional[int]) -> List[object]:
        vals: List[object] = []
        for k, e in enumerate(exprs):
            if k == len(exprs) - 1 and e[0] == "call":
                vals.extend(self.call(e, scope))  # the last expression expands
            else:
                vals.append(self.eval(e, scope))
        if want is not None:
            vals = (vals + [None] * want)[:want]
        return vals

    def call(self, e, scope) -> List[object]:
        fn = self.eval(e[1], scope)
        args = self.eval_list(e[2], scope, None)
        if isinstance(fn, _Function):
            return fn(*args)
        if callable(fn):
            r = fn(*args)
            return r if isinstance(r, list) else [r]
        raise LuaError(f"line {e[3]}: attempt to call a {type(fn).__name__} value")

    def eval(self, e, scope):
        kind = e[0]
        if kind == "const":
            return e[1]
        if kind == "name":
            return self._lookup(e[1], scope)
        if kind == "paren":
            return self.eval(e[1], scope)
        if kind == "index":
            tbl = self.eval(e[1], scope)
            if not isinstance(tbl, dict):
                raise LuaError(f"line {e[3]}: attempt to index a {type(tbl).__name__} value")
            return tbl.get(self.eval(e[2], scope))
        if kind == "call":
            r = self.call(e, scope)
            return r[0] if r else None
        if kind == "function":
            return _Function(e[1][0], e[1][1], list(scope), self)
        if kind == "unop":
            v = self.eval(e[2], scope)
            if e[1] == "-":
                return -_num(v)
            if e[1] == "not":
                return not _truthy(v)
            if isinstance(v, str):
                return float(len(v))
            raise LuaError(f"line {e[3]}: attempt to get length of a {type(v).__name__} value")
        if kind == "binop":
            op = e[1]
            if op == "and":
                a = self.eval(e[2], scope)
                return self.eval(e[3], scope) if _truthy(a) else a
            if op == "or":
                a = self.eval(e[2], scope)
                return a if _truthy(a) else self.eval(e[3], scope)
            a, b = self.eval(e[2], scope), self.eval(e[3], scope)
            if op == "+":
                return _num(a) + _num(b)
            if op == "-":
                return _num(a) - _num(b)
            if op == "*":
                return _num(a) * _num(b)
            if op == "/":
                return _div(_num(a), _num(b))
            if op == "%":
                return _mod(_num(a), _num(b))
            if op == "^":
                return _libm.pow(_num(a), _num(b))
            if op == "..":
                def s(v):
                    if isinstance(v, str):
                        return v
                    if isinstance(v, float):
                        return "%.14g" % v
                    raise LuaError(f"line {e[4]}: attempt to concatenate a {type(v).__name__} value")
                return s(a) + s(b)
            if op == "==":
                return a == b and type(a) is type(b)
            if op == "~=":
                return not (a == b and type(a) is type(b))
            if isinstance(a, float) and isinstance(b, float) or isinstance(a, str) and isinstance(b, str):
                return {"<": a < b, ">": a > b, "<=": a <= b, ">=": a >= b}[op]
            raise LuaError(f"line {e[4]}: attempt to compare {type(a).__name__} with {type(b).__name__}")
        raise LuaError(f"unsupported expression {kind}")

    def call_global(self, name: str, *args) -> List[object]:
        fn = self.globals.get(name)
        if not isinstance(fn, _Function):
            raise LuaError(f"the setup script defines no function '{name}'")
        return fn(*[float(a) for a in args])


def evaluate_setup(script: LuaScript, x, y, z, star) -> Dict[str, np.ndarray]:
    """Calls the script's ``initialise(x, y, z, xs, ys, zs)`` for every cell
    (Torch::setUpLua, src/Torch/Torch.cpp:196-228) and returns its nine
    results as arrays: den, pre, hii, vel [3][N], grav [3][N] (cgs)."""
    N = len(x)
    out = np.zeros((9, N))
    xs, ys, zs = (float(v) for v in star)
    for i in range(N):
        r = script.call_global("initialise", float(x[i]), float(y[i]), float(z[i]), xs, ys, zs)
        if len(r) < 9:
            r = list(r) + [None] * (9 - len(r))
        for k in range(9):
            v = r[k]
            if v is None:
                raise LuaError(f"initialise returned {len(r)} values for cell {i}; 9 numbers expected "
                               "(den, pre, hii, v0, v1, v2, grav0, grav1, grav2)")
            out[k, i] = _num(v, "conversion")
    return {"den": out[0], "pre": out[1], "hii": out[2], "vel": out[3:6].copy(), "grav": out[6:9].copy()}
