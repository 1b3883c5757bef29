"""A CPU evaluator for the subset of WGSL that the Fire-X compute shaders use — TEST
INFRASTRUCTURE ONLY (it generates golden fixtures; nothing in the library uses it).

It parses WGSL source text and runs a compute entry point for every invocation of a dispatch
at once, SIMT style: each value is a numpy array over the invocations (lanes), statements run
in lockstep for all lanes, and control flow is a lane mask (an `if` runs both arms under
complementary masks, a loop runs while any lane's condition holds, a `return` retires its
lanes). Lockstep execution is one of the schedules a workgroupBarrier permits, so the
barrier is a no-op here; every kernel evaluated writes each storage element from at most
one invocation, so scatters need no ordering.

Arithmetic follows the WGSL specification with one fixed choice wherever the specification
allows a range of results:
  * f32 and f16 values are numpy float32 / float16 arrays; +, -, *, / and sqrt are IEEE
    operations with round-to-nearest-even (the specification allows inexact division; this
    evaluator divides exactly);
  * sin, cos, exp, pow, exp2, log, log2, tan, atan2 of f32 call the C library's
    single-precision functions (sinf, ...), or, for a module created with
    transcendentals="f64", the double-precision ones rounded to f32; both are within the
    error bounds the specification allows;
  * AbstractFloat / AbstractInt literals and constant expressions built only from them are
    evaluated in float64 / int64 and converted (rounded to nearest) when they meet a
    concrete type or initialise a let/var (WGSL's concretisation rules);
  * builtins are evaluated by their specification formulas: mix(a, b, t) = a * (1 - t) +
    b * t; smoothstep(l, h, x) = t * t * (3 - 2 t) with t = clamp((x - l) / (h - l), 0, 1);
    clamp(e, l, h) = min(max(e, l), h); fract(x) = x - floor(x); length(v) = sqrt(dot(v, v));
    normalize(v) = v / length(v); cross as the usual determinant; max(a, b) = b if a < b
    else a, min(a, b) = b if b < a else a;
  * f32 -> f16 conversion rounds to nearest even (numpy's conversion); f32 -> i32 / u32
    truncates toward zero and saturates; i32 <-> u32 reinterpret the bits.
"""
from __future__ import annotations

import ctypes
import ctypes.util
import math
import re
from dataclasses import dataclass, field

import numpy as np

# ---------------------------------------------------------------- tokens -------------------

_TOKEN = re.compile(r"""
    (?P<ws>\s+|//[^\n]*|/\*.*?\*/)
  | (?P<num>(?:0[xX][0-9a-fA-F]+[iu]?)|(?:(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?[fhiu]?))
  | (?P<id>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>->|\+\+|--|<<=|>>=|&&|\|\||==|!=|<=|>=|<<|>>|\+=|-=|\*=|/=|%=|&=|\|=|\^=|[-+*/%<>=!&|^~.,;:(){}\[\]@])
""", re.S | re.X)


@dataclass
class Tok:
    kind: str
    text: str


def tokenize(src: str) -> list:
    out, pos = [], 0
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise SyntaxError(f"unexpected character {src[pos]!r} at {pos}")
        pos = m.end()
        if m.lastgroup != "ws":
            out.append(Tok(m.lastgroup, m.group()))
    out.append(Tok("eof", ""))
    return out


# ---------------------------------------------------------------- syntax tree --------------

@dataclass
class Node:
    kind: str
    a: object = None
    b: object = None
    c: object = None
    d: object = None


@dataclass
class Func:
    name: str
    params: list  # (name, type, builtin or None)
    ret: object
    body: list
    attrs: dict = field(default_factory=dict)


class Parser:
    """Recursive descent over the token list. Types are kept as nested tuples:
    ('scalar', 'f32') / ('vec', n, 'f32') / ('array', elemtype, count or None) / ('struct', name)."""

    SCALARS = {"f32", "f16", "i32", "u32", "bool"}
    VEC_ALIASES = {f"vec{n}{s}": ("vec", n, t) for n in (2, 3, 4) for s, t in
                   (("f", "f32"), ("h", "f16"), ("i", "i32"), ("u", "u32"))}

    def __init__(self, src: str):
        self.t = tokenize(src)
        self.i = 0
        self.structs, self.consts, self.globals, self.funcs = {}, {}, {}, {}

    # token helpers
    def peek(self, k=0):
        return self.t[self.i + k]

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def accept(self, text):
        if self.peek().text == text:
            self.i += 1
            return True
        return False

    def expect(self, text):
        tok = self.next()
        if tok.text != text:
            raise SyntaxError(f"expected {text!r}, got {tok.text!r} near token {self.i}")
        return tok

    def expect_close(self):
        """A template's closing '>' (the tokenizer reads '>>' in array<atomic<u32>> as one)."""
        tok = self.peek()
        if tok.text == ">>":
            self.t[self.i] = Tok("op", ">")
            return
        self.expect(">")

    # types
    def parse_type(self):
        name = self.next().text
        if name in self.SCALARS:
            return ("scalar", name)
        if name in self.VEC_ALIASES:
            return self.VEC_ALIASES[name]
        if name in ("vec2", "vec3", "vec4"):
            self.expect("<")
            el = self.next().text
            self.expect_close()
            return ("vec", int(name[3]), el)
        if name == "array":
            self.expect("<")
            el = self.parse_type()
            count = None
            if self.accept(","):
                count = self.parse_unary()  # not parse_expr: the closing '>' is not an operator here
            self.expect_close()
            return ("array", el, count)
        if name == "atomic":
            self.expect("<")
            el = self.parse_type()
            self.expect_close()
            return ("atomic", el)
        if name in self.structs:
            return ("struct", name)
        raise SyntaxError(f"unknown type {name}")

    def parse_attrs(self):
        attrs = {}
        while self.accept("@"):
            name = self.next().text
            args = []
            if self.accept("("):
                while not self.accept(")"):
                    args.append(self.next().text)
                    self.accept(",")
            attrs[name] = args
        return attrs

    # module
    def parse_module(self):
        while self.peek().kind != "eof":
            if self.accept(";"):
                continue
            if self.peek().text == "enable":
                while self.next().text != ";":
                    pass
                continue
            attrs = self.parse_attrs()
            kw = self.next().text
            if kw == "struct":
                name = self.next().text
                self.expect("{")
                fields = []
                while not self.accept("}"):
                    self.parse_attrs()
                    fname = self.next().text
                    self.expect(":")
                    fields.append((fname, self.parse_type()))
                    self.accept(",")
                self.structs[name] = fields
            elif kw == "const":
                name = self.next().text
                ty = None
                if self.accept(":"):
                    ty = self.parse_type()
                self.expect("=")
                self.consts[name] = (ty, self.parse_expr())
                self.expect(";")
            elif kw == "var":
                space = []
                if self.accept("<"):
                    while not self.accept(">"):
                        space.append(self.next().text)
                        self.accept(",")
                name = self.next().text
                self.expect(":")
                ty = self.parse_type()
                self.expect(";")
                self.globals[name] = (space, ty, attrs)
            elif kw == "fn":
                name = self.next().text
                self.expect("(")
                params = []
                while not self.accept(")"):
                    pattrs = self.parse_attrs()
                    pname = self.next().text
                    self.expect(":")
                    pty = self.parse_type()
                    params.append((pname, pty, (pattrs.get("builtin") or [None])[0]))
                    self.accept(",")
                ret = None
                if self.accept("->"):
                    self.parse_attrs()
                    ret = self.parse_type()
                self.funcs[name] = Func(name, params, ret, self.parse_block(), attrs)
            else:
                raise SyntaxError(f"unexpected {kw!r} at module scope")
        return self

    # statements
    def parse_block(self):
        self.expect("{")
        out = []
        while not self.accept("}"):
            out.append(self.parse_stmt())
        return out

    def parse_stmt(self):
        tok = self.peek()
        if tok.text == "{":
            return Node("block", self.parse_block())
        if tok.text in ("let", "var", "const"):
            self.next()
            if tok.text == "var" and self.accept("<"):
                while not self.accept(">"):
                    self.next()
            name = self.next().text
            ty = None
            if self.accept(":"):
                ty = self.parse_type()
            init = None
            if self.accept("="):
                init = self.parse_expr()
            self.expect(";")
            return Node("decl", name, ty, init, tok.text)
        if tok.text == "if":
            self.next()
            cond = self.parse_expr()
            then = self.parse_block()
            other = None
            if self.accept("else"):
                other = [self.parse_stmt()] if self.peek().text == "if" else self.parse_block()
            return Node("if", cond, then, other)
        if tok.text == "while":
            self.next()
            cond = self.parse_expr()
            return Node("for", None, cond, None, self.parse_block())
        if tok.text == "for":
            self.next()
            self.expect("(")
            init = None if self.peek().text == ";" else self.parse_simple()
            self.expect(";")
            cond = None if self.peek().text == ";" else self.parse_expr()
            self.expect(";")
            upd = None if self.peek().text == ")" else self.parse_simple()
            self.expect(")")
            return Node("for", init, cond, upd, self.parse_block())
        if tok.text == "loop":
            self.next()
            return Node("for", None, None, None, self.parse_block())
        if tok.text == "return":
            self.next()
            val = None if self.peek().text == ";" else self.parse_expr()
            self.expect(";")
            return Node("return", val)
        if tok.text in ("break", "continue"):
            self.next()
            self.expect(";")
            return Node(tok.text)
        s = self.parse_simple()
        self.expect(";")
        return s

    def parse_simple(self):
        """Declaration, assignment, increment or call (no trailing ';')."""
        tok = self.peek()
        if tok.text in ("let", "var"):
            self.next()
            name = self.next().text
            ty = None
            if self.accept(":"):
                ty = self.parse_type()
            self.expect("=")
            return Node("decl", name, ty, self.parse_expr(), tok.text)
        if tok.text == "_":
            self.next()
            self.expect("=")
            return Node("expr", self.parse_expr())
        lhs = self.parse_expr()
        op = self.peek().text
        if op in ("=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>="):
            self.next()
            return Node("assign", lhs, op, self.parse_expr())
        if op in ("++", "--"):
            self.next()
            return Node("assign", lhs, "+=" if op == "++" else "-=", Node("lit", ("ai", 1)))
        return Node("expr", lhs)

    # expressions (WGSL precedence, lowest first)
    BIN = [("||",), ("&&",), ("|",), ("^",), ("&",), ("==", "!="), ("<", "<=", ">", ">="), ("<<", ">>"),
           ("+", "-"), ("*", "/", "%")]

    def parse_expr(self, level=0):
        if level == len(self.BIN):
            return self.parse_unary()
        lhs = self.parse_expr(level + 1)
        while self.peek().text in self.BIN[level]:
            op = self.next().text
            lhs = Node("bin", op, lhs, self.parse_expr(level + 1))
        return lhs

    def parse_unary(self):
        if self.peek().text in ("-", "!", "~", "&", "*"):
            op = self.next().text
            return Node("un", op, self.parse_unary())
        return self.parse_postfix(self.parse_primary())

    def parse_primary(self):
        tok = self.next()
        if tok.kind == "num":
            return Node("lit", parse_number(tok.text))
        if tok.text == "(":
            e = self.parse_expr()
            self.expect(")")
            return e
        if tok.text in ("true", "false"):
            return Node("lit", ("bool", tok.text == "true"))
        if tok.kind == "id":
            name = tok.text
            if name in ("vec2", "vec3", "vec4", "array") and self.peek().text == "<":
                self.i -= 1
                ty = self.parse_type()
                return Node("call", ty, self.parse_args())
            if self.peek().text == "(":
                ty = self.VEC_ALIASES.get(name) or (("scalar", name) if name in self.SCALARS else None)
                if name in ("vec2", "vec3", "vec4"):
                    ty = ("vec", int(name[3]), None)  # element type inferred from the arguments
                return Node("call", ty or name, self.parse_args())
            return Node("id", name)
        raise SyntaxError(f"unexpected {tok.text!r}")

    def parse_args(self):
        self.expect("(")
        args = []
        while not self.accept(")"):
            args.append(self.parse_expr())
            self.accept(",")
        return args

    def parse_postfix(self, e):
        while True:
            if self.accept("."):
                e = Node("member", e, self.next().text)
            elif self.accept("["):
                idx = self.parse_expr()
                self.expect("]")
                e = Node("index", e, idx)
            else:
                return e


def parse_number(text):
    t = text
    if t.startswith(("0x", "0X")):
        suf = t[-1] if t[-1] in "iu" else ""
        v = int(t[:-1] if suf else t, 16)
        return ({"i": "i32", "u": "u32"}.get(suf, "ai"), v)
    suf = t[-1] if t[-1] in "fhiu" else ""
    body = t[:-1] if suf else t
    is_float = any(ch in body for ch in ".eE") or suf in ("f", "h")
    if is_float:
        return ({"f": "f32", "h": "f16"}.get(suf, "af"), float(body))
    return ({"i": "i32", "u": "u32"}.get(suf, "ai"), int(body))


# ---------------------------------------------------------------- values -------------------

DT = {"f32": np.float32, "f16": np.float16, "i32": np.int32, "u32": np.uint32, "bool": np.bool_,
      "af": np.float64, "ai": np.int64}
FLOATS = ("f32", "f16", "af")


@dataclass
class Val:
    """el: element type; n: 0 for a scalar, else the vector width; v: array shaped (L,) /
    (L, n), or (1,) / (1, n) for a value uniform over the lanes (broadcasts)."""
    el: str
    n: int
    v: np.ndarray

    @property
    def abstract(self):
        return self.el in ("af", "ai")


class SVal(dict):
    """A struct value: field name -> Val (each over the lanes)."""

    def __init__(self, name, fields):
        super().__init__(fields)
        self.name = name


def sel(mask, new, old):
    """new where mask, old elsewhere, for a Val or a struct value."""
    if isinstance(new, SVal):
        return SVal(new.name, {k: sel(mask, new[k], old[k]) for k in new})
    return select_lanes(mask, new, old)


def widen(v, L):
    """A Val or struct value broadcast to L lanes."""
    if isinstance(v, SVal):
        return SVal(v.name, {k: widen(x, L) for k, x in v.items()})
    if v.v.shape[0] != L:
        return Val(v.el, v.n, np.broadcast_to(v.v, (L,) + v.v.shape[1:]).copy())
    return v


def _libm():
    lib = ctypes.CDLL(ctypes.util.find_library("m") or "libm.so.6")
    fns = {}
    for name in ("sinf", "cosf", "tanf", "expf", "exp2f", "logf", "log2f", "powf", "atan2f", "atanf", "asinf",
                 "acosf", "sinhf", "coshf", "tanhf"):
        f = getattr(lib, name)
        nargs = 2 if name in ("powf", "atan2f") else 1
        f.argtypes = [ctypes.c_float] * nargs
        f.restype = ctypes.c_float
        fns[name] = f
    return fns


_LIBM = _libm()


def _map_f32(fname, *arrays):
    """Applies a C library single-precision function elementwise."""
    f = _LIBM[fname]
    arrs = np.broadcast_arrays(*[np.asarray(a, np.float32) for a in arrays])
    out = np.empty(arrs[0].shape, np.float32)
    flat = [a.ravel() for a in arrs]
    o = out.ravel()
    for k in range(o.size):
        o[k] = f(*(float(a[k]) for a in flat))
    return out


def convert(x: Val, el: str) -> Val:
    """Value conversion to element type el (WGSL's conversion rules)."""
    if x.el == el:
        return x
    v = x.v
    if el in ("f32", "f16", "af"):
        if x.el == "bool":
            return Val(el, x.n, v.astype(DT[el]))
        return Val(el, x.n, np.asarray(v, np.float64 if x.el in ("af", "ai") else v.dtype).astype(DT[el]))
    if el in ("i32", "u32"):
        if x.el in FLOATS:
            lo, hi = (-2 ** 31, 2 ** 31 - 128) if el == "i32" else (0, 2 ** 32 - 256)
            f = np.trunc(np.nan_to_num(v.astype(np.float64)))
            return Val(el, x.n, np.clip(f, lo, hi).astype(np.int64).astype(DT[el]))
        if x.el in ("i32", "u32", "ai"):  # bit reinterpretation between 32-bit integers
            return Val(el, x.n, (v.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32).view(np.int32).astype(DT[el])
                       if el == "i32" else (v.astype(np.int64) & 0xFFFFFFFF).astype(np.uint32))
        if x.el == "bool":
            return Val(el, x.n, v.astype(DT[el]))
    if el == "bool":
        return Val(el, x.n, v != 0)
    raise TypeError(f"cannot convert {x.el} to {el}")


def concretize(x: Val) -> Val:
    return convert(x, {"af": "f32", "ai": "i32"}[x.el]) if x.abstract else x


def unify(a: Val, b: Val):
    """Brings two operands to one element type (abstract operands take the concrete type)."""
    if a.el == b.el:
        return a, b
    if a.abstract and b.abstract:
        return convert(a, "af"), convert(b, "af")
    if a.abstract:
        return convert(a, b.el), b
    if b.abstract:
        return a, convert(b, a.el)
    raise TypeError(f"mixed types {a.el} and {b.el}")


def _bc(a: Val, b: Val):
    """numpy operands with a scalar broadcast over a vector's components."""
    av, bv = a.v, b.v
    if a.n and not b.n:
        bv = bv[..., None]
    elif b.n and not a.n:
        av = av[..., None]
    return av, bv, max(a.n, b.n)


def binop(op: str, a: Val, b: Val) -> Val:
    if op in ("<<", ">>"):
        sh = (b.v.astype(np.int64) & 31)
        base = concretize(a) if not (a.abstract and b.abstract) else a
        av, bv, n = _bc(base, Val(base.el, b.n, sh))
        r = (av.astype(np.int64) << bv) if op == "<<" else (av.astype(np.int64) >> bv)
        return convert(Val("ai", n, r), base.el) if not base.abstract else Val("ai", n, r)
    a, b = unify(a, b)
    av, bv, n = _bc(a, b)
    el = a.el
    if op in ("==", "!=", "<", "<=", ">", ">="):
        f = {"==": np.equal, "!=": np.not_equal, "<": np.less, "<=": np.less_equal, ">": np.greater,
             ">=": np.greater_equal}[op]
        return Val("bool", n, f(av, bv))
    if op in ("&&", "||", "&", "|", "^"):
        if el == "bool":
            f = {"&&": np.logical_and, "||": np.logical_or, "&": np.logical_and, "|": np.logical_or,
                 "^": np.logical_xor}[op]
        else:
            f = {"&": np.bitwise_and, "|": np.bitwise_or, "^": np.bitwise_xor}[op]
        return Val(el, n, f(av, bv))
    with np.errstate(all="ignore"):
        if op == "+":
            r = av + bv
        elif op == "-":
            r = av - bv
        elif op == "*":
            r = av * bv
        elif op == "/":
            if el in FLOATS:
                r = av / bv
            else:  # truncating integer division; x / 0 = x (WGSL)
                a64, b64 = av.astype(np.int64), bv.astype(np.int64)
                safe = np.where(b64 == 0, 1, b64)
                r = np.where(b64 == 0, a64, np.trunc(a64 / safe).astype(np.int64))
        elif op == "%":
            if el in FLOATS:
                r = np.fmod(av, bv)  # x - y * trunc(x / y)
            else:
                a64, b64 = av.astype(np.int64), bv.astype(np.int64)
                safe = np.where(b64 == 0, 1, b64)
                r = np.where(b64 == 0, 0, np.fmod(a64, safe))
        else:
            raise SyntaxError(op)
    if el in ("i32", "u32"):
        r = (np.asarray(r).astype(np.int64) & 0xFFFFFFFF).astype(np.uint32)
        r = r.view(np.int32) if el == "i32" else r
    return Val(el, n, np.asarray(r).astype(DT[el]))


def select_lanes(mask, new: Val, old: Val) -> Val:
    """new where mask, old elsewhere (mask is a lane mask, (L,))."""
    m = mask[:, None] if new.n else mask
    return Val(new.el, new.n, np.where(m, new.v, old.v))


SWZ = {c: i for i, c in enumerate("xyzw")}
SWZ.update({c: i for i, c in enumerate("rgba")})


# ---------------------------------------------------------------- interpreter --------------

class Frame:
    def __init__(self, lanes):
        self.alive = np.ones(lanes, bool)
        self.ret = None
        self.scopes = [{}]

    def lookup(self, name):
        for s in reversed(self.scopes):
            if name in s:
                return s
        return None


class Program:
    """A parsed WGSL module with storage bindings; run() dispatches an entry point."""

    def __init__(self, src: str, transcendentals: str = "libm"):
        self.p = Parser(src).parse_module()
        self.transcendentals = transcendentals
        self.bindings = {}  # global name -> numpy array (storage) or dict of Val (uniform struct)
        self.uniform_vals = {}

    # storage / uniform binding
    def bind(self, name, array):
        self.bindings[name] = array

    def bind_uniform(self, name, floats):
        space, ty, _ = self.p.globals[name]
        fields = self.p.structs[ty[1]]
        vals, off = {}, 0
        f = np.asarray(floats, np.float32)
        for fname, fty in fields:
            n = fty[1] if fty[0] == "vec" else 0
            width = n or 1
            chunk = f[off:off + width]
            vals[fname] = Val(fty[2] if n else fty[1], n, chunk.reshape(1, n) if n else chunk.reshape(1))
            off += 4 if n in (3, 4) else width  # vec3/vec4 occupy 16 bytes in a uniform struct
        self.uniform_vals[name] = vals

    # dispatch
    def run(self, entry: str, workgroups):
        fn = self.p.funcs[entry]
        wgs = tuple(int(w) for w in workgroups) + (1,) * (3 - len(workgroups))
        size = [int(s) for s in fn.attrs["workgroup_size"]] + [1] * (3 - len(fn.attrs["workgroup_size"]))
        nwg = wgs[0] * wgs[1] * wgs[2]
        per = size[0] * size[1] * size[2]
        L = nwg * per
        lane = np.arange(L)
        wg_lin, loc_lin = lane // per, lane % per
        wg = np.stack([wg_lin % wgs[0], (wg_lin // wgs[0]) % wgs[1], wg_lin // (wgs[0] * wgs[1])], 1)
        loc = np.stack([loc_lin % size[0], (loc_lin // size[0]) % size[1], loc_lin // (size[0] * size[1])], 1)
        builtins = {
            "global_invocation_id": Val("u32", 3, (wg * np.array(size) + loc).astype(np.uint32)),
            "local_invocation_id": Val("u32", 3, loc.astype(np.uint32)),
            "local_invocation_index": Val("u32", 0, loc_lin.astype(np.uint32)),
            "workgroup_id": Val("u32", 3, wg.astype(np.uint32)),
            "num_workgroups": Val("u32", 3, np.tile(np.array(wgs, np.uint32), (L, 1))),
        }
        self.L, self.wg_of_lane = L, wg_lin
        self.workgroup_mem = {}
        for name, (space, ty, _) in self.p.globals.items():
            if space and space[0] == "workgroup":
                count = int(self.const_eval(ty[2]).v.reshape(-1)[0])
                self.workgroup_mem[name] = np.zeros((nwg, count), DT[ty[1][1]])
        fr = Frame(L)
        for pname, pty, bname in fn.params:
            fr.scopes[0][pname] = builtins[bname]
        self.exec_block(fn.body, fr, np.ones(L, bool))

    def const_eval(self, e):
        fr = Frame(1)
        self.L = getattr(self, "L", 1)
        return self.eval(e, fr, np.ones(1, bool))

    # statements
    def exec_block(self, stmts, fr, mask):
        fr.scopes.append({})
        try:
            for s in stmts:
                mask = mask & fr.alive & ~getattr(fr, "broken", np.zeros_like(mask)) & \
                    ~getattr(fr, "continued", np.zeros_like(mask))
                if not mask.any():
                    break
                self.exec_stmt(s, fr, mask)
        finally:
            fr.scopes.pop()

    def exec_stmt(self, s, fr, mask):
        k = s.kind
        if k == "decl":
            name, ty, init, how = s.a, s.b, s.c, s.d
            if init is None:
                v = self.zero(ty)
            else:
                v = self.eval(init, fr, mask)
                if isinstance(v, SVal):
                    pass
                elif ty is not None:
                    v = convert(v, ty[1] if ty[0] == "scalar" else ty[2])
                else:
                    v = concretize(v)
            fr.scopes[-1][name] = widen(v, self.L)
        elif k == "assign":
            lhs, op, rhs = s.a, s.b, s.c
            val = self.eval(rhs, fr, mask)
            if op != "=":
                val = binop(op[:-1], self.eval(lhs, fr, mask), val)
            self.store(lhs, val, fr, mask)
        elif k == "expr":
            self.eval(s.a, fr, mask)
        elif k == "block":
            self.exec_block(s.a, fr, mask)
        elif k == "if":
            c = self.lane_bool(self.eval(s.a, fr, mask))
            tm, em = mask & c, mask & ~c
            if tm.any():
                self.exec_block(s.b, fr, tm)
            if s.c is not None and em.any():
                self.exec_block(s.c, fr, em)
        elif k == "for":
            init, cond, upd, body = s.a, s.b, s.c, s.d
            fr.scopes.append({})
            outer_broken = getattr(fr, "broken", None)
            outer_cont = getattr(fr, "continued", None)
            fr.broken = np.zeros(self.L, bool)
            try:
                if init is not None:
                    self.exec_stmt(init, fr, mask)
                live = mask.copy()
                while True:
                    live = live & fr.alive & ~fr.broken
                    if cond is not None:
                        live = live & self.lane_bool(self.eval(cond, fr, live))
                    if not live.any():
                        break
                    fr.continued = np.zeros(self.L, bool)
                    self.exec_block(body, fr, live)
                    fr.continued = np.zeros(self.L, bool)
                    live = live & fr.alive & ~fr.broken
                    if upd is not None and live.any():
                        self.exec_stmt(upd, fr, live)
            finally:
                fr.scopes.pop()
                fr.broken = outer_broken if outer_broken is not None else np.zeros(self.L, bool)
                fr.continued = outer_cont if outer_cont is not None else np.zeros(self.L, bool)
        elif k == "break":
            fr.broken = fr.broken | mask
        elif k == "continue":
            fr.continued = fr.continued | mask
        elif k == "return":
            if s.a is not None:
                v = self.eval(s.a, fr, mask)
                if isinstance(v, SVal):
                    v = widen(v, self.L)
                    fr.ret = v if fr.ret is None else sel(mask, v, fr.ret)
                else:
                    if fr.ret is None:
                        fr.ret = Val(v.el, v.n, np.zeros((self.L,) + v.v.shape[1:], v.v.dtype))
                    v = convert(v, fr.ret.el) if v.el != fr.ret.el else v
                    fr.ret = select_lanes(mask, Val(v.el, v.n, np.broadcast_to(v.v, fr.ret.v.shape)), fr.ret)
            fr.alive = fr.alive & ~mask
        else:
            raise SyntaxError(k)

    def struct_layout(self, name):
        """(field, element, width, float offset) of a struct of scalars and vectors, packed
        as a storage array of vec4 / f32 fields lays them out."""
        out, off = [], 0
        for fname, fty in self.p.structs[name]:
            n = fty[1] if fty[0] == "vec" else 0
            el = fty[2] if n else fty[1]
            out.append((fname, el, n, off))
            off += n or 1
        return out

    def zero(self, ty):
        if ty[0] == "struct":
            return SVal(ty[1], {f: Val(el, n, np.zeros((self.L, n) if n else self.L, DT[el]))
                                for f, el, n, _ in self.struct_layout(ty[1])})
        if ty[0] == "scalar":
            return Val(ty[1], 0, np.zeros(self.L, DT[ty[1]]))
        if ty[0] == "vec":
            return Val(ty[2], ty[1], np.zeros((self.L, ty[1]), DT[ty[2]]))
        raise TypeError(ty)

    def lane_bool(self, v: Val):
        b = v.v if v.el == "bool" else v.v != 0
        return np.broadcast_to(b, (self.L,)) if b.shape[0] == 1 else b

    def store(self, lhs, val, fr, mask):
        if lhs.kind == "id":
            scope = fr.lookup(lhs.a)
            if scope is None:
                raise NameError(lhs.a)
            old = scope[lhs.a]
            if isinstance(old, SVal):
                scope[lhs.a] = sel(mask, widen(val, self.L), old)
                return
            val = convert(val, old.el) if val.el != old.el else val
            if val.n == 0 and old.n:
                val = Val(val.el, old.n, np.broadcast_to(val.v[..., None], old.v.shape))
            scope[lhs.a] = select_lanes(mask, Val(val.el, val.n, np.broadcast_to(val.v, old.v.shape)), old)
        elif lhs.kind == "member":  # component write: v.x = ..., v.xyz is not assignable in WGSL
            base = lhs.a
            scope = fr.lookup(base.a)
            old = scope[base.a]
            if isinstance(old, SVal):  # struct field: s.f = ...
                f = old[lhs.b]
                val = convert(val, f.el) if val.el != f.el else val
                if val.n == 0 and f.n:
                    val = Val(val.el, f.n, np.broadcast_to(val.v[..., None], f.v.shape))
                new = dict(old)
                new[lhs.b] = select_lanes(mask, Val(f.el, f.n, np.broadcast_to(val.v, f.v.shape)), f)
                scope[base.a] = SVal(old.name, new)
                return
            comp = SWZ[lhs.b]
            val = convert(val, old.el) if val.el != old.el else val
            newv = old.v.copy()
            newv[:, comp] = np.where(mask, np.broadcast_to(val.v, (self.L,)), old.v[:, comp])
            scope[base.a] = Val(old.el, old.n, newv)
        elif lhs.kind == "index" and isinstance(val, SVal):  # a struct into an array of structs
            arr = self.bindings[lhs.a.a]
            idx = self.eval(lhs.b, fr, mask)
            ii = np.broadcast_to(idx.v.astype(np.int64), (self.L,))
            if mask.any() and (ii[mask].min() < 0 or ii[mask].max() >= arr.shape[0]):
                raise IndexError(f"store out of bounds in {lhs.a.a}")
            for f, el, n, off in self.struct_layout(val.name):
                fv = widen(val[f], self.L).v
                arr[ii[mask], off:off + (n or 1)] = (fv[mask] if n else fv[mask][:, None]).astype(arr.dtype)
        elif lhs.kind == "index":
            arr, el, n = self.buffer(lhs.a)
            idx = self.eval(lhs.b, fr, mask)
            ii = np.broadcast_to(idx.v.astype(np.int64), (self.L,))
            val = convert(val, el) if val.el != el else val
            vv = np.broadcast_to(val.v, (self.L,) + ((n,) if n else ()))
            if lhs.a.a in self.workgroup_mem:
                w = self.wg_of_lane[mask]
                arr[w, ii[mask]] = vv[mask]
            else:
                if mask.any() and (ii[mask].min() < 0 or ii[mask].max() >= arr.shape[0]):
                    raise IndexError(f"store out of bounds in {lhs.a.a}")
                arr[ii[mask]] = vv[mask]
        else:
            raise SyntaxError(f"cannot assign to {lhs.kind}")

    def buffer(self, node):
        name = node.a
        if name in self.workgroup_mem:
            arr = self.workgroup_mem[name]
            ty = self.p.globals[name][1][1]
        else:
            arr = self.bindings[name]
            ty = self.p.globals[name][1][1]
        if ty[0] == "atomic":
            ty = ty[1]
        if ty[0] == "struct":
            return arr, ("struct", ty[1]), 0
        return arr, (ty[1] if ty[0] == "scalar" else ty[2]), (ty[1] if ty[0] == "vec" else 0)

    # expressions
    def eval(self, e, fr, mask) -> Val:
        k = e.kind
        if k == "lit":
            el, v = e.a
            return Val(el, 0, np.array([v], DT[el]))
        if k == "id":
            scope = fr.lookup(e.a)
            if scope is not None:
                return scope[e.a]
            if e.a in self.p.consts:
                ty, ex = self.p.consts[e.a]
                v = self.eval(ex, Frame(1), np.ones(1, bool))
                return convert(v, ty[1] if ty[0] == "scalar" else ty[2]) if ty else v
            if e.a in self.uniform_vals:
                return self.uniform_vals[e.a]
            raise NameError(e.a)
        if k == "member":
            if e.a.kind == "id" and e.a.a in self.uniform_vals:
                return self.uniform_vals[e.a.a][e.b]
            base = self.eval(e.a, fr, mask)
            if isinstance(base, dict):
                return base[e.b]
            comps = [SWZ[c] for c in e.b]
            if len(comps) == 1:
                return Val(base.el, 0, base.v[:, comps[0]])
            return Val(base.el, len(comps), base.v[:, comps])
        if k == "index":
            arr, el, n = self.buffer(e.a)
            idx = self.eval(e.b, fr, mask)
            ii = np.broadcast_to(idx.v.astype(np.int64), (self.L,))
            ii = np.where(mask, ii, 0)  # lanes that do not run this read nothing
            if e.a.a in self.workgroup_mem:
                return Val(el, n, arr[self.wg_of_lane, ii])
            if mask.any() and (ii[mask].min() < 0 or ii[mask].max() >= arr.shape[0]):
                raise IndexError(f"read out of bounds in {e.a.a}")
            if isinstance(el, tuple):  # array of structs: one row of floats per element
                rows = arr[ii]
                return SVal(el[1], {f: Val(fe, fn, rows[:, off:off + fn] if fn else rows[:, off])
                                    for f, fe, fn, off in self.struct_layout(el[1])})
            return Val(el, n, arr[ii])
        if k == "un":
            if e.a == "&":
                return Node("ref", e.b.a)
            x = self.eval(e.b, fr, mask)
            if e.a == "-":
                return Val(x.el, x.n, (-x.v).astype(x.v.dtype))
            if e.a == "!":
                return Val("bool", x.n, ~x.v)
            if e.a == "~":
                return Val(x.el, x.n, ~x.v)
            raise SyntaxError(e.a)
        if k == "bin":
            return binop(e.a, self.eval(e.b, fr, mask), self.eval(e.c, fr, mask))
        if k == "call":
            return self.call(e.a, e.b, fr, mask)
        raise SyntaxError(k)

    def call(self, callee, argn, fr, mask):
        if isinstance(callee, tuple):  # type constructor / conversion
            args = [self.eval(a, fr, mask) for a in argn]
            if callee[0] == "scalar":
                return convert(args[0], callee[1])
            n, el = callee[1], callee[2]
            if el is None:
                el = concretize(args[0]).el if not all(a.abstract for a in args) else "af"
            if len(args) == 1 and args[0].n == n:
                return convert(args[0], el)
            if len(args) == 1 and args[0].n == 0:
                a = convert(args[0], el)
                return Val(el, n, np.repeat(a.v[..., None], n, axis=-1))
            cols = []
            for a in args:
                a = convert(a, el)
                cols.extend([a.v] if a.n == 0 else [a.v[:, j] for j in range(a.n)])
            rows = max(c.shape[0] for c in cols)
            return Val(el, n, np.stack([np.broadcast_to(c, (rows,)) for c in cols], 1))
        name = callee
        if name in self.p.funcs:
            f = self.p.funcs[name]
            args = [self.eval(a, fr, mask) for a in argn]
            sub = Frame(self.L)
            sub.alive = mask.copy()
            for (pname, pty, _), a in zip(f.params, args):
                if not isinstance(a, SVal):
                    a = convert(a, pty[1] if pty[0] == "scalar" else pty[2])
                sub.scopes[0][pname] = widen(a, self.L)
            self.exec_block(f.body, sub, mask)
            return sub.ret
        return self.builtin(name, argn, fr, mask)

    def builtin(self, name, argn, fr, mask):
        if name == "workgroupBarrier" or name == "storageBarrier":
            return None
        if name == "arrayLength":
            ref = argn[0]
            buf = self.bindings[ref.b.a]
            return Val("u32", 0, np.array([buf.shape[0]], np.uint32))
        if name.startswith("atomic"):
            return self.atomic(name, argn, fr, mask)
        args = [self.eval(a, fr, mask) for a in argn]
        if name in ("any", "all"):
            v = args[0].v
            return Val("bool", 0, v.any(-1) if name == "any" else v.all(-1))
        if name == "select":  # select(f, t, cond)
            f_, t_ = unify(args[0], args[1])
            c = args[2].v
            fv, tv, n = _bc(f_, t_)
            if f_.n and not args[2].n:
                c = c[..., None]
            return Val(f_.el, n, np.where(c, tv, fv))
        if all(a.abstract for a in args):  # constant expression in float64
            args = [convert(a, "af") for a in args]
        else:
            first = next(a for a in args if not a.abstract)
            args = [convert(a, first.el) if a.abstract else a for a in args]
        el = args[0].el
        f32 = el != "af"

        def mk(v, n=None):
            return Val(el, args[0].n if n is None else n, np.asarray(v).astype(DT[el]))

        def bc(*xs):
            out, n = [], max(x.n for x in xs)
            for x in xs:
                out.append(x.v[..., None] if (n and not x.n) else x.v)
            return out, n

        if name in ("max", "min"):
            (a, b), n = bc(*args)
            return Val(el, n, np.where(a < b, b, a) if name == "max" else np.where(b < a, b, a))
        if name == "clamp":
            (x, lo, hi), n = bc(*args)
            m = np.where(x < lo, lo, x)
            return Val(el, n, np.where(hi < m, hi, m))
        if name == "abs":
            return mk(np.abs(args[0].v))
        if name == "sqrt":
            return mk(np.sqrt(args[0].v))
        if name == "floor":
            return mk(np.floor(args[0].v))
        if name == "round":  # halfway cases to the even integer
            return mk(np.rint(args[0].v))
        if name == "ceil":
            return mk(np.ceil(args[0].v))
        if name == "fract":
            x = args[0]
            return binop("-", x, mk(np.floor(x.v)))
        if name == "sign":
            return mk(np.sign(args[0].v))
        if name == "mix":  # e1 * (1 - e3) + e2 * e3
            a, b, t = args
            one = Val("af", 0, np.array([1.0]))
            return binop("+", binop("*", a, binop("-", one, t)), binop("*", b, t))
        if name == "smoothstep":
            lo, hi, x = args
            t = self.builtin_val("clamp", [binop("/", binop("-", x, lo), binop("-", hi, lo)),
                                           Val("af", 0, np.array([0.0])), Val("af", 0, np.array([1.0]))])
            return binop("*", binop("*", t, t), binop("-", Val("af", 0, np.array([3.0])),
                                                         binop("*", Val("af", 0, np.array([2.0])), t)))
        if name == "dot":
            a, b = args
            r = None
            for j in range(a.n):
                term = binop("*", Val(el, 0, a.v[:, j]), Val(el, 0, b.v[:, j]))
                r = term if r is None else binop("+", r, term)
            return r
        if name == "length":
            a = args[0]
            if a.n == 0:
                return mk(np.abs(a.v))
            d = self.builtin_val("dot", [a, a])
            return Val(el, 0, np.sqrt(d.v).astype(DT[el]))
        if name == "distance":
            return self.builtin_val("length", [binop("-", args[0], args[1])])
        if name == "normalize":
            a = args[0]
            ln = self.builtin_val("length", [a])
            return binop("/", a, ln)
        if name == "cross":
            a, b = args

            def c(i):
                return Val(el, 0, a.v[:, i]), Val(el, 0, b.v[:, i])

            (ax, bx), (ay, by), (az, bz) = c(0), c(1), c(2)
            x = binop("-", binop("*", ay, bz), binop("*", az, by))
            y = binop("-", binop("*", az, bx), binop("*", ax, bz))
            z = binop("-", binop("*", ax, by), binop("*", ay, bx))
            rows = max(x.v.shape[0], y.v.shape[0], z.v.shape[0])
            return Val(el, 3, np.stack([np.broadcast_to(q.v, (rows,)) for q in (x, y, z)], 1))
        libf = {"sin": "sinf", "cos": "cosf", "tan": "tanf", "exp": "expf", "exp2": "exp2f", "log": "logf",
                "log2": "log2f", "pow": "powf", "atan2": "atan2f", "atan": "atanf", "asin": "asinf", "acos": "acosf",
                "sinh": "sinhf", "cosh": "coshf", "tanh": "tanhf"}
        if name in libf:
            if not f32:
                fn = {"pow": math.pow, "atan2": math.atan2, "exp2": lambda x: 2.0 ** x}.get(name) or getattr(math, name)
                vs = np.broadcast_arrays(*[a.v for a in args])
                return mk(np.vectorize(fn)(*vs))
            if el == "f16":
                raise NotImplementedError("f16 transcendentals")
            vs, n = bc(*args)
            if self.transcendentals == "f64":
                fn = {"pow": math.pow, "atan2": math.atan2, "exp2": lambda x: 2.0 ** x}.get(name) or getattr(math, name)
                ws = np.broadcast_arrays(*[np.asarray(v, np.float64) for v in vs])
                return Val(el, n, np.vectorize(fn, otypes=[np.float64])(*ws).astype(np.float32))
            return Val(el, n, _map_f32(libf[name], *vs))
        raise NameError(f"builtin {name}")

    def builtin_val(self, name, vals):
        """Calls a builtin on already-evaluated values."""
        tmp = Frame(self.L)
        nodes = []
        for i, v in enumerate(vals):
            tmp.scopes[0][f"__a{i}"] = v
            nodes.append(Node("id", f"__a{i}"))
        return self.builtin(name, nodes, tmp, np.ones(self.L, bool))

    def atomic(self, name, argn, fr, mask):
        """atomicAdd / atomicLoad / atomicStore / atomicMax / atomicMin on storage arrays of
        atomic<u32> or atomic<i32>: integer atomics commute, so lanes apply in lane order."""
        ref = argn[0]
        target = ref.b  # &arr[idx]
        arr, el, _ = self.buffer(target.a)
        idx = np.broadcast_to(self.eval(target.b, fr, mask).v.astype(np.int64), (self.L,))
        if name == "atomicLoad":
            return Val(el, 0, arr[np.where(mask, idx, 0)])
        val = convert(self.eval(argn[1], fr, mask), el)
        vv = np.broadcast_to(val.v, (self.L,))
        old = np.zeros(self.L, arr.dtype)
        for lane in np.nonzero(mask)[0]:
            i = idx[lane]
            old[lane] = arr[i]
            if name == "atomicAdd":
                arr[i] = (int(arr[i]) + int(vv[lane])) & 0xFFFFFFFF if el == "u32" else np.int32(arr[i] + vv[lane])
            elif name == "atomicStore":
                arr[i] = vv[lane]
            elif name == "atomicMax":
                arr[i] = max(arr[i], vv[lane])
            elif name == "atomicMin":
                arr[i] = min(arr[i], vv[lane])
            else:
                raise NameError(name)
        return Val(el, 0, old)


def wgsl_from_ts(ts_source: str, export_name: str) -> str:
    """The text of `export const <name> = /* wgsl */ \\`...\\`;` in a TypeScript module."""
    m = re.search(r"export const " + re.escape(export_name) + r"\s*=\s*(?:/\*\s*wgsl\s*\*/)?\s*`(.*?)`;", ts_source, re.S)
    if not m:
        raise ValueError(f"{export_name} not found")
    body = m.group(1)
    if "${" in body:
        raise ValueError(f"{export_name} has template substitutions")
    return body
