"""WGSL -> C++ source translator: the recipe that compiles the reference's
own shader math for the CPU oracle.  TEST INFRASTRUCTURE ONLY.

It reads the reference's WGSL where it lies (src/shaders/*.wgsl) and writes
C++ into oracle/_ref/ (git-ignored); nothing it emits is committed.  The
emitted code keeps WGSL semantics via oracle/wgsl_rt.hpp:

* full static typing (WGSL is explicitly typed at every function boundary),
  so abstract literals are concretised exactly as WGSL does -- abstract
  constant sub-expressions are evaluated in double / int64 and converted
  once, concrete f32 arithmetic stays f32 (no silent promotion to double);
* every binary expression is parenthesised, `%`, `/`, `<<`, `>>` go through
  wg::mod / wg::div / wg::shl / wg::shr (WGSL integer and float rules);
* user functions are renamed `U_<name>` (no clash with libm), module-scope
  storage/uniform variables become thread_local pointers / values that the
  glue (oracle/ref_glue.cpp) binds before calling an entry point.

Only the subset of WGSL the reference shaders use is supported; anything
else raises, so a silently wrong translation cannot happen.
"""
from __future__ import annotations

import re
import sys

# --------------------------------------------------------------------------
# tokenizer

_TOKEN_RE = re.compile(r"""
    (?P<ws>\s+)
  | (?P<lcomment>//[^\n]*)
  | (?P<bcomment>/\*.*?\*/)
  | (?P<float>(?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?[fh]?|\d+[eE][+-]?\d+[fh]?|\d+[fh])
  | (?P<hex>0[xX][0-9a-fA-F]+[iu]?)
  | (?P<int>\d+[iu]?)
  | (?P<ident>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op><<=|>>=|->|==|!=|<=|>=|&&|\|\||<<|>>|\+=|-=|\*=|/=|%=|&=|\|=|\^=|\+\+|--|[-+*/%<>=!&|^~(){}\[\],;:.@])
""", re.S | re.X)


class Tok:
    __slots__ = ("kind", "text", "line")

    def __init__(self, kind, text, line):
        self.kind, self.text, self.line = kind, text, line

    def __repr__(self):
        return f"{self.kind}:{self.text}@{self.line}"


def tokenize(src: str):
    out, pos, line = [], 0, 1
    while pos < len(src):
        m = _TOKEN_RE.match(src, pos)
        if not m:
            raise SyntaxError(f"line {line}: cannot tokenize {src[pos:pos + 30]!r}")
        kind = m.lastgroup
        text = m.group(kind)
        if kind not in ("ws", "lcomment", "bcomment"):
            out.append(Tok(kind, text, line))
        line += text.count("\n")
        pos = m.end()
    out.append(Tok("eof", "", line))
    return out


# --------------------------------------------------------------------------
# types: tuples
#   ("s", k)  scalar, k in f32 i32 u32 bool af ai
#   ("v", n, k)  vector
#   ("a", elemtype, n|None)  array (None = runtime-sized)
#   ("st", name)  struct
#   ("at", k)  atomic
#   ("p", t)  pointer (only for &expr passed to atomics)
#   ("void",)

F32, I32, U32, BOOL, AF, AI = (("s", k) for k in ("f32", "i32", "u32", "bool", "af", "ai"))
VOID = ("void",)
SCALAR_NAMES = {"f32": F32, "i32": I32, "u32": U32, "bool": BOOL}
VEC_SHORT = {}
for _n in (2, 3, 4):
    for _suf, _k in (("f", "f32"), ("i", "i32"), ("u", "u32")):
        VEC_SHORT[f"vec{_n}{_suf}"] = ("v", _n, _k)
CPP_SCALAR = {"f32": "float", "i32": "int32_t", "u32": "uint32_t", "bool": "bool",
              "af": "double", "ai": "int64_t"}

CPP_KEYWORDS = set("""alignas alignof and and_eq asm auto bitand bitor char char8_t char16_t
char32_t class compl concept consteval constexpr constinit const_cast co_await co_return
co_yield decltype delete do double dynamic_cast enum explicit export extern float friend goto
inline int long mutable namespace new noexcept not not_eq nullptr operator or or_eq private
protected public register reinterpret_cast requires short signed sizeof static static_assert
static_cast template this thread_local throw try typedef typeid typename union unsigned using
virtual volatile wchar_t xor xor_eq main""".split())


def is_abstract(t):
    return t[0] == "s" and t[1] in ("af", "ai")


def scal_kind(t):
    if t[0] == "s":
        return t[1]
    if t[0] == "v":
        return t[2]
    if t[0] == "at":
        return t[1]
    raise TypeError(f"no scalar kind for {t}")


def with_kind(t, k):
    if t[0] == "s":
        return ("s", k)
    if t[0] == "v":
        return ("v", t[1], k)
    raise TypeError(t)


def concretize(t):
    """Default concretisation of an abstract type (WGSL: af->f32, ai->i32)."""
    if t[0] == "s" and t[1] == "af":
        return F32
    if t[0] == "s" and t[1] == "ai":
        return I32
    return t


# --------------------------------------------------------------------------
# AST


class Node:
    pass


class Lit(Node):
    def __init__(self, text, kind):
        self.text, self.kind = text, kind


class Ident(Node):
    def __init__(self, name):
        self.name = name


class Call(Node):
    def __init__(self, name, targs, args):
        self.name, self.targs, self.args = name, targs, args


class Member(Node):
    def __init__(self, obj, name):
        self.obj, self.name = obj, name


class Index(Node):
    def __init__(self, obj, idx):
        self.obj, self.idx = obj, idx


class Unary(Node):
    def __init__(self, op, e):
        self.op, self.e = op, e


class Binary(Node):
    def __init__(self, op, a, b):
        self.op, self.a, self.b = op, a, b


BIN_PREC = {
    "||": 1, "&&": 2, "|": 3, "^": 4, "&": 5,
    "==": 6, "!=": 6, "<": 7, ">": 7, "<=": 7, ">=": 7,
    "<<": 8, ">>": 8, "+": 9, "-": 9, "*": 10, "/": 10, "%": 10,
}


# --------------------------------------------------------------------------
# parser


class Parser:
    def __init__(self, toks):
        self.t = toks
        self.i = 0

    def peek(self, k=0):
        return self.t[self.i + k]

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def at(self, text):
        return self.t[self.i].text == text and self.t[self.i].kind in ("op", "ident")

    def eat(self, text):
        if self.at(text):
            self.i += 1
            return True
        return False

    def expect(self, text):
        tok = self.next()
        if tok.text != text:
            raise SyntaxError(f"line {tok.line}: expected {text!r}, got {tok.text!r}")
        return tok

    def ident(self):
        tok = self.next()
        if tok.kind != "ident":
            raise SyntaxError(f"line {tok.line}: expected identifier, got {tok.text!r}")
        return tok.text

    # ---- types
    def close_angle(self):
        tok = self.peek()
        if tok.text == ">":
            self.i += 1
        elif tok.text == ">>":
            tok.text = ">"  # split '>>' into two closers
        elif tok.text == ">=":
            tok.text = "="
        else:
            raise SyntaxError(f"line {tok.line}: expected '>'")

    def parse_type(self):
        name = self.ident()
        if name in SCALAR_NAMES:
            return SCALAR_NAMES[name]
        if name in VEC_SHORT:
            return VEC_SHORT[name]
        if name in ("vec2", "vec3", "vec4"):
            self.expect("<")
            el = self.parse_type()
            self.close_angle()
            return ("v", int(name[3]), el[1])
        if name == "array":
            self.expect("<")
            el = self.parse_type()
            n = None
            if self.eat(","):
                n = self.parse_const_int()
            self.close_angle()
            return ("a", el, n)
        if name == "atomic":
            self.expect("<")
            el = self.parse_type()
            self.close_angle()
            return ("at", el[1])
        return ("st", name)

    def parse_const_int(self):
        tok = self.next()
        if tok.kind in ("int", "hex"):
            return int(tok.text.rstrip("iu"), 0)
        if tok.kind == "ident":
            return ("const", tok.text)
        raise SyntaxError(f"line {tok.line}: bad array size {tok.text}")

    def skip_attrs(self):
        attrs = []
        while self.at("@"):
            self.next()
            name = self.ident()
            args = []
            if self.at("("):
                depth = 0
                while True:
                    tok = self.next()
                    if tok.text == "(":
                        depth += 1
                    elif tok.text == ")":
                        depth -= 1
                        if depth == 0:
                            break
                    else:
                        args.append(tok.text)
            attrs.append((name, args))
        return attrs

    # ---- module
    def parse_module(self):
        items = []
        while self.peek().kind != "eof":
            attrs = self.skip_attrs()
            tok = self.peek()
            if tok.text == "struct":
                self.next()
                name = self.ident()
                self.expect("{")
                fields = []
                while not self.eat("}"):
                    self.skip_attrs()
                    fname = self.ident()
                    self.expect(":")
                    ftype = self.parse_type()
                    fields.append((fname, ftype))
                    self.eat(",")
                self.eat(";")
                items.append(("struct", name, fields))
            elif tok.text in ("const", "override"):
                self.next()
                name = self.ident()
                ty = None
                if self.eat(":"):
                    ty = self.parse_type()
                self.expect("=")
                e = self.parse_expr()
                self.expect(";")
                items.append(("const", name, ty, e))
            elif tok.text == "var":
                self.next()
                space = None
                if self.eat("<"):
                    space = [self.ident()]
                    while self.eat(","):
                        space.append(self.ident())
                    self.close_angle()
                name = self.ident()
                self.expect(":")
                ty = self.parse_type()
                init = None
                if self.eat("="):
                    init = self.parse_expr()
                self.expect(";")
                items.append(("var", name, space, ty, init))
            elif tok.text == "fn":
                self.next()
                name = self.ident()
                self.expect("(")
                params = []
                while not self.eat(")"):
                    self.skip_attrs()
                    pname = self.ident()
                    self.expect(":")
                    pty = self.parse_type()
                    params.append((pname, pty))
                    self.eat(",")
                ret = VOID
                if self.eat("->"):
                    self.skip_attrs()
                    ret = self.parse_type()
                body = self.parse_block()
                items.append(("fn", name, params, ret, body, attrs))
            elif tok.text == ";":
                self.next()
            else:
                raise SyntaxError(f"line {tok.line}: unexpected {tok.text!r} at module scope")
        return items

    # ---- statements
    def parse_block(self):
        self.expect("{")
        stmts = []
        while not self.eat("}"):
            stmts.append(self.parse_stmt())
        return stmts

    def parse_stmt(self):
        tok = self.peek()
        t = tok.text
        if t == "{":
            return ("block", self.parse_block())
        if t in ("let", "var", "const"):
            self.next()
            name = self.ident()
            ty = None
            if self.eat(":"):
                ty = self.parse_type()
            init = None
            if self.eat("="):
                init = self.parse_expr()
            self.expect(";")
            return ("decl", t, name, ty, init)
        if t == "if":
            self.next()
            cond = self.parse_expr()
            then = self.parse_block()
            other = None
            if self.eat("else"):
                if self.at("if"):
                    other = [self.parse_stmt()]
                else:
                    other = self.parse_block()
            return ("if", cond, then, other)
        if t == "for":
            self.next()
            self.expect("(")
            init = None if self.at(";") else self.parse_simple()
            self.expect(";")
            cond = None if self.at(";") else self.parse_expr()
            self.expect(";")
            upd = None if self.at(")") else self.parse_simple(no_semi=True)
            self.expect(")")
            body = self.parse_block()
            return ("for", init, cond, upd, body)
        if t == "while":
            self.next()
            cond = self.parse_expr()
            body = self.parse_block()
            return ("while", cond, body)
        if t == "loop":
            self.next()
            self.expect("{")
            body = []
            while not self.eat("}"):
                if self.at("continuing"):
                    raise NotImplementedError(f"line {tok.line}: continuing blocks")
                body.append(self.parse_stmt())
            return ("loop", body)
        if t == "switch":
            self.next()
            sel = self.parse_expr()
            self.expect("{")
            cases = []
            while not self.eat("}"):
                labels = []
                if self.eat("default"):
                    labels.append(None)
                else:
                    self.expect("case")
                    while True:
                        if self.eat("default"):
                            labels.append(None)
                        else:
                            labels.append(self.parse_expr())
                        if not self.eat(","):
                            break
                        if self.at(":") or self.at("{"):
                            break
                self.eat(":")
                body = self.parse_block()
                cases.append((labels, body))
            return ("switch", sel, cases)
        if t == "break":
            self.next()
            if self.at("if"):
                raise NotImplementedError("break if")
            self.expect(";")
            return ("break",)
        if t == "continue":
            self.next()
            self.expect(";")
            return ("continue",)
        if t == "return":
            self.next()
            e = None if self.at(";") else self.parse_expr()
            self.expect(";")
            return ("return", e)
        if t == "discard":
            self.next()
            self.expect(";")
            return ("discard",)
        s = self.parse_simple()
        self.expect(";")
        return s

    def parse_simple(self, no_semi=False):
        tok = self.peek()
        if tok.text in ("let", "var", "const"):
            self.next()
            name = self.ident()
            ty = None
            if self.eat(":"):
                ty = self.parse_type()
            init = None
            if self.eat("="):
                init = self.parse_expr()
            return ("decl", tok.text, name, ty, init)
        if tok.text == "_" and self.peek(1).text == "=":
            self.next()
            self.next()
            return ("phony", self.parse_expr())
        lhs = self.parse_expr()
        op = self.peek().text
        if op in ("=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>="):
            self.next()
            rhs = self.parse_expr()
            return ("assign", op, lhs, rhs)
        if op in ("++", "--"):
            self.next()
            return ("incdec", op, lhs)
        return ("expr", lhs)

    # ---- expressions
    def parse_expr(self, min_prec=1):
        lhs = self.parse_unary()
        while True:
            op = self.peek().text
            if self.peek().kind != "op" or op not in BIN_PREC:
                break
            prec = BIN_PREC[op]
            if prec < min_prec:
                break
            self.next()
            rhs = self.parse_expr(prec + 1)
            lhs = Binary(op, lhs, rhs)
        return lhs

    def parse_unary(self):
        tok = self.peek()
        if tok.kind == "op" and tok.text in ("-", "!", "~", "&", "*"):
            self.next()
            return Unary(tok.text, self.parse_unary())
        return self.parse_postfix(self.parse_primary())

    def parse_primary(self):
        tok = self.next()
        if tok.kind == "float":
            return Lit(tok.text, "float")
        if tok.kind in ("int", "hex"):
            return Lit(tok.text, "int")
        if tok.kind == "ident":
            if tok.text in ("true", "false"):
                return Lit(tok.text, "bool")
            name = tok.text
            targs = None
            # templated constructor / bitcast: name<...>(...)
            if self.at("<") and name in ("vec2", "vec3", "vec4", "array", "bitcast"):
                self.next()
                targs = [self.parse_type()]
                if self.eat(","):
                    targs.append(self.parse_const_int())
                self.close_angle()
            if self.at("("):
                self.next()
                args = []
                while not self.eat(")"):
                    args.append(self.parse_expr())
                    self.eat(",")
                return Call(name, targs, args)
            if targs is not None:
                raise SyntaxError(f"line {tok.line}: template without call")
            return Ident(name)
        if tok.text == "(":
            e = self.parse_expr()
            self.expect(")")
            return e
        raise SyntaxError(f"line {tok.line}: unexpected {tok.text!r} in expression")

    def parse_postfix(self, e):
        while True:
            if self.at("."):
                self.next()
                e = Member(e, self.ident())
            elif self.at("["):
                self.next()
                idx = self.parse_expr()
                self.expect("]")
                e = Index(e, idx)
            else:
                return e


# --------------------------------------------------------------------------
# type checker + emitter

FLOAT_UNARY = {"sin", "cos", "tan", "asin", "acos", "atan", "sinh", "cosh", "tanh", "asinh",
               "acosh", "atanh", "exp", "exp2", "log", "log2", "sqrt", "inverseSqrt", "floor",
               "ceil", "trunc", "round", "fract", "saturate", "degrees", "radians", "sign",
               "abs", "normalize", "countOneBits", "reverseBits"}
SAME_TYPE_N = {"atan2": 2, "pow": 2, "min": 2, "max": 2, "step": 2, "reflect": 2, "cross": 2,
               "clamp": 3, "smoothstep": 3, "fma": 3}
SWZ = {"x": 0, "y": 1, "z": 2, "w": 3, "r": 0, "g": 1, "b": 2, "a": 3}


class Emitter:
    def __init__(self, ns, skip_fns=()):
        self.ns = ns
        self.structs = {}  # name -> [(field, type)]
        self.consts = {}  # name -> type
        self.globals = {}  # name -> type
        self.fns = {}  # name -> (params, ret)
        self.scopes = []
        self.cur_ret = None
        self.out = []
        self.skip_fns = set(skip_fns)
        self.subst = {}  # id(Call node) -> temporary holding its value
        self.impure = set()  # user functions that (transitively) draw RNG / write state
        self.tmp_n = 0

    # ---- helpers
    def err(self, msg):
        raise TypeError(f"[{self.ns}] {msg}")

    def cname(self, name):
        return name + "_" if name in CPP_KEYWORDS else name

    def ctype(self, t):
        k = t[0]
        if k == "s":
            return CPP_SCALAR[t[1]]
        if k == "v":
            return f"wg::vec<{CPP_SCALAR[t[2]]}, {t[1]}>"
        if k == "a":
            n = t[2]
            if isinstance(n, tuple):
                n = self.cname(n[1])
            return f"std::array<{self.ctype(t[1])}, {n}>"
        if k == "st":
            return self.cname(t[1])
        if k == "at":
            return CPP_SCALAR[t[1]]
        if k == "void":
            return "void"
        self.err(f"no C++ type for {t}")

    def lookup(self, name):
        for sc in reversed(self.scopes):
            if name in sc:
                return sc[name]
        if name in self.consts:
            return self.consts[name]
        if name in self.globals:
            return self.globals[name]
        self.err(f"unknown identifier {name}")

    # ---- type inference
    def typeof(self, e):
        if isinstance(e, Lit):
            if e.kind == "bool":
                return BOOL
            txt = e.text
            if e.kind == "float":
                return F32 if txt.endswith("f") else AF
            if txt.endswith("u"):
                return U32
            if txt.endswith("i"):
                return I32
            return AI
        if isinstance(e, Ident):
            return self.lookup(e.name)
        if isinstance(e, Member):
            ot = self.typeof(e.obj)
            if ot[0] == "st":
                for f, ft in self.structs[ot[1]]:
                    if f == e.name:
                        return ft
                self.err(f"struct {ot[1]} has no field {e.name}")
            if ot[0] == "v":
                n = len(e.name)
                return ("s", ot[2]) if n == 1 else ("v", n, ot[2])
            self.err(f"member {e.name} of {ot}")
        if isinstance(e, Index):
            ot = self.typeof(e.obj)
            if ot[0] == "a":
                return ot[1]
            if ot[0] == "v":
                return ("s", ot[2])
            if ot[0] == "p":
                return self.typeof(Index(e.obj, e.idx))
            self.err(f"index of {ot}")
        if isinstance(e, Unary):
            t = self.typeof(e.e)
            if e.op == "&":
                return ("p", t)
            if e.op == "*":
                return t[1]
            if e.op == "!":
                return t
            return t
        if isinstance(e, Binary):
            ta, tb = self.typeof(e.a), self.typeof(e.b)
            if e.op in ("&&", "||"):
                return BOOL
            if e.op in ("==", "!=", "<", ">", "<=", ">="):
                n = ta[1] if ta[0] == "v" else (tb[1] if tb[0] == "v" else None)
                return ("v", n, "bool") if n else BOOL
            if e.op in ("<<", ">>"):
                return ta
            return self.arith_result(ta, tb)
        if isinstance(e, Call):
            return self.call_type(e)
        self.err(f"cannot type {e}")

    def arith_result(self, ta, tb):
        if is_abstract(ta) and is_abstract(tb):
            return AF if "af" in (ta[1], tb[1]) else AI
        if is_abstract(ta):
            return tb
        if is_abstract(tb):
            return ta
        if ta[0] == "v":
            return ta
        return tb

    def common_kind(self, types):
        """Concrete scalar kind shared by builtin args, or None if all abstract."""
        conc = [t for t in types if not is_abstract(t)]
        if conc:
            return scal_kind(conc[0])
        return None

    def call_type(self, e):
        n = e.name
        if e.targs is not None:
            if n == "bitcast":
                return e.targs[0]
            if n == "array":
                return ("a", e.targs[0], e.targs[1] if len(e.targs) > 1 else len(e.args))
            return ("v", int(n[3]), e.targs[0][1])
        if n in SCALAR_NAMES:
            return SCALAR_NAMES[n]
        if n in VEC_SHORT:
            return VEC_SHORT[n]
        if n in self.structs:
            return ("st", n)
        if n in self.fns:
            return self.fns[n][1]
        args = [self.typeof(a) for a in e.args]
        if n in FLOAT_UNARY:
            return args[0]
        if n in SAME_TYPE_N:
            k = self.common_kind(args)
            shape = next((a for a in args if a[0] == "v"), args[0])
            if k is None:
                return shape
            return with_kind(shape, k)
        if n == "mix":
            k = self.common_kind(args)
            shape = next((a for a in args[:2] if a[0] == "v"), args[0])
            return with_kind(shape, k) if k else shape
        if n == "select":
            k = self.common_kind(args[:2])
            shape = next((a for a in args[:2] if a[0] == "v"), args[0])
            return with_kind(shape, k) if k else shape
        if n in ("length", "distance", "dot"):
            a = args[0]
            return ("s", a[2]) if a[0] == "v" else a
        if n in ("any", "all"):
            return BOOL
        if n in ("atomicLoad", "atomicAdd", "atomicMax", "atomicSub"):
            return U32
        if n == "atomicStore":
            return VOID
        if n == "atomicCompareExchangeWeak":
            return ("st", "__cmpxchg")
        self.err(f"unknown function {n}")

    # ---- emission
    def emit_conv(self, e, want):
        """Emit `e` converted (if abstract) to concrete type `want`."""
        t = self.typeof(e)
        if want is None or not is_abstract(t):
            return self.emit(e)
        wk = scal_kind(want) if want[0] in ("s", "v") else None
        if wk is None:
            self.err(f"cannot concretise abstract to {want}")
        code = self.emit(e)
        return f"(({CPP_SCALAR[wk]})({code}))"

    def emit_abstract(self, e):
        """Emit an all-abstract expression evaluated in double / int64."""
        if isinstance(e, Lit):
            txt = e.text
            if e.kind == "float":
                return txt.rstrip("fh") if not txt.rstrip("fh").endswith(".") else txt.rstrip("fh") + "0"
            return f"INT64_C({txt})"
        return None

    def emit(self, e):
        sub = self.subst.get(id(e))
        if sub is not None:
            return sub
        if isinstance(e, Lit):
            t = self.typeof(e)
            if e.kind == "bool":
                return e.text
            if t == AF:
                return self.emit_abstract(e)
            if t == AI:
                return f"INT64_C({e.text})"
            if t == F32:
                txt = e.text.rstrip("f")
                if txt.endswith("."):
                    txt += "0"
                if not any(c in txt for c in ".eE"):
                    txt += ".0"
                return f"((float)({txt}))"
            txt = e.text.rstrip("iu")
            return f"(({CPP_SCALAR[t[1]]})({txt}))"
        if isinstance(e, Ident):
            return self.cname(e.name)
        if isinstance(e, Member):
            ot = self.typeof(e.obj)
            obj = self.emit(e.obj)
            if ot[0] == "st":
                return f"{obj}.{self.cname(e.name)}"
            if len(e.name) == 1:
                return f"{obj}.{'xyzw'[SWZ[e.name]]}"
            idx = ", ".join(str(SWZ[c]) for c in e.name)
            return f"wg::swz<{CPP_SCALAR[ot[2]]}, {idx}>({obj})"
        if isinstance(e, Index):
            return f"{self.emit(e.obj)}[{self.emit_conv(e.idx, I32)}]"
        if isinstance(e, Unary):
            if e.op == "&":
                return f"(&{self.emit(e.e)})"
            if e.op == "*":
                return f"(*{self.emit(e.e)})"
            return f"({e.op}{self.emit(e.e)})"
        if isinstance(e, Binary):
            return self.emit_binary(e)
        if isinstance(e, Call):
            return self.emit_call(e)
        self.err(f"cannot emit {e}")

    def emit_binary(self, e):
        ta, tb = self.typeof(e.a), self.typeof(e.b)
        op = e.op
        if op in ("&&", "||"):
            return f"({self.emit(e.a)} {op} {self.emit(e.b)})"
        if is_abstract(ta) and is_abstract(tb):
            # constant-folded in double / int64 by the C++ compiler
            a, b = self.emit(e.a), self.emit(e.b)
            if op in ("%",):
                return f"wg::mod_s({a}, {b})"
            return f"({a} {op} {b})"
        if op in ("<<", ">>"):
            a = self.emit_conv(e.a, ta)
            b = self.emit_conv(e.b, U32)
            return f"wg::{'shl' if op == '<<' else 'shr'}({a}, {b})"
        # concretise abstract operand to the other operand's scalar kind
        if is_abstract(ta):
            a = self.emit_conv(e.a, ("s", scal_kind(tb)))
            b = self.emit(e.b)
        elif is_abstract(tb):
            a = self.emit(e.a)
            b = self.emit_conv(e.b, ("s", scal_kind(ta)))
        else:
            a, b = self.emit(e.a), self.emit(e.b)
        vec = ta[0] == "v" or tb[0] == "v"
        cmp = {"==": "eq", "!=": "ne", "<": "lt", ">": "gt", "<=": "le", ">=": "ge"}
        if op in cmp:
            return f"wg::{cmp[op]}({a}, {b})" if vec else f"({a} {op} {b})"
        if op == "/":
            return f"wg::div({a}, {b})"
        if op == "%":
            return f"wg::mod({a}, {b})"
        return f"({a} {op} {b})"

    def emit_call(self, e):
        n = e.name
        rt = self.typeof(e)
        if e.targs is not None:
            if n == "bitcast":
                return f"wg::bitcast<{self.ctype(rt)}>({self.emit(e.args[0])})"
            if n == "array":
                el = rt[1]
                return "{}{{{}}}".format(self.ctype(rt), ", ".join(self.emit_conv(a, el) for a in e.args))
            return self.emit_ctor(rt, e.args)
        if n in SCALAR_NAMES or n in VEC_SHORT:
            return self.emit_ctor(rt, e.args)
        if n in self.structs:
            fields = self.structs[n]
            if len(e.args) != len(fields):
                self.err(f"struct ctor {n} arity")
            parts = [self.emit_conv(a, ft) for a, (_, ft) in zip(e.args, fields)]
            return f"{self.cname(n)}{{{', '.join(parts)}}}"
        if n in self.fns:
            params, _ = self.fns[n]
            if len(params) != len(e.args):
                self.err(f"call {n} arity")
            parts = [self.emit_conv(a, pt) for a, (_, pt) in zip(e.args, params)]
            return f"U_{n}({', '.join(parts)})"
        args = e.args
        types = [self.typeof(a) for a in args]
        if n.startswith("atomic"):
            parts = [self.emit(args[0])] + [self.emit_conv(a, U32) for a in args[1:]]
            return f"wg::{n}({', '.join(parts)})"
        if n == "select":
            k = self.common_kind(types[:2])
            want = ("s", k) if k else None
            if want is None:  # all abstract: concretise by default
                want = concretize(types[0])
            parts = [self.emit_conv(args[0], want), self.emit_conv(args[1], want), self.emit(args[2])]
            return f"wg::select({', '.join(parts)})"
        k = self.common_kind(types)
        if k is None:
            # builtin of purely abstract args: evaluate in double
            return f"wg::{n}({', '.join(self.emit(a) for a in args)})"
        want = ("s", k)
        parts = [self.emit_conv(a, want) for a in args]
        return f"wg::{n}({', '.join(parts)})"

    def emit_ctor(self, rt, args):
        if rt[0] == "s":
            if not args:
                return f"(({self.ctype(rt)})0)"
            a = args[0]
            at = self.typeof(a)
            if is_abstract(at):
                return self.emit_conv(a, rt)
            return f"wg::cvt<{self.ctype(rt)}>({self.emit(a)})"
        if not args:
            return f"{self.ctype(rt)}{{}}"
        want = ("s", rt[2])
        if len(args) == 1 and self.typeof(args[0])[0] == "v":
            return f"wg::conv<{self.ctype(rt)}>({self.emit(args[0])})"
        parts = [self.emit_conv(a, want) for a in args]
        return f"wg::make<{self.ctype(rt)}>({', '.join(parts)})"

    # ---- statements
    def w(self, line, ind):
        self.out.append("  " * ind + line)

    def emit_block(self, stmts, ind):
        self.scopes.append({})
        for s in stmts:
            self.emit_stmt(s, ind)
        self.scopes.pop()

    def decl_type(self, ty, init):
        if ty is not None:
            return ty
        return concretize(self.typeof(init))

    # ---- left-to-right evaluation of impure calls
    def _impure_calls(self, e, acc):
        """Collect impure user calls in WGSL evaluation order (operands left
        to right, a call's arguments before the call).  The right operand of
        && / || is conditional and is left in place (C++ sequences it)."""
        if isinstance(e, Call):
            for a in e.args:
                self._impure_calls(a, acc)
            if e.name in self.impure:
                acc.append(e)
        elif isinstance(e, Binary):
            self._impure_calls(e.a, acc)
            if e.op not in ("&&", "||"):
                self._impure_calls(e.b, acc)
        elif isinstance(e, Unary):
            self._impure_calls(e.e, acc)
        elif isinstance(e, Member):
            self._impure_calls(e.obj, acc)
        elif isinstance(e, Index):
            self._impure_calls(e.obj, acc)
            self._impure_calls(e.idx, acc)

    def hoist(self, exprs, ind):
        acc = []
        for e in exprs:
            if e is not None:
                self._impure_calls(e, acc)
        if len(acc) < 2:
            return
        for c in acc:
            t = concretize(self.typeof(c))
            code = self.emit(c)
            name = f"__t{self.tmp_n}"
            self.tmp_n += 1
            self.w(f"const {self.ctype(t)} {name} = {code};", ind)
            self.subst[id(c)] = name

    def simple_text(self, s):
        k = s[0]
        if k == "decl":
            _, kw, name, ty, init = s
            t = self.decl_type(ty, init)
            cn = self.cname(name)
            q = "const " if kw in ("let", "const") else ""
            self.scopes[-1][name] = t
            if init is None:
                return f"{self.ctype(t)} {cn}{{}}"
            return f"{q}{self.ctype(t)} {cn} = {self.emit_conv(init, t)}"
        if k == "assign":
            _, op, lhs, rhs = s
            lt = self.typeof(lhs)
            if lt[0] == "at":
                lt = ("s", lt[1])
            l = self.emit(lhs)
            want = ("s", scal_kind(lt)) if lt[0] in ("s", "v") else lt
            if op == "=":
                return f"{l} = {self.emit_conv(rhs, want)}"
            return f"{l} = {self.emit_binary(Binary(op[:-1], lhs, rhs))}"
        if k == "incdec":
            return f"{self.emit(s[2])}{s[1]}"
        self.err(f"simple stmt {k}")

    def emit_stmt(self, s, ind):
        k = s[0]
        if k == "block":
            self.w("{", ind)
            self.emit_block(s[1], ind + 1)
            self.w("}", ind)
        elif k in ("decl", "assign", "incdec"):
            if k == "decl":
                self.hoist([s[4]], ind)
            elif k == "assign":
                self.hoist([s[2], s[3]], ind)
            self.w(self.simple_text(s) + ";", ind)
        elif k == "phony":
            self.hoist([s[1]], ind)
            self.w(f"(void)({self.emit(s[1])});", ind)
        elif k == "expr":
            self.hoist([s[1]], ind)
            self.w(f"{self.emit(s[1])};", ind)
        elif k == "if":
            _, cond, then, other = s
            self.hoist([cond], ind)
            self.w(f"if ({self.emit(cond)}) {{", ind)
            self.emit_block(then, ind + 1)
            if other is None:
                self.w("}", ind)
            else:
                self.w("} else {", ind)
                self.emit_block(other, ind + 1)
                self.w("}", ind)
        elif k == "for":
            _, init, cond, upd, body = s
            self.scopes.append({})
            chk = []
            self._impure_calls(cond, chk) if cond is not None else None
            if upd is not None and upd[0] == "assign":
                self._impure_calls(upd[3], chk)
            if chk:
                self.err("impure call in a for-loop condition/update")
            if init is not None and init[0] == "decl":
                self.hoist([init[4]], ind)
            init_s = self.simple_text(init) if init is not None else ""
            c = self.emit(cond) if cond is not None else ""
            upd_s = self.simple_text(upd) if upd is not None else ""
            self.w(f"for ({init_s}; {c}; {upd_s}) {{", ind)
            self.emit_block(body, ind + 1)
            self.w("}", ind)
            self.scopes.pop()
        elif k == "while":
            self.w(f"while ({self.emit(s[1])}) {{", ind)
            self.emit_block(s[2], ind + 1)
            self.w("}", ind)
        elif k == "loop":
            self.w("for (;;) {", ind)
            self.emit_block(s[1], ind + 1)
            self.w("}", ind)
        elif k == "switch":
            _, sel, cases = s
            st = concretize(self.typeof(sel))
            self.hoist([sel], ind)
            self.w(f"switch ({self.emit_conv(sel, st)}) {{", ind)
            for labels, body in cases:
                for lab in labels:
                    if lab is None:
                        self.w("default:", ind + 1)
                    else:
                        self.w(f"case {self.emit_conv(lab, st)}:", ind + 1)
                self.w("{", ind + 1)
                self.emit_block(body, ind + 2)
                self.w("} break;", ind + 1)
            self.w("}", ind)
        elif k == "break":
            self.w("break;", ind)
        elif k == "continue":
            self.w("continue;", ind)
        elif k == "return":
            self.hoist([s[1]], ind)
            if s[1] is None:
                self.w("return;", ind)
            else:
                self.w(f"return {self.emit_conv(s[1], self.cur_ret)};", ind)
        elif k == "discard":
            self.w("return {};", ind)
        else:
            self.err(f"stmt {k}")

    def _scan_calls(self, node, names):
        if isinstance(node, list):
            for x in node:
                self._scan_calls(x, names)
        elif isinstance(node, tuple):
            for x in node:
                self._scan_calls(x, names)
        elif isinstance(node, Call):
            names.add(node.name)
            for a in node.args:
                self._scan_calls(a, names)
        elif isinstance(node, Binary):
            self._scan_calls(node.a, names)
            self._scan_calls(node.b, names)
        elif isinstance(node, Unary):
            self._scan_calls(node.e, names)
        elif isinstance(node, Member):
            self._scan_calls(node.obj, names)
        elif isinstance(node, Index):
            self._scan_calls(node.obj, names)
            self._scan_calls(node.idx, names)

    # ---- module
    def translate(self, items):
        # pass 1: declarations
        for it in items:
            if it[0] == "struct":
                self.structs[it[1]] = it[2]
            elif it[0] == "fn":
                if it[1] in self.skip_fns:
                    continue
                self.fns[it[1]] = (it[2], it[3])
        self.structs["__cmpxchg"] = [("old_value", U32), ("exchanged", BOOL)]
        calls = {}
        for it in items:
            if it[0] == "fn":
                names = set()
                self._scan_calls(it[4], names)
                calls[it[1]] = names
        self.impure = {"isaac_irand", "isaac_round", "rand01", "rand_11",
                       "atomic_add_sat", "atomic_add_sat_idx"} & set(calls)
        changed = True
        while changed:
            changed = False
            for f, names in calls.items():
                if f not in self.impure and names & self.impure:
                    self.impure.add(f)
                    changed = True
        o = self.out
        o.append(f"namespace {self.ns} {{")
        o.append("using __cmpxchg = wg::atomic_cmpxchg_u32;")
        for it in items:
            if it[0] == "struct":
                o.append(f"struct {self.cname(it[1])} {{")
                for f, ft in it[2]:
                    o.append(f"  {self.ctype(ft)} {self.cname(f)};")
                o.append("};")
        for it in items:
            if it[0] == "const":
                _, name, ty, e = it
                et = self.typeof(e)
                if ty is None and is_abstract(et):
                    ct = "double" if et == AF else "int64_t"
                    o.append(f"constexpr {ct} {self.cname(name)} = {self.emit(e)};")
                    self.consts[name] = et
                else:
                    t = ty or concretize(et)
                    if t[0] == "a":
                        o.append(f"static const {self.ctype(t)} {self.cname(name)} = {self.emit(e)};")
                    else:
                        o.append(f"static const {self.ctype(t)} {self.cname(name)} = {self.emit_conv(e, t)};")
                    self.consts[name] = t
            elif it[0] == "var":
                _, name, space, ty, init = it
                if ty[0] == "a" and ty[2] is None:
                    el = ty[1]
                    elc = self.ctype(("s", el[1])) if el[0] == "at" else self.ctype(el)
                    o.append(f"thread_local {elc}* {self.cname(name)} = nullptr;")
                else:
                    o.append(f"thread_local {self.ctype(ty)} {self.cname(name)}{{}};")
                self.globals[name] = ty
        # prototypes
        for it in items:
            if it[0] == "fn" and it[1] not in self.skip_fns:
                _, name, params, ret, body, attrs = it
                ps = ", ".join(f"{self.ctype(pt)} {self.cname(pn)}" for pn, pt in params)
                o.append(f"{self.ctype(ret)} U_{name}({ps});")
        for it in items:
            if it[0] == "fn" and it[1] not in self.skip_fns:
                _, name, params, ret, body, attrs = it
                ps = ", ".join(f"{self.ctype(pt)} {self.cname(pn)}" for pn, pt in params)
                o.append(f"{self.ctype(ret)} U_{name}({ps}) {{")
                self.cur_ret = ret
                self.scopes = [{pn: pt for pn, pt in params}]
                self.emit_block(body, 1)
                self.scopes = []
                o.append("}")
        o.append(f"}}  // namespace {self.ns}")
        return "\n".join(o)


def translate(sources, ns, skip_fns=(), f32_type="float"):
    """C++ for the WGSL `sources` in namespace `ns`.  f32_type="double"
    emits every f32 value, literal and conversion as a C++ double: the same
    expressions evaluated in FP64, for measuring the f32 shaders' error."""
    text = "\n".join(sources)
    items = Parser(tokenize(text)).parse_module()
    saved = CPP_SCALAR["f32"]
    CPP_SCALAR["f32"] = f32_type
    try:
        return Emitter(ns, skip_fns).translate(items)
    finally:
        CPP_SCALAR["f32"] = saved


if __name__ == "__main__":
    # usage: wgsl2cpp.py NAMESPACE OUT.cpp IN1.wgsl [IN2.wgsl ...]
    ns, out = sys.argv[1], sys.argv[2]
    srcs = [open(p).read() for p in sys.argv[3:]]
    code = translate(srcs, ns, skip_fns=("vs",))
    with open(out, "w") as f:
        f.write(code + "\n")
