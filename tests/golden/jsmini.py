"""jsmini -- run the reference solver's own JavaScript here, without a JS engine.

No JavaScript engine exists on this machine, so the golden vectors that pin the
oracle come from the reference's sources (src/lattices.js, src/solid.js,
src/sim.js) translated mechanically into Python and executed.  This module is
that translator.  It accepts the small subset those files use -- ES classes,
let/const with object destructuring, for/while/if, typed arrays, Math.*,
ternaries, ++/--, compound assignment, `??`, an IIFE -- and rejects anything
else loudly instead of guessing.

Semantics preserved (the ones the solver's results depend on):
  * JS numbers are IEEE doubles: integer-valued quantities stay Python ints
    (exact below 2**53, as in JS), everything else is a Python float; every
    arithmetic operator maps to the same correctly rounded double operation,
    evaluated in the same order (every binary expression is parenthesised, so
    Python neither re-associates nor chains comparisons).
  * Float32Array / Int32Array / Int8Array / Uint8Array are array.array of the
    same element type: a store rounds to the element type exactly like a JS
    typed-array store, a load widens to double.
  * `|`, `&`, `^`, `<<`, `>>`, `>>>`, `~` apply ToInt32 / ToUint32.
  * Math.min / Math.max propagate NaN, Math.sqrt of a negative is NaN.
  * A `for (let v = a; v < b; v++)` loop whose bound and counter the body does
    not assign becomes a Python range loop; every other loop becomes a while
    loop whose `continue` runs the update first.
Known difference: Math.tanh is the C library's tanh (V8 may differ by one ulp;
it only enters through Sim.initFlat).

Used only to generate test fixtures (tests/golden/make_golden.py); nothing in
the library or its tests imports it at run time.
"""
import array
import math
import re

# ----------------------------------------------------------------- tokenizer
_TOKEN = re.compile(r"""
  (?P<ws>\s+) | (?P<lc>//[^\n]*) | (?P<bc>/\*.*?\*/)
| (?P<num>(?:\d+\.\d*|\.\d+|\d+)(?:[eE][+-]?\d+)?)
| (?P<str>'(?:[^'\\\n]|\\.)*'|"(?:[^"\\\n]|\\.)*")
| (?P<id>[A-Za-z_$][\w$]*)
| (?P<op>>>>=|===|!==|\*\*=|<<=|>>=|>>>|\?\?=|\.\.\.|\?\?|\?\.|=>|\+\+|--|&&|\|\||<=|>=|==|!=|\+=|-=|\*=|/=|%=|&=|\|=|\^=|<<|>>|\*\*|[{}()\[\];,.<>+\-*/%&|^!~?:=])
""", re.S | re.X)


class JSSyntaxError(Exception):
    pass


def tokenize(src):
    out, pos = [], 0
    while pos < len(src):
        m = _TOKEN.match(src, pos)
        if not m:
            raise JSSyntaxError(f"unexpected character {src[pos]!r} at offset {pos}")
        pos = m.end()
        kind = m.lastgroup
        if kind in ("ws", "lc", "bc"):
            continue
        out.append((kind, m.group()))
    out.append(("eof", ""))
    return out


# ----------------------------------------------------------------- parser
_BINARY = {  # precedence, right-associative
    "??": (3, False), "||": (4, False), "&&": (5, False), "|": (6, False), "^": (7, False),
    "&": (8, False), "==": (9, False), "!=": (9, False), "===": (9, False), "!==": (9, False),
    "<": (10, False), ">": (10, False), "<=": (10, False), ">=": (10, False),
    "<<": (11, False), ">>": (11, False), ">>>": (11, False), "+": (12, False), "-": (12, False),
    "*": (13, False), "/": (13, False), "%": (13, False), "**": (14, True),
}
_ASSIGN = {"=", "+=", "-=", "*=", "/=", "%=", "&=", "|=", "^=", "<<=", ">>=", ">>>=", "**=", "??="}
_RESERVED = {"class", "constructor", "function", "return", "if", "else", "for", "while", "do",
             "break", "continue", "const", "let", "var", "new", "this", "throw", "import",
             "export", "from", "switch", "case", "typeof", "instanceof", "in", "of", "yield",
             "async", "await", "try", "catch", "finally", "delete", "void"}


class Parser:
    def __init__(self, tokens):
        self.t = tokens
        self.i = 0

    # helpers
    def peek(self, k=0):
        return self.t[self.i + k]

    def at(self, val, k=0):
        tok = self.t[self.i + k]
        return tok[0] in ("op", "id") and tok[1] == val

    def next(self):
        tok = self.t[self.i]
        self.i += 1
        return tok

    def expect(self, val):
        tok = self.next()
        if tok[1] != val or tok[0] not in ("op", "id"):
            raise JSSyntaxError(f"expected {val!r}, got {tok[1]!r} (token {self.i})")
        return tok

    def ident(self):
        tok = self.next()
        if tok[0] != "id":
            raise JSSyntaxError(f"expected identifier, got {tok[1]!r}")
        return tok[1]

    # program
    def program(self):
        body = []
        while self.peek()[0] != "eof":
            body.append(self.statement())
        return body

    def statement(self):
        tok = self.peek()
        v = tok[1]
        if tok[0] == "op":
            if v == "{":
                return ("block", self.block())
            if v == ";":
                self.next()
                return ("empty",)
        if tok[0] == "id":
            if v == "import":
                while not self.at(";"):
                    self.next()
                self.next()
                return ("empty",)
            if v == "export":
                self.next()
                return self.statement()
            if v in ("const", "let", "var"):
                s = self.declaration()
                self.expect(";")
                return s
            if v == "class":
                return self.class_decl()
            if v == "function":
                return self.function(True)
            if v == "if":
                self.next()
                self.expect("(")
                c = self.expression()
                self.expect(")")
                a = self.statement()
                b = None
                if self.at("else"):
                    self.next()
                    b = self.statement()
                return ("if", c, a, b)
            if v == "for":
                self.next()
                self.expect("(")
                init = None
                if not self.at(";"):
                    init = self.declaration() if self.peek()[1] in ("let", "const", "var") \
                        else ("expr", self.expression())
                    if self.at("of") or self.at("in"):
                        raise JSSyntaxError("for-of / for-in is outside the supported subset")
                self.expect(";")
                cond = None if self.at(";") else self.expression()
                self.expect(";")
                upd = None if self.at(")") else self.expression()
                self.expect(")")
                return ("for", init, cond, upd, self.statement())
            if v == "while":
                self.next()
                self.expect("(")
                c = self.expression()
                self.expect(")")
                return ("while", c, self.statement())
            if v == "return":
                self.next()
                e = None if self.at(";") else self.expression()
                self.expect(";")
                return ("return", e)
            if v in ("break", "continue"):
                self.next()
                self.expect(";")
                return (v,)
            if v == "throw":
                self.next()
                e = self.expression()
                self.expect(";")
                return ("throw", e)
            if v in ("switch", "do", "try", "yield", "async", "await", "delete"):
                raise JSSyntaxError(f"'{v}' is outside the supported subset")
        e = self.expression()
        self.expect(";")
        return ("expr", e)

    def block(self):
        self.expect("{")
        body = []
        while not self.at("}"):
            body.append(self.statement())
        self.expect("}")
        return body

    def declaration(self):
        self.next()  # const / let / var
        decls = []
        while True:
            if self.at("{"):
                self.next()
                names = []
                while not self.at("}"):
                    names.append(self.ident())
                    if self.at(":") or self.at("="):
                        raise JSSyntaxError("renaming / default destructuring is not supported")
                    if self.at(","):
                        self.next()
                self.expect("}")
                target = ("objpat", names)
            elif self.at("["):
                raise JSSyntaxError("array destructuring is not supported")
            else:
                target = ("id", self.ident())
            init = None
            if self.at("="):
                self.next()
                init = self.assignment()
            decls.append((target, init))
            if not self.at(","):
                break
            self.next()
        return ("var", decls)

    def params(self):
        self.expect("(")
        ps = []
        while not self.at(")"):
            name = self.ident()
            default = None
            if self.at("="):
                self.next()
                default = self.assignment()
            ps.append((name, default))
            if self.at(","):
                self.next()
        self.expect(")")
        return ps

    def function(self, is_decl):
        self.expect("function")
        name = self.ident() if self.peek()[0] == "id" else None
        ps = self.params()
        body = self.block()
        return ("funcdecl" if is_decl else "func", name, ps, body)

    def class_decl(self):
        self.expect("class")
        name = self.ident()
        if self.at("extends"):
            raise JSSyntaxError("class inheritance is not supported")
        self.expect("{")
        methods = []
        while not self.at("}"):
            if self.at(";"):
                self.next()
                continue
            if self.at("static") or self.at("get") or self.at("set"):
                if self.peek(1)[0] == "id":
                    raise JSSyntaxError("static members and accessors are not supported")
            mname = self.ident()
            ps = self.params()
            body = self.block()
            methods.append((mname, ps, body))
        self.expect("}")
        return ("class", name, methods)

    # expressions
    def expression(self):
        e = self.assignment()
        if self.at(","):
            raise JSSyntaxError("the comma operator is not supported")
        return e

    def assignment(self):
        if self.at("(") and self._arrow_ahead():
            raise JSSyntaxError("arrow functions are not supported")
        left = self.conditional()
        tok = self.peek()
        if tok[0] == "op" and tok[1] in _ASSIGN:
            self.next()
            if left[0] not in ("id", "member", "index"):
                raise JSSyntaxError("invalid assignment target")
            return ("assign", tok[1], left, self.assignment())
        return left

    def _arrow_ahead(self):
        depth, j = 0, self.i
        while True:
            kind, v = self.t[j]
            if kind == "eof":
                return False
            if v == "(":
                depth += 1
            elif v == ")":
                depth -= 1
                if depth == 0:
                    return self.t[j + 1][1] == "=>"
            j += 1

    def conditional(self):
        c = self.binary(0)
        if self.at("?"):
            self.next()
            a = self.assignment()
            self.expect(":")
            b = self.assignment()
            return ("cond", c, a, b)
        return c

    def binary(self, min_prec):
        left = self.unary()
        while True:
            tok = self.peek()
            if tok[0] != "op" or tok[1] not in _BINARY:
                return left
            prec, right_assoc = _BINARY[tok[1]]
            if prec < min_prec:
                return left
            self.next()
            right = self.binary(prec if right_assoc else prec + 1)
            left = ("bin", tok[1], left, right)

    def unary(self):
        tok = self.peek()
        if tok[0] == "op" and tok[1] in ("!", "-", "+", "~"):
            self.next()
            return ("unary", tok[1], self.unary())
        if tok[0] == "op" and tok[1] in ("++", "--"):
            self.next()
            return ("prefix", tok[1], self.unary())
        if tok[0] == "id" and tok[1] in ("typeof", "void", "delete", "await"):
            raise JSSyntaxError(f"'{tok[1]}' is not supported")
        e = self.postfix()
        return e

    def postfix(self):
        e = self.call_member()
        tok = self.peek()
        if tok[0] == "op" and tok[1] in ("++", "--"):
            self.next()
            return ("postfix", tok[1], e)
        return e

    def call_member(self):
        if self.at("new"):
            self.next()
            ctor = self.primary()
            while self.at("."):
                self.next()
                ctor = ("member", ctor, self.ident())
            args = self.arguments() if self.at("(") else []
            e = ("new", ctor, args)
        else:
            e = self.primary()
        while True:
            if self.at("."):
                self.next()
                e = ("member", e, self.ident())
            elif self.at("["):
                self.next()
                idx = self.expression()
                self.expect("]")
                e = ("index", e, idx)
            elif self.at("("):
                e = ("call", e, self.arguments())
            elif self.at("?."):
                raise JSSyntaxError("optional chaining is not supported")
            else:
                return e

    def arguments(self):
        self.expect("(")
        args = []
        while not self.at(")"):
            if self.at("..."):
                raise JSSyntaxError("spread is not supported")
            args.append(self.assignment())
            if self.at(","):
                self.next()
        self.expect(")")
        return args

    def primary(self):
        kind, v = self.next()
        if kind == "num":
            return ("num", v)
        if kind == "str":
            return ("str", v)
        if kind == "id":
            if v == "this":
                return ("this",)
            if v == "function":
                self.i -= 1
                return self.function(False)
            if v in ("true", "false"):
                return ("bool", v == "true")
            if v in ("null", "undefined"):
                return ("none",)
            if v in _RESERVED:
                raise JSSyntaxError(f"unexpected keyword {v!r}")
            return ("id", v)
        if v == "(":
            e = self.expression()
            self.expect(")")
            return ("paren", e)
        if v == "[":
            elems = []
            while not self.at("]"):
                elems.append(self.assignment())
                if self.at(","):
                    self.next()
            self.expect("]")
            return ("array", elems)
        if v == "{":
            props = []
            while not self.at("}"):
                key = self.next()[1]
                self.expect(":")
                props.append((key, self.assignment()))
                if self.at(","):
                    self.next()
            self.expect("}")
            return ("object", props)
        raise JSSyntaxError(f"unexpected token {v!r}")


# ----------------------------------------------------------------- code generator
_MATH = {"min": "_js_min", "max": "_js_max", "abs": "abs", "sqrt": "_js_sqrt",
         "tanh": "math.tanh", "floor": "math.floor", "ceil": "math.ceil", "exp": "math.exp",
         "log": "_js_log", "pow": "_js_pow", "round": "_js_round", "sign": "_js_sign",
         "hypot": "math.hypot", "cos": "math.cos", "sin": "math.sin", "atan2": "math.atan2"}
_MATH_CONST = {"PI": "math.pi", "E": "math.e", "SQRT2": "math.sqrt(2.0)"}
_BITOP = {"|": "_js_or", "&": "_js_and", "^": "_js_xor", "<<": "_js_shl", ">>": "_js_sar",
          ">>>": "_js_shr"}
_CMP = {"<": "<", ">": ">", "<=": "<=", ">=": ">=", "===": "==", "!==": "!=", "==": "==",
        "!=": "!="}
_BOOLEAN_KINDS = ("bool",)


def _assigned_names(node, out):
    """Names of plain identifiers assigned (or ++/--) anywhere inside node."""
    if isinstance(node, tuple):
        if node and node[0] == "assign" and node[2][0] == "id":
            out.add(node[2][1])
        if node and node[0] in ("postfix", "prefix") and node[2][0] == "id":
            out.add(node[2][1])
        if node and node[0] == "var":
            for target, _ in node[1]:
                if target[0] == "id":
                    out.add(target[1])
                else:
                    out.update(target[1])
        for x in node:
            _assigned_names(x, out)
    elif isinstance(node, list):
        for x in node:
            _assigned_names(x, out)
    return out


def _idents(node, out):
    if isinstance(node, tuple):
        if node and node[0] == "id":
            out.add(node[1])
        for x in node:
            _idents(x, out)
    elif isinstance(node, list):
        for x in node:
            _idents(x, out)
    return out


def _simple_bound(node):
    """A loop bound made of identifiers, numbers, this.<field> and + - *."""
    k = node[0]
    if k in ("num", "id"):
        return True
    if k == "member":
        return node[1][0] in ("this", "id") and node[2] != "length"
    if k == "paren":
        return _simple_bound(node[1])
    if k == "bin" and node[1] in ("+", "-", "*"):
        return _simple_bound(node[2]) and _simple_bound(node[3])
    if k == "unary" and node[1] == "-":
        return _simple_bound(node[2])
    return False


class CodeGen:
    def __init__(self):
        self.lines = []
        self.tmp = 0
        self.loop_updates = []   # update code of the enclosing while-loops (None = range loop)
        self.scopes = []         # stack of sets of names declared per JS block

    # ---- emission
    def emit(self, depth, text):
        self.lines.append("    " * depth + text)

    def fresh(self):
        self.tmp += 1
        return f"_t{self.tmp}"

    # ---- scoping: JS block scope is flattened into the Python function scope,
    # which is only sound when no inner block re-declares a name of an enclosing one.
    def declare(self, name):
        for s in self.scopes[:-1]:
            if name in s:
                raise JSSyntaxError(f"'{name}' shadows a binding of an enclosing block")
        self.scopes[-1].add(name)

    # ---- expressions; `pre` collects statements that must run first (hoisted ++/--)
    def expr(self, n, pre):
        k = n[0]
        if k == "num":
            txt = n[1]
            if re.fullmatch(r"\d+", txt):
                return str(int(txt))
            return repr(float(txt))
        if k == "str":
            return repr(bytes(n[1][1:-1], "utf-8").decode("unicode_escape"))
        if k == "bool":
            return "True" if n[1] else "False"
        if k == "none":
            return "None"
        if k == "this":
            return "self"
        if k == "id":
            return n[1]
        if k == "paren":
            return self.expr(n[1], pre)
        if k == "array":
            return "[" + ", ".join(self.expr(e, pre) for e in n[1]) + "]"
        if k == "object":
            return "_JSObject(" + ", ".join(f"{key}={self.expr(v, pre)}" for key, v in n[1]) + ")"
        if k == "member":
            obj, name = n[1], n[2]
            if obj == ("id", "Math"):
                if name not in _MATH_CONST:
                    raise JSSyntaxError(f"Math.{name} is not supported")
                return _MATH_CONST[name]
            if name == "length":
                return f"len({self.expr(obj, pre)})"
            return f"{self.expr(obj, pre)}.{name}"
        if k == "index":
            return f"{self.expr(n[1], pre)}[{self.expr(n[2], pre)}]"
        if k == "call":
            fn, args = n[1], n[2]
            a = ", ".join(self.expr(x, pre) for x in args)
            if fn[0] == "member" and fn[1] == ("id", "Math"):
                if fn[2] not in _MATH:
                    raise JSSyntaxError(f"Math.{fn[2]} is not supported")
                return f"{_MATH[fn[2]]}({a})"
            return f"{self.expr(fn, pre)}({a})"
        if k == "new":
            ctor = n[1]
            if ctor[0] != "id":
                raise JSSyntaxError("new of a non-identifier")
            name = ctor[1]
            if name == "Error":
                name = "_JSError"
            return f"{name}(" + ", ".join(self.expr(x, pre) for x in n[2]) + ")"
        if k == "unary":
            op, e = n[1], n[2]
            if op == "!":
                return f"(not {self.cond(e, pre)})"
            if op == "-":
                return f"(-{self.expr(e, pre)})"
            if op == "+":
                return f"_js_number({self.expr(e, pre)})"
            if op == "~":
                return f"_js_not({self.expr(e, pre)})"
        if k == "bin":
            op, l, r = n[1], n[2], n[3]
            if op == "&&":
                return f"({self.cond_value(l, pre)} and {self.cond_value(r, pre)})"
            if op == "||":
                return f"({self.cond_value(l, pre)} or {self.cond_value(r, pre)})"
            if op == "??":
                return f"_js_nullish({self.expr(l, pre)}, {self.expr(r, pre)})"
            if op in _BITOP:
                return f"{_BITOP[op]}({self.expr(l, pre)}, {self.expr(r, pre)})"
            if op in _CMP:
                return f"({self.expr(l, pre)} {_CMP[op]} {self.expr(r, pre)})"
            if op == "+" and (l[0] == "str" or r[0] == "str"):
                return f"_js_concat({self.expr(l, pre)}, {self.expr(r, pre)})"
            if op == "%":
                return f"_js_mod({self.expr(l, pre)}, {self.expr(r, pre)})"
            if op in ("+", "-", "*", "/", "**"):
                return f"({self.expr(l, pre)} {op} {self.expr(r, pre)})"
            raise JSSyntaxError(f"operator {op} is not supported")
        if k == "cond":
            return (f"({self.expr(n[2], pre)} if {self.cond(n[1], pre)} "
                    f"else {self.expr(n[3], pre)})")
        if k in ("postfix", "prefix"):
            target = n[2]
            if target[0] != "id":
                raise JSSyntaxError("++/-- on a non-identifier inside an expression")
            t = self.fresh()
            step = "+ 1" if n[1] == "++" else "- 1"
            if k == "postfix":
                pre.append(f"{t} = {target[1]}")
                pre.append(f"{target[1]} = {t} {step}")
            else:
                pre.append(f"{target[1]} = {target[1]} {step}")
                pre.append(f"{t} = {target[1]}")
            return t
        if k == "assign":
            raise JSSyntaxError("assignment inside an expression is not supported")
        if k in ("func", "funcdecl"):
            raise JSSyntaxError("function expressions are only supported as an IIFE statement")
        raise JSSyntaxError(f"cannot translate expression {k}")

    def is_boolean(self, n):
        k = n[0]
        if k == "paren":
            return self.is_boolean(n[1])
        if k == "bool":
            return True
        if k == "bin" and (n[1] in _CMP or n[1] in ("&&", "||")):
            return n[1] in _CMP or (self.is_boolean(n[2]) and self.is_boolean(n[3]))
        if k == "unary" and n[1] == "!":
            return True
        return False

    def cond(self, n, pre):
        """A JS condition as a Python bool (NaN is falsy in JS)."""
        if self.is_boolean(n):
            return self.expr(n, pre)
        return f"_js_truthy({self.expr(n, pre)})"

    def cond_value(self, n, pre):
        """Operand of && / ||: JS returns the operand itself."""
        if self.is_boolean(n):
            return self.expr(n, pre)
        return f"_js_falsy_nan({self.expr(n, pre)})"

    # ---- statements
    def stmt_expr(self, n, depth):
        """An expression statement: assignments, ++/--, calls."""
        pre = []
        k = n[0]
        if k in ("postfix", "prefix"):
            tgt = n[2]
            if tgt[0] not in ("id", "member", "index"):
                raise JSSyntaxError("bad ++/-- target")
            code = f"{self.expr(tgt, pre)} {'+=' if n[1] == '++' else '-='} 1"
        elif k == "assign":
            targets, value, op = [], n, None
            # a = b = c chains (plain '=') become one Python chained assignment
            while value[0] == "assign" and value[1] == "=" and (op is None or op == "="):
                targets.append(value[2])
                op = "="
                value = value[3]
                if targets and n[1] != "=":
                    break
            if n[1] != "=":
                if n[1] not in ("+=", "-=", "*=", "/=", "**="):
                    raise JSSyntaxError(f"compound assignment {n[1]} is not supported")
                code = f"{self.expr(n[2], pre)} {n[1]} {self.expr(n[3], pre)}"
            else:
                lhs = [self.expr(t, pre) for t in targets]
                rhs = self.expr(value, pre)
                code = " = ".join(lhs + [rhs])
        elif k == "call":
            code = self.expr(n, pre)
        else:
            raise JSSyntaxError(f"expression statement of kind {k} is not supported")
        for p in pre:
            self.emit(depth, p)
        self.emit(depth, code)

    def body(self, stmts, depth, new_scope=True):
        if new_scope:
            self.scopes.append(set())
        start = len(self.lines)
        for s in stmts:
            self.stmt(s, depth)
        if len(self.lines) == start:
            self.emit(depth, "pass")
        if new_scope:
            self.scopes.pop()

    def as_list(self, s):
        return s[1] if s[0] == "block" else [s]

    def stmt(self, n, depth):
        k = n[0]
        if k == "empty":
            return
        if k == "block":
            self.scopes.append(set())
            for s in n[1]:
                self.stmt(s, depth)
            self.scopes.pop()
            return
        if k == "expr":
            e = n[1]
            if e[0] == "call" and e[1][0] in ("func", "paren") and not e[2]:
                fn = e[1][1] if e[1][0] == "paren" else e[1]
                if fn[0] in ("func", "funcdecl"):  # IIFE
                    name = fn[1] or self.fresh()
                    self.function(("funcdecl", name, fn[2], fn[3]), depth)
                    self.emit(depth, f"{name}()")
                    return
            self.stmt_expr(e, depth)
            return
        if k == "var":
            for target, init in n[1]:
                pre = []
                if target[0] == "objpat":
                    if init is None:
                        raise JSSyntaxError("destructuring without an initialiser")
                    src = self.expr(init, pre)
                    for p in pre:
                        self.emit(depth, p)
                    if src != "self" and not re.fullmatch(r"\w+", src):
                        t = self.fresh()
                        self.emit(depth, f"{t} = {src}")
                        src = t
                    for name in target[1]:
                        self.declare(name)
                        self.emit(depth, f"{name} = {src}.{name}")
                else:
                    self.declare(target[1])
                    val = "None" if init is None else self.expr(init, pre)
                    for p in pre:
                        self.emit(depth, p)
                    self.emit(depth, f"{target[1]} = {val}")
            return
        if k == "if":
            pre = []
            c = self.cond(n[1], pre)
            for p in pre:
                self.emit(depth, p)
            self.emit(depth, f"if {c}:")
            self.body(self.as_list(n[2]), depth + 1)
            if n[3] is not None:
                self.emit(depth, "else:")
                self.body(self.as_list(n[3]), depth + 1)
            return
        if k == "for":
            self.for_loop(n, depth)
            return
        if k == "while":
            pre = []
            c = self.cond(n[1], pre)
            if pre:
                raise JSSyntaxError("side effects in a while condition")
            self.emit(depth, f"while {c}:")
            self.loop_updates.append(None)
            self.body(self.as_list(n[2]), depth + 1)
            self.loop_updates.pop()
            return
        if k == "return":
            pre = []
            v = "None" if n[1] is None else self.expr(n[1], pre)
            for p in pre:
                self.emit(depth, p)
            self.emit(depth, f"return {v}")
            return
        if k == "break":
            self.emit(depth, "break")
            return
        if k == "continue":
            upd = self.loop_updates[-1] if self.loop_updates else None
            if upd:
                for line in upd:
                    self.emit(depth, line)
            self.emit(depth, "continue")
            return
        if k == "throw":
            pre = []
            v = self.expr(n[1], pre)
            for p in pre:
                self.emit(depth, p)
            self.emit(depth, f"raise {v}")
            return
        if k == "funcdecl":
            self.function(n, depth)
            return
        if k == "class":
            self.class_def(n, depth)
            return
        raise JSSyntaxError(f"cannot translate statement {k}")

    def for_loop(self, n, depth):
        _, init, cond, upd, body = n
        body_list = self.as_list(body)
        self.scopes.append(set())
        # range fast path: for (let v = INT; v < B | v <= B; v++) with v, B untouched in the body
        if (init is not None and init[0] == "var" and len(init[1]) == 1
                and init[1][0][0][0] == "id" and init[1][0][1] is not None
                and cond is not None and cond[0] == "bin" and cond[1] in ("<", "<=")
                and cond[2] == ("id", init[1][0][0][1]) and _simple_bound(cond[3])
                and upd is not None and upd[0] in ("postfix", "prefix") and upd[1] == "++"
                and upd[2] == ("id", init[1][0][0][1])):
            v = init[1][0][0][1]
            start = init[1][0][1]
            is_int = start[0] == "num" and re.fullmatch(r"\d+", start[1]) or (
                start[0] == "unary" and start[1] == "-" and start[2][0] == "num"
                and re.fullmatch(r"\d+", start[2][1]))
            touched = _assigned_names(body_list, set())
            if is_int and v not in touched and not (_idents(cond[3], set()) & touched):
                self.declare(v)
                pre = []
                a = self.expr(start, pre)
                b = self.expr(cond[3], pre)
                bound = f"_js_ub_lt({b})" if cond[1] == "<" else f"_js_ub_le({b})"
                for p in pre:
                    self.emit(depth, p)
                self.emit(depth, f"for {v} in range({a}, {bound}):")
                self.loop_updates.append(None)
                self.body(body_list, depth + 1)
                self.loop_updates.pop()
                self.scopes.pop()
                return
        # general form
        if init is not None:
            if init[0] == "var":
                self.stmt(init, depth)
            else:
                self.stmt_expr(init[1], depth)
        pre = []
        c = "True" if cond is None else self.cond(cond, pre)
        if pre:
            raise JSSyntaxError("side effects in a for condition")
        upd_lines = []
        if upd is not None:
            save = self.lines
            self.lines = []
            self.stmt_expr(upd, 0)
            upd_lines = self.lines
            self.lines = save
        self.emit(depth, f"while {c}:")
        self.loop_updates.append(upd_lines)
        self.body(body_list, depth + 1)
        self.loop_updates.pop()
        for line in upd_lines:
            self.emit(depth + 1, line)
        self.scopes.pop()

    def params(self, ps, depth_body):
        names, defaults = [], []
        for name, default in ps:
            if default is None:
                names.append(name)
            else:
                names.append(f"{name}=None")
                defaults.append((name, default))
        return names, defaults

    def function(self, n, depth, method=False):
        _, name, ps, body = n
        names, defaults = self.params(ps, depth + 1)
        args = (["self"] if method else []) + names
        self.emit(depth, f"def {name}({', '.join(args)}):")
        saved_scopes, saved_loops = self.scopes, self.loop_updates
        self.scopes, self.loop_updates = [set(p for p, _ in ps)], []
        for pname, default in defaults:
            pre = []
            dv = self.expr(default, pre)
            self.emit(depth + 1, f"if {pname} is None:")
            self.emit(depth + 2, f"{pname} = {dv}")
        self.body(body, depth + 1, new_scope=False)
        self.scopes, self.loop_updates = saved_scopes, saved_loops

    def class_def(self, n, depth):
        _, name, methods = n
        self.emit(depth, f"class {name}:")
        if not methods:
            self.emit(depth + 1, "pass")
        for mname, ps, body in methods:
            pyname = "__init__" if mname == "constructor" else mname
            self.function(("funcdecl", pyname, ps, body), depth + 1, method=True)


def translate(src):
    """JavaScript source -> Python source (module level)."""
    prog = Parser(tokenize(src)).program()
    g = CodeGen()
    g.scopes = [set()]
    for s in prog:
        g.stmt(s, 0)
    return "\n".join(g.lines) + "\n"


# ----------------------------------------------------------------- runtime
class _JSError(Exception):
    pass


class _JSObject(dict):
    """A plain JS object literal: missing properties read as undefined (None)."""

    def __getattr__(self, k):
        return self.get(k)


def _typed(code, itemsize, name):
    class TypedArray(array.array):
        def __new__(cls, n):
            if isinstance(n, int):
                return super().__new__(cls, code, bytes(itemsize * n))
            return super().__new__(cls, code, n)

        def set(self, src, offset=0):  # TypedArray.prototype.set
            self[offset:offset + len(src)] = array.array(code, src)

        def fill(self, v):  # TypedArray.prototype.fill (whole array)
            self[:] = array.array(code, [v]) * len(self)
            return self

    TypedArray.__name__ = TypedArray.__qualname__ = name
    assert array.array(code).itemsize == itemsize
    return TypedArray


Float32Array = _typed("f", 4, "Float32Array")
Float64Array = _typed("d", 8, "Float64Array")
Int32Array = _typed("i", 4, "Int32Array")
Int8Array = _typed("b", 1, "Int8Array")
Uint8Array = _typed("B", 1, "Uint8Array")


def _js_truthy(x):
    return bool(x) and x == x


class _NanFalseType(float):
    """NaN that Python treats as falsy, as JS does."""

    def __bool__(self):
        return False


_NanFalse = _NanFalseType("nan")


def _js_falsy_nan(x):
    # a NaN operand of && / || behaves as falsy; other values pass through
    if isinstance(x, float) and x != x:
        return _NanFalse
    return x


def _js_nullish(a, b):
    return b if a is None else a


def _js_number(x):
    return float(x) if not isinstance(x, (int, float)) else x


def _js_toint32(x):
    if isinstance(x, bool):
        x = int(x)
    if not isinstance(x, int):
        if x != x or x in (math.inf, -math.inf):
            return 0
        x = int(x)  # truncation toward zero
    x &= 0xFFFFFFFF
    return x - (1 << 32) if x >= (1 << 31) else x


def _js_or(a, b):
    return _js_toint32(_js_toint32(a) | _js_toint32(b))


def _js_and(a, b):
    return _js_toint32(_js_toint32(a) & _js_toint32(b))


def _js_xor(a, b):
    return _js_toint32(_js_toint32(a) ^ _js_toint32(b))


def _js_shl(a, b):
    return _js_toint32(_js_toint32(a) << (_js_toint32(b) & 31))


def _js_sar(a, b):
    return _js_toint32(a) >> (_js_toint32(b) & 31)


def _js_shr(a, b):
    return (_js_toint32(a) & 0xFFFFFFFF) >> (_js_toint32(b) & 31)


def _js_not(a):
    return _js_toint32(~_js_toint32(a))


def _js_min(*a):
    if not a:
        return math.inf
    if any(x != x for x in a):
        return math.nan
    return min(a)


def _js_max(*a):
    if not a:
        return -math.inf
    if any(x != x for x in a):
        return math.nan
    return max(a)


def _js_sqrt(x):
    return math.sqrt(x) if x >= 0 else math.nan


def _js_log(x):
    if x != x or x < 0:
        return math.nan
    return math.log(x) if x > 0 else -math.inf


def _js_pow(a, b):
    return float(a) ** b


def _js_round(x):
    return math.floor(x + 0.5)


def _js_sign(x):
    return (x > 0) - (x < 0) if x == x else math.nan


def _js_mod(a, b):
    return math.fmod(a, b)


def _js_concat(a, b):
    return str(a) + str(b)


def _js_ub_lt(b):
    """Exclusive upper bound of `v < b` for integer v."""
    return b if isinstance(b, int) else math.ceil(b)


def _js_ub_le(b):
    """Exclusive upper bound of `v <= b` for integer v."""
    return b + 1 if isinstance(b, int) else math.floor(b) + 1


RUNTIME = {k: v for k, v in globals().items()
           if k.startswith("_js") or k in ("_JSError", "_JSObject", "Float32Array", "Float64Array",
                                           "Int32Array", "Int8Array", "Uint8Array")}


def load(sources):
    """Translate and execute JS sources (in order) in one namespace; returns it."""
    ns = {"math": math, "__name__": "jsmini_module"}
    ns.update(RUNTIME)
    for name, src in sources:
        code = translate(src)
        exec(compile(code, f"<{name} (translated)>", "exec"), ns)
    return ns
