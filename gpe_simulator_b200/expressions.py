"""Potential expressions: the reference's formula language, compiled for the C ABI.

The language (the one the reference's config editor accepts): finite numbers,
the variables ``x y z`` and the constant ``pi`` (plus ``t`` for time-dependent
potentials), ``+ - * / **``, unary ``+ -``, parentheses, and the one-argument
functions ``sin cos tan exp sqrt tanh abs log``.  Precedence and associativity
are Python's, which the reference parses with: ``-x**2`` is ``-(x**2)``,
``2**-1`` is ``2**(-1)``, ``**`` groups to the right, the others to the left.

This module has its own front end (a tokenizer and a recursive-descent parser
producing a small tuple tree), whose acceptance rules come from what the
device evaluator can run:

* every number must be a finite real (decimal literals only);
* the compiled program must fit ``GPE_PROGRAM_MAX`` doubles and need at most
  ``GPE_STACK_MAX - 1`` stack slots (``include/gpe_ssf.h``);
* nesting (parentheses, signs, powers) is bounded at 100 levels, which keeps
  the recursive descent within Python's recursion limit.

Integer literals in other bases (``0x10``) and comments are not accepted.

Outputs:

* ``cuda_expression`` renders the CUDA double text in the reference's format
  (``gpe/expressions.py:9-30``: constants as ``repr(float)``, ``**`` as ``pow``,
  ``abs`` as ``fabs``, every operation parenthesised), so a stage whose
  expressions the reference's YAML parser rendered carries identical strings;
* ``compile_program`` emits the stack-machine bytecode of ``include/gpe_ssf.h``;
* ``split_static`` separates a static potential into ``vx(x) + vy(y) + vz(z)``
  (terms of at most one coordinate, read from per-axis tables) and a general
  remainder (evaluated once into a device array);
* ``from_cuda_text`` reads such CUDA text back (``pow(a, b)``, ``fabs``).
"""

import math
import re

FUNCTIONS = ("sin", "cos", "tan", "exp", "sqrt", "tanh", "abs", "log")

OP_CONST, OP_X, OP_Y, OP_Z, OP_T = 1, 2, 3, 4, 5
OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_POW, OP_NEG = 6, 7, 8, 9, 10, 11
_FUNC_OP = {"sin": 13, "cos": 14, "tan": 15, "exp": 16, "sqrt": 17, "tanh": 18, "abs": 19, "log": 20}
_BIN_OP = {"+": OP_ADD, "-": OP_SUB, "*": OP_MUL, "/": OP_DIV, "**": OP_POW}
_VAR_OP = {"x": OP_X, "y": OP_Y, "z": OP_Z, "t": OP_T}
STACK_MAX = 32        # GPE_STACK_MAX
PROGRAM_MAX = 2048    # GPE_PROGRAM_MAX (doubles)
_SOURCE_MAX = 16384   # characters
_DEPTH_MAX = 100      # nesting of the recursive descent (parentheses, signs, powers)

_TOKEN = re.compile(r"""
    (?P<ws>\s+)
  | (?P<num>(?:\d(?:_?\d)*(?:\.(?:\d(?:_?\d)*)?)?|\.\d(?:_?\d)*)(?:[eE][+-]?\d(?:_?\d)*)?)
  | (?P<name>[A-Za-z_][A-Za-z0-9_]*)
  | (?P<op>\*\*|[-+*/(),])
""", re.VERBOSE)


class _Parser:
    """Recursive descent over the token list; ``cuda`` also reads the CUDA
    rendering's two-argument ``pow`` and its ``fabs``."""

    def __init__(self, source, time_dependent, cuda=False):
        if not isinstance(source, str):
            raise ValueError("a potential expression must be a string")
        if len(source) > _SOURCE_MAX:
            raise ValueError(f"potential expression longer than {_SOURCE_MAX} characters")
        self.src = source
        self.names = {"x", "y", "z"} | ({"t"} if time_dependent else set())
        self.cuda = cuda
        self.toks = []
        pos = 0
        while pos < len(source):
            m = _TOKEN.match(source, pos)
            if not m:
                raise ValueError(f"potential expression: unexpected {source[pos]!r} at column {pos + 1}")
            kind = m.lastgroup
            if kind != "ws":
                self.toks.append((kind, m.group(), pos))
            pos = m.end()
        self.i = 0
        self.depth = 0

    # token helpers
    def peek(self):
        return self.toks[self.i] if self.i < len(self.toks) else ("end", "", len(self.src))

    def take(self, text=None):
        tok = self.peek()
        if text is not None and tok[1] != text:
            self.fail(tok, f"expected {text!r}")
        self.i += 1
        return tok

    def fail(self, tok, why):
        where = "at the end" if tok[0] == "end" else f"at column {tok[2] + 1} ({tok[1]!r})"
        raise ValueError(f"potential expression: {why} {where}")

    def nest(self):
        self.depth += 1
        if self.depth > _DEPTH_MAX:
            raise ValueError("potential expression nested too deeply")

    # grammar
    def parse(self):
        if not self.toks:
            raise ValueError("potential expression is empty (write 0 for no potential)")
        tree = self.sum()
        if self.peek()[0] != "end":
            self.fail(self.peek(), "unexpected token")
        return tree

    def sum(self):
        left = self.product()
        while self.peek()[1] in ("+", "-"):
            op = self.take()[1]
            left = ("bin", op, left, self.product())
        return left

    def product(self):
        left = self.unary()
        while self.peek()[1] in ("*", "/"):
            op = self.take()[1]
            left = ("bin", op, left, self.unary())
        return left

    def unary(self):
        tok = self.peek()
        if tok[1] in ("+", "-"):
            self.take()
            self.nest()
            inner = self.unary()
            self.depth -= 1
            return ("neg" if tok[1] == "-" else "pos", inner)
        return self.power()

    def power(self):
        base = self.atom()
        if self.peek()[1] == "**":
            self.take()
            self.nest()
            exponent = self.unary()     # right operand may carry its own sign; groups right
            self.depth -= 1
            return ("bin", "**", base, exponent)
        return base

    def atom(self):
        tok = self.take()
        kind, text = tok[0], tok[1]
        if kind == "num":
            nxt = self.peek()
            if nxt[0] == "name" and nxt[2] == tok[2] + len(text):
                self.fail(nxt, "a number runs into a name")
            digits = text.replace("_", "")
            if re.fullmatch(r"0\d+", digits) and set(digits) != {"0"}:
                self.fail(tok, "decimal integers do not start with 0")
            try:
                value = float(digits)
            except OverflowError:
                value = math.inf
            if not math.isfinite(value):
                self.fail(tok, "numbers must be finite")
            return ("num", value)
        if kind == "name":
            if self.peek()[1] == "(":
                return self.call(tok)
            if text == "pi":
                return ("pi",)
            if text in self.names:
                return ("var", text)
            if text in FUNCTIONS:
                self.fail(tok, f"{text} is a function: write {text}(...)")
            self.fail(tok, "unknown name (variables are " + ", ".join(sorted(self.names)) + " and pi)")
        if text == "(":
            self.nest()
            inner = self.sum()
            self.depth -= 1
            self.take(")")
            return inner
        self.fail(tok, "expected a number, a name or '('")

    def call(self, tok):
        name = tok[1]
        self.take("(")
        self.nest()
        if self.cuda and name == "pow":
            a = self.sum()
            self.take(",")
            b = self.sum()
            self.take(")")
            self.depth -= 1
            return ("bin", "**", a, b)
        if self.cuda and name == "fabs":
            name = "abs"
        if name not in FUNCTIONS:
            self.fail(tok, "unknown function (functions are " + ", ".join(FUNCTIONS) + ")")
        arg = self.sum()
        if self.peek()[1] == ",":
            self.fail(self.peek(), f"{name} takes one argument")
        self.take(")")
        self.depth -= 1
        return ("call", name, arg)


def parse_expression(source, time_dependent=False):
    """The expression tree of ``source``; ``ValueError`` for anything outside the
    language or beyond the device evaluator's limits."""
    tree = _Parser(source.strip() if isinstance(source, str) else source, time_dependent).parse()
    program_of(tree)   # size and stack limits of the device evaluator
    return tree


# ------------------------------------------------------------------ tree walks
# Trees of long sums are deep on their left spine, so every walk is iterative.
def _children(node):
    kind = node[0]
    if kind in ("neg", "pos"):
        return (node[1],)
    if kind == "call":
        return (node[2],)
    if kind == "bin":
        return (node[2], node[3])
    return ()


def _postorder(node):
    """Nodes of the tree in post-order (children before their parent)."""
    order, stack = [], [(node, False)]
    while stack:
        nd, expanded = stack.pop()
        kids = _children(nd)
        if kids and not expanded:
            stack.append((nd, True))
            stack.extend((k, False) for k in reversed(kids))
        else:
            order.append(nd)
    return order


def _render(node, cuda):
    vals = []
    for nd in _postorder(node):
        kind = nd[0]
        if kind == "num":
            vals.append(repr(float(nd[1])))
        elif kind == "pi":
            vals.append(repr(math.pi) if cuda else "pi")
        elif kind == "var":
            vals.append(nd[1])
        elif kind in ("neg", "pos"):
            vals.append(f"({'-' if kind == 'neg' else '+'}{vals.pop()})")
        elif kind == "call":
            name = "fabs" if cuda and nd[1] == "abs" else nd[1]
            vals.append(f"{name}({vals.pop()})")
        else:
            b, a = vals.pop(), vals.pop()
            vals.append(f"pow({a}, {b})" if cuda and nd[1] == "**" else f"({a} {nd[1]} {b})")
    return vals[0]


def cuda_expression(source, time_dependent=False):
    """CUDA double text of an expression, in the reference's format."""
    return _render(parse_expression(source, time_dependent), cuda=True)


def from_cuda_text(text):
    """The expression (in the formula language) of the reference's CUDA text.

    ``stage.potential_params[...]['expression']`` holds ``cuda_expression``'s
    output (``gpe/yaml_parser.py:44-46``); ``pow(a, b)`` reads as ``a ** b`` and
    ``fabs`` as ``abs``.  ``t`` is allowed; the caller's compile step decides
    whether the potential may depend on time.
    """
    return _render(_Parser(text.strip(), True, cuda=True).parse(), cuda=False)


# ------------------------------------------------------------------ bytecode
def _emit(node, out):
    """Append the post-order bytecode of ``node`` to ``out``; returns the stack
    depth it needs."""
    depths = []
    for nd in _postorder(node):
        kind = nd[0]
        if kind in ("num", "pi"):
            out += [OP_CONST, float(nd[1]) if kind == "num" else math.pi]
            depths.append(1)
        elif kind == "var":
            out.append(_VAR_OP[nd[1]])
            depths.append(1)
        elif kind == "neg":
            out.append(OP_NEG)
        elif kind == "call":
            out.append(_FUNC_OP[nd[1]])
        elif kind == "bin":
            d2, d1 = depths.pop(), depths.pop()
            out.append(_BIN_OP[nd[1]])
            depths.append(max(d1, d2 + 1))
    return depths[0]


def _checked(out, depth):
    if depth > STACK_MAX - 1:
        raise ValueError(f"potential expression needs {depth} stack slots; the device evaluator has "
                         f"{STACK_MAX - 1}")
    if len(out) > PROGRAM_MAX:
        raise ValueError(f"potential expression compiles to {len(out)} values; the device evaluator "
                         f"takes at most {PROGRAM_MAX}")
    return [float(v) for v in out]


def program_of(tree):
    out = []
    depth = _emit(tree, out)
    return _checked(out, depth)


def is_zero(node):
    while node[0] in ("neg", "pos"):
        node = node[1]
    return node[0] == "num" and node[1] == 0.0


def compile_program(source, time_dependent=False):
    """Bytecode for ``source`` (empty list for the zero potential)."""
    tree = parse_expression(source, time_dependent)
    return [] if is_zero(tree) else program_of(tree)


def _variables(node):
    return {nd[1] for nd in _postorder(node) if nd[0] == "var"}


def _terms(node):
    """The top-level sum as (sign, term) pairs, in order."""
    out, stack = [], [(node, 1)]
    while stack:
        nd, sign = stack.pop()
        if nd[0] == "bin" and nd[1] in ("+", "-"):
            stack.append((nd[3], sign if nd[1] == "+" else -sign))
            stack.append((nd[2], sign))
        elif nd[0] in ("neg", "pos"):
            stack.append((nd[1], -sign if nd[0] == "neg" else sign))
        else:
            out.append((sign, nd))
    return out


def _sum_program(terms):
    if not terms:
        return []
    out, depth = [], 0
    for idx, (sign, node) in enumerate(terms):
        depth = max(depth, _emit(node, out) + (1 if idx else 0))
        if sign < 0:
            out.append(OP_NEG)
        if idx:
            out.append(OP_ADD)
    return _checked(out, depth)


def split_static(source):
    """Programs ``(vx, vy, vz, vg)`` whose sum is the static potential ``source``."""
    tree = parse_expression(source, time_dependent=False)
    groups = {"x": [], "y": [], "z": [], "g": []}
    if not is_zero(tree):
        for sign, term in _terms(tree):
            names = _variables(term)
            key = "x" if not names else (names.pop() if len(names) == 1 else "g")
            groups[key].append((sign, term))
    return tuple(_sum_program(groups[key]) for key in ("x", "y", "z", "g"))
