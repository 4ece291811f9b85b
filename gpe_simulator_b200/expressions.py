"""Potential expressions: the reference grammar, compiled for the C ABI.

Grammar (``config_editor/expressions.py:8-58``): finite numbers, ``x y z pi``
(and ``t`` for time-dependent potentials), ``+ - * / **``, unary ``+ -`` and
``sin cos tan exp sqrt tanh abs log`` of one argument.

* ``cuda_expression`` renders the same CUDA double text as the reference
  (``gpe/expressions.py:9-30``), so YAML-parsed stages carry identical strings.
* ``compile_program`` turns an expression into the stack-machine bytecode of
  ``include/gpe_ssf.h`` (evaluated in FP64 on the device).
* ``split_static`` separates a static potential into ``vx(x) + vy(y) + vz(z)``
  (terms of at most one coordinate, read from per-axis tables) and a general
  remainder (evaluated once into a device array).
"""

import ast
import math

FUNCTIONS = {"sin", "cos", "tan", "exp", "sqrt", "tanh", "abs", "log"}
_BINARY = (ast.Add, ast.Sub, ast.Mult, ast.Div, ast.Pow)

OP_CONST, OP_X, OP_Y, OP_Z, OP_T = 1, 2, 3, 4, 5
OP_ADD, OP_SUB, OP_MUL, OP_DIV, OP_POW, OP_NEG = 6, 7, 8, 9, 10, 11
_FUNC_OP = {"sin": 13, "cos": 14, "tan": 15, "exp": 16, "sqrt": 17, "tanh": 18, "abs": 19, "log": 20}
_BIN_OP = {ast.Add: OP_ADD, ast.Sub: OP_SUB, ast.Mult: OP_MUL, ast.Div: OP_DIV, ast.Pow: OP_POW}
_VAR_OP = {"x": OP_X, "y": OP_Y, "z": OP_Z, "t": OP_T}
STACK_MAX = 32


def parse_expression(source, time_dependent=False):
    """Validate ``source``; same acceptance and messages' intent as the reference."""
    if not isinstance(source, str) or not source.strip():
        raise ValueError("Enter a formula, or 0 to disable this potential.")
    if len(source) > 4096:
        raise ValueError("Keep the formula within 4096 characters.")
    try:
        tree = ast.parse(source.strip(), mode="eval").body
    except (SyntaxError, RecursionError) as exc:
        raise ValueError(f"Syntax error: {getattr(exc, 'msg', 'expression is too deeply nested')}.") from exc
    if sum(1 for _ in ast.walk(tree)) > 256:
        raise ValueError("The formula is too complex; use a shorter expression.")
    names = {"x", "y", "z", "pi"} | ({"t"} if time_dependent else set())

    def check(node):
        if isinstance(node, ast.Constant):
            ok = type(node.value) in (int, float)
            try:
                ok = ok and math.isfinite(node.value)
            except OverflowError:
                ok = False
            if not ok:
                raise ValueError("Use finite real numbers in the formula.")
        elif isinstance(node, ast.Name):
            if node.id not in names:
                raise ValueError(f"Unrecognised variable {node.id}.")
        elif isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.UAdd, ast.USub)):
            check(node.operand)
        elif isinstance(node, ast.BinOp) and isinstance(node.op, _BINARY):
            check(node.left)
            check(node.right)
        elif isinstance(node, ast.Call):
            if not isinstance(node.func, ast.Name) or node.func.id not in FUNCTIONS:
                raise ValueError("Unrecognised function.")
            if len(node.args) != 1 or node.keywords:
                raise ValueError(f"{node.func.id} expects one positional argument.")
            check(node.args[0])
        else:
            raise ValueError("Use numbers, coordinates, + - * / **, parentheses and the listed functions.")

    check(tree)
    return tree


def cuda_expression(source, time_dependent=False):
    """CUDA double text of an expression (output format of ``gpe/expressions.py``)."""
    tree = parse_expression(source, time_dependent)

    def render(node):
        if isinstance(node, ast.Constant):
            return repr(float(node.value))
        if isinstance(node, ast.Name):
            return repr(math.pi) if node.id == "pi" else node.id
        if isinstance(node, ast.UnaryOp):
            return f"({'-' if isinstance(node.op, ast.USub) else '+'}{render(node.operand)})"
        if isinstance(node, ast.Call):
            return f"{'fabs' if node.func.id == 'abs' else node.func.id}({render(node.args[0])})"
        left, right = render(node.left), render(node.right)
        if isinstance(node.op, ast.Pow):
            return f"pow({left}, {right})"
        op = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*", ast.Div: "/"}[type(node.op)]
        return f"({left} {op} {right})"

    return render(tree)


def _emit(node, out):
    """Post-order bytecode; returns the stack depth the subtree needs."""
    if isinstance(node, ast.Constant):
        out += [OP_CONST, float(node.value)]
        return 1
    if isinstance(node, ast.Name):
        if node.id == "pi":
            out += [OP_CONST, math.pi]
        else:
            out.append(_VAR_OP[node.id])
        return 1
    if isinstance(node, ast.UnaryOp):
        d = _emit(node.operand, out)
        if isinstance(node.op, ast.USub):
            out.append(OP_NEG)
        return d
    if isinstance(node, ast.Call):
        d = _emit(node.args[0], out)
        out.append(_FUNC_OP[node.func.id])
        return d
    d1 = _emit(node.left, out)
    d2 = _emit(node.right, out)
    out.append(_BIN_OP[type(node.op)])
    return max(d1, d2 + 1)


def program_of(tree):
    out = []
    depth = _emit(tree, out)
    if depth > STACK_MAX - 1:
        raise ValueError("The formula is nested too deeply for the device evaluator.")
    return [float(v) for v in out]


def compile_program(source, time_dependent=False):
    """Bytecode for ``source`` (empty list for the zero potential)."""
    tree = parse_expression(source, time_dependent)
    if is_zero(tree):
        return []
    return program_of(tree)


def is_zero(node):
    while isinstance(node, ast.UnaryOp):
        node = node.operand
    return isinstance(node, ast.Constant) and node.value == 0


def _variables(node):
    return {n.id for n in ast.walk(node) if isinstance(n, ast.Name) and n.id in ("x", "y", "z", "t")}


def _terms(node, sign=1):
    """Flatten top-level sums into (sign, term) pairs."""
    if isinstance(node, ast.BinOp) and isinstance(node.op, (ast.Add, ast.Sub)):
        left = _terms(node.left, sign)
        right = _terms(node.right, sign if isinstance(node.op, ast.Add) else -sign)
        return left + right
    if isinstance(node, ast.UnaryOp):
        return _terms(node.operand, sign if isinstance(node.op, ast.UAdd) else -sign)
    return [(sign, node)]


def _sum_program(terms):
    if not terms:
        return []
    out = []
    for idx, (sign, node) in enumerate(terms):
        depth = _emit(node, out)
        if depth > STACK_MAX - 2:
            raise ValueError("The formula is nested too deeply for the device evaluator.")
        if sign < 0:
            out.append(OP_NEG)
        if idx:
            out.append(OP_ADD)
    return [float(v) for v in out]


def split_static(source):
    """Programs ``(vx, vy, vz, vg)`` whose sum is the static potential ``source``."""
    tree = parse_expression(source, time_dependent=False)
    groups = {"x": [], "y": [], "z": [], "g": []}
    if not is_zero(tree):
        for sign, term in _terms(tree):
            names = _variables(term)
            if not names:
                groups["x"].append((sign, term))
            elif len(names) == 1:
                groups[names.pop()].append((sign, term))
            else:
                groups["g"].append((sign, term))
    return tuple(_sum_program(groups[key]) for key in ("x", "y", "z", "g"))


def from_cuda_text(text):
    """Recover an expression tree from the reference's CUDA text.

    ``stage.potential_params[...]['expression']`` holds the output of
    ``cuda_expression`` (``gpe/yaml_parser.py:44-46``); it is valid Python once
    ``pow(a, b)`` is read as ``a ** b`` and ``fabs`` as ``abs``.
    """
    tree = ast.parse(text.strip(), mode="eval").body

    class Fix(ast.NodeTransformer):
        def visit_Call(self, node):
            self.generic_visit(node)
            if isinstance(node.func, ast.Name) and node.func.id == "pow" and len(node.args) == 2:
                return ast.copy_location(ast.BinOp(left=node.args[0], op=ast.Pow(), right=node.args[1]), node)
            if isinstance(node.func, ast.Name) and node.func.id == "fabs":
                node.func.id = "abs"
            return node

    return ast.unparse(ast.fix_missing_locations(Fix().visit(tree)))
