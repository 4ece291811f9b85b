"""NumPy evaluator for the reference's potential-expression grammar.

TEST INFRASTRUCTURE ONLY (see ``oracle/__init__.py``).

The grammar is the one accepted by ``config_editor/expressions.py:12-58``
(``parse_expression``): finite numbers, the variables ``x y z pi`` (plus ``t``
for time-dependent potentials), ``+ - * / **``, unary ``+``/``-`` and the
one-argument functions ``sin cos tan exp sqrt tanh abs log``
(``config_editor/expressions.py:8``).  ``gpe/expressions.py:9-30`` renders the
same tree into CUDA double arithmetic (``**`` -> ``pow``, ``abs`` -> ``fabs``,
``pi`` -> ``repr(math.pi)``); evaluating the tree with float64 NumPy ufuncs
gives the same values up to libm rounding.
"""

import ast
import math

import numpy as np

_FUNCS = {"sin": np.sin, "cos": np.cos, "tan": np.tan, "exp": np.exp,
          "sqrt": np.sqrt, "tanh": np.tanh, "abs": np.abs, "log": np.log}


def parse(source, time_dependent=False):
    """Parse and validate ``source``; raises ValueError like the reference."""
    if not isinstance(source, str) or not source.strip():
        raise ValueError("empty expression")
    tree = ast.parse(source.strip(), mode="eval").body
    names = {"x", "y", "z", "pi"} | ({"t"} if time_dependent else set())

    def check(node):
        if isinstance(node, ast.Constant):
            if type(node.value) not in (int, float) or not math.isfinite(node.value):
                raise ValueError("non-finite constant")
        elif isinstance(node, ast.Name):
            if node.id not in names:
                raise ValueError(f"unknown variable {node.id}")
        elif isinstance(node, ast.UnaryOp) and isinstance(node.op, (ast.UAdd, ast.USub)):
            check(node.operand)
        elif isinstance(node, ast.BinOp) and isinstance(
                node.op, (ast.Add, ast.Sub, ast.Mult, ast.Div, ast.Pow)):
            check(node.left)
            check(node.right)
        elif (isinstance(node, ast.Call) and isinstance(node.func, ast.Name)
              and node.func.id in _FUNCS and len(node.args) == 1 and not node.keywords):
            check(node.args[0])
        else:
            raise ValueError("unsupported syntax")

    check(tree)
    return tree


def evaluate(source, x, y, z, t=0.0, time_dependent=False):
    """Evaluate ``source`` in float64 on broadcastable coordinate arrays."""
    tree = parse(source, time_dependent)
    env = {"x": np.asarray(x, np.float64), "y": np.asarray(y, np.float64),
           "z": np.asarray(z, np.float64), "t": np.float64(t), "pi": np.float64(math.pi)}

    def ev(node):
        if isinstance(node, ast.Constant):
            return np.float64(node.value)
        if isinstance(node, ast.Name):
            return env[node.id]
        if isinstance(node, ast.UnaryOp):
            value = ev(node.operand)
            return -value if isinstance(node.op, ast.USub) else +value
        if isinstance(node, ast.Call):
            return _FUNCS[node.func.id](ev(node.args[0]))
        a, b = ev(node.left), ev(node.right)
        op = type(node.op)
        if op is ast.Add:
            return a + b
        if op is ast.Sub:
            return a - b
        if op is ast.Mult:
            return a * b
        if op is ast.Div:
            return a / b
        return np.power(a, b)

    return ev(tree)
