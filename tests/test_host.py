"""Host-side logic that needs no GPU: expressions, bytecode, shells, C-ABI symbols."""

import ctypes
import math
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from oracle import expr as oexpr
from oracle import ssf

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "gpe_ssf.h"


# ------------------------------------------------------------------ expressions
def test_cuda_expression_matches_reference_rendering():
    """Strings the reference's own tests pin (``tests/test_workflow.py:25-32``)."""
    from gpe_simulator_b200.expressions import cuda_expression
    assert cuda_expression("1/2*y**2") == "((1.0 / 2.0) * pow(y, 2.0))"
    assert cuda_expression("abs(-x) + cos(t)", True) == "(fabs((-x)) + cos(t))"
    assert cuda_expression("pi") == repr(np.pi)
    with pytest.raises(ValueError):
        cuda_expression("t*y")
    with pytest.raises(ValueError):
        cuda_expression("x; return 0")


def test_expression_front_end_matches_the_reference_renderings():
    """Every formula of the fixture (generated by the reference's own
    ``cuda_expression``, ``tests/golden/make_expr_cases.py``) renders to the same
    CUDA text here, and what the reference rejects is rejected here too."""
    import json
    from gpe_simulator_b200.expressions import cuda_expression
    rows = json.loads((ROOT / "tests" / "golden" / "expr_cases.json").read_text())
    assert len(rows) > 40
    for row in rows:
        if row["cuda"] is None:
            with pytest.raises(ValueError):
                cuda_expression(row["source"], row["time_dependent"])
        else:
            assert cuda_expression(row["source"], row["time_dependent"]) == row["cuda"], row["source"]


def test_expression_limits_come_from_the_device_evaluator():
    from gpe_simulator_b200.expressions import compile_program, STACK_MAX, PROGRAM_MAX
    deep = "x*" + "(y+" * STACK_MAX + "z" + ")" * STACK_MAX
    with pytest.raises(ValueError, match="stack"):
        compile_program(deep)
    long_sum = "+".join(["x*y"] * (PROGRAM_MAX // 2))
    with pytest.raises(ValueError, match="at most"):
        compile_program(long_sum)
    with pytest.raises(ValueError, match="nested"):
        compile_program("(" * 150 + "x" + ")" * 150)
    assert compile_program("0") == [] and compile_program("-(0.0)") == []


def run_program(prog, x, y, z, t=0.0):
    """Python model of the device stack machine (same opcodes as include/gpe_ssf.h)."""
    st = []
    pc = 0
    fn = {13: np.sin, 14: np.cos, 15: np.tan, 16: np.exp, 17: np.sqrt, 18: np.tanh, 19: np.abs, 20: np.log}
    while pc < len(prog):
        op = int(prog[pc]); pc += 1
        if op == 1:
            st.append(prog[pc]); pc += 1
        elif op in (2, 3, 4, 5):
            st.append({2: x, 3: y, 4: z, 5: t}[op])
        elif op in (6, 7, 8, 9, 10):
            b, a = st.pop(), st.pop()
            ops = {6: lambda: a + b, 7: lambda: a - b, 8: lambda: a * b, 9: lambda: a / b,
                   10: lambda: a ** b}
            st.append(ops[op]())
        elif op == 11:
            st.append(-st.pop())
        else:
            st.append(fn[op](st.pop()))
    assert len(st) == 1
    return st[0]


EXPRS = ["x**2+1.44*y**2+2.25*z**2", "x/2 + y**2/10 + abs(z)/5", "0.002*(x*x + y*y + z*z)",
         "-(x-1)**2 + 3*sin(y)*cos(z) - exp(-x*x)", "sqrt(x*x+y*y) - tanh(z) + log(2+x)", "1/2", "pi*x"]


@pytest.mark.parametrize("source", EXPRS)
def test_bytecode_and_separable_split_evaluate_like_the_oracle(source):
    from gpe_simulator_b200.expressions import compile_program, split_static
    rng = np.random.default_rng(0)
    x, y, z = rng.uniform(0.1, 2.0, 3)
    want = oexpr.evaluate(source, x, y, z)
    assert run_program(compile_program(source), x, y, z) == pytest.approx(want, rel=1e-14, abs=1e-14)
    px, py, pz, pg = split_static(source)
    parts = [run_program(px, x, 0, 0) if px else 0.0, run_program(py, 0, y, 0) if py else 0.0,
             run_program(pz, 0, 0, z) if pz else 0.0, run_program(pg, x, y, z) if pg else 0.0]
    assert sum(parts) == pytest.approx(want, rel=1e-13, abs=1e-13)


def test_separable_trap_has_no_general_part():
    from gpe_simulator_b200.expressions import split_static
    px, py, pz, pg = split_static("x**2+1.44*y**2+2.25*z**2")
    assert px and py and pz and not pg
    assert split_static("x*y")[3]


def test_time_dependent_bytecode():
    from gpe_simulator_b200.expressions import compile_program
    beam = ssf.Beam(20.0, 0.5, 2.0, 1.0, 0.05)
    src = beam.expression()
    for t in (0.0, 0.01, 0.07):
        got = run_program(compile_program(src, time_dependent=True), 1.2, -0.3, 0.4, t)
        assert got == pytest.approx(float(beam.value(1.2, -0.3, t)), rel=1e-13)


def test_reference_cuda_text_round_trips():
    from gpe_simulator_b200.expressions import cuda_expression, from_cuda_text
    for source in EXPRS:
        back = from_cuda_text(cuda_expression(source))
        x, y, z = 0.7, -1.1, 0.3
        assert oexpr.evaluate(back, x, y, z) == pytest.approx(oexpr.evaluate(source, x, y, z), rel=1e-15)


# ------------------------------------------------------------------ n(k) geometry
@pytest.mark.parametrize("n", [2, 7, 8, 18, 256, 512])
def test_reference_shell_count(n):
    from gpe_simulator_b200.nk_extraction import shell_geometry
    nb, width = shell_geometry(n, 0.5)
    assert nb == ssf.reference_nbins(n) and width == 0.5
    assert ssf.reference_nbins(256) == 223 and ssf.reference_nbins(512) == 444


def test_assemble_matches_oracle_dictionary():
    from gpe_simulator_b200.nk_extraction import assemble
    n, L = 8, 2 * np.pi
    x, k = ssf.get_grids(n, L)
    F = np.fft.fftn(np.random.default_rng(1).normal(size=(n, n, n)) + 0j)
    want = ssf.nk_extraction(F, x, k)
    got = assemble(want["Nk"], want["counts"], n, 1.0)
    for key in want:
        np.testing.assert_allclose(got[key], want[key])


# ------------------------------------------------------------------ C ABI
def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^\s*(?:int|const char\*)\s+(gpe_\w+)\s*\(", text, re.M)))


def test_library_exports_every_declared_symbol():
    from gpe_simulator_b200 import _lib, build
    build.build()
    lib = ctypes.CDLL(str(_lib.LIB_PATH))
    names = declared_functions()
    assert len(names) >= 15
    for name in names:
        assert hasattr(lib, name), name
        assert name in _lib.SIGNATURES, f"{name} has no ctypes signature"


def test_desc_struct_layout_matches_header(tmp_path):
    """Offsets of gpe_desc as compiled by gcc equal the ctypes Structure's."""
    from gpe_simulator_b200 import _lib
    fields = [f for f, _ in _lib.Desc._fields_]
    src = tmp_path / "layout.c"
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    lines += [f'printf("%zu\\n", offsetof(gpe_desc, {f}));' for f in fields]
    lines += ['printf("%zu\\n", sizeof(gpe_desc));', "return 0;}"]
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", str(src), "-o", str(exe)], check=True)
    out = [int(v) for v in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    want = [getattr(_lib.Desc, f).offset for f in fields] + [ctypes.sizeof(_lib.Desc)]
    assert out == want


def test_status_codes_map_to_reference_exceptions():
    from gpe_simulator_b200 import _lib
    _lib.load()
    _lib.check(_lib.GPE_OK)
    with pytest.raises(ValueError):
        _lib.check(_lib.GPE_ERR_ARG)
    with pytest.raises(MemoryError):
        _lib.check(_lib.GPE_ERR_OOM)
    with pytest.raises(_lib.GpeError):
        _lib.check(_lib.GPE_ERR_CUDA)


def test_plan_create_rejects_bad_descriptors_without_a_gpu():
    """Argument validation runs before any device call."""
    from gpe_simulator_b200 import _lib
    lib = _lib.load()
    d = _lib.Desc()
    d.n = 17 * 19
    h = ctypes.c_void_p()
    assert lib.gpe_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.GPE_ERR_UNSUPPORTED
    assert "prime factor" in _lib.last_error()
    d.n = 1
    assert lib.gpe_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.GPE_ERR_UNSUPPORTED
    d.n, d.dtype = 16, 7
    assert lib.gpe_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.GPE_ERR_ARG
    x = (ctypes.c_double * 16)(*np.linspace(-1, 1, 16))
    d.dtype, d.kind, d.x_array, d.k_array = 0, 0, x, x
    bad = (ctypes.c_double * 3)(2.0, 6.0, 6.0)  # x, ADD with one operand on the stack
    d.static_g, d.static_g_len = bad, 3
    assert lib.gpe_plan_create(ctypes.byref(d), ctypes.byref(h)) == _lib.GPE_ERR_ARG
    assert "program" in _lib.last_error()


def test_path_tuner_picks_and_caches_the_fastest_candidate(tmp_path, monkeypatch):
    """``Plan(path="auto")``'s choice: every candidate timed once per (device, n,
    dtype, kind), the fastest kept in the JSON cache; no timing on a cache hit or
    where only one path exists."""
    import json
    import torch
    from gpe_simulator_b200 import tune
    monkeypatch.setenv("GPE_TUNE_CACHE", str(tmp_path / "paths.json"))
    x = np.linspace(-6, 6, 128, endpoint=False)
    k = 2 * np.pi * np.fft.fftfreq(128, 12 / 128)
    calls = []
    times = {"default": 0.30, "tma": 0.31, "plane": 0.29}

    def timer(p):
        calls.append(p)
        return times[p]

    def choose(n=128, dtype=torch.complex64, kind="real", dev="gpu-a"):
        return tune.choose_path(n, x, k, dtype, kind, device_name=dev, timer=timer)

    assert choose() == "plane"
    assert sorted(calls) == sorted(tune.CANDIDATES)
    calls.clear()
    assert choose() == "plane" and calls == []                     # cached
    assert choose(kind="imaginary") == "plane" and len(calls) == 3   # keyed by kind
    calls.clear()
    times["plane"] = 0.5
    assert choose(n=256) == "default" and len(calls) == 3           # keyed by size
    assert choose(dev="gpu-b") == "default"                          # keyed by device
    calls.clear()
    assert choose(n=64) == "default" and calls == []                # one path only
    assert choose(dtype=torch.complex128) == "default" and calls == []
    cache = json.loads((tmp_path / "paths.json").read_text())
    entry = cache["gpu-a|n=128|complex64|real"]
    assert entry["path"] == "plane" and set(entry["ms_per_step"]) == set(tune.CANDIDATES)


def test_ctypes_signatures_match_the_header_prototypes():
    """Every prototype in include/gpe_ssf.h and its ctypes argtypes agree in the
    number of parameters and in each scalar type (pointers as any pointer type)."""
    from gpe_simulator_b200 import _lib
    text = Path(HEADER).read_text()
    text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
    protos = dict(re.findall(r"^\s*(?:int|const char\*)\s+(gpe_\w+)\s*\(([^)]*)\)\s*;", text, re.M))
    assert set(protos) == set(declared_functions())
    scalar = {"double": ctypes.c_double, "int": ctypes.c_int, "long long": ctypes.c_longlong,
              "unsigned": ctypes.c_uint, "size_t": ctypes.c_size_t}
    pointer_like = (ctypes.c_void_p, ctypes.c_char_p)
    for name, params in protos.items():
        params = " ".join(params.split())
        parts = [] if params in ("", "void") else [p.strip() for p in params.split(",")]
        argtypes = _lib.SIGNATURES[name]
        assert len(parts) == len(argtypes), (name, parts, argtypes)
        for p, t in zip(parts, argtypes):
            if "*" in p:
                assert t in pointer_like or issubclass(t, ctypes._Pointer), (name, p, t)
            else:
                base = re.sub(r"^const\s+", "", p).rsplit(" ", 1)[0]
                assert t is scalar[base], (name, p, t)


def test_python_constants_match_the_header():
    """Status codes, dtype/kind/potential kinds, bytecode opcodes and projection
    bits as the Python layer spells them equal the header's #defines."""
    from gpe_simulator_b200 import _lib, expressions
    from gpe_simulator_b200.plan import Plan
    defs = {k: int(v) for k, v in re.findall(r"^#define\s+(GPE_\w+)\s+(\d+)u?\b", Path(HEADER).read_text(), re.M)}
    for name in ("GPE_OK", "GPE_ERR_ARG", "GPE_ERR_UNSUPPORTED", "GPE_ERR_CUDA", "GPE_ERR_OOM",
                 "GPE_ERR_NONFINITE", "GPE_ERR_TIMEOUT"):
        assert getattr(_lib, name) == defs[name], name
    for py, c in (("C64", "GPE_C64"), ("C128", "GPE_C128"), ("IMAGINARY", "GPE_IMAGINARY"), ("REAL", "GPE_REAL"),
                  ("V_NONE", "GPE_V_NONE"), ("V_REAL64", "GPE_V_REAL64"), ("V_CPLX128", "GPE_V_CPLX128")):
        assert getattr(_lib, py) == defs[c], py
    for op in ("CONST", "X", "Y", "Z", "T", "ADD", "SUB", "MUL", "DIV", "POW", "NEG"):
        assert getattr(expressions, "OP_" + op) == defs["GPE_OP_" + op], op
    for fn, code in expressions._FUNC_OP.items():
        assert code == defs["GPE_OP_" + fn.upper()], fn
    for i, name in enumerate(Plan.PROJECTIONS):
        assert defs["GPE_PROJ_" + name.upper()] == 1 << i, name


def test_product_code_does_not_reach_the_oracle():
    """The package never imports ``oracle``; bench.py imports it only inside its
    CPU legs (``cpu_baseline``, whose caller ``reference`` is the CPU arm)."""
    import ast
    root = Path(__file__).resolve().parents[1]

    def oracle_imports(path):
        tree = ast.parse(path.read_text())
        found = []

        def visit(node, func):
            for child in ast.iter_child_nodes(node):
                f = child.name if isinstance(child, (ast.FunctionDef, ast.AsyncFunctionDef)) else func
                mods = []
                if isinstance(child, ast.Import):
                    mods = [a.name for a in child.names]
                elif isinstance(child, ast.ImportFrom):
                    mods = [child.module or ""]
                if any(m == "oracle" or m.startswith("oracle.") for m in mods):
                    found.append(f)
                visit(child, f)

        visit(tree, None)
        return found

    for src in sorted((root / "gpe_simulator_b200").rglob("*.py")):
        assert oracle_imports(src) == [], src
    assert set(oracle_imports(root / "bench.py")) <= {"cpu_baseline"}


def test_missing_library_and_missing_gpu_fail_loudly(tmp_path, monkeypatch):
    """No CPU fallback: without the built library the loader raises, and a plan
    refuses to exist without a CUDA device (this container has none)."""
    import torch
    from gpe_simulator_b200 import _lib
    from gpe_simulator_b200.plan import Plan
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "libgpe_ssf.so")
    with pytest.raises(RuntimeError, match="not built"):
        _lib.load()
    if not torch.cuda.is_available():
        x = np.linspace(-4, 4, 16, endpoint=False)
        with pytest.raises(RuntimeError, match="CUDA device"):
            Plan(16, x, 2 * np.pi * np.fft.fftfreq(16, 0.5), dtype=torch.complex64, kind="imaginary",
                 beta=1.0, dt=1e-3)
