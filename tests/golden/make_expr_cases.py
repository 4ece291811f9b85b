"""Golden renderings of potential expressions by the reference itself.

Runs ONLY where the reference sources are present (the location the oracle
recipe uses, ``oracle/ref_shim.py``).  For each formula of the corpus below the
reference's ``gpe/expressions.py:9-30`` ``cuda_expression`` (with its validator,
``config_editor/expressions.py:12-58``; both pure Python) gives the CUDA text, or
rejects the formula; ``expr_cases.json`` stores the source, the time flag and
that text (``null`` when rejected).

Usage: ``python tests/golden/make_expr_cases.py``.
"""

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

CORPUS = [
    # potentials as stages write them
    ("x**2+1.44*y**2+2.25*z**2", False), ("0.5*(x*x + y*y) + 2.25*z**2/2", False),
    ("x/2 + y**2/10 + abs(z)/5", False), ("0.002*(x*x + y*y + z*z)", False),
    ("-(x-1)**2 + 3*sin(y)*cos(z) - exp(-x*x)", False), ("sqrt(x*x+y*y) - tanh(z) + log(2+x)", False),
    ("1/2", False), ("pi*x", False), ("0", False), ("-0", False), ("10*exp(-((x-2)**2+y**2)/0.25)", False),
    ("20.0*exp(-((x-2.0*cos((1.0*(((t+0.025-abs(t-0.025))/2)**2/(2*0.025)+t-((t+0.025-abs(t-0.025))/2)))))**2"
     "+(y-2.0*sin((1.0*(((t+0.025-abs(t-0.025))/2)**2/(2*0.025)+t-((t+0.025-abs(t-0.025))/2)))))**2)/0.5**2)", True),
    ("0.3*sin(5*t)*x", True), ("abs(-x) + cos(t)", True), ("(1+0.1*sin(2*t))*(x**2+y**2+z**2)", True),
    # precedence, signs and literals
    ("-x**2", False), ("2**-1", False), ("2**3**2", False), ("--x", False), ("+-+x", False), ("x*-y", False),
    ("(-x)**2", False), ("x**-y**2", False), ("-2**2", False), ("1/2/3", False), ("1-2-3", False),
    ("1.e5+.5+5.+1_000", False), ("05.5 + 00", False), ("1e-3*x", False), ("2.50E+2", False),
    ("  x  +  y  ", False), ("((((x))))", False), ("tan(x)*tanh(y)", False), ("exp(log(z+3))", False),
    # rejected by both
    ("t*y", False), ("x; return 0", False), ("", False), ("   ", False), ("2x", False), ("007", False),
    ("sin", False), ("foo(x)", False), ("sin(x, y)", False), ("1e999", False), ("x <= y", False),
    ("True", False), ("x @ y", False), ("x % 2", False), ("1j", False), ("x^2", False), ("np.sin(x)", False),
    ("x // 2", False), ("lambda: 0", False), ("x if y else z", False), ("[x]", False), ("sin(x=1)", False),
]


def main():
    from oracle import ref_shim
    if not ref_shim.available():
        raise SystemExit(ref_shim.UNSET if ref_shim.REFERENCE is None else "the reference sources are not present")
    sys.path.insert(0, str(ref_shim.REFERENCE))
    from gpe.expressions import cuda_expression   # pure Python in the reference
    rows = []
    for source, td in CORPUS:
        try:
            text = cuda_expression(source, time_dependent=td)
        except ValueError:
            text = None
        rows.append({"source": source, "time_dependent": td, "cuda": text})
    out = Path(__file__).with_name("expr_cases.json")
    out.write_text(json.dumps(rows, indent=1) + "\n")
    print(f"wrote {out} ({len(rows)} cases)")


if __name__ == "__main__":
    main()
