"""Extract the Ram-Lak known-answer vectors from the reference's own test.

Reads src/aprict/tests/ramp_kernels/test_ramp_kernels_precision.py (as text,
through the ast module -- nothing of the reference is imported or executed)
and writes ramlak_golden.json: the three (input, expected output) pairs of its
``Test_RampFilter`` parametrisation (:33-147). The expected outputs there are
high-precision values of the linear "same"-mode convolution of the input with
the Ram-Lak taps of a window 2*len+1, physpixsize 1 (:162-175).

Usage: python tests/golden/make_ramp_golden.py REFERENCE_ROOT
(or set APRICT_REF_DIR to the reference checkout).
"""

from __future__ import annotations

import ast
import json
import pathlib
import sys

import os

_ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("APRICT_REF_DIR")
if not _ref:
    sys.exit("usage: make_ramp_golden.py REFERENCE_ROOT (or set APRICT_REF_DIR)")
REF = pathlib.Path(_ref)
SRC = REF / "src/aprict/tests/ramp_kernels/test_ramp_kernels_precision.py"
OUT = pathlib.Path(__file__).resolve().parent / "ramlak_golden.json"


def _numbers(node: ast.AST) -> list[float]:
    """Flatten the literal numbers of an np.array(...) call, expanding `(x,) * n` products."""
    if isinstance(node, ast.Call):
        return _numbers(node.args[0])
    if isinstance(node, (ast.Tuple, ast.List)):
        out: list[float] = []
        for e in node.elts:
            out.extend(_numbers(e))
        return out
    if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Mult):
        return _numbers(node.left) * int(ast.literal_eval(node.right))
    if isinstance(node, ast.BinOp) and isinstance(node.op, ast.Add):
        return _numbers(node.left) + _numbers(node.right)
    return [float(ast.literal_eval(node))]


def main() -> None:
    tree = ast.parse(SRC.read_text())
    cases = []
    for node in ast.walk(tree):
        if isinstance(node, ast.Call) and getattr(node.func, "attr", "") == "parametrize":
            kw = {k.arg: k.value for k in node.keywords}
            if "argvalues" not in kw:
                continue
            ids = ast.literal_eval(kw["ids"]) if "ids" in kw else None
            for i, tup in enumerate(kw["argvalues"].elts):
                _factory, inp, expected = tup.elts
                # keep the literal text of the expected values (more digits than a float64 holds)
                exp_text = [ast.get_source_segment(SRC.read_text(), e) for e in expected.args[0].elts]
                cases.append(
                    {
                        "id": ids[i] if ids else str(i),
                        "input": _numbers(inp),
                        "input_dtype": "float32",
                        "expected": [float(t) for t in exp_text],
                        "expected_text": exp_text,
                    }
                )
    meta = {
        "source": "src/aprict/tests/ramp_kernels/test_ramp_kernels_precision.py:33-147",
        "window": "2*len(input)+1, physpixsize 1, ramp_kernel_ramlak (src/aprict/ramp_kernels.py:43-59)",
        "convolution": "scipy.signal.convolve(x, kern, mode='same')",
        "cases": cases,
    }
    OUT.write_text(json.dumps(meta, indent=1))
    print(f"wrote {OUT} ({len(cases)} cases)")


if __name__ == "__main__":
    main()
