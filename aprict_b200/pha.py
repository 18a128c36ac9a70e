"""FORBILD phantom files (``.pha``): reader and writer.

The reference reads these files with a C preprocessor and regular
expressions (src/aprict/lib/process_pha_file.py:89-388) into FORBILD_Shape
records (src/aprict/data/cusrc/FORBILD_volumes.h:1395-1415). This module is an
independent reader of the same format into the same 156-byte records:

* preprocessing: ``//`` and ``/* */`` comments, ``#include "file"`` (relative
  to the including file), ``#define NAME value`` and function-like
  ``#define F(a, b) body`` macros, expanded until stable;
* the German keywords ``achse`` (axis) and ``dichte`` (rho), ``mm`` units
  after numbers, ``Detector{...}`` blocks (dropped);
* one object per ``{ ... }``: ``[ShapeName: key=expr ... vec(x,y,z) ...
  clip ...]`` plus ``key=expr`` properties after the brackets (``formel`` /
  ``formula`` ignored); vectors ``axis``, ``a_x``, ``a_y``, ``a_z``; clip
  planes ``x<e``, ``y>e``, ``z<e``, ``r(a,b,c)>e`` (axis normalised; ``<`` is
  mode 1, ``>`` mode 2; at most three);
* expressions: numbers, ``+ - * /``, parentheses and ``sin cos tan`` of
  degrees, ``sqrt``, ``pi``;
* a missing third axis of an Ellipsoid_free (a_x, a_y, a_z) or Ellipt_Cyl
  (a_x, a_y, axis) is the cross product of the other two (right-handed; both
  solids are symmetric, so the sign does not matter).

:func:`format_shapes` writes records back in the same syntax.
"""

from __future__ import annotations

import ast
import math
import operator
import pathlib
import re

import numpy as np

from . import _structs as S

SHAPE_TYPES = {
    "Box": 1, "Cone": 2, "Cone_x": 3, "Cone_y": 4, "Cone_z": 5, "Cylinder": 6, "Cylinder_x": 7,
    "Cylinder_y": 8, "Cylinder_z": 9, "Ellipsoid": 10, "Ellipsoid_free": 11, "Ellipt_Cyl": 12, "Sphere": 13,
    "Ellipt_Cyl_x": 14, "Ellipt_Cyl_y": 15, "Ellipt_Cyl_z": 16,
}
TYPE_NAMES = {v: k for k, v in SHAPE_TYPES.items()}
SCALARS = ("x", "y", "z", "dx", "dy", "dz", "r", "r1", "r2", "l", "rho")
VECTORS = ("axis", "a_x", "a_y", "a_z")


# ----------------------------------------------------------------- expressions
_BIN = {ast.Add: operator.add, ast.Sub: operator.sub, ast.Mult: operator.mul, ast.Div: operator.truediv,
        ast.Pow: operator.pow}
_FUN = {
    "sin": lambda d: math.sin(math.radians(d)), "cos": lambda d: math.cos(math.radians(d)),
    "tan": lambda d: math.tan(math.radians(d)), "sqrt": math.sqrt, "abs": abs,
}


def evaluate(expr: str) -> float:
    """Value of an arithmetic expression of the .pha format (angles in degrees)."""
    try:
        return float(expr)
    except ValueError:
        pass

    def ev(n: ast.AST) -> float:
        if isinstance(n, ast.Expression):
            return ev(n.body)
        if isinstance(n, ast.Constant) and isinstance(n.value, (int, float)):
            return float(n.value)
        if isinstance(n, ast.BinOp) and type(n.op) in _BIN:
            return _BIN[type(n.op)](ev(n.left), ev(n.right))
        if isinstance(n, ast.UnaryOp) and isinstance(n.op, (ast.USub, ast.UAdd)):
            v = ev(n.operand)
            return -v if isinstance(n.op, ast.USub) else v
        if isinstance(n, ast.Call) and isinstance(n.func, ast.Name) and n.func.id in _FUN and len(n.args) == 1:
            return float(_FUN[n.func.id](ev(n.args[0])))
        if isinstance(n, ast.Name) and n.id == "pi":
            return math.pi
        msg = f"unsupported expression in a phantom file: {expr!r}"
        raise ValueError(msg)

    return ev(ast.parse(expr.strip(), mode="eval"))


# ---------------------------------------------------------------- preprocessor
_COMMENTS = re.compile(r"//[^\n]*|/\*.*?\*/", re.S)


def _macros_expand(text: str, macros: dict) -> str:
    ident = re.compile(r"\b([A-Za-z_]\w*)\b")
    for _ in range(64):
        changed = False
        out, pos = [], 0
        for m in ident.finditer(text):
            name = m.group(1)
            if name not in macros or m.start() < pos:
                continue
            params, body = macros[name]
            if params is None:
                out.append(text[pos:m.start()])
                out.append(body)
                pos = m.end()
                changed = True
                continue
            j = m.end()
            while j < len(text) and text[j] in " \t":
                j += 1
            if j >= len(text) or text[j] != "(":
                continue
            depth, k, args, start = 0, j, [], j + 1
            while k < len(text):
                c = text[k]
                if c == "(":
                    depth += 1
                elif c == ")":
                    depth -= 1
                    if depth == 0:
                        args.append(text[start:k])
                        break
                elif c == "," and depth == 1:
                    args.append(text[start:k])
                    start = k + 1
                k += 1
            else:
                msg = f"unbalanced macro call {name}("
                raise ValueError(msg)
            if len(args) == 1 and not args[0].strip() and not params:
                args = []
            if len(args) != len(params):
                msg = f"macro {name} takes {len(params)} arguments, got {len(args)}"
                raise ValueError(msg)
            rep = body
            for p, a in zip(params, args, strict=True):
                rep = re.sub(rf"\b{re.escape(p)}\b", a.strip(), rep)
            out.append(text[pos:m.start()])
            out.append(rep)
            pos = k + 1
            changed = True
        out.append(text[pos:])
        text = "".join(out)
        if not changed:
            return text
    msg = "macro expansion does not terminate"
    raise ValueError(msg)


def preprocess(text: str, *, base_dir: pathlib.Path | None = None, macros: dict | None = None) -> str:
    """Comments, #include and #define handled; macros expanded."""
    macros = {} if macros is None else macros
    text = _COMMENTS.sub(" ", text.replace("\\\n", " "))
    out = []
    define = re.compile(r"#\s*define\s+([A-Za-z_]\w*)(\(([^)]*)\))?\s*(.*)$")
    include = re.compile(r'#\s*include\s+["<]([^">]+)[">]')
    for line in text.splitlines():
        s = line.strip()
        if s.startswith("#"):
            if m := include.match(s):
                if base_dir is None:
                    msg = "#include needs the including file's directory"
                    raise ValueError(msg)
                inc = base_dir / m.group(1)
                out.append(preprocess(inc.read_text(encoding="ISO-8859-1"), base_dir=inc.parent, macros=macros))
            elif m := define.match(s):
                params = None if m.group(2) is None else [p.strip() for p in m.group(3).split(",") if p.strip()]
                macros[m.group(1)] = (params, m.group(4).strip())
            continue  # other directives (#undef, #if ...) are not used by the phantom files
        out.append(line)
    return _macros_expand("\n".join(out), macros)


# -------------------------------------------------------------------- objects
_NUM_MM = re.compile(r"(?<=[0-9.])mm\b")
_VEC = re.compile(r"\b(axis|a_x|a_y|a_z)\s*\(")
_KEYVAL = re.compile(r"\b([A-Za-z_]\w*)\s*=\s*")


def _split_top(s: str, seps: str = " \t\n") -> list[str]:
    """Whitespace-separated tokens, keeping parenthesised parts together."""
    toks, depth, cur = [], 0, []
    for c in s:
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        if c in seps and depth == 0:
            if cur:
                toks.append("".join(cur))
                cur = []
        else:
            cur.append(c)
    if cur:
        toks.append("".join(cur))
    return toks


def _paren_args(s: str) -> list[str]:
    """'(a, b, c)' -> ['a', 'b', 'c'] (top-level commas)."""
    s = s.strip()
    if not (s.startswith("(") and s.endswith(")")):
        msg = f"expected a parenthesised triple, got {s!r}"
        raise ValueError(msg)
    inner, depth, cur, out = s[1:-1], 0, [], []
    for c in inner:
        if c == "(":
            depth += 1
        elif c == ")":
            depth -= 1
        if c == "," and depth == 0:
            out.append("".join(cur))
            cur = []
        else:
            cur.append(c)
    out.append("".join(cur))
    return out


def _normalise_tokens(body: str) -> list[str]:
    # join "key = value" and "name (x,y,z)" into single tokens
    body = re.sub(r"\s*=\s*", "=", body)
    body = re.sub(r"\b(axis|a_x|a_y|a_z|r)\s+\(", r"\1(", body)
    body = re.sub(r"\s*([<>])\s*", r"\1", body)
    body = re.sub(r"-\s+(?=[0-9.(])", "-", body)
    return _split_top(body)


def _cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.cross(a.astype(np.float64), b.astype(np.float64))


def parse_object(obj: str) -> np.ndarray:
    """One ``{ ... }`` object -> a forbild_shape record."""
    m = re.search(r"\[(.*)\]", obj, re.S)
    if m is None:
        msg = f"no [Shape: ...] in object {obj[:60]!r}"
        raise ValueError(msg)
    inside, outside = m.group(1), obj[: m.start()] + " " + obj[m.end():]
    head, _, rest = inside.partition(":")
    name = head.strip()
    if name not in SHAPE_TYPES:
        msg = f"unknown FORBILD shape {name!r}"
        raise ValueError(msg)
    rec = np.zeros((), S.forbild_shape)
    rec["type"] = SHAPE_TYPES[name]
    vecs: dict[str, np.ndarray] = {}
    clips: list[tuple[np.ndarray, float, int]] = []
    for tok in _normalise_tokens(rest) + [("@" + t) for t in _normalise_tokens(outside)]:
        from_outside = tok.startswith("@")
        tok = tok.lstrip("@")
        if not tok or tok.startswith('"'):
            continue
        if "=" in tok and not re.match(r"^[^=]*[<>]", tok):
            k, v = tok.split("=", 1)
            if k in ("formel", "formula"):
                continue
            if k not in SCALARS:
                msg = f"unknown property {k!r} in {name}"
                raise ValueError(msg)
            rec[k] = evaluate(v)
            continue
        if from_outside:
            continue  # labels and other free text outside the brackets
        vm = re.match(r"^(axis|a_x|a_y|a_z)(\(.*\))$", tok)
        if vm:
            vecs[vm.group(1)] = np.array([evaluate(e) for e in _paren_args(vm.group(2))])
            continue
        cm = re.match(r"^(x|y|z|r\(.*\))([<>])(.+)$", tok)
        if cm:
            lhs, sign, rhs = cm.groups()
            if lhs in ("x", "y", "z"):
                ax = np.eye(3)["xyz".index(lhs)]
            else:
                ax = np.array([evaluate(e) for e in _paren_args(lhs[1:])])
                ax = ax / np.linalg.norm(ax)
            clips.append((ax, evaluate(rhs), 1 if sign == "<" else 2))
            continue
        msg = f"cannot read {tok!r} in {name}"
        raise ValueError(msg)
    if name == "Ellipsoid_free":
        trio = ("a_x", "a_y", "a_z")
    elif name == "Ellipt_Cyl":
        trio = ("a_x", "a_y", "axis")
    else:
        trio = ()
    if trio:
        missing = [k for k in trio if k not in vecs]
        if len(missing) == 1:
            i = trio.index(missing[0])
            vecs[missing[0]] = _cross(vecs[trio[(i + 1) % 3]], vecs[trio[(i + 2) % 3]])
    for k, v in vecs.items():
        rec[k] = tuple(float(c) for c in v)
    if len(clips) > 3:
        msg = "Too many clip planes encountered."
        raise ValueError(msg)
    for i, (ax, d, mode) in enumerate(clips):
        c = rec[f"cas{i + 1}"]
        c["axis"] = tuple(float(a) for a in ax)
        c["dotprod"] = d
        c["mode"] = mode
    return rec


def parse_text(text: str, *, base_dir: pathlib.Path | None = None) -> np.ndarray:
    """All shapes of a phantom description, in file order."""
    s = preprocess(text, base_dir=base_dir)
    s = re.sub(r"\bachse\b", "axis", s)
    s = re.sub(r"\bdichte\b", "rho", s)
    s = _NUM_MM.sub("", s)
    s = re.sub(r"Detector\s*\{[^{}]*\}", " ", s)
    objs = re.findall(r"\{[^{}]*\}", s)
    out = np.zeros(len(objs), S.forbild_shape)
    for i, o in enumerate(objs):
        out[i] = parse_object(o[1:-1])
    return out


def load(path: str | pathlib.Path) -> np.ndarray:
    """Shapes of a ``.pha`` file (``#include`` resolved next to it)."""
    p = pathlib.Path(path)
    return parse_text(p.read_text(encoding="ISO-8859-1"), base_dir=p.parent)


def _fmt(v: float) -> str:
    return repr(float(np.float32(v)))


def format_shape(rec: np.ndarray) -> str:
    """One record in .pha syntax (read back by :func:`parse_text`)."""
    name = TYPE_NAMES[int(rec["type"])]
    parts = [f"{k}={_fmt(rec[k])}" for k in SCALARS if k != "rho" and float(rec[k]) != 0.0]
    for k in VECTORS:
        v = rec[k]
        if any(float(v[c]) != 0.0 for c in "xyz"):
            parts.append(f"{k}({_fmt(v['x'])},{_fmt(v['y'])},{_fmt(v['z'])})")
    for i in (1, 2, 3):
        c = rec[f"cas{i}"]
        if int(c["mode"]) == 0:
            continue
        a = c["axis"]
        parts.append(f"r({_fmt(a['x'])},{_fmt(a['y'])},{_fmt(a['z'])}){'<' if int(c['mode']) == 1 else '>'}{_fmt(c['dotprod'])}")
    return "{ [" + name + ": " + " ".join(parts) + "] rho=" + _fmt(rec["rho"]) + " }"


def format_shapes(shapes: np.ndarray) -> str:
    """A phantom description with one object per line."""
    return "\n".join(format_shape(s) for s in shapes)


__all__ = ["SHAPE_TYPES", "evaluate", "format_shapes", "load", "parse_text", "preprocess"]
