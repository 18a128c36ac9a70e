"""Regenerate tests/golden/forbild_head_shapes.npy: the FORBILD head phantom of
the reference checkout (src/aprict/data/FORBILD/head/HeadPhantom.pha, with its
#include "TableOfTissues"), read by aprict_b200.pha, as 156-byte FORBILD_Shape
records. The GPU tests use it where the reference checkout is absent.

Run from the repository root: python tests/golden/make_forbild_golden.py REFERENCE_ROOT
(or set APRICT_REF_DIR to the reference checkout).
"""

from __future__ import annotations

import os
import pathlib
import sys

import numpy as np

ROOT = pathlib.Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from aprict_b200 import pha  # noqa: E402

PHA = "src/aprict/data/FORBILD/head/HeadPhantom.pha"


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("APRICT_REF_DIR")
    if not ref:
        sys.exit("usage: make_forbild_golden.py REFERENCE_ROOT (or set APRICT_REF_DIR)")
    shapes = pha.load(pathlib.Path(ref) / PHA)
    np.save(pathlib.Path(__file__).with_name("forbild_head_shapes.npy"), shapes)
    print(len(shapes), "shapes")


if __name__ == "__main__":
    main()
