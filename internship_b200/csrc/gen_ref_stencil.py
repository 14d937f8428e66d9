"""Writes mr_ref_stencil.inc: the 160 stencil directions of the reference's
core/vector.cu:77-172 (arrays Spn0..Spn4, SpVn5..SpVn7), as fp32 literals.

The reference network's weights (core/NNWeight.cuh) were trained on
descriptors gathered at these points, so a drop-in renderer must gather at
the same points; the table is data, kept identical for that reason.

usage: python gen_ref_stencil.py <reference checkout>
(or set MRPNN_REFERENCE). Only needed when the reference table changes; the
generated file is committed.
"""
import importlib.util
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def _lit(c):
    t = "%.9g" % np.float32(c)
    if "." not in t and "e" not in t:
        t += ".0"
    return t + "f"


def main():
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("MRPNN_REFERENCE")
    if not ref:
        sys.exit("usage: gen_ref_stencil.py <reference checkout> (or set MRPNN_REFERENCE)")
    spec = importlib.util.spec_from_file_location("_mr_weights", os.path.join(os.path.dirname(HERE), "weights.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    pts = mod.load_stencil_source(os.path.join(ref, "core", "vector.cu")).reshape(160, 3)
    lines = ["// Generated by gen_ref_stencil.py from the reference's core/vector.cu:77-172",
             "// (160 stencil directions: shells of 8, 8, 16, 16, 16 points on the unit",
             "// sphere, then three shells of 32 points in the unit ball). Do not edit.",
             "static const float kRefStencil[160 * 3] = {"]
    for p in pts:
        lines.append("    " + ", ".join(_lit(c) for c in p) + ",")
    lines.append("};")
    out = os.path.join(HERE, "mr_ref_stencil.inc")
    with open(out, "w") as f:
        f.write("\n".join(lines) + "\n")
    print(out)


if __name__ == "__main__":
    main()
