"""Writes csrc/hg_breakpoints.h: the 255 iSAX breakpoints of cardinality 256.

Breakpoint s (0-based) is the standard normal quantile Phi^-1((s+1)/256),
evaluated in double precision (scipy.special.ndtri) and rounded to float32,
which is how the reference's generated table (include/sax_breakpoints.h,
offset (c-1)(c-2)/2 = 32385 for c = 256) is stored.  Run once; the header
is committed.
"""
import os

import numpy as np
import scipy.special as sp

HERE = os.path.dirname(os.path.abspath(__file__))


def breakpoints():
    return np.array([sp.ndtri((s + 1) / 256.0) for s in range(255)], dtype=np.float64).astype(np.float32)


def main():
    bp = breakpoints()
    lines = ["// Generated by hercules_b200/gen_breakpoints.py: Phi^-1((s+1)/256), s = 0..254,",
             "// double precision rounded to float32.  Do not edit.",
             "#pragma once", "", "static const float kHgBreakpoints[255] = {"]
    for i in range(0, 255, 4):
        lines.append("    " + " ".join("%.9ef," % v for v in bp[i:i + 4]))
    lines += ["};", ""]
    with open(os.path.join(HERE, "csrc", "hg_breakpoints.h"), "w") as f:
        f.write("\n".join(lines))


if __name__ == "__main__":
    main()
