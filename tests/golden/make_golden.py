"""Regenerates the golden fixtures of tests/golden from the reference's own data files.

Reads (only when the mumax/2 tree is available; its root is the first argument or $REF_ROOT):
  tests/stdsolution4.txt   muMAG standard problem 4, <m>(t) with t in ns
and writes subsampled copies next to this script.  Run: python tests/golden/make_golden.py [REF_ROOT]
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref_root):
    src = os.path.join(ref_root, "tests", "stdsolution4.txt")
    a = np.loadtxt(src)
    sub = a[::8]
    if sub[-1, 0] != a[-1, 0]:
        sub = np.vstack([sub, a[-1]])
    hdr = ("muMAG standard problem 4 golden <m>(t) of the reference (tests/stdsolution4.txt),\n"
           "every 8th row.  columns: t (ns), <mx>, <my>, <mz> (user axes)")
    np.savetxt(os.path.join(HERE, "sp4_stdsolution4.txt"), sub, fmt="%.7g", header=hdr)
    print("wrote", len(sub), "rows")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("REF_ROOT")
    if not root:
        sys.exit("usage: make_golden.py REF_ROOT (or set REF_ROOT)")
    main(root)
