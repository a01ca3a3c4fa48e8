"""Regenerate the golden fixtures of tests/golden/ from the reference's example data.

Reads (never at test time) the reference's own known-answer files and writes small text
fixtures next to this script:
  sod_exact.txt  <- example/sodShockTube/exact.dat (exact Sod solution at t = 0.2:
                    x, u, rho, p on 2000 points; every 4th point is kept)
Usage: python tests/golden/make_golden.py [/path/to/reference]  (default: oracle/ref_build.py's
reference_dir())
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_tecplot_columns(path, ncol):
    vals = []
    with open(path) as f:
        for line in f:
            s = line.strip()
            if not s or s.lower().startswith("variables"):
                continue
            vals.extend(float(t) for t in s.split())
    a = np.array(vals)
    return a.reshape(-1, ncol)


def main(ref):
    sod = read_tecplot_columns(os.path.join(ref, "example", "sodShockTube", "exact.dat"), 4)
    sub = sod[::4]
    np.savetxt(os.path.join(HERE, "sod_exact.txt"), sub, fmt="%.15e",
               header="exact Sod solution at t=0.2 from example/sodShockTube/exact.dat (every 4th point)\n"
                      "columns: x u rho p")


if __name__ == "__main__":
    sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
    import ref_build
    ref = ref_build.reference_dir(sys.argv[1] if len(sys.argv) > 1 else None)
    if ref is None:
        sys.exit("reference sources not found: pass the path or set COREFL_REFERENCE")
    main(ref)
