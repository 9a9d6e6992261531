"""Generate tests/golden/estimate_k.json from the reference itself.

Runs the reference's estimate_K and crt_overflowed
(python/euler2ai_full_verify.py:40-93, 152-167) on fixed inputs.  Needs the
reference checkout (read-only) and sympy/mpmath; run from the repo root:

    python tests/golden/make_estimate_k.py /path/to/reference
"""

import importlib.util
import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_estimate_k.py <reference checkout>")
ref = sys.argv[1]
sys.path.insert(0, os.path.join(ref, "python"))
spec = importlib.util.spec_from_file_location(
    "euler2ai_full_verify", os.path.join(ref, "python", "euler2ai_full_verify.py"))
mod = importlib.util.module_from_spec(spec)
spec.loader.exec_module(mod)

k_cases = [("2", "n**2", 2000), ("3*n+1", "-2*n**2+5", 500), ("n", "1/n", 100), ("5", "7", 0),
           ("n**2+n+1", "-n**4", 8000), ("-9*n**2", "10*n**4-3", 1), ("1", "n**3", 50000),
           ("2*n+1", "n**2", 12345), ("not an expr", "n", 300)]
o_cases = [(355, 113, 3.14159292), (355, 113, 3.2), (0, 5, 0.0), (7, 0, 1.0), (10 ** 400, 1, 1e300),
           (-3, 4, -0.75), (-3, 4, 0.75), (1, 10 ** 12, 1e-12), (1, 10 ** 12, 0.02),
           (2 ** 2000 + 1, 2 ** 1999, 2.0), (5, 7, float("nan"))]
out = {"estimate_K": [[a, b, d, mod.estimate_K(a, b, d)] for a, b, d in k_cases],
       "crt_overflowed": [[str(p), str(q), repr(e), mod.crt_overflowed(p, q, e)] for p, q, e in o_cases]}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "estimate_k.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1)
print("wrote", path)
