"""Generate tests/golden/constants.json from the reference's constants module.

Records the registry (names, expressions), compute_match_digits and
compute_delta_against_constant (python/dreams_rns/constants.py:21-207) on
fixed inputs.  Run from the repo root with the reference checkout:

    python tests/golden/make_constants.py /path/to/reference
"""

import json
import os
import sys

if len(sys.argv) != 2:
    sys.exit("usage: python tests/golden/make_constants.py <reference checkout>")
ref = sys.argv[1]
sys.path.insert(0, os.path.join(ref, "python"))
from dreams_rns import constants as C  # noqa: E402  (the reference package)

consts = C.load_constants(200)
estimates = [3.141592653589793, 1.2020569031595942, 1.0000009536743164, 1.000001, 0.6931471805599453,
             2.5, 1.6449340668482264, 0.0, -1.0, 1.0, 1e-12, 1.2]
match = [[e, *C.compute_match_digits(e, consts)] for e in estimates]
near = [[e, [m["name"] for m in C.match_against_constants(e, consts, 1e-2)]] for e in estimates]
pairs = [(355, 113, "pi"), (103993, 33102, "pi"), (0, 7, "pi"), (5, 0, "e"), (1, 1, "e"),
         (6, 5, "zeta3"), (-7, 5, "ln2"), (1393, 985, "sqrt2"), (10 ** 40 + 1, 10 ** 40, "zeta30")]
by = {c["name"]: c for c in consts}
deltas = [[str(p), str(q), n, C.compute_delta_against_constant(p, q, by[n]["value"], 200)]
          for p, q, n in pairs]
out = {"registry": [[e["name"], e["sympy_expr"]] for e in C.CONSTANTS_REGISTRY],
       "match_digits": match, "near": near, "delta_against": deltas}
path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "constants.json")
with open(path, "w") as f:
    json.dump(out, f, indent=1)
print("wrote", path)
