"""Generate tests/golden/golden.json from the reference itself.

For every recipe in tests/cases.py this runs the reference's own msd_CE6
(rantala/string-sorting src/msd_ce.cpp:367-419), compiled from its sources
into oracle/_ref/libref.so by oracle/Makefile, and records the permutation it
produces (in full for small cases, as a SHA-256 digest otherwise) together with
the LCP array of that order by the reference's lcp() definition
(src/mergesort_lcp.cpp:88-100).  msd_CE2 is run as a cross-check and must agree.

Usage (needs the reference sources and `make -C oracle ref`):
    python tests/golden/make_golden.py
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import cases  # noqa: E402
import pyoracle  # noqa: E402


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def main():
    out = {}
    for name, build in cases.CASES.items():
        strings = build()
        arena, offs = cases.arena_of(strings)
        n = len(strings)
        if n:
            p6 = pyoracle.ref_sort_perm("msd_CE6", arena, offs)
            p2 = pyoracle.ref_sort_perm("msd_CE2", arena, offs)
            if not np.array_equal(p6, p2):
                raise SystemExit(f"{name}: msd_CE6 and msd_CE2 disagree")
        else:
            p6 = np.zeros(0, dtype=np.uint32)
        lcp = cases.lcp_of(strings, p6)
        rec = {"n": n, "routine": "msd_CE6", "perm_sha256": digest(p6), "lcp_sha256": digest(lcp)}
        if n <= 64:
            rec["perm"] = [int(x) for x in p6]
            rec["lcp"] = [int(x) for x in lcp]
        out[name] = rec
        print(f"{name:28s} n={n}")
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main()
