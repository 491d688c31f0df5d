"""Golden decisions of the REFERENCE fixed group-by planner.

Run where the reference checkout is readable:

    python tests/golden/make_plan_golden.py /path/to/numfast-reference

For a grid of probe observables (n, sortedness, key range, aggregate count) it calls the
reference's own Planner.plan_groupby exactly as the executor's dense gate does
(src/Drivers/CPU/_lib/cpu.py:381-421: span, dense_estimate_bytes, bycode_estimate_bytes,
budget from the CPU capability) and writes plan_fixed.json next to this file.  Tests
compare nfc_plan_fixed against these decisions; the reference is not needed at test time.
"""

import json
import os
import sys


def main(ref_root):
    os.environ["NUMFAST_NATIVE_DISABLE"] = "1"
    os.environ["PYTHONDONTWRITEBYTECODE"] = "1"
    sys.path.insert(0, os.path.join(ref_root, "src"))
    import numfast as nf

    plan_groupby = nf.get_kernel(fresh=True).alias["plan_groupby"]

    # groupindex.py:72-83 (the executor imports these as _dense_est / _bycode_est).
    def dense_estimate_bytes(r, n):
        return 16 * int(r) + 8 * int(n)

    def bycode_estimate_bytes(m, n, keys_is_int64):
        return 16 * int(m) + (0 if keys_is_int64 else 8 * int(n))

    cases = []
    ns = [1, 7, 1000, 100_000, 1_000_000, 10_000_000, 50_000_000, 100_000_000]
    spans = [1, 10, 1000, 65_536, 1_000_000, 4_000_000, 10_000_000, 40_000_000, 63_999_999, 64_000_001,
             200_000_000, 2 ** 32]
    kmins = [0, 5, 1_000_000, -1, -2 ** 31]
    for n in ns:
        for r in spans:
            for kmin in kmins:
                if kmin + r - 1 > 2 ** 31 - 1:
                    continue
                for naggs in (1, 2, 6):
                    for is_sorted in ((False, True) if naggs == 1 and kmin == 0 else (False,)):
                        est = dense_estimate_bytes(r, n)
                        m_code = kmin + r if kmin >= 0 else None
                        est_code = bycode_estimate_bytes(m_code, n, False) if m_code is not None else None
                        dec = plan_groupby(n, is_sorted, span=r, est_dense_bytes=est, budget_bytes=None,
                                                   kmin=kmin, est_code_bytes=est_code, naggs=naggs)
                        cases.append({"n": n, "span": r, "kmin": kmin, "naggs": naggs, "sorted": is_sorted,
                                      "strategy": dec["strategy"]})
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "plan_fixed.json")
    fields = ["n", "span", "kmin", "naggs", "sorted", "strategy"]
    with open(out, "w") as f:
        json.dump({"source": "Planner.plan_groupby (src/Runtime/Planner/Planner.py:54-65 -> "
                             "_lib/planner.py:200-262)", "fields": fields,
                   "cases": [[c[k] for k in fields] for c in cases]}, f, separators=(",", ":"))
    print("wrote %d cases to %s" % (len(cases), out))


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NUMFAST_REFERENCE")
    if not root:
        sys.exit("usage: %s <reference checkout> (or set NUMFAST_REFERENCE)" % sys.argv[0])
    main(root)
