"""Regenerate tests/golden/qs_tables.json from the reference's QS coefficient tables.

The reference keeps the coefficients of symmetry QS as C++ fragments under
``c++/symmetry/coefnew/qs/`` (``qs-{1,2}ch-{offdiag,diag,spinup*,spindown*,doublet*,triplet*}.dat``):
each row names its combinations and a closed-form factor in the spin S of a subspace; the
two-channel global charge tables (``qs-2ch-{q1,q2,qdiff,qtot}.dat``) hold integers. This
script evaluates every row's factor for SS = 1..11 (S = 0..5) in IEEE double arithmetic, as
the C++ evaluates it (so 1/0 is inf and sqrt of a negative number is nan), and writes the
values in file order. The test tests/test_qs_tables.py compares nrgljubljana_b200/qs.py
against them. Usage:

    python tests/golden/make_qs_tables.py /path/to/nrgljubljana
"""
import json
import os
import re
import sys

import numpy as np

SS = list(range(1, 12))
FILES = ["offdiag", "diag", "spinupa", "spindowna", "spinupb", "spindownb", "doubletp", "doubletm",
         "triplets", "tripletp", "tripletm", "q1", "q2", "qdiff", "qtot"]
GLOBAL = ("q1", "q2", "qdiff", "qtot")


def value(expr: str, s: float) -> float:
    e = re.sub(r"S\(ss[1p]?\)", "s", expr)
    e = e.replace("Power(", "pw(")
    with np.errstate(all="ignore"):
        return float(eval(e, {"s": np.float64(s), "sqrt": np.sqrt, "pw": lambda a, b: np.float64(a) ** b}))


def split_args(body: str):
    """Top-level comma split of a C++ argument list."""
    out, depth, cur = [], 0, ""
    for ch in body:
        if ch == "(":
            depth += 1
        elif ch == ")":
            depth -= 1
        if ch == "," and depth == 0:
            out.append(cur.strip())
            cur = ""
        else:
            cur += ch
    out.append(cur.strip())
    return out


def rows_of(path: str, kind: str):
    rows = []
    for line in open(path):
        line = line.strip()
        if not line:
            continue
        if kind in ("offdiag", "diag") + GLOBAL:
            body = line[line.index("(") + 1:line.rindex(")")]
        else:
            body = line.rstrip(",")[1:-1]
        args = split_args(body)
        if kind == "offdiag":      # OFFDIAG(i, j, ch, factor(S(ss)))
            rows.append([int(args[0]), int(args[1]), int(args[2]), [value(args[3], (ss - 1) / 2) for ss in SS]])
        elif kind in GLOBAL:       # Q1(i1, ip, ch, value) and the like: integer values
            rows.append([int(args[0]), int(args[1]), int(args[2]), int(args[3])])
        elif kind == "diag":       # DIAG(i, ch, number)
            rows.append([int(args[0]), int(args[1]), float(args[2])])
        elif kind.startswith("spin"):   # { i1, ip, factor(S(ssp)) }
            rows.append([int(args[0]), int(args[1]), [value(args[2], (ss - 1) / 2) for ss in SS]])
        else:                      # { i1, ip, Invar(..), Invar(..), factor(S(ss1)) }
            rows.append([int(args[0]), int(args[1]), [value(args[4], (ss - 1) / 2) for ss in SS]])
    return rows


def main(ref_root: str) -> None:
    d = os.path.join(ref_root, "c++", "symmetry", "coefnew", "qs")
    out = {"ss": SS}
    for ch in (1, 2):
        for kind in FILES:
            path = os.path.join(d, f"qs-{ch}ch-{kind}.dat")
            if os.path.exists(path):
                out[f"{ch}ch-{kind}"] = rows_of(path, kind)
    dst = os.path.join(os.path.dirname(os.path.abspath(__file__)), "qs_tables.json")
    with open(dst, "w") as f:
        json.dump(out, f)
    print(f"wrote {len(out) - 1} tables to {dst}")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NRG_REFERENCE")
    if not ref:
        sys.exit(f"usage: {sys.argv[0]} REFERENCE_DIR (or set NRG_REFERENCE): the NRG Ljubljana source tree")
    main(ref)
