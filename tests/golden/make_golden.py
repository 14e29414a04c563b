"""Generate the golden fixtures in tests/golden/*.npz from the reference's own CPU build.

Run in a container that holds the reference sources (oracle/Makefile builds ``oracle/_ref`` from
them); the GPU box never runs this.  Each fixture stores the result of one case in
``tests/golden/cases.py`` as computed by the reference ``oscars.sr`` (gpu=0, nthreads=1), plus the
per-entry stop levels from a second ``quantity='level'`` call where the case returns values.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py flux_und_41
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import CASES, run_case  # noqa: E402


def reference():
    subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref"])
    from oracle.oracle import reference_module
    return reference_module()


def exact_sums(a):
    """Correctly rounded row sums (independent of memory layout and summation order)."""
    import math
    return np.array([math.fsum(row) for row in np.asarray(a)])


def flatten(result):
    """Return (positions, values) arrays for any of the API's list results."""
    if isinstance(result[0][0], list):            # [[x, y, z], value]
        pos = np.array([r[0] for r in result], dtype=np.float64)
        val = np.array([r[1] for r in result], dtype=np.float64)
    else:                                          # [energy, value]
        pos = np.array([r[0] for r in result], dtype=np.float64)
        val = np.array([r[1] for r in result], dtype=np.float64)
    return pos, val


def make(name, S):
    calls = CASES[name]
    obj = S.sr(nthreads=1, gpu=0)
    last, kw = calls[-1]
    if last == "calculate_trajectory":
        res = run_case(obj, calls)
        a = np.array([[p[0]] + p[1] + p[2] + p[3] for p in res], dtype=np.float64).T
        idx = np.arange(0, a.shape[1], 100)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), n=a.shape[1], idx=idx, sub=a[:, idx],
                            sums=exact_sums(a), abssums=exact_sums(np.abs(a)))
        return
    kw = dict(kw)
    if last != "calculate_trajectory":
        kw.setdefault("nthreads", 1)
    res = run_case(obj, calls[:-1] + [(last, kw)])
    pos, val = flatten(res)
    extra = {}
    if kw.get("quantity", "flux") in ("flux", "power density"):
        obj2 = S.sr(nthreads=1, gpu=0)
        kw2 = dict(kw)
        kw2["quantity"] = "level"
        _, lev = flatten(run_case(obj2, calls[:-1] + [(last, kw2)]))
        extra["level"] = lev
    np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=pos, val=val, **extra)


def main(argv):
    S = reference()
    names = argv[1:] or sorted(CASES)
    for n in names:
        make(n, S)
        print("wrote", n)


if __name__ == "__main__":
    main(sys.argv)
