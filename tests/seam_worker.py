"""Runs the golden radiation cases through the reference's own `oscars.sr`, built with its GPU seam
served by liboscars_b200 (oscars_b200/seam/Makefile), with gpu=1.  Run as a separate process with
that build first on sys.path:

    python tests/seam_worker.py <seam build dir> <output .npz> <case> [<case> ...]

For each case it stores <case>/pos, <case>/val and, with --levels, <case>/level (quantity='level'),
plus the module's file, check_gpu() and the first GPU's description as reported through the seam.
"""
import os
import sys

import numpy as np


def main():
    build, out, names = sys.argv[1], sys.argv[2], sys.argv[3:]
    sys.path.insert(0, build)
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(here, "golden"))
    saved = os.dup(1)  # the reference prints a banner on import; keep stdout for the caller
    os.dup2(os.open(os.devnull, os.O_WRONLY), 1)
    try:
        import oscars.sr as S
    finally:
        os.dup2(saved, 1)
    from cases import CASES, run_case
    res = {"module": np.array(S.__file__), "ngpu": np.array(S.sr().check_gpu())}
    for name in names:
        calls = list(CASES[name])
        last, kw = calls[-1]
        r = run_case(S.sr(), calls[:-1] + [(last, dict(kw, gpu=1))])
        res[name + "/pos"] = np.array([p[0] for p in r], dtype=np.float64)
        res[name + "/val"] = np.array([p[1] for p in r], dtype=np.float64)
        if kw.get("quantity", "flux") == "flux":
            r = run_case(S.sr(), calls[:-1] + [(last, dict(kw, gpu=1, quantity="level"))])
            res[name + "/level"] = np.array([p[1] for p in r], dtype=np.float64)
    np.savez(out, **res)


if __name__ == "__main__":
    main()
