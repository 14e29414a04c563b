"""Generate the golden fixtures in tests/golden/*.npz from the reference's own CPU build.

Run in a container that holds the reference sources (oracle/Makefile builds ``oracle/_ref`` from
them); the GPU box never runs this.  Each fixture stores the result of one case in
``tests/golden/cases.py`` as computed by the reference ``oscars.sr`` (gpu=0, nthreads=1), plus the
per-entry stop levels from a second ``quantity='level'`` call where the case returns values.

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py flux_und_41
    python tests/golden/make_golden.py files      # the reference's output files (files.npz)
    python tests/golden/make_golden.py adjoint_fd # finite-difference gradients (adjoint_fd.npz)
    python tests/golden/make_golden.py stl_files  # the mesh file of stlofile (stl_files.npz)
    python tests/golden/make_golden.py deep_levels  # extended levels up to 27 (deep_levels.npz)
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


def make_files(S):
    """Output files written by the reference for FILE_CASES (ofile and bofile) -> files.npz: per case
    the text and binary bytes and the returned result (positions / energies / trajectory and values)
    that the files hold."""
    import tempfile
    from cases import FILE_CASES
    out = {}
    with tempfile.TemporaryDirectory() as d:
        for name, (setup, call, kw) in FILE_CASES.items():
            obj = S.sr(nthreads=1, gpu=0)
            txt, binf = os.path.join(d, name + ".txt"), os.path.join(d, name + ".bin")
            kw = dict(kw, ofile=txt, bofile=binf)
            if call != "calculate_trajectory":
                kw.setdefault("nthreads", 1)
            res = run_case(obj, setup + [(call, kw)])
            out[name + "/txt"] = np.frombuffer(open(txt, "rb").read(), dtype=np.uint8)
            out[name + "/bin"] = np.frombuffer(open(binf, "rb").read(), dtype=np.uint8)
            if call == "calculate_trajectory":
                out[name + "/traj"] = np.array([[p[0]] + p[1] + p[2] + p[3] for p in res], dtype=np.float64).T
            else:
                pos, val = flatten(res)
                out[name + "/pos"] = pos
                out[name + "/val"] = val
    np.savez_compressed(os.path.join(HERE, "files.npz"), **out)


def make_stl_file(S):
    """The mesh file the reference writes for calculate_power_density_stl(stlofile=...) on the plate
    and the shield (stl_files.npz: the bytes after the 80-byte header, which the reference leaves
    partly uninitialised)."""
    import tempfile
    from cases import stl_file
    obj = S.sr(nthreads=1, gpu=0)
    run_case(obj, CASES["stl_shadow"][:-1])
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "out.stl")
        obj.calculate_power_density_stl([0, 0, 0], stlofile=path, nthreads=1, max_level=9)
        with open(path, "rb") as f:
            data = f.read()
    np.savez_compressed(os.path.join(HERE, "stl_files.npz"), head=np.frombuffer(data[:37], dtype=np.uint8),
                        body=np.frombuffer(data[80:], dtype=np.uint8))


def make_deep_levels(S):
    """The spectrum of cases.DEEP_LEVELS (extended levels up to 27) -> deep_levels.npz."""
    from cases import DEEP_LEVELS
    pos, val = flatten(run_case(S.sr(nthreads=1, gpu=0), DEEP_LEVELS))
    np.savez_compressed(os.path.join(HERE, "deep_levels.npz"), pos=pos, val=val)


def make_adjoint(S):
    """Central finite differences of loss = sum (F(s) - F(1))^2 over the adjoint configuration, every
    one of the 82 half-period factors, with the reference's CPU path (the scaled undulator given to it
    as a Python field function), at the steps ADJ_FD_STEPS -> adjoint_fd.npz (grad_h<i> per step).
    The FP64 retarded phase (~7e10 rad here) carries ~1e-5 rad of rounding, so differences with
    h = 1e-6 are dominated by rounding; the tests extrapolate the larger steps (Richardson)."""
    import math
    from cases import ADJ_FD_STEPS, BEAM, adjoint_config, halfscale_41, halfscale_function
    obs, energies, level = adjoint_config()
    s0 = np.array(halfscale_41())

    def flux(s):
        o = S.sr(nthreads=1, gpu=0)
        o.add_bfield_function(halfscale_function([0, 0.5, 0], [0, 0, 0.05], 41, -math.pi / 2, list(s)))
        o.set_particle_beam(**BEAM[1])
        o.set_ctstartstop(-1.5, 1.5)
        o.set_npoints_trajectory(20001)
        F = np.zeros((obs.shape[0], energies.size))
        for j, e in enumerate(energies):
            res = o.calculate_flux_rectangle(energy_eV=float(e), npoints=[5, 5], width=[0.001, 0.001],
                                             translation=[0, 0, 30], precision=0, max_level=level, nthreads=1,
                                             dim=3)
            assert np.array_equal(np.array([r[0] for r in res]), obs)
            F[:, j] = [r[1] for r in res]
        return F
    F1 = flux(np.ones(82))
    F = flux(s0)
    loss = lambda s: float(np.sum((flux(s) - F1) ** 2))
    out = dict(s=s0, F=F, F1=F1, h=np.array(ADJ_FD_STEPS), level=level)
    for i, h in enumerate(ADJ_FD_STEPS):
        g = np.zeros(82)
        for k in range(82):
            e = np.zeros(82)
            e[k] = h
            g[k] = (loss(s0 + e) - loss(s0 - e)) / (2 * h)
        out["grad_h%d" % i] = g
    np.savez_compressed(os.path.join(HERE, "adjoint_fd.npz"), **out)


def main(argv):
    S = reference()
    if argv[1:] == ["adjoint_fd"]:
        make_adjoint(S)
        print("wrote adjoint_fd")
        return
    if argv[1:] == ["files"]:
        make_files(S)
        print("wrote files")
        return
    if argv[1:] == ["deep_levels"]:
        make_deep_levels(S)
        print("wrote deep_levels")
        return
    if argv[1:] == ["stl_files"]:
        make_stl_file(S)
        print("wrote stl_files")
        return
    names = argv[1:] or sorted(CASES)
    for n in names:
        make(n, S)
        print("wrote", n)


if __name__ == "__main__":
    main(sys.argv)
