"""Generates tests/golden/golden.npz from the UNMODIFIED reference FP64 solver
(oracle/_ref/libdgref.so, compiled in place from the reference tree by
oracle/Makefile).  Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py

For every case in tests/cases.py it stores the inputs and the reference's
outputs: residual R and f = -Minv R (solve.cpp:150), and for time-step cases
the state after nsteps RK steps plus the per-step residual norms the
reference prints (time_distributed.cpp:23-102)."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle  # noqa: E402
import cases  # noqa: E402


def main():
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libdgref.so is not built (make -C oracle ref)")
    out = {}
    for c in cases.residual_cases():
        m = oracle.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)
        R, f = ref.residual(m, c.prm, c.U)
        out[f"{c.name}/U"] = c.U
        out[f"{c.name}/R"] = R
        out[f"{c.name}/f"] = f
        print(f"{c.name:20s} |f| = {np.linalg.norm(f):.6e}")
    for c in cases.run_cases():
        m = oracle.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)
        U, norms = ref.run(m, c.prm, c.U, c.scheme, c.dt, c.nsteps)
        out[f"{c.name}/U0"] = c.U
        out[f"{c.name}/UN"] = U
        out[f"{c.name}/norms"] = norms
        print(f"{c.name:20s} |U_N - U_0| = {np.linalg.norm(U - c.U):.6e} norms[0] = {norms[0]:.6e}")
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
