"""Generates tests/golden/long_runs.npz: long-horizon runs of the UNMODIFIED
reference FP64 solver (oracle/_ref/libdgref.so, compiled in place from the
reference tree by oracle/Makefile), for the GPU parity tests at the
benchmark configurations' own step counts.  Run from the repository root:

    make -C oracle ref && python tests/golden/make_long_runs.py

  vortex_8_p2_100   the isentropic-vortex configuration in full: periodic
                    [0,10]^3, 8^3 hexes, p = 2, Euler, RK4, dt = 0.01, 100 steps
  tgv_8_p3_1000     the Taylor-Green configuration (Re 1600, Ma 0.1, BR2,
                    RK4, dt = 0.2 h / ((2p+1)(c + |u|max))) at 8^3 hexes, p = 3,
                    for its 1000 steps

Only the final states and the per-step residual norms are stored; the
initial states come from tests/cases.py at test time."""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from tests import cases  # noqa: E402


def main():
    ref = oracle.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libdgref.so is not built (make -C oracle ref)")
    out = {}
    for c in cases.long_run_cases():
        t0 = time.time()
        m = oracle.Mesh(c.nx, c.ny, c.nz, c.p, c.q, c.nodes, c.bounds)
        U, norms = ref.run(m, c.prm, c.U, c.scheme, c.dt, c.nsteps)
        out[f"{c.name}/UN"] = U
        out[f"{c.name}/norms"] = norms
        print(f"{c.name:20s} {c.nsteps} steps in {time.time() - t0:.0f} s, |U_N - U_0| = "
              f"{np.linalg.norm(U - c.U):.6e}", flush=True)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "long_runs.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()
