"""Generates tests/golden/cfg2_steps.json: the FP64 oracle's state over the 10
time steps of the 64^3 x 6 tetrahedral configuration (1,572,864 tets,
274,625 nodes, nu = 1e-3, dt = 5e-3, lid-driven cavity), for the GPU parity
test of the full configuration (tests/test_cfg_parity.py).  The oracle's serial
solve of this system takes minutes per step, too long to repeat inline, so its
result is recorded once: per step the L2 norm of each field (u, v, w, p) and the
full state of 256 seeded sample nodes, with the solver's iterations and final
relative residual.

    python tests/golden/make_cfg2_steps.py [threads]

The inputs are the seeded synthetic problem (oracle.lid_driven_problem, bitwise
equal to the product's generator); the oracle assembles on `threads` host
threads (bitwise equal to serial) and solves with ILU(0)-GMRES(100) to 1e-13.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402

N_CELLS, NU, DT, STEPS, SAMPLES, TOL = 64, 1e-3, 5e-3, 10, 256, 1e-13
OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cfg2_steps.json")


def main():
    threads = int(sys.argv[1]) if len(sys.argv) > 1 else (os.cpu_count() or 1)
    pb = O.lid_driven_problem(3, N_CELLS, NU, DT)
    o = O.Oracle(pb["coords"], pb["conn"], O.options(dt=DT, use_specializations=False))
    o.set_state(pb["up"], pb["lin"], pb["nu"])
    o.add_dirichlet(pb["bc_nodes"], pb["bc_comps"], pb["bc_values"])
    nodes = np.sort(np.random.default_rng(20261203).choice(pb["coords"].shape[0], SAMPLES, replace=False))
    steps = []
    for k in range(STEPS):
        t0 = time.time()
        o.assemble(threads)
        o.apply_dirichlet()
        res = o.solve(tol=TOL, maxit=20000, restart=100)
        o.update()
        up, _ = o.state()
        steps.append({"step": k + 1, "solver": {"rc": int(res["rc"]), "iterations": int(res["iterations"]),
                                                "rel_residual": float(res["rel_residual"])},
                      "norms": [float(np.linalg.norm(up[:, c])) for c in range(4)],
                      "samples": up[nodes].tolist(), "seconds": round(time.time() - t0, 1)})
        print(f"step {k + 1}: {steps[-1]['solver']} {steps[-1]['seconds']} s", flush=True)
    out = {"config": f"3D P1 tets {N_CELLS}^3x6, nu {NU}, dt {DT}, lid-driven cavity (walls then lid, p pinned "
                     "at node 0), generic element expression, theta 1",
           "oracle_solve": f"ILU(0)-GMRES(100) to relative residual {TOL}",
           "sample_nodes": nodes.tolist(), "steps": steps}
    with open(OUT, "w") as f:
        json.dump(out, f)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
