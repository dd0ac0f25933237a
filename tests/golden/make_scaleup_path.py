"""Golden fixture of a complete load path of the scale-up workload, shrunk to
16^3 hexes x 6 tets (24,576 tets, 14,739 DOF): interior jitter 0.15 h,
log-normal mu (sigma 0.3), top face u_z = -0.2 in 10 load steps, exactly the
block of the 64^3 benchmark at a quarter of the resolution.

The C oracle (oracle/fm_oracle.c, pinned bit for bit to the reference's own
build by tests/test_oracle_golden.py) runs the reference's Newton loop in
FP64: the Dirichlet predictor, PCG-ILU(0) to 1e-12, Newton to 1e-10 and
Armijo backtracking on every iteration as armijo_line_search_true
(FEM/adaptive_fem_engine.hpp:933-985, c = 1e-4, 10 trials) - without it
the reference's tangent stops contracting at load levels 8-10 and Newton
diverges (oracle: level 8 hits 400 iterations, level 9 grows 10x).

Writes tests/golden/scaleup16_path.npz: u after load levels 5 and 10, and
per level the Newton and PCG counts and the Armijo step lengths.

    python tests/golden/make_scaleup_path.py     (about 3 minutes, 1 core)
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "atlas-flexmesh_b200"))

import oracle as O  # noqa: E402
from flexmesh_b200 import configs  # noqa: E402

N = 16
LINE_SEARCH, LS_C = 10, 1e-4


def main():
    P = configs.scaleup_block(N, mesher=O.unit_cube)
    rp, ci = O.pattern(P.n_nodes, P.conn, "solve")
    slot = O.slot_map(P.n_nodes, P.conn, rp, ci)
    mu, lam = P.lame()
    act = (P.elem_volume >= 1e-30).astype(np.uint8)
    u = np.zeros(P.xyz.size)
    out = {"N": N, "line_search": LINE_SEARCH, "ls_c": LS_C}
    newton, pcg, alphas, alpha_ptr = [], [], [], [0]
    t0 = time.time()
    for s in range(1, P.n_steps + 1):
        u, st, nps, pps, al = O.newton_ex(P.xyz, P.conn, mu, lam, P.nu, rp, ci, slot, P.mask,
                                          P.bc_value, P.n_steps, first_step=s, last_step=s,
                                          rtol=1e-10, inner_tol=1e-12, max_newton=400,
                                          max_pcg=20000, line_search=LINE_SEARCH, ls_c=LS_C,
                                          u0=u, active=act)
        assert st == 0, (s, st)
        newton.append(int(nps[0]))
        pcg.append(int(pps[0]))
        alphas.extend(al.tolist())
        alpha_ptr.append(len(alphas))
        if s == 5:
            out["u_level5"] = u.copy()
        print(f"level {s}: newton {nps[0]} pcg {pps[0]} backtracked {(al < 1).sum()} "
              f"({time.time() - t0:.0f} s)", flush=True)
    out["u_level10"] = u
    out["newton"] = np.array(newton, np.int32)
    out["pcg"] = np.array(pcg, np.int32)
    out["alpha"] = np.array(alphas)
    out["alpha_ptr"] = np.array(alpha_ptr, np.int32)
    np.savez_compressed(os.path.join(HERE, "scaleup16_path.npz"), **out)


if __name__ == "__main__":
    main()
