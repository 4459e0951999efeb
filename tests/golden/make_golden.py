"""Generates tests/golden/*.npz by running the reference's own C code.

Needs oracle/_ref/libparadmm_ref.so, i.e. the reference compiled from its
sources (core/paradmm.c, packing/host.c) by oracle/Makefile with parity
flags.  Each fixture records a seeded circle-packing problem (the reference
demo's graph, packing/host.c:283-343, in a box or the demo's triangle), its
initial state, and the reference's X, M, N, U, Z after selected sweeps of
updateG, with the per-sweep metrics of oracle/harness.c.

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import engine_b200 as eb  # noqa: E402
import oracle_lib  # noqa: E402

CASES = [
    # name, N, container, W, H, rmax, rho, rho_radius, alpha, order, seed, snapshots
    ("box_n12_order0", 12, "box", 1.0, 1.0, 0.15, 10.0, 5.0, 1.0, 0, 101, (1, 10, 100, 400)),
    ("box_n10_order1", 10, "box", 1.5, 1.0, 0.2, 10.0, 5.0, 0.5, 1, 202, (1, 25, 200)),
    ("triangle_n8", 8, "triangle", 1.0, 0.87, 0.2, 10.0, 5.0, 0.1, 0, 303, (1, 50, 300)),
]


def walls_for(kind, W, H):
    return eb.box_walls(W, H) if kind == "box" else eb.triangle_walls()


def main():
    ref = oracle_lib.ref()
    if ref is None:
        raise SystemExit("oracle/_ref/libparadmm_ref.so is missing (needs the reference sources)")
    for name, N, kind, W, H, rmax, rho, rho_r, alpha, order, seed, snaps in CASES:
        walls = walls_for(kind, W, H)
        P = oracle_lib.OraclePacking(ref, N, walls, 2.0, order=order)
        P.init(seed, W, H, rmax, rho, rho_r, alpha)
        out = dict(N=N, walls=walls, W=W, H=H, rmax=rmax, rho=rho, rho_radius=rho_r, alpha=alpha, order=order,
                   seed=seed, snaps=np.array(snaps))
        for k, v in P.state().items():
            out[f"init_{k}"] = v
        out["RHOS"] = P.G.arr("RHOS").copy()
        done = 0
        traces = []
        for s in snaps:
            _, tr = P.run(s - done)
            traces.append(tr)
            done = s
            for k, v in P.state().items():
                out[f"it{s}_{k}"] = v
        out["trace"] = np.concatenate(traces)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, "edges", P.G.num_edges, "final metrics", out["trace"][-1])
        P.close()


if __name__ == "__main__":
    main()
