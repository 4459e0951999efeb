"""Edge cases and a full-size property of the packing engine.

Edge cases: the smallest instances (2 and 3 circles), ragged last circle
blocks (N just above and below a tile side), no walls, both tile sides,
teacher-forced against the reference's own sweep (core/paradmm.c:736-741)
like the box case of test_gpu_parity.py.

Full size: N = 8000 circles of the benchmark's 2 x 1 box on a grid, equal
radii far below the spacing, so that no pair overlaps and no circle touches
a wall.  Then every pair and wall prox returns its input (packing/host.c:
31-65, 83-132) and every circle sees the same edges, so all radii follow one
scalar ADMM recurrence (N + 3 identity edges of weight rho and one radius
edge whose prox is rho_r n / (rho_r - 2) for exponent 2) and the centres do
not move.  The recurrence is computed here in FP64; the engine keeps FP32
edge state, so radii must agree to FP32 accuracy after every sweep.
"""
import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4
RHO, RHO_R, ALPHA, EXP = 10.0, 5.0, 1.0, 2.0


@pytest.mark.parametrize("N,bw,walls", [(2, 64, "box"), (3, 64, "none"), (63, 64, "box"), (65, 64, "none"),
                                        (127, 128, "box"), (129, 128, "box"), (130, 64, "triangle")])
def test_teacher_forced_edge_cases(N, bw, walls):
    W, H = (1.0, 0.87) if walls == "triangle" else (1.0, 1.0)
    wl = {"box": eb.box_walls(W, H), "none": np.zeros((0, 4)), "triangle": eb.triangle_walls()}[walls]
    seed = 70 + N
    pg = eb.PackingGraph(N, wl, EXP)
    pg.init_seeded(eb.seeded_circles(N, W, H, 0.05, seed), RHO, RHO_R, ALPHA)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, wl, EXP)
    orc.init(seed, W, H, 0.05, RHO, RHO_R, ALPHA)
    done = 0
    for k in (0, 4, 60):
        orc.run(k - done, trace=False)
        done = k
        for key, v in orc.state().items():
            pg.G.arr(key)[:] = v
        with eb.Handle.from_graph(pg.G, engine=eb.ENGINE_PACKING, block_width=bw) as h:
            h.iterate(1)
            h.download(pg.G)
        orc.sweep()
        done += 1
        ref, got = orc.state(), pg.G.state()
        d = max(float(np.max(np.abs(got[q] - ref[q]))) for q in ("X", "M", "N", "U", "Z"))
        assert d <= TOL_F32, f"N={N} k={k}: max diff {d}"


def _radius_recurrence(r0: float, n_identity: int, sweeps: int) -> np.ndarray:
    """Radius consensus of one circle whose n_identity edges (pairs, walls)
    have the identity prox and whose radius edge has the exponent-2 prox,
    from X = Z, U = 0 (core/paradmm.c:569-715 restated for two edge
    classes); returns the radius after each sweep."""
    w1, w2 = RHO * n_identity, RHO_R
    z, u1, u2 = r0, 0.0, 0.0
    out = []
    for _ in range(sweeps):
        x1 = z - u1                               # identity prox of N = Z - U
        x2 = RHO_R * (z - u2) / (RHO_R - 2.0)     # radius prox, exponent 2
        zn = (w1 * (x1 + u1) + w2 * (x2 + u2)) / (w1 + w2)
        u1 += ALPHA * (x1 - zn)
        u2 += ALPHA * (x2 - zn)
        z = zn
        out.append(z)
    return np.array(out)


@pytest.mark.parametrize("N,nx,ny,K", [(8000, 126, 64, 40),      # the bench's size, spacing ~0.0159 x 0.0156
                                      (32767, 256, 128, 200)])  # the largest instance the engine takes
def test_full_size_separated_grid_follows_the_scalar_recurrence(N, nx, ny, K):
    """N = 32767 has 536,821,761 pair factors (2.1e9 reference edges, 12.9 GB
    of pair state): indices beyond 2^31 in every tile and partial-sum
    address."""
    W, H = 2.0, 1.0
    gx, gy = np.meshgrid((np.arange(nx) + 0.5) * W / nx, (np.arange(ny) + 0.5) * H / ny, indexing="ij")
    pts = np.stack([gx.ravel(), gy.ravel()], axis=1)[:N]
    r0 = 0.002
    circles = np.concatenate([pts, np.full((N, 1), r0)], axis=1)
    d = dict(n_circles=N, walls=eb.box_walls(W, H), exponent=EXP, rho=RHO, rho_radius=RHO_R, alpha=ALPHA,
             init=circles)
    want = _radius_recurrence(r0, N - 1 + 4, K)
    assert want[-1] < 0.0045  # still far from any contact: the identity-prox premise holds
    assert (want[-1] - r0) / r0 > 100 * 1e-5  # the radii move well beyond the tolerance below
    with eb.Handle.packing([d]) as h:
        prev = 0
        for k in sorted({1, 2, 10, K}):
            assert h.solve(k - prev, -1.0)["iterations"] == k - prev
            prev = k
            c = h.circles(0, N)
            assert np.abs(c[:, :2] - pts).max() <= 1e-6, f"centres moved at sweep {k}"
            rel = np.abs(c[:, 2] - want[k - 1]) / want[k - 1]
            assert rel.max() <= 1e-5, f"sweep {k}: radius off the recurrence by {rel.max():.2e}"
            # circles sum their edges in different orders (row vs column tiles): FP32 rounding only
            assert np.ptp(c[:, 2]) <= 1e-5 * want[k - 1], f"sweep {k}: radii differ between circles"
