"""Pins the oracle: the C restatement (oracle/paradmm_port.c) against the
reference compiled from its own sources (oracle/_ref) and against the golden
fixtures that the reference produced (tests/golden/make_golden.py)."""
import glob
import os

import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

GOLDEN = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "*.npz")))


def _walls(kind_w, W, H):
    return eb.box_walls(W, H) if kind_w == "box" else eb.triangle_walls()


def _same(a: dict, b: dict):
    for k in ("X", "M", "N", "U", "Z"):
        assert np.array_equal(a[k], b[k]), f"{k}: max |diff| {np.max(np.abs(a[k] - b[k]))}"


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("container", ["box", "triangle"])
def test_port_bit_identical_to_reference(order, container):
    ref = oracle_lib.ref()
    if ref is None:
        pytest.skip("reference sources not available here")
    port = oracle_lib.port()
    N = 30
    walls = _walls(container, 1.2, 1.0)
    a = oracle_lib.OraclePacking(ref, N, walls, 2.0, order=order)
    b = oracle_lib.OraclePacking(port, N, walls, 2.0, order=order)
    a.init(9, 1.2, 1.0, 0.06, 10.0, 5.0, 1.0)
    b.init(9, 1.2, 1.0, 0.06, 10.0, 5.0, 1.0)
    _, ta = a.run(500)
    _, tb = b.run(500)
    _same(a.state(), b.state())
    assert np.array_equal(ta, tb)


def test_port_openmp_equals_serial():
    port = oracle_lib.port()
    N = 40
    walls = eb.box_walls(1, 1)
    a = oracle_lib.OraclePacking(port, N, walls, 2.0)
    b = oracle_lib.OraclePacking(port, N, walls, 2.0)
    a.init(3, 1, 1, 0.05, 10, 5, 1)
    b.init(3, 1, 1, 0.05, 10, 5, 1)
    a.run(100, nthreads=0, trace=False)
    b.run(100, nthreads=4, trace=False)
    _same(a.state(), b.state())


@pytest.mark.parametrize("path", GOLDEN, ids=[os.path.basename(p) for p in GOLDEN])
@pytest.mark.parametrize("which", ["port", "ref"])
def test_oracle_reproduces_golden(path, which):
    lib = oracle_lib.port() if which == "port" else oracle_lib.ref()
    if lib is None:
        pytest.skip("reference sources not available here")
    g = np.load(path)
    N = int(g["N"])
    P = oracle_lib.OraclePacking(lib, N, g["walls"], 2.0, order=int(g["order"]))
    P.init(int(g["seed"]), float(g["W"]), float(g["H"]), float(g["rmax"]), float(g["rho"]),
           float(g["rho_radius"]), float(g["alpha"]))
    for k in ("X", "M", "N", "U", "Z"):
        assert np.array_equal(P.state()[k], g[f"init_{k}"]), k
    done = 0
    traces = []
    for s in g["snaps"]:
        _, tr = P.run(int(s) - done)
        traces.append(tr)
        done = int(s)
        st = P.state()
        for k in ("X", "M", "N", "U", "Z"):
            assert np.array_equal(st[k], g[f"it{s}_{k}"]), f"{k} at sweep {s}"
    assert np.array_equal(np.concatenate(traces), g["trace"])


def test_harness_metrics_match_numpy():
    """The residual definitions (RMS over all (edge, dim)) recomputed here."""
    port = oracle_lib.port()
    N = 15
    walls = eb.box_walls(1, 1)
    P = oracle_lib.OraclePacking(port, N, walls, 2.0)
    P.init(5, 1, 1, 0.1, 10, 5, 1)
    P.run(20, trace=False)
    zprev = P.state()["Z"].copy()
    P.sweep()
    m = P.metrics(zprev)
    G = P.G
    e2v = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
    st = P.state()
    r = np.sqrt(np.mean((st["X"] - st["Z"][e2v]) ** 2))
    s = np.sqrt(np.mean((st["Z"][e2v] - zprev[e2v]) ** 2))
    assert abs(r - m[0]) <= 1e-14 * max(1, r) and abs(s - m[1]) <= 1e-14 * max(1, s)
    Z = st["Z"]
    c, rad = Z[0::2], Z[1::2, 0]
    viol = max(0.0, float(np.max(-rad)))
    for w in walls:
        viol = max(viol, float(np.max(w[0] * (c[:, 0] - w[2]) + w[1] * (c[:, 1] - w[3]) + rad)))
    for i in range(N):
        for j in range(i + 1, N):
            viol = max(viol, rad[i] + rad[j] - float(np.hypot(*(c[i] - c[j]))))
    assert abs(viol - m[2]) <= 1e-12 and abs(rad.sum() - m[3]) <= 1e-12


def test_balanced_run_restates_the_rule():
    """orc_packing_run_balanced (the residual-balancing rule the engine
    implements, over the reference's own updateG): before the first decision
    applies it is the plain run bit for bit; afterwards every penalty is its
    base value times 2^(log2 scale), the scaled duals moved by the inverse
    factor (so rho U is continuous), and N = Z - U."""
    lib = oracle_lib.best()
    N = 24
    walls = eb.box_walls(1.0, 1.0)
    a = oracle_lib.OraclePacking(lib, N, walls, 2.0)
    b = oracle_lib.OraclePacking(lib, N, walls, 2.0)
    a.init(11, 1.0, 1.0, 0.05, 10.0, 5.0, 1.0)
    b.init(11, 1.0, 1.0, 0.05, 10.0, 5.0, 1.0)
    base = a.G.arr("RHOS").copy()
    n, tr = a.run_balanced(26, 25, 2.0, -1, 4)  # the first decision (age 25) applies after sweep 27
    b.run(26, trace=False)
    _same(a.state(), b.state())
    assert not tr[:, 3].any()
    # one more sweep each: the balanced run now applies its first decision
    n2, tr2 = a.run_balanced(200, 25, 2.0, -1, 4)
    assert n2 == 200 and tr2[:, 3].any()
    G = a.G
    l2 = int(tr2[-1, 2])
    assert np.array_equal(G.arr("RHOS"), base * 2.0 ** l2)
    U, Z = G.arr("U"), G.arr("Z")
    v = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
    applied_last = np.nonzero(tr2[:, 3])[0][-1]
    if applied_last == len(tr2) - 1:  # N was reset from the rescaled U right after the last sweep
        assert np.array_equal(G.arr("N"), Z[v] - U)
    # a period below 3 is refused
    assert a.lib.orc_packing_run_balanced(a.P, 5, 0.0, 2, 10.0, -1, 4, None) == -1


@pytest.mark.parametrize("maxiter", [1, 7])
def test_port_optimal_init_bit_identical_to_reference(maxiter):
    """initialize_X_N_Z_M_U_optimal (core/paradmm.c:266-375) restated in the
    port: same arrays as the reference's own, bit for bit, from a mid-solve
    Zinit and Uinit; the engine's device-side dual initialiser is checked
    against it on the GPU."""
    import ctypes as C
    ref = oracle_lib.ref()
    if ref is None:
        pytest.skip("reference sources not available here")
    port = oracle_lib.port()
    N = 30
    walls = eb.box_walls(1.0, 1.0)
    out = []
    for lib in (ref, port):
        o = oracle_lib.OraclePacking(lib, N, walls, 2.0)
        o.init(5, 1.0, 1.0, 0.05, 10.0, 5.0, 1.0)
        o.run(120, trace=False)
        z, u = o.G.arr("Z").copy(), o.G.arr("U").copy()
        lib.initialize_X_N_Z_M_U_optimal(o.graph_ptr(), z.ctypes.data_as(C.POINTER(C.c_double)),
                                         u.ctypes.data_as(C.POINTER(C.c_double)), maxiter)
        out.append(o.state())
    _same(out[0], out[1])
