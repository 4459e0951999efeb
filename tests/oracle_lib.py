"""Loaders for the oracle libraries (test infrastructure only).

  oracle/libparadmm_port.so        C restatement of the reference + harness
  oracle/_ref/libparadmm_ref.so    the reference's own sources + harness

Both export the paradmm.h API and the packing harness (oracle/harness.h).
They are built by `make -C oracle` (``__graft_entry__.build()`` does it).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from engine_b200 import Graph

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE = os.path.join(ROOT, "oracle")
PORT = os.path.join(ORACLE, "libparadmm_port.so")
REF = os.path.join(ORACLE, "_ref", "libparadmm_ref.so")
REF_OFAST = os.path.join(ORACLE, "_ref", "libparadmm_ref_ofast.so")

_cache: dict[str, C.CDLL] = {}


def ensure_built() -> None:
    """Builds what is missing: the restatement always, the reference's own
    build when PARADMM_REFERENCE names the reference tree."""
    ref_tree = os.environ.get("PARADMM_REFERENCE", "")
    want_ref = bool(ref_tree) and os.path.isdir(ref_tree) and not os.path.exists(REF)
    if not os.path.exists(PORT) or want_ref:
        cmd = ["make", "-C", ORACLE] + ([f"REF={ref_tree}"] if want_ref else [])
        subprocess.run(cmd, check=True, capture_output=True)


def _load(path: str) -> C.CDLL:
    if path in _cache:
        return _cache[path]
    L = C.CDLL(path)
    L.orc_packing_new.restype = C.c_void_p
    L.orc_packing_new.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_double, C.c_int]
    L.orc_packing_free.argtypes = [C.c_void_p]
    L.orc_packing_graph.restype = C.POINTER(Graph)
    L.orc_packing_graph.argtypes = [C.c_void_p]
    L.orc_packing_init.argtypes = [C.c_void_p, C.c_uint64, C.c_double, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double]
    L.orc_packing_metrics.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.orc_packing_run.restype = C.c_int
    L.orc_packing_run.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_double, C.c_void_p]
    L.orc_time_sweeps.restype = C.c_double
    L.orc_time_sweeps.argtypes = [C.c_void_p, C.c_int, C.c_int]
    L.orc_max_threads.restype = C.c_int
    L.orc_u01.restype = C.c_double
    L.orc_u01.argtypes = [C.POINTER(C.c_uint64)]
    for n in ("updateG", "updateXM", "updateX", "updateM", "updateZ", "updateUN", "updateU", "updateN",
              "initialize_X_N_Z_M_U_zeros", "closeG"):
        getattr(L, n).argtypes = [C.POINTER(Graph)]
        getattr(L, n).restype = None
    L.updateGOpenMP.argtypes = [C.POINTER(Graph), C.c_int, C.c_int]
    L.startG.argtypes = [C.POINTER(Graph), C.c_int]
    L.addNode.argtypes = [C.POINTER(Graph), C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.initialize_RHOS_APHAS.argtypes = [C.POINTER(Graph), C.c_double, C.c_double]
    L.initialize_X_N_Z_M_U_optimal.argtypes = [C.POINTER(Graph), C.POINTER(C.c_double), C.POINTER(C.c_double),
                                                 C.c_int]
    L.initialize_X_N_Z_M_U_optimal.restype = None
    L.orc_packing_run_balanced.restype = C.c_int
    L.orc_packing_run_balanced.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int,
                                           C.c_void_p]
    L.max_alpha_radius.restype = C.c_double
    L.max_alpha_radius.argtypes = [C.c_double, C.c_double, C.c_double]
    for n in ("disk_collision_variable_radius", "disk_plane_collision_variable_radius",
              "maximize_sum_of_squared_disk_radii_alpha"):
        getattr(L, n).argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_int, C.c_int, C.c_void_p]
        getattr(L, n).restype = None
    _cache[path] = L
    return L


def omp_threads(G, want: int) -> int:
    """The most host threads (<= want) the reference's updateGOpenMP can use
    on graph G.  It splits each loop as id * N / numthreads in int
    (core/paradmm.c:964-965, 990-991, 1002-1003, 1044-1045, 1069-1070), with
    N up to num_edges * num_dims; past INT_MAX / N threads the product
    overflows and the threads write outside the state arrays (the N = 8000
    bench graph, 2 x 128,056,000 components, allows 8)."""
    n = max(int(G.num_edges) * int(G.num_dims), int(G.num_opts), int(G.num_vars), 1)
    return max(1, min(int(want), (2 ** 31 - 1) // n))


def port() -> C.CDLL:
    ensure_built()
    return _load(PORT)


def ref() -> C.CDLL | None:
    ensure_built()
    return _load(REF) if os.path.exists(REF) else None


def best() -> C.CDLL:
    """The reference build when present, else the restatement."""
    return ref() or port()


class OraclePacking:
    """A packing graph built and iterated by an oracle library."""

    def __init__(self, lib: C.CDLL, N: int, walls: np.ndarray, exponent: float = 2.0, order: int = 0):
        self.lib = lib
        self.N = N
        self.walls = np.ascontiguousarray(walls, dtype=np.float64)
        self.P = lib.orc_packing_new(N, len(self.walls), self.walls.ctypes.data, exponent, order)
        assert self.P, "orc_packing_new failed"

    @property
    def G(self) -> Graph:
        return self.lib.orc_packing_graph(self.P).contents

    def graph_ptr(self):
        return self.lib.orc_packing_graph(self.P)

    def init(self, seed: int, W: float, H: float, rmax: float, rho: float, rho_radius: float, alpha: float):
        self.lib.orc_packing_init(self.P, seed, W, H, rmax, rho, rho_radius, alpha)

    def run(self, iters: int, nthreads: int = 0, tol: float = 0.0, trace: bool = True):
        if nthreads > 0:
            nthreads = omp_threads(self.G, nthreads)
        tr = np.zeros((iters, 4)) if trace else None
        n = self.lib.orc_packing_run(self.P, iters, nthreads, tol, tr.ctypes.data if trace else None)
        return n, (tr[:n] if trace else None)

    def sweep(self):
        self.lib.updateG(self.graph_ptr())

    def metrics(self, Zprev=None) -> np.ndarray:
        out = np.zeros(4)
        zp = None if Zprev is None else np.ascontiguousarray(Zprev, dtype=np.float64)
        self.lib.orc_packing_metrics(self.P, None if zp is None else zp.ctypes.data, out.ctypes.data)
        return out

    def state(self) -> dict:
        return self.G.state()

    def run_balanced(self, iters: int, period: int, mu: float, lmin: int, lmax: int, tol: float = 0.0):
        """orc_packing_run_balanced: updateG with residual balancing of the
        penalties between sweeps; trace rows (r, s, log2 scale, applied)."""
        tr = np.zeros((iters, 4))
        n = self.lib.orc_packing_run_balanced(self.P, iters, tol, period, mu, lmin, lmax, tr.ctypes.data)
        assert n >= 0, "orc_packing_run_balanced refused its arguments"
        return n, tr[:n]

    def duals(self, order: int = 0):
        """The duals U of the current state in the engine's warm-start order
        (paradmm_gpu_warm_start_duals): pair_duals [P, 6] (pairs i < j
        row-major: u_cx_i, u_cy_i, u_r_i, u_cx_j, u_cy_j, u_r_j),
        wall_duals [N * nwalls, 3] (circle by circle, walls in order) and
        radius_duals [N]; radius edges give their dim 0.  Graph order 0
        (packing/host.c: radius factors, then walls, then pairs)."""
        assert order == 0
        N, nw = self.N, len(self.walls)
        U = self.G.arr("U").reshape(-1, 2)
        rad = U[:N, 0].copy()
        wall = np.zeros((N * nw, 3))
        for w in range(nw):
            e = N + 2 * (w * N + np.arange(N))
            wall[np.arange(N) * nw + w, 0:2] = U[e]
            wall[np.arange(N) * nw + w, 2] = U[e + 1, 0]
        base = N + 2 * nw * N
        q = U[base:].reshape(-1, 4, 2)
        pair = np.stack([q[:, 0, 0], q[:, 0, 1], q[:, 1, 0], q[:, 2, 0], q[:, 2, 1], q[:, 3, 0]], axis=1)
        return pair, wall, rad

    def circles(self) -> np.ndarray:
        Z = self.G.arr("Z").reshape(-1, 4)
        return np.ascontiguousarray(Z[:, :3])

    def set_circles_plain(self, circles: np.ndarray) -> None:
        """Plain start from given circles: Z, X = N = M = Z_v(e), U = 0."""
        G = self.G
        Z = G.arr("Z").reshape(-1, 4)
        Z[:, 0:3] = circles
        Z[:, 3] = circles[:, 2]
        Zv = Z.reshape(-1, 2)
        v = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
        for k in ("X", "N", "M"):
            G.arr(k).reshape(-1, 2)[:] = Zv[v]
        G.arr("U")[:] = 0.0

    def set_state(self, st: dict) -> None:
        G = self.G
        for k, v in st.items():
            G.arr(k)[:] = v

    def close(self):
        if self.P:
            self.lib.orc_packing_free(self.P)
            self.P = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
