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
    if not os.path.exists(PORT) or (os.path.isdir("/root/reference") and not os.path.exists(REF)):
        subprocess.run(["make", "-C", ORACLE], check=True, capture_output=True)


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
    L.max_alpha_radius.restype = C.c_double
    L.max_alpha_radius.argtypes = [C.c_double, C.c_double, C.c_double]
    for n in ("disk_collision_variable_radius", "disk_plane_collision_variable_radius",
              "maximize_sum_of_squared_disk_radii_alpha"):
        getattr(L, n).argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_int, C.c_int, C.c_void_p]
        getattr(L, n).restype = None
    _cache[path] = L
    return L


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
