"""Python view of libparadmm_b200.so (paradmm.h + paradmm_gpu.h).

The library is the product: a C-ABI shared object whose sweep functions and
``paradmm_gpu_*`` entry points run sm_100a kernels.  This module only binds
it with ctypes so that tests and the benchmark can drive it the way a C host
does (``startG``/``addNode``/``initialize_*``/``updateG``, or the handle API),
plus a few conveniences for building circle-packing problems.

There is no fallback: if the shared library is missing, ``load()`` raises, and
every compute call fails with the engine's own error code when no CUDA device
is present.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libparadmm_b200.so")

# ---- status codes / enums (paradmm_gpu.h) ----
OK, EINVAL, ENOMEM, ECUDA, EUNSUPPORTED_OP, EUNSUPPORTED_GRAPH, ENONFINITE, ETIMEOUT, ENODEVICE = (
    0, -1, -2, -3, -4, -5, -6, -7, -8)
OP_UNKNOWN, OP_PAIR, OP_WALL, OP_RADIUS = 0, 1, 2, 3
ENGINE_AUTO, ENGINE_PACKING, ENGINE_GENERIC_F64, ENGINE_GENERIC_F32 = 0, 1, 2, 3
SCHEDULE_AUTO, SCHEDULE_GRID, SCHEDULE_INSTANCE, SCHEDULE_ONCHIP = 0, 1, 2, 3

OP_FN = C.CFUNCTYPE(None, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double),
                    C.c_int, C.c_int, C.c_void_p)


class Graph(C.Structure):
    """``graph`` of paradmm.h (reference core/paradmm.h:33-63), same layout."""
    _fields_ = [
        ("num_opts", C.c_int), ("num_vars", C.c_int), ("num_dims", C.c_int), ("num_edges", C.c_int),
        ("list_of_operators_functions_pointers", C.POINTER(C.c_void_p)),
        ("list_of_operators_param_pointers", C.POINTER(C.c_void_p)),
        ("list_of_operators_param_sizes", C.POINTER(C.c_int)),
        ("operatorix_to_numedges", C.POINTER(C.c_int)),
        ("operatorix_to_edgelistix", C.POINTER(C.POINTER(C.c_int))),
        ("varix_to_numedges", C.POINTER(C.c_int)),
        ("varix_to_edgelistix", C.POINTER(C.POINTER(C.c_int))),
        ("edgeix_to_varlistix", C.POINTER(C.c_int)),
        ("X", C.POINTER(C.c_double)), ("M", C.POINTER(C.c_double)), ("N", C.POINTER(C.c_double)),
        ("U", C.POINTER(C.c_double)), ("Z", C.POINTER(C.c_double)),
        ("RHOS", C.POINTER(C.c_double)), ("ALPHAS", C.POINTER(C.c_double)),
    ]

    # numpy views of the state arrays (no copies)
    def arr(self, name: str) -> np.ndarray:
        if name in ("X", "M", "N", "U"):
            shape = (self.num_edges, self.num_dims)
        elif name == "Z":
            shape = (self.num_vars, self.num_dims)
        elif name in ("RHOS", "ALPHAS"):
            shape = (self.num_edges,)
        else:
            raise KeyError(name)
        p = getattr(self, name)
        if not p:
            raise ValueError(f"graph array {name} is not allocated")
        return np.ctypeslib.as_array(p, shape=shape)

    def state(self) -> dict:
        return {k: self.arr(k).copy() for k in ("X", "M", "N", "U", "Z")}


class Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("engine", C.c_int), ("block_width", C.c_int), ("ctas_per_sm", C.c_int),
                ("check_every", C.c_int), ("schedule", C.c_int), ("cluster_size", C.c_int), ("reserved", C.c_int * 6)]


class Stats(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("converged", C.c_int), ("status", C.c_int),
                ("primal", C.c_double), ("dual", C.c_double), ("max_violation", C.c_double),
                ("total_radius", C.c_double), ("device_ms", C.c_double)]

    def as_dict(self) -> dict:
        return {k: getattr(self, k) for k, _ in self._fields_}


class PackingDesc(C.Structure):
    _fields_ = [("n_circles", C.c_int), ("n_walls", C.c_int), ("walls", C.POINTER(C.c_double)),
                ("exponent", C.c_double), ("rho", C.c_double), ("rho_radius", C.c_double),
                ("alpha", C.c_double), ("init", C.POINTER(C.c_double))]


class Tuning(C.Structure):
    """paradmm_gpu_tuning."""
    _fields_ = [("schedule", C.c_int), ("cluster_size", C.c_int), ("coop_min_n", C.c_int), ("candidates", C.c_int),
                ("ms", C.c_double), ("worst_ms", C.c_double), ("block_width", C.c_int), ("reserved", C.c_int * 3)]


class ParadmmError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"paradmm status {status}: {msg}")
        self.status = status


_lib = None

_SIGS = {
    # paradmm.h
    "startG": (None, [C.POINTER(Graph), C.c_int]),
    "closeG": (None, [C.POINTER(Graph)]),
    "printG": (None, [C.POINTER(Graph)]),
    "initialize_RHOS_APHAS": (None, [C.POINTER(Graph), C.c_double, C.c_double]),
    "initialize_X_N_Z_M_U_zeros": (None, [C.POINTER(Graph)]),
    "initialize_X_N_Z_M_U_rand": (None, [C.POINTER(Graph)] + [C.c_double] * 10),
    "initialize_X_N_Z_M_U_optimal": (None, [C.POINTER(Graph), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]),
    "addNode": (None, [C.POINTER(Graph), C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "addNodeWithParamSize": (None, [C.POINTER(Graph), C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "update_outgoing_rhos": (None, [C.POINTER(Graph)]),
    "updateXM": (None, [C.POINTER(Graph)]), "updateX": (None, [C.POINTER(Graph)]),
    "updateM": (None, [C.POINTER(Graph)]), "updateZ": (None, [C.POINTER(Graph)]),
    "updateUN": (None, [C.POINTER(Graph)]), "updateU": (None, [C.POINTER(Graph)]),
    "updateN": (None, [C.POINTER(Graph)]), "updateG": (None, [C.POINTER(Graph)]),
    "updateXOpenMP": (None, [C.POINTER(Graph)]), "updateMOpenMP": (None, [C.POINTER(Graph)]),
    "updateZOpenMP": (None, [C.POINTER(Graph)]), "updateUOpenMP": (None, [C.POINTER(Graph)]),
    "updateNOpenMP": (None, [C.POINTER(Graph)]),
    "updateGOpenMP": (None, [C.POINTER(Graph), C.c_int, C.c_int]),
    "abs_d": (C.c_double, [C.c_double]),
    "quicksort": (None, [C.POINTER(C.c_int), C.c_int]),
    "get_random": (C.c_double, [C.c_double, C.c_double]),
    "realloc2": (C.c_void_p, [C.c_void_p, C.c_size_t, C.c_size_t]),
    "max_alpha_radius": (C.c_double, [C.c_double, C.c_double, C.c_double]),
    "paradmm_add_packing_factors": (C.c_int, [C.POINTER(Graph), C.c_int, C.c_int, C.POINTER(C.c_double),
                                              C.POINTER(C.c_double), C.c_int]),
    # paradmm_gpu.h
    "paradmm_gpu_default_opts": (None, [C.POINTER(Opts)]),
    "paradmm_gpu_register_op": (C.c_int, [C.c_void_p, C.c_int]),
    "paradmm_gpu_create": (C.c_int, [C.POINTER(Graph), C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "paradmm_gpu_upload": (C.c_int, [C.c_void_p, C.POINTER(Graph)]),
    "paradmm_gpu_iterate": (C.c_int, [C.c_void_p, C.c_int]),
    "paradmm_gpu_solve": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.POINTER(Stats)]),
    "paradmm_gpu_download": (C.c_int, [C.c_void_p, C.POINTER(Graph)]),
    "paradmm_gpu_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "paradmm_gpu_engine": (C.c_int, [C.c_void_p]),
    "paradmm_gpu_destroy": (None, [C.c_void_p]),
    "paradmm_gpu_create_packing": (C.c_int, [C.POINTER(PackingDesc), C.c_int, C.POINTER(Opts), C.POINTER(C.c_void_p)]),
    "paradmm_gpu_instances": (C.c_int, [C.c_void_p]),
    "paradmm_gpu_instance_stats": (C.c_int, [C.c_void_p, C.POINTER(Stats)]),
    "paradmm_gpu_get_circles": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "paradmm_gpu_warm_start": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_float)]),
    "paradmm_gpu_warm_start_duals": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
                                               C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]),
    "paradmm_gpu_device_bytes": (C.c_int64, [C.c_void_p]),
    "paradmm_gpu_launches": (C.c_int64, [C.c_void_p]),
    "paradmm_gpu_instance_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "paradmm_gpu_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
    "paradmm_gpu_set_tail_handoff": (C.c_int, [C.c_void_p, C.c_int]),
    "paradmm_gpu_tail_handoffs": (C.c_int, [C.c_void_p]),
    "paradmm_gpu_set_fallback": (C.c_int, [C.c_void_p, C.c_int64]),
    "paradmm_gpu_set_rho_balance": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int, C.c_int]),
    "paradmm_gpu_rho_scale": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_int)]),
    "paradmm_gpu_selftest_barrier_timeout": (C.c_int, [C.c_int, C.c_int]),
    "paradmm_gpu_register_op_source": (C.c_int, [C.c_void_p, C.c_char_p, C.c_char_p]),
    "paradmm_gpu_autotune": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_void_p]),
    "paradmm_gpu_create_packing_tuned": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Opts), C.c_int, C.c_double,
                                                   C.POINTER(C.c_void_p), C.c_void_p]),
    "paradmm_gpu_instance_fallbacks": (C.c_int, [C.c_void_p, C.POINTER(C.c_int)]),
    "paradmm_gpu_phase_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_double)]),
    "paradmm_gpu_pin_graph": (C.c_int, [C.POINTER(Graph)]),
    "paradmm_gpu_unpin_graph": (C.c_int, [C.POINTER(Graph)]),
    "paradmm_noalloc_state_bytes": (C.c_int64, [C.c_int, C.c_int]),
    "paradmm_gpu_packing_iterate_noalloc": (C.c_int, [C.POINTER(PackingDesc), C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                                                      C.c_double, C.POINTER(Stats), C.c_int, C.c_void_p]),
    "paradmm_gpu_shard_rows": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int)]),
    "paradmm_gpu_create_packing_shard": (C.c_int, [C.POINTER(PackingDesc), C.c_int, C.c_int, C.POINTER(Opts),
                                                   C.POINTER(C.c_void_p)]),
    "paradmm_gpu_shard_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
    "paradmm_gpu_shard_start": (C.c_int, [C.c_void_p, C.c_int, C.c_double, C.c_int]),
    "paradmm_gpu_shard_begin": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "paradmm_gpu_shard_end": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "paradmm_gpu_shard_poll": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int)]),
    "paradmm_gpu_shard_finish": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(Stats)]),
    "paradmm_gpu_shard_fused_buffers": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p)]),
    "paradmm_gpu_shard_run_fused": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(C.c_void_p),
                                              C.POINTER(C.c_void_p), C.c_int, C.c_void_p]),
    "paradmm_gpu_ipc_export": (C.c_int, [C.c_void_p, C.c_void_p]),
    "paradmm_gpu_ipc_import": (C.c_int, [C.c_int, C.c_void_p, C.POINTER(C.c_void_p)]),
    "paradmm_gpu_ipc_close": (C.c_int, [C.c_int, C.c_void_p]),
    "paradmm_last_status": (C.c_int, []),
    "paradmm_last_error_string": (C.c_char_p, []),
    "paradmm_set_sweep_options": (None, [C.POINTER(Opts)]),
}

OP_NAMES = ("disk_collision_variable_radius", "disk_plane_collision_variable_radius",
            "maximize_sum_of_squared_disk_radii_alpha")


def load() -> C.CDLL:
    """Loads the in-tree shared library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FileNotFoundError(f"{LIB_PATH} is missing: run `python -m engine_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def op_ptr(name: str, lib: C.CDLL | None = None) -> int:
    """Address of an exported operator (for addNode)."""
    lib = lib or load()
    return C.cast(getattr(lib, name), C.c_void_p).value


def check(rc: int) -> None:
    if rc != OK:
        lib = load()
        raise ParadmmError(rc, (lib.paradmm_last_error_string() or b"").decode())


def last_status() -> int:
    return load().paradmm_last_status()


def last_error() -> str:
    return (load().paradmm_last_error_string() or b"").decode()


def opts(**kw) -> Opts:
    """paradmm_gpu_opts with defaults; coop_min_n sets reserved[0] (per-instance
    schedule: the smallest instance solved by a whole cluster)."""
    o = Opts()
    load().paradmm_gpu_default_opts(C.byref(o))
    for k, v in kw.items():
        if k == "coop_min_n":
            o.reserved[0] = int(v)
        elif k == "no_graphs":
            o.reserved[1] = 1 if v else 0
        else:
            setattr(o, k, v)
    return o


# ---------------------------------------------------------------------------
# Circle-packing problems (the reference demo's graph, packing/host.c:256-343)
# ---------------------------------------------------------------------------
def box_walls(W: float, H: float) -> np.ndarray:
    """Four half-planes v.(c - p) + r <= 0 keeping a circle inside [0,W]x[0,H]."""
    return np.array([[-1.0, 0.0, 0.0, 0.0], [1.0, 0.0, W, 0.0], [0.0, -1.0, 0.0, 0.0], [0.0, 1.0, 0.0, H]])


def triangle_walls() -> np.ndarray:
    """The reference demo's triangle container (packing/host.c:141-149)."""
    t = np.deg2rad(60.0)
    return np.array([[0.0, -1.0, 0.0, 0.0], [-np.sin(t), np.cos(t), 0.0, 0.0], [np.sin(t), np.cos(t), 1.0, 0.0]])


def splitmix64_u01(seed: int, n: int) -> np.ndarray:
    """n uniforms in [0,1) from a splitmix64 stream (top 53 bits / 2^53)."""
    out = np.empty(n, dtype=np.float64)
    s = seed & 0xFFFFFFFFFFFFFFFF
    M = 0xFFFFFFFFFFFFFFFF
    for i in range(n):
        s = (s + 0x9E3779B97F4A7C15) & M
        z = s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        z ^= z >> 31
        out[i] = (z >> 11) * (1.0 / 9007199254740992.0)
    return out


def seeded_circles(N: int, W: float, H: float, rmax: float, seed: int) -> np.ndarray:
    """Seeded plain init: circle i draws (cx, cy, r) = (W u, H u, rmax u)."""
    u = splitmix64_u01(seed, 3 * N).reshape(N, 3)
    return np.ascontiguousarray(u * np.array([W, H, rmax]))


class PackingGraph:
    """A circle-packing factor graph built through this library's addNode,
    in the reference demo's factor order (radius, walls, pairs)."""

    def __init__(self, N: int, walls: np.ndarray, exponent: float = 2.0, order: int = 0, lib=None,
                 ops: tuple[int, int, int] | None = None):
        self.lib = lib or load()
        self.N = N
        self.walls = np.ascontiguousarray(walls, dtype=np.float64)
        self.exponent = (C.c_double * 1)(exponent)
        self.G = Graph()
        self._extra_radius_ops = [] if ops is None else [ops[2]]
        lib = self.lib
        lib.startG(C.byref(self.G), 2)
        if ops is None:
            # the library's C-side builder: same addNode sequence, no per-factor Python call
            check(lib.paradmm_add_packing_factors(C.byref(self.G), N, len(self.walls),
                                                  self.walls.ctypes.data_as(C.POINTER(C.c_double)),
                                                  C.cast(self.exponent, C.POINTER(C.c_double)), order))
            return
        pair, wall, rad = ops
        wall_rows = [self.walls[w].ctypes.data for w in range(len(self.walls))]
        v1 = (C.c_int * 1)()
        v2 = (C.c_int * 2)()
        v4 = (C.c_int * 4)()

        def radius():
            for i in range(N):
                v1[0] = 2 * i + 1
                lib.addNode(C.byref(self.G), rad, C.cast(self.exponent, C.c_void_p), 1, v1)

        def wallf():
            for w in range(len(self.walls)):
                for i in range(N):
                    v2[0], v2[1] = 2 * i, 2 * i + 1
                    lib.addNode(C.byref(self.G), wall, wall_rows[w], 2, v2)

        if order == 0:
            radius(); wallf()
        else:
            wallf(); radius()
        for i in range(N - 1):
            for j in range(i + 1, N):
                v4[0], v4[1], v4[2], v4[3] = 2 * i, 2 * i + 1, 2 * j, 2 * j + 1
                lib.addNode(C.byref(self.G), pair, None, 4, v4)

    def init_seeded(self, circles: np.ndarray, rho: float, rho_radius: float, alpha: float) -> None:
        """Z from circles; X = N = M = Z_v(e); U = 0; RHOS = rho except the
        radius-factor edges (rho_radius); ALPHAS = alpha."""
        lib, G = self.lib, self.G
        lib.initialize_X_N_Z_M_U_zeros(C.byref(G))
        lib.initialize_RHOS_APHAS(C.byref(G), rho, alpha)
        e2v = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
        Z = G.arr("Z")
        Z[0::2, 0] = circles[:, 0]
        Z[0::2, 1] = circles[:, 1]
        Z[1::2, 0] = circles[:, 2]
        Z[1::2, 1] = circles[:, 2]
        for k in ("X", "N", "M"):
            G.arr(k)[:] = Z[e2v]
        G.arr("U")[:] = 0.0
        rh = G.arr("RHOS")
        o2n = np.ctypeslib.as_array(G.operatorix_to_numedges, shape=(G.num_opts,))
        fps = np.ctypeslib.as_array(C.cast(G.list_of_operators_functions_pointers, C.POINTER(C.c_uint64)),
                                    shape=(G.num_opts,))
        first_edge = np.concatenate([[0], np.cumsum(o2n)[:-1]])
        rad_ops = {op_ptr(OP_NAMES[2], lib)} | set(self._extra_radius_ops)
        is_rad = np.isin(fps, np.array(sorted(rad_ops), dtype=np.uint64))
        for f in np.nonzero(is_rad)[0]:
            rh[first_edge[f]:first_edge[f] + o2n[f]] = rho_radius

    def close(self) -> None:
        if self.G.num_edges or self.G.num_opts:
            self.lib.closeG(C.byref(self.G))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Handle:
    """Owns a paradmm_gpu handle."""

    def __init__(self, ptr: int, lib=None):
        self.lib = lib or load()
        self.ptr = C.c_void_p(ptr)

    @classmethod
    def from_graph(cls, G: Graph, **kw) -> "Handle":
        lib = load()
        p = C.c_void_p()
        o = opts(**kw)
        check(lib.paradmm_gpu_create(C.byref(G), C.byref(o), C.byref(p)))
        return cls(p.value, lib)

    @staticmethod
    def _descs(descs: list[dict]):
        arr = (PackingDesc * len(descs))()
        keep = []
        for i, d in enumerate(descs):
            walls = np.ascontiguousarray(d["walls"], dtype=np.float64)
            init = np.ascontiguousarray(d["init"], dtype=np.float64)
            keep += [walls, init]
            arr[i].n_circles = int(d["n_circles"])
            arr[i].n_walls = int(walls.shape[0])
            arr[i].walls = walls.ctypes.data_as(C.POINTER(C.c_double))
            arr[i].exponent = float(d.get("exponent", 2.0))
            arr[i].rho = float(d["rho"])
            arr[i].rho_radius = float(d["rho_radius"])
            arr[i].alpha = float(d["alpha"])
            arr[i].init = init.ctypes.data_as(C.POINTER(C.c_double))
        return arr, keep

    @classmethod
    def packing_tuned(cls, descs: list[dict], sweeps: int, tol: float = -1.0, **kw) -> tuple["Handle", dict]:
        """paradmm_gpu_create_packing_tuned: tile side and schedule from probes."""
        lib = load()
        arr, keep = cls._descs(descs)
        p = C.c_void_p()
        o = opts(**kw)
        t = Tuning()
        check(lib.paradmm_gpu_create_packing_tuned(arr, len(descs), C.byref(o), int(sweeps), float(tol), C.byref(p),
                                                   C.byref(t)))
        return cls(p.value, lib), {k: getattr(t, k) for k, _ in Tuning._fields_ if k != "reserved"}

    @classmethod
    def packing(cls, descs: list[dict], **kw) -> "Handle":
        """descs: dicts with n_circles, walls (k x 4), exponent, rho, rho_radius, alpha, init (N x 3)."""
        lib = load()
        arr, keep = cls._descs(descs)  # keep: the arrays arr points into, alive until the call returns
        p = C.c_void_p()
        o = opts(**kw)
        check(lib.paradmm_gpu_create_packing(arr, len(descs), C.byref(o), C.byref(p)))
        del keep
        return cls(p.value, lib)

    def iterate(self, n: int) -> None:
        check(self.lib.paradmm_gpu_iterate(self.ptr, n))

    def solve(self, maxiter: int, tol: float) -> dict:
        s = Stats()
        rc = self.lib.paradmm_gpu_solve(self.ptr, maxiter, tol, C.byref(s))
        if rc not in (OK, ENONFINITE):
            check(rc)
        return s.as_dict()

    def upload(self, G: Graph) -> None:
        check(self.lib.paradmm_gpu_upload(self.ptr, C.byref(G)))

    def download(self, G: Graph) -> None:
        check(self.lib.paradmm_gpu_download(self.ptr, C.byref(G)))

    def stats(self) -> dict:
        s = Stats()
        check(self.lib.paradmm_gpu_stats(self.ptr, C.byref(s)))
        return s.as_dict()

    def instances(self) -> int:
        return self.lib.paradmm_gpu_instances(self.ptr)

    def instance_stats(self) -> list[dict]:
        n = self.instances()
        arr = (Stats * n)()
        check(self.lib.paradmm_gpu_instance_stats(self.ptr, arr))
        return [a.as_dict() for a in arr]

    def circles(self, instance: int, n: int) -> np.ndarray:
        out = np.zeros((n, 3), dtype=np.float64)
        check(self.lib.paradmm_gpu_get_circles(self.ptr, instance, out.ctypes.data_as(C.POINTER(C.c_double))))
        return out

    def warm_start(self, instance: int, circles: np.ndarray, pair_duals: np.ndarray | None = None) -> None:
        c = np.ascontiguousarray(circles, dtype=np.float64)
        du = None if pair_duals is None else np.ascontiguousarray(pair_duals, dtype=np.float32)
        check(self.lib.paradmm_gpu_warm_start(self.ptr, instance, c.ctypes.data_as(C.POINTER(C.c_double)),
                                              None if du is None else du.ctypes.data_as(C.POINTER(C.c_float))))

    def warm_start_duals(self, instance: int, circles: np.ndarray, pair_duals=None, wall_duals=None,
                         radius_duals=None, dual_iters: int = 0) -> None:
        """paradmm_gpu_warm_start_duals: Z = circles, X = Z, U from the given
        duals (None = 0), then dual_iters rounds of the reference's
        optimal-initialisation map."""
        def p(a):
            if a is None:
                return None, None
            a = np.ascontiguousarray(a, dtype=np.float64)
            return a, a.ctypes.data_as(C.POINTER(C.c_double))
        keep = [p(circles), p(pair_duals), p(wall_duals), p(radius_duals)]
        check(self.lib.paradmm_gpu_warm_start_duals(self.ptr, instance, keep[0][1], keep[1][1], keep[2][1], keep[3][1],
                                                    int(dual_iters)))

    def engine(self) -> int:
        return self.lib.paradmm_gpu_engine(self.ptr)

    def device_bytes(self) -> int:
        return self.lib.paradmm_gpu_device_bytes(self.ptr)

    def instance_times(self) -> tuple[np.ndarray, np.ndarray]:
        """Per-instance schedule: (start_ms, stop_ms) of every instance in the last call."""
        n = self.instances()
        b = np.zeros(n)
        e = np.zeros(n)
        check(self.lib.paradmm_gpu_instance_times(self.ptr, b.ctypes.data_as(C.POINTER(C.c_double)),
                                                  e.ctypes.data_as(C.POINTER(C.c_double))))
        return b, e

    def launches(self) -> int:
        return self.lib.paradmm_gpu_launches(self.ptr)

    def set_tail_handoff(self, instances: int) -> None:
        """paradmm_gpu_set_tail_handoff: the last `instances` unfinished
        instances of a per-instance solve finish on the grid schedule."""
        check(self.lib.paradmm_gpu_set_tail_handoff(self.ptr, int(instances)))

    def tail_handoffs(self) -> int:
        return self.lib.paradmm_gpu_tail_handoffs(self.ptr)

    def set_profiling(self, on: bool) -> None:
        check(self.lib.paradmm_gpu_set_profiling(self.ptr, 1 if on else 0))

    def set_rho_balance(self, period: int, mu: float = 10.0, log2_min: int = -1, log2_max: int = 4) -> None:
        """paradmm_gpu_set_rho_balance: residual balancing of the penalties
        every `period` iterates (0: off)."""
        check(self.lib.paradmm_gpu_set_rho_balance(self.ptr, int(period), float(mu), int(log2_min), int(log2_max)))

    def rho_scale(self, instance: int = 0) -> int:
        """log2 of the penalty scale of the instance's next sweep."""
        v = C.c_int()
        check(self.lib.paradmm_gpu_rho_scale(self.ptr, int(instance), C.byref(v)))
        return v.value

    def set_fallback(self, after_sweeps: int) -> None:
        """Per-instance schedule: restart unconverged instances from their plain
        start after this many sweeps of a solve call (0: off)."""
        check(self.lib.paradmm_gpu_set_fallback(self.ptr, int(after_sweeps)))

    def autotune(self, sweeps: int = 100, tol: float = -1.0) -> dict:
        """Times the schedule candidates on a probe solve(sweeps, tol), keeps
        the fastest (state unchanged).  Returns the chosen configuration."""
        t = Tuning()
        check(self.lib.paradmm_gpu_autotune(self.ptr, int(sweeps), float(tol), C.byref(t)))
        return {k: getattr(t, k) for k, _ in Tuning._fields_ if k != "reserved"}

    def instance_fallbacks(self) -> np.ndarray:
        """1 for every instance that fell back to its plain start in the last call."""
        out = np.zeros(self.instances(), dtype=np.int32)
        check(self.lib.paradmm_gpu_instance_fallbacks(self.ptr, out.ctypes.data_as(C.POINTER(C.c_int))))
        return out

    def phase_times(self) -> list[float]:
        """Mean block time per sweep (us): pass, barrier 1, finalise, barrier 2
        (per-instance schedule: pass, barrier, consensus, barrier + stop test)."""
        out = (C.c_double * 4)()
        check(self.lib.paradmm_gpu_phase_times(self.ptr, out))
        return list(out)

    def close(self) -> None:
        if self.ptr and self.ptr.value:
            self.lib.paradmm_gpu_destroy(self.ptr)
            self.ptr = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
