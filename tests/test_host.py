"""Host-side tests (no GPU): the C-ABI library loads and exports every
declared symbol, graph construction reproduces the reference's structures,
the plain-C operators equal the reference's, and the engine reports errors
instead of failing when no device (or an unknown operator) is present."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("paradmm.h", "paradmm_gpu.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:MY_EXTERN_C\s+)?(?:const\s+)?[A-Za-z_][\w]*[\s\*]+\**\s*([A-Za-z_]\w*)\s*\(",
                             text, flags=re.M):
            if m.group(1) not in ("typedef", "return", "if", "while", "for", "sizeof", "void"):
                names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_function():
    lib = eb.load()
    names = declared_functions()
    assert "paradmm_gpu_create" in names and "updateGOpenMP" in names and "addNode" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def topo(G):
    d = dict(num=(G.num_opts, G.num_vars, G.num_dims, G.num_edges))
    d["o2n"] = [G.operatorix_to_numedges[f] for f in range(G.num_opts)]
    d["o2e"] = [[G.operatorix_to_edgelistix[f][k] for k in range(G.operatorix_to_numedges[f])]
                for f in range(G.num_opts)]
    d["v2n"] = [G.varix_to_numedges[v] for v in range(G.num_vars)]
    d["v2e"] = [[G.varix_to_edgelistix[v][k] for k in range(G.varix_to_numedges[v])] for v in range(G.num_vars)]
    d["e2v"] = [G.edgeix_to_varlistix[e] for e in range(G.num_edges)]
    return d


@pytest.mark.parametrize("order", [0, 1])
def test_construction_matches_reference(order):
    """addNode (called per factor) and the bulk builder both produce the
    reference's topology arrays."""
    ref = oracle_lib.best()
    N = 15
    walls = eb.box_walls(1.0, 1.0)
    orc = oracle_lib.OraclePacking(ref, N, walls, 2.0, order=order)
    lib = eb.load()
    ops = tuple(eb.op_ptr(n, lib) for n in eb.OP_NAMES)
    per_factor = eb.PackingGraph(N, walls, 2.0, order=order, ops=ops)
    bulk = eb.PackingGraph(N, walls, 2.0, order=order)
    t_ref = topo(orc.G)
    assert topo(per_factor.G) == t_ref
    assert topo(bulk.G) == t_ref


def test_addnode_sorts_and_grows():
    lib = eb.load()
    G = eb.Graph()
    lib.startG(C.byref(G), 2)
    pair = eb.op_ptr(eb.OP_NAMES[0], lib)
    rng = np.random.default_rng(1)
    for f in range(3000):
        v = rng.choice(500, size=4, replace=False).astype(np.int32)
        arr = (C.c_int * 4)(*v)
        lib.addNode(C.byref(G), pair, None, 4, arr)
        assert list(arr) == sorted(v)
    assert G.num_edges == 12000 and G.num_opts == 3000
    e2v = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
    for v in range(0, G.num_vars, 37):
        edges = [G.varix_to_edgelistix[v][k] for k in range(G.varix_to_numedges[v])]
        assert edges == sorted(edges) and all(e2v[e] == v for e in edges)
    lib.closeG(C.byref(G))
    lib.closeG(C.byref(G))  # a second close is harmless


@pytest.mark.parametrize("name", eb.OP_NAMES)
def test_host_operators_bit_identical_to_reference(name):
    ref = oracle_lib.best()
    lib = eb.load()
    f_ref = getattr(ref, name)
    f_me = getattr(lib, name)
    f_me.argtypes = [C.POINTER(C.c_double)] * 3 + [C.c_int, C.c_int, C.c_void_p]
    rng = np.random.default_rng(abs(hash(name)) % 2**32)
    nv = {eb.OP_NAMES[0]: 4, eb.OP_NAMES[1]: 2, eb.OP_NAMES[2]: 3}[name]
    P = C.POINTER(C.c_double)
    for trial in range(3000):
        n = rng.uniform(-0.5, 1.5, size=2 * nv)
        if trial % 3 == 0:  # radius dims equal
            for e in range(nv):
                n[2 * e + 1] = n[2 * e]
        rh = rng.uniform(0.5, 20, size=nv)
        params = np.array([2.0]) if name == eb.OP_NAMES[2] else rng.uniform(-1, 1, size=4)
        if trial % 7 == 0 and name == eb.OP_NAMES[2]:
            params = np.array([rng.choice([1.0, 2.0, 3.0])])
        xa = np.zeros(2 * nv)
        xb = np.zeros(2 * nv)
        f_ref(xa.ctypes.data_as(P), n.copy().ctypes.data_as(P), rh.copy().ctypes.data_as(P), nv, 2,
              params.ctypes.data)
        f_me(xb.ctypes.data_as(P), n.copy().ctypes.data_as(P), rh.copy().ctypes.data_as(P), nv, 2,
             params.ctypes.data)
        assert np.array_equal(xa, xb, equal_nan=True)


def test_seeded_init_matches_harness():
    N = 25
    walls = eb.box_walls(2.0, 1.0)
    pg = eb.PackingGraph(N, walls, 2.0)
    circles = eb.seeded_circles(N, 2.0, 1.0, 0.01, 77)
    pg.init_seeded(circles, 10.0, 5.0, 1.0)
    orc = oracle_lib.OraclePacking(oracle_lib.best(), N, walls, 2.0)
    orc.init(77, 2.0, 1.0, 0.01, 10.0, 5.0, 1.0)
    a, b = pg.G.state(), orc.state()
    for k in a:
        assert np.array_equal(a[k], b[k]), k
    assert np.array_equal(pg.G.arr("RHOS"), orc.G.arr("RHOS"))
    assert np.array_equal(pg.G.arr("ALPHAS"), orc.G.arr("ALPHAS"))


def test_initialize_optimal_matches_reference():
    ref = oracle_lib.best()
    N = 8
    walls = eb.box_walls(1.0, 1.0)
    orc = oracle_lib.OraclePacking(ref, N, walls, 2.0)
    pg = eb.PackingGraph(N, walls, 2.0)
    rng = np.random.default_rng(5)
    Gr, Gm = orc.G, pg.G
    ref.initialize_RHOS_APHAS(orc.graph_ptr(), 10.0, 1.0)
    lib = eb.load()
    lib.initialize_RHOS_APHAS(C.byref(Gm), 10.0, 1.0)
    Z = rng.uniform(0, 1, size=Gm.num_vars * 2)
    U = rng.uniform(-0.1, 0.1, size=Gm.num_edges * 2)
    P = C.POINTER(C.c_double)
    ref.initialize_X_N_Z_M_U_optimal.argtypes = [C.POINTER(eb.Graph), P, P, C.c_int]
    ref.initialize_X_N_Z_M_U_optimal(orc.graph_ptr(), Z.ctypes.data_as(P), U.ctypes.data_as(P), 3)
    lib.initialize_X_N_Z_M_U_optimal(C.byref(Gm), Z.ctypes.data_as(P), U.ctypes.data_as(P), 3)
    a, b = Gm.state(), Gr.state()
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_unknown_operator_is_rejected_before_any_device_work():
    lib = eb.load()
    cb = eb.OP_FN(lambda x, n, r, nv, nd, p: None)
    G = eb.Graph()
    lib.startG(C.byref(G), 2)
    v = (C.c_int * 2)(0, 1)
    lib.addNode(C.byref(G), C.cast(cb, C.c_void_p), None, 2, v)
    lib.initialize_RHOS_APHAS(C.byref(G), 1.0, 1.0)
    lib.initialize_X_N_Z_M_U_zeros(C.byref(G))
    h = C.c_void_p()
    rc = lib.paradmm_gpu_create(C.byref(G), None, C.byref(h))
    assert rc == eb.EUNSUPPORTED_OP
    assert "not one of the packing operators" in eb.last_error()
    lib.updateG(C.byref(G))
    assert eb.last_status() == eb.EUNSUPPORTED_OP
    lib.closeG(C.byref(G))


def test_registered_operator_is_recognised():
    """A caller's own copy of an operator, registered by kind."""
    lib = eb.load()
    ref = oracle_lib.best()
    assert lib.paradmm_gpu_register_op(C.cast(ref.disk_collision_variable_radius, C.c_void_p), eb.OP_PAIR) == eb.OK
    assert lib.paradmm_gpu_register_op(None, eb.OP_PAIR) == eb.EINVAL
    assert lib.paradmm_gpu_register_op(C.cast(ref.disk_collision_variable_radius, C.c_void_p), 9) == eb.EINVAL


@pytest.mark.skipif(_has_gpu(), reason="checks the no-device path")
def test_no_device_reports_enodevice():
    lib = eb.load()
    pg = eb.PackingGraph(6, eb.box_walls(1, 1), 2.0)
    pg.init_seeded(eb.seeded_circles(6, 1, 1, 0.05, 1), 10, 5, 1)
    h = C.c_void_p()
    rc = lib.paradmm_gpu_create(C.byref(pg.G), None, C.byref(h))
    assert rc == eb.ENODEVICE, eb.last_error()
    before = pg.G.state()
    lib.updateG(C.byref(pg.G))
    assert eb.last_status() == eb.ENODEVICE
    after = pg.G.state()
    for k in before:
        assert np.array_equal(before[k], after[k])  # graph untouched on failure


def test_packing_desc_validation():
    lib = eb.load()
    h = C.c_void_p()
    assert lib.paradmm_gpu_create_packing(None, 1, None, C.byref(h)) == eb.EINVAL
    d = (eb.PackingDesc * 1)()
    d[0].n_circles = 1
    assert lib.paradmm_gpu_create_packing(d, 1, None, C.byref(h)) == eb.EINVAL


def test_fused_shard_and_tail_handoff_arguments_are_checked_without_a_device():
    """The fused shard run, its buffers, the IPC helpers and the tail
    hand-off validate their arguments before any device work."""
    lib = eb.load()
    vp = C.c_void_p
    assert lib.paradmm_gpu_shard_run_fused(None, 1, None, None, 0, None) == eb.EINVAL
    hs = (vp * 1)()
    assert lib.paradmm_gpu_shard_run_fused(hs, 0, None, None, 0, None) == eb.EINVAL  # nlocal < 1
    assert lib.paradmm_gpu_shard_run_fused(hs, 9, None, None, 0, None) == eb.EINVAL  # more than 8 ranks
    assert lib.paradmm_gpu_shard_run_fused(hs, 1, None, None, 0, None) == eb.EINVAL  # no buffers
    ex, fl = vp(), vp()
    assert lib.paradmm_gpu_shard_fused_buffers(None, C.byref(ex), C.byref(fl)) == eb.EINVAL
    assert lib.paradmm_gpu_ipc_export(None, C.create_string_buffer(64)) == eb.EINVAL
    assert lib.paradmm_gpu_ipc_import(0, None, C.byref(ex)) == eb.EINVAL
    assert lib.paradmm_gpu_set_tail_handoff(None, 8) == eb.EINVAL
    assert lib.paradmm_gpu_tail_handoffs(None) == 0
