"""Operators the engine does not know, given by the caller as device source
(paradmm_gpu_register_op_source): the drop-in updateG runs them on the GPU
(generic FP64 engine, the operators compiled at run time) and must match the
reference's own CPU updateG, which calls the host twins of the same
operators, on the same graph and state."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

import engine_b200 as eb
import oracle_lib

pytestmark = pytest.mark.gpu

# Two operators of a smoothing problem on 2-D points: a weighted pull of one
# variable toward a target (params: weight, target x, target y), and a
# coupling lam ||x0 - x1||^2 between two variables (params: lam).  Host and
# device bodies are the same statements in the same order.
BODY_PULL = """
    const double *p = (const double *)params;
    const double w = p[0];
    for (int k = 0; k < numdims; ++k) x[k] = (rhos[0] * n[k] + w * p[1 + k]) / (rhos[0] + w);
"""
BODY_COUPLE = """
    const double L = 2.0 * ((const double *)params)[0];
    const double a = rhos[0], b = rhos[1];
    const double det = a * b + L * (a + b);
    for (int k = 0; k < numdims; ++k) {
        const double n0 = n[k], n1 = n[numdims + k];
        x[k] = (a * n0 * (b + L) + L * b * n1) / det;
        x[numdims + k] = (b * n1 * (a + L) + L * a * n0) / det;
    }
"""
SIG = "(double *x, double *n, double *rhos, int numvars, int numdims, void *params)"
HOST_SRC = f"void pull{SIG} {{{BODY_PULL}}}\nvoid couple{SIG} {{{BODY_COUPLE}}}\n"
DEV_PULL = f"__device__ void dev_pull{SIG} {{{BODY_PULL}}}"
DEV_COUPLE = f"__device__ void dev_couple{SIG} {{{BODY_COUPLE}}}"


@pytest.fixture(scope="module")
def host_ops(tmp_path_factory):
    d = tmp_path_factory.mktemp("userops")
    src, so = os.path.join(d, "ops.c"), os.path.join(d, "libops.so")
    open(src, "w").write(HOST_SRC)
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-shared", "-fPIC", src, "-o", so], check=True)
    lib = C.CDLL(so)
    return C.cast(lib.pull, C.c_void_p).value, C.cast(lib.couple, C.c_void_p).value, lib


def _bind(L):
    L.startG.argtypes = [C.POINTER(eb.Graph), C.c_int]
    L.addNodeWithParamSize.argtypes = [C.POINTER(eb.Graph), C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int)]
    L.initialize_RHOS_APHAS.argtypes = [C.POINTER(eb.Graph), C.c_double, C.c_double]
    for n in ("updateG", "initialize_X_N_Z_M_U_zeros", "closeG"):
        getattr(L, n).argtypes = [C.POINTER(eb.Graph)]
        getattr(L, n).restype = None
    return L


def _build(L, pull, couple, nvar, pairs, targets, keep):
    G = eb.Graph()
    L.startG(C.byref(G), 2)
    for v in range(nvar):
        p = np.array([1.0 + 0.1 * (v % 7), targets[v, 0], targets[v, 1]])
        keep.append(p)
        vi = (C.c_int * 1)(v)
        keep.append(vi)
        L.addNodeWithParamSize(C.byref(G), pull, p.ctypes.data, p.nbytes, 1, vi)
    for (a, b), lam in pairs:
        p = np.array([lam])
        keep.append(p)
        vi = (C.c_int * 2)(a, b)
        keep.append(vi)
        L.addNodeWithParamSize(C.byref(G), couple, p.ctypes.data, p.nbytes, 2, vi)
    L.initialize_RHOS_APHAS(C.byref(G), 3.0, 1.0)
    L.initialize_X_N_Z_M_U_zeros(C.byref(G))
    return G


def test_user_operators_match_reference_updateG(host_ops):
    pull, couple, _ = host_ops
    lib = eb.load()
    assert lib.paradmm_gpu_register_op_source(pull, DEV_PULL.encode(), b"dev_pull") == eb.OK
    assert lib.paradmm_gpu_register_op_source(couple, DEV_COUPLE.encode(), b"dev_couple") == eb.OK
    rng = np.random.default_rng(9)
    nvar = 300
    targets = rng.uniform(-1, 1, (nvar, 2))
    pairs = [((int(a), int(b)), float(rng.uniform(0.1, 2.0)))
             for a, b in rng.integers(0, nvar, (900, 2)) if a < b]
    keep = []
    ref = _bind(oracle_lib.best())
    Ge = _build(_bind(lib), pull, couple, nvar, pairs, targets, keep)
    Gr = _build(ref, pull, couple, nvar, pairs, targets, keep)
    z0 = rng.uniform(-1, 1, (nvar, 2))
    for G in (Ge, Gr):
        G.arr("Z")[:] = z0
        e2v = np.ctypeslib.as_array(G.edgeix_to_varlistix, shape=(G.num_edges,))
        for k in ("X", "N", "M"):
            G.arr(k)[:] = z0[e2v]
        G.arr("U")[:] = 0.0
    for _ in range(40):
        lib.updateG(C.byref(Ge))
        assert lib.paradmm_last_status() == eb.OK, lib.paradmm_last_error_string()
        ref.updateG(C.byref(Gr))
    se, sr = Ge.state(), Gr.state()
    for k in ("X", "M", "N", "U", "Z"):
        assert np.max(np.abs(se[k] - sr[k])) <= 1e-12, k
    lib.closeG(C.byref(Ge))
    ref.closeG(C.byref(Gr))


def test_operator_source_errors(host_ops):
    pull, _, _ = host_ops
    lib = eb.load()
    bad = b"__device__ void broken(double *x) { this is not C++ }"
    assert lib.paradmm_gpu_register_op_source(pull, bad, b"broken") == eb.OK  # compiled when a graph needs it
    keep = []
    G = _build(_bind(lib), pull, pull, 4, [], np.zeros((4, 2)), keep)
    h = C.c_void_p()
    o = eb.opts()
    rc = lib.paradmm_gpu_create(C.byref(G), C.byref(o), C.byref(h))
    assert rc == eb.EINVAL
    assert b"does not compile" in lib.paradmm_last_error_string()
    assert lib.paradmm_gpu_register_op_source(pull, DEV_PULL.encode(), b"not an id") == eb.EINVAL
    lib.paradmm_gpu_register_op_source(pull, DEV_PULL.encode(), b"dev_pull")  # leave it valid
    lib.closeG(C.byref(G))
