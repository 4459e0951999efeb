"""The allocation-free entry point, paradmm_gpu_packing_iterate_noalloc.

It exists for callers that may not allocate device memory while they run
(services that reserve their device memory up front, latency-critical loops
where cudaMalloc/cudaFree could synchronise the device).  The test plays such
a caller: it owns the circle and edge-state buffers (allocated here through
torch, i.e. by the caller, not by the library), calls the entry point twice in
a row through the C-ABI, and checks each result against the handle API
(paradmm_gpu_create_packing + paradmm_gpu_iterate) on the same problem.
The file is named to be collected last; it also passes on its own in a fresh
process.
"""
import ctypes as C

import numpy as np
import pytest

import engine_b200 as eb

pytestmark = pytest.mark.gpu

TOL_F32 = 1e-4


def _desc(N, walls, circles):
    d = eb.PackingDesc()
    d.n_circles = N
    d.n_walls = len(walls)
    d.walls = walls.ctypes.data_as(C.POINTER(C.c_double))
    d.exponent = 2.0
    d.rho = 10.0
    d.rho_radius = 5.0
    d.alpha = 1.0
    d.init = circles.ctypes.data_as(C.POINTER(C.c_double))
    return d


@pytest.mark.parametrize("N", [300, 301])  # odd N: the state's FP32 circles still start 16-byte aligned
def test_noalloc_matches_handle_api_on_two_calls(N):
    import torch

    lib = eb.load()
    walls = np.ascontiguousarray(eb.box_walls(1.5, 1.0))
    circles = eb.seeded_circles(N, 1.5, 1.0, 0.05, 42)
    desc = _desc(N, walls, circles)

    nbytes = lib.paradmm_noalloc_state_bytes(N, len(walls))
    assert nbytes > 0
    d_circles = torch.from_numpy(circles.copy()).to("cuda:0")
    d_state = torch.empty(nbytes, dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()

    ref = eb.Handle.packing([dict(n_circles=N, walls=walls, exponent=2.0, rho=10.0, rho_radius=5.0, alpha=1.0,
                                  init=circles)], device=0, block_width=64)
    for call, init in ((1, 1), (2, 0)):
        st = eb.Stats()
        rc = lib.paradmm_gpu_packing_iterate_noalloc(C.byref(desc), C.c_void_p(d_circles.data_ptr()),
                                                     C.c_void_p(d_state.data_ptr()), init, 60, -1.0, C.byref(st),
                                                     0, None)
        assert rc == eb.OK, eb.last_error()
        assert st.iterations == 60
        ref.iterate(60)
        got = d_circles.cpu().numpy()
        want = ref.circles(0, N)
        d = float(np.max(np.abs(got - want)))
        assert d <= TOL_F32, f"call {call}: max |diff| vs handle API = {d}"
        assert np.isfinite(st.primal) and np.isfinite(st.dual)
    ref.close()


def test_noalloc_rejects_sizes_beyond_its_limit():
    lib = eb.load()
    N = 600  # above PARADMM_NOALLOC_MAX_CIRCLES (512)
    walls = np.ascontiguousarray(eb.box_walls(1.0, 1.0))
    circles = eb.seeded_circles(N, 1.0, 1.0, 0.05, 1)
    desc = _desc(N, walls, circles)
    assert lib.paradmm_noalloc_state_bytes(N, 4) == -1
    rc = lib.paradmm_gpu_packing_iterate_noalloc(C.byref(desc), C.c_void_p(8), C.c_void_p(8), 1, 1, -1.0, None, 0,
                                                 None)
    assert rc == eb.EINVAL
    assert "limit of the fixed scratch" in eb.last_error()


def test_noalloc_refuses_a_buffer_it_never_initialised():
    """A caller that passes a zero-filled state buffer with init_state = 0
    (forgetting the first, initialising call) gets PARADMM_EINVAL instead of
    sweeps from an all-zero edge state."""
    import torch

    lib = eb.load()
    N = 100
    walls = np.ascontiguousarray(eb.box_walls(1.0, 1.0))
    circles = eb.seeded_circles(N, 1.0, 1.0, 0.05, 4)
    desc = _desc(N, walls, circles)
    d_circles = torch.from_numpy(circles.copy()).to("cuda:0")
    d_state = torch.zeros(lib.paradmm_noalloc_state_bytes(N, len(walls)), dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    rc = lib.paradmm_gpu_packing_iterate_noalloc(C.byref(desc), C.c_void_p(d_circles.data_ptr()),
                                                 C.c_void_p(d_state.data_ptr()), 0, 5, -1.0, None, 0, None)
    assert rc == eb.EINVAL and "never initialised" in eb.last_error()
    assert np.array_equal(d_circles.cpu().numpy(), circles)  # nothing ran


def test_noalloc_early_stop_then_continue():
    """tol >= 0: the call stops at the tolerance like the handle API's solve,
    and a following init_state = 0 call resumes from the state it left."""
    import torch

    lib = eb.load()
    N = 120
    walls = np.ascontiguousarray(eb.box_walls(1.0, 1.0))
    circles = eb.seeded_circles(N, 1.0, 1.0, 0.05, 8)
    desc = _desc(N, walls, circles)
    d_circles = torch.from_numpy(circles.copy()).to("cuda:0")
    d_state = torch.empty(lib.paradmm_noalloc_state_bytes(N, len(walls)), dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    ref = eb.Handle.packing([dict(n_circles=N, walls=walls, exponent=2.0, rho=10.0, rho_radius=5.0, alpha=1.0,
                                  init=circles)], device=0, block_width=64)
    st = eb.Stats()
    rc = lib.paradmm_gpu_packing_iterate_noalloc(C.byref(desc), C.c_void_p(d_circles.data_ptr()),
                                                 C.c_void_p(d_state.data_ptr()), 1, 20000, 1e-4, C.byref(st), 0, None)
    assert rc == eb.OK, eb.last_error()
    want = ref.solve(20000, 1e-4)
    assert st.converged == 1 and 0 < st.iterations < 20000
    assert st.iterations == want["iterations"]
    assert float(np.max(np.abs(d_circles.cpu().numpy() - ref.circles(0, N)))) <= TOL_F32
    rc = lib.paradmm_gpu_packing_iterate_noalloc(C.byref(desc), C.c_void_p(d_circles.data_ptr()),
                                                 C.c_void_p(d_state.data_ptr()), 0, 40, -1.0, C.byref(st), 0, None)
    assert rc == eb.OK, eb.last_error()
    assert st.iterations == 40
    ref.iterate(40)
    assert float(np.max(np.abs(d_circles.cpu().numpy() - ref.circles(0, N)))) <= TOL_F32
    ref.close()
