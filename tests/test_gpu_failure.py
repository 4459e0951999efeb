"""Failure detection on the device without a GPU fault: a grid barrier that
one block never reaches runs out its (short) wait limit, the kernel records
the error and returns, the host reports PARADMM_ETIMEOUT, and the device
keeps working."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_barrier_wait_runs_out_and_device_stays_usable():
    import engine_b200 as eb
    lib = eb.load()
    t = time.perf_counter()
    rc = lib.paradmm_gpu_selftest_barrier_timeout(0, 200)
    dt = time.perf_counter() - t
    assert rc == eb.ETIMEOUT, (rc, lib.paradmm_last_error_string())
    assert b"ran out" in lib.paradmm_last_error_string()
    assert dt < 5.0
    # the context is intact: a small solve on the same device still works
    desc = dict(n_circles=30, walls=eb.box_walls(1.0, 1.0), exponent=2.0, rho=10.0, rho_radius=5.0, alpha=1.0,
                init=eb.seeded_circles(30, 1.0, 1.0, 0.05, 9))
    h = eb.Handle.packing([desc])
    s = h.solve(50, -1.0)
    assert s["iterations"] == 50
    c = h.circles(0, 30)
    assert np.all(np.isfinite(c))
    h.close()


def test_selftest_rejects_bad_arguments():
    import engine_b200 as eb
    lib = eb.load()
    assert lib.paradmm_gpu_selftest_barrier_timeout(0, 0) == eb.EINVAL
    assert lib.paradmm_gpu_selftest_barrier_timeout(-1, 100) == eb.ENODEVICE
