"""The drop-in from C: one host program written against paradmm.h only
(tests/c_host/host_demo.c), built once against the reference's own library
(compiled from its sources into oracle/_ref, or the oracle restatement) and
once against libparadmm_b200.so.  Both runs print the consensus after
updateGOpenMP; the engine (FP32 packing path) must agree within the FP32
parity tolerance over a few sweeps (the early phase is chaotic)."""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_host", "host_demo.c")


def _build(tmp, name, libdir, lib, extra=()):
    exe = os.path.join(tmp, name)
    cmd = ["gcc", "-O2", "-std=gnu11", *extra, "-I" + os.path.join(ROOT, "include"), SRC, "-o", exe,
           "-L" + libdir, "-l:" + lib, "-Wl,-rpath," + libdir, "-lm"]
    subprocess.run(cmd, check=True, capture_output=True)
    return exe


def test_same_c_host_against_reference_and_engine(tmp_path):
    oracle_lib.ensure_built()
    ref = oracle_lib.REF if os.path.exists(oracle_lib.REF) else oracle_lib.PORT
    exe_ref = _build(str(tmp_path), "host_ref", os.path.dirname(ref), os.path.basename(ref))
    exe_eng = _build(str(tmp_path), "host_eng", os.path.join(ROOT, "engine_b200"), "libparadmm_b200.so",
                     ("-DPARADMM_B200",))
    out = []
    for exe in (exe_ref, exe_eng):
        r = subprocess.run([exe, "60", "6"], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, r.stderr
        out.append(np.array([[float(x) for x in l.split()] for l in r.stdout.split("\n") if l.strip()]))
    assert out[0].shape == out[1].shape == (120, 2)
    assert np.max(np.abs(out[0] - out[1])) <= 1e-4
