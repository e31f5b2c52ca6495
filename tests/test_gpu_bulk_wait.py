"""The plane kernels load each M-form plane with one bulk copy (TMA engine) and wait on an
mbarrier for at most fz::BULK_WAIT_POLLS polls (csrc/fused.cuh).  A test-only kernel
(tests/probes/mbar_wait_probe.cu) runs the same copy and wait: once normally, once with
an mbarrier that expects bytes no copy delivers, where the wait must run out, record
MEU_ERR_TIMEOUT (105) and return, and the context must stay usable."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "probes", "mbar_wait_probe.cu")
OUT = os.path.join(HERE, "probes", "_build", "libmbarprobe.so")
POLLS = 1 << 18  # fz::BULK_WAIT_POLLS
DEPS = [SRC, os.path.join(HERE, "..", "meumapps_ss_b200", "csrc", "fused.cuh")]


def _lib():
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < max(os.path.getmtime(d) for d in DEPS):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        subprocess.run(["/usr/local/cuda/bin/nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
                        "-Xcompiler", "-fPIC", "-shared", "--expt-relaxed-constexpr", SRC, "-o", OUT], check=True)
    L = C.CDLL(OUT)
    L.probe_mbar.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_float)]
    return L


def test_probe_source_uses_the_product_wait():
    src = open(SRC).read()
    for name in ("fz::mbar_init1", "fz::bulk_load", "fz::mbar_wait"):
        assert name in src
    hdr = open(DEPS[1]).read()
    assert "constexpr int BULK_WAIT_POLLS = 1 << 18;" in hdr


@pytest.mark.gpu
def test_bulk_copy_wait_completes_and_runs_out():
    import torch
    L = _lib()
    n = 32 * 1024
    x = torch.arange(n // 4, dtype=torch.float32, device="cuda")
    y = torch.zeros_like(x)
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    ms = C.c_float()
    res = {}
    assert L.probe_mbar(0, POLLS, x.data_ptr(), y.data_ptr(), n, err.data_ptr(), C.byref(ms)) == 0
    assert int(err.item()) == 0 and torch.equal(x, y)
    res["copy_ms"] = ms.value
    assert L.probe_mbar(1, POLLS, x.data_ptr(), y.data_ptr(), n, err.data_ptr(), C.byref(ms)) == 0
    assert int(err.item()) == 105
    res["run_out_ms"] = ms.value
    assert ms.value < 20000.0
    # the context is still usable
    err.zero_()
    y.zero_()
    assert L.probe_mbar(0, POLLS, x.data_ptr(), y.data_ptr(), n, err.data_ptr(), C.byref(ms)) == 0
    assert int(err.item()) == 0 and torch.equal(x, y)
    print("MBAR_PROBE " + json.dumps(res))
