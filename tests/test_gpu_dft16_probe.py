"""Is a tensor-core DFT stage worth it for the transforms?  A measurement, not a
product path: one radix-16 stage from and to shared memory, on the CUDA cores (the
butterfly the fused transforms run) and on the tensor pipe (the stage as a 32x32 real
GEMM in TF32 with the 3xTF32 split, mma.sync m16n8k8), over tiles held on chip
(tests/probes/dft16_probe.cu).  Checks both against an FP64 DFT and prints the time per
point of one pass of each."""
import ctypes as C
import json
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "probes", "dft16_probe.cu")
OUT = os.path.join(HERE, "probes", "_build", "libdft16probe.so")


def _lib():
    if not os.path.exists(OUT) or os.path.getmtime(OUT) < os.path.getmtime(SRC):
        os.makedirs(os.path.dirname(OUT), exist_ok=True)
        nvcc = "/usr/local/cuda/bin/nvcc"
        subprocess.run([nvcc, "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "-Xcompiler",
                        "-fPIC", "-shared", "--expt-relaxed-constexpr", SRC, "-o", OUT], check=True)
    L = C.CDLL(OUT)
    L.probe_dft16.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.POINTER(C.c_float)]
    return L


@pytest.mark.gpu
def test_dft16_stage_tensor_pipe_against_cuda_cores():
    import torch
    L = _lib()
    rng = np.random.default_rng(4)
    nb = 148 * 8
    x = (rng.standard_normal((nb, 16, 256)) + 1j * rng.standard_normal((nb, 16, 256))).astype(np.complex64)
    d_in = torch.from_numpy(x.view(np.float32)).cuda()
    d_out = torch.empty_like(d_in)
    ref = np.fft.fft(x.astype(np.complex128), axis=1) / 4
    res = {}
    for mode, name in ((0, "cuda_cores"), (1, "tensor_3xtf32")):
        ms = C.c_float()
        assert L.probe_dft16(mode, nb, 1, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), C.byref(ms)) == 0
        y = d_out.cpu().numpy().view(np.complex64)
        err = float(np.max(np.abs(y - ref)) / np.max(np.abs(ref)))
        reps = 400
        L.probe_dft16(mode, nb, 20, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()), C.byref(ms))
        assert L.probe_dft16(mode, nb, reps, C.c_void_p(d_in.data_ptr()), C.c_void_p(d_out.data_ptr()),
                             C.byref(ms)) == 0
        pts = nb * 16 * 256 * reps
        res[name] = {"max_rel_err_vs_fp64": err, "ms": ms.value, "ps_per_point_pass": ms.value * 1e9 / pts}
    print("DFT16_PROBE " + json.dumps(res))
    assert res["cuda_cores"]["max_rel_err_vs_fp64"] < 1e-6
    assert res["tensor_3xtf32"]["max_rel_err_vs_fp64"] < 1e-5
