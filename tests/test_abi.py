"""C-ABI surface (CPU): the library loads without a GPU, exports every
function include/meu.h declares, and the ctypes mirrors of meu_params /
meu_diag have the C layout."""
import ctypes as C
import os
import subprocess
import tempfile

from meumapps_ss_b200 import _lib
from meumapps_ss_b200 import params as P

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_header_symbols():
    L = _lib.lib()
    names = _lib.header_functions()
    assert "meu_run" in names and "meu_create" in names
    for n in names:
        assert hasattr(L, n), n


def _c_layout(struct, fields):
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"meu.h\"\nint main(){\n"
    src += f'printf("%zu\\n", sizeof({struct}));\n'
    for f in fields:
        src += f'printf("%zu\\n", offsetof({struct}, {f}));\n'
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        cfile, exe = os.path.join(d, "t.c"), os.path.join(d, "t")
        open(cfile, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), cfile, "-o", exe], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    return [int(x) for x in out]


def test_struct_layouts_match_c():
    for cls, cname in ((P.MeuParams, "meu_params"), (P.MeuDiag, "meu_diag"), (_lib.Ran2State, "meu_ran2_state")):
        names = [f[0] for f in cls._fields_]
        got = _c_layout(cname, names)
        assert got[0] == C.sizeof(cls), cname
        for n, off in zip(names, got[1:]):
            assert getattr(cls, n).offset == off, (cname, n)


def test_bad_arguments_fail_without_gpu():
    L = _lib.lib()
    assert L.meu_run(None, 1, None) == 100
    assert L.meu_destroy(None) == 100
    assert L.meu_get_step(None) == -1


def test_ensemble_bad_arguments():
    L = _lib.lib()
    h = C.c_void_p()
    assert L.meu_ensemble_create(0, None, 0, C.byref(h)) == 100  # MEU_ERR_BADARG
    assert L.meu_ensemble_run(None, 1, None) == 100  # MEU_ERR_BADARG
    assert L.meu_ensemble_get_step(None) == -1
    assert L.meu_set_schedule(None, None) == 100  # MEU_ERR_BADARG


def test_transform_entry_points_validate_before_any_gpu_work():
    """Argument checks of the transform entry points run on the host before any
    device call, so they answer without a GPU (and never launch on bad input)."""
    import pytest
    import torch
    if torch.cuda.is_available():
        pytest.skip("host-only argument checks; the addresses below are not device memory")
    L = _lib.lib()
    buf = (C.c_double * 8)()
    assert L.meu_fft_roundtrip(16, 16, 16, 7, buf, buf, buf) == 100  # unknown precision
    assert L.meu_fft_roundtrip(16, 16, 16, P.PREC_F64, None, buf, buf) == 100
    assert L.meu_fft_roundtrip(14, 16, 16, P.PREC_F64, buf, buf, buf) == 103  # 7 is not 2^a 3^b
    # FP64 needs 16-byte aligned arrays, FP32 8-byte: an address 8 past a 16-byte boundary
    # is rejected in FP64; one 4 past an 8-byte boundary in FP32
    a16, off8, off4 = C.c_void_p(0x10000), C.c_void_p(0x10008), C.c_void_p(0x10004)
    assert L.meu_fft_roundtrip_noalloc(16, 16, 16, P.PREC_F64, off8, a16, a16) == 100
    assert b"16-byte aligned" in L.meu_last_error(None)
    assert L.meu_fft_roundtrip_noalloc(16, 16, 16, P.PREC_F64, a16, a16, off8) == 100
    assert L.meu_fft_roundtrip_noalloc(16, 16, 16, P.PREC_F32, a16, off4, a16) == 100
    assert b"8-byte aligned" in L.meu_last_error(None)
    assert L.meu_fft_roundtrip_noalloc(16, 16, 16, 7, a16, a16, a16) == 100
