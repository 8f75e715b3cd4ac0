"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, the ctypes struct matches the C struct byte for byte, and
argument validation fails with status codes instead of crashing."""
import ctypes
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from diablo3_test_b200 import _lib
from diablo3_test_b200.config import ChannelParams, CParams

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "diablo_gpu.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(diablo_[a-z0-9_]+)\s*\(", src)))


def test_header_declares_what_the_binding_binds():
    assert declared_functions() == sorted(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert lib.diablo_abi_version() == 1


def test_status_strings():
    lib = _lib.load()
    for code in range(-8, 1):
        assert lib.diablo_status_string(code)


def test_struct_layout_matches_c():
    fields = [f[0] for f in CParams._fields_]
    prog = ["#include <stdio.h>", "#include <stddef.h>", '#include "diablo_gpu.h"', "int main(void){",
            'printf("size %zu\\n", sizeof(diablo_params));']
    for f in fields:
        prog.append(f'printf("{f} %zu\\n", offsetof(diablo_params, {f}));')
    prog.append("return 0;}")
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write("\n".join(prog))
        subprocess.check_call(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe])
        out = subprocess.check_output([exe]).decode().split("\n")
    got = dict(line.split() for line in out if line)
    assert int(got["size"]) == ctypes.sizeof(CParams)
    for f in fields:
        assert int(got[f]) == getattr(CParams, f).offset, f


def _create(p, gy=None):
    lib = _lib.load()
    c = p.to_c()
    st = ctypes.c_int(123)
    if gy is None:
        gy = np.linspace(-1, 1, p.ny + 1)
    ctx = lib.diablo_create(ctypes.byref(c), gy.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st))
    return ctx, st.value, c


def test_create_rejects_bad_arguments_before_touching_the_device():
    lib = _lib.load()
    p = ChannelParams.with_scalars(1, nx=32, ny=33, nz=24)
    c = p.to_c()
    c.struct_size = 4
    st = ctypes.c_int(0)
    gy = np.linspace(-1, 1, 34)
    assert not lib.diablo_create(ctypes.byref(c), gy.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st))
    assert st.value == _lib.ERR_ARG
    for bad in (dict(nz=20), dict(nx=34), dict(nx=1024)):
        kw = dict(nx=32, ny=33, nz=24)
        kw.update(bad)
        ctx, st, _ = _create(ChannelParams.with_scalars(1, **kw))
        assert not ctx and st == _lib.ERR_SIZE, bad
    ctx, st, _ = _create(ChannelParams.with_scalars(1, nx=32, ny=33, nz=24, re=-1.0))
    assert not ctx and st == _lib.ERR_ARG
    assert lib.diablo_create(None, None, None) is None


def test_null_context_calls_return_arg_error():
    lib = _lib.load()
    assert lib.diablo_step(None, 1) == _lib.ERR_ARG
    assert lib.diablo_rk_substep(None, 1) == _lib.ERR_ARG
    assert lib.diablo_destroy(None) == _lib.ERR_ARG
    assert lib.diablo_kernel_launches(None) == -1


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    ctx, st, _ = _create(ChannelParams.with_scalars(1, nx=32, ny=33, nz=24))
    assert not ctx and st in (_lib.ERR_CUDA, _lib.ERR_NOMEM)
