"""The drop-in boundary from a compiled C caller: tests/c_caller/fftlib_caller.c
includes <fftlib.h>, is built with gcc against include/ and linked against
libfftlib_b200.so, and calls the reference's entry points in the reference
test drivers' order. Drift between the headers, the shared object and the
Python binding (struct layouts, enum values, prototypes) shows up here."""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "c_caller", "fftlib_caller.c")
LIBDIR = os.path.join(ROOT, "c7x_fftlib_b200")


@pytest.fixture(scope="module")
def caller(tmp_path_factory):
    if not shutil.which("gcc"):
        pytest.skip("gcc not available")
    F.lib()  # the shared object exists
    exe = str(tmp_path_factory.mktemp("c_caller") / "fftlib_caller")
    cmd = ["gcc", "-std=c99", "-D_POSIX_C_SOURCE=200112L", "-O1", "-Wall", "-Wextra", "-Werror", "-I",
           os.path.join(ROOT, "include"), SRC, "-o", exe, "-L", LIBDIR, "-lfftlib_b200", f"-Wl,-rpath,{LIBDIR}", "-lm"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
    return exe


def _lines(out):
    return [ln.split() for ln in out.strip().splitlines()]


def test_layout_matches_python_binding(caller):
    r = subprocess.run([caller, "layout"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    got = {k: int(v) for k, v in _lines(r.stdout)}
    assert got["sizeof_bufParams1D"] == C.sizeof(F.BufParams) == 8
    assert got["offset_bufParams1D_dim_x"] == F.BufParams.dim_x.offset
    assert got["sizeof_bufParams2D"] == C.sizeof(F.BufParams2D)
    assert got["sizeof_mma_initargs"] == C.sizeof(F.MmaInitArgs)
    assert got["offset_mma_fftSize"] == F.MmaInitArgs.fftSize.offset
    assert got["offset_mma_shiftVector"] == F.MmaInitArgs.shiftVector.offset
    assert got["sizeof_status"] == 4
    assert got["FFTLIB_FLOAT32"] == F.FFTLIB_FLOAT32 == 12
    assert got["FFTLIB_INT16"] == F.FFTLIB_INT16 == 1
    assert got["FFTLIB_UINT32"] == F.FFTLIB_UINT32 == 8
    assert got["FFTLIB_ERR_NULL_POINTER"] == 5
    assert got["FFTLIB_FUNCTION_OPTIMIZED"] == F.FFTLIB_FUNCTION_OPTIMIZED == 1
    assert got["PBLOCK_C2C"] >= 64 and got["PBLOCK_I16"] >= 64


# testNum: (optimized status, natural-C status for c2c, for ifft); the
# reference driver's coverage cases (..._d.c:370-534)
COVERAGE = {1000: (5, 5, 5), 1001: (5, 5, 5), 1002: (5, 5, 5), 1003: (5, 0, 0), 1004: (4, 4, 4), 1005: (4, 4, 4),
            1006: (3, 3, 3), 1007: (3, 3, 3), 1008: (3, 3, 3), 1009: (8, 0, 0), 1010: (4, 4, 6), 1011: (0, 0, 0)}


def test_checkparams_coverage_from_c(caller):
    r = subprocess.run([caller, "checkparams"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    seen = 0
    for kind, tc, so, sc in _lines(r.stdout):
        exp_opt, exp_cn, exp_cn_inv = COVERAGE[int(tc)]
        assert int(so) == exp_opt, (kind, tc)
        assert int(sc) == (exp_cn_inv if kind == "ifft" else exp_cn), (kind, tc)
        seen += 1
    assert seen == 24


def _load(d, name, dt):
    return np.fromfile(os.path.join(d, name), dtype=dt)


@pytest.mark.gpu
def test_c_caller_transforms(caller, tmp_path):
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    d = str(tmp_path)
    r = subprocess.run([caller, "run", d], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "failures 0" in r.stdout
    for kind, n, ch in (("c2c", 256, 16), ("c2c", 4096, 64), ("ifft", 960, 5), ("c2c", 31250, 2)):
        x = _load(d, f"{kind}_{n}_{ch}_in.f32", np.float32)
        y = _load(d, f"{kind}_{n}_{ch}_out.f32", np.float32)
        assert O.rel_l2(y, O.fp64_c2c(x, n, ch, kind == "ifft")) <= 2e-6, (kind, n, ch)
    n, ch = 4096, 8
    x = _load(d, "r2c_in.f32", np.float32)
    y = _load(d, "r2c_out.f32", np.float32)
    assert O.rel_l2(O.as_complex(y, n // 2 + 1, ch), O.fp64_r2c(x, n, ch, 0)) <= 2e-6
    z = _load(d, "c2r_out.f32", np.float32)
    assert O.rel_l2(z, O.fp64_c2r(y, n, ch, 0).ravel()) <= 2e-6
    xi = _load(d, "i16_in.i16", np.int16)
    np.testing.assert_array_equal(_load(d, "i16_out.i16", np.int16), O.fft_c2c_i16(xi, 1024, 32, [2] * 5))
    paths = {ln[0]: int(ln[2]) for ln in _lines(r.stdout) if len(ln) == 3 and ln[1] == "path"}
    assert paths["mma_f32_256"] == F.MMA_PATH_TC
    xf = _load(d, "mma_f32_256_in.bin", np.float32)
    yf = _load(d, "mma_f32_256_out.bin", np.float32)
    assert O.rel_l2(yf, O.fp64_c2c(xf, 256, 300)) <= 2e-6
    xm = _load(d, "mma_i16_32_in.bin", np.int16)
    ym = _load(d, "mma_i16_32_out.bin", np.int16)
    np.testing.assert_array_equal(ym, O.mma_exec(16, 32, 100, 1, [12, 0, 0, 0, 0], xm))
