"""Host-side behaviour of the fft_c7xmma coordinator API (no GPU needed):
buffer sizes, parameter checks with the reference's status codes, and the
FP32 computational matrix generated in FP64."""
import ctypes as C

import numpy as np
import pytest

import c7x_fftlib_b200 as F

M = "FFTLIB_FFT_fft_ixX_cxX_oxX_"


def _sizes(n, batch, style=F.FFTLIB_FUNCTION_OPTIMIZED, interleave=1, dtype=F.FFTLIB_FLOAT32):
    a = F.MmaInitArgs(style, n, batch, interleave)
    bx, bw, by = F.BufParams(dtype, 0), F.BufParams(dtype, 0), F.BufParams(dtype, 0)
    st = getattr(F.lib(), M + "getSizes")(C.byref(a), bx, bw, by)
    return st, bx.dim_x, bw.dim_x, by.dim_x


@pytest.mark.parametrize("n,wsize", [(8, 256), (64, 128 * 128), (128, 32 * 32 + 16 * 16 + 256),
                                     (4096, 2 * 128 * 128 + 8192)])
def test_sizes_tensor_core_path(n, wsize):
    st, x, w, y = _sizes(n, 10)
    assert st == F.FFTLIB_SUCCESS
    assert x == y == 2 * n * 10 and w == wsize


def test_sizes_fft_path():
    assert _sizes(3000, 4)[:3] == (F.FFTLIB_SUCCESS, 24000, 6000)
    # NATC style always takes the FFT path and its 2N table
    assert _sizes(64, 4, style=F.FFTLIB_FUNCTION_NATC)[2] == 128


def test_status_codes():
    assert _sizes(7, 4)[0] == F.FFTLIB_ERR_INVALID_DIMENSION
    assert _sizes(0, 4)[0] == F.FFTLIB_ERR_INVALID_DIMENSION
    assert _sizes(64, 0)[0] == F.FFTLIB_ERR_INVALID_DIMENSION
    assert _sizes(64, 4, interleave=0)[0] == F.FFTLIB_ERR_NOT_IMPLEMENTED
    assert _sizes(64, 4, dtype=F.FFTLIB_UINT32)[0] == F.FFTLIB_ERR_NOT_IMPLEMENTED
    L = F.lib()
    a = F.MmaInitArgs(1, 64, 4, 1)
    bx, bw, by = F.BufParams(F.FFTLIB_FLOAT32, 512), F.BufParams(F.FFTLIB_FLOAT32, 128 * 128), \
        F.BufParams(F.FFTLIB_FLOAT32, 512)
    h = C.create_string_buffer(getattr(L, M + "getHandleSize")(C.byref(a)))
    chk = getattr(L, M + "init_checkParams")
    assert chk(None, bx, bw, by, C.byref(a)) == F.FFTLIB_ERR_NULL_POINTER
    assert chk(h, bx, bw, by, C.byref(a)) == F.FFTLIB_SUCCESS
    assert chk(h, bx, F.BufParams(F.FFTLIB_FLOAT32, 100), by, C.byref(a)) == F.FFTLIB_ERR_INVALID_DIMENSION
    assert chk(h, bx, bw, F.BufParams(F.FFTLIB_FLOAT32, 510), C.byref(a)) == F.FFTLIB_ERR_INVALID_DIMENSION
    assert chk(h, bx, F.BufParams(F.FFTLIB_INT32, 128 * 128), by, C.byref(a)) == F.FFTLIB_ERR_INVALID_TYPE
    ex = getattr(L, M + "exec_checkParams")
    buf = C.create_string_buffer(8)
    assert ex(h, buf, buf, None) == F.FFTLIB_ERR_NULL_POINTER
    assert ex(h, buf, buf, buf) == F.FFTLIB_SUCCESS
    # exec on a handle init never set up
    assert getattr(L, M + "exec")(C.create_string_buffer(64), buf, buf, buf) == F.FFTLIB_ERR_NULL_POINTER


def _fp64_embedding(m):
    j = np.arange(m)
    ang = 2 * np.pi * ((j[:, None] * j[None, :]) % m) / m
    w = np.zeros((2 * m, 2 * m))
    w[0::2, 0::2] = np.cos(ang)
    w[0::2, 1::2] = -np.sin(ang)
    w[1::2, 0::2] = np.sin(ang)
    w[1::2, 1::2] = np.cos(ang)
    return w


@pytest.mark.parametrize("n", [8, 32, 64, 256, 2048])
def test_twgen_host_matrix(n):
    st, _, wsize, _ = _sizes(n, 1)
    a = F.MmaInitArgs(1, n, 1, 1)
    w = np.zeros(wsize, np.float32)
    assert getattr(F.lib(), M + "twGen")(C.byref(a), F.ptr(w), F.BufParams(F.FFTLIB_FLOAT32, wsize)) == 0
    if n <= 64:
        want = _fp64_embedding(n).ravel()
    else:
        n1, n2 = {256: (16, 16), 2048: (64, 32)}[n]
        tw = np.exp(-2j * np.pi * np.arange(n) / n)
        tws = np.empty(2 * n)
        tws[0::2], tws[1::2] = tw.real, tw.imag
        want = np.concatenate([_fp64_embedding(n1).ravel(), _fp64_embedding(n2).ravel(), tws])
    # FP64 values rounded once to FP32
    assert np.abs(w.astype(np.float64) - want).max() <= 6e-8
    # the one-stage matrix applied in FP64 is the DFT
    if n <= 64:
        x = np.random.default_rng(0).uniform(-1, 1, 2 * n)
        y = x @ w.astype(np.float64).reshape(2 * n, 2 * n)
        ref = np.fft.fft(x[0::2] + 1j * x[1::2])
        assert np.abs(y[0::2] + 1j * y[1::2] - ref).max() < 1e-5


def test_twgen_rejects_wrong_size():
    a = F.MmaInitArgs(1, 64, 1, 1)
    w = np.zeros(10, np.float32)
    st = getattr(F.lib(), M + "twGen")(C.byref(a), F.ptr(w), F.BufParams(F.FFTLIB_FLOAT32, 10))
    assert st == F.FFTLIB_ERR_INVALID_DIMENSION
