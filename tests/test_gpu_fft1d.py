"""Parity of the single-transform kernels FFTLIB_{fft,ifft}1d_* (through the
FFTLIB C API, CUDA path) against the oracle, the reference's own _cn code,
the reference's committed vectors and FP64.

Tolerances:
* relative L2 error against the FP64 transform <= 2e-6 (FP32 paths);
* max abs difference to the reference's static vectors: r2c 2^-3
  (FFTLIB_fft1d_i32f_c32fc_o32fc_d.c:194), c2r 0.1
  (FFTLIB_ifft1d_i32fc_c32fc_o32f_d.c:192);
* int16: bit-exact with the reference _cn.
"""
import os

import numpy as np
import pytest

import fftcall
import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REL_L2 = 2e-6

C2C_SIZES = [1, 2, 3, 4, 5, 8, 12, 16, 60, 64, 125, 256, 1000, 1024, 3000, 4096, 6561, 16384,
             32768, 65536, 59049, 1 << 20]
REAL_SIZES = [2, 4, 6, 8, 64, 120, 1000, 6000, 8192, 32768, 65536, 1 << 20]


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("n", C2C_SIZES)
def test_c2c_vs_fp64_and_oracle(gpu, n, inverse):
    x = O.uniform_c2c(n, 1, seed=3 * n + int(inverse), lo=-256.0, hi=256.0)
    y = fftcall.fft1d_c2c(x, n, inverse=inverse)
    assert O.rel_l2(y, O.fp64_c2c(x, n, 1, inverse)) <= REL_L2
    if n <= 16384:
        yo = O.fft1d_c2c_f32(x, n, inverse)
        assert O.rel_l2(y, O.as_complex(yo, n, 1)) <= REL_L2


@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("n", [16, 60, 4096, 65536])
def test_c2c_cn_and_host_buffers(gpu, n, inverse):
    x = O.uniform_c2c(n, 1, seed=11 * n)
    ref = O.fp64_c2c(x, n, 1, inverse)
    assert O.rel_l2(fftcall.fft1d_c2c(x, n, inverse, entry="cn"), ref) <= REL_L2
    assert O.rel_l2(fftcall.fft1d_c2c(x, n, inverse, on_device=False), ref) <= REL_L2


def test_c2c_vs_reference_python_model(gpu):
    d = np.load(os.path.join(GOLD, "fft1d_c2c_pymodel.npz"))
    for i, n in enumerate(d["sizes"]):
        n = int(n)
        x = d[f"case{i}_in"]
        assert O.rel_l2(fftcall.fft1d_c2c(x, n), O.as_complex(d[f"case{i}_fwd"], n, 1)[0]) < 1e-6
        # the model's inverse is rounded to 6 decimals
        assert np.abs(fftcall.fft1d_c2c(x, n, True) - d[f"case{i}_inv"]).max() < 2e-6


def test_c2c_vs_reference_cn(gpu, ref_cn):
    if not O.ref1d_available():
        pytest.skip("single-transform reference _cn not built")
    for n in (64, 256, 3000, 4096, 6561):
        x = O.uniform_c2c(n, 1, seed=5 * n, lo=-256.0, hi=256.0)
        for inverse in (False, True):
            r = O.ref_fft1d_c2c_f32(x, n, inverse)
            y = fftcall.fft1d_c2c(x, n, inverse)
            assert O.rel_l2(y, O.as_complex(r, n, 1)) <= REL_L2
            assert np.abs(y - r).max() <= (2.0 ** -5 if not inverse else 1e-5)


def test_round_trip_large(gpu):
    """ifft1d(fft1d(x)) == x at 2^22 points (three global passes), a
    size-independent check beyond the oracle's reach."""
    n = 1 << 22
    x = O.uniform_c2c(n, 1, seed=99)
    y = fftcall.fft1d_c2c(x, n)
    z = fftcall.fft1d_c2c(y, n, inverse=True)
    assert O.rel_l2(z, O.as_complex(x, n, 1)) <= 4e-6
    # Parseval: sum |X|^2 = N sum |x|^2
    ex = float(np.sum(x.astype(np.float64) ** 2))
    ey = float(np.sum(y.astype(np.float64) ** 2))
    assert abs(ey / (n * ex) - 1.0) < 1e-5


# ---- real-input kernels ---------------------------------------------------------

@pytest.mark.parametrize("n", REAL_SIZES)
def test_r2c_vs_fp64(gpu, n):
    x = O.real_signal(n, 1, seed=n + 5)
    y = fftcall.fft1d_r2c(x, n)
    f = np.fft.fft(x.astype(np.float64))
    assert O.rel_l2(y, f) <= REL_L2
    if n <= 16384:
        assert O.rel_l2(y, O.as_complex(O.fft1d_r2c_f32(x, n), n, 1)[0]) <= REL_L2


@pytest.mark.parametrize("n", REAL_SIZES)
def test_c2r_vs_fp64(gpu, n):
    x = O.real_signal(n, 1, seed=n + 9)
    f = np.fft.fft(x.astype(np.float64))
    spec = np.stack([f.real, f.imag], -1).ravel().astype(np.float32)
    y = fftcall.fft1d_c2r(spec, n)
    assert O.rel_l2(y, O.fp64_c2r(spec, n, 1, 1)[0]) <= REL_L2
    assert O.rel_l2(y, x.astype(np.float64)) <= 4e-6


@pytest.mark.parametrize("kind", ["r2c", "c2r"])
def test_real_vs_reference_static_vectors(gpu, kind):
    d = np.load(os.path.join(GOLD, f"fft1d_{kind}_static.npz"))
    for cid in d["ids"]:
        n = int(d[f"n_{cid}"])
        xin, yout = d[f"in_{cid}"], d[f"out_{cid}"]
        if kind == "r2c":
            y = fftcall.fft1d_r2c(xin, n)
            assert np.abs(y - yout).max() <= 2.0 ** -3, (cid, n)
            assert O.rel_l2(y, np.fft.fft(xin.astype(np.float64))) <= REL_L2
        else:
            y = fftcall.fft1d_c2r(xin, n)
            assert np.abs(y - yout).max() <= 0.1, (cid, n)
            assert O.rel_l2(y, O.fp64_c2r(xin, n, 1, 1)[0]) <= REL_L2


@pytest.mark.parametrize("n", [64, 1000, 4096])
def test_real_cn_and_host_buffers(gpu, n):
    x = O.real_signal(n, 1, seed=n + 17)
    f = np.fft.fft(x.astype(np.float64))
    assert O.rel_l2(fftcall.fft1d_r2c(x, n, entry="cn"), f) <= REL_L2
    assert O.rel_l2(fftcall.fft1d_r2c(x, n, on_device=False), f) <= REL_L2
    spec = np.stack([f.real, f.imag], -1).ravel().astype(np.float32)
    want = O.fp64_c2r(spec, n, 1, 1)[0]
    assert O.rel_l2(fftcall.fft1d_c2r(spec, n, entry="cn"), want) <= REL_L2
    assert O.rel_l2(fftcall.fft1d_c2r(spec, n, on_device=False), want) <= REL_L2


def test_real_vs_reference_cn(gpu, ref_cn):
    if not O.ref1d_available():
        pytest.skip("single-transform reference _cn not built")
    for n in (64, 120, 4096, 6000):
        x = O.real_signal(n, 1, seed=n + 23)
        r = O.ref_fft1d_r2c_f32(x, n)
        y = fftcall.fft1d_r2c(x, n)
        assert O.rel_l2(y, O.as_complex(r, n, 1)[0]) <= REL_L2
        rc = O.ref_fft1d_c2r_f32(r, n)
        yc = fftcall.fft1d_c2r(r, n)
        assert O.rel_l2(yc, rc.astype(np.float64)) <= REL_L2


# ---- int16 ------------------------------------------------------------------------

def test_i16_vs_reference_fixture(gpu):
    d = np.load(os.path.join(GOLD, "fft1d_i16_pymodel.npz"))
    for i in range(int(d["n_cases"])):
        n = int(d[f"case{i}_n"])
        y = fftcall.fft1d_i16(d[f"case{i}_in"], n, d[f"case{i}_shift"])
        assert np.array_equal(y, d[f"case{i}_out"]), (i, n)


@pytest.mark.parametrize("n,shifts", [(2, []), (4, [1]), (8, [1]), (16, [1, 1]), (32, [0, 1]), (64, [0, 1, 1]),
                                      (128, [1, 1, 1]), (256, [3, 3, 3, 3]), (2048, [1, 1, 1, 1, 2]),
                                      (16384, [0, 0, 0, 1, 0, 1, 1])])
def test_i16_vs_oracle_and_reference_cn(gpu, n, shifts):
    """Every length from 2 (the natural-C entry accepts the short ones the
    optimized check refuses) with full-range inputs that overflow 16-bit
    intermediates; bit-exact."""
    entry = "cn" if n < 64 else "kernel"
    for seed, (lo, hi) in enumerate([(-1000, 1000), (-32768, 32767)]):
        x = O.int16_input(n, 1, 300 + n + seed, lo, hi)
        y = fftcall.fft1d_i16(x, n, shifts, entry=entry)
        assert np.array_equal(y, O.fft1d_c2c_i16(x, n, shifts)), (n, lo)
        if O.ref1d_available():
            assert np.array_equal(y, O.ref_fft1d_c2c_i16(x, n, shifts)), (n, lo)


def test_i16_host_buffers(gpu):
    n, sh = 1024, [2, 2, 2, 2, 2]
    x = O.int16_input(n, 1, 77, -32768, 32767)
    assert np.array_equal(fftcall.fft1d_i16(x, n, sh, on_device=False), O.fft1d_c2c_i16(x, n, sh))


# ---- plan records ------------------------------------------------------------------

def test_kernel_refuses_a_pblock_for_another_length(gpu):
    import c7x_fftlib_b200 as F

    n = 64
    X = gpu.zeros(4 * n, dtype=gpu.float32, device="cuda")
    base = F.KERNELS["1d_c2c"]
    b = F.bp(F.FFTLIB_FLOAT32, 2 * n)
    pb = F.pblock("1d_c2c")
    F.check(F.fn(base + "_init")(F.ptr(X), b, F.ptr(X), b, F.ptr(X), b, pb), "init")
    b2 = F.bp(F.FFTLIB_FLOAT32, 4 * n)
    assert F.fn(base + "_kernel")(F.ptr(X), b2, F.ptr(X), b2, F.ptr(X), b2, pb) == F.FFTLIB_ERR_INVALID_DIMENSION
    # a single-transform record is not a batched one, and the reverse
    assert F.fn(F.KERNELS["c2c"] + "_kernel")(F.ptr(X), b, F.ptr(X), b, F.ptr(X), b, n, 1, pb) == \
        F.FFTLIB_ERR_FAILURE
