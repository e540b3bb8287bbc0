"""int16 batched FFT: the CUDA kernel (through the FFTLIB C API) must be
bit-exact with the reference _cn (memcmp, as
test/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._d.c:232-236 does)."""
import os

import numpy as np
import pytest

import fftcall
import oracle as O

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def nshifts(n):
    s, m = 0, n
    while m > 2:
        s, m = s + 1, m // 4
    return s


@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384])
@pytest.mark.parametrize("full_range", [False, True])
def test_i16_bit_exact_vs_oracle(gpu, n, full_range):
    rng = np.random.default_rng(n)
    ch = 5
    for trial in range(2):
        sh = rng.integers(0, 3, max(nshifts(n), 1)).astype(np.uint32)
        lo, hi = (-32768, 32767) if full_range else (-2048, 2047)
        x = O.int16_input(n, ch, 31 * n + trial, lo, hi)
        y = fftcall.i16(x, n, ch, sh)
        np.testing.assert_array_equal(y, O.fft_c2c_i16(x, n, ch, sh))


def test_i16_headline_config(gpu, ref_cn):
    """N=1024, batch 4096, inputs in [-2048, 2047], shift 2 per radix-4 stage."""
    n, ch = 1024, 4096
    sh = np.full(5, 2, np.uint32)
    x = O.int16_input(n, ch, 2024)
    y = fftcall.i16(x, n, ch, sh)
    sel = slice(0, 64 * 2 * n)  # reference _cn on the first 64 channels (the full batch is slow on CPU)
    np.testing.assert_array_equal(y[sel], O.ref_c2c_i16(x[sel], n, 64, sh))
    np.testing.assert_array_equal(y, O.fft_c2c_i16(x, n, ch, sh))


@pytest.mark.parametrize("shift", [0, 1, 3, 15, 16, 17, 31])
def test_i16_shift_edge_values(gpu, ref_cn, shift):
    """Shift amounts whose rounding mask the reference forms by 32-bit
    truncation (0 is a no-op, >= 17 drops the rounding bit)."""
    n, ch = 64, 3
    sh = np.full(3, shift, np.uint32)
    x = O.int16_input(n, ch, shift, -32768, 32767)
    y = fftcall.i16(x, n, ch, sh)
    np.testing.assert_array_equal(y, O.ref_c2c_i16(x, n, ch, sh))


def test_i16_golden_pymodel(gpu):
    d = np.load(os.path.join(GOLD, "i16_pymodel.npz"))
    for i in range(int(d["n_cases"])):
        ch, n = (int(v) for v in d[f"case{i}_meta"])
        y = fftcall.i16(d[f"case{i}_in"], n, ch, d[f"case{i}_shift"], w=d[f"case{i}_tw"])
        np.testing.assert_array_equal(y, d[f"case{i}_out"], err_msg=f"case {i} N={n}")


def test_i16_golden_ref_cn(gpu):
    d = np.load(os.path.join(GOLD, "ref_cn.npz"))
    for i in range(int(d["i16_n"])):
        ch, n = (int(v) for v in d[f"i16{i}_meta"])
        y = fftcall.i16(d[f"i16{i}_in"], n, ch, d[f"i16{i}_shift"])
        np.testing.assert_array_equal(y, d[f"i16{i}_out"], err_msg=f"case {i} N={n}")


def test_i16_host_buffers(gpu):
    n, ch = 256, 7
    sh = np.array([1, 1, 1, 1], np.uint32)
    x = O.int16_input(n, ch, 3)
    np.testing.assert_array_equal(fftcall.i16(x, n, ch, sh), fftcall.i16(x, n, ch, sh, on_device=False))


@pytest.mark.parametrize("n", [64, 128, 256, 512, 1024, 2048, 4096, 8192, 16384])
def test_i16_every_cta_walks_several_transforms(gpu, n):
    """Batches large enough that every persistent CTA takes three or more
    steps, so each group's input copied ahead (while the previous transform
    is computed) is the one transformed next; the last step is partial, and
    full-range inputs with mixed shifts. Bit-exact with the oracle."""
    per_step = 148 * (4 * max(1, 4096 // n) if n <= 4096 else 2)  # CTAs per GPU x transforms per CTA
    ch = 3 * per_step + 5
    rng = np.random.default_rng(7 * n)
    sh = rng.integers(0, 3, nshifts(n)).astype(np.uint32)
    x = O.int16_input(n, ch, 11 * n, -32768, 32767)
    np.testing.assert_array_equal(fftcall.i16(x, n, ch, sh), O.fft_c2c_i16(x, n, ch, sh))
