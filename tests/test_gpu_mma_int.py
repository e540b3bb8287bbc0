"""Bit-exact parity of the coordinator's integer paths (INT16 / INT32) on
the GPU against the integer oracle and the reference's own natural C, and
the reference test's 50-LSB tolerance against its committed vectors
(FFTLIB_FFT_fft_ixX_cxX_oxX_d.c:159-170)."""
import os

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DT = {16: F.FFTLIB_INT16, 32: F.FFTLIB_INT32}
NP = {16: np.int16, 32: np.int32}

CASES = [(4, 3, 1), (8, 2, 0), (16, 4, 1), (16, 1, 0), (32, 8, 1), (32, 4, 0), (64, 4, 1), (64, 8, 0), (64, 32, 1),
         (64, 16, 0), (64, 16, 1), (128, 2, 1), (256, 3, 0), (1024, 2, 1), (4096, 2, 1), (512, 1, 1), (80, 2, 1),
         (16, 1000, 1), (32, 777, 0), (256, 300, 1), (65536, 1, 1)]


# Shifts that reach every branch of the tensor-core kernels' 32-bit rounding:
# exactly 8 (the low byte folds in), 9..37 (a partial shift of the folded
# value), the cap at 37 and above, and values with bits above the low byte
# (the reference's shift arithmetic keeps only the low byte).
WIDE_SHIFTS = ([8] * 5, [16] * 5, [24] * 5, [37] * 5, [40] * 5, [0x108] * 5, [8, 16, 0x108, 24, 9])


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def run(torch, bits, n, batch, il, shifts, x, on_device=True, stream=False):
    d = F.DftMma(n, batch, dtype=DT[bits], interleave=il, shifts=shifts, w_device=on_device)
    if on_device:
        X = torch.from_numpy(np.ascontiguousarray(x, NP[bits])).cuda()
        Y = torch.zeros_like(X)
        if stream:
            s = torch.cuda.current_stream()
            d.exec_async(X, Y, F.ptr(s.cuda_stream))
            F.check(F.lib().FFTLIB_b200_FFT_fft_sync(F.ptr(s.cuda_stream)), "sync")
        else:
            d.exec(X, Y)
        return Y.cpu().numpy()
    X = np.array(x, NP[bits])
    Y = np.zeros_like(X)
    d.exec(X, Y, w=d.w_host)
    return Y


def _rand(bits, size, seed, full):
    mx = (1 << (bits - 1)) - 1
    lo, hi = (-mx - 1, mx) if full else (-1000, 1000)
    return np.random.default_rng(seed).integers(lo, hi + 1, size)


@pytest.mark.parametrize("bits", [16, 32])
@pytest.mark.parametrize("n,batch,il", CASES)
def test_bit_exact_with_oracle_and_reference_cn(torch_cuda, bits, n, batch, il):
    if bits == 32 and n in (80, 65536):
        pytest.skip("not a d0 x 8^L length within four stages")
    for seed, full in ((1, False), (2, True)):
        x = _rand(bits, 2 * n * batch, 7 * n + seed, full)
        for sh in ([1, 1, 1, 1, 1], [4, 4, 4, 4, 4], [0, 0, 0, 0, 0], [bits - 1] * 5, [0, 3, 1, 2, 5]) + WIDE_SHIFTS:
            y = run(torch_cuda, bits, n, batch, il, sh, x)
            want = O.mma_exec(bits, n, batch, il, sh, x)
            assert np.array_equal(y, want), (bits, n, batch, il, sh, full)
            if O.ref_mma_available() and n * batch <= 8192:
                assert np.array_equal(y, O.ref_mma_exec(bits, n, batch, il, sh, x))


@pytest.mark.parametrize("bits,n,batch,il", [(16, 16, 8, 1), (16, 64, 4, 0), (16, 1024, 2, 1), (32, 32, 4, 1),
                                              (32, 64, 8, 0)])
def test_host_buffers_and_stream_entry(torch_cuda, bits, n, batch, il):
    x = _rand(bits, 2 * n * batch, 11 * n, True)
    sh = [2, 2, 2, 2, 2]
    want = O.mma_exec(bits, n, batch, il, sh, x)
    assert np.array_equal(run(torch_cuda, bits, n, batch, il, sh, x, on_device=False), want)
    assert np.array_equal(run(torch_cuda, bits, n, batch, il, sh, x, stream=True), want)


def test_reference_committed_vectors(torch_cuda):
    d = np.load(os.path.join(GOLDEN, "mma_int_static.npz"))
    for cid in d["ids"]:
        bits, batch, n, il = (int(v) for v in d[f"meta_{cid}"])
        sh = d[f"shift_{cid}"]
        y = run(torch_cuda, bits, n, batch, il, sh, d[f"in_{cid}"])
        assert np.array_equal(y, O.mma_exec(bits, n, batch, il, sh, d[f"in_{cid}"])), cid
        assert np.abs(y.astype(np.int64) - d[f"out_{cid}"].astype(np.int64)).max() <= 50, cid


def test_high_radix_needs_distinct_buffers(torch_cuda):
    import torch

    d = F.DftMma(64, 4, dtype=F.FFTLIB_INT16, interleave=1)
    X = torch.zeros(2 * 64 * 4, dtype=torch.int16, device="cuda")
    st = F.lib().FFTLIB_FFT_fft_ixX_cxX_oxX_exec(d.handle, F.ptr(X), F.ptr(d.w), F.ptr(X))
    assert st == F.FFTLIB_ERR_INVALID_VALUE
    assert d.path == 3


@pytest.mark.parametrize("bits,n,batch,il", [(16, 16, 1 << 16, 1), (16, 32, 40000, 0), (16, 64, 20001, 1),
                                             (16, 8, 3333, 1), (16, 1, 999, 1), (16, 2, 70, 0), (16, 4, 513, 1)])
def test_tensor_core_and_cuda_core_products_agree(torch_cuda, bits, n, batch, il):
    """The INT16 dftSmall / dftLarge product on the tensor cores (byte limbs
    of offset-binary values, exact) against the CUDA-core kernel on the same
    full-range inputs, ragged batches included, and against the oracle."""
    L = F.lib()
    x = _rand(bits, 2 * n * batch, 3 * n + batch, True)
    for sh in ([0] * 5, [bits - 1] * 5, [7] * 5):
        try:
            L.FFTLIB_b200_FFT_setIntTensorCores(0)
            y_cc = run(torch_cuda, bits, n, batch, il, sh, x)
        finally:
            L.FFTLIB_b200_FFT_setIntTensorCores(1)
        y_tc = run(torch_cuda, bits, n, batch, il, sh, x)
        assert np.array_equal(y_tc, y_cc), sh
        k = min(batch, 257)
        assert np.array_equal(y_tc[: 2 * n * k], O.mma_exec(bits, n, k, il, sh, x[: 2 * n * k])), sh


def test_tensor_core_product_in_place(torch_cuda):
    import torch

    bits, n, batch = 16, 32, 5000
    x = _rand(bits, 2 * n * batch, 77, True)
    sh = [3] * 5
    d = F.DftMma(n, batch, dtype=F.FFTLIB_INT16, interleave=1, shifts=sh)
    X = torch.from_numpy(np.ascontiguousarray(x, np.int16)).cuda()
    d.exec(X, X)
    assert np.array_equal(X.cpu().numpy(), O.mma_exec(bits, n, batch, 1, sh, x))


@pytest.mark.parametrize("n,batch,il", [(256, 301, 1), (1024, 77, 1), (4096, 9, 1), (65536, 3, 1), (128, 100, 1),
                                        (64, 513, 1), (512, 33, 1), (2048, 5, 1), (256, 7, 0), (1024, 1, 1),
                                        (16384, 2, 1)])
def test_high_radix_tensor_core_stages_agree(torch_cuda, n, batch, il):
    """The INT16 highRadix radix-16 stages and final stage on the tensor cores
    against the CUDA-core kernels and the oracle: full-range inputs with
    imaginary parts of -32768 planted (the reference's saturating negation),
    ragged batches, shifts that saturate and shifts that do not."""
    L = F.lib()
    x = _rand(16, 2 * n * batch, 5 * n + batch, True)
    x[1::37] = -32768
    x[0::53] = -32768
    x[3::41] = 32767
    for sh in ([0] * 5, [15] * 5, [2, 2, 2, 2, 4], [1, 3, 0, 2, 5]) + WIDE_SHIFTS:
        try:
            L.FFTLIB_b200_FFT_setIntTensorCores(0)
            y_cc = run(torch_cuda, 16, n, batch, il, sh, x)
        finally:
            L.FFTLIB_b200_FFT_setIntTensorCores(1)
        y_tc = run(torch_cuda, 16, n, batch, il, sh, x)
        assert np.array_equal(y_tc, y_cc), sh
        k = max(1, min(batch, 16384 // n))
        assert np.array_equal(y_tc[: 2 * n * k], O.mma_exec(16, n, k, il, sh, x[: 2 * n * k])), sh


def test_high_radix_tensor_core_unaligned_rows_fall_back(torch_cuda):
    """Rows that start off a 16-byte boundary take the CUDA-core kernels with
    the same bits."""
    import torch

    n, batch, sh = 256, 9, [2, 2, 2, 2, 4]
    x = _rand(16, 2 * n * batch, 99, True)
    d = F.DftMma(n, batch, dtype=F.FFTLIB_INT16, interleave=1, shifts=sh)
    X = torch.zeros(2 * n * batch + 8, dtype=torch.int16, device="cuda")
    X[2:2 + 2 * n * batch] = torch.from_numpy(np.ascontiguousarray(x, np.int16)).cuda()
    Y = torch.zeros(2 * n * batch + 8, dtype=torch.int16, device="cuda")
    st = F.lib().FFTLIB_FFT_fft_ixX_cxX_oxX_exec(d.handle, F.ptr(X.data_ptr() + 4), F.ptr(d.w),
                                                 F.ptr(Y.data_ptr() + 4))
    F.check(st, "exec")
    torch.cuda.synchronize()
    assert np.array_equal(Y[2:2 + 2 * n * batch].cpu().numpy(), O.mma_exec(16, n, batch, 1, sh, x))
