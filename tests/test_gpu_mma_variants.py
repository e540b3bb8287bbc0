"""The coordinator's three integer kernels called on their own
(FFTLIB_FFT_dftSmall / dftLarge / highRadixDecompositions_ixX_cxX_oxX_*) on
the GPU: bit-exact with the integer oracle and the reference's own natural C,
and within the reference tests' 50-LSB tolerance of their committed vectors
(..._d.c:160-175)."""
import os

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
DT = {16: F.FFTLIB_INT16, 32: F.FFTLIB_INT32}
NP = {16: np.int16, 32: np.int32}
VARIANT = {"dftSmall": 1, "dftLarge": 2, "highRadix": 3}
FIXTURE = {"dftSmall": "mma_dft_small_static.npz", "dftLarge": "mma_dft_large_static.npz",
           "highRadix": "mma_high_radix_static.npz"}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def run(torch, variant, bits, n, batch, il, shifts, x, on_device=True, in_place=False):
    d = F.DftMma(n, batch, dtype=DT[bits], interleave=il, shifts=shifts, w_device=on_device, variant=variant)
    if on_device:
        X = torch.from_numpy(np.ascontiguousarray(x, NP[bits])).cuda()
        Y = X if in_place else torch.zeros_like(X)
        d.exec(X, Y)
        return Y.cpu().numpy()
    X = np.array(x, NP[bits])
    Y = X if in_place else np.zeros_like(X)
    d.exec(X, Y, w=d.w_host)
    return Y


def _rand(bits, size, seed, full):
    mx = (1 << (bits - 1)) - 1
    lo, hi = (-mx - 1, mx) if full else (-1000, 1000)
    return np.random.default_rng(seed).integers(lo, hi + 1, size)


# includes dftLarge lengths whose table leaves shared memory (200 INT16,
# 120 INT32: the tiled multiply) and highRadix with a batch the coordinator
# would give to dftLarge
CASES = [("dftSmall", 16, 5, 135, 1), ("dftSmall", 16, 13, 70, 1), ("dftSmall", 16, 16, 2048, 0),
         ("dftSmall", 32, 7, 43, 0), ("dftSmall", 32, 8, 64, 1), ("dftLarge", 16, 40, 5, 0),
         ("dftLarge", 16, 64, 43, 1), ("dftLarge", 16, 17, 300, 1), ("dftLarge", 16, 200, 37, 1),
         ("dftLarge", 32, 16, 32, 1), ("dftLarge", 32, 40, 5, 0), ("dftLarge", 32, 120, 19, 0),
         ("highRadix", 16, 64, 64, 1), ("highRadix", 16, 128, 6, 0), ("highRadix", 16, 2048, 2, 1),
         ("highRadix", 32, 32, 8, 1), ("highRadix", 32, 64, 3, 0), ("highRadix", 32, 8192, 1, 1)]


@pytest.mark.parametrize("variant,bits,n,batch,il", CASES)
def test_bit_exact_with_oracle_and_reference_cn(torch_cuda, variant, bits, n, batch, il):
    v = VARIANT[variant]
    for seed, full in ((1, False), (2, True)):
        x = _rand(bits, 2 * n * batch, 17 * n + seed, full)
        for sh in ([1, 1, 1, 1, 1], [0, 0, 0, 0, 0], [bits - 1] * 5, [3, 2, 4, 1, 2]):
            y = run(torch_cuda, variant, bits, n, batch, il, sh, x)
            want = O.mma_exec(bits, n, batch, il, sh, x, variant=v)
            assert np.array_equal(y, want), (sh, full)
            if O.ref_mma_available() and n * batch <= 8192:
                assert np.array_equal(y, O.ref_mma_exec(bits, n, batch, il, sh, x, variant=v))


@pytest.mark.parametrize("variant", list(VARIANT))
def test_reference_committed_vectors(torch_cuda, variant):
    d = np.load(os.path.join(GOLDEN, FIXTURE[variant]))
    for cid in d["ids"]:
        bits, batch, n, il = (int(v) for v in d[f"meta_{cid}"])
        sh = d[f"shift_{cid}"]
        y = run(torch_cuda, variant, bits, n, batch, il, sh, d[f"in_{cid}"])
        assert np.array_equal(y, O.mma_exec(bits, n, batch, il, sh, d[f"in_{cid}"], variant=VARIANT[variant])), cid
        assert np.abs(y.astype(np.int64) - d[f"out_{cid}"].astype(np.int64)).max() <= 50, cid


@pytest.mark.parametrize("variant,bits,n,batch,il", [("dftSmall", 16, 16, 33, 1), ("dftLarge", 16, 200, 9, 1),
                                                     ("dftLarge", 32, 16, 40, 0), ("highRadix", 16, 256, 3, 1)])
def test_host_buffers_and_in_place(torch_cuda, variant, bits, n, batch, il):
    x = _rand(bits, 2 * n * batch, 5 * n, True)
    sh = [2, 2, 2, 2, 2]
    want = O.mma_exec(bits, n, batch, il, sh, x, variant=VARIANT[variant])
    assert np.array_equal(run(torch_cuda, variant, bits, n, batch, il, sh, x, on_device=False), want)
    if variant != "highRadix":  # highRadix works in pX and refuses pX == pY
        assert np.array_equal(run(torch_cuda, variant, bits, n, batch, il, sh, x, in_place=True), want)


def test_variant_handles_are_not_interchangeable(torch_cuda):
    import torch

    d = F.DftMma(16, 4, dtype=F.FFTLIB_INT16, interleave=1, variant="dftSmall")
    X = torch.zeros(2 * 16 * 4, dtype=torch.int16, device="cuda")
    Y = torch.zeros_like(X)
    st = F.lib().FFTLIB_FFT_dftLarge_ixX_cxX_oxX_exec(d.handle, F.ptr(X), F.ptr(d.w), F.ptr(Y))
    assert st == F.FFTLIB_ERR_INVALID_VALUE
    # the coordinator's exec runs any of its variants' handles
    assert F.lib().FFTLIB_FFT_fft_ixX_cxX_oxX_exec(d.handle, F.ptr(X), F.ptr(d.w), F.ptr(Y)) == F.FFTLIB_SUCCESS


def test_high_radix_init_leaves_the_internal_table_in_twdata(torch_cuda):
    import ctypes as C

    for bits, n in ((16, 64), (16, 2048), (32, 512)):
        h = F.DftMma(n, 2, dtype=DT[bits], interleave=1, variant="highRadix")
        assert h.path == 3
        mma = 32 if bits == 16 else 16
        raw = (C.c_uint8 * (32 * 32 * 3 * 2)).in_dll(F.lib(), "FFTLIB_FFT_twData")
        got = np.frombuffer(bytes(raw), NP[bits])[: mma * mma]
        assert np.array_equal(got, O.mma_w1(bits, n))
