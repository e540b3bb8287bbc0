"""Host-side checks of the coordinator's three integer kernels called on
their own (FFTLIB_FFT_dftSmall / dftLarge / highRadixDecompositions
_ixX_cxX_oxX_*), no GPU needed: getSizes and twGen against the oracle's
restatement of the reference generators (c71/..._ci.cpp), the status codes of
each variant's init_checkParams (..._oxX.cpp), the oracle bit-exact with the
reference's natural C for every variant, and within the reference tests'
50-LSB tolerance of their committed vectors (..._d.c:160-175)."""
import ctypes as C
import os

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
NP = {16: np.int16, 32: np.int32}
DT = {16: F.FFTLIB_INT16, 32: F.FFTLIB_INT32}
VARIANT = {"dftSmall": 1, "dftLarge": 2, "highRadix": 3}
FIXTURE = {"dftSmall": "mma_dft_small_static.npz", "dftLarge": "mma_dft_large_static.npz",
           "highRadix": "mma_high_radix_static.npz"}


def call(variant, fn, *args):
    prefix, _ = F.DFT_VARIANTS[variant]
    return getattr(F.lib(), prefix + fn)(*args)


def sizes(variant, bits, n, batch, il):
    _, t = F.DFT_VARIANTS[variant]
    a = t(1, n, batch, il)
    bx, bw, by = (F.BufParams(DT[bits], 0) for _ in range(3))
    st = call(variant, "getSizes", C.byref(a), bx, bw, by)
    return st, a, bx, bw, by


# (variant, bits, fftSize, batch, interleave), including lengths the
# coordinator would route elsewhere (dftLarge of 40 and 64 with any batch,
# highRadix of 64 with a large batch)
CASES = [("dftSmall", 16, 5, 6, 1), ("dftSmall", 16, 13, 5, 1), ("dftSmall", 16, 16, 64, 0), ("dftSmall", 32, 7, 43, 0),
         ("dftSmall", 32, 8, 2, 1), ("dftLarge", 16, 40, 5, 0), ("dftLarge", 16, 32, 8, 1), ("dftLarge", 16, 64, 43, 1),
         ("dftLarge", 32, 16, 32, 1), ("dftLarge", 32, 40, 5, 0), ("dftLarge", 16, 17, 3, 1),
         ("highRadix", 16, 64, 64, 1), ("highRadix", 16, 128, 3, 0), ("highRadix", 16, 512, 2, 1),
         ("highRadix", 32, 32, 6, 1), ("highRadix", 32, 64, 3, 0), ("highRadix", 32, 1024, 1, 1)]


@pytest.mark.parametrize("variant,bits,n,batch,il", CASES)
def test_sizes_and_twgen(variant, bits, n, batch, il):
    st, a, bx, bw, by = sizes(variant, bits, n, batch, il)
    assert st == F.FFTLIB_SUCCESS
    want = O.mma_twgen(bits, n, batch, il, VARIANT[variant])
    assert bx.dim_x == by.dim_x == 2 * n * batch and bw.dim_x == want.size
    got = np.zeros(bw.dim_x, NP[bits])
    assert call(variant, "twGen", C.byref(a), F.ptr(got), C.byref(bw)) == F.FFTLIB_SUCCESS
    assert np.array_equal(got, want)


def test_size_limits_of_each_variant():
    for bits in (16, 32):
        mma = 32 if bits == 16 else 16
        assert sizes("dftSmall", bits, mma // 2, 4, 1)[0] == F.FFTLIB_SUCCESS
        assert sizes("dftSmall", bits, mma // 2 + 1, 4, 1)[0] == F.FFTLIB_ERR_INVALID_DIMENSION
        assert sizes("dftLarge", bits, mma // 2, 4, 1)[0] == F.FFTLIB_ERR_INVALID_DIMENSION
        assert sizes("dftLarge", bits, mma // 2 + 1, 4, 1)[0] == F.FFTLIB_SUCCESS
        st, a, bx, bw, by = sizes("highRadix", bits, 2 * mma, 4, 1)
        assert st == F.FFTLIB_SUCCESS
    for variant in VARIANT:
        _, t = F.DFT_VARIANTS[variant]
        a = t(1, 8, 4, 1)
        bx = F.BufParams(F.FFTLIB_FLOAT32, 0)
        assert call(variant, "getSizes", C.byref(a), bx, F.BufParams(12, 0), F.BufParams(12, 0)) == \
            F.FFTLIB_ERR_NOT_IMPLEMENTED


def test_status_codes():
    for variant in VARIANT:
        for bits in (16, 32):
            mma = 32 if bits == 16 else 16
            n = {"dftSmall": mma // 2, "dftLarge": mma, "highRadix": 2 * mma}[variant]
            st, a, bx, bw, by = sizes(variant, bits, n, 4, 1)
            h = C.create_string_buffer(call(variant, "getHandleSize", C.byref(a)))
            chk = lambda *b: call(variant, "init_checkParams", *b, C.byref(a))  # noqa: E731
            assert chk(None, bx, bw, by) == F.FFTLIB_ERR_NULL_POINTER
            assert chk(h, bx, bw, by) == F.FFTLIB_SUCCESS
            assert chk(h, F.BufParams(DT[bits], bx.dim_x + 2), bw, by) == F.FFTLIB_ERR_INVALID_DIMENSION
            assert chk(h, bx, bw, F.BufParams(DT[bits], 2)) == F.FFTLIB_ERR_INVALID_DIMENSION
            assert chk(h, bx, F.BufParams(DT[bits], bw.dim_x - 1), by) == F.FFTLIB_ERR_INVALID_DIMENSION
            other = F.FFTLIB_INT32 if bits == 16 else F.FFTLIB_INT16
            assert chk(h, bx, F.BufParams(other, bw.dim_x), by) == F.FFTLIB_ERR_INVALID_TYPE
            assert chk(h, F.BufParams(F.FFTLIB_UINT32, bx.dim_x), bw, by) == F.FFTLIB_ERR_NOT_IMPLEMENTED
            assert call(variant, "exec_checkParams", h, None, C.addressof(bx), C.addressof(by)) == \
                F.FFTLIB_ERR_NULL_POINTER
    # highRadix below 2 MMA points
    st, a, bx, bw, by = sizes("highRadix", 16, 48, 2, 1)
    h = C.create_string_buffer(call("highRadix", "getHandleSize", C.byref(a)))
    assert call("highRadix", "init_checkParams", h, bx, bw, by, C.byref(a)) == F.FFTLIB_ERR_INVALID_VALUE
    # dftLarge: the LINALG shift bound (int8_t shift above 64 for INT16, 128 for INT32)
    for bits, bad in ((16, 65), (32, 127)):
        st, a, bx, bw, by = sizes("dftLarge", bits, 32, 2, 1)
        a.shiftVector[0] = bad
        h = C.create_string_buffer(call("dftLarge", "getHandleSize", C.byref(a)))
        want = F.FFTLIB_ERR_INVALID_SHIFT if bits == 16 else F.FFTLIB_SUCCESS
        assert call("dftLarge", "init_checkParams", h, bx, bw, by, C.byref(a)) == want


def _rand(bits, size, seed, full):
    mx = (1 << (bits - 1)) - 1
    lo, hi = (-mx - 1, mx) if full else (-1000, 1000)
    return np.random.default_rng(seed).integers(lo, hi + 1, size)


needs_ref = pytest.mark.skipif(not O.ref_mma_available(), reason="oracle/_ref/libref_mma.so not built")


@needs_ref
@pytest.mark.parametrize("variant,bits,n,batch,il", CASES)
def test_oracle_bit_exact_with_reference_cn(variant, bits, n, batch, il):
    v = VARIANT[variant]
    for seed, full in ((1, False), (2, True)):
        x = _rand(bits, 2 * n * batch, 31 * n + seed, full)
        for sh in ([1, 1, 1, 1, 1], [0, 0, 0, 0, 0], [bits - 1] * 5, [3, 2, 4, 1, 2]):
            assert np.array_equal(O.mma_exec(bits, n, batch, il, sh, x, variant=v),
                                  O.ref_mma_exec(bits, n, batch, il, sh, x, variant=v)), (sh, full)


@pytest.mark.parametrize("variant", list(VARIANT))
def test_oracle_within_reference_tolerance_of_committed_vectors(variant):
    d = np.load(os.path.join(GOLDEN, FIXTURE[variant]))
    assert len(d["ids"]) >= 11
    for cid in d["ids"]:
        bits, batch, n, il = (int(v) for v in d[f"meta_{cid}"])
        y = O.mma_exec(bits, n, batch, il, d[f"shift_{cid}"], d[f"in_{cid}"], variant=VARIANT[variant])
        diff = np.abs(y.astype(np.int64) - d[f"out_{cid}"].astype(np.int64))
        assert diff.max() <= 50, (cid, diff.max())
