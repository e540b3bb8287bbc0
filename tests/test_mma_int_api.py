"""Host-side checks of the coordinator's integer paths (INT16 / INT32, the
reference's own data types), no GPU needed: the variant choice, getSizes,
twGen tables bit-identical to the oracle's restatement of the reference
generators, the reference's status codes, and the integer oracle pinned
against the reference's own natural C (dftSmall / LINALG / highRadix _cn,
compiled here) and within the reference test's tolerance of its committed
vectors."""
import ctypes as C
import os

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

M = "FFTLIB_FFT_fft_ixX_cxX_oxX_"
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BITS = {F.FFTLIB_INT16: 16, F.FFTLIB_INT32: 32}
NP = {16: np.int16, 32: np.int32}

# (fftSize, batch, interleave) across all three variants of both types
CASES = [(4, 3, 1), (8, 2, 0), (16, 4, 1), (16, 1, 0), (32, 8, 1), (32, 4, 0), (64, 4, 1), (64, 8, 0), (64, 32, 1),
         (64, 16, 0), (64, 16, 1), (128, 2, 1), (256, 2, 0), (1024, 2, 1), (4096, 1, 1), (512, 1, 1), (80, 2, 1)]


def _sizes(n, batch, interleave, dtype):
    a = F.MmaInitArgs(1, n, batch, interleave)
    bx, bw, by = F.BufParams(dtype, 0), F.BufParams(dtype, 0), F.BufParams(dtype, 0)
    st = getattr(F.lib(), M + "getSizes")(C.byref(a), bx, bw, by)
    return st, bx.dim_x, bw.dim_x, by.dim_x


@pytest.mark.parametrize("dtype", [F.FFTLIB_INT16, F.FFTLIB_INT32])
@pytest.mark.parametrize("n,batch,il", CASES)
def test_sizes_and_twgen_match_the_reference_generators(dtype, n, batch, il):
    bits = BITS[dtype]
    st, x, w, y = _sizes(n, batch, il, dtype)
    assert st == F.FFTLIB_SUCCESS
    want = O.mma_twgen(bits, n, batch, il)
    assert x == y == 2 * n * batch and w == want.size
    got = np.zeros(w, NP[bits])
    a = F.MmaInitArgs(1, n, batch, il)
    assert getattr(F.lib(), M + "twGen")(C.byref(a), F.ptr(got), C.byref(F.BufParams(dtype, w))) == 0
    assert np.array_equal(got, want)
    bad = F.BufParams(dtype, w + 1)
    assert getattr(F.lib(), M + "twGen")(C.byref(a), F.ptr(got), C.byref(bad)) == F.FFTLIB_ERR_INVALID_DIMENSION


def test_variant_choice_follows_the_reference():
    """FFTLIB_FFT_fft_ixX_cxX_oxX.cpp:13-50: MMA 32 (INT16), 16 (INT32)."""
    v = O.mma_variant
    assert [v(16, n, 4, 1) for n in (2, 16, 32, 64, 128)] == [1, 1, 2, 3, 3]
    assert [v(16, 64, b, il) for b, il in ((15, 0), (16, 1), (16, 0), (17, 1))] == [3, 3, 2, 2]
    assert [v(32, n, 4, 1) for n in (8, 16, 32, 64)] == [1, 2, 3, 3]
    assert v(32, 32, 9, 1) == 2


def test_status_codes():
    L = F.lib()
    chk = getattr(L, M + "init_checkParams")
    for dtype in (F.FFTLIB_INT16, F.FFTLIB_INT32):
        bits = BITS[dtype]
        mma = 32 if bits == 16 else 16
        a = F.MmaInitArgs(1, 2 * mma, 4, 1)
        st, x, w, y = _sizes(2 * mma, 4, 1, dtype)
        h = C.create_string_buffer(getattr(L, M + "getHandleSize")(C.byref(a)))
        bx, bw, by = F.BufParams(dtype, x), F.BufParams(dtype, w), F.BufParams(dtype, y)
        assert chk(None, bx, bw, by, C.byref(a)) == F.FFTLIB_ERR_NULL_POINTER
        assert chk(h, bx, bw, by, C.byref(a)) == F.FFTLIB_SUCCESS
        assert chk(h, F.BufParams(dtype, x - 2), bw, by, C.byref(a)) == F.FFTLIB_ERR_INVALID_DIMENSION
        assert chk(h, bx, F.BufParams(dtype, w - 1), by, C.byref(a)) == F.FFTLIB_ERR_INVALID_DIMENSION
        other = F.FFTLIB_INT32 if dtype == F.FFTLIB_INT16 else F.FFTLIB_INT16
        assert chk(h, bx, F.BufParams(other, w), by, C.byref(a)) == F.FFTLIB_ERR_INVALID_TYPE
        # highRadix below 2 MMA points: INVALID_VALUE (the size mma + mma/2 is
        # neither dftSmall nor dftLarge)
        a2 = F.MmaInitArgs(1, mma + mma // 2, 4, 1)
        st, x2, w2, y2 = _sizes(mma + mma // 2, 4, 1, dtype)
        assert chk(h, F.BufParams(dtype, x2), F.BufParams(dtype, w2), F.BufParams(dtype, y2), C.byref(a2)) == \
            F.FFTLIB_ERR_INVALID_VALUE
    # dftLarge: the LINALG shift bound (shift > 64 for INT16)
    a = F.MmaInitArgs(1, 32, 4, 1)
    a.shiftVector[0] = 65
    st, x, w, y = _sizes(32, 4, 1, F.FFTLIB_INT16)
    h = C.create_string_buffer(getattr(L, M + "getHandleSize")(C.byref(a)))
    assert chk(h, F.BufParams(1, x), F.BufParams(1, w), F.BufParams(1, y), C.byref(a)) == F.FFTLIB_ERR_INVALID_SHIFT


def _rand(bits, size, seed, full):
    mx = (1 << (bits - 1)) - 1
    lo, hi = (-mx - 1, mx) if full else (-1000, 1000)
    return np.random.default_rng(seed).integers(lo, hi + 1, size)


needs_ref = pytest.mark.skipif(not O.ref_mma_available(), reason="oracle/_ref/libref_mma.so not built")


@needs_ref
@pytest.mark.parametrize("bits", [16, 32])
@pytest.mark.parametrize("n,batch,il", CASES)
def test_oracle_bit_exact_with_reference_cn(bits, n, batch, il):
    if bits == 32 and n == 80:
        pytest.skip("80 = 10 x 8: not a d0 x 8^L length")
    for seed, full in ((1, False), (2, True)):
        x = _rand(bits, 2 * n * batch, 100 * n + seed, full)
        for sh in ([1, 1, 1, 1, 1], [4, 4, 4, 4, 4], [0, 0, 0, 0, 0], [bits - 1] * 5, [0, 3, 1, 2, 5]):
            a = O.mma_exec(bits, n, batch, il, sh, x)
            b = O.ref_mma_exec(bits, n, batch, il, sh, x)
            assert np.array_equal(a, b), (bits, n, batch, il, sh, full)


def test_oracle_within_reference_tolerance_of_committed_vectors():
    """The coordinator's 23 committed static cases
    (test/fft_c7xmma/FFTLIB_FFT_fft_ixX_cxX_oxX/..._idat.c); the reference
    test compares its kernel with them within 50 LSB (..._d.c:159-170):
    the vectors come from the MMA hardware, whose rounding differs from the
    natural C by a few LSB."""
    d = np.load(os.path.join(GOLDEN, "mma_int_static.npz"))
    exact = 0
    for cid in d["ids"]:
        bits, batch, n, il = (int(v) for v in d[f"meta_{cid}"])
        y = O.mma_exec(bits, n, batch, il, d[f"shift_{cid}"], d[f"in_{cid}"]).astype(np.int64)
        diff = np.abs(y - d[f"out_{cid}"].astype(np.int64))
        assert diff.max() <= 50, (cid, diff.max())
        exact += int(diff.max() == 0)
    assert len(d["ids"]) == 23 and exact >= 8
