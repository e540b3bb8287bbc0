"""Host-side checks of the integer matrix multiply
FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_*, no GPU needed: the status
codes of its init_checkParams (src/linalg_c7xmma/.../..._oxX.cpp:14-62, in the
same order) and the oracle bit-exact with the reference's natural C
(..._cn.cpp:27-62, compiled here) for INT8, INT16 and INT32."""
import ctypes as C

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

L_ = F.LINALG
DT = {8: F.FFTLIB_INT8, 16: F.FFTLIB_INT16, 32: F.FFTLIB_INT32}


def chk(a, b, c, shift=0, handle=True):
    args = F.LinalgInitArgs(1, shift)
    h = C.create_string_buffer(getattr(F.lib(), L_ + "getHandleSize")(C.byref(args))) if handle else None
    return getattr(F.lib(), L_ + "init_checkParams")(h, C.byref(a), C.byref(b), C.byref(c), C.byref(args))


def bp(dt, rows, cols, stride=None):
    es = {F.FFTLIB_INT8: 1, F.FFTLIB_INT16: 2, F.FFTLIB_INT32: 4}.get(dt, 4)
    return F.BufParams2D(dt, cols, rows, (cols if stride is None else stride) * es)


def test_status_codes():
    for bits, dt in DT.items():
        a, b, c = bp(dt, 4, 6), bp(dt, 6, 5), bp(dt, 4, 5)
        assert chk(a, b, c, handle=False) == F.FFTLIB_ERR_NULL_POINTER
        assert chk(a, b, c) == F.FFTLIB_SUCCESS
        assert chk(a, bp(dt, 7, 5), c) == F.FFTLIB_ERR_INVALID_DIMENSION      # A cols != B rows
        assert chk(a, b, bp(dt, 3, 5)) == F.FFTLIB_ERR_INVALID_DIMENSION      # C rows
        assert chk(a, b, bp(dt, 4, 4)) == F.FFTLIB_ERR_INVALID_DIMENSION      # C cols
        other = F.FFTLIB_INT32 if bits != 32 else F.FFTLIB_INT16
        assert chk(a, bp(other, 6, 5), c) == F.FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_TYPE_COMBINATION
        assert chk(a, b, bp(other, 4, 5)) == F.FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_TYPE_COMBINATION
        # the accumulator width bounds the shift (an int8_t: any value passes INT32's 128)
        if bits < 32:
            assert chk(a, b, c, shift=4 * bits) == F.FFTLIB_SUCCESS
            assert chk(a, b, c, shift=4 * bits + 1) == F.FFTLIB_ERR_INVALID_SHIFT
        else:
            assert chk(a, b, c, shift=127) == F.FFTLIB_SUCCESS
        assert chk(a, b, c, shift=-3) == F.FFTLIB_SUCCESS
    for bad in (F.FFTLIB_FLOAT32, F.FFTLIB_UINT32, 5):
        assert chk(bp(bad, 2, 2), bp(bad, 2, 2), bp(bad, 2, 2)) == \
            F.FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_INPUT_TYPE
    assert getattr(F.lib(), L_ + "exec_checkParams")(None, None, None, None) == F.FFTLIB_ERR_NULL_POINTER


needs_ref = pytest.mark.skipif(not O.ref_mma_available(), reason="oracle/_ref/libref_mma.so not built")


@needs_ref
@pytest.mark.parametrize("bits", [8, 16, 32])
@pytest.mark.parametrize("m,k,n", [(1, 1, 1), (5, 7, 3), (64, 64, 64), (33, 100, 17), (3, 0, 4), (70, 129, 65)])
def test_oracle_bit_exact_with_reference_cn(bits, m, k, n):
    rng = np.random.default_rng(1000 * bits + m + k + n)
    mx = (1 << (bits - 1)) - 1
    for full in (False, True):
        lo, hi = (-mx - 1, mx) if full else (-100, 100)
        a = rng.integers(lo, hi + 1, (m, k))
        b = rng.integers(lo, hi + 1, (k, n))
        for sh in (0, 1, 4, bits - 1, bits, 2 * bits):
            assert np.array_equal(O.linalg_mm(bits, a, b, sh), O.ref_linalg_mm(bits, a, b, sh)), (full, sh)
