"""FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX on the GPU: bit-exact with
the oracle and the reference's natural C (..._cn.cpp:27-62) for INT8, INT16
and INT32, ragged shapes, row strides wider than the rows, host and device
buffers, and the stream-ordered entry point."""
import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

pytestmark = pytest.mark.gpu

DT = {8: F.FFTLIB_INT8, 16: F.FFTLIB_INT16, 32: F.FFTLIB_INT32}
NP = {8: np.int8, 16: np.int16, 32: np.int32}


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _mats(bits, m, k, n, seed, full):
    rng = np.random.default_rng(seed)
    mx = (1 << (bits - 1)) - 1
    lo, hi = (-mx - 1, mx) if full else (-300, 300)
    return rng.integers(lo, hi + 1, (m, k)).astype(NP[bits]), rng.integers(lo, hi + 1, (k, n)).astype(NP[bits])


SHAPES = [(1, 1, 1), (5, 7, 3), (64, 64, 64), (65, 33, 129), (200, 300, 100), (1000, 64, 64), (3, 0, 5),
          (128, 1024, 96)]


@pytest.mark.parametrize("bits", [8, 16, 32])
@pytest.mark.parametrize("m,k,n", SHAPES)
def test_bit_exact_device(torch_cuda, bits, m, k, n):
    torch = torch_cuda
    for full in (False, True):
        a, b = _mats(bits, m, k, n, 7 * m + k + n + bits, full)
        for sh in (0, 1, bits - 1, bits + 3):
            mm = F.MatMul(m, k, n, DT[bits], shift=sh)
            # an empty A or B (k = 0) still needs a non-NULL buffer, as in the reference
            A = torch.from_numpy(a).cuda() if a.size else torch.zeros(1, dtype=torch.from_numpy(a).dtype).cuda()
            B = torch.from_numpy(b).cuda() if b.size else torch.zeros(1, dtype=A.dtype).cuda()
            Cd = torch.zeros((m, n), dtype=A.dtype, device="cuda")
            mm.exec(A, B, Cd)
            want = O.linalg_mm(bits, a, b, sh)
            assert np.array_equal(Cd.cpu().numpy(), want), (full, sh)
            if O.ref_mma_available() and m * n * k <= 1 << 22:
                assert np.array_equal(want, O.ref_linalg_mm(bits, a, b, sh))


@pytest.mark.parametrize("bits", [8, 16, 32])
def test_strides_host_buffers_and_stream(torch_cuda, bits):
    torch = torch_cuda
    m, k, n = 37, 50, 70
    lda, ldb, ldc = 64, 75, 80
    a, b = _mats(bits, m, k, n, 99 + bits, True)
    sh = 5
    want = O.linalg_mm(bits, a, b, sh)
    A = np.zeros((m, lda), NP[bits])
    A[:, :k] = a
    B = np.zeros((k, ldb), NP[bits])
    B[:, :n] = b
    Cm = np.full((m, ldc), 77, NP[bits])
    mm = F.MatMul(m, k, n, DT[bits], shift=sh, lda=lda, ldb=ldb, ldc=ldc)
    mm.exec(A, B, Cm)  # host buffers
    assert np.array_equal(Cm[:, :n], want)
    assert (Cm[:, n:] == 77).all()  # the gaps between rows of C are left alone
    Ad, Bd = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    Cd = torch.full((m, ldc), 77, dtype=Ad.dtype, device="cuda")
    s = torch.cuda.current_stream()
    mm.exec_async(Ad, Bd, Cd, F.ptr(s.cuda_stream))
    torch.cuda.synchronize()
    got = Cd.cpu().numpy()
    assert np.array_equal(got[:, :n], want) and (got[:, n:] == 77).all()
    # mixed: device A, host B, device C
    Cd.fill_(0)
    mm.exec(Ad, B, Cd)
    assert np.array_equal(Cd.cpu().numpy()[:, :n], want)


def test_overlapping_source_rows(torch_cuda):
    """A with a row stride smaller than its width (rows overlap), as the
    reference's strided indexing allows for the inputs."""
    bits, m, k, n = 16, 6, 8, 5
    rng = np.random.default_rng(3)
    flat = rng.integers(-500, 500, (m - 1) * 3 + k).astype(np.int16)
    a = np.stack([flat[r * 3: r * 3 + k] for r in range(m)])
    b = rng.integers(-500, 500, (k, n)).astype(np.int16)
    mm = F.MatMul(m, k, n, DT[bits], shift=2, lda=3)
    Cm = np.zeros((m, n), np.int16)
    mm.exec(flat, b, Cm)
    assert np.array_equal(Cm, O.linalg_mm(bits, a, b, 2))


@pytest.mark.parametrize("bits", [8, 16])
@pytest.mark.parametrize("m,k,n,lda,ldb,ldc", [(128, 128, 128, 128, 128, 128), (300, 100, 70, 112, 72, 70),
                                               (300, 100, 70, 112, 80, 70), (129, 257, 65, 272, 68, 80),
                                               (129, 257, 65, 272, 80, 80), (1000, 64, 64, 64, 64, 64),
                                               (64, 1000, 200, 1008, 200, 203), (64, 1000, 200, 1008, 208, 203),
                                               (1, 16, 4, 16, 4, 4), (1, 16, 4, 16, 16, 4),
                                               (300, 200, 130, 208, 144, 133), (129, 129, 129, 144, 144, 129),
                                               (520, 384, 256, 384, 256, 256)])
def test_tensor_core_and_cuda_core_agree(torch_cuda, bits, m, k, n, lda, ldb, ldc):
    """The tensor-core multiplies (rows of A and B 16-byte aligned; INT8 with
    N and K of a full tile or more through the bulk tensor copies) against the
    CUDA-core kernel on the same full-range data, ragged
    tiles and K chunks included, and against the oracle."""
    torch = torch_cuda
    L = F.lib()
    rng = np.random.default_rng(m * 7 + k + n + bits)
    mx = (1 << (bits - 1)) - 1
    A = rng.integers(-mx - 1, mx + 1, (m, lda)).astype(NP[bits])
    B = rng.integers(-mx - 1, mx + 1, (k, ldb)).astype(NP[bits])
    Ad, Bd = torch.from_numpy(A).cuda(), torch.from_numpy(B).cuda()
    for sh in (0, 3, bits + 5, 2 * bits - 1, 4 * bits):
        mm = F.MatMul(m, k, n, DT[bits], shift=sh, lda=lda, ldb=ldb, ldc=ldc)
        outs = []
        for tc in (0, 1):
            L.FFTLIB_b200_FFT_setIntTensorCores(tc)
            try:
                Cd = torch.full((m, ldc), 5, dtype=Ad.dtype, device="cuda")
                mm.exec(Ad, Bd, Cd)
                outs.append(Cd.cpu().numpy())
            finally:
                L.FFTLIB_b200_FFT_setIntTensorCores(1)
        assert np.array_equal(outs[0], outs[1]), sh
        want = O.linalg_mm(bits, A[:, :k], B[:, :n], sh)
        assert np.array_equal(outs[1][:, :n], want), sh
        assert (outs[1][:, n:] == 5).all()
