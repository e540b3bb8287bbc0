"""The allocation-free c2c entry point (FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc).

It exists for callers that cannot allocate memory when they call the library
(a device-memory budget fixed at start-up, a real-time loop that must not
enter an allocator, a host whose allocator belongs to another runtime). It
keeps its twiddle table and error word in one static device array instead of
memory from cudaMalloc, so its results must equal those of the regular
_init/_kernel path. Collected last (file name) so a stop-at-first-failure run
has run every other test first; it needs nothing from them and also passes
alone in a fresh process.
"""
import numpy as np
import pytest

import c7x_fftlib_b200 as F
import fftcall
import oracle as O

pytestmark = pytest.mark.gpu
REL_L2 = 2e-6


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def no_alloc(torch, x, n, ch):
    X = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    Y = torch.zeros_like(X)
    torch.cuda.synchronize()
    st = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc")(F.ptr(X), F.ptr(Y), n, ch, None)
    F.check(st, "kernelNoAlloc")
    # the input stays unmodified
    np.testing.assert_array_equal(X.cpu().numpy(), np.asarray(x, np.float32))
    return Y.cpu().numpy()


def test_no_alloc_matches_kernel_on_consecutive_calls(torch):
    """Two (and more) calls in a row, with different lengths, each against the
    regular entry point and FP64."""
    for n, ch in [(4096, 300), (960, 7), (4096, 5), (16, 1000)]:
        x = O.uniform_c2c(n, ch, seed=n * 7 + ch)
        y = no_alloc(torch, x, n, ch)
        y_ref = fftcall.c2c(x, n, ch)
        assert O.rel_l2(y, O.as_complex(y_ref, n, ch)) <= REL_L2, (n, ch)
        assert O.rel_l2(y, O.fp64_c2c(x, n, ch)) <= REL_L2, (n, ch)


def test_no_alloc_allocates_no_device_memory(torch):
    """After a warm-up call of each length (CUDA loads a kernel's code on its
    first launch), calls of those lengths leave the device's free memory
    exactly unchanged."""
    fn = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc")
    cases = [(4096, 64), (960, 33), (16384, 4), (12, 500), (3000, 9)]
    bufs = [(torch.rand(2 * n * ch, device="cuda") * 2 - 1, torch.empty(2 * n * ch, device="cuda"), n, ch)
            for n, ch in cases]
    for x, y, n, ch in bufs:
        F.check(fn(F.ptr(x), F.ptr(y), n, ch, None), "kernelNoAlloc warm-up")
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for _ in range(2):
        for x, y, n, ch in bufs:
            F.check(fn(F.ptr(x), F.ptr(y), n, ch, None), "kernelNoAlloc")
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_no_alloc_rejects_lengths_beyond_its_scratch(torch):
    X = torch.zeros(2 * 31250, device="cuda")
    fn = F.fn("FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc")
    assert fn(F.ptr(X), F.ptr(X), 31250, 1, None) == F.FFTLIB_ERR_INVALID_DIMENSION
    assert "16384" in F.last_error()
    assert fn(F.ptr(X), F.ptr(X), 7, 1, None) == F.FFTLIB_ERR_INVALID_DIMENSION
