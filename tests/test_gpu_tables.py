"""The table generators on the GPU (FFTLIB_b200_*_device and the device
form of the coordinator's twGen) against the host generators, which
reproduce the reference's tables bit for bit: every FP32 stage-twiddle,
Q15 and split-factor table of the reference test lists' lengths, and the
dftLarge matrix, compared as raw bytes including the entries the generators
leave unwritten."""
import ctypes as C

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def lengths_235(limit):
    out = []
    for a in range(0, 21):
        for b in range(0, 13):
            for c in range(0, 9):
                n = 2 ** a * 3 ** b * 5 ** c
                if n <= limit:
                    out.append(n)
    return sorted(out)


def _compare(torch, host_fn, dev_fn, n_elems, np_dt, arg):
    host = np.full(n_elems, 7, np_dt)
    host_fn(F.ptr(host), arg)
    dev = torch.full((n_elems,), 7, dtype={np.float32: torch.float32, np.int16: torch.int16}[np_dt], device="cuda")
    assert dev_fn(F.ptr(dev), arg, None) == F.FFTLIB_SUCCESS
    torch.cuda.synchronize()
    got = dev.cpu().numpy()
    return np.array_equal(host.view(np.uint8), got.view(np.uint8))


def test_stage_twiddles_c2c(torch_cuda):
    L = F.lib()
    bad = [n for n in lengths_235(1 << 16) + [1 << 20, 3 * (1 << 18), 78125, 5 ** 8]
           if not _compare(torch_cuda, L.FFTLIB_b200_tw_gen_c2c, L.FFTLIB_b200_tw_gen_c2c_device, 2 * n + 2,
                           np.float32, n)]
    assert not bad, bad


def test_q15_twiddles(torch_cuda):
    L = F.lib()
    bad = [n for n in [1 << k for k in range(0, 21)]
           if not _compare(torch_cuda, L.FFTLIB_b200_tw_gen_i16, L.FFTLIB_b200_tw_gen_i16_device, 2 * n + 2,
                           np.int16, n)]
    assert not bad, bad
    import torch

    d = torch.zeros(256, dtype=torch.int16, device="cuda")
    assert L.FFTLIB_b200_tw_gen_i16_device(F.ptr(d), 96, None) == F.FFTLIB_ERR_INVALID_DIMENSION


@pytest.mark.parametrize("host,dev", [("tw_gen_r2c", "FFTLIB_b200_tw_gen_r2c_device"),
                                      ("split_factor_gen_r2c", "FFTLIB_b200_split_factor_gen_r2c_device"),
                                      ("ifft_c2r_tw_gen", "FFTLIB_b200_ifft_c2r_tw_gen_device"),
                                      ("ifft_c2r_split_factor_gen",
                                       "FFTLIB_b200_ifft_c2r_split_factor_gen_device")])
def test_r2c_c2r_tables(torch_cuda, host, dev):
    L = F.lib()
    ns = [2 * n for n in lengths_235(1 << 15)] + [1 << 21, 2 * 78125]
    bad = [n for n in ns if not _compare(torch_cuda, getattr(L, host), getattr(L, dev), 2 * n + 2, np.float32, n)]
    assert not bad, bad


def test_device_generators_refuse_host_memory(torch_cuda):
    L = F.lib()
    buf = np.zeros(64, np.float32)
    assert L.FFTLIB_b200_tw_gen_c2c_device(F.ptr(buf), 16, None) == F.FFTLIB_ERR_INVALID_VALUE
    assert L.FFTLIB_b200_tw_gen_c2c_device(None, 16, None) == F.FFTLIB_ERR_NULL_POINTER
    import torch

    d = torch.zeros(64, device="cuda")
    assert L.FFTLIB_b200_split_factor_gen_r2c_device(F.ptr(d), -4, None) == F.FFTLIB_ERR_INVALID_DIMENSION


@pytest.mark.parametrize("bits", [16, 32])
@pytest.mark.parametrize("n,il", [(32, 1), (64, 0), (40, 1), (200, 1), (1000, 0)])
def test_dft_large_matrix_on_the_device(torch_cuda, bits, n, il):
    import torch

    dt = {16: F.FFTLIB_INT16, 32: F.FFTLIB_INT32}[bits]
    pre, t = F.DFT_VARIANTS["dftLarge"]
    a = t(1, n, 2, il)
    bw = F.BufParams(dt, 4 * n * n)
    w = torch.zeros(4 * n * n, dtype={16: torch.int16, 32: torch.int32}[bits], device="cuda")
    assert getattr(F.lib(), pre + "twGen")(C.byref(a), F.ptr(w), C.byref(bw)) == F.FFTLIB_SUCCESS
    assert np.array_equal(w.cpu().numpy(), O.mma_twgen(bits, n, 2, il, 2))
