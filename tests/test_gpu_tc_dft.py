"""Split-precision tensor-core DFT through the fft_c7xmma coordinator API
(FFTLIB_FFT_fft_ixX_cxX_oxX_*), against the FP64 oracle: relative L2 error
<= 2e-6 per transform, for every tensor-core length, partial tiles, extreme
magnitudes and mixed-magnitude batches."""
import numpy as np
import pytest

import c7x_fftlib_b200 as F

pytestmark = pytest.mark.gpu

TOL = 2e-6
TC_SIZES = [8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096]


def _run(x: np.ndarray, n: int, batch: int, style=F.FFTLIB_FUNCTION_OPTIMIZED) -> tuple[np.ndarray, int]:
    import torch

    d = F.DftMma(n, batch, style)
    X = torch.from_numpy(np.ascontiguousarray(x, np.float32)).cuda()
    Y = torch.zeros_like(X)
    d.exec(X, Y)
    return Y.cpu().numpy(), d.path


def _per_transform_err(y, ref, n, batch):
    g = y.astype(np.float64).reshape(batch, 2 * n)
    ref = np.asarray(ref)
    if np.iscomplexobj(ref):
        c = ref.reshape(batch, n)
        r = np.empty((batch, 2 * n))
        r[:, 0::2], r[:, 1::2] = c.real, c.imag
    else:
        r = ref.reshape(batch, 2 * n)
    den = np.linalg.norm(r, axis=1)
    return np.linalg.norm(g - r, axis=1) / np.where(den == 0, 1, den)


@pytest.mark.parametrize("n", TC_SIZES)
def test_tc_dft_matches_fp64(oracle_mod, n):
    O = oracle_mod
    batch = 300  # not a multiple of any tile size
    x = O.uniform_c2c(n, batch, seed=n)
    y, path = _run(x, n, batch)
    assert path == F.MMA_PATH_TC
    ref = O.fp64_c2c(x, n, batch)
    assert O.rel_l2(y, ref) <= TOL
    assert _per_transform_err(y, ref, n, batch).max() <= TOL


@pytest.mark.parametrize("n", [16, 64, 256, 4096])
@pytest.mark.parametrize("scale", [1e-30, 1e-8, 1e8, 1e30])
def test_tc_dft_extreme_magnitudes(oracle_mod, n, scale):
    O = oracle_mod
    batch = 130
    x = (O.uniform_c2c(n, batch, seed=7) * scale).astype(np.float32)
    y, _ = _run(x, n, batch)
    ref = O.fp64_c2c(x, n, batch)
    assert np.isfinite(y).all()
    assert _per_transform_err(y, ref, n, batch).max() <= TOL


@pytest.mark.parametrize("n", [32, 128, 1024, 4096])
def test_tc_dft_mixed_magnitudes(oracle_mod, n):
    """Rows of very different size in one tile, an all-zero transform, and a
    transform with one huge point: the per-row and per-transform scaling
    keep each transform accurate on its own."""
    O = oracle_mod
    batch = 260
    rng = np.random.default_rng(11)
    x = O.uniform_c2c(n, batch, seed=3).reshape(batch, 2 * n)
    x *= (10.0 ** rng.uniform(-12, 12, size=(batch, 1))).astype(np.float32)
    x[5] = 0
    x[6, 10] = 3e20
    x = x.ravel().astype(np.float32)
    y, _ = _run(x, n, batch)
    ref = O.fp64_c2c(x, n, batch)
    err = _per_transform_err(y, ref, n, batch)
    assert err.max() <= TOL
    assert not y.reshape(batch, 2 * n)[5].any()


@pytest.mark.parametrize("n", [64, 4096])
def test_tc_dft_impulses_and_tones(n):
    """Known answers: the DFT of a unit impulse at m is W_n^(m k); of a pure
    tone at bin f, n at bin f and 0 elsewhere."""
    batch = 4
    t = np.arange(n)
    sig = np.zeros((batch, n), np.complex128)
    sig[0, 0] = 1
    sig[1, 3] = 1
    sig[2] = np.exp(2j * np.pi * 5 * t / n)
    sig[3] = np.exp(2j * np.pi * (n - 1) * t / n)
    x = np.empty((batch, 2 * n), np.float32)
    x[:, 0::2], x[:, 1::2] = sig.real, sig.imag
    y, _ = _run(x.ravel(), n, batch)
    yc = y.reshape(batch, 2 * n)
    got = yc[:, 0::2] + 1j * yc[:, 1::2]
    want = np.fft.fft(sig, axis=1)
    assert np.abs(got - want).max() <= 2e-6 * n


@pytest.mark.parametrize("n", [64, 1024])
def test_tc_dft_host_buffers_match_device(oracle_mod, n):
    O = oracle_mod
    batch = 200
    x = O.uniform_c2c(n, batch, seed=5)
    y_dev, _ = _run(x, n, batch)
    d = F.DftMma(n, batch, w_device=False)
    xh = np.array(x, np.float32)
    yh = np.zeros_like(xh)
    d.exec(xh, yh, d.w_host)
    assert np.array_equal(yh, y_dev)


def test_tc_dft_device_and_host_matrices_agree():
    for n in TC_SIZES:
        d = F.DftMma(n, 1)
        wd = d.w.cpu().numpy()
        assert np.abs(wd - d.w_host).max() <= 6e-8, n


@pytest.mark.parametrize("n", [48, 3000, 12, 4])
def test_coordinator_fft_path(oracle_mod, n):
    """Lengths without a tensor-core kernel take the CUDA-core FFT."""
    O = oracle_mod
    batch = 33
    x = O.uniform_c2c(n, batch, seed=2)
    y, path = _run(x, n, batch)
    assert path == F.MMA_PATH_FFT
    assert O.rel_l2(y, O.fp64_c2c(x, n, batch)) <= TOL


def test_coordinator_natc_style_uses_fft(oracle_mod):
    O = oracle_mod
    n, batch = 256, 64
    x = O.uniform_c2c(n, batch, seed=9)
    y_natc, p_natc = _run(x, n, batch, F.FFTLIB_FUNCTION_NATC)
    y_opt, p_opt = _run(x, n, batch, F.FFTLIB_FUNCTION_OPTIMIZED)
    assert (p_natc, p_opt) == (F.MMA_PATH_FFT, F.MMA_PATH_TC)
    ref = O.fp64_c2c(x, n, batch)
    assert O.rel_l2(y_natc, ref) <= TOL and O.rel_l2(y_opt, ref) <= TOL


def test_tc_dft_large_batch_properties():
    """Full-size batch (2^20 rows of 64 points): linearity and Parseval on
    the device, without the oracle."""
    import torch

    n, batch = 64, 1 << 20
    d = F.DftMma(n, batch)
    g = torch.Generator(device="cuda").manual_seed(1)
    a = torch.rand(2 * n * batch, device="cuda", generator=g) * 2 - 1
    b = torch.rand(2 * n * batch, device="cuda", generator=g) * 2 - 1
    ya, yb, yab = (torch.empty_like(a) for _ in range(3))
    d.exec(a, ya)
    d.exec(b, yb)
    d.exec(a + 2 * b, yab)
    lin = torch.linalg.norm(yab - (ya + 2 * yb)) / torch.linalg.norm(yab)
    assert float(lin) <= 4e-6
    pa = (ya.double() ** 2).view(batch, -1).sum(1) / n
    pt = (a.double() ** 2).view(batch, -1).sum(1)
    assert float(((pa - pt).abs() / pt).max()) <= 4e-6


def test_tc_handle_with_8_byte_aligned_buffers(oracle_mod):
    """Buffers that are 8- but not 16-byte aligned are transformed correctly
    (they take the CUDA-core FFT inside the same handle)."""
    import torch

    O = oracle_mod
    n, batch = 64, 100
    x = O.uniform_c2c(n, batch, seed=4)
    d = F.DftMma(n, batch)
    X = torch.zeros(2 * n * batch + 2, device="cuda")
    Y = torch.zeros_like(X)
    X[2:] = torch.from_numpy(x).cuda()
    d.exec(X[2:], Y[2:])
    assert O.rel_l2(Y[2:].cpu().numpy(), O.fp64_c2c(x, n, batch)) <= TOL
