"""FP32 parity of the CUDA kernels (through the FFTLIB C API) against the
oracle, the reference's own _cn code, its golden vectors and FP64.

Tolerances, as the reference's tests and the FP32 target state them:
* relative L2 error against the FP64 transform <= 2e-6;
* c2c / ifft c2c: max abs difference to the reference _cn <= 2^-5 on inputs
  of magnitude 256 (FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_d.c:304-311);
* r2c: 2^-3, c2r: 1e-3 absolute against the committed static vectors
  (..._i32f_c32fc_o32fc_d.c:208-234, ..._ifft1dBatched_i32fc_c32fc_o32f_d.c:196-201).
"""
import os

import numpy as np
import pytest

import fftcall
import oracle as O

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
REL_L2 = 2e-6
ABS_C2C = 2.0 ** -5

# every c2c size of the reference test lists
# (test/fft_c7x/FFTLIB_idat_gen/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/test_cases_list.csv)
REF_C2C_SIZES = [1, 2, 3, 4, 5, 8, 9, 15, 16, 18, 25, 27, 32, 36, 45, 50, 64, 72, 81, 96, 100, 125, 128, 135, 144,
                 160, 192, 200, 243, 256, 320, 384, 400, 512, 576, 625, 640, 800, 864, 960, 1024, 1152, 1280, 1440,
                 1600, 1728, 1920, 2048, 2430, 2560, 2592, 2880, 3125, 3200, 4000, 4096, 4374, 6075, 6250, 6400,
                 6561, 8000, 8192, 10935, 13122, 15625, 19683, 21870, 31250]


def _channels(n):
    return 3 if n <= 4096 else 2


@pytest.fixture(scope="module")
def gpu():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.mark.parametrize("n", REF_C2C_SIZES)
def test_c2c_fwd_vs_fp64_and_oracle(gpu, n):
    ch = _channels(n)
    x = O.uniform_c2c(n, ch, seed=n)
    y = fftcall.c2c(x, n, ch)
    assert O.rel_l2(y, O.fp64_c2c(x, n, ch)) <= REL_L2
    yo = O.fft_c2c_f32(x, n, ch)
    assert O.rel_l2(y, O.as_complex(yo, n, ch)) <= REL_L2


@pytest.mark.parametrize("n", REF_C2C_SIZES)
def test_ifft_c2c_vs_fp64(gpu, n):
    ch = _channels(n)
    x = O.uniform_c2c(n, ch, seed=7 * n + 1)
    y = fftcall.c2c(x, n, ch, inverse=True)
    assert O.rel_l2(y, O.fp64_c2c(x, n, ch, inverse=True)) <= REL_L2


@pytest.mark.parametrize("n,ch", [(256, 16), (4096, 4), (960, 8), (64, 512), (3000, 2), (12, 33), (8192, 2),
                                  (30, 7), (6561, 1)])
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_vs_reference_cn(gpu, ref_cn, n, ch, inverse):
    x = O.uniform_c2c(n, ch, seed=11 * n + ch, lo=-256.0, hi=256.0)
    y = fftcall.c2c(x, n, ch, inverse=inverse)
    yr = O.ref_c2c_f32(x, n, ch, inverse)
    assert np.abs(y - yr).max() <= ABS_C2C
    assert O.rel_l2(y, O.fp64_c2c(x, n, ch, inverse)) <= REL_L2


@pytest.mark.parametrize("n,ch", [(4096, 1), (4096, 297), (4096, 1000), (2048, 593), (8192, 300), (16384, 150),
                                  (1024, 777), (960, 301)])
def test_c2c_batch_counts(gpu, n, ch):
    """Batch counts below, around and above the number of persistent CTAs
    (148 SMs x resident CTAs) exercise the pipelined kernels' tile loop."""
    x = O.uniform_c2c(n, ch, seed=n + ch)
    for inverse in (False, True):
        y = fftcall.c2c(x, n, ch, inverse=inverse)
        assert O.rel_l2(y, O.fp64_c2c(x, n, ch, inverse)) <= REL_L2


def test_c2c_golden_ref_cn(gpu):
    d = np.load(os.path.join(GOLD, "ref_cn.npz"))
    for i in range(int(d["c2c_n"])):
        ch, n = (int(v) for v in d[f"c2c{i}_meta"])
        x = d[f"c2c{i}_in"]
        for inv, key in ((False, "fwd"), (True, "inv")):
            y = fftcall.c2c(x, n, ch, inverse=inv)
            assert np.abs(y - d[f"c2c{i}_{key}"]).max() <= ABS_C2C, (n, ch, key)


def test_c2c_golden_pymodel(gpu):
    d = np.load(os.path.join(GOLD, "c2c_pymodel.npz"))
    for i in range(int(d["n_cases"])):
        ch, n = (int(v) for v in d[f"case{i}_meta"])
        x = d[f"case{i}_in"]
        for inv, key in ((False, "fwd"), (True, "inv")):
            y = fftcall.c2c(x, n, ch, inverse=inv)
            ref = d[f"case{i}_{key}"]
            # golden values are rounded to 6 decimals by the reference generator
            assert np.abs(y - ref).max() <= 1e-5 + 1e-6 * np.abs(ref).max(), (n, ch, key)


def test_c2c_headline_size_properties(gpu):
    """N=4096 x 8192 (the benchmark size): sampled channels against FP64,
    linearity and inverse(forward(x)) == x over the whole batch."""
    torch = gpu
    import c7x_fftlib_b200 as F

    n, ch = 4096, 8192
    g = torch.Generator(device="cuda").manual_seed(1)
    x = torch.rand(2 * n * ch, device="cuda", generator=g) * 2 - 1
    x2 = torch.rand(2 * n * ch, device="cuda", generator=g) * 2 - 1
    w = torch.zeros(2 * n, device="cuda")
    bX, bW = F.bp(F.FFTLIB_FLOAT32, 2 * n * ch), F.bp(F.FFTLIB_FLOAT32, 2 * n)

    def run(kind, inp):
        out = torch.empty_like(inp)
        src = inp.clone()
        pb = F.pblock(kind)
        base = F.KERNELS[kind]
        F.check(F.fn(base + "_init")(F.ptr(src), bX, F.ptr(w), bW, F.ptr(out), bX, n, ch, pb))
        F.check(F.fn(base + "_kernel")(F.ptr(src), bX, F.ptr(w), bW, F.ptr(out), bX, n, ch, pb))
        return out

    y = run("c2c", x)
    idx = np.linspace(0, ch - 1, 16).astype(int)
    xs = x.view(ch, 2 * n)[idx].cpu().numpy().ravel()
    ys = y.view(ch, 2 * n)[idx].cpu().numpy().ravel()
    assert O.rel_l2(ys, O.fp64_c2c(xs, n, len(idx))) <= REL_L2
    # linearity: F(x + 2 x2) = F(x) + 2 F(x2)
    y2 = run("c2c", x2)
    ysum = run("c2c", x + 2 * x2)
    err = torch.linalg.norm(ysum - (y + 2 * y2)) / torch.linalg.norm(ysum)
    assert float(err) <= 4 * REL_L2
    # round trip
    xr = run("ifft", y)
    err = torch.linalg.norm(xr - x) / torch.linalg.norm(x)
    assert float(err) <= 2 * REL_L2


@pytest.mark.parametrize("n", [2, 4, 6, 10, 12, 18, 30, 50, 64, 128, 250, 256, 480, 960, 1024, 2304, 4096, 5760, 8192,
                               12800, 16000, 26244, 62500, 118098])
@pytest.mark.parametrize("mode", [0, 1])
def test_r2c_c2r_vs_fp64(gpu, n, mode):
    ch = 3 if n <= 8192 else 2
    x = O.real_signal(n, ch, seed=n + mode)
    y = fftcall.r2c(x, n, ch, outmode=mode)
    nout = n if mode else n // 2 + 1
    assert O.rel_l2(O.as_complex(y, nout, ch), O.fp64_r2c(x, n, ch, mode)) <= REL_L2
    xr = fftcall.c2r(y, n, ch, inmode=mode)
    assert O.rel_l2(xr, O.fp64_c2r(y, n, ch, mode).ravel()) <= REL_L2
    assert O.rel_l2(xr, x) <= REL_L2


@pytest.mark.parametrize("n", [27648, 28800, 32000, 32768])
def test_c2r_full_spectrum_longest_single_kernel(gpu, n):
    """inMode 1 at the longest single-kernel half lengths (13824..16384),
    whose staged full-spectrum row exceeds a CTA's shared memory: the split
    runs as a pre-pass into pXFFT."""
    x = O.real_signal(n, 2, seed=n + 3)
    y = fftcall.r2c(x, n, 2, outmode=1)
    assert O.rel_l2(O.as_complex(y, n, 2), O.fp64_r2c(x, n, 2, 1)) <= REL_L2
    xr = fftcall.c2r(y, n, 2, inmode=1)
    assert O.rel_l2(xr, O.fp64_c2r(y, n, 2, 1).ravel()) <= REL_L2


@pytest.mark.parametrize("n,ch,mode", [(4096, 2, 0), (4096, 2, 1), (480, 3, 0), (250, 1, 1), (64, 4, 0), (6, 2, 0)])
def test_r2c_c2r_vs_reference_cn(gpu, ref_cn, n, ch, mode):
    x = O.real_signal(n, ch, seed=4000 + n)
    y = fftcall.r2c(x, n, ch, outmode=mode)
    yr = O.ref_r2c_f32(x, n, ch, mode)
    assert np.abs(y - yr).max() <= 2.0 ** -3
    xr = fftcall.c2r(yr, n, ch, inmode=mode)
    assert np.abs(xr - O.ref_c2r_f32(yr, n, ch, mode)).max() <= 1e-3


def test_r2c_extended_golden(gpu):
    d = np.load(os.path.join(GOLD, "r2c_extended.npz"))
    for cid, ch, n, mode in zip(d["ids"], d["channels"], d["points"], d["mode"]):
        y = fftcall.r2c(d[f"in_{cid}"], int(n), int(ch), outmode=int(mode))
        assert np.abs(y - d[f"out_{cid}"]).max() <= 2.0 ** -3, cid


def test_c2r_extended_golden(gpu):
    d = np.load(os.path.join(GOLD, "c2r_extended.npz"))
    for cid, ch, n, mode in zip(d["ids"], d["channels"], d["points"], d["mode"]):
        y = fftcall.c2r(d[f"in_{cid}"], int(n), int(ch), inmode=int(mode))
        assert np.abs(y - d[f"out_{cid}"]).max() <= 1e-3, cid


def test_rc_golden_ref_cn(gpu):
    d = np.load(os.path.join(GOLD, "ref_cn.npz"))
    for i in range(int(d["rc_n"])):
        ch, n, mode = (int(v) for v in d[f"rc{i}_meta"])
        y = fftcall.r2c(d[f"rc{i}_in"], n, ch, outmode=mode)
        assert np.abs(y - d[f"rc{i}_r2c"]).max() <= 2.0 ** -3
        xr = fftcall.c2r(d[f"rc{i}_r2c"], n, ch, inmode=mode)
        assert np.abs(xr - d[f"rc{i}_c2r"]).max() <= 1e-3


@pytest.mark.parametrize("n,ch", [(4096, 5), (60, 9), (31250, 1)])
def test_host_buffers_match_device(gpu, n, ch):
    """Host (numpy) buffers go through the staged path and give the same
    result as device buffers."""
    x = O.uniform_c2c(n, ch, seed=99)
    yd = fftcall.c2c(x, n, ch)
    yh = fftcall.c2c(x, n, ch, on_device=False)
    np.testing.assert_array_equal(yd, yh)


def test_cn_entry_points_run_the_same_path(gpu):
    n, ch = 960, 4
    x = O.uniform_c2c(n, ch, seed=5)
    np.testing.assert_array_equal(fftcall.c2c(x, n, ch), fftcall.c2c(x, n, ch, entry="cn"))
