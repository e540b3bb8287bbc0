"""The batched-path autotuner (FFTLIB_B200_AUTOTUNE=1): _init times the
launch candidates of its call shape (radix schedule, transforms per CTA,
persistent kernel and its CTA count; for int16 the threads per transform and
CTA count), records the winner in pBlock and in the cache file
(FFTLIB_B200_TUNE_CACHE), and the tuned launch is parity-green:

* FP32 c2c / ifft / r2c / c2r against the GPU FP64 oracle, relative L2 error
  <= 2e-6 for the whole batch and for every transform on its own;
* int16 bit-exact with the CPU oracle.

The reference takes the same decision -- how to factor N into stages -- once
per length in _init (FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_ci.cpp:99-118).
"""
import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

pytestmark = pytest.mark.gpu
REL_L2 = 2e-6


@pytest.fixture(scope="module")
def torch():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    return torch


@pytest.fixture
def tuning(tmp_path, monkeypatch):
    path = tmp_path / "tune.txt"
    monkeypatch.setenv("FFTLIB_B200_AUTOTUNE", "1")
    monkeypatch.setenv("FFTLIB_B200_TUNE_CACHE", str(path))
    return path


def bucket(batch):
    b = 1
    while b < batch and b < (1 << 20):
        b <<= 2
    return b


def cache_lines(path, n, batch, tag):
    if not path.exists():
        return []
    return [ln for ln in path.read_text().splitlines() if f"|{n}|{bucket(batch)}|{tag} " in ln + " "]


def c2c_init_run(torch, kind, x, n, ch):
    w = torch.zeros(2 * n, device="cuda")
    bX, bW = F.bp(F.FFTLIB_FLOAT32, 2 * n * ch), F.bp(F.FFTLIB_FLOAT32, 2 * n)
    out = torch.empty_like(x)
    src = x.clone()
    pb = F.pblock(kind)
    base = F.KERNELS[kind]
    F.check(F.fn(base + "_init")(F.ptr(src), bX, F.ptr(w), bW, F.ptr(out), bX, n, ch, pb))
    F.check(F.fn(base + "_kernel")(F.ptr(src), bX, F.ptr(w), bW, F.ptr(out), bX, n, ch, pb))
    return out, F.describe_block(pb)


@pytest.mark.parametrize("kind", ["c2c", "ifft"])
@pytest.mark.parametrize("n,ch", [(4096, 8192), (1024, 3000), (3000, 64), (720, 1000), (64, 20000), (16, 3)])
def test_tuned_c2c_cache_written_and_parity(torch, tuning, kind, n, ch):
    g = torch.Generator(device="cuda").manual_seed(n + ch)
    x = torch.rand(2 * n * ch, device="cuda", generator=g) * 2 - 1
    y, desc = c2c_init_run(torch, kind, x, n, ch)
    assert desc.startswith("tuned: "), desc
    lines = cache_lines(tuning, n, ch, f"{kind}:f32")
    assert len(lines) == 1, tuning.read_text() if tuning.exists() else "no cache file"
    overall, worst = O.gpu_check_c2c(x, y, n, ch, inverse=(kind == "ifft"))
    assert overall <= REL_L2 and worst <= REL_L2, (desc, overall, worst)


def test_tuned_choice_read_back_from_the_file(torch, tuning, tmp_path, monkeypatch):
    """A second cache path holding the first one's entry: the choice comes
    from the file (no new line is timed and appended) and is the same."""
    n, ch = 2048, 4000
    x = torch.rand(2 * n * ch, device="cuda") * 2 - 1
    _, desc = c2c_init_run(torch, "c2c", x, n, ch)
    line = cache_lines(tuning, n, ch, "c2c:f32")
    assert len(line) == 1
    second = tmp_path / "second.txt"
    second.write_text(line[0] + "\n")
    monkeypatch.setenv("FFTLIB_B200_TUNE_CACHE", str(second))
    y, desc2 = c2c_init_run(torch, "c2c", x, n, ch)
    assert desc2 == desc
    assert second.read_text().splitlines() == [line[0]]
    overall, worst = O.gpu_check_c2c(x, y, n, ch)
    assert overall <= REL_L2 and worst <= REL_L2


def test_stale_cache_entry_is_ignored(torch, tuning, monkeypatch):
    """An entry naming a schedule that is not a candidate (here 3 x 5 for
    N = 1000) is not used: the call shape is timed again and a valid line
    appended."""
    n, ch = 1000, 500
    x = torch.rand(2 * n * ch, device="cuda") * 2 - 1
    c2c_init_run(torch, "c2c", x, n, ch)  # learns this device's key
    key = cache_lines(tuning, n, ch, "c2c:f32")[0].split(" ")[0]
    tuning.write_text(f"{key} 16 8 2 3 5 0 0 0\n")
    # a detour through another path makes the tuner re-read the edited file
    monkeypatch.setenv("FFTLIB_B200_TUNE_CACHE", str(tuning) + ".b")
    c2c_init_run(torch, "c2c", x, n, ch)
    monkeypatch.setenv("FFTLIB_B200_TUNE_CACHE", str(tuning))
    y, desc = c2c_init_run(torch, "c2c", x, n, ch)
    assert desc.startswith("tuned: ")
    lines = cache_lines(tuning, n, ch, "c2c:f32")
    assert len(lines) == 2 and lines[0].endswith(" 16 8 2 3 5 0 0 0"), lines
    overall, worst = O.gpu_check_c2c(x, y, n, ch)
    assert overall <= REL_L2 and worst <= REL_L2


def real_workload(torch, n, ch, seed):
    g = torch.Generator(device="cuda").manual_seed(seed)
    return torch.randn(ch * n, device="cuda", generator=g)


@pytest.mark.parametrize("n,ch,mode", [(4096, 2048, 0), (1000, 700, 1), (64, 5000, 0), (250, 33, 1)])
def test_tuned_r2c_c2r_cache_written_and_parity(torch, tuning, n, ch, mode):
    h = n // 2
    bins = n if mode else h + 1
    x = real_workload(torch, n, ch, seed=n)
    yc = torch.empty(2 * bins * ch, device="cuda")
    xb = torch.empty(n * ch, device="cuda")
    work = torch.empty(n * ch, device="cuda")
    b = F.bp(F.FFTLIB_FLOAT32, n * ch)  # the reference's checks want every buffer's dim_x equal
    pr, pc = F.pblock("r2c"), F.pblock("c2r")
    F.check(F.fn(F.KERNELS["r2c"] + "_init")(F.ptr(x), b, F.ptr(x), b, F.ptr(work), b, F.ptr(x), b, F.ptr(yc), b, n,
                                             ch, mode, pr))
    F.check(F.fn(F.KERNELS["c2r"] + "_init")(F.ptr(yc), b, F.ptr(yc), b, F.ptr(work), b, F.ptr(yc), b, F.ptr(xb), b,
                                             n, ch, mode, pc))
    for pb, tag in ((pr, f"r2c:f32:m{mode}"), (pc, f"c2r:f32:m{mode}")):
        assert F.describe_block(pb).startswith("tuned: ")
        assert len(cache_lines(tuning, h, ch, tag)) == 1, tag
    st = torch.cuda.current_stream().cuda_stream
    F.check(F.fn("FFTLIB_b200_fft1dBatched_i32f_c32fc_o32fc_kernelAsync")(F.ptr(x), F.ptr(work), F.ptr(yc), n, ch,
                                                                          mode, pr, F.ptr(st)))
    yc_in = yc.clone()
    F.check(F.fn("FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32f_kernelAsync")(F.ptr(yc), F.ptr(work), F.ptr(xb), n, ch,
                                                                           mode, pc, F.ptr(st)))
    torch.cuda.synchronize()
    ref = O.gpu_fp64_r2c(x.view(ch, n), n, ch, mode)
    overall, worst = O.gpu_rel_l2_rows(yc.view(ch, bins, 2), ref, ch)
    assert overall <= REL_L2 and worst <= REL_L2, ("r2c", overall, worst)
    ref = O.gpu_fp64_c2r(yc_in.view(ch, bins, 2), n, ch, mode)
    overall, worst = O.gpu_rel_l2_rows(xb.view(ch, n), ref, ch)
    assert overall <= REL_L2 and worst <= REL_L2, ("c2r", overall, worst)


@pytest.mark.parametrize("n,ch", [(1024, 4096), (4096, 300), (64, 2000), (16384, 20)])
def test_tuned_i16_cache_written_and_bit_exact(torch, tuning, n, ch):
    nsh = 0
    m = n
    while m > 2:
        nsh, m = nsh + 1, m // 4
    sh = np.full(nsh, 2, np.uint32)
    x = O.int16_input(n, ch, 77 + n)
    w = np.zeros(2 * n, np.int16)
    F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
    X = torch.from_numpy(x).cuda()
    W = torch.from_numpy(w).cuda()
    Y = torch.zeros(2 * n * ch, dtype=torch.int16, device="cuda")
    S = torch.from_numpy(sh.view(np.int32)).cuda()
    dim = 2 * n * ch
    bX, bW, bS = F.bp(F.FFTLIB_INT16, dim), F.bp(F.FFTLIB_INT16, 2 * n), F.bp(F.FFTLIB_UINT32, nsh)
    pb = F.pblock("i16")
    base = F.KERNELS["i16"]
    args = (F.ptr(X), bX, F.ptr(W), bW, F.ptr(Y), bX, F.ptr(S), bS, n, ch)
    F.check(F.fn(base + "_init")(*args, pb))
    assert F.describe_block(pb).startswith("tuned: int16")
    assert len(cache_lines(tuning, n, ch, "c2c:i16")) == 1
    F.check(F.fn(base + "_kernel")(*args, pb))
    np.testing.assert_array_equal(Y.cpu().numpy(), O.fft_c2c_i16(x, n, ch, sh))


def test_untuned_block_says_planner(torch, monkeypatch):
    monkeypatch.delenv("FFTLIB_B200_AUTOTUNE", raising=False)
    n, ch = 4096, 16
    x = torch.rand(2 * n * ch, device="cuda") * 2 - 1
    _, desc = c2c_init_run(torch, "c2c", x, n, ch)
    assert desc.startswith("planner: ") and "fixed-size pipelined kernel" in desc, desc


@pytest.mark.parametrize("n,ch", [(32, 20000), (16, 30000), (1024, 4096), (256, 3000)])
def test_i16_64_register_build_bit_exact(torch, tuning, n, ch):
    """A cache entry selects the int16 kernel built for 64 registers (four
    CTAs per SM) when shared memory admits a fourth CTA; that build is
    bit-exact too. Lengths 64...4096 have fixed-length kernels: whether their
    64-register build admits more CTAs than the default one depends on both
    builds' register counts, so there the entry may be a candidate or be
    timed afresh; either way the result is bit-exact."""
    nsh = 0
    m = n
    while m > 2:
        nsh, m = nsh + 1, m // 4
    sh = np.full(nsh, 2, np.uint32)
    dev = torch.cuda.get_device_name(0).replace(" ", "_")
    tgs = [t for t in (n // 16, n // 32, n // 64) if t >= 1]
    tuning.write_text("".join(f"{dev}|{n}|{bucket(ch)}|c2c:i16 {tg} 0 4\n" for tg in tgs[::-1]))
    x = O.int16_input(n, ch, 5 + n)
    w = np.zeros(2 * n, np.int16)
    F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
    X, W = torch.from_numpy(x).cuda(), torch.from_numpy(w).cuda()
    Y = torch.zeros(2 * n * ch, dtype=torch.int16, device="cuda")
    S = torch.from_numpy(sh.view(np.int32)).cuda()
    bX, bW, bS = F.bp(F.FFTLIB_INT16, 2 * n * ch), F.bp(F.FFTLIB_INT16, 2 * n), F.bp(F.FFTLIB_UINT32, nsh)
    pb = F.pblock("i16")
    args = (F.ptr(X), bX, F.ptr(W), bW, F.ptr(Y), bX, F.ptr(S), bS, n, ch)
    F.check(F.fn(F.KERNELS["i16"] + "_init")(*args, pb))
    desc = F.describe_block(pb)
    F.check(F.fn(F.KERNELS["i16"] + "_kernel")(*args, pb))
    np.testing.assert_array_equal(Y.cpu().numpy(), O.fft_c2c_i16(x, n, ch, sh))
    if n < 64:
        assert "64 registers" in desc, desc
