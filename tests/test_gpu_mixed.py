"""Uneven-length batches (FFTLIB_b200_fftMixed_*): one persistent launch over
a descriptor table must give every transform the result of its own FFT."""
import os

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


def check_all(x, y, lengths, inverse=False):
    off = 0
    worst = 0.0
    segs = {}
    for i, n in enumerate(lengths):
        segs.setdefault(int(n), []).append(off)
        off += 2 * int(n)
    for n, offs in segs.items():
        xs = np.concatenate([x[o: o + 2 * n] for o in offs])
        ys = np.concatenate([y[o: o + 2 * n] for o in offs])
        err = O.rel_l2(ys, O.fp64_c2c(xs, n, len(offs), inverse))
        worst = max(worst, err)
        assert err <= REL_L2, (n, err)
    return worst


@pytest.mark.parametrize("inverse", [False, True])
def test_mixed_matches_fp64(torch, inverse):
    lengths = fftcall.mixed_lengths(3000, seed=4)
    total = int(lengths.sum())
    x = O.uniform_c2c(total, 1, seed=9)
    X = torch.from_numpy(x).cuda()
    Y = torch.zeros_like(X)
    mb = F.MixedBatch(lengths, inverse=inverse)
    mb.exec(X, Y)
    torch.cuda.synchronize()
    check_all(x, Y.cpu().numpy(), lengths, inverse)
    # one launch per length computes the same numbers
    Y2 = torch.zeros_like(X)
    mb.exec_per_size(X, Y2)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(Y.cpu().numpy(), Y2.cpu().numpy())
    mb.close()


def test_mixed_buffer_change_and_repeat(torch):
    lengths = np.array([12, 4096, 60, 60, 1536, 3000, 12, 960, 2880, 240] * 37, np.uint32)
    total = int(lengths.sum())
    mb = F.MixedBatch(lengths)
    for seed in (1, 2):
        x = O.uniform_c2c(total, 1, seed=seed)
        X = torch.from_numpy(x).cuda()
        Y = torch.zeros_like(X)
        for _ in range(2):
            mb.exec(X, Y)
        torch.cuda.synchronize()
        check_all(x, Y.cpu().numpy(), lengths)
    mb.close()


def test_mixed_every_allowed_length(torch):
    lengths = np.array(sorted(set(fftcall.mixed_lengths(20000, seed=1)) | {1, 2, 3, 4, 5, 8, 16, 25, 4096}),
                       np.uint32)
    total = int(lengths.sum())
    x = O.uniform_c2c(total, 1, seed=3)
    X = torch.from_numpy(x).cuda()
    Y = torch.zeros_like(X)
    mb = F.MixedBatch(lengths)
    mb.exec(X, Y)
    torch.cuda.synchronize()
    check_all(x, Y.cpu().numpy(), lengths)


def test_mixed_autotuned(torch, tmp_path, monkeypatch):
    monkeypatch.setenv("FFTLIB_B200_TUNE_CACHE", str(tmp_path / "tune.txt"))
    lengths = fftcall.mixed_lengths(500, seed=11)
    total = int(lengths.sum())
    x = O.uniform_c2c(total, 1, seed=12)
    X = torch.from_numpy(x).cuda()
    Y = torch.zeros_like(X)
    mb = F.MixedBatch(lengths, autotune=True)
    mb.exec(X, Y)
    torch.cuda.synchronize()
    check_all(x, Y.cpu().numpy(), lengths)
    assert os.path.exists(tmp_path / "tune.txt")
    assert len(open(tmp_path / "tune.txt").read().splitlines()) >= len(set(lengths.tolist())) - 1


def test_mixed_buffers_off_16_byte_boundary(torch):
    """pX and pY 8 bytes past a 16-byte boundary: no tile may be bulk-copied,
    the threads copy every tile in; results as for aligned buffers."""
    lengths = np.array([4096, 60, 60, 12, 3888, 960, 1536, 240] * 11, np.uint32)
    total = int(lengths.sum())
    x = O.uniform_c2c(total, 1, seed=21)
    X = torch.zeros(2 * total + 4, device="cuda")
    X[2:2 + 2 * total] = torch.from_numpy(x).cuda()
    Y = torch.zeros_like(X)
    mb = F.MixedBatch(lengths)
    mb.exec(X.data_ptr() + 8, Y.data_ptr() + 8)
    torch.cuda.synchronize()
    check_all(x, Y[2:2 + 2 * total].cpu().numpy(), lengths)
    mb.close()


@pytest.mark.parametrize("inverse", [False, True])
def test_mixed_grouped_and_persistent_agree(torch, inverse):
    """Lengths stored grouped (fixed-size kernels on grid shares) and the same
    batch in the single persistent kernel: both against FP64."""
    lengths = np.sort(fftcall.mixed_lengths(2000, seed=31))[::-1].copy()
    total = int(lengths.sum())
    x = O.uniform_c2c(total, 1, seed=32)
    X = torch.from_numpy(x).cuda()
    for po in (False, True):
        Y = torch.zeros_like(X)
        mb = F.MixedBatch(lengths, inverse=inverse, persistent_only=po)
        assert ("fixed-size groups" in mb.describe())
        mb.exec(X, Y)
        torch.cuda.synchronize()
        check_all(x, Y.cpu().numpy(), lengths, inverse)
        mb.close()


@pytest.mark.parametrize("branches", ["1", "3", "8"])
def test_mixed_chained_launches_on_branches(torch, monkeypatch, branches):
    """The fixed-size groups' launches chained by programmatic dependent
    launch, on one branch (the default) or spread over several, replayed
    twice from the graph: every transform against FP64."""
    monkeypatch.setenv("FFTLIB_B200_MIXED_BRANCHES", branches)
    lengths = np.sort(fftcall.mixed_lengths(3000, seed=77))[::-1].copy()
    total = int(lengths.sum())
    x = O.uniform_c2c(total, 1, seed=78)
    X = torch.from_numpy(x).cuda()
    Y = torch.zeros_like(X)
    mb = F.MixedBatch(lengths)
    for _ in range(2):
        mb.exec(X, Y)
    torch.cuda.synchronize()
    check_all(x, Y.cpu().numpy(), lengths, False)
    mb.close()
