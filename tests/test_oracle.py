"""The oracle is pinned before anything is checked against it: its tables and
kernels against the reference's own _cn code (compiled from the reference
sources into oracle/_ref) and against the committed golden vectors."""
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")
C2C_SIZES = [1, 2, 3, 4, 5, 6, 8, 9, 12, 15, 16, 25, 27, 30, 60, 64, 96, 125, 240, 256, 625, 960, 1024, 1536, 3000,
             4096, 6561, 15625]


@pytest.mark.parametrize("n", C2C_SIZES + [31250])
def test_twiddle_table_bit_exact(ref_cn, n):
    a, b = O.tw_gen_f32(n), O.ref_tw_gen_c2c(n)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("n", [2, 4, 8, 12, 20, 64, 128, 480, 4096, 62500])
def test_real_tables_bit_exact(ref_cn, n):
    assert np.array_equal(O.tw_gen_f32(n // 2), O.ref_tw_gen_r2c(n))
    assert np.array_equal(O.tw_gen_f32(n // 2), O.ref_tw_gen_c2r(n))
    assert np.array_equal(O.split_factor_r2c(n), O.ref_split_factor_r2c(n))
    assert np.array_equal(O.split_factor_c2r(n), O.ref_split_factor_c2r(n))


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048, 4096])
def test_q15_table_bit_exact(ref_cn, n):
    assert np.array_equal(O.tw_gen_i16(n), O.ref_tw_gen_i16(n))


@pytest.mark.parametrize("n", C2C_SIZES)
@pytest.mark.parametrize("inverse", [False, True])
def test_c2c_oracle_vs_reference(ref_cn, n, inverse):
    ch = 3
    x = O.uniform_c2c(n, ch, seed=n)
    a = O.fft_c2c_f32(x, n, ch, inverse)
    b = O.ref_c2c_f32(x, n, ch, inverse)
    f = O.fp64_c2c(x, n, ch, inverse)
    assert O.rel_l2(a, f) <= 2e-6
    assert O.rel_l2(b, f) <= 2e-6
    assert O.rel_l2(a, O.as_complex(b, n, ch)) <= 2e-6


@pytest.mark.parametrize("n", [2, 4, 8, 10, 12, 64, 128, 250, 480, 1024, 4096])
@pytest.mark.parametrize("mode", [0, 1])
def test_real_oracle_vs_reference(ref_cn, n, mode):
    ch = 2
    x = O.real_signal(n, ch, 7)
    nout = n if mode else n // 2 + 1
    a, b = O.fft_r2c_f32(x, n, ch, mode), O.ref_r2c_f32(x, n, ch, mode)
    f = O.fp64_r2c(x, n, ch, mode)
    assert O.rel_l2(O.as_complex(a, nout, ch), f) <= 2e-6
    assert O.rel_l2(O.as_complex(b, nout, ch), f) <= 2e-6
    a2, b2 = O.fft_c2r_f32(a, n, ch, mode), O.ref_c2r_f32(a, n, ch, mode)
    f2 = O.fp64_c2r(a, n, ch, mode).ravel()
    assert O.rel_l2(a2, f2) <= 2e-6
    assert O.rel_l2(b2, f2) <= 2e-6
    assert O.rel_l2(a2, x) <= 2e-6


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 64, 128, 256, 512, 1024, 2048])
def test_i16_oracle_bit_exact_vs_reference(ref_cn, n):
    rng = np.random.default_rng(0)
    ns, m = 0, n
    while m > 2:
        ns, m = ns + 1, m // 4
    for trial in range(4):
        sh = rng.integers(0, 4, max(ns, 1)).astype(np.uint32)
        lo, hi = [(-2048, 2047), (-32768, 32767)][trial % 2]
        x = O.int16_input(n, 3, trial + n, lo, hi)
        assert np.array_equal(O.fft_c2c_i16(x, n, 3, sh), O.ref_c2c_i16(x, n, 3, sh))


def test_oracle_vs_golden_ref_cn():
    d = np.load(os.path.join(GOLD, "ref_cn.npz"))
    for i in range(int(d["c2c_n"])):
        ch, n = (int(v) for v in d[f"c2c{i}_meta"])
        for inv, key in ((False, "fwd"), (True, "inv")):
            y = O.fft_c2c_f32(d[f"c2c{i}_in"], n, ch, inv)
            assert np.abs(y - d[f"c2c{i}_{key}"]).max() <= 2.0 ** -5
    for i in range(int(d["rc_n"])):
        ch, n, mode = (int(v) for v in d[f"rc{i}_meta"])
        assert np.abs(O.fft_r2c_f32(d[f"rc{i}_in"], n, ch, mode) - d[f"rc{i}_r2c"]).max() <= 2.0 ** -3
        assert np.abs(O.fft_c2r_f32(d[f"rc{i}_r2c"], n, ch, mode) - d[f"rc{i}_c2r"]).max() <= 1e-3
    for i in range(int(d["i16_n"])):
        ch, n = (int(v) for v in d[f"i16{i}_meta"])
        y = O.fft_c2c_i16(d[f"i16{i}_in"], n, ch, d[f"i16{i}_shift"])
        assert np.array_equal(y, d[f"i16{i}_out"])


def test_oracle_vs_golden_pymodels():
    d = np.load(os.path.join(GOLD, "i16_pymodel.npz"))
    for i in range(int(d["n_cases"])):
        ch, n = (int(v) for v in d[f"case{i}_meta"])
        assert np.array_equal(O.tw_gen_i16(n), d[f"case{i}_tw"])
        assert np.array_equal(O.fft_c2c_i16(d[f"case{i}_in"], n, ch, d[f"case{i}_shift"]), d[f"case{i}_out"])
    d = np.load(os.path.join(GOLD, "c2c_pymodel.npz"))
    for i in range(int(d["n_cases"])):
        ch, n = (int(v) for v in d[f"case{i}_meta"])
        for inv, key in ((False, "fwd"), (True, "inv")):
            ref = d[f"case{i}_{key}"]
            y = O.fft_c2c_f32(d[f"case{i}_in"], n, ch, inv)
            assert np.abs(y - ref).max() <= 1e-5 + 1e-6 * np.abs(ref).max()


def test_oracle_vs_extended_vectors():
    for kind, run, tol in (("r2c", O.fft_r2c_f32, 2.0 ** -3), ("c2r", O.fft_c2r_f32, 1e-3)):
        d = np.load(os.path.join(GOLD, f"{kind}_extended.npz"))
        assert len(d["ids"]) >= 10
        for cid, ch, n, mode in zip(d["ids"], d["channels"], d["points"], d["mode"]):
            y = run(d[f"in_{cid}"], int(n), int(ch), int(mode))
            assert np.abs(y - d[f"out_{cid}"]).max() <= tol, (kind, cid)


def test_oracle_catches_a_planted_mistake():
    """A wrong twiddle sign in the oracle must be detected by the FP64
    check: guards against an oracle that agrees with anything."""
    n, ch = 64, 2
    x = O.uniform_c2c(n, ch, 3)
    good = O.fft_c2c_f32(x, n, ch)
    bad = O.fft_c2c_f32(x, n, ch, inverse=True) * n  # conjugate-direction transform
    f = O.fp64_c2c(x, n, ch)
    assert O.rel_l2(good, f) <= 2e-6
    assert O.rel_l2(bad, f) > 0.1
