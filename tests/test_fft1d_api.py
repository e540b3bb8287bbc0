"""Host-side checks of the single-transform kernels FFTLIB_{fft,ifft}1d_*
that need no GPU: the reference drivers' coverage cases for every
_checkParams / _checkParams_cn, the pBlock sizes, the _init argument checks
that run before any device work, and the oracle's single-transform
restatement against the committed golden vectors and the reference's own
_cn code."""
import ctypes as C
import os

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _buf(n, dtype=np.float32):
    # 128-byte aligned host buffer, like TI_memalign(128, ...)
    raw = np.zeros(n * np.dtype(dtype).itemsize + 256, np.uint8)
    off = (-raw.ctypes.data) % 128
    return raw[off: off + n * np.dtype(dtype).itemsize].view(dtype)


def _addr(a, byte_offset=0):
    return C.c_void_p(a.ctypes.data + byte_offset)


# ---- FP32 coverage cases ------------------------------------------------------
# test/fft_c7x/FFTLIB_{fft,ifft}1d_i32fc_c32fc_o32fc/..._d.c coverage_test_main
# (numPoints 64, dim_x 128); test/fft_c7x/FFTLIB_fft1d_i32f_c32fc_o32fc/..._d.c
# and FFTLIB_ifft1d_i32fc_c32fc_o32f/..._d.c (numPoints 60, dim_x 60).
# mutation -> (optimized status, natural-C status)
C2C_CASES = {
    "null_x": (5, 5), "null_w": (5, 5), "null_y": (5, 5), "wdim": (4, 4), "ydim": (4, 4),
    "xtype": (3, 3), "wtype": (3, 3), "ytype": (3, 3), "misaligned": (8, 0), "dim14": (4, 4), "dim60": (0, 0),
}
R2C_CASES = dict(C2C_CASES, dim61=(0, 4), dim254=(4, 4), base=(0, 0))
del R2C_CASES["dim14"], R2C_CASES["dim60"]
C2R_CASES = dict(C2C_CASES, base=(0, 0))
del C2R_CASES["dim60"]


def _f32_args(mut, dim):
    X, W, Y = _buf(2 * dim + 8), _buf(2 * dim + 8), _buf(2 * dim + 8)
    bX, bW, bY = F.bp(F.FFTLIB_FLOAT32, dim), F.bp(F.FFTLIB_FLOAT32, dim), F.bp(F.FFTLIB_FLOAT32, dim)
    px, pw, py = _addr(X), _addr(W), _addr(Y)
    if mut == "null_x":
        px = None
    elif mut == "null_w":
        pw = None
    elif mut == "null_y":
        py = None
    elif mut == "wdim":
        bW.dim_x = dim // 2
    elif mut == "ydim":
        bY.dim_x = dim // 2
    elif mut == "xtype":
        bX.data_type = F.FFTLIB_UINT32
    elif mut == "wtype":
        bW.data_type = F.FFTLIB_UINT32
    elif mut == "ytype":
        bY.data_type = F.FFTLIB_UINT32
    elif mut == "misaligned":
        px = _addr(X, 4)
    elif mut.startswith("dim"):
        for b in (bX, bW, bY):
            b.dim_x = int(mut[3:])
    return px, bX, pw, bW, py, bY


@pytest.mark.parametrize("kind", ["1d_c2c", "1d_ifft"])
@pytest.mark.parametrize("mut", sorted(C2C_CASES))
def test_c2c_checkparams_coverage(kind, mut):
    exp_opt, exp_cn = C2C_CASES[mut]
    base = F.KERNELS[kind]
    px, bX, pw, bW, py, bY = _f32_args(mut, 128)
    pb = F.pblock(kind)
    assert F.fn(base + "_checkParams")(px, bX, pw, bW, py, bY, pb) == exp_opt
    assert F.fn(base + "_checkParams_cn")(px, bX, pw, bW, py, bY) == exp_cn


@pytest.mark.parametrize("kind,cases", [("1d_r2c", R2C_CASES), ("1d_c2r", C2R_CASES)])
def test_real_checkparams_coverage(kind, cases):
    base = F.KERNELS[kind]
    for mut, (exp_opt, exp_cn) in sorted(cases.items()):
        px, bX, pw, bW, py, bY = _f32_args(mut, 60)
        pb = F.pblock(kind)
        assert F.fn(base + "_checkParams")(px, bX, pw, bW, py, bY, pb) == exp_opt, mut
        assert F.fn(base + "_checkParams_cn")(px, bX, pw, bW, py, bY) == exp_cn, mut


# ---- int16 coverage cases -------------------------------------------------------
# test/fft_c7x/FFTLIB_fft1d_i16sc_c16sc_o16sc/..._d.c coverage_test_main
# (numPoints 64, dim_x 128, three shifts)
I16_CASES = {
    1000: ("null_x", 5, 5), 1001: ("null_w", 5, 5), 1002: ("null_y", 5, 5), 1003: ("null_shift", 5, 5),
    1004: ("null_block", 5, 0), 1005: ("wdim", 4, 4), 1006: ("ydim", 4, 4), 1007: ("dim64", 4, 4),
    1008: ("xtype", 3, 3), 1009: ("wtype", 3, 3), 1010: ("ytype", 3, 3), 1011: ("stype", 3, 3),
    1012: ("misaligned", 8, 0), 1013: ("dim256", 0, 0), 1014: ("dim192", 4, 4), 1015: ("base", 0, 0),
}


@pytest.mark.parametrize("case", sorted(I16_CASES))
def test_i16_checkparams_coverage(case):
    mut, exp_opt, exp_cn = I16_CASES[case]
    base = F.KERNELS["1d_i16"]
    X, W, Y, S = _buf(512, np.int16), _buf(512, np.int16), _buf(512, np.int16), _buf(4, np.uint32)
    bX, bW, bY = (F.bp(F.FFTLIB_INT16, 128) for _ in range(3))
    bS = F.bp(F.FFTLIB_UINT32, 3)
    px, pw, py, ps = _addr(X), _addr(W), _addr(Y), _addr(S)
    pb = F.pblock("1d_i16")
    if mut == "null_x":
        px = None
    elif mut == "null_w":
        pw = None
    elif mut == "null_y":
        py = None
    elif mut == "null_shift":
        ps = None
    elif mut == "null_block":
        pb = None
    elif mut == "wdim":
        bW.dim_x = 64
    elif mut == "ydim":
        bY.dim_x = 64
    elif mut in ("dim64", "dim256", "dim192"):
        for b in (bX, bW, bY):
            b.dim_x = int(mut[3:])
    elif mut == "xtype":
        bX.data_type = F.FFTLIB_UINT32
    elif mut == "wtype":
        bW.data_type = F.FFTLIB_UINT32
    elif mut == "ytype":
        bY.data_type = F.FFTLIB_UINT32
    elif mut == "stype":
        bS.data_type = F.FFTLIB_INT16
    elif mut == "misaligned":
        px = _addr(X, 2)
    assert F.fn(base + "_checkParams")(px, bX, pw, bW, py, bY, ps, bS, pb) == exp_opt
    assert F.fn(base + "_checkParams_cn")(px, bX, pw, bW, py, bY, ps, bS) == exp_cn


def test_init_rejects_before_device_work():
    """Argument errors come back from _init without touching a GPU: a NULL
    pBlock (the optimized FP32 checks do not test it), a failed check, an
    odd real length the c71 checks let through."""
    X, W, Y = _buf(256), _buf(256), _buf(256)
    b = F.bp(F.FFTLIB_FLOAT32, 128)
    for kind in ("1d_c2c", "1d_ifft"):
        base = F.KERNELS[kind]
        assert F.fn(base + "_init")(_addr(X), b, _addr(W), b, _addr(Y), b, None) == F.FFTLIB_ERR_NULL_POINTER
        bad = F.bp(F.FFTLIB_FLOAT32, 14)
        assert F.fn(base + "_init")(_addr(X), bad, _addr(W), bad, _addr(Y), bad,
                                    F.pblock(kind)) == F.FFTLIB_ERR_INVALID_DIMENSION
    odd = F.bp(F.FFTLIB_FLOAT32, 61)
    for kind in ("1d_r2c", "1d_c2r"):
        base = F.KERNELS[kind]
        args = (_addr(X), odd, _addr(W), odd, _addr(X), odd, _addr(W), odd, _addr(Y), odd)
        assert F.fn(base + "_checkParams")(_addr(X), odd, _addr(W), odd, _addr(Y), odd, None) == 0
        assert F.fn(base + "_init")(*args, F.pblock(kind)) == F.FFTLIB_ERR_INVALID_DIMENSION
        args = (_addr(X), b, _addr(W), b, _addr(X), b, _addr(W), b, _addr(Y), b)
        assert F.fn(base + "_init")(*args, None) == F.FFTLIB_ERR_NULL_POINTER


def test_kernel_rejects_foreign_pblock():
    """A pBlock that no matching _init filled is refused before any launch."""
    X, W, Y = _buf(256), _buf(256), _buf(256)
    b = F.bp(F.FFTLIB_FLOAT32, 128)
    pb = F.pblock("1d_c2c")
    assert F.fn(F.KERNELS["1d_c2c"] + "_kernel")(_addr(X), b, _addr(W), b, _addr(Y), b, pb) == F.FFTLIB_ERR_FAILURE
    assert F.fn(F.KERNELS["1d_c2c"] + "_kernel")(_addr(X), b, _addr(W), b, _addr(Y), b, None) == \
        F.FFTLIB_ERR_NULL_POINTER


def test_pblock_sizes_cover_the_plan_record():
    for kind in ("1d_c2c", "1d_ifft", "1d_r2c", "1d_c2r", "1d_i16"):
        assert F.PBLOCK_SIZE[kind] >= 64


# ---- oracle: single-transform restatement, pinned --------------------------------

@pytest.mark.parametrize("kind", ["r2c", "c2r"])
def test_oracle_matches_reference_static_vectors(kind):
    """The reference drivers' static vectors for the single real-input
    kernels (tolerances of the drivers: r2c 2^-3, c2r 0.1 absolute)."""
    d = np.load(os.path.join(GOLDEN, f"fft1d_{kind}_static.npz"))
    assert len(d["ids"]) == 8
    for cid in d["ids"]:
        n = int(d[f"n_{cid}"])
        got = O.fft1d_r2c_f32(d[f"in_{cid}"], n) if kind == "r2c" else O.fft1d_c2r_f32(d[f"in_{cid}"], n)
        tol = 2.0 ** -3 if kind == "r2c" else 0.1
        assert np.abs(got - d[f"out_{cid}"]).max() <= tol, (kind, cid, n)


def test_oracle_int16_matches_reference_fixture():
    d = np.load(os.path.join(GOLDEN, "fft1d_i16_pymodel.npz"))
    agree = 0
    for i in range(int(d["n_cases"])):
        n = int(d[f"case{i}_n"])
        if f"tw_{n}" in d:
            assert np.array_equal(O.tw_gen_i16(n), d[f"tw_{n}"])
        got = O.fft1d_c2c_i16(d[f"case{i}_in"], n, d[f"case{i}_shift"])
        assert np.array_equal(got, d[f"case{i}_out"]), (i, n)
        agree += int(d[f"case{i}_model_agrees"])
    assert agree >= 10  # the Python model itself agrees wherever nothing overflows


def test_oracle_c2c_matches_reference_python_model():
    d = np.load(os.path.join(GOLDEN, "fft1d_c2c_pymodel.npz"))
    for i, n in enumerate(d["sizes"]):
        n = int(n)
        x = d[f"case{i}_in"]
        fwd = O.fft1d_c2c_f32(x, n)
        inv = O.fft1d_c2c_f32(x, n, True)
        # the model rounds to 6 decimals (then FP32 storage)
        assert O.rel_l2(fwd, O.as_complex(d[f"case{i}_fwd"], n, 1)[0]) < 1e-6
        assert np.abs(inv - d[f"case{i}_inv"]).max() < 2e-6


needs_ref = pytest.mark.skipif(not O.ref1d_available(), reason="oracle/_ref single-transform libraries not built")


@needs_ref
@pytest.mark.parametrize("n", [1, 2, 4, 8, 16, 64, 256, 1024, 4096, 16384, 12, 60, 125, 1000, 3000, 6561])
def test_oracle_matches_reference_cn_c2c(n):
    """pow2 lengths are bit-identical; 3 and 5 radices agree to FP32
    rounding (the restatement orders the radix-3/5 arithmetic differently)."""
    x = O.uniform_c2c(n, 1, 50 + n, -128, 128)
    for inv in (False, True):
        r, o = O.ref_fft1d_c2c_f32(x, n, inv), O.fft1d_c2c_f32(x, n, inv)
        if n & (n - 1) == 0:
            assert np.array_equal(r, o), (n, inv)
        else:
            assert O.rel_l2(o, O.as_complex(r, n, 1)[0]) < 5e-7, (n, inv)
        # the single kernel is the batched kernel with one channel: bit for
        # bit forward; the inverse scales at the end (..._cn.c:436-437) where
        # the batched one scales the input, which moves FP32 roundings
        b = O.ref_c2c_f32(x, n, 1, inv)
        if inv and n & (n - 1):
            assert O.rel_l2(r, O.as_complex(b, n, 1)[0]) < 5e-7
        else:
            assert np.array_equal(r, b), (n, inv)


@needs_ref
@pytest.mark.parametrize("n", [4, 8, 16, 64, 120, 256, 1000, 4096, 6000, 8192])
def test_oracle_matches_reference_cn_real(n):
    x = O.real_signal(n, 1, 70 + n)
    r, o = O.ref_fft1d_r2c_f32(x, n), O.fft1d_r2c_f32(x, n)
    f = np.fft.fft(x.astype(np.float64))
    spec = np.stack([f.real, f.imag], -1).ravel().astype(np.float32)
    rc, oc = O.ref_fft1d_c2r_f32(spec, n), O.fft1d_c2r_f32(spec, n)
    if n & (n - 1) == 0:
        assert np.array_equal(r, o) and np.array_equal(rc, oc)
    else:
        assert O.rel_l2(o, f) < 5e-7 and O.rel_l2(r, f) < 5e-7
        assert np.abs(rc - oc).max() <= 1e-5 * np.abs(x).max()
    # batched with one channel: bit for bit forward (and pow2 inverse); the
    # single c2r's ifft scales at the end instead of on input
    assert np.array_equal(r, O.ref_r2c_f32(x, n, 1, 1))
    bc = O.ref_c2r_f32(spec, n, 1, 1)
    if n & (n - 1) == 0:
        assert np.array_equal(rc, bc)
    else:
        assert np.abs(rc - bc).max() <= 1e-5 * np.abs(x).max()


@needs_ref
@pytest.mark.parametrize("n,shifts", [(2, []), (4, [1]), (8, [1]), (16, [1, 1]), (32, [0, 1]), (64, [0, 1, 1]),
                                      (128, [0, 1, 1]), (1024, [2, 2, 2, 2, 2]), (4096, [1, 0, 0, 0, 0, 1]),
                                      (16384, [1, 0, 1, 1, 1, 1, 0])])
def test_oracle_matches_reference_cn_i16(n, shifts):
    for seed, (lo, hi) in enumerate([(-1000, 1000), (-32768, 32767)]):
        x = O.int16_input(n, 1, 90 + n + seed, lo, hi)
        assert np.array_equal(O.ref_fft1d_c2c_i16(x, n, shifts), O.fft1d_c2c_i16(x, n, shifts)), (n, lo)
