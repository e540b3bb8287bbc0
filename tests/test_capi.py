"""Host-side checks of libfftlib_b200.so that need no GPU: the library loads,
exports every entry point its headers declare, its parameter checks return
the reference's status codes on the reference's own coverage cases, its
table generators reproduce the reference tables bit for bit, and the planner
finds a schedule for every length the reference tests."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

import c7x_fftlib_b200 as F
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
S = F  # status / type constants


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "**", "*.h"), recursive=True):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:FFTLIB_STATUS|void|int32_t|uint32_t|int|const char \*)\s+\**\s*(\w+)\s*\(",
                             text, re.M):
            if m.group(1) != "FFTLIB_sizeof":
                names.add(m.group(1))
        for m in re.finditer(r"^\s*extern\s+\w+\s+(\w+)\s*\[", text, re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    L = F.lib()
    names = declared_functions()
    assert len(names) >= 40
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_error_string():
    assert F.lib().FFTLIB_b200_version() >= 100
    assert isinstance(F.last_error(), str)


def test_product_does_not_link_the_oracle():
    with open(F.LIB_PATH, "rb") as f:
        blob = f.read()
    assert b"orc_fft" not in blob and b"liboracle" not in blob


# ---- checkParams: reference coverage cases -----------------------------------

def _buf(n, dtype=np.float32):
    # 128-byte aligned host buffer, like TI_memalign(128, ...)
    raw = np.zeros(n * np.dtype(dtype).itemsize + 256, np.uint8)
    off = (-raw.ctypes.data) % 128
    return raw[off: off + n * np.dtype(dtype).itemsize].view(dtype)


def _addr(a, byte_offset=0):
    return C.c_void_p(a.ctypes.data + byte_offset)


C2C_CASES = {
    # testNum: (mutation, expected optimized status, expected _cn status, _cn status for ifft)
    1000: ("null_x", 5, 5, 5), 1001: ("null_w", 5, 5, 5), 1002: ("null_y", 5, 5, 5), 1003: ("null_block", 5, 0, 0),
    1004: ("ydim", 4, 4, 4), 1005: ("wdim", 4, 4, 4), 1006: ("xtype", 3, 3, 3), 1007: ("wtype", 3, 3, 3),
    1008: ("ytype", 3, 3, 3), 1009: ("misaligned", 8, 0, 0), 1010: ("n7", 4, 4, 6), 1011: ("n30", 0, 0, 0),
}


@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("case", sorted(C2C_CASES))
def test_c2c_checkparams_coverage(case, inverse):
    """test/fft_c7x/FFTLIB_{fft,ifft}1dBatched_i32fc_c32fc_o32fc/..._d.c coverage_test_main."""
    mut, exp_opt, exp_cn, exp_cn_inv = C2C_CASES[case]
    n, ch = 64, 4
    dim = ch * n * 2
    X, W, Y = _buf(dim), _buf(2 * n), _buf(dim)
    bX, bW, bY = F.bp(F.FFTLIB_FLOAT32, dim), F.bp(F.FFTLIB_FLOAT32, 2 * n), F.bp(F.FFTLIB_FLOAT32, dim)
    pX, pW, pY, pb = _addr(X), _addr(W), _addr(Y), F.pblock("c2c")
    if mut == "null_x": pX = None
    if mut == "null_w": pW = None
    if mut == "null_y": pY = None
    if mut == "null_block": pb = None
    if mut == "ydim": bY.dim_x = dim // 2
    if mut == "wdim": bW.dim_x = n
    if mut == "xtype": bX.data_type = F.FFTLIB_UINT32
    if mut == "wtype": bW.data_type = F.FFTLIB_UINT32
    if mut == "ytype": bY.data_type = F.FFTLIB_UINT32
    if mut == "misaligned": pX = _addr(X, 4)
    if mut in ("n7", "n30"):
        n, ch = (7, 1) if mut == "n7" else (30, 1)
        bX.dim_x = bY.dim_x = ch * n * 2
        bW.dim_x = 2 * n
    base = F.KERNELS["ifft" if inverse else "c2c"]
    st_opt = F.fn(base + "_checkParams")(pX, bX, pW, bW, pY, bY, n, ch, pb)
    st_cn = F.fn(base + "_checkParams_cn")(pX, bX, pW, bW, pY, bY, n, ch)
    assert st_opt == exp_opt
    assert st_cn == (exp_cn_inv if inverse else exp_cn)


@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("case", sorted(C2C_CASES))
def test_c2c_checkparams_cn_matches_reference(ref_cn, case, inverse):
    mut = C2C_CASES[case][0]
    if mut in ("null_block", "misaligned"):
        pytest.skip("optimized-only condition")
    n, ch = 64, 4
    dim = ch * n * 2
    X, W, Y = _buf(dim), _buf(2 * n), _buf(dim)
    bX, bW, bY = O.BufParams(12, dim), O.BufParams(12, 2 * n), O.BufParams(12, dim)
    args = {"null_x": 0, "null_w": 1, "null_y": 2}
    ptrs = [_addr(X), _addr(W), _addr(Y)]
    if mut in args: ptrs[args[mut]] = None
    if mut == "ydim": bY.dim_x = dim // 2
    if mut == "wdim": bW.dim_x = n
    if mut == "xtype": bX.data_type = 8
    if mut == "wtype": bW.data_type = 8
    if mut == "ytype": bY.data_type = 8
    if mut in ("n7", "n30"):
        n, ch = (7, 1) if mut == "n7" else (30, 1)
        bX.dim_x = bY.dim_x = ch * n * 2
        bW.dim_x = 2 * n
    kind = "ifft" if inverse else "c2c"
    ref = getattr(O.ref_lib(kind), F.KERNELS[kind] + "_checkParams_cn")
    ours = F.fn(F.KERNELS[kind] + "_checkParams_cn")
    r = ref(ptrs[0], C.byref(bX), ptrs[1], C.byref(bW), ptrs[2], C.byref(bY), C.c_uint32(n), C.c_uint32(ch))
    o = ours(ptrs[0], F.bp(bX.data_type, bX.dim_x), ptrs[1], F.bp(bW.data_type, bW.dim_x), ptrs[2],
             F.bp(bY.data_type, bY.dim_x), n, ch)
    assert o == r


REAL_CASES = {
    # r2c: test/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._d.c coverage_test_main
    "r2c": {1000: ("null_x", 5, 5), 1001: ("null_w", 5, 5), 1002: ("null_y", 5, 5), 1003: ("wdim", 4, 4),
            1004: ("ydim", 4, 4), 1005: ("xtype", 3, 3), 1006: ("wtype", 3, 3), 1007: ("ytype", 3, 3),
            1008: ("misaligned", 8, 0), 1009: ("outmode2", 14, 0), 1010: ("dim61", 0, 4), 1011: ("n254", 4, 4),
            1012: ("ok", 0, 0)},
    # c2r: test/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/..._d.c coverage_test_main
    "c2r": {1000: ("null_x", 5, 5), 1001: ("null_w", 5, 5), 1002: ("null_y", 5, 5), 1003: ("wdim", 4, 4),
            1004: ("ydim", 4, 4), 1005: ("xtype", 3, 3), 1006: ("wtype", 3, 3), 1007: ("ytype", 3, 3),
            1008: ("misaligned", 8, 0), 1009: ("n14", 4, 4), 1010: ("ok", 0, 0)},
}


@pytest.mark.parametrize("kind,case", [(k, c) for k in REAL_CASES for c in sorted(REAL_CASES[k])])
def test_real_checkparams_coverage(kind, case):
    mut, exp_opt, exp_cn = REAL_CASES[kind][case]
    n, ch, mode = 60, 4, 0
    dim = n
    X, W, Y = _buf(4 * n * ch), _buf(4 * n), _buf(4 * n * ch)
    b = [F.bp(F.FFTLIB_FLOAT32, dim) for _ in range(3)]
    p = [_addr(X), _addr(W), _addr(Y)]
    if mut == "null_x": p[0] = None
    if mut == "null_w": p[1] = None
    if mut == "null_y": p[2] = None
    if mut == "wdim": b[1].dim_x = dim // 2
    if mut == "ydim": b[2].dim_x = dim // 2
    if mut == "xtype": b[0].data_type = F.FFTLIB_UINT32
    if mut == "wtype": b[1].data_type = F.FFTLIB_UINT32
    if mut == "ytype": b[2].data_type = F.FFTLIB_UINT32
    if mut == "misaligned": p[0] = _addr(X, 4)
    if mut == "outmode2": mode = 2
    if mut == "dim61":
        for bb in b: bb.dim_x = 61
    if mut == "n254":
        n = 254
        for bb in b: bb.dim_x = n * ch
    if mut == "n14": n = 14
    base = F.KERNELS[kind]
    st_opt = F.fn(base + "_checkParams")(p[0], b[0], p[1], b[1], p[2], b[2], n, ch, mode, F.pblock(kind))
    st_cn = F.fn(base + "_checkParams_cn")(p[0], b[0], p[1], b[1], p[2], b[2], n, ch, mode)
    assert (st_opt, st_cn) == (exp_opt, exp_cn)


I16_CASES = {
    # test/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._d.c coverage_test_main
    1000: ("null_x", 5, 5), 1001: ("null_block", 5, 0), 1002: ("ydim", 0, 4), 1003: ("xdim_small", 0, 4),
    1004: ("wdim", 0, 4), 1005: ("xtype", 0, 3), 1006: ("shifttype", 0, 3), 1007: ("n96", 0, 4), 1008: ("ok", 0, 0),
}


@pytest.mark.parametrize("case", sorted(I16_CASES))
def test_i16_checkparams_coverage(case):
    mut, exp_opt, exp_cn = I16_CASES[case]
    n, ch, nsh = 64, 4, 3
    dim = n * ch * 2
    X, W, Y, Sh = _buf(dim, np.int16), _buf(2 * n, np.int16), _buf(dim, np.int16), _buf(nsh, np.uint32)
    bX, bW, bY, bS = F.bp(F.FFTLIB_INT16, dim), F.bp(F.FFTLIB_INT16, 2 * n), F.bp(F.FFTLIB_INT16, dim), \
        F.bp(F.FFTLIB_UINT32, nsh)
    pX, pb = _addr(X), F.pblock("i16")
    if mut == "null_x": pX = None
    if mut == "null_block": pb = None
    if mut == "ydim": bY.dim_x = dim // 2
    if mut == "xdim_small": bX.dim_x = bY.dim_x = dim - 2
    if mut == "wdim": bW.dim_x = n
    if mut == "xtype": bX.data_type = F.FFTLIB_UINT32
    if mut == "shifttype": bS.data_type = F.FFTLIB_INT16
    if mut == "n96":
        n = 96
        bX.dim_x = bY.dim_x = n * ch * 2
        bW.dim_x = 2 * n
    base = F.KERNELS["i16"]
    args = (pX, bX, _addr(W), bW, _addr(Y), bY, _addr(Sh), bS, n, ch)
    assert F.fn(base + "_checkParams")(*args, pb) == exp_opt
    assert F.fn(base + "_checkParams_cn")(*args) == exp_cn


# ---- table generators --------------------------------------------------------

@pytest.mark.parametrize("n", [2, 4, 8, 12, 64, 128, 480, 4096, 6250, 62500])
def test_table_generators_bit_exact(ref_cn, n):
    L = F.lib()
    for ours, ref, size in (("tw_gen_r2c", O.ref_tw_gen_r2c, n), ("ifft_c2r_tw_gen", O.ref_tw_gen_c2r, n),
                            ("split_factor_gen_r2c", O.ref_split_factor_r2c, 2 * n),
                            ("ifft_c2r_split_factor_gen", O.ref_split_factor_c2r, 2 * n)):
        buf = np.zeros(max(size, 2), np.float32)
        getattr(L, ours)(F.ptr(buf), n)
        assert np.array_equal(buf[:size].view(np.uint32), ref(n)[:size].view(np.uint32)), ours


@pytest.mark.parametrize("n", [1, 4, 12, 30, 64, 960, 3000, 4096, 15625, 31250])
def test_test_driver_tables_bit_exact(ref_cn, n):
    w = np.zeros(max(2 * n, 2), np.float32)
    F.lib().FFTLIB_b200_tw_gen_c2c(F.ptr(w), n)
    assert np.array_equal(w[: 2 * n].view(np.uint32), O.ref_tw_gen_c2c(n).view(np.uint32))


@pytest.mark.parametrize("n", [4, 16, 64, 256, 1024, 4096])
def test_q15_table_bit_exact(ref_cn, n):
    w = np.zeros(2 * n, np.int16)
    F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
    assert np.array_equal(w, O.ref_tw_gen_i16(n))


# ---- planner -----------------------------------------------------------------

def _sizes_235(limit):
    out = []
    a = 1
    while a <= limit:
        b = a
        while b <= limit:
            c = b
            while c <= limit:
                out.append(c)
                c *= 5
            b *= 3
        a *= 2
    return sorted(out)


def test_planner_covers_every_235_length_up_to_16384():
    for n in _sizes_235(16384):
        desc = F.describe_plan(n)
        m = re.match(r"N=(\d+) E=(\d+) T=(\d+) radices=([\dx]+)", desc)
        if m is None:
            assert desc.startswith("global passes"), (n, desc)
            continue
        radices = [int(r) for r in m.group(4).split("x")]
        assert int(np.prod(radices)) == n, (n, desc)
        e, t = int(m.group(2)), int(m.group(3))
        assert t <= 1024
        for r in radices:
            assert r <= e
            # every pass fits the register capacity with T threads
            assert -(-(n // r) // t) * r <= e, (n, desc)


def test_planner_headline_schedule():
    """N=4096: three radix-16 passes, 32 values per thread (128 threads), the
    fixed-size schedule measured fastest on B200."""
    assert F.describe_plan(4096) == "N=4096 E=32 T=128 radices=16x16x16 (fixed-size kernel)"


def test_planner_prefers_the_measured_wide_schedules():
    """Lengths whose 32-wide fixed-size schedule (fewer passes, radices up to
    27 and 32) measured faster than the heuristic pick run that schedule."""
    want = {250: "25x10", 270: "27x10", 576: "24x24", 864: "32x27", 2000: "25x10x8", 2916: "27x12x9",
            3000: "25x12x10", 3645: "27x15x9", 4050: "27x15x10"}
    for n, radices in want.items():
        d = F.describe_plan(n)
        assert d.startswith(f"N={n} E=32 ") and f"radices={radices} " in d, d
    # and the heuristic keeps the lengths where the 16-wide schedule won
    for n in (1024, 2048, 1875, 3600):
        assert " E=16 " in F.describe_plan(n), F.describe_plan(n)


def test_every_length_from_8_to_4096_has_a_fixed_size_kernel():
    """Every 2^a 3^b 5^c length in [8, 4096] runs a kernel compiled for its
    planned schedule (the runtime-radix engine serves the rest)."""
    small = {8, 9, 10, 12, 15, 16, 18, 20, 24, 25, 27, 30, 32, 45}  # c2c: one transform per thread
    for n in _sizes_235(4096):
        if n >= 8:
            want = "(fixed-size kernel; c2c: one transform per thread)" if n in small else "(fixed-size kernel)"
            assert F.describe_plan(n).endswith(want), (n, F.describe_plan(n))


def test_planner_rejects_other_primes():
    assert F.lib().FFTLIB_b200_describePlan(7, C.create_string_buffer(64), 64) == F.FFTLIB_ERR_INVALID_DIMENSION


def test_mixed_batch_supports_every_length_up_to_4096():
    import fftcall

    for n in _sizes_235(4096):
        assert F.lib().FFTLIB_b200_fftMixed_supported(n) == F.FFTLIB_SUCCESS, n
    for n in set(fftcall.mixed_lengths(2000, seed=0).tolist()):
        assert n % 12 == 0 and n <= 4096
    assert F.lib().FFTLIB_b200_fftMixed_supported(7) == F.FFTLIB_ERR_INVALID_DIMENSION
