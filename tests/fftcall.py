"""Test-side driver: runs the FFTLIB entry points of libfftlib_b200.so the
way the reference test drivers do (bufParams, pBlock, _init then _kernel),
with device buffers from torch (plumbing only) or host numpy buffers."""
from __future__ import annotations

import numpy as np

import c7x_fftlib_b200 as F


def _dev(a: np.ndarray):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t) -> np.ndarray:
    return t.cpu().numpy()


def c2c(x: np.ndarray, n: int, ch: int, inverse=False, on_device=True, entry="kernel") -> np.ndarray:
    """Batched FP32 c2c (forward or inverse) through the C API."""
    kind = "ifft" if inverse else "c2c"
    base = F.KERNELS[kind]
    dim = max(2 * n * ch, 2)
    w = np.zeros(max(2 * n, 2), np.float32)
    F.lib().FFTLIB_b200_tw_gen_c2c(F.ptr(w), n)
    if on_device:
        X, Y, W = _dev(np.asarray(x, np.float32)), _dev(np.zeros(dim, np.float32)), _dev(w)
    else:
        X, Y, W = np.array(x, np.float32), np.zeros(dim, np.float32), w
    bX, bW, bY = F.bp(F.FFTLIB_FLOAT32, dim), F.bp(F.FFTLIB_FLOAT32, 2 * n), F.bp(F.FFTLIB_FLOAT32, dim)
    if entry == "cn":
        F.check(F.fn(base + "_cn")(F.ptr(X), bX, F.ptr(W), bW, F.ptr(Y), bY, n, ch), base + "_cn")
    else:
        pb = F.pblock(kind)
        F.check(F.fn(base + "_init")(F.ptr(X), bX, F.ptr(W), bW, F.ptr(Y), bY, n, ch, pb), base + "_init")
        F.check(F.fn(base + "_kernel")(F.ptr(X), bX, F.ptr(W), bW, F.ptr(Y), bY, n, ch, pb), base + "_kernel")
    y = _host(Y) if on_device else Y
    return y[: 2 * n * ch]


def r2c(x: np.ndarray, n: int, ch: int, outmode=0, on_device=True) -> np.ndarray:
    base = F.KERNELS["r2c"]
    nout = n if outmode else n // 2 + 1
    w = np.zeros(max(n, 2), np.float32)
    F.lib().tw_gen_r2c(F.ptr(w), n)
    sf = np.zeros(2 * n, np.float32)
    F.lib().split_factor_gen_r2c(F.ptr(sf), n)
    if on_device:
        X, W, SF = _dev(np.asarray(x, np.float32)), _dev(w), _dev(sf)
        XF, Y = _dev(np.zeros(n * ch, np.float32)), _dev(np.zeros(2 * nout * ch, np.float32))
    else:
        X, W, SF = np.array(x, np.float32), w, sf
        XF, Y = np.zeros(n * ch, np.float32), np.zeros(2 * nout * ch, np.float32)
    b = F.bp(F.FFTLIB_FLOAT32, n * ch)
    pb = F.pblock("r2c")
    args = (F.ptr(X), b, F.ptr(W), b, F.ptr(XF), b, F.ptr(SF), b, F.ptr(Y), b, n, ch, outmode)
    F.check(F.fn(base + "_init")(*args, pb), base + "_init")
    F.check(F.fn(base + "_kernel")(*args, pb), base + "_kernel")
    return _host(Y) if on_device else Y


def c2r(x: np.ndarray, n: int, ch: int, inmode=0, on_device=True) -> np.ndarray:
    base = F.KERNELS["c2r"]
    w = np.zeros(max(n, 2), np.float32)
    F.lib().ifft_c2r_tw_gen(F.ptr(w), n)
    sf = np.zeros(2 * n, np.float32)
    F.lib().ifft_c2r_split_factor_gen(F.ptr(sf), n)
    if on_device:
        X, W, SF = _dev(np.asarray(x, np.float32)), _dev(w), _dev(sf)
        XF, Y = _dev(np.zeros((n + 1) * 2 * ch, np.float32)), _dev(np.zeros(n * ch, np.float32))
    else:
        X, W, SF = np.array(x, np.float32), w, sf
        XF, Y = np.zeros((n + 1) * 2 * ch, np.float32), np.zeros(n * ch, np.float32)
    b = F.bp(F.FFTLIB_FLOAT32, n * ch)
    pb = F.pblock("c2r")
    args = (F.ptr(X), b, F.ptr(W), b, F.ptr(XF), b, F.ptr(SF), b, F.ptr(Y), b, n, ch, inmode)
    F.check(F.fn(base + "_init")(*args, pb), base + "_init")
    F.check(F.fn(base + "_kernel")(*args, pb), base + "_kernel")
    return _host(Y) if on_device else Y


def i16(x: np.ndarray, n: int, ch: int, shifts, w=None, on_device=True) -> np.ndarray:
    base = F.KERNELS["i16"]
    if w is None:
        w = np.zeros(2 * n, np.int16)
        F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
    sh = np.ascontiguousarray(shifts, np.uint32)
    dim = 2 * n * ch
    if on_device:
        X, W, Y, S = _dev(np.asarray(x, np.int16)), _dev(np.asarray(w, np.int16)), _dev(np.zeros(dim, np.int16)), \
            _dev(sh.view(np.int32)).view(dtype=__import__("torch").int32)
    else:
        X, W, Y, S = np.array(x, np.int16), np.asarray(w, np.int16), np.zeros(dim, np.int16), sh
    bX, bW, bS = F.bp(F.FFTLIB_INT16, dim), F.bp(F.FFTLIB_INT16, 2 * n), F.bp(F.FFTLIB_UINT32, len(sh))
    pb = F.pblock("i16")
    args = (F.ptr(X), bX, F.ptr(W), bW, F.ptr(Y), bX, F.ptr(S), bS, n, ch)
    F.check(F.fn(base + "_init")(*args, pb), base + "_init")
    F.check(F.fn(base + "_kernel")(*args, pb), base + "_kernel")
    return _host(Y) if on_device else Y


# ---- single-transform kernels (length from dim_x) ------------------------------

def _run(base, args, entry, pb_kind):
    if entry == "cn":
        F.check(F.fn(base + "_cn")(*args), base + "_cn")
    else:
        pb = F.pblock(pb_kind)
        F.check(F.fn(base + "_init")(*args, pb), base + "_init")
        F.check(F.fn(base + "_kernel")(*args, pb), base + "_kernel")


def fft1d_c2c(x: np.ndarray, n: int, inverse=False, on_device=True, entry="kernel") -> np.ndarray:
    kind = "1d_ifft" if inverse else "1d_c2c"
    dim = 2 * n
    w = np.zeros(max(dim, 2), np.float32)
    F.lib().FFTLIB_b200_tw_gen_c2c(F.ptr(w), n)
    if on_device:
        X, Y, W = _dev(np.asarray(x, np.float32)), _dev(np.zeros(dim, np.float32)), _dev(w)
    else:
        X, Y, W = np.array(x, np.float32), np.zeros(dim, np.float32), w
    b = F.bp(F.FFTLIB_FLOAT32, dim)
    _run(F.KERNELS[kind], (F.ptr(X), b, F.ptr(W), b, F.ptr(Y), b), entry, kind)
    return _host(Y) if on_device else Y


def fft1d_r2c(x: np.ndarray, n: int, on_device=True, entry="kernel") -> np.ndarray:
    """n reals in, n complex bins out (as 2n floats)."""
    w = np.zeros(max(n, 2), np.float32)
    F.lib().tw_gen_r2c(F.ptr(w), n)
    sf = np.zeros(2 * n, np.float32)
    F.lib().split_factor_gen_r2c(F.ptr(sf), n)
    if on_device:
        X, W, SF = _dev(np.asarray(x, np.float32)), _dev(w), _dev(sf)
        XF, Y = _dev(np.zeros(2 * n + 2, np.float32)), _dev(np.zeros(2 * n, np.float32))
    else:
        X, W, SF = np.array(x, np.float32), w, sf
        XF, Y = np.zeros(2 * n + 2, np.float32), np.zeros(2 * n, np.float32)
    b = F.bp(F.FFTLIB_FLOAT32, n)
    _run(F.KERNELS["1d_r2c"], (F.ptr(X), b, F.ptr(W), b, F.ptr(XF), b, F.ptr(SF), b, F.ptr(Y), b), entry, "1d_r2c")
    return _host(Y) if on_device else Y


def fft1d_c2r(x: np.ndarray, n: int, on_device=True, entry="kernel") -> np.ndarray:
    """n complex bins in (2n floats), n reals out."""
    w = np.zeros(max(n, 2), np.float32)
    F.lib().ifft_c2r_tw_gen(F.ptr(w), n)
    sf = np.zeros(2 * n, np.float32)
    F.lib().ifft_c2r_split_factor_gen(F.ptr(sf), n)
    if on_device:
        X, W, SF = _dev(np.asarray(x, np.float32)), _dev(w), _dev(sf)
        XF, Y = _dev(np.zeros(2 * n + 2, np.float32)), _dev(np.zeros(n, np.float32))
    else:
        X, W, SF = np.array(x, np.float32), w, sf
        XF, Y = np.zeros(2 * n + 2, np.float32), np.zeros(n, np.float32)
    b = F.bp(F.FFTLIB_FLOAT32, n)
    _run(F.KERNELS["1d_c2r"], (F.ptr(X), b, F.ptr(W), b, F.ptr(XF), b, F.ptr(SF), b, F.ptr(Y), b), entry, "1d_c2r")
    return _host(Y) if on_device else Y


def fft1d_i16(x: np.ndarray, n: int, shifts, w=None, on_device=True, entry="kernel") -> np.ndarray:
    if w is None:
        w = np.zeros(2 * n, np.int16)
        F.lib().FFTLIB_b200_tw_gen_i16(F.ptr(w), n)
    sh = np.ascontiguousarray(shifts, np.uint32)
    if sh.size == 0:
        sh = np.zeros(1, np.uint32)  # a valid pointer; no radix-4 stage reads it
        nsh = 0
    else:
        nsh = sh.size
    dim = 2 * n
    if on_device:
        import torch

        X, W, Y = _dev(np.asarray(x, np.int16)), _dev(np.asarray(w, np.int16)), _dev(np.zeros(dim, np.int16))
        S = _dev(sh.view(np.int32)).view(dtype=torch.int32)
    else:
        X, W, Y, S = np.array(x, np.int16), np.asarray(w, np.int16), np.zeros(dim, np.int16), sh
    b, bS = F.bp(F.FFTLIB_INT16, dim), F.bp(F.FFTLIB_UINT32, nsh)
    _run(F.KERNELS["1d_i16"], (F.ptr(X), b, F.ptr(W), b, F.ptr(Y), b, F.ptr(S), bS), entry, "1d_i16")
    return _host(Y) if on_device else Y


def mixed_lengths(count: int, seed: int, nmax: int = 4096):
    """Lengths 12 * 2^a 3^b 5^c <= nmax drawn log-uniformly: log N uniform on
    [log 12, log nmax], snapped to the nearest allowed length in log space."""
    allowed = []
    a = 1
    while 12 * a <= nmax:
        b = a
        while 12 * b <= nmax:
            c = b
            while 12 * c <= nmax:
                allowed.append(12 * c)
                c *= 5
            b *= 3
        a *= 2
    allowed = np.array(sorted(allowed))
    g = np.random.default_rng(seed)
    u = g.uniform(np.log(12), np.log(nmax), count)
    idx = np.abs(np.log(allowed)[None, :] - u[:, None]).argmin(axis=1)
    return allowed[idx].astype(np.uint32)
