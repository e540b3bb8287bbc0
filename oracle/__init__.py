"""CPU oracle for the FFTLIB batched FFT hot path.

TEST INFRASTRUCTURE ONLY. Imported by ``tests/``, ``__graft_entry__.smoke()``
and the CPU-baseline leg of ``bench.py`` as the checker, never by the product
package ``c7x_fftlib_b200``.

Three layers, all on the CPU:

* ``liboracle.so`` -- this repository's C restatement of the reference
  natural-C (``_cn``) kernels (``oracle/fftlib_oracle.c``), with the same
  buffer layouts and twiddle tables as the reference.
* ``_ref/libref_*.so`` -- the reference's own ``_cn`` sources, compiled by
  ``oracle/Makefile`` from the reference tree (present only where that tree
  was available at build time; the shared objects travel with the checkout).
* FP64 references through numpy's ``pocketfft`` (``np.fft``), against which
  every result reports relative L2 error.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_i16p = np.ctypeslib.ndpointer(np.int16, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u32 = C.c_uint32


REF_ENV = "FFTLIB_REFERENCE_ROOT"


def reference_root(ref_root: str | None = None) -> str | None:
    """The reference tree oracle/_ref is compiled from: the argument, else
    $FFTLIB_REFERENCE_ROOT, else None (no default location)."""
    return ref_root or os.environ.get(REF_ENV) or None


def build(ref_root: str | None = None, with_ref: bool = True) -> None:
    """Compile this repository's checkers (liboracle.so, liboracle_gpu.so)
    and, when a reference tree is named (argument or $FFTLIB_REFERENCE_ROOT),
    oracle/_ref from the reference's own sources."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    root = reference_root(ref_root)
    if with_ref and root:
        build_ref(root)


def build_ref(ref_root: str | None = None) -> None:
    """Compile oracle/_ref from the reference tree; a clear error when none is
    named or the path holds no reference sources."""
    root = reference_root(ref_root)
    if not root or not os.path.isdir(os.path.join(root, "src")):
        raise RuntimeError(f"oracle/_ref is compiled from the reference's own sources: pass the c7x_fftlib tree "
                           f"or set {REF_ENV} (got {root!r})")
    subprocess.run(["make", "-s", "-C", HERE, f"REF={root}", "all"], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build(with_ref=False)
        L = C.CDLL(path)
        L.orc_tw_gen_f32.argtypes = [_f32p, _u32]
        L.orc_tw_gen_i16.argtypes = [_i16p, _u32]
        L.orc_split_factor_r2c.argtypes = [_f32p, _u32]
        L.orc_split_factor_c2r.argtypes = [_f32p, _u32]
        L.orc_fft_c2c_f32.argtypes = [_f32p, _f32p, _f32p, _u32, _u32, C.c_int]
        L.orc_fft_r2c_f32.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _u32, _u32, C.c_int]
        L.orc_fft_c2r_f32.argtypes = [_f32p, _f32p, _f32p, _f32p, _f32p, _u32, _u32, C.c_int]
        L.orc_fft_c2c_i16.argtypes = [_i16p, _i16p, _i16p, _u32p, _u32, _u32, _u32]
        for fn in ("orc_fft_c2c_f32", "orc_fft_r2c_f32", "orc_fft_c2r_f32", "orc_fft_c2c_i16"):
            getattr(L, fn).restype = C.c_int
        _lib = L
    return _lib


# --------------------------------------------------------------------------
# Tables
# --------------------------------------------------------------------------

def tw_gen_f32(n: int) -> np.ndarray:
    """FP32 twiddle table (2n floats) in the reference tw_gen layout."""
    w = np.zeros(max(2 * n, 2), np.float32)
    lib().orc_tw_gen_f32(w, n)
    return w[: 2 * n] if n else w[:0]


def tw_gen_i16(n: int) -> np.ndarray:
    """Q15 radix-4 twiddle table (2n int16) in the reference layout."""
    w = np.zeros(max(2 * n, 2), np.int16)
    lib().orc_tw_gen_i16(w, n)
    return w[: 2 * n]


def split_factor_r2c(n: int) -> np.ndarray:
    sf = np.zeros(2 * n, np.float32)
    lib().orc_split_factor_r2c(sf, n)
    return sf


def split_factor_c2r(n: int) -> np.ndarray:
    sf = np.zeros(2 * n, np.float32)
    lib().orc_split_factor_c2r(sf, n)
    return sf


# --------------------------------------------------------------------------
# Restated kernels (inputs are copied; the C code clobbers its input like
# the reference does)
# --------------------------------------------------------------------------

def fft_c2c_f32(x: np.ndarray, n: int, channels: int, inverse: bool = False) -> np.ndarray:
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(max(2 * n * channels, 1), np.float32)
    w = tw_gen_f32(n) if n else np.zeros(2, np.float32)
    rc = lib().orc_fft_c2c_f32(xin, np.ascontiguousarray(w), y, n, channels, int(inverse))
    if rc:
        raise ValueError(f"oracle c2c rejected N={n} (rc={rc})")
    return y[: 2 * n * channels]


def fft_r2c_f32(x: np.ndarray, n: int, channels: int, outmode: int = 0) -> np.ndarray:
    xin = np.ascontiguousarray(x, np.float32).copy()
    nout = n if outmode else n // 2 + 1
    y = np.zeros(2 * nout * channels, np.float32)
    xfft = np.zeros(n * channels, np.float32)
    rc = lib().orc_fft_r2c_f32(xin, tw_gen_f32(n // 2), xfft, split_factor_r2c(n), y, n, channels, int(outmode))
    if rc:
        raise ValueError(f"oracle r2c rejected N={n}")
    return y


def fft_c2r_f32(x: np.ndarray, n: int, channels: int, inmode: int = 0) -> np.ndarray:
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(n * channels, np.float32)
    xfft = np.zeros(n * channels, np.float32)
    rc = lib().orc_fft_c2r_f32(xin, tw_gen_f32(n // 2), xfft, split_factor_c2r(n), y, n, channels, int(inmode))
    if rc:
        raise ValueError(f"oracle c2r rejected N={n}")
    return y


def fft_c2c_i16(x: np.ndarray, n: int, channels: int, shifts) -> np.ndarray:
    xin = np.ascontiguousarray(x, np.int16).copy()
    y = np.zeros(2 * n * channels, np.int16)
    sh = np.ascontiguousarray(shifts, np.uint32)
    rc = lib().orc_fft_c2c_i16(xin, tw_gen_i16(n), y, sh, len(sh), n, channels)
    if rc:
        raise ValueError(f"oracle int16 rejected N={n} shifts={list(shifts)} (rc={rc})")
    return y


# --------------------------------------------------------------------------
# FP64 references and error metric
# --------------------------------------------------------------------------

def as_complex(a: np.ndarray, n: int, channels: int) -> np.ndarray:
    a = np.asarray(a, np.float64).reshape(channels, n, 2)
    return a[..., 0] + 1j * a[..., 1]


def fp64_c2c(x: np.ndarray, n: int, channels: int, inverse: bool = False) -> np.ndarray:
    z = as_complex(x, n, channels)
    return np.fft.ifft(z, axis=1) if inverse else np.fft.fft(z, axis=1)


def fp64_r2c(x: np.ndarray, n: int, channels: int, outmode: int = 0) -> np.ndarray:
    z = np.fft.fft(np.asarray(x, np.float64).reshape(channels, n), axis=1)
    return z if outmode else z[:, : n // 2 + 1]


def fp64_c2r(x: np.ndarray, n: int, channels: int, inmode: int = 0) -> np.ndarray:
    """The reference c2r algorithm in exact arithmetic (FP64, exact pi):
    Z[i] = X[i] A'[i] + b[i] B'[i] with A' = (1 - sin t)/2 + i cos t/2,
    B' = (1 + sin t)/2 - i cos t/2, t = 2 pi i / N, b[i] = conj(X[N/2-i])
    (inMode 0) or X[i+N/2] (inMode 1); then the N/2-point inverse DFT read as
    N interleaved reals. For a Hermitian spectrum this is numpy's irfft."""
    h = n // 2
    nin = h + 1 if inmode == 0 else n
    z = as_complex(x, nin, channels)
    i = np.arange(h)
    t = 2 * np.pi * i / n
    a = 0.5 * (1 - np.sin(t)) + 0.5j * np.cos(t)
    bb = 0.5 * (1 + np.sin(t)) - 0.5j * np.cos(t)
    b = np.conj(z[:, h - i]) if inmode == 0 else z[:, i + h]
    zz = z[:, :h] * a + b * bb
    y = np.fft.ifft(zz, axis=1)
    out = np.empty((channels, n))
    out[:, 0::2] = y.real
    out[:, 1::2] = y.imag
    return out


def rel_l2(got, ref) -> float:
    got = np.asarray(got)
    ref = np.asarray(ref)
    if np.iscomplexobj(ref) and not np.iscomplexobj(got):
        got = got.astype(np.float64).reshape(ref.shape + (2,))
        got = got[..., 0] + 1j * got[..., 1]
    den = np.linalg.norm(ref.ravel())
    num = np.linalg.norm((np.asarray(got, np.complex128) - ref).ravel())
    return float(num / den) if den > 0 else float(num)


# --------------------------------------------------------------------------
# The reference's own _cn code (oracle/_ref)
# --------------------------------------------------------------------------

class BufParams(C.Structure):
    """FFTLIB_bufParams1D_t (src/common/FFTLIB_bufParams.h:62-67)."""
    _fields_ = [("data_type", C.c_uint32), ("dim_x", C.c_uint32)]


FFTLIB_INT16, FFTLIB_UINT32, FFTLIB_FLOAT32 = 1, 8, 12


def ref_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"libref_{k}.so"))
               for k in ("c2c", "ifft", "r2c", "c2r", "i16", "twgen"))


_ref = {}


def ref_lib(kind: str) -> C.CDLL:
    if kind not in _ref:
        path = os.path.join(REF_DIR, f"libref_{kind}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} not built (make -C oracle all)")
        _ref[kind] = C.CDLL(path)
    return _ref[kind]


def _bp(dtype, dim):
    return C.byref(BufParams(dtype, dim))


def ref_tw_gen_c2c(n: int) -> np.ndarray:
    w = np.zeros(max(2 * n, 2), np.float32)
    ref_lib("twgen").ref_tw_gen_c2c(w.ctypes.data_as(C.c_void_p), _u32(n))
    return w[: 2 * n]


def ref_tw_gen_i16(n: int) -> np.ndarray:
    w = np.zeros(max(2 * n, 2), np.int16)
    ref_lib("twgen").ref_tw_gen_i16(w.ctypes.data_as(C.c_void_p), _u32(n))
    return w[: 2 * n]


def ref_tw_gen_r2c(n: int) -> np.ndarray:
    w = np.zeros(max(n, 2), np.float32)
    ref_lib("r2c").tw_gen_r2c(w.ctypes.data_as(C.c_void_p), C.c_int32(n))
    return w[:n]


def ref_tw_gen_c2r(n: int) -> np.ndarray:
    w = np.zeros(max(n, 2), np.float32)
    ref_lib("c2r").ifft_c2r_tw_gen(w.ctypes.data_as(C.c_void_p), C.c_int32(n))
    return w[:n]


def ref_split_factor_r2c(n: int) -> np.ndarray:
    sf = np.zeros(2 * n, np.float32)
    ref_lib("r2c").split_factor_gen_r2c(sf.ctypes.data_as(C.c_void_p), C.c_int32(n))
    return sf


def ref_split_factor_c2r(n: int) -> np.ndarray:
    sf = np.zeros(2 * n, np.float32)
    ref_lib("c2r").ifft_c2r_split_factor_gen(sf.ctypes.data_as(C.c_void_p), C.c_int32(n))
    return sf


def _vp(a):
    return a.ctypes.data_as(C.c_void_p)


def ref_c2c_f32(x, n, channels, inverse=False, w=None):
    """Reference FFTLIB_{fft,ifft}1dBatched_i32fc_c32fc_o32fc_cn."""
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(max(2 * n * channels, 2), np.float32)
    w = ref_tw_gen_c2c(n) if w is None else np.ascontiguousarray(w, np.float32)
    L = ref_lib("ifft" if inverse else "c2c")
    fn = L.FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_cn if inverse else L.FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn
    dim = 2 * n * channels
    rc = fn(_vp(xin), _bp(FFTLIB_FLOAT32, dim), _vp(w), _bp(FFTLIB_FLOAT32, 2 * n), _vp(y),
            _bp(FFTLIB_FLOAT32, dim), _u32(n), _u32(channels))
    if rc:
        raise ValueError(f"reference c2c returned {rc}")
    return y[: 2 * n * channels]


def ref_r2c_f32(x, n, channels, outmode=0):
    xin = np.ascontiguousarray(x, np.float32).copy()
    nout = n if outmode else n // 2 + 1
    y = np.zeros(2 * nout * channels, np.float32)
    xfft = np.zeros(n * channels + 2, np.float32)
    w = ref_tw_gen_r2c(n)
    sf = ref_split_factor_r2c(n)
    L = ref_lib("r2c")
    dim = n * channels
    rc = L.FFTLIB_fft1dBatched_i32f_c32fc_o32fc_cn(
        _vp(xin), _bp(FFTLIB_FLOAT32, dim), _vp(w), _bp(FFTLIB_FLOAT32, dim), _vp(xfft),
        _bp(FFTLIB_FLOAT32, dim), _vp(sf), _bp(FFTLIB_FLOAT32, 2 * n), _vp(y), _bp(FFTLIB_FLOAT32, dim),
        _u32(n), _u32(channels), C.c_uint8(outmode))
    if rc:
        raise ValueError(f"reference r2c returned {rc}")
    return y


def ref_c2r_f32(x, n, channels, inmode=0):
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(n * channels, np.float32)
    xfft = np.zeros((n + 1) * 2 * channels, np.float32)
    w = ref_tw_gen_c2r(n)
    sf = ref_split_factor_c2r(n)
    L = ref_lib("c2r")
    dim = n * channels
    rc = L.FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_cn(
        _vp(xin), _bp(FFTLIB_FLOAT32, dim), _vp(w), _bp(FFTLIB_FLOAT32, dim), _vp(xfft),
        _bp(FFTLIB_FLOAT32, dim), _vp(sf), _bp(FFTLIB_FLOAT32, 2 * n), _vp(y), _bp(FFTLIB_FLOAT32, dim),
        _u32(n), _u32(channels), C.c_uint8(inmode))
    if rc:
        raise ValueError(f"reference c2r returned {rc}")
    return y


def ref_c2c_i16(x, n, channels, shifts, w=None):
    xin = np.ascontiguousarray(x, np.int16).copy()
    y = np.zeros(2 * n * channels, np.int16)
    w = ref_tw_gen_i16(n) if w is None else np.ascontiguousarray(w, np.int16)
    sh = np.ascontiguousarray(shifts, np.uint32)
    L = ref_lib("i16")
    dim = 2 * n * channels
    rc = L.FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_cn(
        _vp(xin), _bp(FFTLIB_INT16, dim), _vp(w), _bp(FFTLIB_INT16, 2 * n), _vp(y), _bp(FFTLIB_INT16, dim),
        _vp(sh), _bp(FFTLIB_UINT32, len(sh)), _u32(n), _u32(channels))
    if rc:
        raise ValueError(f"reference int16 returned {rc}")
    return y


# --------------------------------------------------------------------------
# Single-transform kernels FFTLIB_{fft,ifft}1d_* (length from dim_x)
#
# Restatement: each is the batched kernel with one channel --
#   fft1d c2c / ifft1d c2c : FFTLIB_{fft,ifft}1d_i32fc_c32fc_o32fc_cn.c, the
#       same mixed-radix DIF + digit reversal (ifft: conjugate in, conjugate
#       and 1/N out, ..._ifft1d_i32fc_c32fc_o32fc_cn.c:436-437)
#   fft1d r2c  : FFTLIB_fft1d_i32f_c32fc_o32fc_cn.c:34-140, the N/2-point
#       batched c2c then the split post-process over the full spectrum
#       (outmode 1 of the batched kernel)
#   ifft1d c2r : FFTLIB_ifft1d_i32fc_c32fc_o32f_cn.c:39-74, the split
#       pre-process reading bins i and i+N/2 (inMode 1) then the single
#       N/2-point ifft
#   fft1d int16: FFTLIB_fft1d_i16sc_c16sc_o16sc_cn.c:189-306, the batched
#       int16 loop with one channel
# --------------------------------------------------------------------------

def fft1d_c2c_f32(x: np.ndarray, n: int, inverse: bool = False) -> np.ndarray:
    return fft_c2c_f32(x, n, 1, inverse)


def fft1d_r2c_f32(x: np.ndarray, n: int) -> np.ndarray:
    return fft_r2c_f32(x, n, 1, 1)


def fft1d_c2r_f32(x: np.ndarray, n: int) -> np.ndarray:
    return fft_c2r_f32(x, n, 1, 1)


def fft1d_c2c_i16(x: np.ndarray, n: int, shifts) -> np.ndarray:
    return fft_c2c_i16(x, n, 1, shifts)


def ref1d_available() -> bool:
    return all(os.path.exists(os.path.join(REF_DIR, f"libref_1d_{k}.so"))
               for k in ("c2c", "ifft", "r2c", "c2r", "i16"))


def ref_fft1d_c2c_f32(x, n, inverse=False, w=None):
    """Reference FFTLIB_{fft,ifft}1d_i32fc_c32fc_o32fc_cn (dim_x = 2n)."""
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(max(2 * n, 2), np.float32)
    w = ref_tw_gen_c2c(n) if w is None else np.ascontiguousarray(w, np.float32)
    L = ref_lib("1d_ifft" if inverse else "1d_c2c")
    fn = L.FFTLIB_ifft1d_i32fc_c32fc_o32fc_cn if inverse else L.FFTLIB_fft1d_i32fc_c32fc_o32fc_cn
    b = _bp(FFTLIB_FLOAT32, 2 * n)
    rc = fn(_vp(xin), b, _vp(w), b, _vp(y), b)
    if rc:
        raise ValueError(f"reference fft1d c2c returned {rc}")
    return y[: 2 * n]


def ref_fft1d_r2c_f32(x, n):
    """Reference FFTLIB_fft1d_i32f_c32fc_o32fc_cn (dim_x = n). Its output
    buffer gets one spare bin: the reference also stores bin n (the conjugate
    of bin 0) there."""
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(2 * (n + 1), np.float32)
    xfft = np.zeros(2 * (n + 1), np.float32)
    w = ref_tw_gen_r2c(n)
    sf = ref_split_factor_r2c(n)
    b = _bp(FFTLIB_FLOAT32, n)
    rc = ref_lib("1d_r2c").FFTLIB_fft1d_i32f_c32fc_o32fc_cn(_vp(xin), b, _vp(w), b, _vp(xfft), b, _vp(sf), b,
                                                             _vp(y), b)
    if rc:
        raise ValueError(f"reference fft1d r2c returned {rc}")
    return y[: 2 * n]


def ref_fft1d_c2r_f32(x, n):
    """Reference FFTLIB_ifft1d_i32fc_c32fc_o32f_cn (dim_x = n; n bins in)."""
    xin = np.ascontiguousarray(x, np.float32).copy()
    y = np.zeros(max(n, 2), np.float32)
    xfft = np.zeros(2 * (n + 1), np.float32)
    w = ref_tw_gen_c2r(n)
    sf = ref_split_factor_c2r(n)
    b = _bp(FFTLIB_FLOAT32, n)
    rc = ref_lib("1d_c2r").FFTLIB_ifft1d_i32fc_c32fc_o32f_cn(_vp(xin), b, _vp(w), b, _vp(xfft), b, _vp(sf), b,
                                                              _vp(y), b)
    if rc:
        raise ValueError(f"reference ifft1d c2r returned {rc}")
    return y[:n]


def ref_fft1d_c2c_i16(x, n, shifts, w=None):
    """Reference FFTLIB_fft1d_i16sc_c16sc_o16sc_cn (dim_x = 2n)."""
    xin = np.ascontiguousarray(x, np.int16).copy()
    y = np.zeros(2 * n, np.int16)
    w = ref_tw_gen_i16(n) if w is None else np.ascontiguousarray(w, np.int16)
    sh = np.ascontiguousarray(shifts, np.uint32)
    b = _bp(FFTLIB_INT16, 2 * n)
    rc = ref_lib("1d_i16").FFTLIB_fft1d_i16sc_c16sc_o16sc_cn(_vp(xin), b, _vp(w), b, _vp(y), b, _vp(sh),
                                                              _bp(FFTLIB_UINT32, len(sh)))
    if rc:
        raise ValueError(f"reference fft1d int16 returned {rc}")
    return y


# --------------------------------------------------------------------------
# Integer DFT coordinator (FFTLIB_FFT_fft_ixX_cxX_oxX, INT16 / INT32):
# oracle/mma_int_oracle.c, values carried in int32 arrays
# --------------------------------------------------------------------------

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")


def _mma_lib():
    L = lib()
    if not getattr(L, "_mma_bound", False):
        L.orc_mma_variant.argtypes = [C.c_int, _u32, _u32, _u32]
        L.orc_mma_w_size.argtypes = [C.c_int, _u32, _u32, _u32]
        L.orc_mma_w_size.restype = _u32
        L.orc_mma_twgen.argtypes = [C.c_int, _u32, _u32, _u32, _i32p]
        L.orc_mma_exec.argtypes = [C.c_int, _u32, _u32, _u32, _u32p, _i32p, _i32p, _i32p]
        L.orc_mma_w1.argtypes = [C.c_int, _u32, _i32p]
        L.orc_mma_w_size_v.argtypes = [C.c_int, C.c_int, _u32]
        L.orc_mma_w_size_v.restype = _u32
        L.orc_mma_twgen_v.argtypes = [C.c_int, C.c_int, _u32, _u32, _u32, _i32p]
        L.orc_mma_exec_v.argtypes = [C.c_int, C.c_int, _u32, _u32, _u32, _u32p, _i32p, _i32p, _i32p]
        L.orc_linalg_mm.argtypes = [C.c_int, _u32, _u32, _u32, _i32p, C.c_uint64, _i32p, C.c_uint64, _i32p,
                                    C.c_uint64, C.c_int32]
        L._mma_bound = True
    return L


_INT_DT = {8: np.int8, 16: np.int16, 32: np.int32}


def mma_variant(bits: int, n: int, batch: int, interleave: int) -> int:
    """1 dftSmall, 2 dftLarge, 3 highRadixDecompositions."""
    return _mma_lib().orc_mma_variant(bits, n, batch, interleave)


def mma_twgen(bits: int, n: int, batch: int, interleave: int, variant: int | None = None) -> np.ndarray:
    """The caller's table of the coordinator (variant None: its rule) or of
    one variant (1 dftSmall, 2 dftLarge, 3 highRadix)."""
    L = _mma_lib()
    v = mma_variant(bits, n, batch, interleave) if variant is None else variant
    w = np.zeros(L.orc_mma_w_size_v(bits, v, n), np.int32)
    L.orc_mma_twgen_v(bits, v, n, batch, interleave, w)
    return w.astype(np.int16 if bits == 16 else np.int32)


def mma_w1(bits: int, n: int) -> np.ndarray:
    """The highRadix internal table (MMA x MMA entries)."""
    L = _mma_lib()
    mma = 32 if bits == 16 else 16
    w = np.zeros(mma * mma, np.int32)
    L.orc_mma_w1(bits, n, w)
    return w.astype(np.int16 if bits == 16 else np.int32)


def ref_mma_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libref_mma.so"))


def ref_mma_exec(bits: int, n: int, batch: int, interleave: int, shifts, x, w=None,
                 variant: int | None = None) -> np.ndarray:
    """The reference's natural-C integer DFT (dftSmall / LINALG / highRadix
    _cn) through oracle/mma_ref_driver.cpp, with this oracle's tables."""
    dt = np.int16 if bits == 16 else np.int32
    v = mma_variant(bits, n, batch, interleave) if variant is None else variant
    if w is None:
        w = mma_twgen(bits, n, batch, interleave, v)
    sh = np.zeros(5, np.uint32)
    sh[: len(shifts)] = shifts
    xin = np.ascontiguousarray(x, dt).copy()
    y = np.zeros(2 * n * batch, dt)
    w1 = mma_w1(bits, n)
    L = ref_lib("mma")
    rc = L.ref_mma_exec(C.c_int(bits), C.c_int(v), _u32(n), _u32(batch), _u32(interleave), _vp(sh),
                        _vp(np.ascontiguousarray(w, dt)), _vp(w1), _vp(xin), _vp(y))
    if rc:
        raise ValueError(f"reference integer DFT returned {rc}")
    return y


def mma_exec(bits: int, n: int, batch: int, interleave: int, shifts, x, w=None,
             variant: int | None = None) -> np.ndarray:
    L = _mma_lib()
    v = mma_variant(bits, n, batch, interleave) if variant is None else variant
    if w is None:
        w = mma_twgen(bits, n, batch, interleave, v)
    sh = np.zeros(5, np.uint32)
    sh[: len(shifts)] = shifts
    y = np.zeros(2 * n * batch, np.int32)
    rc = L.orc_mma_exec_v(bits, v, n, batch, interleave, sh, np.ascontiguousarray(w, np.int32),
                          np.ascontiguousarray(x, np.int32), y)
    if rc:
        raise ValueError(f"oracle integer DFT does not cover N={n}")
    return y.astype(np.int16 if bits == 16 else np.int32)


def linalg_mm(bits: int, a: np.ndarray, b: np.ndarray, shift: int, c_shape=None, ldc=None) -> np.ndarray:
    """The LINALG multiply C = shiftAndRound(A B, shift) (oracle/mma_int_oracle.c).
    a, b: 2-D arrays whose row strides (in elements, from their strides) may
    exceed their widths. Returns C as a dense M x N array of the data type."""
    L = _mma_lib()
    M, K = a.shape
    K2, N = b.shape
    assert K == K2
    a32 = np.ascontiguousarray(a, np.int32)
    b32 = np.ascontiguousarray(b, np.int32)
    c = np.zeros((M, N), np.int32)
    L.orc_linalg_mm(bits, M, K, N, a32, max(K, 1), b32, max(N, 1), c, max(N, 1), int(shift))
    return c.astype(_INT_DT[bits])


def ref_linalg_mm(bits: int, a: np.ndarray, b: np.ndarray, shift: int) -> np.ndarray:
    """The reference's own LINALG _cn (oracle/_ref/libref_mma.so)."""
    dt = _INT_DT[bits]
    M, K = a.shape
    N = b.shape[1]
    A = np.ascontiguousarray(a, dt)
    B = np.ascontiguousarray(b, dt)
    Cm = np.zeros((M, N), dt)
    L = ref_lib("mma")
    rc = L.ref_linalg_exec(C.c_int(bits), C.c_int32(M), C.c_int32(K), C.c_int32(N), _vp(A), C.c_int32(max(K, 1)),
                           _vp(B), C.c_int32(max(N, 1)), _vp(Cm), C.c_int32(max(N, 1)), C.c_int32(shift))
    if rc:
        raise ValueError(f"reference LINALG returned {rc}")
    return Cm


# --------------------------------------------------------------------------
# Seeded synthetic inputs (splitmix64-free: numpy PCG64 with a fixed seed)
# --------------------------------------------------------------------------

def rng(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


def uniform_c2c(n: int, channels: int, seed: int, lo=-1.0, hi=1.0) -> np.ndarray:
    return rng(seed).uniform(lo, hi, 2 * n * channels).astype(np.float32)


def real_signal(n: int, channels: int, seed: int) -> np.ndarray:
    """N(0,1) noise plus 3 sinusoids per channel (amplitude U[1,10], integer
    bins U{1..N/2-1}, phase U[0,2pi)), the real-input workload."""
    g = rng(seed)
    t = np.arange(n, dtype=np.float64)
    x = g.standard_normal((channels, n))
    for _ in range(3):
        amp = g.uniform(1.0, 10.0, (channels, 1))
        k = g.integers(1, max(n // 2, 2), (channels, 1))
        ph = g.uniform(0.0, 2 * np.pi, (channels, 1))
        x += amp * np.cos(2 * np.pi * k * t / n + ph)
    return x.astype(np.float32).ravel()


def int16_input(n: int, channels: int, seed: int, lo=-2048, hi=2047) -> np.ndarray:
    return rng(seed).integers(lo, hi + 1, 2 * n * channels).astype(np.int16)


# --------------------------------------------------------------------------
# CPU baseline timing of the reference _cn code (bench.py's reference arm and
# cpu_baseline leg): one thread per host core, each calling the reference on
# a contiguous slice of channels (channels are independent in the API). The
# input is re-copied before every repetition (the reference overwrites pX);
# the copy is outside the timed region.
# --------------------------------------------------------------------------

def host_threads() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def time_reference_c2c(n: int, channels: int, threads: int | None = None, reps: int = 3,
                       inverse: bool = False, seed: int = 0):
    """Median seconds for the reference _cn to transform `channels` channels
    of length n, split over `threads` threads; returns (seconds, threads)."""
    import threading
    import time

    threads = max(1, min(threads or host_threads(), channels))
    kind = "ifft" if inverse else "c2c"
    L = ref_lib(kind)
    fn = L.FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_cn if inverse else L.FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn
    fn.restype = C.c_int
    x0 = uniform_c2c(n, channels, seed)
    w = ref_tw_gen_c2c(n)
    per = [channels // threads + (1 if i < channels % threads else 0) for i in range(threads)]
    starts = np.cumsum([0] + per[:-1])
    bufs = [(np.empty(2 * n * c, np.float32), np.empty(2 * n * c, np.float32)) for c in per]
    times = []
    for _ in range(reps):
        for (xb, _), s, c in zip(bufs, starts, per):
            xb[:] = x0[2 * n * s: 2 * n * (s + c)]
        barrier = threading.Barrier(threads + 1)

        def work(i):
            xb, yb = bufs[i]
            c = per[i]
            barrier.wait()
            fn(_vp(xb), _bp(FFTLIB_FLOAT32, 2 * n * c), _vp(w), _bp(FFTLIB_FLOAT32, 2 * n), _vp(yb),
               _bp(FFTLIB_FLOAT32, 2 * n * c), _u32(n), _u32(c))

        ts = [threading.Thread(target=work, args=(i,)) for i in range(threads)]
        for t in ts:
            t.start()
        barrier.wait()
        t0 = time.perf_counter()
        for t in ts:
            t.join()
        times.append(time.perf_counter() - t0)
    return float(np.median(times)), threads


# --------------------------------------------------------------------------
# FP64 oracle FFT on the GPU (oracle/fft_f64.cu): the checker for
# benchmark-size batches. Works on torch CUDA tensors (torch is plumbing
# here: device memory, streams and the norms of the comparison).
# --------------------------------------------------------------------------

_glib = None


def gpu_lib() -> C.CDLL:
    global _glib
    if _glib is None:
        path = os.path.join(HERE, "liboracle_gpu.so")
        if not os.path.exists(path):
            subprocess.run(["make", "-s", "-C", HERE, "liboracle_gpu.so"], check=True)
        L = C.CDLL(path)
        L.orc_gpu_fft_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint64, C.c_int,
                                      C.c_void_p]
        L.orc_gpu_fft_f64.restype = C.c_int
        _glib = L
    return _glib


def gpu_fft_f64(x, n: int, batch: int, inverse: bool = False):
    """FP64 DFT (or scaled inverse DFT) of `batch` rows of n interleaved
    complex values held in a CUDA tensor (any float dtype); returns a float64
    CUDA tensor of shape (batch, n, 2)."""
    import torch

    xd = x.reshape(batch, n, 2).to(torch.float64).contiguous()
    y = torch.empty_like(xd)
    w = torch.empty_like(xd)
    st = torch.cuda.current_stream().cuda_stream
    rc = gpu_lib().orc_gpu_fft_f64(xd.data_ptr(), y.data_ptr(), w.data_ptr(), n, batch, int(inverse), st)
    if rc:
        raise RuntimeError(f"orc_gpu_fft_f64 failed (CUDA error {rc})")
    return y


def gpu_rel_l2_rows(got, ref, batch: int):
    """(overall rel-L2, largest per-row rel-L2) of `got` against `ref`, both
    holding `batch` rows (CUDA tensors; compared in FP64). Rows whose
    reference is all zero count by their absolute error."""
    import torch

    g = got.reshape(batch, -1).to(torch.float64)
    r = ref.reshape(batch, -1).to(torch.float64)
    e = torch.linalg.vector_norm(g - r, dim=1)
    d = torch.linalg.vector_norm(r, dim=1)
    overall = float(torch.linalg.vector_norm(e) / torch.linalg.vector_norm(d))
    per = torch.where(d > 0, e / torch.where(d > 0, d, torch.ones_like(d)), e)
    return overall, float(per.max())


def gpu_check_c2c(x, y, n: int, batch: int, inverse: bool = False, chunk_points: int = 1 << 26):
    """Checks FP32 results y of a batched c2c (inverse) FFT of x against the
    GPU FP64 oracle, in chunks of whole rows; returns (overall rel-L2,
    largest per-row rel-L2)."""
    import torch

    rows = max(1, chunk_points // max(n, 1))
    xs = x.reshape(batch, 2 * n)
    ys = y.reshape(batch, 2 * n)
    err2 = 0.0
    ref2 = 0.0
    worst = 0.0
    for b0 in range(0, batch, rows):
        b1 = min(batch, b0 + rows)
        ref = gpu_fft_f64(xs[b0:b1], n, b1 - b0, inverse)
        g = ys[b0:b1].to(torch.float64).reshape(b1 - b0, -1)
        r = ref.reshape(b1 - b0, -1)
        e = torch.linalg.vector_norm(g - r, dim=1)
        d = torch.linalg.vector_norm(r, dim=1)
        err2 += float((e * e).sum())
        ref2 += float((d * d).sum())
        per = torch.where(d > 0, e / torch.where(d > 0, d, torch.ones_like(d)), e)
        worst = max(worst, float(per.max()))
        del ref, g, r
    return (err2 ** 0.5) / (ref2 ** 0.5 if ref2 > 0 else 1.0), worst


def gpu_fp64_r2c(x, n: int, channels: int, outmode: int = 0):
    """FP64 spectrum of `channels` rows of n reals (CUDA tensor): the n-point
    DFT of the real row, its first n/2+1 bins (outmode 0) or all n; returns
    float64 (channels, bins, 2)."""
    import torch

    z = torch.zeros(channels, n, 2, dtype=torch.float64, device=x.device)
    z[..., 0] = x.reshape(channels, n).to(torch.float64)
    y = gpu_fft_f64(z, n, channels)
    return y if outmode else y[:, : n // 2 + 1].contiguous()


def gpu_fp64_c2r(x, n: int, channels: int, inmode: int = 0):
    """The reference c2r algorithm in FP64 on the GPU (the same definition as
    fp64_c2r): Z[i] = X[i] A'[i] + b[i] B'[i], then the n/2-point inverse
    DFT read as n interleaved reals; returns float64 (channels, n)."""
    import math

    import torch

    h = n // 2
    nin = h + 1 if inmode == 0 else n
    z = x.reshape(channels, nin, 2).to(torch.float64)
    zc = torch.complex(z[..., 0], z[..., 1])
    i = torch.arange(h, device=x.device, dtype=torch.float64)
    t = 2 * math.pi * i / n
    a = torch.complex(0.5 * (1 - torch.sin(t)), 0.5 * torch.cos(t))
    bb = torch.complex(0.5 * (1 + torch.sin(t)), -0.5 * torch.cos(t))
    ii = torch.arange(h, device=x.device)
    b = torch.conj(zc[:, h - ii]) if inmode == 0 else zc[:, ii + h]
    zz = zc[:, :h] * a + b * bb
    y = gpu_fft_f64(torch.view_as_real(zz.contiguous()), h, channels, inverse=True)
    return y.reshape(channels, n)
