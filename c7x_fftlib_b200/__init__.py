"""c7x_fftlib_b200 -- B200-native FFTLIB 1-D FFT hot path (batched and
single-transform kernels, the DFT coordinator, mixed-size batches).

The product is ``libfftlib_b200.so`` (hand-written sm_100a CUDA behind the
FFTLIB C API, headers in ``include/``). This package builds it in-tree
(``c7x_fftlib_b200._build``) and binds it with ctypes under the reference
names, so Python callers (tests, benchmarks) drive exactly the C entry points
a C caller would link against. There is no fallback: if the shared library
is missing, ``lib()`` raises.
"""
from __future__ import annotations

import ctypes as C
import os

__all__ = ["lib", "BufParams", "pblock", "ptr", "check", "FftlibError"]

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libfftlib_b200.so")

# FFTLIB_STATUS (src/common/FFTLIB_types.h:168-211)
FFTLIB_SUCCESS = 0
FFTLIB_ERR_FAILURE = 1
FFTLIB_ERR_INVALID_VALUE = 2
FFTLIB_ERR_INVALID_TYPE = 3
FFTLIB_ERR_INVALID_DIMENSION = 4
FFTLIB_ERR_NULL_POINTER = 5
FFTLIB_ERR_NOT_IMPLEMENTED = 6
FFTLIB_ERR_NOT_ALIGNED_PTRS_STRIDES = 8
FFTLIB_ERR_INVALID_SHIFT = 12
FFTLIB_ERR_INVALID_OUTMODE = 14
FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_INPUT_TYPE = 10000
FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_OUTPUT_TYPE = 10001
FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_TYPE_COMBINATION = 10002

# FFTLIB_data_type_e (src/common/FFTLIB_bufParams.h:22-42)
FFTLIB_INT8 = 0
FFTLIB_INT16 = 1
FFTLIB_INT32 = 2
FFTLIB_UINT32 = 8
FFTLIB_FLOAT32 = 12

# FFTLIB_FUNCTION_STYLE
FFTLIB_FUNCTION_NATC = 0
FFTLIB_FUNCTION_OPTIMIZED = 1

SE_PARAM_SIZE = 64
PBLOCK_SIZE = {
    "c2c": 31 * SE_PARAM_SIZE + 18 * 4,
    "ifft": 31 * SE_PARAM_SIZE + 18 * 4,
    "r2c": 41 * SE_PARAM_SIZE + 18 * 4,
    "c2r": 41 * SE_PARAM_SIZE + 18 * 4,
    "i16": 13 * SE_PARAM_SIZE,
    "1d_c2c": 27 * SE_PARAM_SIZE + 16 * 4,
    "1d_ifft": 27 * SE_PARAM_SIZE + 16 * 4,
    "1d_r2c": 35 * SE_PARAM_SIZE + 18 * 4,
    "1d_c2r": 34 * SE_PARAM_SIZE + 16 * 4,
    "1d_i16": 9 * SE_PARAM_SIZE,
}


class FftlibError(RuntimeError):
    pass


class BufParams(C.Structure):
    """FFTLIB_bufParams1D_t (src/common/FFTLIB_bufParams.h:62-67)."""
    _fields_ = [("data_type", C.c_uint32), ("dim_x", C.c_uint32)]


class MmaInitArgs(C.Structure):
    """FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs
    (src/fft_c7xmma/FFTLIB_FFT_fft_ixX_cxX_oxX/FFTLIB_FFT_fft_ixX_cxX_oxX.h:42-64)."""
    _fields_ = [("funcStyle", C.c_int8), ("fftSize", C.c_uint32), ("batchSize", C.c_uint32),
                ("interleave", C.c_uint32), ("shiftVector", C.c_uint32 * 5)]


class DftVariantInitArgs(C.Structure):
    """FFTLIB_FFT_dftSmall_ixX_cxX_oxX_InitArgs and FFTLIB_FFT_dftLarge_ixX_cxX_oxX_InitArgs
    (..._dftSmall_ixX_cxX_oxX.h:40-62, ..._dftLarge_ixX_cxX_oxX.h:42-64: one shift).
    The highRadixDecompositions InitArgs has the coordinator's layout (five shifts)."""
    _fields_ = [("funcStyle", C.c_int8), ("fftSize", C.c_uint32), ("batchSize", C.c_uint32),
                ("interleave", C.c_uint32), ("shiftVector", C.c_uint32 * 1)]


class BufParams2D(C.Structure):
    """FFTLIB_bufParams2D_t (src/common/FFTLIB_bufParams.h:69-78): stride_y in bytes."""
    _fields_ = [("data_type", C.c_uint32), ("dim_x", C.c_uint32), ("dim_y", C.c_uint32), ("stride_y", C.c_int32)]


class LinalgInitArgs(C.Structure):
    """FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs
    (src/linalg_c7xmma/FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/..._oxX.h:48-51)."""
    _fields_ = [("funcStyle", C.c_int8), ("shift", C.c_int8)]


# the coordinator's variants as separate kernels: name prefix and InitArgs type
DFT_VARIANTS = {
    "dftSmall": ("FFTLIB_FFT_dftSmall_ixX_cxX_oxX_", DftVariantInitArgs),
    "dftLarge": ("FFTLIB_FFT_dftLarge_ixX_cxX_oxX_", DftVariantInitArgs),
    "highRadix": ("FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX_", MmaInitArgs),
}
LINALG = "FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_"

# paths the coordinator's init picks (FFTLIB_b200_FFT_fft_path)
MMA_PATH_TC = 1
MMA_PATH_FFT = 2

_vp = C.c_void_p
_bpp = C.POINTER(BufParams)
_u32 = C.c_uint32
_u8 = C.c_uint8

_SIGS = {
    # name suffix: argtypes (after the common prefix)
    "c2c": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32, _vp],
    "c2c_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32],
    "real": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32, _u8, _vp],
    "real_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32, _u8],
    "real_check": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32, _u8, _vp],
    "real_check_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32, _u8],
    "i16": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32, _vp],
    "i16_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _u32, _u32],
    # single-transform kernels: lengths from bufParamsX->dim_x
    "1d_c2c": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp],
    "1d_c2c_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp],
    "1d_real": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _vp],
    "1d_real_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp],
    "1d_i16": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp, _vp],
    "1d_i16_cn": [_vp, _bpp, _vp, _bpp, _vp, _bpp, _vp, _bpp],
}

KERNELS = {
    "c2c": "FFTLIB_fft1dBatched_i32fc_c32fc_o32fc",
    "ifft": "FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc",
    "r2c": "FFTLIB_fft1dBatched_i32f_c32fc_o32fc",
    "c2r": "FFTLIB_ifft1dBatched_i32fc_c32fc_o32f",
    "i16": "FFTLIB_fft1dBatched_i16sc_c16sc_o16sc",
    "1d_c2c": "FFTLIB_fft1d_i32fc_c32fc_o32fc",
    "1d_ifft": "FFTLIB_ifft1d_i32fc_c32fc_o32fc",
    "1d_r2c": "FFTLIB_fft1d_i32f_c32fc_o32fc",
    "1d_c2r": "FFTLIB_ifft1d_i32fc_c32fc_o32f",
    "1d_i16": "FFTLIB_fft1d_i16sc_c16sc_o16sc",
}

_lib = None


def lib() -> C.CDLL:
    """Load libfftlib_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise FftlibError(f"{LIB_PATH} is missing; build it with `python -m c7x_fftlib_b200._build`")
    L = C.CDLL(LIB_PATH)
    for kind, base in KERNELS.items():
        if kind in ("c2c", "ifft"):
            fam = {"_init": "c2c", "_kernel": "c2c", "_checkParams": "c2c", "_cn": "c2c_cn", "_checkParams_cn": "c2c_cn"}
        elif kind in ("r2c", "c2r"):
            fam = {"_init": "real", "_kernel": "real", "_checkParams": "real_check", "_cn": "real_cn",
                   "_checkParams_cn": "real_check_cn"}
        elif kind == "i16":
            fam = {"_init": "i16", "_kernel": "i16", "_checkParams": "i16", "_cn": "i16_cn", "_checkParams_cn": "i16_cn"}
        elif kind in ("1d_c2c", "1d_ifft"):
            fam = {"_init": "1d_c2c", "_kernel": "1d_c2c", "_checkParams": "1d_c2c", "_cn": "1d_c2c_cn",
                   "_checkParams_cn": "1d_c2c_cn"}
        elif kind in ("1d_r2c", "1d_c2r"):
            fam = {"_init": "1d_real", "_kernel": "1d_real", "_checkParams": "1d_c2c", "_cn": "1d_real_cn",
                   "_checkParams_cn": "1d_c2c_cn"}
        else:
            fam = {"_init": "1d_i16", "_kernel": "1d_i16", "_checkParams": "1d_i16", "_cn": "1d_i16_cn",
                   "_checkParams_cn": "1d_i16_cn"}
        for suffix, sig in fam.items():
            fn = getattr(L, base + suffix)
            fn.argtypes = _SIGS[sig]
            fn.restype = C.c_int
    L.FFTLIB_b200_lastError.restype = C.c_char_p
    L.FFTLIB_b200_lastError.argtypes = []
    L.FFTLIB_b200_version.restype = C.c_int
    L.FFTLIB_b200_describePlan.argtypes = [_u32, C.c_char_p, _u32]
    L.FFTLIB_b200_describePlan.restype = C.c_int
    L.FFTLIB_b200_describeBlock.argtypes = [_vp, C.c_char_p, _u32]
    L.FFTLIB_b200_describeBlock.restype = C.c_int
    L.FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync.argtypes = [_vp, _vp, _u32, _u32, _vp, _vp]
    L.FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32fc_kernelAsync.argtypes = [_vp, _vp, _u32, _u32, _vp, _vp]
    L.FFTLIB_b200_fft1dBatched_i32f_c32fc_o32fc_kernelAsync.argtypes = [_vp, _vp, _vp, _u32, _u32, _u8, _vp, _vp]
    L.FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32f_kernelAsync.argtypes = [_vp, _vp, _vp, _u32, _u32, _u8, _vp, _vp]
    L.FFTLIB_b200_fft1dBatched_i16sc_c16sc_o16sc_kernelAsync.argtypes = [_vp, _vp, _vp, _vp, _u32, _u32, _u32, _vp,
                                                                         _vp]
    L.FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc.argtypes = [_vp, _vp, _u32, _u32, _vp]
    L.FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc.restype = C.c_int
    L.FFTLIB_b200_fftMixed_supported.argtypes = [_u32]
    L.FFTLIB_b200_fftMixed_create.argtypes = [C.POINTER(C.c_uint32), _u32, _u32, C.POINTER(_vp)]
    L.FFTLIB_b200_fftMixed_exec.argtypes = [_vp, _vp, _vp, _vp]
    L.FFTLIB_b200_fftMixed_execPerSize.argtypes = [_vp, _vp, _vp, _vp]
    L.FFTLIB_b200_fftMixed_describe.argtypes = [_vp, C.c_char_p, _u32]
    L.FFTLIB_b200_fftMixed_destroy.argtypes = [_vp]
    for fname in ("fftMixed_supported", "fftMixed_create", "fftMixed_exec", "fftMixed_execPerSize",
                  "fftMixed_describe", "fftMixed_destroy"):
        getattr(L, "FFTLIB_b200_" + fname).restype = C.c_int
    M = "FFTLIB_FFT_fft_ixX_cxX_oxX_"
    _ia = C.POINTER(MmaInitArgs)
    getattr(L, M + "getHandleSize").argtypes = [_ia]
    getattr(L, M + "getHandleSize").restype = C.c_int32
    getattr(L, M + "getSizes").argtypes = [_ia, _bpp, _bpp, _bpp]
    getattr(L, M + "twGen").argtypes = [_ia, _vp, _bpp]
    getattr(L, M + "init").argtypes = [_vp, _bpp, _bpp, _bpp, _ia]
    getattr(L, M + "init_checkParams").argtypes = [_vp, _bpp, _bpp, _bpp, _ia]
    getattr(L, M + "exec").argtypes = [_vp, _vp, _vp, _vp]
    getattr(L, M + "exec_checkParams").argtypes = [_vp, _vp, _vp, _vp]
    for f in ("getSizes", "twGen", "init", "init_checkParams", "exec", "exec_checkParams"):
        getattr(L, M + f).restype = C.c_int
    for prefix, args_t in DFT_VARIANTS.values():
        _va = C.POINTER(args_t)
        getattr(L, prefix + "getHandleSize").argtypes = [_va]
        getattr(L, prefix + "getHandleSize").restype = C.c_int32
        getattr(L, prefix + "getSizes").argtypes = [_va, _bpp, _bpp, _bpp]
        getattr(L, prefix + "twGen").argtypes = [_va, _vp, _bpp]
        getattr(L, prefix + "init").argtypes = [_vp, _bpp, _bpp, _bpp, _va]
        getattr(L, prefix + "init_checkParams").argtypes = [_vp, _bpp, _bpp, _bpp, _va]
        getattr(L, prefix + "exec").argtypes = [_vp, _vp, _vp, _vp]
        getattr(L, prefix + "exec_checkParams").argtypes = [_vp, _vp, _vp, _vp]
        for f in ("getSizes", "twGen", "init", "init_checkParams", "exec", "exec_checkParams"):
            getattr(L, prefix + f).restype = C.c_int
    _la, _b2 = C.POINTER(LinalgInitArgs), C.POINTER(BufParams2D)
    getattr(L, LINALG + "getHandleSize").argtypes = [_la]
    getattr(L, LINALG + "getHandleSize").restype = C.c_int32
    getattr(L, LINALG + "init").argtypes = [_vp, _b2, _b2, _b2, _la]
    getattr(L, LINALG + "init_checkParams").argtypes = [_vp, _b2, _b2, _b2, _la]
    getattr(L, LINALG + "exec").argtypes = [_vp, _vp, _vp, _vp]
    getattr(L, LINALG + "exec_checkParams").argtypes = [_vp, _vp, _vp, _vp]
    for f in ("init", "init_checkParams", "exec", "exec_checkParams"):
        getattr(L, LINALG + f).restype = C.c_int
    L.FFTLIB_b200_LINALG_matrixMatrixMultiply_execAsync.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.FFTLIB_b200_LINALG_matrixMatrixMultiply_execAsync.restype = C.c_int
    L.FFTLIB_b200_FFT_fft_execAsync.argtypes = [_vp, _vp, _vp, _vp, _vp]
    L.FFTLIB_b200_FFT_fft_execAsync.restype = C.c_int
    L.FFTLIB_b200_FFT_fft_sync.argtypes = [_vp]
    L.FFTLIB_b200_FFT_fft_sync.restype = C.c_int
    L.FFTLIB_b200_FFT_setIntTensorCores.argtypes = [C.c_int32]
    L.FFTLIB_b200_FFT_setIntTensorCores.restype = None
    L.FFTLIB_b200_FFT_fft_path.argtypes = [_vp]
    L.FFTLIB_b200_FFT_fft_path.restype = C.c_int32
    L.FFTLIB_b200_tw_gen_c2c.argtypes = [_vp, _u32]
    L.FFTLIB_b200_tw_gen_i16.argtypes = [_vp, _u32]
    for fn in ("tw_gen_r2c", "split_factor_gen_r2c", "ifft_c2r_tw_gen", "ifft_c2r_split_factor_gen"):
        getattr(L, fn).argtypes = [_vp, C.c_int32]
        getattr(L, fn).restype = None
        getattr(L, "FFTLIB_b200_" + fn + "_device").argtypes = [_vp, C.c_int32, _vp]
        getattr(L, "FFTLIB_b200_" + fn + "_device").restype = C.c_int
    for fn in ("tw_gen_c2c_device", "tw_gen_i16_device"):
        getattr(L, "FFTLIB_b200_" + fn).argtypes = [_vp, _u32, _vp]
        getattr(L, "FFTLIB_b200_" + fn).restype = C.c_int
    _lib = L
    return L


def ptr(x) -> C.c_void_p | None:
    """Address of a buffer: None, an int address, a numpy array, a torch
    tensor (device or host) or a ctypes object."""
    if x is None:
        return None
    if isinstance(x, int):
        return C.c_void_p(x)
    if hasattr(x, "data_ptr"):
        return C.c_void_p(x.data_ptr())
    if hasattr(x, "ctypes"):
        return C.c_void_p(x.ctypes.data)
    return C.cast(x, C.c_void_p)


def pblock(kind: str):
    """A zeroed pBlock of the reference size for kernel kind."""
    return C.create_string_buffer(PBLOCK_SIZE[kind])


def bp(data_type: int, dim_x: int) -> BufParams:
    return BufParams(data_type, dim_x)


def last_error() -> str:
    return lib().FFTLIB_b200_lastError().decode()


def check(status: int, what: str = "FFTLIB call") -> None:
    if status != FFTLIB_SUCCESS:
        raise FftlibError(f"{what} returned {status}: {last_error()}")


def describe_plan(n: int) -> str:
    buf = C.create_string_buffer(256)
    check(lib().FFTLIB_b200_describePlan(n, buf, 256), "describePlan")
    return buf.value.decode()


def describe_block(pblock) -> str:
    """The launch an _init recorded in pblock ("tuned: ..." or "planner: ...")."""
    buf = C.create_string_buffer(256)
    check(lib().FFTLIB_b200_describeBlock(ptr(pblock), buf, 256), "describeBlock")
    return buf.value.decode()


MIXED_INVERSE = 1
MIXED_AUTOTUNE = 2
MIXED_PERSISTENT_ONLY = 4


class MixedBatch:
    """FFTLIB_b200_fftMixed_*: uneven-length c2c batch (device buffers)."""

    def __init__(self, lengths, inverse=False, autotune=False, persistent_only=False):
        import numpy as _np

        self.lengths = _np.ascontiguousarray(lengths, _np.uint32)
        self.h = C.c_void_p()
        flags = (MIXED_INVERSE if inverse else 0) | (MIXED_AUTOTUNE if autotune else 0) | \
            (MIXED_PERSISTENT_ONLY if persistent_only else 0)
        arr = self.lengths.ctypes.data_as(C.POINTER(C.c_uint32))
        check(lib().FFTLIB_b200_fftMixed_create(arr, len(self.lengths), flags, C.byref(self.h)), "fftMixed_create")

    def exec(self, x, y, stream=None):
        check(lib().FFTLIB_b200_fftMixed_exec(self.h, ptr(x), ptr(y), stream), "fftMixed_exec")

    def exec_per_size(self, x, y, stream=None):
        check(lib().FFTLIB_b200_fftMixed_execPerSize(self.h, ptr(x), ptr(y), stream), "fftMixed_execPerSize")

    def describe(self) -> str:
        buf = C.create_string_buffer(8192)
        check(lib().FFTLIB_b200_fftMixed_describe(self.h, buf, 8192), "fftMixed_describe")
        return buf.value.decode()

    def close(self):
        if self.h:
            lib().FFTLIB_b200_fftMixed_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def fn(name: str):
    """The exported C function `name` (reference name or FFTLIB_b200_*)."""
    return getattr(lib(), name)


class DftMma:
    """FFTLIB_FFT_fft_ixX_cxX_oxX_*: the DFT coordinator (getSizes, twGen,
    init_checkParams, init, then exec or the stream-ordered execAsync) for
    FLOAT32 interleaved data or the reference's INT16 / INT32 data
    (dtype, interleave and the five-entry shift vector as in its InitArgs)."""

    def __init__(self, n: int, batch: int, func_style: int = FFTLIB_FUNCTION_OPTIMIZED, w_device=True,
                 dtype: int = FFTLIB_FLOAT32, interleave: int = 1, shifts=None, variant: str | None = None):
        """variant None: the coordinator; "dftSmall", "dftLarge" or "highRadix":
        that kernel on its own (FFTLIB_FFT_<variant>_ixX_cxX_oxX_*)."""
        import numpy as _np

        L = lib()
        M, args_t = ("FFTLIB_FFT_fft_ixX_cxX_oxX_", MmaInitArgs) if variant is None else DFT_VARIANTS[variant]
        self.prefix = M
        self.n, self.batch, self.dtype = n, batch, dtype
        self.args = args_t(func_style, n, batch, interleave)
        nsh = len(self.args.shiftVector)
        for i, v in enumerate([] if shifts is None else list(shifts)[:nsh]):
            self.args.shiftVector[i] = int(v)
        self.bx, self.bw, self.by = (BufParams(dtype, 0) for _ in range(3))
        check(getattr(L, M + "getSizes")(C.byref(self.args), self.bx, self.bw, self.by), "getSizes")
        self.handle = C.create_string_buffer(getattr(L, M + "getHandleSize")(C.byref(self.args)))
        check(getattr(L, M + "init_checkParams")(self.handle, self.bx, self.bw, self.by, C.byref(self.args)),
              "init_checkParams")
        check(getattr(L, M + "init")(self.handle, self.bx, self.bw, self.by, C.byref(self.args)), "init")
        np_dt = {FFTLIB_FLOAT32: _np.float32, FFTLIB_INT16: _np.int16, FFTLIB_INT32: _np.int32}[dtype]
        self.w_host = _np.zeros(self.bw.dim_x, np_dt)
        check(getattr(L, M + "twGen")(C.byref(self.args), ptr(self.w_host), self.bw), "twGen")
        self.w = None
        if w_device:
            import torch

            t_dt = {FFTLIB_FLOAT32: torch.float32, FFTLIB_INT16: torch.int16, FFTLIB_INT32: torch.int32}[dtype]
            self.w = torch.empty(self.bw.dim_x, dtype=t_dt, device="cuda")
            check(getattr(L, M + "twGen")(C.byref(self.args), ptr(self.w), self.bw), "twGen (device)")

    @property
    def path(self) -> int:
        return lib().FFTLIB_b200_FFT_fft_path(self.handle)

    def exec(self, x, y, w=None):
        w = self.w if w is None else w
        check(getattr(lib(), self.prefix + "exec")(self.handle, ptr(x), ptr(w), ptr(y)), "exec")

    def exec_async(self, x, y, stream=None, w=None):
        w = self.w if w is None else w
        check(lib().FFTLIB_b200_FFT_fft_execAsync(self.handle, ptr(x), ptr(w), ptr(y), stream), "execAsync")


class MatMul:
    """FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_*: C = shiftAndRound(A B)
    for INT8 / INT16 / INT32 (init_checkParams, init, then exec or the
    stream-ordered execAsync). Strides are row strides in elements (default:
    dense rows)."""

    ELEM = {FFTLIB_INT8: 1, FFTLIB_INT16: 2, FFTLIB_INT32: 4}

    def __init__(self, m: int, k: int, n: int, dtype: int, shift: int = 0,
                 func_style: int = FFTLIB_FUNCTION_OPTIMIZED, lda=None, ldb=None, ldc=None):
        L = lib()
        es = self.ELEM.get(dtype, 1)
        self.m, self.k, self.n, self.dtype = m, k, n, dtype
        self.args = LinalgInitArgs(func_style, shift)
        self.a = BufParams2D(dtype, k, m, (k if lda is None else lda) * es)
        self.b = BufParams2D(dtype, n, k, (n if ldb is None else ldb) * es)
        self.c = BufParams2D(dtype, n, m, (n if ldc is None else ldc) * es)
        self.handle = C.create_string_buffer(getattr(L, LINALG + "getHandleSize")(C.byref(self.args)))
        check(getattr(L, LINALG + "init_checkParams")(self.handle, self.a, self.b, self.c, C.byref(self.args)),
              "init_checkParams")
        check(getattr(L, LINALG + "init")(self.handle, self.a, self.b, self.c, C.byref(self.args)), "init")

    def exec(self, a, b, c):
        check(getattr(lib(), LINALG + "exec")(self.handle, ptr(a), ptr(b), ptr(c)), "exec")

    def exec_async(self, a, b, c, stream=None):
        check(lib().FFTLIB_b200_LINALG_matrixMatrixMultiply_execAsync(self.handle, ptr(a), ptr(b), ptr(c), stream),
              "execAsync")
