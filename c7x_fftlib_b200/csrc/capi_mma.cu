// capi_mma.cu -- FFTLIB_FFT_fft_ixX_cxX_oxX_*: the DFT coordinator of the
// reference's src/fft_c7xmma/FFTLIB_FFT_fft_ixX_cxX_oxX/
// FFTLIB_FFT_fft_ixX_cxX_oxX.cpp:7-282.
//
// INT16 / INT32 (the reference's types): the reference's own variant choice
// (dftSmall / dftLarge / highRadixDecompositions, ..._oxX.cpp:13-50), tables
// and arithmetic, bit-exact with its natural C (dft_int.cu).
// FLOAT32 (added): init picks between two GPU paths:
//   PATH_TC  -- funcStyle OPTIMIZED and fftSize a power of two in [8, 4096]:
//               the split-precision tensor-core DFT (one DFT-GEMM up to 64,
//               two DFT-GEMM stages with the twiddle fused between above);
//   PATH_FFT -- otherwise, for fftSize = 2^a 3^b 5^c: the CUDA-core FP32 FFT
//               of the fft1dBatched c2c kernel.
#include <string.h>

#include "capi_common.h"
#include "dft_int.h"
#include "fft_c7xmma.h"
#include "fft_c7xmma_variants.h"
#include "fftlib_b200_ext.h"
#include "plan.h"
#include "tables.h"
#include "tc_dft.h"

using namespace fftb200;

namespace {

constexpr uint32_t kMmaMagic = 0x32414D4Du;  // "MMA2"
enum MmaPath : int32_t { PATH_NONE = 0, PATH_TC = 1, PATH_FFT = 2, PATH_INT = 3 };

struct MmaHandle {
    uint32_t magic;
    int32_t path;
    int32_t device;
    int32_t bits;       // PATH_INT: 16 or 32
    int32_t variant;    // PATH_INT: the variant fixed by a variant's init (0: the coordinator's rule)
    FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs init;
    ComplexPlan* plan;  // CUDA-core FFT plan of fftSize (FLOAT32)
};

int variant_of(const MmaHandle* m)
{
    return m->variant ? m->variant : int_dft_variant(m->bits, m->init.fftSize, m->init.batchSize, m->init.interleave);
}

int int_bits(uint32_t type) { return type == FFTLIB_INT16 ? 16 : (type == FFTLIB_INT32 ? 32 : 0); }

// INT16 / INT32 buffer sizes in elements (the reference's getSizes).
FFTLIB_STATUS sizes_int(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* a, int bits, uint32_t* x, uint32_t* w,
                        uint32_t* y)
{
    const uint64_t xy = 2ull * a->fftSize * a->batchSize;
    if (xy > 0xFFFFFFFFull) {
        set_error("fftSize x batchSize x 2 = %llu exceeds the 32-bit dim_x", (unsigned long long)xy);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    *x = *y = (uint32_t)xy;
    *w = int_dft_w_size(bits, a->fftSize, a->batchSize, a->interleave);
    return FFTLIB_SUCCESS;
}

int32_t choose_path(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* a)
{
    if (a->fftSize == 0 || a->batchSize == 0) return PATH_NONE;
    if (a->funcStyle == FFTLIB_FUNCTION_OPTIMIZED && tc_dft_supported(a->fftSize)) return PATH_TC;
    if (is_235(a->fftSize)) return PATH_FFT;
    return PATH_NONE;
}

// FLOAT32 buffer sizes in elements.
FFTLIB_STATUS sizes_f32(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* a, uint32_t* x, uint32_t* w, uint32_t* y)
{
    if (!a->interleave) {
        set_error("FLOAT32 data must be interleaved (interleave = 1)");
        return FFTLIB_ERR_NOT_IMPLEMENTED;
    }
    const int32_t path = choose_path(a);
    if (path == PATH_NONE) {
        set_error("fftSize %u (batchSize %u) has no FLOAT32 path: it must be 2^a 3^b 5^c", a->fftSize, a->batchSize);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const uint64_t xy = 2ull * a->fftSize * a->batchSize;
    if (xy > 0xFFFFFFFFull) {
        set_error("fftSize x batchSize x 2 = %llu exceeds the 32-bit dim_x", (unsigned long long)xy);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    *x = *y = (uint32_t)xy;
    *w = path == PATH_TC ? (uint32_t)tc_dft_w_floats(a->fftSize) : 2u * a->fftSize;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS unsupported_type(uint32_t type)
{
    set_error("data type %u: the coordinator implements INT16 (%d), INT32 (%d) and FLOAT32 (%d)", type,
              FFTLIB_INT16, FFTLIB_INT32, FFTLIB_FLOAT32);
    return FFTLIB_ERR_NOT_IMPLEMENTED;
}

MmaHandle* handle_of(FFTLIB_kernelHandle h)
{
    MmaHandle* m = static_cast<MmaHandle*>(h);
    if (!m || m->magic != kMmaMagic || m->path == PATH_NONE) {
        set_error("handle was not set up by the init of the coordinator or of one of its variants");
        return nullptr;
    }
    return m;
}

cudaError_t enqueue(const MmaHandle* m, const float* x, const float* w, float* y, uint32_t batch, cudaStream_t s)
{
    if (m->path == PATH_INT)
        return int_dft_launch_v(m->bits, variant_of(m), m->init.fftSize, batch, m->init.interleave,
                                m->init.shiftVector, const_cast<float*>(x), w, y, s);
    // the tensor-core kernels read and prefetch whole 16-byte lines; buffers
    // that are only 8-byte aligned take the FFT
    const bool aligned = (((uintptr_t)x | (uintptr_t)y) & 15u) == 0;
    if (m->path == PATH_TC && aligned)
        return launch_tc_dft(m->init.fftSize, reinterpret_cast<const float2*>(x), reinterpret_cast<float2*>(y), w,
                             batch, error_word().dev, s);
    // above 16384 points the FFT may use pX as scratch of its global passes,
    // as the fft1dBatched kernels do
    return run_c2c(m->plan, const_cast<float2*>(reinterpret_cast<const float2*>(x)), reinterpret_cast<float2*>(y),
                   batch, false, s);
}

// The caller's integer table of `elems` entries: host memory from the host
// generator; device memory from the device generator for the dense dftLarge
// matrix (4 n^2 entries), else from the host one and one copy.
FFTLIB_STATUS int_tw_gen(int bits, int variant, uint32_t n, uint32_t batch, uint32_t il, void* pW, uint32_t elems)
{
    if (!is_device_ptr(pW)) {
        int_dft_twgen_host_v(bits, variant, n, batch, il, pW);
        return FFTLIB_SUCCESS;
    }
    cudaError_t e;
    if (variant == INT_DFT_LARGE) {
        e = dft_large_matrix_device(pW, bits, n, il, cudaStreamPerThread);
        if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
        return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "twGen");
    }
    std::vector<unsigned char> tmp((size_t)elems * (bits / 8));
    int_dft_twgen_host_v(bits, variant, n, batch, il, tmp.data());
    e = cudaMemcpy(pW, tmp.data(), tmp.size(), cudaMemcpyHostToDevice);
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "twGen copy");
}

} // namespace

extern "C" {

int32_t FFTLIB_FFT_fft_ixX_cxX_oxX_getHandleSize(FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* pKerInitArgs)
{
    (void)pKerInitArgs;
    return (int32_t)sizeof(MmaHandle);
}

FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_getSizes(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* pKerInitArgs,
                                                  FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_bufParams1D_t* bufParamsW,
                                                  FFTLIB_bufParams1D_t* bufParamsY)
{
    if (!pKerInitArgs || !bufParamsX || !bufParamsW || !bufParamsY) return FFTLIB_ERR_NULL_POINTER;
    const int bits = int_bits(bufParamsX->data_type);
    if (!bits && bufParamsX->data_type != FFTLIB_FLOAT32) return unsupported_type(bufParamsX->data_type);
    uint32_t x, w, y;
    const FFTLIB_STATUS st = bits ? sizes_int(pKerInitArgs, bits, &x, &w, &y) : sizes_f32(pKerInitArgs, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    bufParamsX->dim_x = x;
    bufParamsW->dim_x = w;
    bufParamsY->dim_x = y;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_twGen(const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* pKerInitArgs, void* pW,
                                               const FFTLIB_bufParams1D_t* bufParamsW)
{
    if (!pKerInitArgs || !pW || !bufParamsW) return FFTLIB_ERR_NULL_POINTER;
    const int bits = int_bits(bufParamsW->data_type);
    if (bits) {
        const uint32_t n = pKerInitArgs->fftSize, b = pKerInitArgs->batchSize, il = pKerInitArgs->interleave;
        const uint32_t w = int_dft_w_size(bits, n, b, il);
        if (bufParamsW->dim_x != w) {
            set_error("bufParamsW->dim_x %u, expected %u", bufParamsW->dim_x, w);
            return FFTLIB_ERR_INVALID_DIMENSION;
        }
        return int_tw_gen(bits, int_dft_variant(bits, n, b, il), n, b, il, pW, w);
    }
    if (bufParamsW->data_type != FFTLIB_FLOAT32) return unsupported_type(bufParamsW->data_type);
    uint32_t x, w, y;
    FFTLIB_STATUS st = sizes_f32(pKerInitArgs, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    if (bufParamsW->dim_x != w) {
        set_error("bufParamsW->dim_x %u, expected %u", bufParamsW->dim_x, w);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const uint32_t n = pKerInitArgs->fftSize;
    float* out = static_cast<float*>(pW);
    const bool dev = is_device_ptr(pW);
    if (choose_path(pKerInitArgs) == PATH_TC) {
        if (!dev) {
            tc_dft_gen_w_host(out, n);
            return FFTLIB_SUCCESS;
        }
        cudaError_t e = tc_dft_gen_w_device(out, n, cudaStreamPerThread);
        if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
        return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "twGen");
    }
    if (!dev) {
        FFTLIB_b200_tw_gen_c2c(out, n);
        return FFTLIB_SUCCESS;
    }
    cudaError_t e = stage_twiddles_device(out, n, false, cudaStreamPerThread);
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamPerThread);
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "twGen");
}

FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_init_checkParams(FFTLIB_kernelHandle handle,
                                                          const FFTLIB_bufParams1D_t* bufParamsX,
                                                          const FFTLIB_bufParams1D_t* bufParamsW,
                                                          const FFTLIB_bufParams1D_t* bufParamsY,
                                                          const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* pKerInitArgs)
{
    if (!handle || !bufParamsX || !bufParamsW || !bufParamsY || !pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;
    const int bits = int_bits(bufParamsX->data_type);
    if (!bits && bufParamsX->data_type != FFTLIB_FLOAT32) return unsupported_type(bufParamsX->data_type);
    uint32_t x, w, y;
    const FFTLIB_STATUS st = bits ? sizes_int(pKerInitArgs, bits, &x, &w, &y) : sizes_f32(pKerInitArgs, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    const int variant = bits ? int_dft_variant(bits, pKerInitArgs->fftSize, pKerInitArgs->batchSize,
                                               pKerInitArgs->interleave)
                             : 0;
    // highRadix: at least 2 MMA points
    // (FFTLIB_FFT_highRadixDecompositions_ixX_cxX_oxX.cpp:41-43)
    if (variant == INT_HIGH_RADIX && pKerInitArgs->fftSize < 2u * (uint32_t)int_mma_size(bits))
        return FFTLIB_ERR_INVALID_VALUE;
    if (bufParamsX->dim_x != x || bufParamsY->dim_x != y || bufParamsW->dim_x != w) {
        set_error("dim_x X/W/Y = %u/%u/%u, expected %u/%u/%u", bufParamsX->dim_x, bufParamsW->dim_x,
                  bufParamsY->dim_x, x, w, y);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (bufParamsW->data_type != bufParamsX->data_type || bufParamsY->data_type != bufParamsX->data_type)
        return FFTLIB_ERR_INVALID_TYPE;
    // dftLarge runs the LINALG matrix multiply, whose check bounds the shift
    // by the accumulator width (FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.cpp:41-56)
    if (variant == INT_DFT_LARGE && (int8_t)pKerInitArgs->shiftVector[0] > (bits == 16 ? 64 : 128))
        return FFTLIB_ERR_INVALID_SHIFT;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_init(FFTLIB_kernelHandle handle, FFTLIB_bufParams1D_t* bufParamsX,
                                              FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_bufParams1D_t* bufParamsY,
                                              const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs* pKerInitArgs)
{
    if (!handle || !bufParamsX || !pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;
    (void)bufParamsW;
    (void)bufParamsY;
    MmaHandle* m = static_cast<MmaHandle*>(handle);
    memset(m, 0, sizeof(*m));
    const int bits = int_bits(bufParamsX->data_type);
    if (bits) {
        const uint32_t n = pKerInitArgs->fftSize;
        if (n == 0 || pKerInitArgs->batchSize == 0) return FFTLIB_ERR_INVALID_DIMENSION;
        if (int_dft_variant(bits, n, pKerInitArgs->batchSize, pKerInitArgs->interleave) == INT_HIGH_RADIX &&
            !int_high_radix_covered(bits, n)) {
            set_error("INT%d fftSize %u: the high-radix decomposition needs d0 x %u^L points, d0 <= %u, L <= 4",
                      bits, n, int_mma_size(bits) / 2, int_mma_size(bits) / 2);
            return FFTLIB_ERR_NOT_IMPLEMENTED;
        }
        int dev = 0;
        const cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
        m->init = *pKerInitArgs;
        m->device = dev;
        m->bits = bits;
        m->path = PATH_INT;
        m->magic = kMmaMagic;
        return FFTLIB_SUCCESS;
    }
    if (bufParamsX->data_type != FFTLIB_FLOAT32) return unsupported_type(bufParamsX->data_type);
    uint32_t x, w, y;
    const FFTLIB_STATUS st = sizes_f32(pKerInitArgs, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    m->init = *pKerInitArgs;
    m->device = dev;
    m->path = choose_path(pKerInitArgs);
    // the FFT plan also serves tensor-core handles called with buffers that
    // are not 16-byte aligned
    m->plan = get_complex_plan(pKerInitArgs->fftSize, false, &e);
    if (!m->plan) return cuda_fail(e, "plan creation");
    m->magic = kMmaMagic;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_exec_checkParams(FFTLIB_kernelHandle handle, const void* pX, const void* pW,
                                                          const void* pY)
{
    (void)handle;
    if (!pX || !pW || !pY) return FFTLIB_ERR_NULL_POINTER;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_FFT_fft_ixX_cxX_oxX_exec(FFTLIB_kernelHandle handle, void* pX, void* pW, void* pY)
{
    MmaHandle* m = handle_of(handle);
    if (!m) return FFTLIB_ERR_NULL_POINTER;
    if (!pX || !pW || !pY) return FFTLIB_ERR_NULL_POINTER;
    DeviceScope scope(m->device);
    const uint32_t n = m->init.fftSize;
    const void* w = pW;
    const size_t elem = m->path == PATH_INT ? (size_t)m->bits / 8u : sizeof(float);
    if (m->path == PATH_TC || m->path == PATH_INT) {
        const size_t wbytes = m->path == PATH_TC ? tc_dft_w_floats(n) * sizeof(float)
                                                 : (size_t)int_dft_w_size_v(m->bits, variant_of(m), n) * elem;
        cudaError_t e = device_table(pW, wbytes, 2, &w);
        if (e != cudaSuccess) return cuda_fail(e, "computational matrix copy");
    }
    if (m->path == PATH_INT && pX == pY && variant_of(m) == INT_HIGH_RADIX) {
        set_error("the high-radix path works in pX and needs pY != pX");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    const size_t bytes = (size_t)n * 2u * elem;
    std::vector<ChannelBuf> bufs = {{pX, bytes, true, false}, {pY, bytes, false, true}};
    cudaError_t e = run_channels(bufs, m->init.batchSize,
                                 [&](const std::vector<void*>& d, uint32_t, uint32_t cnt, cudaStream_t s) {
                                     return enqueue(m, (const float*)d[0], (const float*)w, (float*)d[1], cnt, s);
                                 });
    if (e != cudaSuccess) return cuda_fail(e, "FFT_fft_ixX_cxX_oxX_exec");
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_FFT_fft_execAsync(FFTLIB_kernelHandle handle, void* pX, void* pW, void* pY, void* stream)
{
    MmaHandle* m = handle_of(handle);
    if (!m) return FFTLIB_ERR_NULL_POINTER;
    if (!pX || !pW || !pY) return FFTLIB_ERR_NULL_POINTER;
    if (!is_device_ptr(pX) || !is_device_ptr(pY) || !is_device_ptr(pW)) {
        set_error("execAsync needs device buffers");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    if (m->path == PATH_INT && pX == pY && variant_of(m) == INT_HIGH_RADIX) {
        set_error("the high-radix path works in pX and needs pY != pX");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    DeviceScope scope(m->device);
    const cudaError_t e = enqueue(m, (const float*)pX, (const float*)pW, (float*)pY, m->init.batchSize,
                                  (cudaStream_t)stream);
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "FFT_fft execAsync");
}

FFTLIB_STATUS FFTLIB_b200_FFT_fft_sync(void* stream)
{
    cudaError_t e = cudaStreamSynchronize((cudaStream_t)stream);
    if (e == cudaSuccess && take_device_error()) e = cudaErrorLaunchTimeout;
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "FFT_fft sync");
}

int32_t FFTLIB_b200_FFT_fft_path(FFTLIB_kernelHandle handle)
{
    const MmaHandle* m = static_cast<const MmaHandle*>(handle);
    return (m && m->magic == kMmaMagic) ? m->path : PATH_NONE;
}

uint8_t FFTLIB_FFT_twData[32 * 32 * 3 * sizeof(int16_t)];

void FFTLIB_b200_FFT_setIntTensorCores(int32_t enable) { int_set_tensor_cores(enable != 0); }

} // extern "C"

// ---- the variants on their own (fft_c7xmma_variants.h) ----------------------------
//
// The same handle, tables and kernels as the coordinator, with the variant
// fixed by which init was called. The checks follow each variant's
// init_checkParams (src/fft_c7xmma/FFTLIB_FFT_dftSmall_ixX_cxX_oxX/
// FFTLIB_FFT_dftSmall_ixX_cxX_oxX.cpp:13-52, ..._dftLarge_ixX_cxX_oxX.cpp:13-75,
// ..._highRadixDecompositions_ixX_cxX_oxX.cpp:14-66) and getSizes
// (c71/..._ci.cpp: dftSmall 74-106, dftLarge 43-75, highRadix 1975-2025).
namespace {

template <class VArgs>
FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs coordinator_args(const VArgs* a)
{
    FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs c;
    memset(&c, 0, sizeof(c));
    c.funcStyle = a->funcStyle;
    c.fftSize = a->fftSize;
    c.batchSize = a->batchSize;
    c.interleave = a->interleave;
    for (size_t i = 0; i < sizeof(a->shiftVector) / sizeof(a->shiftVector[0]); ++i) c.shiftVector[i] = a->shiftVector[i];
    return c;
}

// getSizes of one variant: X, W and Y elements.
FFTLIB_STATUS variant_sizes(int variant, const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs& a, uint32_t type, uint32_t* x,
                            uint32_t* w, uint32_t* y)
{
    const int bits = int_bits(type);
    if (!bits) {
        set_error("data type %u: the DFT variants implement INT16 (%d) and INT32 (%d)", type, FFTLIB_INT16,
                  FFTLIB_INT32);
        return FFTLIB_ERR_NOT_IMPLEMENTED;
    }
    const uint32_t mma = (uint32_t)int_mma_size(bits), n = a.fftSize;
    if (variant == INT_DFT_SMALL && n > mma / 2) {
        set_error("dftSmall: fftSize %u above MMA/2 = %u", n, mma / 2);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (variant == INT_DFT_LARGE && n <= mma / 2) {
        set_error("dftLarge: fftSize %u not above MMA/2 = %u", n, mma / 2);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const uint64_t xy = 2ull * n * a.batchSize;
    if (xy > 0xFFFFFFFFull || (variant == INT_DFT_LARGE && 4ull * n * n > 0xFFFFFFFFull)) {
        set_error("fftSize %u x batchSize %u exceeds the 32-bit dim_x", n, a.batchSize);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    *x = *y = (uint32_t)xy;
    *w = int_dft_w_size_v(bits, variant, n);
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS variant_get_sizes(int variant, const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs& a,
                                FFTLIB_bufParams1D_t* bx, FFTLIB_bufParams1D_t* bw, FFTLIB_bufParams1D_t* by)
{
    if (!bx || !bw || !by) return FFTLIB_ERR_NULL_POINTER;
    uint32_t x, w, y;
    const FFTLIB_STATUS st = variant_sizes(variant, a, bx->data_type, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    bx->dim_x = x;
    bw->dim_x = w;
    by->dim_x = y;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS variant_tw_gen(int variant, const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs& a, void* pW,
                             const FFTLIB_bufParams1D_t* bw)
{
    if (!pW || !bw) return FFTLIB_ERR_NULL_POINTER;
    uint32_t x, w, y;
    const FFTLIB_STATUS st = variant_sizes(variant, a, bw->data_type, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    if (bw->dim_x != w) {
        set_error("bufParamsW->dim_x %u, expected %u", bw->dim_x, w);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    return int_tw_gen(int_bits(bw->data_type), variant, a.fftSize, a.batchSize, a.interleave, pW, w);
}

FFTLIB_STATUS variant_check(int variant, FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t* bx,
                            const FFTLIB_bufParams1D_t* bw, const FFTLIB_bufParams1D_t* by,
                            const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs& a)
{
    if (!handle) return FFTLIB_ERR_NULL_POINTER;
    if (!bx || !bw || !by) return FFTLIB_ERR_NULL_POINTER;
    uint32_t x, w, y;
    const FFTLIB_STATUS st = variant_sizes(variant, a, bx->data_type, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    const int bits = int_bits(bx->data_type);
    if (variant == INT_HIGH_RADIX && a.fftSize < 2u * (uint32_t)int_mma_size(bits)) {
        set_error("highRadix: fftSize %u below 2 MMA = %d", a.fftSize, 2 * int_mma_size(bits));
        return FFTLIB_ERR_INVALID_VALUE;
    }
    if (bx->dim_x != x || by->dim_x != y || bw->dim_x != w) {
        set_error("dim_x X/W/Y = %u/%u/%u, expected %u/%u/%u", bx->dim_x, bw->dim_x, by->dim_x, x, w, y);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (bw->data_type != bx->data_type || by->data_type != bx->data_type) return FFTLIB_ERR_INVALID_TYPE;
    // dftLarge: the LINALG multiply's own check (its shift is int8_t)
    if (variant == INT_DFT_LARGE && (int8_t)a.shiftVector[0] > (bits == 16 ? 64 : 128))
        return FFTLIB_ERR_INVALID_SHIFT;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS variant_init(int variant, FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t* bx,
                           const FFTLIB_FFT_fft_ixX_cxX_oxX_InitArgs& a)
{
    if (!handle || !bx) return FFTLIB_ERR_NULL_POINTER;
    MmaHandle* m = static_cast<MmaHandle*>(handle);
    memset(m, 0, sizeof(*m));
    uint32_t x, w, y;
    const FFTLIB_STATUS st = variant_sizes(variant, a, bx->data_type, &x, &w, &y);
    if (st != FFTLIB_SUCCESS) return st;
    const int bits = int_bits(bx->data_type);
    const uint32_t n = a.fftSize;
    if (n == 0 || a.batchSize == 0) return FFTLIB_ERR_INVALID_DIMENSION;
    if (variant == INT_HIGH_RADIX) {
        if (n < 2u * (uint32_t)int_mma_size(bits)) {
            set_error("highRadix: fftSize %u below 2 MMA = %d", n, 2 * int_mma_size(bits));
            return FFTLIB_ERR_INVALID_VALUE;
        }
        if (!int_high_radix_covered(bits, n)) {
            set_error("INT%d fftSize %u: the high-radix decomposition needs d0 x %u^L points, d0 <= %u, L <= 4",
                      bits, n, int_mma_size(bits) / 2, int_mma_size(bits) / 2);
            return FFTLIB_ERR_NOT_IMPLEMENTED;
        }
        // the reference's init leaves the internal table in FFTLIB_FFT_twData
        int_dft_w1_host(bits, n, FFTLIB_FFT_twData);
    }
    int dev = 0;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    m->init = a;
    m->device = dev;
    m->bits = bits;
    m->variant = variant;
    m->path = PATH_INT;
    m->magic = kMmaMagic;
    return FFTLIB_SUCCESS;
}

} // namespace

extern "C" {

#define FFTLIB_B200_DFT_VARIANT(NAME, VARIANT, INIT_CONST, EXEC_X_CONST, EXEC_W_CONST)                              \
    int32_t FFTLIB_FFT_##NAME##_getHandleSize(FFTLIB_FFT_##NAME##_InitArgs* pKerInitArgs)                            \
    {                                                                                                                \
        (void)pKerInitArgs;                                                                                          \
        return (int32_t)sizeof(MmaHandle);                                                                           \
    }                                                                                                                \
    FFTLIB_STATUS FFTLIB_FFT_##NAME##_getSizes(const FFTLIB_FFT_##NAME##_InitArgs* pKerInitArgs,                     \
                                               FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_bufParams1D_t* bufParamsW,    \
                                               FFTLIB_bufParams1D_t* bufParamsY)                                     \
    {                                                                                                                \
        if (!pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;                                                           \
        return variant_get_sizes(VARIANT, coordinator_args(pKerInitArgs), bufParamsX, bufParamsW, bufParamsY);      \
    }                                                                                                                \
    FFTLIB_STATUS FFTLIB_FFT_##NAME##_twGen(const FFTLIB_FFT_##NAME##_InitArgs* pKerInitArgs, void* pW,              \
                                            const FFTLIB_bufParams1D_t* bufParamsW)                                  \
    {                                                                                                                \
        if (!pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;                                                           \
        return variant_tw_gen(VARIANT, coordinator_args(pKerInitArgs), pW, bufParamsW);                              \
    }                                                                                                                \
    FFTLIB_STATUS FFTLIB_FFT_##NAME##_init_checkParams(                                                              \
        FFTLIB_kernelHandle handle, const FFTLIB_bufParams1D_t* bufParamsX, const FFTLIB_bufParams1D_t* bufParamsW,  \
        const FFTLIB_bufParams1D_t* bufParamsY, const FFTLIB_FFT_##NAME##_InitArgs* pKerInitArgs)                    \
    {                                                                                                                \
        if (!pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;                                                           \
        return variant_check(VARIANT, handle, bufParamsX, bufParamsW, bufParamsY, coordinator_args(pKerInitArgs));   \
    }                                                                                                                \
    FFTLIB_STATUS FFTLIB_FFT_##NAME##_init(FFTLIB_kernelHandle handle, INIT_CONST FFTLIB_bufParams1D_t* bufParamsX,  \
                                           INIT_CONST FFTLIB_bufParams1D_t* bufParamsW,                              \
                                           INIT_CONST FFTLIB_bufParams1D_t* bufParamsY,                              \
                                           INIT_CONST FFTLIB_FFT_##NAME##_InitArgs* pKerInitArgs)                    \
    {                                                                                                                \
        (void)bufParamsW;                                                                                            \
        (void)bufParamsY;                                                                                            \
        if (!pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;                                                           \
        return variant_init(VARIANT, handle, bufParamsX, coordinator_args(pKerInitArgs));                            \
    }                                                                                                                \
    FFTLIB_STATUS FFTLIB_FFT_##NAME##_exec_checkParams(FFTLIB_kernelHandle handle, const void* pX, const void* pW,   \
                                                       const void* pY)                                               \
    {                                                                                                                \
        (void)handle;                                                                                                \
        return (!pX || !pW || !pY) ? FFTLIB_ERR_NULL_POINTER : FFTLIB_SUCCESS;                                       \
    }                                                                                                                \
    FFTLIB_STATUS FFTLIB_FFT_##NAME##_exec(FFTLIB_kernelHandle handle, EXEC_X_CONST void* pX,                        \
                                           EXEC_W_CONST void* pW, void* pY)                                          \
    {                                                                                                                \
        const MmaHandle* m = handle_of(handle);                                                                      \
        if (!m) return FFTLIB_ERR_NULL_POINTER;                                                                      \
        if (m->variant != VARIANT) {                                                                                 \
            set_error("handle was set up for another DFT variant");                                                  \
            return FFTLIB_ERR_INVALID_VALUE;                                                                         \
        }                                                                                                            \
        return FFTLIB_FFT_fft_ixX_cxX_oxX_exec(handle, const_cast<void*>(pX), const_cast<void*>(pW), pY);            \
    }

FFTLIB_B200_DFT_VARIANT(dftSmall_ixX_cxX_oxX, INT_DFT_SMALL, , , )
FFTLIB_B200_DFT_VARIANT(dftLarge_ixX_cxX_oxX, INT_DFT_LARGE, const, const, const)
FFTLIB_B200_DFT_VARIANT(highRadixDecompositions_ixX_cxX_oxX, INT_HIGH_RADIX, , , )

#undef FFTLIB_B200_DFT_VARIANT

} // extern "C"
