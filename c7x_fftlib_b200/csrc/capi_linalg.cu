// capi_linalg.cu -- FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_*: the
// integer matrix multiply of the reference's src/linalg_c7xmma/
// FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX/
// FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX.cpp:7-152, computed by the
// tiled integer GEMM of dft_int.cu (bit-exact with ..._cn.cpp:27-62).
#include <string.h>

#include "capi_common.h"
#include "dft_int.h"
#include "linalg_c7xmma.h"

using namespace fftb200;

namespace {

constexpr uint32_t kLinalgMagic = 0x4C474C41u;  // "ALGL"

struct LinalgHandle {
    uint32_t magic;
    int32_t device;
    int32_t bits;                // 8, 16 or 32
    uint32_t M, K, N;
    size_t lda, ldb, ldc;        // row strides in elements
    uint32_t shift;              // InitArgs.shift as the reference's uint8_t shiftAndRound parameter
    FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs init;
};

int type_bits(uint32_t type)
{
    return type == FFTLIB_INT8 ? 8 : (type == FFTLIB_INT16 ? 16 : (type == FFTLIB_INT32 ? 32 : 0));
}

LinalgHandle* handle_of(FFTLIB_kernelHandle h)
{
    LinalgHandle* m = static_cast<LinalgHandle*>(h);
    if (!m || m->magic != kLinalgMagic) {
        set_error("handle was not set up by FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_init");
        return nullptr;
    }
    return m;
}

// A matrix argument of exec: the device pointer the kernel reads or writes,
// staged through device memory when the caller's buffer is host memory.
struct Operand {
    const void* user;
    void* dev = nullptr;   // temporary device copy (host operands)
    size_t ld = 0;         // row stride the kernel uses, in elements
};

// Host rows of `rows` x `cols` elements with stride `ld` into a dense device
// buffer (row stride cols), or the whole strided extent when rows overlap.
cudaError_t stage_in(Operand& o, uint32_t rows, uint32_t cols, size_t ld, size_t es, cudaStream_t s)
{
    if (rows == 0 || cols == 0) {
        o.ld = ld;
        return cudaSuccess;
    }
    const bool dense = ld >= cols;
    const size_t bytes = dense ? (size_t)rows * cols * es : ((size_t)(rows - 1) * ld + cols) * es;
    cudaError_t e = cudaMallocAsync(&o.dev, bytes, s);
    if (e != cudaSuccess) return e;
    if (!dense) {
        o.ld = ld;
        return cudaMemcpyAsync(o.dev, o.user, bytes, cudaMemcpyHostToDevice, s);
    }
    o.ld = cols;
    return cudaMemcpy2DAsync(o.dev, cols * es, o.user, ld * es, cols * es, rows, cudaMemcpyHostToDevice, s);
}

cudaError_t enqueue(const LinalgHandle* m, const void* a, size_t lda, const void* b, size_t ldb, void* c, size_t ldc,
                    cudaStream_t s)
{
    return int_matmul_launch(m->bits, m->M, m->K, m->N, a, lda, b, ldb, c, ldc, m->shift, s);
}

} // namespace

extern "C" {

int32_t FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_getHandleSize(
    FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs* pKerInitArgs)
{
    (void)pKerInitArgs;
    return (int32_t)sizeof(LinalgHandle);
}

FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_init_checkParams(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams2D_t* src0_addr, const FFTLIB_bufParams2D_t* src1_addr,
    const FFTLIB_bufParams2D_t* dst_addr, const FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs* pKerInitArgs)
{
    if (!handle) return FFTLIB_ERR_NULL_POINTER;
    if (!src0_addr || !src1_addr || !dst_addr || !pKerInitArgs) return FFTLIB_ERR_NULL_POINTER;
    // A is m x k, B is k x n, C is m x n
    if (src0_addr->dim_x != src1_addr->dim_y || src0_addr->dim_y != dst_addr->dim_y ||
        src1_addr->dim_x != dst_addr->dim_x) {
        set_error("dimensions: A %u x %u, B %u x %u, C %u x %u (rows x columns)", src0_addr->dim_y, src0_addr->dim_x,
                  src1_addr->dim_y, src1_addr->dim_x, dst_addr->dim_y, dst_addr->dim_x);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const int bits = type_bits(src0_addr->data_type);
    if (!bits) return FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_INPUT_TYPE;
    if (src1_addr->data_type != src0_addr->data_type || dst_addr->data_type != src0_addr->data_type)
        return FFTLIB_ERR_MATRIX_MATRIX_MULTIPLY_UNSUPPORTED_TYPE_COMBINATION;
    // the accumulator width: 32, 64 and 128 bits for INT8, INT16 and INT32
    if (pKerInitArgs->shift > 4 * bits) return FFTLIB_ERR_INVALID_SHIFT;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_init(
    FFTLIB_kernelHandle handle, const FFTLIB_bufParams2D_t* src0_addr, const FFTLIB_bufParams2D_t* src1_addr,
    const FFTLIB_bufParams2D_t* dst_addr, const FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_InitArgs* pKerInitArgs)
{
    const FFTLIB_STATUS st = FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_init_checkParams(
        handle, src0_addr, src1_addr, dst_addr, pKerInitArgs);
    if (st != FFTLIB_SUCCESS) return st;
    LinalgHandle* m = static_cast<LinalgHandle*>(handle);
    memset(m, 0, sizeof(*m));
    const int bits = type_bits(dst_addr->data_type);
    const int32_t es = bits / 8;
    if (src0_addr->stride_y < 0 || src1_addr->stride_y < 0 || dst_addr->stride_y < 0) {
        set_error("negative row strides are not supported");
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    m->M = src0_addr->dim_y;
    m->K = src0_addr->dim_x;
    m->N = src1_addr->dim_x;
    // element strides as the reference's init computes them (..._oxX.cpp:100-102)
    m->lda = (size_t)(src0_addr->stride_y / es);
    m->ldb = (size_t)(src1_addr->stride_y / es);
    m->ldc = (size_t)(dst_addr->stride_y / es);
    if (m->M > 1 && m->ldc < m->N) {
        set_error("dst stride %d bytes makes rows of C overlap (%u columns)", dst_addr->stride_y, m->N);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if ((m->M + 63ull) / 64ull > 0x7FFFFFFFull || (m->N + 63ull) / 64ull > 65535ull) {
        set_error("C of %u x %u exceeds the launch grid", m->M, m->N);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    int dev = 0;
    const cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    m->device = dev;
    m->bits = bits;
    m->shift = (uint32_t)(uint8_t)pKerInitArgs->shift;
    m->init = *pKerInitArgs;
    m->magic = kLinalgMagic;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec_checkParams(FFTLIB_kernelHandle handle,
                                                                              const void* src0, const void* src1,
                                                                              const void* dst)
{
    (void)handle;
    return (!src0 || !src1 || !dst) ? FFTLIB_ERR_NULL_POINTER : FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_LINALG_matrixMatrixMultiply_ixX_ixX_oxX_exec(FFTLIB_kernelHandle handle, const void* src0,
                                                                  const void* src1, void* dst)
{
    const LinalgHandle* m = handle_of(handle);
    if (!m) return FFTLIB_ERR_NULL_POINTER;
    if (!src0 || !src1 || !dst) return FFTLIB_ERR_NULL_POINTER;
    DeviceScope scope(m->device);
    const size_t es = (size_t)m->bits / 8u;
    cudaStream_t s = cudaStreamPerThread;
    Operand a{src0}, b{src1};
    cudaError_t e = cudaSuccess;
    if (is_device_ptr(src0)) a.ld = m->lda;
    else e = stage_in(a, m->M, m->K, m->lda, es, s);
    if (e == cudaSuccess) {
        if (is_device_ptr(src1)) b.ld = m->ldb;
        else e = stage_in(b, m->K, m->N, m->ldb, es, s);
    }
    const bool c_dev = is_device_ptr(dst);
    void* c = dst;
    size_t ldc = m->ldc;
    if (e == cudaSuccess && !c_dev && m->M && m->N) {
        e = cudaMallocAsync(&c, (size_t)m->M * m->N * es, s);
        ldc = m->N;
    }
    if (e == cudaSuccess)
        e = enqueue(m, a.dev ? a.dev : a.user, a.ld, b.dev ? b.dev : b.user, b.ld, c, ldc, s);
    if (e == cudaSuccess && !c_dev && m->M && m->N) {
        // only the M x N elements: the gaps between the caller's rows stay as they were
        e = m->M == 1 ? cudaMemcpyAsync(dst, c, m->N * es, cudaMemcpyDeviceToHost, s)
                      : cudaMemcpy2DAsync(dst, m->ldc * es, c, m->N * es, m->N * es, m->M, cudaMemcpyDeviceToHost, s);
    }
    if (!c_dev && c != dst && c) cudaFreeAsync(c, s);
    if (a.dev) cudaFreeAsync(a.dev, s);
    if (b.dev) cudaFreeAsync(b.dev, s);
    const cudaError_t f = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = f;
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "LINALG_matrixMatrixMultiply exec");
}

FFTLIB_STATUS FFTLIB_b200_LINALG_matrixMatrixMultiply_execAsync(FFTLIB_kernelHandle handle, const void* src0,
                                                                const void* src1, void* dst, void* stream)
{
    const LinalgHandle* m = handle_of(handle);
    if (!m) return FFTLIB_ERR_NULL_POINTER;
    if (!src0 || !src1 || !dst) return FFTLIB_ERR_NULL_POINTER;
    if (!is_device_ptr(src0) || !is_device_ptr(src1) || !is_device_ptr(dst)) {
        set_error("execAsync needs device buffers");
        return FFTLIB_ERR_INVALID_VALUE;
    }
    DeviceScope scope(m->device);
    const cudaError_t e = enqueue(m, src0, m->lda, src1, m->ldb, dst, m->ldc, (cudaStream_t)stream);
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, "LINALG_matrixMatrixMultiply execAsync");
}

} // extern "C"
