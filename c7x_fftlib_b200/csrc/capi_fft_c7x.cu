// capi_fft_c7x.cu -- exported FFTLIB batched-kernel API (include/fftlib_b200/fft_c7x.h).
//
// Parameter checks reproduce the reference's status codes and their order:
//   c2c   _checkParams  src/fft_c7x/FFTLIB_fft1dBatched_i32fc_c32fc_o32fc/c7504/..._ci.cpp:2806-2855
//         _checkParams_cn                                   ..._cn.c:497-543
//   ifft  _checkParams  src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc/c7504/..._ci.cpp (checkParams)
//         _checkParams_cn                                   ..._cn.c (checkParams_cn)
//   r2c   _checkParams  src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/c71/..._ci.cpp:442-500
//         _checkParams_cn                                   ..._cn.c:127-175
//   c2r   _checkParams  src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/c71/..._ci.cpp (checkParams)
//         _checkParams_cn                                   ..._cn.c:93-136
//   int16 _checkParams  src/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/c7504/..._ci.cpp:793-835
//         _checkParams_cn                                   ..._cn.c:340-385
// The optimized checks are the reference's; _init and _kernel add the
// conditions this implementation needs to stay in bounds (numPoints that the
// c7504/c71 checks let through but the kernels cannot run, undersized shift
// vectors), reported with FFTLIB_ERR_INVALID_DIMENSION.
#include <string.h>

#include "capi_exec.h"
#include "fft_c7x.h"
#include "fft_i16.h"
#include "plan.h"

using namespace fftb200;

namespace {

bool has_235(uint32_t n) { return is_235(n); }

} // namespace

namespace fftb200 {

FFTLIB_STATUS write_record(void* pBlock, uint32_t kind, uint32_t n, uint32_t c, uint32_t mode, ComplexPlan* plan)
{
    PlanRecord r{};
    r.magic = kRecordMagic;
    r.kind = kind;
    r.numPoints = n;
    r.numChannels = c;
    r.mode = mode;
    cudaGetDevice(&r.device);
    r.plan = plan;
    memcpy(pBlock, &r, sizeof(r));
    return FFTLIB_SUCCESS;
}

// Validates the record left by _init for this call.
FFTLIB_STATUS read_record(void* pBlock, uint32_t kind, uint32_t n, PlanRecord* out)
{
    if (!pBlock) {
        set_error("pBlock is NULL");
        return FFTLIB_ERR_NULL_POINTER;
    }
    memcpy(out, pBlock, sizeof(*out));
    if (out->magic != kRecordMagic || out->kind != kind) {
        set_error("pBlock was not initialised by the matching _init");
        return FFTLIB_ERR_FAILURE;
    }
    if (out->numPoints != n) {
        set_error("numPoints %u differs from the %u given to _init", n, out->numPoints);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    return FFTLIB_SUCCESS;
}

} // namespace fftb200

namespace {

// ---- checks ---------------------------------------------------------------

FFTLIB_STATUS check_c2c(const void* pX, const FFTLIB_bufParams1D_t* bX, const void* pW,
                        const FFTLIB_bufParams1D_t* bW, const void* pY, const FFTLIB_bufParams1D_t* bY,
                        uint32_t n, const void* pBlock, bool optimized, bool inverse)
{
    if (!pX || !pW || !pY || (optimized && !pBlock)) return FFTLIB_ERR_NULL_POINTER;
    if (!bX || !bW || !bY) return FFTLIB_ERR_NULL_POINTER;
    if (bX->dim_x != bY->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bW->dim_x != n * 2u) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bX->data_type != FFTLIB_FLOAT32 || bW->data_type != FFTLIB_FLOAT32 || bY->data_type != FFTLIB_FLOAT32)
        return FFTLIB_ERR_INVALID_TYPE;
    if (optimized && ((uintptr_t)pX & 0xFu)) return FFTLIB_ERR_NOT_ALIGNED_PTRS_STRIDES;
    if (!has_235(n)) return (!optimized && inverse) ? FFTLIB_ERR_NOT_IMPLEMENTED : FFTLIB_ERR_INVALID_DIMENSION;
    return FFTLIB_SUCCESS;
}

// r2c and c2r share the check; the natural-C version also rejects odd dim_x
// (r2c) and has no alignment / outmode checks.
FFTLIB_STATUS check_real(const void* pX, const FFTLIB_bufParams1D_t* bX, const void* pW,
                         const FFTLIB_bufParams1D_t* bW, const void* pY, const FFTLIB_bufParams1D_t* bY,
                         uint32_t n, uint8_t mode, bool optimized, bool r2c)
{
    if (!pX || !pW || !pY) return FFTLIB_ERR_NULL_POINTER;
    if (!bX || !bW || !bY) return FFTLIB_ERR_NULL_POINTER;
    if (bX->dim_x != bW->dim_x || bX->dim_x != bY->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bX->data_type != FFTLIB_FLOAT32 || bW->data_type != FFTLIB_FLOAT32 || bY->data_type != FFTLIB_FLOAT32)
        return FFTLIB_ERR_INVALID_TYPE;
    if (optimized) {
        if ((uintptr_t)pX & 0xFu) return FFTLIB_ERR_NOT_ALIGNED_PTRS_STRIDES;
        if (r2c && mode != 0 && mode != 1) return FFTLIB_ERR_INVALID_OUTMODE;
    } else if (r2c && (bX->dim_x & 1u)) {
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (!has_235(n / 2u)) return FFTLIB_ERR_INVALID_DIMENSION;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS check_i16(const void* pX, const FFTLIB_bufParams1D_t* bX, const void* pW,
                        const FFTLIB_bufParams1D_t* bW, const void* pY, const FFTLIB_bufParams1D_t* bY,
                        const void* pShift, const FFTLIB_bufParams1D_t* bS, uint32_t n, uint32_t c,
                        const void* pBlock, bool optimized)
{
    if (!pX || !pW || !pY || !pShift || (optimized && !pBlock)) return FFTLIB_ERR_NULL_POINTER;
    if (optimized) return FFTLIB_SUCCESS; // the c7504 optimized check stops here
    if (!bX || !bW || !bY || !bS) return FFTLIB_ERR_NULL_POINTER;
    if (bX->dim_x != bY->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bX->dim_x < n * c * 2u) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bW->dim_x != n * 2u) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bX->data_type != FFTLIB_INT16 || bW->data_type != FFTLIB_INT16 || bY->data_type != FFTLIB_INT16)
        return FFTLIB_ERR_INVALID_TYPE;
    if (bS->data_type != FFTLIB_UINT32) return FFTLIB_ERR_INVALID_TYPE;
    const uint32_t p4 = (1u << ((bS->dim_x * 2u) & 31u)) * 2u;
    if (p4 != bW->dim_x && p4 * 2u != bW->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    return FFTLIB_SUCCESS;
}

} // namespace

namespace fftb200 {

// ---- execution ----------------------------------------------------------------

FFTLIB_STATUS exec_c2c(float* pX, float* pY, uint32_t n, uint32_t c, bool inverse, ComplexPlan* plan)
{
    if (!plan) {
        cudaError_t e;
        plan = get_complex_plan(n, false, &e);
        if (!plan) return cuda_fail(e, "plan creation");
    }
    DeviceScope scope(plan->device);
    const size_t bytes = (size_t)n * 2u * sizeof(float);
    std::vector<ChannelBuf> bufs = {{pX, bytes, true, false}, {pY, bytes, false, true}};
    cudaError_t e = run_channels(bufs, c, [&](const std::vector<void*>& d, uint32_t, uint32_t cnt, cudaStream_t s) {
        return run_c2c(plan, (float2*)d[0], (float2*)d[1], cnt, inverse, s);
    });
    if (e != cudaSuccess) return cuda_fail(e, inverse ? "ifft1dBatched c2c" : "fft1dBatched c2c");
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS exec_r2c(float* pX, float* pXFFT, float* pY, uint32_t n, uint32_t c, int outmode, ComplexPlan* plan)
{
    if (n & 1u) {
        set_error("numPoints %u is odd", n);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const uint32_t h = n / 2u;
    if (!plan || !plan->twSplit) {
        cudaError_t e;
        plan = get_complex_plan(h, true, &e);
        if (!plan) return cuda_fail(e, "plan creation");
    }
    DeviceScope scope(plan->device);
    if (plan->multiPass && !pXFFT) {
        set_error("pXFFT work buffer required for numPoints %u", n);
        return FFTLIB_ERR_NULL_POINTER;
    }
    const size_t nOut = outmode ? n : h + 1u;
    std::vector<ChannelBuf> bufs = {{pX, (size_t)n * sizeof(float), true, false},
                                    {plan->multiPass ? pXFFT : nullptr, (size_t)h * sizeof(float2), false, false},
                                    {pY, nOut * sizeof(float2), false, true}};
    cudaError_t e = run_channels(bufs, c, [&](const std::vector<void*>& d, uint32_t, uint32_t cnt, cudaStream_t s) {
        return run_r2c(plan, (float*)d[0], (float2*)d[1], (float2*)d[2], cnt, outmode, s);
    });
    if (e != cudaSuccess) return cuda_fail(e, "fft1dBatched r2c");
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS exec_c2r(float* pX, float* pXFFT, float* pY, uint32_t n, uint32_t c, int inmode, ComplexPlan* plan)
{
    if (n & 1u) {
        set_error("numPoints %u is odd", n);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const uint32_t h = n / 2u;
    if (!plan || !plan->twSplit) {
        cudaError_t e;
        plan = get_complex_plan(h, true, &e);
        if (!plan) return cuda_fail(e, "plan creation");
    }
    DeviceScope scope(plan->device);
    const bool scratch = c2r_needs_scratch(plan, inmode);
    if (scratch && !pXFFT) {
        set_error("pXFFT work buffer required for numPoints %u", n);
        return FFTLIB_ERR_NULL_POINTER;
    }
    const size_t nIn = inmode ? n : h + 1u;
    std::vector<ChannelBuf> bufs = {{pX, nIn * sizeof(float2), true, false},
                                    {scratch ? pXFFT : nullptr, (size_t)h * sizeof(float2), false, false},
                                    {pY, (size_t)n * sizeof(float), false, true}};
    cudaError_t e = run_channels(bufs, c, [&](const std::vector<void*>& d, uint32_t, uint32_t cnt, cudaStream_t s) {
        return run_c2r(plan, (const float2*)d[0], (float2*)d[1], (float*)d[2], cnt, inmode, s);
    });
    if (e != cudaSuccess) return cuda_fail(e, "ifft1dBatched c2r");
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS exec_i16(int16_t* pX, const int16_t* pW, int16_t* pY, const uint32_t* pShift, uint32_t numShifts,
                       uint32_t n, uint32_t c, uint32_t tg, uint32_t gridCap, uint32_t minBlocks)
{
    if (n == 0 || (n & (n - 1u)) || n > 16384u) {
        set_error("int16 numPoints %u must be a power of two <= 16384", n);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (numShifts < i16_num_shifts(n)) {
        set_error("shift vector has %u entries, numPoints %u needs %u", numShifts, n, i16_num_shifts(n));
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    const void* dW = nullptr;
    const void* dS = pShift; // not read on the device when no radix-4 stage runs (n <= 2)
    cudaError_t e = device_table(pW, (size_t)n * 2u * sizeof(int16_t), 0, &dW);
    if (e == cudaSuccess && i16_num_shifts(n) > 0)
        e = device_table(pShift, (size_t)i16_num_shifts(n) * sizeof(uint32_t), 1, &dS);
    if (e != cudaSuccess) return cuda_fail(e, "int16 table upload");
    const size_t bytes = (size_t)n * 2u * sizeof(int16_t);
    std::vector<ChannelBuf> bufs = {{pX, bytes, true, false}, {pY, bytes, false, true}};
    e = run_channels(bufs, c, [&](const std::vector<void*>& d, uint32_t, uint32_t cnt, cudaStream_t s) {
        return launch_fft_i16((const int16_t*)d[0], (int16_t*)d[1], (const int16_t*)dW, (const uint32_t*)dS, n, cnt, s,
                              tg, gridCap, minBlocks);
    });
    if (e != cudaSuccess) return cuda_fail(e, "fft1dBatched int16");
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS init_fp32(void* pBlock, uint32_t kind, uint32_t n, uint32_t c, uint32_t mode, bool real)
{
    if (real && (n & 1u)) {
        set_error("numPoints %u is odd", n);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    cudaError_t e;
    const uint32_t len = real ? n / 2u : n;
    // the batched kinds take the autotuner's choice when it is enabled
    ComplexPlan* plan;
    switch (kind) {
    case REC_C2C: plan = get_batched_plan(len, real, TUNE_C2C, 0, c, &e); break;
    case REC_IFFT: plan = get_batched_plan(len, real, TUNE_IFFT, 0, c, &e); break;
    case REC_R2C: plan = get_batched_plan(len, real, TUNE_R2C, (int)mode, c, &e); break;
    case REC_C2R: plan = get_batched_plan(len, real, TUNE_C2R, (int)mode, c, &e); break;
    default: plan = get_complex_plan(len, real, &e); break;
    }
    if (!plan) return cuda_fail(e, "plan creation");
    return write_record(pBlock, kind, n, c, mode, plan);
}

} // namespace fftb200

extern "C" {

// ---- c2c forward -------------------------------------------------------------

FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                uint32_t numPoints, uint32_t numChannels,
                                                                void* pBlock)
{
    FFTLIB_STATUS st = check_c2c(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, pBlock, true, false);
    if (st == FFTLIB_SUCCESS && bufParamsX->dim_x < numPoints * numChannels * 2u) st = FFTLIB_ERR_INVALID_DIMENSION;
    return st;
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                   FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                   FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                   uint32_t numPoints, uint32_t numChannels)
{
    (void)numChannels;
    return check_c2c(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, nullptr, false, false);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                         FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                         FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                         uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    FFTLIB_STATUS st = FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY,
                                                                         numPoints, numChannels, pBlock);
    if (st != FFTLIB_SUCCESS) return st;
    return init_fp32(pBlock, REC_C2C, numPoints, numChannels, 0, false);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                           FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                           FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                           uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    (void)bufParamsX; (void)pW; (void)bufParamsW; (void)bufParamsY;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, REC_C2C, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, numPoints, numChannels, false, r.plan);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                       FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                       FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                       uint32_t numPoints, uint32_t numChannels)
{
    FFTLIB_STATUS st = FFTLIB_fft1dBatched_i32fc_c32fc_o32fc_checkParams_cn(pX, bufParamsX, pW, bufParamsW, pY,
                                                                            bufParamsY, numPoints, numChannels);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, numPoints, numChannels, false, nullptr);
}

// ---- c2c inverse -------------------------------------------------------------

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                 FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                 FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                 uint32_t numPoints, uint32_t numChannels,
                                                                 void* pBlock)
{
    FFTLIB_STATUS st = check_c2c(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, pBlock, true, true);
    if (st == FFTLIB_SUCCESS && bufParamsX->dim_x < numPoints * numChannels * 2u) st = FFTLIB_ERR_INVALID_DIMENSION;
    return st;
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                    FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                    FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                    uint32_t numPoints, uint32_t numChannels)
{
    (void)numChannels;
    return check_c2c(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, nullptr, false, true);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                          FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                          FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                          uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    FFTLIB_STATUS st = FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams(pX, bufParamsX, pW, bufParamsW, pY,
                                                                          bufParamsY, numPoints, numChannels, pBlock);
    if (st != FFTLIB_SUCCESS) return st;
    return init_fp32(pBlock, REC_IFFT, numPoints, numChannels, 0, false);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                            FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                            FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                            uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    (void)bufParamsX; (void)pW; (void)bufParamsW; (void)bufParamsY;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, REC_IFFT, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, numPoints, numChannels, true, r.plan);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                        FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                        FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                        uint32_t numPoints, uint32_t numChannels)
{
    FFTLIB_STATUS st = FFTLIB_ifft1dBatched_i32fc_c32fc_o32fc_checkParams_cn(pX, bufParamsX, pW, bufParamsW, pY,
                                                                             bufParamsY, numPoints, numChannels);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, numPoints, numChannels, true, nullptr);
}

// ---- r2c ---------------------------------------------------------------------

FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                               FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                               FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                               uint32_t numPoints, uint32_t numChannels,
                                                               uint8_t outmode, void* pBlock)
{
    (void)numChannels; (void)pBlock;
    return check_real(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, outmode, true, true);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                  FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                  FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                  uint32_t numPoints, uint32_t numChannels,
                                                                  uint8_t outmode)
{
    (void)numChannels;
    return check_real(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, outmode, false, true);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                        FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                        FFTLIB_F32* pXFFT, FFTLIB_bufParams1D_t* bufParamsXFFT,
                                                        FFTLIB_F32* pSf, FFTLIB_bufParams1D_t* bufParamsSf,
                                                        FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                        uint32_t numPoints, uint32_t numChannels, uint8_t outmode,
                                                        void* pBlock)
{
    (void)pXFFT; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = FFTLIB_fft1dBatched_i32f_c32fc_o32fc_checkParams(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY,
                                                                        numPoints, numChannels, outmode, pBlock);
    if (st != FFTLIB_SUCCESS) return st;
    if (!pBlock) return FFTLIB_ERR_NULL_POINTER;
    return init_fp32(pBlock, REC_R2C, numPoints, numChannels, outmode, true);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                          FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                          FFTLIB_F32* pXFFT, FFTLIB_bufParams1D_t* bufParamsXFFT,
                                                          FFTLIB_F32* pSf, FFTLIB_bufParams1D_t* bufParamsSf,
                                                          FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                          uint32_t numPoints, uint32_t numChannels, uint8_t outmode,
                                                          void* pBlock)
{
    (void)bufParamsX; (void)pW; (void)bufParamsW; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    (void)bufParamsY;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, REC_R2C, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    if (outmode != 0 && outmode != 1) return FFTLIB_ERR_INVALID_OUTMODE;
    return exec_r2c(pX, pXFFT, pY, numPoints, numChannels, outmode, r.plan);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i32f_c32fc_o32fc_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                      FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                      FFTLIB_F32* pXFFT, FFTLIB_bufParams1D_t* bufParamsXFFT,
                                                      FFTLIB_F32* pSf, FFTLIB_bufParams1D_t* bufParamsSf,
                                                      FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                      uint32_t numPoints, uint32_t numChannels, uint8_t outmode)
{
    (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = FFTLIB_fft1dBatched_i32f_c32fc_o32fc_checkParams_cn(pX, bufParamsX, pW, bufParamsW, pY,
                                                                           bufParamsY, numPoints, numChannels, outmode);
    if (st != FFTLIB_SUCCESS) return st;
    // the natural-C kernel treats any outmode other than 1 as the half spectrum
    return exec_r2c(pX, pXFFT, pY, numPoints, numChannels, outmode == 1 ? 1 : 0, nullptr);
}

// ---- c2r ---------------------------------------------------------------------

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                uint32_t numPoints, uint32_t numChannels,
                                                                uint8_t inMode, void* pBlock)
{
    (void)numChannels; (void)pBlock;
    return check_real(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, inMode, true, false);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                   FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                   FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                   uint32_t numPoints, uint32_t numChannels,
                                                                   uint8_t inMode)
{
    (void)numChannels;
    return check_real(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, numPoints, inMode, false, false);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                         FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                         FFTLIB_F32* pXFFT, FFTLIB_bufParams1D_t* bufParamsXFFT,
                                                         FFTLIB_F32* pSf, FFTLIB_bufParams1D_t* bufParamsSf,
                                                         FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                         uint32_t numPoints, uint32_t numChannels, uint8_t inMode,
                                                         void* pBlock)
{
    (void)pXFFT; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_checkParams(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY,
                                                                         numPoints, numChannels, inMode, pBlock);
    if (st != FFTLIB_SUCCESS) return st;
    if (!pBlock) return FFTLIB_ERR_NULL_POINTER;
    return init_fp32(pBlock, REC_C2R, numPoints, numChannels, inMode, true);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                           FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                           FFTLIB_F32* pXFFT, FFTLIB_bufParams1D_t* bufParamsXFFT,
                                                           FFTLIB_F32* pSf, FFTLIB_bufParams1D_t* bufParamsSf,
                                                           FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                           uint32_t numPoints, uint32_t numChannels, uint8_t inMode,
                                                           void* pBlock)
{
    (void)bufParamsX; (void)pW; (void)bufParamsW; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    (void)bufParamsY;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, REC_C2R, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    // the reference treats any inMode other than 0 as the full spectrum
    return exec_c2r(pX, pXFFT, pY, numPoints, numChannels, inMode ? 1 : 0, r.plan);
}

FFTLIB_STATUS FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                       FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                       FFTLIB_F32* pXFFT, FFTLIB_bufParams1D_t* bufParamsXFFT,
                                                       FFTLIB_F32* pSf, FFTLIB_bufParams1D_t* bufParamsSf,
                                                       FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                       uint32_t numPoints, uint32_t numChannels, uint8_t inMode)
{
    (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = FFTLIB_ifft1dBatched_i32fc_c32fc_o32f_checkParams_cn(pX, bufParamsX, pW, bufParamsW, pY,
                                                                            bufParamsY, numPoints, numChannels, inMode);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2r(pX, pXFFT, pY, numPoints, numChannels, inMode ? 1 : 0, nullptr);
}

// ---- int16 -------------------------------------------------------------------

FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                int16_t* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                int16_t* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                uint32_t* pShift, FFTLIB_bufParams1D_t* bufParamsShift,
                                                                uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    return check_i16(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, numPoints, numChannels,
                     pBlock, true);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams_cn(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                                   int16_t* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                                   int16_t* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                                   uint32_t* pShift,
                                                                   FFTLIB_bufParams1D_t* bufParamsShift,
                                                                   uint32_t numPoints, uint32_t numChannels)
{
    return check_i16(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, numPoints, numChannels,
                     nullptr, false);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_init(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                         int16_t* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                         int16_t* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                         uint32_t* pShift, FFTLIB_bufParams1D_t* bufParamsShift,
                                                         uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    FFTLIB_STATUS st = FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams(
        pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, numPoints, numChannels, pBlock);
    if (st != FFTLIB_SUCCESS) return st;
    if (numPoints == 0 || (numPoints & (numPoints - 1u)) || numPoints > 16384u) {
        set_error("int16 numPoints %u must be a power of two <= 16384", numPoints);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    st = write_record(pBlock, REC_I16, numPoints, numChannels, 0, nullptr);
    I16Choice ch{};
    if (st == FFTLIB_SUCCESS && autotune_enabled() && tune_i16(numPoints, numChannels, &ch)) {
        PlanRecord r;
        memcpy(&r, pBlock, sizeof(r));
        r.i16Tg = ch.tg;
        r.i16GridCap = ch.gridCap;
        r.i16MinBlocks = ch.minBlocks;
        r.i16Tuned = 1u;
        memcpy(pBlock, &r, sizeof(r));
    }
    return st;
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_kernel(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                           int16_t* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                           int16_t* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                           uint32_t* pShift, FFTLIB_bufParams1D_t* bufParamsShift,
                                                           uint32_t numPoints, uint32_t numChannels, void* pBlock)
{
    (void)bufParamsX; (void)bufParamsW; (void)bufParamsY;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, REC_I16, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    if (!pX || !pW || !pY || !pShift || !bufParamsShift) return FFTLIB_ERR_NULL_POINTER;
    DeviceScope scope(r.device);
    return exec_i16(pX, pW, pY, pShift, bufParamsShift->dim_x, numPoints, numChannels, r.i16Tg, r.i16GridCap,
                    r.i16MinBlocks ? r.i16MinBlocks : 3u);
}

FFTLIB_STATUS FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_cn(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                       int16_t* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                       int16_t* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                       uint32_t* pShift, FFTLIB_bufParams1D_t* bufParamsShift,
                                                       uint32_t numPoints, uint32_t numChannels)
{
    FFTLIB_STATUS st = FFTLIB_fft1dBatched_i16sc_c16sc_o16sc_checkParams_cn(
        pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, numPoints, numChannels);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_i16(pX, pW, pY, pShift, bufParamsShift->dim_x, numPoints, numChannels);
}

} // extern "C"
