// capi_fft1d.cu -- exported FFTLIB single-transform API
// (include/fftlib_b200/fft1d_c7x.h).
//
// Each kernel is the batched transform with one channel (the reference's own
// natural-C r2c and c2r call the batched / single c2c code the same way:
// FFTLIB_fft1d_i32f_c32fc_o32fc_cn.c:34, FFTLIB_ifft1d_i32fc_c32fc_o32f_cn.c:74), so the
// work goes through the batched execution helpers; what is specific here is
// the length taken from bufParamsX->dim_x and the parameter checks, which
// reproduce the reference's status codes and their order:
//   c2c   _checkParams  src/fft_c7x/FFTLIB_fft1d_i32fc_c32fc_o32fc/c7504/..._ci.cpp:2279-2323
//         _checkParams_cn                                   ..._cn.c:491-532
//   ifft  _checkParams  src/fft_c7x/FFTLIB_ifft1d_i32fc_c32fc_o32fc/c7504/..._ci.cpp:2381-2425
//         _checkParams_cn                                   ..._cn.c:506-547
//   r2c   _checkParams  src/fft_c7x/FFTLIB_fft1d_i32f_c32fc_o32fc/c71/..._ci.cpp:277-322
//         _checkParams_cn                                   ..._cn.c:150-197
//   c2r   _checkParams  src/fft_c7x/FFTLIB_ifft1d_i32fc_c32fc_o32f/c71/..._ci.cpp:166-210
//         _checkParams_cn                                   ..._cn.c:80-120
//   int16 _checkParams  src/fft_c7x/FFTLIB_fft1d_i16sc_c16sc_o16sc/c7504/..._ci.cpp:659-699
//         _checkParams_cn                                   ..._cn.c:310-343
// The optimized FP32 checks do not test pBlock; _init answers
// FFTLIB_ERR_NULL_POINTER for a NULL pBlock after them. _init and _kernel add
// the conditions this implementation needs to stay in bounds (an odd real
// length that the c71 checks let through), reported with
// FFTLIB_ERR_INVALID_DIMENSION.
#include <string.h>

#include "capi_exec.h"
#include "fft1d_c7x.h"
#include "plan.h"

using namespace fftb200;

namespace {

enum Family { FAM_C2C, FAM_REAL_FWD, FAM_REAL_INV };

// FP32 checks; `optimized` selects the c7504/c71 variant (alignment of pX)
// over the natural-C one (odd length, r2c only).
FFTLIB_STATUS check_f32(const void* pX, const FFTLIB_bufParams1D_t* bX, const void* pW,
                        const FFTLIB_bufParams1D_t* bW, const void* pY, const FFTLIB_bufParams1D_t* bY,
                        bool optimized, Family fam)
{
    if (!pX || !pW || !pY) return FFTLIB_ERR_NULL_POINTER;
    if (!bX || !bW || !bY) return FFTLIB_ERR_NULL_POINTER;
    if (bX->dim_x != bW->dim_x || bX->dim_x != bY->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    if (bX->data_type != FFTLIB_FLOAT32 || bW->data_type != FFTLIB_FLOAT32 || bY->data_type != FFTLIB_FLOAT32)
        return FFTLIB_ERR_INVALID_TYPE;
    if (optimized) {
        if ((uintptr_t)pX & 0xFu) return FFTLIB_ERR_NOT_ALIGNED_PTRS_STRIDES;
    } else if (fam == FAM_REAL_FWD && (bX->dim_x & 1u)) {
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    if (!is_235(bX->dim_x / 2u)) return FFTLIB_ERR_INVALID_DIMENSION;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS check_i16(const void* pX, const FFTLIB_bufParams1D_t* bX, const void* pW,
                        const FFTLIB_bufParams1D_t* bW, const void* pY, const FFTLIB_bufParams1D_t* bY,
                        const void* pShift, const FFTLIB_bufParams1D_t* bS, const void* pBlock, bool optimized)
{
    if (!pX || !pW || !pY || !pShift || (optimized && !pBlock)) return FFTLIB_ERR_NULL_POINTER;
    if (!bX || !bW || !bY || !bS) return FFTLIB_ERR_NULL_POINTER;
    if (bX->dim_x != bW->dim_x || bX->dim_x != bY->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    if (optimized && bX->dim_x < 64u * 2u) return FFTLIB_ERR_INVALID_DIMENSION;  // at least 64 points
    if (bX->data_type != FFTLIB_INT16 || bW->data_type != FFTLIB_INT16 || bY->data_type != FFTLIB_INT16)
        return FFTLIB_ERR_INVALID_TYPE;
    if (bS->data_type != FFTLIB_UINT32) return FFTLIB_ERR_INVALID_TYPE;
    if (optimized && ((uintptr_t)pX & 0xFu)) return FFTLIB_ERR_NOT_ALIGNED_PTRS_STRIDES;
    // dim_x = 2 * 4^numShifts (powers of 4) or 4 * 4^numShifts (powers of 2)
    const uint32_t p4 = (1u << ((bS->dim_x * 2u) & 31u)) * 2u;
    if (p4 != bX->dim_x && p4 * 2u != bX->dim_x) return FFTLIB_ERR_INVALID_DIMENSION;
    return FFTLIB_SUCCESS;
}

// Real length of an r2c / c2r call; odd lengths pass the reference's c71
// checks (only dim_x / 2 is examined) but have no split-radix form.
FFTLIB_STATUS real_length(const FFTLIB_bufParams1D_t* bX, uint32_t* n)
{
    *n = bX->dim_x;
    if (*n & 1u) {
        set_error("real length %u is odd", *n);
        return FFTLIB_ERR_INVALID_DIMENSION;
    }
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS init_c2c(const FFTLIB_bufParams1D_t* bX, void* pBlock, uint32_t kind)
{
    if (!pBlock) return FFTLIB_ERR_NULL_POINTER;
    return init_fp32(pBlock, kind, bX->dim_x / 2u, 1u, 0u, false);
}

FFTLIB_STATUS run_c2c_kernel(float* pX, const FFTLIB_bufParams1D_t* bX, float* pY, void* pBlock, uint32_t kind)
{
    if (!pX || !pY || !bX) return FFTLIB_ERR_NULL_POINTER;
    const uint32_t n = bX->dim_x / 2u;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, kind, n, &r);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, n, 1u, kind == REC_1D_IFFT, r.plan);
}

FFTLIB_STATUS init_real(const FFTLIB_bufParams1D_t* bX, void* pBlock, uint32_t kind)
{
    if (!pBlock) return FFTLIB_ERR_NULL_POINTER;
    uint32_t n;
    FFTLIB_STATUS st = real_length(bX, &n);
    if (st != FFTLIB_SUCCESS) return st;
    return init_fp32(pBlock, kind, n, 1u, 1u, true);
}

FFTLIB_STATUS run_real_kernel(float* pX, const FFTLIB_bufParams1D_t* bX, float* pXFFT, float* pY, void* pBlock,
                              uint32_t kind)
{
    if (!pX || !pY || !bX) return FFTLIB_ERR_NULL_POINTER;
    uint32_t n;
    FFTLIB_STATUS st = real_length(bX, &n);
    if (st != FFTLIB_SUCCESS) return st;
    PlanRecord r;
    st = read_record(pBlock, kind, n, &r);
    if (st != FFTLIB_SUCCESS) return st;
    return kind == REC_1D_R2C ? exec_r2c(pX, pXFFT, pY, n, 1u, 1, r.plan) : exec_c2r(pX, pXFFT, pY, n, 1u, 1, r.plan);
}

FFTLIB_STATUS run_i16(int16_t* pX, const FFTLIB_bufParams1D_t* bX, int16_t* pW, int16_t* pY, uint32_t* pShift,
                      const FFTLIB_bufParams1D_t* bS)
{
    return exec_i16(pX, pW, pY, pShift, bS->dim_x, bX->dim_x / 2u, 1u);
}

} // namespace

extern "C" {

// ---- c2c forward -------------------------------------------------------------

FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                         FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                         FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                         void* pBlock)
{
    (void)pBlock;
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_C2C);
}

FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                            FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                            FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY)
{
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_C2C);
}

FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                  FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pY,
                                                  FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_C2C);
    if (st != FFTLIB_SUCCESS) return st;
    return init_c2c(bufParamsX, pBlock, REC_1D_C2C);
}

FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                    FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pY,
                                                    FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    (void)pW; (void)bufParamsW; (void)bufParamsY;
    return run_c2c_kernel(pX, bufParamsX, pY, pBlock, REC_1D_C2C);
}

FFTLIB_STATUS FFTLIB_fft1d_i32fc_c32fc_o32fc_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pY,
                                                FFTLIB_bufParams1D_t* bufParamsY)
{
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_C2C);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, bufParamsX->dim_x / 2u, 1u, false, nullptr);
}

// ---- c2c inverse -------------------------------------------------------------

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                          FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                          FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                          void* pBlock)
{
    (void)pBlock;
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_C2C);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                             FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                             FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY)
{
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_C2C);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                   FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pY,
                                                   FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_C2C);
    if (st != FFTLIB_SUCCESS) return st;
    return init_c2c(bufParamsX, pBlock, REC_1D_IFFT);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                     FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pY,
                                                     FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    (void)pW; (void)bufParamsW; (void)bufParamsY;
    return run_c2c_kernel(pX, bufParamsX, pY, pBlock, REC_1D_IFFT);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32fc_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                 FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pY,
                                                 FFTLIB_bufParams1D_t* bufParamsY)
{
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_C2C);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2c(pX, pY, bufParamsX->dim_x / 2u, 1u, true, nullptr);
}

// ---- r2c ---------------------------------------------------------------------

FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                        FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                        FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                        void* pBlock)
{
    (void)pBlock;
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_REAL_FWD);
}

FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                           FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                           FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY)
{
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_REAL_FWD);
}

FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                 FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pXFFT,
                                                 FFTLIB_bufParams1D_t* bufParamsXFFT, FFTLIB_F32* pSf,
                                                 FFTLIB_bufParams1D_t* bufParamsSf, FFTLIB_F32* pY,
                                                 FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    (void)pXFFT; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_REAL_FWD);
    if (st != FFTLIB_SUCCESS) return st;
    return init_real(bufParamsX, pBlock, REC_1D_R2C);
}

FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                   FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pXFFT,
                                                   FFTLIB_bufParams1D_t* bufParamsXFFT, FFTLIB_F32* pSf,
                                                   FFTLIB_bufParams1D_t* bufParamsSf, FFTLIB_F32* pY,
                                                   FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    (void)pW; (void)bufParamsW; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf; (void)bufParamsY;
    return run_real_kernel(pX, bufParamsX, pXFFT, pY, pBlock, REC_1D_R2C);
}

FFTLIB_STATUS FFTLIB_fft1d_i32f_c32fc_o32fc_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                               FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pXFFT,
                                               FFTLIB_bufParams1D_t* bufParamsXFFT, FFTLIB_F32* pSf,
                                               FFTLIB_bufParams1D_t* bufParamsSf, FFTLIB_F32* pY,
                                               FFTLIB_bufParams1D_t* bufParamsY)
{
    (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_REAL_FWD);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_r2c(pX, pXFFT, pY, bufParamsX->dim_x, 1u, 1, nullptr);
}

// ---- c2r ---------------------------------------------------------------------

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_checkParams(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                         FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                         FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                         void* pBlock)
{
    (void)pBlock;
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_REAL_INV);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_checkParams_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                            FFTLIB_F32* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                            FFTLIB_F32* pY, FFTLIB_bufParams1D_t* bufParamsY)
{
    return check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_REAL_INV);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_init(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                  FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pXFFT,
                                                  FFTLIB_bufParams1D_t* bufParamsXFFT, FFTLIB_F32* pSf,
                                                  FFTLIB_bufParams1D_t* bufParamsSf, FFTLIB_F32* pY,
                                                  FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    (void)pXFFT; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, true, FAM_REAL_INV);
    if (st != FFTLIB_SUCCESS) return st;
    return init_real(bufParamsX, pBlock, REC_1D_C2R);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_kernel(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                    FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pXFFT,
                                                    FFTLIB_bufParams1D_t* bufParamsXFFT, FFTLIB_F32* pSf,
                                                    FFTLIB_bufParams1D_t* bufParamsSf, FFTLIB_F32* pY,
                                                    FFTLIB_bufParams1D_t* bufParamsY, void* pBlock)
{
    (void)pW; (void)bufParamsW; (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf; (void)bufParamsY;
    return run_real_kernel(pX, bufParamsX, pXFFT, pY, pBlock, REC_1D_C2R);
}

FFTLIB_STATUS FFTLIB_ifft1d_i32fc_c32fc_o32f_cn(FFTLIB_F32* pX, FFTLIB_bufParams1D_t* bufParamsX, FFTLIB_F32* pW,
                                                FFTLIB_bufParams1D_t* bufParamsW, FFTLIB_F32* pXFFT,
                                                FFTLIB_bufParams1D_t* bufParamsXFFT, FFTLIB_F32* pSf,
                                                FFTLIB_bufParams1D_t* bufParamsSf, FFTLIB_F32* pY,
                                                FFTLIB_bufParams1D_t* bufParamsY)
{
    (void)bufParamsXFFT; (void)pSf; (void)bufParamsSf;
    FFTLIB_STATUS st = check_f32(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, false, FAM_REAL_INV);
    if (st != FFTLIB_SUCCESS) return st;
    uint32_t n;
    st = real_length(bufParamsX, &n);
    if (st != FFTLIB_SUCCESS) return st;
    return exec_c2r(pX, pXFFT, pY, n, 1u, 1, nullptr);
}

// ---- int16 -------------------------------------------------------------------

FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_checkParams(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX, int16_t* pW,
                                                         FFTLIB_bufParams1D_t* bufParamsW, int16_t* pY,
                                                         FFTLIB_bufParams1D_t* bufParamsY, uint32_t* pShift,
                                                         FFTLIB_bufParams1D_t* bufParamsShift, void* pBlock)
{
    return check_i16(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, pBlock, true);
}

FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_checkParams_cn(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX,
                                                            int16_t* pW, FFTLIB_bufParams1D_t* bufParamsW,
                                                            int16_t* pY, FFTLIB_bufParams1D_t* bufParamsY,
                                                            uint32_t* pShift, FFTLIB_bufParams1D_t* bufParamsShift)
{
    return check_i16(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, nullptr, false);
}

FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_init(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX, int16_t* pW,
                                                  FFTLIB_bufParams1D_t* bufParamsW, int16_t* pY,
                                                  FFTLIB_bufParams1D_t* bufParamsY, uint32_t* pShift,
                                                  FFTLIB_bufParams1D_t* bufParamsShift, void* pBlock)
{
    FFTLIB_STATUS st =
        check_i16(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, pBlock, true);
    if (st != FFTLIB_SUCCESS) return st;
    return write_record(pBlock, REC_1D_I16, bufParamsX->dim_x / 2u, 1u, 0u, nullptr);
}

FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_kernel(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX, int16_t* pW,
                                                    FFTLIB_bufParams1D_t* bufParamsW, int16_t* pY,
                                                    FFTLIB_bufParams1D_t* bufParamsY, uint32_t* pShift,
                                                    FFTLIB_bufParams1D_t* bufParamsShift, void* pBlock)
{
    (void)bufParamsW; (void)bufParamsY;
    if (!pX || !pW || !pY || !pShift || !bufParamsX || !bufParamsShift) return FFTLIB_ERR_NULL_POINTER;
    PlanRecord r;
    FFTLIB_STATUS st = read_record(pBlock, REC_1D_I16, bufParamsX->dim_x / 2u, &r);
    if (st != FFTLIB_SUCCESS) return st;
    DeviceScope scope(r.device);
    return run_i16(pX, bufParamsX, pW, pY, pShift, bufParamsShift);
}

FFTLIB_STATUS FFTLIB_fft1d_i16sc_c16sc_o16sc_cn(int16_t* pX, FFTLIB_bufParams1D_t* bufParamsX, int16_t* pW,
                                                FFTLIB_bufParams1D_t* bufParamsW, int16_t* pY,
                                                FFTLIB_bufParams1D_t* bufParamsY, uint32_t* pShift,
                                                FFTLIB_bufParams1D_t* bufParamsShift)
{
    FFTLIB_STATUS st =
        check_i16(pX, bufParamsX, pW, bufParamsW, pY, bufParamsY, pShift, bufParamsShift, nullptr, false);
    if (st != FFTLIB_SUCCESS) return st;
    return run_i16(pX, bufParamsX, pW, pY, pShift, bufParamsShift);
}

} // extern "C"
