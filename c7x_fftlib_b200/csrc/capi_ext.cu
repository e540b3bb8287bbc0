// capi_ext.cu -- libfftlib_b200 extensions (include/fftlib_b200/fftlib_b200_ext.h)
// and the reference's host-side table generators.
#include <math.h>
#include <string.h>

#include <string>

#include "capi_common.h"
#include "fft_engine.h"
#include "fft_c7x.h"
#include "fft_i16.h"
#include "fftlib_b200_ext.h"
#include "plan.h"

using namespace fftb200;

namespace {

// The reference generators use pi truncated to 3.141592654
// (src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._tw_gen.cpp:12); the
// tables below reproduce the reference tables bit for bit, so the same
// value is used.
const double kTablePi = 3.141592654;

// One radix block (5, 3 or 4) of the FP32 stage-twiddle table: for each stage
// of that radix, r-1 sub-blocks of m0/r/stride twiddles W^(m*i) with i
// stepping by the stage stride; returns the size left for the next block.
uint32_t twiddle_block(float* w, uint32_t* k, uint32_t m0, uint32_t r)
{
    uint32_t rest = m0, t = m0 / r;
    for (uint32_t j = 1; j <= m0 / r && rest % r == 0; j *= r) {
        for (uint32_t i = 0; i < m0 / r; i += j) {
            for (uint32_t m = 1; m < r; ++m) {
                const double ang = (double)(2u * m) * kTablePi * (double)i / (double)m0;
                w[*k + 2u * (m - 1u) * t] = (float)cos(ang);
                w[*k + 2u * (m - 1u) * t + 1u] = (float)-sin(ang);
            }
            *k += 2u;
        }
        *k += 2u * t * (r - 2u);
        t /= r;
        rest /= r;
    }
    return rest;
}

void twiddle_table_f32(float* w, uint32_t n)
{
    uint32_t k = 0;
    if (n % 5u == 0u) n = twiddle_block(w, &k, n, 5u);
    if (n % 3u == 0u) n = twiddle_block(w, &k, n, 3u);
    if (n % 4u == 0u) twiddle_block(w, &k, n, 4u);
}

int16_t round_q15(double x)
{
    x = floor(0.5 + x);
    if (x >= 32767.0) return 32767;
    if (x <= -32768.0) return -32768;
    return (int16_t)x;
}

FFTLIB_STATUS async_record(void* pBlock, uint32_t kind, uint32_t n, PlanRecord* r)
{
    if (!pBlock) return FFTLIB_ERR_NULL_POINTER;
    memcpy(r, pBlock, sizeof(*r));
    if (r->magic != kRecordMagic || r->kind != kind) {
        set_error("pBlock was not initialised by the matching _init");
        return FFTLIB_ERR_FAILURE;
    }
    if (r->numPoints != n) return FFTLIB_ERR_INVALID_DIMENSION;
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS launched(cudaError_t e, const char* what)
{
    return e == cudaSuccess ? FFTLIB_SUCCESS : cuda_fail(e, what);
}

} // namespace

extern "C" {

const char* FFTLIB_b200_lastError(void) { return last_error(); }

int FFTLIB_b200_version(void) { return 100; }

void FFTLIB_b200_releasePlans(void) { release_all_plans(); }

FFTLIB_STATUS FFTLIB_b200_describePlan(uint32_t numPoints, char* buf, uint32_t len)
{
    if (!buf || len == 0) return FFTLIB_ERR_NULL_POINTER;
    std::string s;
    EnginePlan e;
    if (!is_235(numPoints)) return FFTLIB_ERR_INVALID_DIMENSION;
    int G = 0;
    uint32_t R[kMaxGlobal];
    if (plan_engine(numPoints, &e)) {
        // (c2c of these lengths runs one transform per thread instead)
        s = describe(e) + (small_fft_length(numPoints) ? " (fixed-size kernel; c2c: one transform per thread)"
                           : static_max_threads(numPoints, e.emax, e.T, e.P, e.R) ? " (fixed-size kernel)"
                                                                                : " (runtime-radix engine)");
    } else if (split_global(numPoints, &G, R)) {
        s = "global passes";
        for (int g = 0; g < G; ++g) {
            EnginePlan eg;
            plan_engine(R[g], &eg);
            s += (g ? " x " : " ") + std::to_string(R[g]) + " [" + describe(eg) + "]";
        }
    } else {
        return FFTLIB_ERR_NOT_IMPLEMENTED;
    }
    strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_describeBlock(const void* pBlock, char* buf, uint32_t len)
{
    if (!pBlock || !buf || len == 0) return FFTLIB_ERR_NULL_POINTER;
    PlanRecord r;
    memcpy(&r, pBlock, sizeof(r));
    if (r.magic != kRecordMagic) {
        set_error("pBlock was not initialised by an _init");
        return FFTLIB_ERR_FAILURE;
    }
    std::string s;
    if (r.kind == REC_I16 || r.kind == REC_1D_I16) {
        const uint32_t tg = r.i16Tg ? r.i16Tg : i16_default_tg(r.numPoints);
        s = std::string(r.i16Tuned ? "tuned: " : "planner: ") + "int16 radix-4 (" +
            (i16_fixed_length(r.numPoints, tg) ? "fixed-length" : "run-time-length") + " kernel), " + std::to_string(tg) +
            " threads per transform, " + std::to_string(i16_block_threads(tg) / tg) + " transforms per CTA";
        if (r.i16GridCap) s += ", " + std::to_string(r.i16GridCap) + " CTAs";
        if (r.i16MinBlocks == 4u) s += ", 64 registers (4 CTAs per SM)";
    } else if (r.plan) {
        s = describe_plan(r.plan);
    } else {
        return FFTLIB_ERR_FAILURE;
    }
    strncpy(buf, s.c_str(), len - 1);
    buf[len - 1] = '\0';
    return FFTLIB_SUCCESS;
}

FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync(FFTLIB_F32* pX, FFTLIB_F32* pY,
                                                                     uint32_t numPoints, uint32_t numChannels,
                                                                     void* pBlock, void* stream)
{
    PlanRecord r;
    FFTLIB_STATUS st = async_record(pBlock, REC_C2C, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    return launched(run_c2c(r.plan, (float2*)pX, (float2*)pY, numChannels, false, (cudaStream_t)stream),
                    "fft1dBatched c2c");
}

FFTLIB_STATUS FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32fc_kernelAsync(FFTLIB_F32* pX, FFTLIB_F32* pY,
                                                                      uint32_t numPoints, uint32_t numChannels,
                                                                      void* pBlock, void* stream)
{
    PlanRecord r;
    FFTLIB_STATUS st = async_record(pBlock, REC_IFFT, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    return launched(run_c2c(r.plan, (float2*)pX, (float2*)pY, numChannels, true, (cudaStream_t)stream),
                    "ifft1dBatched c2c");
}

FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i32f_c32fc_o32fc_kernelAsync(FFTLIB_F32* pX, FFTLIB_F32* pXFFT,
                                                                    FFTLIB_F32* pY, uint32_t numPoints,
                                                                    uint32_t numChannels, uint8_t outmode,
                                                                    void* pBlock, void* stream)
{
    PlanRecord r;
    FFTLIB_STATUS st = async_record(pBlock, REC_R2C, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    if (outmode > 1) return FFTLIB_ERR_INVALID_OUTMODE;
    if (r.plan->multiPass && !pXFFT) return FFTLIB_ERR_NULL_POINTER;
    return launched(run_r2c(r.plan, pX, (float2*)pXFFT, (float2*)pY, numChannels, outmode, (cudaStream_t)stream),
                    "fft1dBatched r2c");
}

FFTLIB_STATUS FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32f_kernelAsync(FFTLIB_F32* pX, FFTLIB_F32* pXFFT,
                                                                     FFTLIB_F32* pY, uint32_t numPoints,
                                                                     uint32_t numChannels, uint8_t inMode,
                                                                     void* pBlock, void* stream)
{
    PlanRecord r;
    FFTLIB_STATUS st = async_record(pBlock, REC_C2R, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    if (c2r_needs_scratch(r.plan, inMode ? 1 : 0) && !pXFFT) return FFTLIB_ERR_NULL_POINTER;
    return launched(run_c2r(r.plan, (const float2*)pX, (float2*)pXFFT, pY, numChannels, inMode ? 1 : 0,
                            (cudaStream_t)stream),
                    "ifft1dBatched c2r");
}

FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i16sc_c16sc_o16sc_kernelAsync(int16_t* pX, int16_t* pW, int16_t* pY,
                                                                     uint32_t* pShift, uint32_t numShifts,
                                                                     uint32_t numPoints, uint32_t numChannels,
                                                                     void* pBlock, void* stream)
{
    PlanRecord r;
    FFTLIB_STATUS st = async_record(pBlock, REC_I16, numPoints, &r);
    if (st != FFTLIB_SUCCESS) return st;
    if (!pX || !pW || !pY || !pShift) return FFTLIB_ERR_NULL_POINTER;
    if (numShifts < i16_num_shifts(numPoints)) return FFTLIB_ERR_INVALID_DIMENSION;
    return launched(launch_fft_i16(pX, pY, pW, pShift, numPoints, numChannels, (cudaStream_t)stream, r.i16Tg,
                                   r.i16GridCap, r.i16MinBlocks ? r.i16MinBlocks : 3u),
                    "fft1dBatched int16");
}

void FFTLIB_b200_tw_gen_c2c(FFTLIB_F32* pW, uint32_t numPoints) { twiddle_table_f32(pW, numPoints); }

// Q15 table of test/fft_c7x/FFTLIB_fft1dBatched_i16sc_c16sc_o16sc/..._d.c:39-61:
// radix-4 stages, 3 sub-blocks each, scaled by 32767.5 with round-half-up.
void FFTLIB_b200_tw_gen_i16(int16_t* pW, uint32_t numPoints)
{
    uint32_t k = 0, t = numPoints >> 2;
    for (uint32_t j = 1; j <= (numPoints >> 2); j <<= 2) {
        for (uint32_t i = 0; i < (numPoints >> 2); i += j) {
            for (uint32_t m = 1; m < 4; ++m) {
                const double ang = (double)(2u * m) * kTablePi * (double)i / (double)numPoints;
                pW[k + 2u * (m - 1u) * t] = round_q15(32767.5 * cos(ang));
                pW[k + 2u * (m - 1u) * t + 1u] = round_q15(32767.5 * (-sin(ang)));
            }
            k += 2;
        }
        k += 4u * t;
        t >>= 2;
    }
}

// src/fft_c7x/FFTLIB_fft1dBatched_i32f_c32fc_o32fc/..._tw_gen.cpp:9-78: the
// c2c table of the half-length transform.
void tw_gen_r2c(FFTLIB_F32* pW, int32_t numPoints) { twiddle_table_f32(pW, (uint32_t)numPoints >> 1); }

// ..._i32f_c32fc_o32fc_tw_gen.cpp:80-97
void split_factor_gen_r2c(FFTLIB_F32* pSFactor, int32_t numPoints)
{
    for (int32_t i = 0; i < numPoints / 2; ++i) {
        const double ang = 2.0 * kTablePi * (double)i / (double)numPoints;
        pSFactor[2 * i] = (float)(0.5 * (1.0 - sin(ang)));
        pSFactor[2 * i + 1] = (float)(0.5 * (-cos(ang)));
        pSFactor[2 * numPoints - 2 * i - 2] = (float)(0.5 * (1.0 + sin(ang)));
        pSFactor[2 * numPoints - 2 * i - 1] = (float)(0.5 * cos(ang));
    }
}

// src/fft_c7x/FFTLIB_ifft1dBatched_i32fc_c32fc_o32f/..._tw_gen.cpp:9-79
void ifft_c2r_tw_gen(FFTLIB_F32* pW, int32_t numPoints) { twiddle_table_f32(pW, (uint32_t)numPoints >> 1); }

// ..._i32fc_c32fc_o32f_tw_gen.cpp:81-95
void ifft_c2r_split_factor_gen(FFTLIB_F32* pSFactor, int32_t numPoints)
{
    for (int32_t i = 0; i < numPoints / 2; ++i) {
        const double ang = 2.0 * kTablePi * (double)i / (double)numPoints;
        pSFactor[2 * i] = (float)(0.5 * (1.0 - sin(ang)));
        pSFactor[2 * i + 1] = (float)(0.5 * cos(ang));
        pSFactor[2 * i + numPoints] = (float)(0.5 * (1.0 + sin(ang)));
        pSFactor[2 * i + numPoints + 1] = (float)(0.5 * (-cos(ang)));
    }
}

} // extern "C"
