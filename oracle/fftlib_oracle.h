/*
 * fftlib_oracle.h -- CPU oracle for the FFTLIB batched FFT hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C restatement of the reference
 * FFTLIB natural-C (_cn) algorithms, used by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg as the checker. The product library
 * (c7x_fftlib_b200/libfftlib_b200.so) never links, loads or calls it.
 *
 * Parity is pinned: tests/test_oracle.py checks every function here against
 * the reference's own _cn code compiled from its sources (oracle/_ref/), and
 * against the golden vectors committed in tests/golden/ (generated from the
 * reference's Python models and committed extended test cases).
 *
 * All buffers follow the reference layouts: interleaved re/im, one row of
 * numPoints complex values per channel, channels contiguous.
 */
#ifndef FFTLIB_ORACLE_H
#define FFTLIB_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Twiddle tables in the reference layout. */
void orc_tw_gen_f32(float *pW, uint32_t numPoints);
void orc_tw_gen_i16(int16_t *pW, uint32_t numPoints);
void orc_split_factor_r2c(float *pSf, uint32_t numPoints);
void orc_split_factor_c2r(float *pSf, uint32_t numPoints);

/* Batched FP32 c2c forward (inverse = 0) or inverse (inverse = 1).
 * pX is used as the work buffer and is overwritten, as in the reference. */
int orc_fft_c2c_f32(float *pX, const float *pW, float *pY,
                    uint32_t numPoints, uint32_t numChannels, int inverse);

/* Batched FP32 real-to-complex: pX holds numChannels x numPoints reals,
 * pW the tables of orc_tw_gen_f32(numPoints/2), pSf orc_split_factor_r2c.
 * pXFFT is scratch of numChannels x numPoints floats. outmode 0 writes
 * numPoints/2+1 bins per channel, outmode 1 writes numPoints bins. */
int orc_fft_r2c_f32(float *pX, const float *pW, float *pXFFT, const float *pSf,
                    float *pY, uint32_t numPoints, uint32_t numChannels,
                    int outmode);

/* Batched FP32 complex-to-real: pX holds numPoints/2+1 (inMode 0) or
 * numPoints (inMode 1) bins per channel; pY receives numPoints reals per
 * channel. pXFFT is scratch of numChannels x numPoints floats. */
int orc_fft_c2r_f32(const float *pX, const float *pW, float *pXFFT,
                    const float *pSf, float *pY, uint32_t numPoints,
                    uint32_t numChannels, int inMode);

/* Batched int16 c2c forward with per-stage shift; bit-exact model of the
 * reference. pX is overwritten. */
int orc_fft_c2c_i16(int16_t *pX, const int16_t *pW, int16_t *pY,
                    const uint32_t *pShift, uint32_t numShifts,
                    uint32_t numPoints, uint32_t numChannels);

#ifdef __cplusplus
}
#endif

#endif
