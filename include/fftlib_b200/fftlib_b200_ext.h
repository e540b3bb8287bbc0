/*
 * fftlib_b200_ext.h -- extensions of libfftlib_b200.so beyond the FFTLIB API.
 * None of these has a counterpart in the reference library; existing FFTLIB
 * callers do not need them.
 */
#ifndef FFTLIB_B200_EXT_H_
#define FFTLIB_B200_EXT_H_

#include "FFTLIB_types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* exported from libfftlib_b200.so (built with hidden default visibility) */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* Text of the last failure on the calling thread ("" if none). */
const char *FFTLIB_b200_lastError(void);

/* Library version, major * 10000 + minor * 100 + patch. */
int FFTLIB_b200_version(void);

/* Frees every cached plan (twiddle tables) on every device. pBlocks
 * initialised earlier must be initialised again before use. */
void FFTLIB_b200_releasePlans(void);

/* Writes the kernel schedule chosen for a complex length-numPoints transform
 * (radices per pass, threads per transform, or the four-step split) into buf. */
FFTLIB_STATUS FFTLIB_b200_describePlan(uint32_t numPoints, char *buf, uint32_t len);

/* Writes the launch an _init recorded in pBlock into buf: "tuned: " when the
 * autotuner chose it (FFTLIB_B200_AUTOTUNE set to a non-zero value when
 * _init ran), "planner: " otherwise, then the radix schedule, the kernel
 * (fixed-size pipelined, fixed-size, or runtime-radix engine) and any CTA or
 * transforms-per-CTA choice; for int16, the threads per transform. No
 * reference counterpart (the reference keeps its plan in pBlock opaquely). */
FFTLIB_STATUS FFTLIB_b200_describeBlock(const void *pBlock, char *buf, uint32_t len);

/* Asynchronous variants of the _kernel calls: every buffer must be device
 * (or managed) memory; the work is enqueued on `stream` (a cudaStream_t;
 * NULL is the legacy default stream) and the call returns without waiting.
 * pBlock must come from the matching _init. These calls can be captured in
 * a CUDA graph. */
FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelAsync(FFTLIB_F32 *pX, FFTLIB_F32 *pY,
                                                                     uint32_t numPoints, uint32_t numChannels,
                                                                     void *pBlock, void *stream);
FFTLIB_STATUS FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32fc_kernelAsync(FFTLIB_F32 *pX, FFTLIB_F32 *pY,
                                                                      uint32_t numPoints, uint32_t numChannels,
                                                                      void *pBlock, void *stream);
FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i32f_c32fc_o32fc_kernelAsync(FFTLIB_F32 *pX, FFTLIB_F32 *pXFFT,
                                                                    FFTLIB_F32 *pY, uint32_t numPoints,
                                                                    uint32_t numChannels, uint8_t outmode,
                                                                    void *pBlock, void *stream);
FFTLIB_STATUS FFTLIB_b200_ifft1dBatched_i32fc_c32fc_o32f_kernelAsync(FFTLIB_F32 *pX, FFTLIB_F32 *pXFFT,
                                                                     FFTLIB_F32 *pY, uint32_t numPoints,
                                                                     uint32_t numChannels, uint8_t inMode,
                                                                     void *pBlock, void *stream);
FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i16sc_c16sc_o16sc_kernelAsync(int16_t *pX, int16_t *pW, int16_t *pY,
                                                                     uint32_t *pShift, uint32_t numShifts,
                                                                     uint32_t numPoints, uint32_t numChannels,
                                                                     void *pBlock, void *stream);

/* FP32 complex-to-complex forward FFT that allocates no memory.
 * No counterpart in the reference library. For callers that cannot allocate
 * at call time: code that runs under a device-memory budget fixed at start-up,
 * real-time loops that must not enter an allocator, or hosts whose allocator
 * belongs to another runtime. The regular _init/_kernel path allocates device
 * memory for plan tables and staging; this call uses only one scratch array
 * that is part of the library image (a static device array of 128 KiB + 256 B,
 * held on every GPU that loads the library until the process exits), so it
 * calls no cudaMalloc, cudaFree or other allocator.
 * - pX, pY: device buffers, numChannels rows of numPoints interleaved complex
 *   floats (the layout of FFTLIB_fft1dBatched_i32fc_c32fc_o32fc); pX is not
 *   modified.
 * - numPoints: 2^a 3^b 5^c, at most 16384, the longest length the
 *   single-kernel planner accepts (the array holds the twiddle table of any
 *   such length; longer or other lengths return FFTLIB_ERR_INVALID_DIMENSION);
 *   stream: a cudaStream_t (NULL = legacy default stream). The call
 *   synchronizes `stream` and reads the device error word back before it
 *   returns, so the result is in pY on return; for the same reason it must
 *   not be called while `stream` (or any stream) is being captured into a
 *   graph.
 * - Every call looks up the scratch array's device address
 *   (cudaGetSymbolAddress). The first call in a process builds the host-side
 *   schedule tables and loads the library's device code on the current
 *   device; CUDA's lazy module loading (the default) loads each kernel's code
 *   on its first launch, so make one warm-up call per length at start-up
 *   (or run with CUDA_MODULE_LOADING=EAGER), and later calls touch no
 *   allocator at all.
 * - Every call shares the one array and rebuilds its contents; calls that
 *   overlap on the GPU (other threads or streams) race on it. */
FFTLIB_STATUS FFTLIB_b200_fft1dBatched_i32fc_c32fc_o32fc_kernelNoAlloc(FFTLIB_F32 *pX, FFTLIB_F32 *pY,
                                                                       uint32_t numPoints, uint32_t numChannels,
                                                                       void *stream);

/* Batches of FP32 complex-to-complex transforms of uneven lengths, replayed
 * from one CUDA graph. No counterpart in the reference library (its batched
 * kernels take one length per call). Transform i has length numPoints[i]
 * (2^a 3^b 5^c, at most 4096) and occupies 2 * numPoints[i] floats of pX and
 * of pY, the transforms packed back to back in the order given. create()
 * groups the transforms by length. A group whose transforms lie back to back
 * runs its length's persistent fixed-size kernel; these launches follow one
 * another, each starting while the previous one drains (programmatic
 * dependent launch; $FFTLIB_B200_MIXED_BRANCHES = 2..8 spreads them over that
 * many parallel graph branches, each on a share of the GPU proportional to
 * its work); the other groups (or all,
 * with FFTLIB_B200_MIXED_PERSISTENT_ONLY) run in one persistent kernel over a
 * device-resident tile table, with radix schedules picked by the planner or
 * timed by the autotuner (FFTLIB_B200_MIXED_AUTOTUNE, or $FFTLIB_B200_AUTOTUNE
 * non-zero; results cached in $FFTLIB_B200_TUNE_CACHE, default
 * $HOME/.cache/fftlib_b200_tune.txt). exec() enqueues the transform on `stream`
 * (device buffers) and returns; execPerSize() runs the persistent kernel once
 * per distinct length, for comparison. create() synchronizes the device
 * (its descriptor uploads must land before any graph replay). */
typedef struct FFTLIB_b200_mixed *FFTLIB_b200_mixedHandle;
#define FFTLIB_B200_MIXED_INVERSE  1u
#define FFTLIB_B200_MIXED_AUTOTUNE 2u
/* every group in the single persistent kernel (no fixed-size groups) */
#define FFTLIB_B200_MIXED_PERSISTENT_ONLY 4u
FFTLIB_STATUS FFTLIB_b200_fftMixed_supported(uint32_t numPoints);
FFTLIB_STATUS FFTLIB_b200_fftMixed_create(const uint32_t *numPoints, uint32_t count, uint32_t flags,
                                          FFTLIB_b200_mixedHandle *handle);
FFTLIB_STATUS FFTLIB_b200_fftMixed_exec(FFTLIB_b200_mixedHandle handle, const FFTLIB_F32 *pX, FFTLIB_F32 *pY,
                                        void *stream);
FFTLIB_STATUS FFTLIB_b200_fftMixed_execPerSize(FFTLIB_b200_mixedHandle handle, const FFTLIB_F32 *pX,
                                               FFTLIB_F32 *pY, void *stream);
FFTLIB_STATUS FFTLIB_b200_fftMixed_describe(FFTLIB_b200_mixedHandle handle, char *buf, uint32_t len);
FFTLIB_STATUS FFTLIB_b200_fftMixed_destroy(FFTLIB_b200_mixedHandle handle);

/* The twiddle tables the reference test drivers build for the c2c/ifft
 * kernels and the int16 kernel, bit-identical to theirs. */
void FFTLIB_b200_tw_gen_c2c(FFTLIB_F32 *pW, uint32_t numPoints);
void FFTLIB_b200_tw_gen_i16(int16_t *pW, uint32_t numPoints);

/* The INT16 dftSmall / dftLarge products of the DFT coordinator and its
 * variants run on the tensor cores (exact u8 x u8 limb products) where the
 * row length divides 128 values; 0 selects the CUDA-core kernel instead,
 * which gives the same bits (for comparisons), 1 restores the default. */
void FFTLIB_b200_FFT_setIntTensorCores(int32_t enable);

/* The same generators on the GPU, for callers that keep no host copy of the
 * tables: the reference's formulas with pi truncated to 3.141592654 and the
 * same order of double operations, so the tables are bit-identical to the
 * host generators' (FFTLIB_b200_tw_gen_c2c / _i16 above; tw_gen_r2c,
 * split_factor_gen_r2c, ifft_c2r_tw_gen, ifft_c2r_split_factor_gen of
 * fft_c7x.h). The buffer is device memory of the host generator's size;
 * entries the host generator leaves unwritten are left unwritten. Enqueued
 * on `stream` (a cudaStream_t). FFTLIB_ERR_INVALID_VALUE for host memory,
 * FFTLIB_ERR_INVALID_DIMENSION for a negative numPoints, and for a Q15
 * numPoints that is not a power of two (the int16 kernel's lengths; for
 * others the host generator's stage blocks overlap and its table depends on
 * its write order). */
FFTLIB_STATUS FFTLIB_b200_tw_gen_c2c_device(FFTLIB_F32 *pW, uint32_t numPoints, void *stream);
FFTLIB_STATUS FFTLIB_b200_tw_gen_i16_device(int16_t *pW, uint32_t numPoints, void *stream);
FFTLIB_STATUS FFTLIB_b200_tw_gen_r2c_device(FFTLIB_F32 *pW, int32_t numPoints, void *stream);
FFTLIB_STATUS FFTLIB_b200_split_factor_gen_r2c_device(FFTLIB_F32 *pSFactor, int32_t numPoints, void *stream);
FFTLIB_STATUS FFTLIB_b200_ifft_c2r_tw_gen_device(FFTLIB_F32 *pW, int32_t numPoints, void *stream);
FFTLIB_STATUS FFTLIB_b200_ifft_c2r_split_factor_gen_device(FFTLIB_F32 *pSFactor, int32_t numPoints, void *stream);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* FFTLIB_B200_EXT_H_ */
