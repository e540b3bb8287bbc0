// fft_i16.h -- launcher of the bit-exact int16 FFT kernel (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fftb200 {

// Number of radix-4 stages (= shift-vector entries read) for length n.
uint32_t i16_num_shifts(uint32_t n);

// Launch shape of the int16 kernel: tg threads per transform (a power of
// two up to i16_max_tg(n); a CTA of max(256, tg) threads holds
// max(256, tg) / tg transforms), at most gridCap CTAs (0: all that are
// resident), and the register budget minBlocks (3: at most 80 registers per
// thread; 4: at most 64, four CTAs per SM; 0: 3).
struct I16Choice {
    uint32_t tg;
    uint32_t gridCap;
    uint32_t minBlocks;
};
// The launcher's default tg: n / 16 for the fixed-length kernels, n / 32 for the
// run-time-length one, within [1, i16_max_tg(n)].
uint32_t i16_default_tg(uint32_t n);
// The largest tg: 1024 for n = 8192 and 16384 (one transform per CTA of tg
// threads), else 256. A CTA has i16_block_threads(tg) threads: max(256, tg).
uint32_t i16_max_tg(uint32_t n);
uint32_t i16_block_threads(uint32_t tg);
// The default launch of lengths 64...2048 on 16-byte aligned input copies the
// next transform's input into shared memory while the current one is
// transformed (an extra flat buffer per transform).
bool i16_prefetch(uint32_t n, uint32_t tg, uint32_t minBlocks);
// Dynamic shared memory of a CTA with that tg, and CTAs resident per SM.
size_t i16_smem_bytes(uint32_t n, uint32_t tg, bool prefetch = false);
int i16_resident(uint32_t n, uint32_t tg, uint32_t minBlocks = 3);
// n with tg threads per transform takes a kernel built for that length (64...4096;
// 8192 and 16384 with tg > 256), its stage constants folded
bool i16_fixed_length(uint32_t n, uint32_t tg);

// x, y: batch x n interleaved int16 complex; w: the caller's Q15 radix-4
// table (2n int16); shifts: i16_num_shifts(n) entries. All device pointers.
// n must be a power of two, 1 <= n <= 16384. tg = 0: i16_default_tg(n).
cudaError_t launch_fft_i16(const int16_t* x, int16_t* y, const int16_t* w, const uint32_t* shifts,
                           uint32_t n, uint32_t batch, cudaStream_t s, uint32_t tg = 0, uint32_t gridCap = 0,
                           uint32_t minBlocks = 3);

// Autotuner of the int16 launch shape for (device, n, batch bucket): times
// the candidate tg and CTA counts on synthetic data; cached like the FP32
// choices. False if nothing could be timed (the caller keeps the default).
bool tune_i16(uint32_t n, uint32_t batch, I16Choice* out);

} // namespace fftb200
