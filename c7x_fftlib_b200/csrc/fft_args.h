// fft_args.h -- launch descriptors shared by host planning code and the
// FP32 FFT kernels (plain C++ structs, no CUDA types beyond float2).
#pragma once

#include <stdint.h>
#include <vector_types.h>

#if defined(__CUDACC__)
#define FFTB_HD __host__ __device__
#else
#define FFTB_HD
#endif

namespace fftb200 {

constexpr int kMaxPasses = 8;

// Magic multiplier for floor(j / d) = umulhi(j, m), m = floor(2^32 / d) + 1,
// exact whenever j * d < 2^32 (all indices here are below 2^16).
inline FFTB_HD constexpr uint32_t fastdiv_magic(uint32_t d)
{
    return d <= 1u ? 0u : (uint32_t)((0x100000000ull / d) + 1ull);
}

// Shared-memory length (complex values) of one length-n region with one pad
// slot per 16 values.
inline FFTB_HD constexpr uint32_t smem_len(uint32_t n) { return n + (n >> 4) + 1u; }

// One Stockham pass of radix R: butterfly j reads in[j + q*N/R] (q < R),
// multiplies input q by W_{Ns*R}^{q*(j mod Ns)} and writes output q to
// out[(j/Ns)*Ns*R + (j mod Ns) + q*Ns]. Ns is the product of the radices of
// the passes before it, so the last pass writes out[j + q*N/R] (natural order).
struct PassInfo {
    int32_t  R;
    uint32_t Ns;
    uint32_t nsMagic;   // fastdiv_magic(Ns)
    uint32_t stride;    // N / R
    uint32_t twOffset;  // this pass's block in the twiddle table: entry
                        // (q-1)*Ns + k holds W_{Ns*R}^{q*k}, q = 1..R-1, k < Ns
};

enum IoMode : int32_t {
    IO_C2C = 0,        // complex in, complex out
    IO_R2C_SPLIT = 1,  // packed reals in, split post-process epilogue
    IO_C2R_SPLIT = 2,  // split pre-process prologue, packed reals out
};

struct FftArgs {
    const float2* in;
    float2*       out;
    const float2* tw;        // per-pass twiddle blocks (PassInfo::twOffset)
    uint32_t N;              // complex transform length handled by the passes
    uint32_t T;              // threads per transform (N / E)
    uint32_t M;              // transforms per CTA
    uint32_t P;              // number of passes
    PassInfo pass[kMaxPasses];
    int64_t  inBatch, inElem;    // strides in complex elements
    int64_t  outBatch, outElem;
    uint32_t batch;              // number of transforms
    int32_t  conjIn;             // conjugate on load  (inverse DFT = conj(FFT(conj x)))
    int32_t  conjOut;            // conjugate on store
    float    scale;              // applied on store
    int32_t  batchMinor;         // thread layout: transform index fastest
    int32_t  staged;             // tile through shared memory on load/store
    // real-input kernels (N = h = half the real length)
    int32_t  ioMode;             // IoMode
    int32_t  realMode;           // r2c outmode / c2r inMode
    const float2* twSplit;       // W_{2h}^i, i < h
    uint32_t nMagic;             // fastdiv_magic(N)
    // shared memory: per-transform stride (complex values) and, for staged
    // input, the input row length
    uint32_t slen;
    uint32_t inCount;
    uint32_t inMagic;            // fastdiv_magic(inCount)
    // error word (host-visible); kernels with bounded waits report here
    uint32_t* err;
    // global Stockham pass (perCh != 0): transform b is column j = b mod
    // perCh of channel c = b / perCh; it reads from c * inChStride +
    // j * inBatch and writes to c * outChStride + (j / outGroup) *
    // outGroupStride + (j mod outGroup) * outBatch (outGroup 0: j * outBatch)
    uint32_t perCh;
    uint32_t outGroup;
    int64_t  inChStride, outChStride, outGroupStride;
    // its input twiddle: element q of column j is multiplied by W_n^p,
    // p = q (j mod twNs) twStep, as twLo[p mod 2^twLoBits] * twHi[p >> twLoBits]
    const float2* twLo;
    const float2* twHi;
    uint32_t twLoBits;
    uint32_t twNs;
    uint32_t twStep;
    // staged tiles of M transforms computed Mc at a time (T * Mc threads;
    // 0: Mc = M); mMagic = fastdiv_magic(M)
    uint32_t Mc;
    uint32_t mMagic;
    // host-side launch hints, read by no kernel: at most gridCap CTAs for the
    // persistent kernels (0: as many as are resident); noPipe != 0 runs a
    // fixed-size schedule's one-tile-per-CTA kernel instead of its persistent
    // pipelined one; overlapPrev != 0 lets the persistent pipelined kernel
    // start while the previous kernel of its stream is still running
    // (programmatic dependent launch: only for launches whose inputs and
    // outputs no earlier kernel of the stream touches)
    uint32_t gridCap;
    uint32_t noPipe;
    uint32_t overlapPrev;
};

// Transforms one CTA computes at a time (its threads: T of them each).
inline FFTB_HD uint32_t tile_group(const FftArgs& a) { return a.Mc && a.staged ? a.Mc : a.M; }

} // namespace fftb200
