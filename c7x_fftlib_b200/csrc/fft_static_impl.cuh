// fft_static_impl.cuh -- fixed-size FFT kernels: the engine of
// fft_stockham.cuh with the whole schedule (length, radices, threads per
// transform, twiddle offsets) known at compile time, so every index and loop
// bound folds to constants. Each fft_static_*.cu instantiates a few
// schedules and registers them; launch_fft() prefers a registered fixed-size
// kernel when the planner's schedule matches one.
#pragma once

#include <algorithm>
#include <mutex>

#include "fft_engine.h"
#include "fft_pipeline.cuh"
#include "fft_stockham.cuh"

namespace fftb200 {

template <class S, int MAXT>
__global__ void __launch_bounds__(MAXT) k_fft_static(const __grid_constant__ FftArgs a)
{
    extern __shared__ __align__(16) float2 smem[];
    fft_tile_static<S>(a, smem, blockIdx.x * a.M);
}

template <class S, int MAXT>
cudaError_t launch_static(const FftArgs& a, cudaStream_t s)
{
    const size_t smem = (size_t)a.M * a.slen * sizeof(float2);
    if (a.T != (uint32_t)S::T || a.T * tile_group(a) > (uint32_t)MAXT) return cudaErrorInvalidConfiguration;
    if (smem > 48u * 1024u) {
        static std::mutex mu;
        static size_t configured[64] = {};
        int dev = 0;
        cudaError_t e = cudaGetDevice(&dev);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64 || configured[dev] < smem) {
            e = cudaFuncSetAttribute(k_fft_static<S, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            if (dev < 64) configured[dev] = smem;
        }
    }
    const uint32_t grid = (a.batch + a.M - 1) / a.M;
    k_fft_static<S, MAXT><<<grid, a.T * tile_group(a), smem, s>>>(a);
    return cudaGetLastError();
}

template <class S, int STAGES, int REGFLOOR, int IO>
__global__ void __launch_bounds__(S::T * pipe_tile(S::T),
                                  pipe_min_blocks(S::N, S::T * pipe_tile(S::T), STAGES, pipe_tile(S::T), REGFLOOR))
    k_fft_pipe(const __grid_constant__ FftArgs a)
{
    fft_pipeline<S, STAGES, pipe_tile(S::T), IO>(a);
}

// Persistent pipelined launch (pipe_tile(T) transforms per tile) of the
// instantiation for transform kind IO: as many CTAs as are resident on the
// device, at most a.gridCap.
template <class S, int STAGES, int REGFLOOR, int IO>
cudaError_t launch_pipe(const FftArgs& a, cudaStream_t s)
{
    constexpr int M = pipe_tile(S::T);
    if (a.T != (uint32_t)S::T || a.ioMode != IO) return cudaErrorInvalidConfiguration;
    const size_t smem = pipe_smem_bytes((uint32_t)S::N, STAGES, M);
    struct Cfg {
        int blocks = -1;
        int sms = 0;
    };
    static std::mutex mu;
    static Cfg cfg[64];
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int resident = 0, sms = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        Cfg& c = cfg[dev & 63];
        if (c.blocks < 0) {
            e = cudaFuncSetAttribute(k_fft_pipe<S, STAGES, REGFLOOR, IO>,
                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
            if (e != cudaSuccess) return e;
            e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&c.blocks, k_fft_pipe<S, STAGES, REGFLOOR, IO>,
                                                              S::T * M, smem);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
        }
        resident = c.blocks;
        sms = c.sms;
    }
    const uint32_t tiles = (a.batch + (uint32_t)M - 1u) / (uint32_t)M;
    uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)std::max(1, resident * sms));
    if (a.gridCap) grid = std::max(1u, std::min(grid, a.gridCap));
    if (a.overlapPrev) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(grid);
        lc.blockDim = dim3((unsigned)(S::T * M));
        lc.dynamicSmemBytes = smem;
        lc.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        lc.attrs = attr;
        lc.numAttrs = 1;
        return cudaLaunchKernelEx(&lc, k_fft_pipe<S, STAGES, REGFLOOR, IO>, a);
    }
    k_fft_pipe<S, STAGES, REGFLOOR, IO><<<grid, S::T * M, smem, s>>>(a);
    return cudaGetLastError();
}

// CTAs per SM of the persistent pipelined kernel.
template <class S, int STAGES, int REGFLOOR, int IO>
int resident_pipe()
{
    constexpr int M = pipe_tile(S::T);
    const size_t smem = pipe_smem_bytes((uint32_t)S::N, STAGES, M);
    int blocks = 0;
    if (cudaFuncSetAttribute(k_fft_pipe<S, STAGES, REGFLOOR, IO>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_fft_pipe<S, STAGES, REGFLOOR, IO>, S::T * M,
                                                      smem) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return blocks;
}

// REGFLOOR: see pipe_min_blocks (0 for the schedules tuned by hand).
// PREFERRED: the planner's choice for its length (see StaticEntry).
template <class S, int REGFLOOR = 0, bool PREFERRED = false>
StaticEntry static_entry()
{
    StaticEntry e{};
    e.preferred = PREFERRED;
    e.n = (uint32_t)S::N;
    e.emax = S::EMAX;
    e.T = (uint32_t)S::T;
    e.P = S::P;
    for (int i = 0; i < S::P; ++i) e.R[i] = S::R[i];
    constexpr int maxt = S::T > 256 ? S::T : 256;
    e.maxThreads = maxt;
    e.launch = &launch_static<S, maxt>;
    // the stage ring and exchange buffer must fit one CTA's shared memory
    // (odd lengths too: a tile's copy starts at the even element at or below
    // its first value, see tile_span); one instantiation per transform kind:
    // c2c for every length, r2c for even ones, c2r for even ones from 64 up
    // (whose stage holds the N + 1 bins beside the exchange layout)
    if constexpr (S::P >= 2 && pipe_smem_bytes(S::N, 2, pipe_tile(S::T)) <= 227u * 1024u) {
        e.launchPipelined[IO_C2C] = &launch_pipe<S, 2, REGFLOOR, IO_C2C>;
        e.residentPipelined[IO_C2C] = &resident_pipe<S, 2, REGFLOOR, IO_C2C>;
        if constexpr (S::N % 2 == 0) {
            e.launchPipelined[IO_R2C_SPLIT] = &launch_pipe<S, 2, REGFLOOR, IO_R2C_SPLIT>;
            e.residentPipelined[IO_R2C_SPLIT] = &resident_pipe<S, 2, REGFLOOR, IO_R2C_SPLIT>;
            e.mirrorLast = pipe_mirrorable<S>(S::P - 1);
        }
        if constexpr (S::N % 2 == 0 && S::N >= 64) {
            e.launchPipelined[IO_C2R_SPLIT] = &launch_pipe<S, 2, REGFLOOR, IO_C2R_SPLIT>;
            e.residentPipelined[IO_C2R_SPLIT] = &resident_pipe<S, 2, REGFLOOR, IO_C2R_SPLIT>;
            e.mirrorFirst = pipe_mirrorable<S>(0);
        }
    }
    return e;
}

} // namespace fftb200
