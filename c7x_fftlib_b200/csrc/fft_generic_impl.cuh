// fft_generic_impl.cuh -- one instantiation of the runtime-planned FP32 FFT
// engine. Each fft_generic_e*.cu includes this with its EMAX / MAXT so the
// instantiations compile as separate translation units.
#pragma once

#include <mutex>

#include "fft_engine.h"
#include "fft_stockham.cuh"

namespace fftb200 {

template <int EMAX, int MAXT>
__global__ void __launch_bounds__(MAXT) k_fft_stockham(const __grid_constant__ FftArgs a)
{
    extern __shared__ __align__(16) float2 smem[];
    fft_tile<EMAX>(a, smem, blockIdx.x * a.M);
}

// Raises the dynamic shared-memory limit of one kernel instantiation, once
// per device, to the largest amount requested so far. The bookkeeping lives
// in the template so every instantiation keeps its own.
template <int EMAX, int MAXT>
cudaError_t ensure_smem(size_t smem)
{
    if (smem <= 48u * 1024u) return cudaSuccess;
    static std::mutex mu;
    static size_t configured[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    if (dev < 64 && configured[dev] >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(k_fft_stockham<EMAX, MAXT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && dev < 64) configured[dev] = smem;
    return e;
}

template <int EMAX, int MAXT>
cudaError_t launch_generic(const FftArgs& a, cudaStream_t s)
{
    const size_t smem = (size_t)a.M * a.slen * sizeof(float2);
    cudaError_t e = ensure_smem<EMAX, MAXT>(smem);
    if (e != cudaSuccess) return e;
    const uint32_t grid = (a.batch + a.M - 1) / a.M;
    k_fft_stockham<EMAX, MAXT><<<grid, a.T * tile_group(a), smem, s>>>(a);
    return cudaGetLastError();
}

} // namespace fftb200
