// tc_dft_launch.cuh -- host launch of one k_tc_dft instantiation (internal).
#pragma once

#include <mutex>

#include "tc_dft.cuh"

namespace fftb200 {

template <int N1, int N2>
cudaError_t launch_tc_shape(const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err, cudaStream_t s)
{
    using S = TcShape<N1, N2>;
    if (batch == 0) return cudaSuccess;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static bool configured[64] = {};
    static int sms[64] = {};
    {
        std::lock_guard<std::mutex> lock(mu);
        if (dev >= 64) return cudaErrorInvalidDevice;
        if (!configured[dev]) {
            e = cudaFuncSetAttribute(k_tc_dft<N1, N2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)S::SMEM);
            if (e != cudaSuccess) return e;
            e = cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev);
            if (e != cudaSuccess) return e;
            configured[dev] = true;
        }
    }
    const uint32_t tiles = (batch + S::T - 1) / S::T;
    const uint32_t grid = tiles < (uint32_t)sms[dev] ? tiles : (uint32_t)sms[dev];
    k_tc_dft<N1, N2><<<grid, S::THREADS, S::SMEM, s>>>(x, y, w, batch, err);
    return cudaGetLastError();
}

} // namespace fftb200
