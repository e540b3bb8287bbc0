// tc_dft_one.cu -- one-stage tensor-core DFT instantiations (n = 8..64).
#include <mutex>

#include "tc_dft.h"
#include "tc_dft_small.cuh"

namespace fftb200 {

cudaError_t launch_tc_one(uint32_t n, const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err,
                          cudaStream_t s)
{
    switch (n) {
    case 8: return launch_tc_small<8>(x, y, w, batch, err, s);
    case 16: return launch_tc_small<16>(x, y, w, batch, err, s);
    case 32: return launch_tc_small<32>(x, y, w, batch, err, s);
    case 64: return launch_tc_small<64>(x, y, w, batch, err, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace fftb200
