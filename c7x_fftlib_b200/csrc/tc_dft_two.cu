// tc_dft_two.cu -- two-stage tensor-core DFT instantiations (n = 128..4096).
#include "tc_dft.h"
#include "tc_dft_launch.cuh"

namespace fftb200 {

cudaError_t launch_tc_two(uint32_t n, const float2* x, float2* y, const float* w, uint32_t batch, uint32_t* err,
                          cudaStream_t s)
{
    switch (n) {
    case 128: return launch_tc_shape<16, 8>(x, y, w, batch, err, s);
    case 256: return launch_tc_shape<16, 16>(x, y, w, batch, err, s);
    case 512: return launch_tc_shape<32, 16>(x, y, w, batch, err, s);
    case 1024: return launch_tc_shape<32, 32>(x, y, w, batch, err, s);
    case 2048: return launch_tc_shape<64, 32>(x, y, w, batch, err, s);
    case 4096: return launch_tc_shape<64, 64>(x, y, w, batch, err, s);
    default: return cudaErrorInvalidValue;
    }
}

} // namespace fftb200
