// Fixed-size FFT kernels (see fft_static_impl.cuh).
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_c(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<960, 16, 64, 16, 15, 4>>());
    out.push_back(static_entry<StaticSchedule<3000, 16, 200, 15, 8, 5, 5>>());
    out.push_back(static_entry<StaticSchedule<1536, 16, 128, 16, 16, 6>>());
    out.push_back(static_entry<StaticSchedule<480, 16, 32, 16, 15, 2>>());
    out.push_back(static_entry<StaticSchedule<240, 16, 16, 16, 15>>());
}

} // namespace fftb200
