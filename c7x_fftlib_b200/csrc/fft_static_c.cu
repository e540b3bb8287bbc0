// Fixed-size FFT kernels (see fft_static_impl.cuh).
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_c(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<960, 32, 32, 32, 30>>());
    out.push_back(static_entry<StaticSchedule<3000, 32, 100, 30, 10, 10>>());
    out.push_back(static_entry<StaticSchedule<1536, 16, 128, 16, 16, 6>>());
    out.push_back(static_entry<StaticSchedule<480, 32, 16, 32, 15>>());
    out.push_back(static_entry<StaticSchedule<240, 16, 16, 16, 15>>());
}

} // namespace fftb200
