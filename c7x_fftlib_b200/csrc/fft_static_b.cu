// Fixed-size FFT kernels (see fft_static_impl.cuh).
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_b(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<8192, 16, 512, 16, 16, 16, 2>>());
    out.push_back(static_entry<StaticSchedule<16384, 32, 512, 32, 32, 16>>());
    out.push_back(static_entry<StaticSchedule<512, 8, 64, 8, 8, 8>>());
    out.push_back(static_entry<StaticSchedule<128, 16, 8, 16, 8>>());
    out.push_back(static_entry<StaticSchedule<64, 8, 8, 8, 8>>());
    out.push_back(static_entry<StaticSchedule<32, 8, 4, 8, 4>>());
    out.push_back(static_entry<StaticSchedule<16, 8, 2, 8, 2>>());
    out.push_back(static_entry<StaticSchedule<8, 8, 1, 4, 2>>());
}

} // namespace fftb200
