// Fixed-size FFT kernels (see fft_static_impl.cuh).
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_a(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<4096, 16, 256, 16, 16, 16>>());
    // twice the values per thread (half the warps per barrier, twice the
    // independent work per warp): 3-4 % faster on B200, the planner's pick
    out.push_back(static_entry<StaticSchedule<4096, 32, 128, 16, 16, 16>, 0, true>());
    // three passes instead of 16x16x16x2: 146 -> 137 us for 4096 transforms
    out.push_back(static_entry<StaticSchedule<8192, 32, 256, 32, 16, 16>, 0, true>());
    out.push_back(static_entry<StaticSchedule<2048, 16, 128, 16, 16, 8>>());
    // radix 8 first: the c2r split of N = 4096 reals runs in its first pass
    out.push_back(static_entry<StaticSchedule<2048, 16, 128, 8, 16, 16>>());
    out.push_back(static_entry<StaticSchedule<1024, 16, 64, 16, 16, 4>>());
    out.push_back(static_entry<StaticSchedule<256, 16, 16, 16, 16>>());
}

} // namespace fftb200
