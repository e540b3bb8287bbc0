// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths (fewer passes: larger radices, up to 27 and 32, with up to 32
// values per thread), registered as the planner's preferred schedules.
// Compiled for at least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_m(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<2592, 32, 144, 18, 18, 8>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3072, 32, 128, 16, 16, 12>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3200, 32, 128, 25, 16, 8>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3456, 32, 128, 27, 16, 8>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3750, 32, 150, 25, 15, 10>, 128, true>());
    out.push_back(static_entry<StaticSchedule<4000, 32, 160, 25, 16, 10>, 128, true>());
}

} // namespace fftb200
