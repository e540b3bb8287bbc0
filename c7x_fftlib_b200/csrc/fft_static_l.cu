// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths (fewer passes: larger radices, up to 27 and 32, with up to 32
// values per thread), registered as the planner's preferred schedules.
// Compiled for at least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_l(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<3125, 32, 125, 25, 25, 5>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3240, 32, 135, 27, 12, 10>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3645, 32, 135, 27, 15, 9>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3888, 32, 144, 27, 16, 9>, 128, true>());
    out.push_back(static_entry<StaticSchedule<4050, 32, 150, 27, 15, 10>, 128, true>());
}

} // namespace fftb200
