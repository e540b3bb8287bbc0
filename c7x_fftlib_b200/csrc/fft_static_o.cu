// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths (fewer passes: larger radices, up to 27 and 32, with up to 32
// values per thread), registered as the planner's preferred schedules.
// Compiled for at least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_o(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<162, 32, 9, 18, 9>, 128, true>());
    out.push_back(static_entry<StaticSchedule<250, 32, 10, 25, 10>, 128, true>());
    out.push_back(static_entry<StaticSchedule<324, 32, 18, 18, 18>, 128, true>());
    out.push_back(static_entry<StaticSchedule<384, 32, 16, 32, 12>, 128, true>());
    out.push_back(static_entry<StaticSchedule<432, 32, 16, 27, 16>, 128, true>());
    out.push_back(static_entry<StaticSchedule<500, 32, 25, 25, 20>, 128, true>());
    out.push_back(static_entry<StaticSchedule<576, 32, 24, 24, 24>, 128, true>());
    out.push_back(static_entry<StaticSchedule<640, 32, 32, 32, 20>, 128, true>());
    out.push_back(static_entry<StaticSchedule<675, 32, 27, 27, 25>, 128, true>());
    out.push_back(static_entry<StaticSchedule<768, 32, 32, 32, 24>, 128, true>());
    out.push_back(static_entry<StaticSchedule<864, 32, 32, 32, 27>, 128, true>());
}

} // namespace fftb200
