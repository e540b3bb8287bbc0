// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths (fewer passes: larger radices, up to 27 and 32, with up to 32
// values per thread), registered as the planner's preferred schedules.
// Compiled for at least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_p(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<200, 32, 10, 20, 10>, 128, true>());
    out.push_back(static_entry<StaticSchedule<288, 32, 12, 24, 12>, 128, true>());
    out.push_back(static_entry<StaticSchedule<375, 32, 15, 25, 15>, 128, true>());
    out.push_back(static_entry<StaticSchedule<400, 32, 20, 20, 20>, 128, true>());
    out.push_back(static_entry<StaticSchedule<486, 32, 27, 27, 18>, 128, true>());
    out.push_back(static_entry<StaticSchedule<540, 32, 27, 27, 20>, 128, true>());
    out.push_back(static_entry<StaticSchedule<600, 32, 25, 25, 24>, 128, true>());
    out.push_back(static_entry<StaticSchedule<648, 32, 27, 27, 24>, 128, true>());
    out.push_back(static_entry<StaticSchedule<729, 32, 27, 27, 27>, 128, true>());
    out.push_back(static_entry<StaticSchedule<800, 32, 32, 32, 25>, 128, true>());
}

} // namespace fftb200
