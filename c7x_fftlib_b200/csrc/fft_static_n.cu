// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths (fewer passes: larger radices, up to 27 and 32, with up to 32
// values per thread), registered as the planner's preferred schedules.
// Compiled for at least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_n(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<625, 32, 25, 25, 25>, 128, true>());
    out.push_back(static_entry<StaticSchedule<1250, 32, 50, 25, 10, 5>, 128, true>());
    out.push_back(static_entry<StaticSchedule<1458, 32, 54, 27, 27, 2>, 128, true>());
    out.push_back(static_entry<StaticSchedule<1944, 32, 72, 27, 9, 8>, 128, true>());
    out.push_back(static_entry<StaticSchedule<2000, 32, 80, 25, 10, 8>, 128, true>());
    out.push_back(static_entry<StaticSchedule<2187, 32, 81, 27, 9, 9>, 128, true>());
    out.push_back(static_entry<StaticSchedule<2500, 32, 100, 25, 10, 10>, 128, true>());
}

} // namespace fftb200
