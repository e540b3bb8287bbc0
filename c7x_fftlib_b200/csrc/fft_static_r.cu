// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths, registered as the planner's preferred schedules. Compiled for at
// least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_r(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<1000, 32, 40, 25, 8, 5>, 128, true>());
    out.push_back(static_entry<StaticSchedule<2916, 32, 122, 27, 12, 9>, 128, true>());
}

} // namespace fftb200
