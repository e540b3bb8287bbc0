// Fixed-size FFT kernels (see fft_static_impl.cuh): 32-wide schedules that
// measured faster on B200 than the planner's heuristic pick for their
// lengths, registered as the planner's preferred schedules. Compiled for at
// least 128 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_q(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<270, 32, 10, 27, 10>, 128, true>());
    out.push_back(static_entry<StaticSchedule<2430, 32, 90, 27, 10, 9>, 128, true>());
    out.push_back(static_entry<StaticSchedule<3000, 32, 125, 25, 12, 10>, 128, true>());
}

} // namespace fftb200
