// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_j(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<24, 16, 2, 12, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<50, 16, 5, 10, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<96, 16, 8, 16, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<160, 16, 16, 16, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<250, 16, 25, 10, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<384, 16, 26, 16, 8, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<576, 16, 48, 12, 12, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<750, 16, 75, 15, 10, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<1080, 16, 90, 15, 12, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<1350, 16, 113, 15, 15, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<1875, 16, 125, 15, 5, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<2304, 16, 192, 16, 12, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<2916, 16, 324, 12, 9, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<3645, 16, 405, 9, 9, 9, 5>, 80>());
}

} // namespace fftb200
