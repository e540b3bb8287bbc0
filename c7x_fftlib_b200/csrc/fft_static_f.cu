// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_f(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<12, 8, 2, 6, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<36, 8, 6, 6, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<75, 16, 5, 15, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<125, 8, 25, 5, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<200, 16, 20, 10, 10, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<320, 16, 22, 16, 5, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<450, 16, 30, 15, 15, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<648, 16, 72, 12, 9, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<864, 16, 72, 12, 12, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<1215, 16, 135, 15, 9, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<1600, 16, 160, 16, 10, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<2025, 16, 225, 15, 15, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<2560, 16, 256, 16, 16, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<3240, 16, 270, 15, 12, 6, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<4000, 16, 400, 10, 10, 10, 4>, 80>());
}

} // namespace fftb200
