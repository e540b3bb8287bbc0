// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_i(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<20, 16, 2, 10, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<48, 16, 4, 12, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<90, 16, 10, 10, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<150, 16, 15, 15, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<243, 16, 27, 9, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<375, 16, 25, 15, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<540, 16, 45, 15, 12, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<729, 16, 81, 9, 9, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<1000, 16, 100, 10, 10, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<1296, 16, 144, 12, 12, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<1800, 16, 120, 15, 15, 8>, 80>());
    out.push_back(static_entry<StaticSchedule<2250, 16, 225, 15, 15, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<2880, 16, 240, 16, 15, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<3600, 16, 240, 16, 15, 15>, 80>());
}

} // namespace fftb200
