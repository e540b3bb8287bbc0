// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_e(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<10, 8, 2, 5, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<30, 8, 6, 6, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<72, 16, 6, 12, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<120, 16, 8, 15, 8>, 80>());
    out.push_back(static_entry<StaticSchedule<192, 16, 16, 16, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<300, 16, 20, 15, 5, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<432, 16, 36, 12, 12, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<640, 16, 43, 16, 8, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<810, 16, 90, 10, 9, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<1200, 16, 80, 16, 15, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<1500, 16, 150, 15, 10, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<2000, 16, 200, 10, 10, 10, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<2500, 16, 250, 10, 10, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<3200, 16, 214, 16, 8, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<3888, 16, 432, 12, 12, 9, 3>, 80>());
}

} // namespace fftb200
