// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_d(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<9, 16, 1, 3, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<27, 16, 3, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<60, 16, 4, 15, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<108, 16, 12, 12, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<180, 16, 15, 15, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<288, 16, 24, 12, 12, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<405, 16, 45, 9, 9, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<625, 8, 125, 5, 5, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<800, 16, 80, 16, 10, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<1152, 16, 96, 16, 12, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<1458, 16, 162, 9, 9, 9, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<1944, 16, 216, 12, 9, 9, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<2430, 16, 270, 10, 9, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<3125, 8, 625, 5, 5, 5, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<3840, 16, 256, 16, 16, 15>, 80>());
}

} // namespace fftb200
