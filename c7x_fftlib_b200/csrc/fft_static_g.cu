// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_g(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<15, 8, 3, 5, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<40, 16, 4, 10, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<80, 16, 6, 16, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<135, 16, 15, 15, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<216, 8, 36, 6, 6, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<324, 16, 36, 12, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<486, 16, 54, 9, 9, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<675, 16, 45, 15, 15, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<900, 16, 60, 15, 15, 4>, 80>());
    out.push_back(static_entry<StaticSchedule<1250, 16, 125, 10, 5, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<1620, 16, 180, 15, 12, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<2160, 16, 180, 15, 12, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<2592, 16, 216, 12, 12, 6, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<3375, 16, 225, 15, 15, 15>, 80>());
    out.push_back(static_entry<StaticSchedule<4050, 16, 450, 10, 9, 9, 5>, 80>());
}

} // namespace fftb200
