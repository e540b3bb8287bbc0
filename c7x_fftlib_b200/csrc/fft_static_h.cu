// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_h(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<18, 8, 3, 6, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<45, 16, 3, 15, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<81, 16, 9, 9, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<144, 16, 12, 12, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<225, 16, 15, 15, 15>, 80>());
    out.push_back(static_entry<StaticSchedule<360, 16, 24, 15, 8, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<500, 16, 50, 10, 10, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<720, 16, 48, 16, 15, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<972, 16, 108, 12, 9, 9>, 80>());
    out.push_back(static_entry<StaticSchedule<1280, 16, 86, 16, 16, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<1728, 16, 144, 12, 12, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<2187, 16, 243, 9, 9, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<2700, 16, 225, 15, 15, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<3456, 16, 288, 12, 12, 12, 2>, 80>());
}

} // namespace fftb200
