// Fixed-size FFT kernels (see fft_static_impl.cuh) for the planner's
// schedules of 2^a 3^b 5^c lengths from 8 to 4096 that the hand-tuned
// entries (fft_static_a/b/c.cu) do not cover, with the pipelined kernel
// compiled for at least 80 registers per thread.
#include "fft_static_impl.cuh"

namespace fftb200 {

void register_static_k(std::vector<StaticEntry>& out)
{
    out.push_back(static_entry<StaticSchedule<25, 8, 5, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<54, 16, 6, 9, 6>, 80>());
    out.push_back(static_entry<StaticSchedule<100, 16, 10, 10, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<162, 16, 18, 9, 9, 2>, 80>());
    out.push_back(static_entry<StaticSchedule<270, 16, 30, 10, 9, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<400, 16, 27, 16, 5, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<600, 16, 40, 15, 8, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<768, 16, 52, 16, 16, 3>, 80>());
    out.push_back(static_entry<StaticSchedule<1125, 16, 75, 15, 15, 5>, 80>());
    out.push_back(static_entry<StaticSchedule<1440, 16, 144, 12, 12, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<1920, 16, 128, 16, 15, 8>, 80>());
    out.push_back(static_entry<StaticSchedule<2400, 16, 240, 16, 15, 10>, 80>());
    out.push_back(static_entry<StaticSchedule<3072, 16, 256, 16, 16, 12>, 80>());
    out.push_back(static_entry<StaticSchedule<3750, 16, 375, 15, 10, 5, 5>, 80>());
}

} // namespace fftb200
