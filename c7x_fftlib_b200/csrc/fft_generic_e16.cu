// Runtime-planned FP32 FFT engine, register capacity 16 complex values per
// thread, at most 512 threads per CTA.
#include "fft_generic_impl.cuh"

namespace fftb200 {
template cudaError_t launch_generic<16, 512>(const FftArgs&, cudaStream_t);
}
