// Runtime-planned FP32 FFT engine, register capacity 8 complex values per
// thread, at most 1024 threads per CTA.
#include "fft_generic_impl.cuh"

namespace fftb200 {
template cudaError_t launch_generic<8, 1024>(const FftArgs&, cudaStream_t);
}
