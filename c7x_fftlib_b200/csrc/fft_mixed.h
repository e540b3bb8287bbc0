// fft_mixed.h -- uneven-length batch kernel (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_args.h"

namespace fftb200 {

// Schedule of one length group (FftArgs with in/out unused: every transform
// is addressed through the offsets array).
struct MixedGroup {
    FftArgs args;
};

// M transforms of one group: offsets[first .. first+count-1].
struct MixedTile {
    uint32_t group;
    uint32_t first;
    uint32_t count;
    uint32_t pad;
};

struct MixedLaunch {
    const MixedGroup* groups;
    const MixedTile* tiles;
    uint32_t numTiles;
    const uint64_t* offsets; // complex-element offset of each transform
    const float2* x;
    float2* y;
    uint32_t* counter;       // tile counter, zeroed by launch_mixed
    uint32_t grid;
    size_t smem;
};

int mixed_emax();   // register capacity the kernel is compiled for
int mixed_block();  // threads per CTA
cudaError_t mixed_configure(size_t smem, int* residentPerSm);
void* mixed_kernel_symbol();
cudaError_t launch_mixed(const MixedLaunch& L, cudaStream_t s);

} // namespace fftb200
