// fft_mixed.h -- uneven-length batch kernel (internal).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "fft_args.h"

namespace fftb200 {

// Schedule of one length group (FftArgs with in/out unused: every transform
// is addressed through the offsets array). args.M transforms make a tile;
// args.slen is the padded shared-memory length of one transform.
struct MixedGroup {
    FftArgs args;
};

// How a tile's inputs reach shared memory.
enum : uint32_t {
    kTileBulk = 1u,  // the tile's transforms lie back to back, 16-byte aligned: one bulk copy
    kTileRows = 2u,  // each transform's row is 16-byte aligned: one bulk copy per transform
    // neither: the first pass loads straight from global memory
};

// `count` transforms of one group: offsets[first .. first+count-1].
struct MixedTile {
    uint32_t group;
    uint32_t first;
    uint32_t count;
    uint32_t flags;
};

// Kernel classes by the register width of the runtime-radix engine:
// W16 (radices up to 16, three 256-thread CTAs per SM) serves every length
// that plans within 16 values per thread; W20 the few that need 20.
enum MixedClass : int { kMixedW16 = 0, kMixedW20 = 1, kMixedClasses = 2 };

struct MixedLaunch {
    int cls;
    const MixedGroup* groups;
    const MixedTile* tiles;  // this launch's tiles, in the order CTAs take them
    uint32_t numTiles;
    const uint64_t* offsets; // complex-element offset of each transform
    const float2* x;
    float2* y;
    uint32_t* err;           // error word of the bounded waits
    uint32_t stageLen;       // complex values per shared-memory stage
    uint32_t grid;
    size_t smem;
};

int mixed_class_emax(int cls);           // register capacity of the class's kernel
uint32_t mixed_block();                  // threads per CTA
uint32_t mixed_stage_max_bytes();        // largest stage a tile may need
size_t mixed_smem(uint32_t stageLen);    // dynamic shared memory of a launch
cudaError_t mixed_configure(int cls, size_t smem, int* residentPerSm);
cudaError_t launch_mixed(const MixedLaunch& L, cudaStream_t s);

} // namespace fftb200
