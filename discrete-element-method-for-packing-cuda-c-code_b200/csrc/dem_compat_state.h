// dem_compat_state.h -- per-device state of the reference-compatible entry
// points: a few device words for reductions/status and a grow-only scratch
// buffer (radix histograms), allocated on the first call on each device and
// kept until exit.
#pragma once
#include "dem_common.cuh"

namespace dem {

struct CompatDevice {
    int device = -1;
    uint* words = nullptr;           // device: [0] status bits, [1] iall, [2] pcntot, [4..5] maxhz bits (u64)
    uint* scratch = nullptr;         // device scratch
    size_t scratch_words = 0;
    uint* host_words = nullptr;      // pinned mirror of words (8 uint)
};

int compat_device(CompatDevice** out);
int compat_scratch(CompatDevice* cd, size_t words, uint** out);
cudaStream_t compat_stream();

size_t radix_scratch_words(uint n);
int radix_sort_pairs(uint2* d0, uint2* d1, uint n, uint keybits, uint* scratch, cudaStream_t s);

}  // namespace dem
