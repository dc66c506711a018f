// Shared device-side definitions: status words, small helpers.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "tables.h"

namespace n2p2b
{

// Status words (device int array), read by the host after a pipeline run.
enum StatusIndex
{
    ST_FLAGS = 0,       // error / path flags below
    ST_TOTAL_NBR = 1,   // total neighbor entries of the last list
    ST_MAX_NBR = 2,     // largest per-atom neighbor count
    ST_BAD_ATOM = 3,    // first atom that raised an error flag (or -1)
    ST_EW_COUNT = 4,    // extrapolation-warning count
    ST_GATE_COUNT = 5,  // symmetry functions outside the student's range
    ST_NUM = 8
};

enum StatusFlags
{
    FLAG_OUTSIDE_CELL  = 1 << 0,  // some atom outside [0,1]^3: brute path
    FLAG_NBR_OVERFLOW  = 1 << 1,  // neighbor entries exceed the capacity
    FLAG_SF_CAPACITY   = 1 << 2,  // an atom has more neighbors than the SF
                                  // kernel's shared-memory staging holds
    FLAG_MIRROR_MISSING = 1 << 3, // mirror entry not found (invariant broken)
    FLAG_ABORT         = 1 << 4,  // stop: later kernels return immediately
    FLAG_TC_TIMEOUT    = 1 << 5,  // a tensor-core wait gave up (bounded)
    FLAG_SF_PATH       = 1 << 6   // SF kernel lacks a needed code path
};

// Physical-unit box used by Structure::remap (before normalization).
struct PhysBox
{
    double box[3][3];
    double invbox[3][3];
};

__device__ __forceinline__ double warpSum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ float warpSumF(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

} // namespace n2p2b
