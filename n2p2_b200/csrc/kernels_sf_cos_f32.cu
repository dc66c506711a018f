// Symmetry-function kernels instantiated for cutoff type 1, FP32 (mixed form).
// One translation unit per (cutoff type, precision) so the variants compile
// in parallel.
#include "sf_impl.cuh"

namespace n2p2b
{

void sfLaunch_1f(SFParams const& P, SFLaunch const& L, std::size_t shm,
                   cudaStream_t s, int variant)
{
    sfk::launchForCT<float, 1>(P, L, shm, s, variant);
}

int sfBlocks_1f(SFParams const& P, std::size_t shm, int variant)
{
    return sfk::blocksForCT<float, 1>(P, shm, variant);
}

} // namespace n2p2b
