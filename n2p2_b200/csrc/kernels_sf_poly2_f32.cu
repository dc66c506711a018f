// Symmetry-function kernels instantiated for cutoff type 6, FP32 (mixed form).
// One translation unit per (cutoff type, precision) so the variants compile
// in parallel.
#include "sf_impl.cuh"

namespace n2p2b
{

void sfLaunch_6f(SFParams const& P, SFLaunch const& L, std::size_t shm,
                   cudaStream_t s, int variant)
{
    sfk::launchForCT<float, 6>(P, L, shm, s, variant);
}

int sfBlocks_6f(SFParams const& P, std::size_t shm, int variant)
{
    return sfk::blocksForCT<float, 6>(P, shm, variant);
}

} // namespace n2p2b
