// Symmetry-function kernels instantiated for cutoff type 6.
// One translation unit per cutoff type so the variants compile in parallel.
#include "sf_impl.cuh"

namespace n2p2b
{

void sfLaunch_6(SFParams const& P, SFLaunch const& L, std::size_t shm,
                  cudaStream_t s, int variant)
{
    sfk::launchForCT<6>(P, L, shm, s, variant);
}

int sfBlocks_6(std::size_t shm, int variant)
{
    return sfk::blocksForCT<6>(shm, variant);
}

} // namespace n2p2b
