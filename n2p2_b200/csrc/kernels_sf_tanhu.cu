// Symmetry-function kernels instantiated for cutoff type 2, FP64 (plain form).
// One translation unit per (cutoff type, precision) so the variants compile
// in parallel.
#include "sf_impl.cuh"

namespace n2p2b
{

void sfLaunch_2(SFParams const& P, SFLaunch const& L, std::size_t shm,
                   cudaStream_t s, int variant)
{
    sfk::launchForCT<double, 2>(P, L, shm, s, variant);
}

int sfBlocks_2(SFParams const& P, std::size_t shm, int variant)
{
    return sfk::blocksForCT<double, 2>(P, shm, variant);
}

} // namespace n2p2b
