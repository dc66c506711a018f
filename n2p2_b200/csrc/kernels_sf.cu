// Host side of the symmetry-function stage: shared-memory sizing, occupancy
// and dispatch to the kernel instantiated for the potential's cutoff type
// (kernels_sf_{cos,tanhu,poly2,any}.cu, templates in sf_impl.cuh).
#include "kernels.h"
#include "sf_impl.cuh"

namespace n2p2b
{

void sfLaunch_1(SFParams const&, SFLaunch const&, std::size_t, cudaStream_t,
                int);
void sfLaunch_2(SFParams const&, SFLaunch const&, std::size_t, cudaStream_t,
                int);
void sfLaunch_6(SFParams const&, SFLaunch const&, std::size_t, cudaStream_t,
                int);
void sfLaunch_any(SFParams const&, SFLaunch const&, std::size_t, cudaStream_t,
                  int);
int sfBlocks_1(std::size_t, int);
int sfBlocks_2(std::size_t, int);
int sfBlocks_6(std::size_t, int);
int sfBlocks_any(std::size_t, int);

long sfWarpDoubles(SFParams const& P, int cap)
{
    long const words = (cap + 31) / 32;
    long d = 7L * cap + (long)P.maxExp * cap + 4L * P.maxSF;
    d += (cap * words + 1) / 2;  // validity bits (uint32) in double units
    d += (long)(sfk::kMaxCats * sizeof(sfk::Cat) + 7) / 8;  // categories
    return d + 1;
}

std::size_t sfSharedBytes(SFParams const& P, int cap)
{
    int const ng = P.groupBeg[P.numElements];
    int nm = 0;
    if (ng > 0) nm = P.groups[ng - 1].mbeg + P.groups[ng - 1].mcnt;
    return sfk::tableBytes(ng, nm)
         + sizeof(double) * sfk::kWarps * sfWarpDoubles(P, cap);
}

int sfAtomsPerBlock() { return sfk::kWarps; }

int sfBlocksPerSM(SFParams const& P, int cap, int variant)
{
    std::size_t const shm = sfSharedBytes(P, cap);
    switch (P.cutoffType)
    {
    case 1: return sfBlocks_1(shm, variant);
    case 2: return sfBlocks_2(shm, variant);
    case 6: return sfBlocks_6(shm, variant);
    default: return sfBlocks_any(shm, variant);
    }
}

int sfDefaultVariant(SFParams const& P)
{
    int const ng = P.groupBeg[P.numElements];
    int n4 = 0, n8 = 0;
    for (int g = 0; g < ng; ++g)
    {
        if (P.groups[g].shapes == 4) ++n4;
        if (P.groups[g].shapes == 8) ++n8;
    }
    return (n8 > n4) ? 2 : 0;
}

void launchSymmetryFunctions(SFParams const& P, SFLaunch const& L0,
                             cudaStream_t s)
{
    SFLaunch L = L0;
    L.warpDoubles = sfWarpDoubles(P, L.cap);
    std::size_t const shm = sfSharedBytes(P, L.cap);
    noteLaunches(1);
    switch (P.cutoffType)
    {
    case 1: sfLaunch_1(P, L, shm, s, L.variant); break;
    case 2: sfLaunch_2(P, L, shm, s, L.variant); break;
    case 6: sfLaunch_6(P, L, shm, s, L.variant); break;
    default: sfLaunch_any(P, L, shm, s, L.variant); break;
    }
}

} // namespace n2p2b
