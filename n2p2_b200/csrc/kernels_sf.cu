// Host side of the symmetry-function stage: shared-memory sizing, occupancy
// and dispatch to the kernel instantiated for the potential's cutoff type and
// the context's precision (kernels_sf_{cos,tanhu,poly2,any}{,_f32}.cu,
// templates in sf_impl.cuh).
#include <algorithm>
#include <cstdlib>

#include "kernels.h"
#include "sf_impl.cuh"

namespace n2p2b
{

#define N2P2B_SF_DECL(SUFFIX)                                                 \
    void sfLaunch_##SUFFIX(SFParams const&, SFLaunch const&, std::size_t,     \
                           cudaStream_t, int);                                \
    int sfBlocks_##SUFFIX(SFParams const&, std::size_t, int);
N2P2B_SF_DECL(1)
N2P2B_SF_DECL(2)
N2P2B_SF_DECL(6)
N2P2B_SF_DECL(any)
N2P2B_SF_DECL(1f)
N2P2B_SF_DECL(2f)
N2P2B_SF_DECL(6f)
N2P2B_SF_DECL(anyf)
#undef N2P2B_SF_DECL

namespace
{

long warpBytesFor(SFParams const& P, int cap, int precision)
{
    return precision != PREC_FP64
        ? sfk::warpBytes<float>(P.maxExp, P.maxSF, cap, P.numElements)
        : sfk::warpBytes<double>(P.maxExp, P.maxSF, cap, P.numElements);
}

bool isStaged(int variant) { return variant == 6 || variant == 7; }
int stagedShapes(int variant) { return variant == 7 ? 8 : 4; }

// The variant that runs: staged variants fall back to the per-owner kernel
// for potentials the staged kernel does not serve.
int effectiveVariant(SFParams const& P, int variant)
{
    if (isStaged(variant) && !sfk::stagedEligible(P, stagedShapes(variant)))
        return variant == 7 ? 5 : 0;
    return variant;
}

// Shared-memory geometry of the staged kernel.
struct StagedGeom
{
    int rb = 0;
    bool tables = false;
    long warpBytes = 0;
    std::size_t shm = 0;
};

template <typename R>
StagedGeom stagedGeomT(SFParams const& P, int cap, int ns)
{
    StagedGeom g;
    g.tables = sfk::stagedTablesShared<R>(P, cap, ns);
    g.rb = sfk::stagedRecordCap<R>(P, cap, ns, g.tables);
    g.warpBytes = sfk::stagedWarpBytes<R>(P.maxSF, ns, g.rb, cap);
    g.shm = sfk::stagedSharedBytes<R>(P, cap, ns, g.rb, g.tables);
    return g;
}

StagedGeom stagedGeom(SFParams const& P, int cap, int precision, int ns)
{
    return precision != PREC_FP64 ? stagedGeomT<float>(P, cap, ns)
                                  : stagedGeomT<double>(P, cap, ns);
}

} // namespace

std::size_t sfSharedBytes(SFParams const& P, int cap, int precision)
{
    return sfk::stagedTableBytes(P)
         + (std::size_t)sfk::kWarps * warpBytesFor(P, cap, precision);
}

int sfAtomsPerBlock(SFParams const& P, int variant)
{
    return isStaged(effectiveVariant(P, variant)) ? 1 : sfk::kWarps;
}

int sfBlocksPerSM(SFParams const& P, int cap, int variant, int precision)
{
    variant = effectiveVariant(P, variant);
    std::size_t const shm = isStaged(variant)
        ? stagedGeom(P, cap, precision, stagedShapes(variant)).shm
        : sfSharedBytes(P, cap, precision);
    bool const f = precision != PREC_FP64;
    switch (P.cutoffType)
    {
    case 1: return f ? sfBlocks_1f(P, shm, variant) : sfBlocks_1(P, shm, variant);
    case 2: return f ? sfBlocks_2f(P, shm, variant) : sfBlocks_2(P, shm, variant);
    case 6: return f ? sfBlocks_6f(P, shm, variant) : sfBlocks_6(P, shm, variant);
    default:
        return f ? sfBlocks_anyf(P, shm, variant) : sfBlocks_any(P, shm, variant);
    }
}

int sfDefaultVariant(SFParams const& P, int precision)
{
    int const ng = P.groupBeg[P.numElements];
    int n4 = 0, n8 = 0;
    for (int g = 0; g < ng; ++g)
    {
        if (P.groups[g].shapes == 4) ++n4;
        if (P.groups[g].shapes == 8) ++n8;
    }
    // Measured on the 24,576-atom water box: the staged-triplet kernel with
    // its lockstep path is the fastest in both precisions (4 shapes in FP32:
    // level with the software-pipelined per-owner kernel, variant 4).
    // Potentials the staged kernel does not serve fall back to the per-owner
    // kernels (0 with 4 shapes; 5 with 8).
    (void)precision;
    return n8 > n4 ? 7 : 6;
}

int sfDefaultSort(SFParams const& P)
{
    int most = 0;
    for (int e = 0; e < P.numElements; ++e)
    {
        int m = 0;
        for (int g = P.groupBeg[e]; g < P.groupBeg[e + 1]; ++g)
            if (P.groups[g].type != 2) m += P.groups[g].mcnt;
        most = std::max(most, m);
    }
    // Bit 2 (the product-form path's segment-wide item order) whenever
    // there are angular members; bits 0 and 1 serve the general paths.
    if (most == 0) return 1;
    return most >= 64 ? 7 : 5;
}

void launchSymmetryFunctions(SFParams const& P, SFLaunch const& L0,
                             cudaStream_t s)
{
    SFLaunch L = L0;
    L.variant = effectiveVariant(P, L.variant);
    std::size_t shm;
    if (isStaged(L.variant))
    {
        StagedGeom const g = stagedGeom(P, L.cap, L.precision,
                                        stagedShapes(L.variant));
        L.recCap = g.rb;
        L.tablesShared = g.tables ? 1 : 0;
        // N2P2B_SF_LOCKSTEP=0 keeps the batched (member, slice) path for
        // every narrow segment (measurements, tests; read per launch).
        char const* lockEnv = std::getenv("N2P2B_SF_LOCKSTEP");
        L.lockstep = lockEnv ? std::atoi(lockEnv) : 1;
        L.warpBytes = g.warpBytes;
        shm = g.shm;
    }
    else
    {
        L.warpBytes = warpBytesFor(P, L.cap, L.precision);
        shm = sfSharedBytes(P, L.cap, L.precision);
    }
    noteLaunches(1);
    bool const f = L.precision != PREC_FP64;
    int const v = L.variant;
    switch (P.cutoffType)
    {
    case 1: f ? sfLaunch_1f(P, L, shm, s, v) : sfLaunch_1(P, L, shm, s, v);
            break;
    case 2: f ? sfLaunch_2f(P, L, shm, s, v) : sfLaunch_2(P, L, shm, s, v);
            break;
    case 6: f ? sfLaunch_6f(P, L, shm, s, v) : sfLaunch_6(P, L, shm, s, v);
            break;
    default: f ? sfLaunch_anyf(P, L, shm, s, v)
               : sfLaunch_any(P, L, shm, s, v);
            break;
    }
}

namespace
{

__global__ void checkExpKernel(double const* x, double* y, long n)
{
    __shared__ double tab[sfk::kExpTableSize];
    for (int j = threadIdx.x; j < sfk::kExpTableSize; j += blockDim.x)
        tab[j] = sfk::kExp2Table[j];
    __syncthreads();
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x)
    {
        y[i] = sfk::expNonPositive(x[i], tab);
        y[n + i] = exp(x[i]);
    }
}

} // namespace

} // namespace n2p2b

extern "C" int n2p2b_check_exp(double const* x, double* y, int64_t n)
{
    using namespace n2p2b;
    if (n <= 0) return 0;
    double* dx = nullptr;
    double* dy = nullptr;
    if (cudaMalloc(&dx, sizeof(double) * n) != cudaSuccess) return -3;
    if (cudaMalloc(&dy, sizeof(double) * 2 * n) != cudaSuccess)
    {
        cudaFree(dx);
        return -3;
    }
    cudaError_t e = cudaMemcpy(dx, x, sizeof(double) * n,
                               cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
    {
        noteLaunches(1);
        checkExpKernel<<<256, 256>>>(dx, dy, (long)n);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(y, dy, sizeof(double) * 2 * n, cudaMemcpyDeviceToHost);
    cudaFree(dx);
    cudaFree(dy);
    return e == cudaSuccess ? 0 : -3;   // N2P2B_ERR_CUDA
}
