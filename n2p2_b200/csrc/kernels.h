// Launch descriptors and host-side launchers of the device pipeline.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "tables.h"
#include "device_common.cuh"

namespace n2p2b
{

struct ElemStarts
{
    int start[kMaxElem + 1];
};

struct NLLaunch
{
    int                 n = 0;
    int                 numElements = 0;
    int                 numCells = 0;
    long                capacity = 0;      // neighbor entries allocated
    NLParams            p{};
    PhysBox             pb{};
    int                 doRemap = 0;
    int                 normalize = 0;
    double              convLength = 1.0;
    double const*       posIn = nullptr;   // physical input positions
    double*             pos = nullptr;     // computing-unit positions
    int const*          elem = nullptr;
    int const*          atomsByElem = nullptr;
    ElemStarts          es{};
    int*                cellOf = nullptr;
    int*                cellCount = nullptr;
    int*                cellStart = nullptr;
    int*                cellFill = nullptr;
    int*                cellAtoms = nullptr;
    int*                cellScanStatus = nullptr;
    int*                nbrCount = nullptr;
    int*                nbrCountElem = nullptr;
    int*                nbrOff = nullptr;
    unsigned long long* keyTmp = nullptr;
    unsigned long long* key = nullptr;
    int*                nbrIdx = nullptr;
    int8_t*             nbrEl = nullptr;
    double*             dx = nullptr;
    double*             dy = nullptr;
    double*             dz = nullptr;
    double*             dd = nullptr;
    int*                entryAtom = nullptr;
    int*                mirror = nullptr;
    int*                status = nullptr;
};

// Running count of kernel launches issued by this library (diagnostics).
void noteLaunches(int k);

void launchNeighborList(NLLaunch const& L, cudaStream_t s);

// Symmetry functions (+ derivatives), FP64.
struct SFLaunch
{
    int            n = 0;
    int            derivatives = 1;
    int            cap = 0;           // neighbor staging capacity per atom
    int            memberChunk = 12;  // members per register chunk
    int            grid = 0;          // persistent grid size
    long           warpDoubles = 0;   // shared memory per warp (set by launcher)
    int            variant = 0;       // product-form shape / run chunking
    int            sortCats = 0;      // order work categories by partners
    int const*     elem = nullptr;
    int const*     nbrOff = nullptr;
    int const*     nbrCountElem = nullptr;
    double const*  dx = nullptr;
    double const*  dy = nullptr;
    double const*  dz = nullptr;
    double const*  dd = nullptr;
    SFScale const* scale = nullptr;   // [element][maxSF]
    double*        G = nullptr;       // [n][maxSF]
    double*        dGdrSelf = nullptr;// [n][maxSF][3]
    double*        dGdr = nullptr;    // per atom block [slot][3][neighbors]
    int*           status = nullptr;
};

void launchSymmetryFunctions(SFParams const& P, SFLaunch const& L,
                             cudaStream_t s);
std::size_t sfSharedBytes(SFParams const& P, int cap);
long sfWarpDoubles(SFParams const& P, int cap);
int sfBlocksPerSM(SFParams const& P, int cap, int variant);
int sfAtomsPerBlock();
// Kernel variant matching the potential's product-form groups:
// 0 = (4 shapes, 3 runs per chunk), 1 = (4, 1), 2 = (8, 1), 3 = (8, 2).
int sfDefaultVariant(SFParams const& P);

// Atomic neural networks (forward + dE/dG), FP64.
struct NNLaunch
{
    int           n = 0;
    int           derivatives = 1;
    int           maxSF = 0;
    int const*    elem = nullptr;
    double const* weights = nullptr;  // blob, offsets in NNParams
    double const* G = nullptr;
    double*       energy = nullptr;   // [n]
    double*       dEdG = nullptr;     // [n][maxSF]
    int const*    status = nullptr;
};

void launchNeuralNetworks(NNParams const& P, NNLaunch const& L,
                          cudaStream_t s);

// Forces (chain rule) and energy.
struct ForceLaunch
{
    int            n = 0;
    int            numElements = 0;
    int            maxSF = 0;
    int            maxSlots = 0;
    int const*     elem = nullptr;
    int const*     nbrOff = nullptr;
    int const*     nbrIdx = nullptr;
    int8_t const*  nbrEl = nullptr;
    int const*     mirror = nullptr;
    int16_t const* slotSF = nullptr;  // [ec][ne][maxSlots] -> SF index
    int            numSF[kMaxElem] = {};
    int            numSlots[kMaxElem][kMaxElem] = {};
    double const*  dEdG = nullptr;
    double const*  dGdrSelf = nullptr;
    double const*  dGdr = nullptr;
    double*        selfF = nullptr;   // [n][3]
    double*        pairF = nullptr;   // [entries][3]
    double*        F = nullptr;       // [n][3] output (physical units)
    double         forceScale = 1.0;  // divide by (convEnergy / convLength)
    int const*     status = nullptr;
};

void launchForces(ForceLaunch const& L, cudaStream_t s);

struct EnergyLaunch
{
    int           n = 0;
    double const* atomicEnergy = nullptr;
    double*       out = nullptr;       // [0] normalized sum, [1] physical
    double        convEnergy = 1.0;
    double        meanEnergy = 0.0;
    int           normalize = 0;
    int           numElements = 0;
    double        offsetTerm[kMaxElem] = {}; // count_e * offset_e, in order
    int const*    status = nullptr;
};

void launchEnergy(EnergyLaunch const& L, cudaStream_t s);

} // namespace n2p2b
