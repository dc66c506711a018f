// Launch descriptors and host-side launchers of the device pipeline.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <string>
#include <vector>

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

// One structure of a batch: its geometry and its atoms sorted by element
// (structAtoms[es[e] .. es[e + 1]) are its atoms of element e, ascending).
struct BatchStruct
{
    NLParams p;
    PhysBox  pb;
    int      doRemap;
    int      atomBeg, atomEnd;       // its atoms in the concatenated arrays
    int      es[kMaxElem + 1];
};

struct NLBatchLaunch
{
    int                 n = 0;               // atoms of all structures
    int                 numElements = 0;
    int                 NIMG = 1;            // largest image count
    long                capacity = 0;
    int                 warpsPerBlock = 4;
    int                 normalize = 0;
    double              convLength = 1.0;
    BatchStruct const*  bs = nullptr;
    int const*          structOf = nullptr;  // [n] structure of each atom
    int const*          structAtoms = nullptr;
    double const*       posIn = nullptr;
    double*             pos = nullptr;
    int const*          elem = nullptr;
    int*                nbrCount = nullptr;
    int*                nbrCountElem = nullptr;
    int*                nbrOff = nullptr;
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

void launchNeighborListBatch(NLBatchLaunch const& L, cudaStream_t s);

// Arithmetic of the per-atom stages: the plain form computes everything in
// FP64.  The mixed forms compute symmetry functions in FP32 and the atomic
// NNs on the tensor cores with BF16 operands and FP32 accumulation, and keep
// FP64 for displacements, energy sums and force accumulation.  PREC_MIXED
// splits every operand into BF16 high and low parts (three MMAs per product:
// hi*hi + hi*lo + lo*hi, about 16 significant bits); PREC_BF16 uses the
// high parts only (one MMA per product, 8 significant bits).
enum Precision
{
    PREC_FP64 = 0,
    PREC_MIXED = 1,
    PREC_BF16 = 2
};

// Symmetry functions (+ derivatives).
struct SFLaunch
{
    int            n = 0;
    int            derivatives = 1;
    int            precision = PREC_FP64;
    int            cap = 0;           // neighbor staging capacity per atom
    int            memberChunk = 12;  // members per register chunk
    int            grid = 0;          // persistent grid size
    long           warpBytes = 0;     // shared memory per warp (set by launcher)
    int            variant = 0;       // product-form shape / run chunking
    int            sortCats = 0;      // bit 0: order work categories by
                                      // partners; bit 1: balanced owners;
                                      // bit 2: one item list of the
                                      // segment ordered by partner count
    int            recCap = 0;        // staged kernel: triplet records per
                                      // warp batch (set by launcher)
    int            tablesShared = 0;  // staged kernel: group / member
                                      // tables staged in shared memory
    int            lockstep = 1;      // staged kernel: the lockstep path
                                      // for groups of at most 3 eta runs
    int const*     elem = nullptr;
    int const*     nbrOff = nullptr;
    int const*     nbrCountElem = nullptr;
    double const*  dx = nullptr;
    double const*  dy = nullptr;
    double const*  dz = nullptr;
    double const*  dd = nullptr;
    SFScale const* scale = nullptr;   // [element][maxSF]
    // Outputs in the compute type (double, or float in the mixed form).
    void*          G = nullptr;       // [n][maxSF]
    void*          dGdr = nullptr;    // per atom block [slot][3][neighbors]
    int*           status = nullptr;
};

void launchSymmetryFunctions(SFParams const& P, SFLaunch const& L,
                             cudaStream_t s);
std::size_t sfSharedBytes(SFParams const& P, int cap, int precision);
int sfBlocksPerSM(SFParams const& P, int cap, int variant, int precision);
int sfAtomsPerBlock(SFParams const& P, int variant);
// Kernel variant matching the potential's product-form groups:
// 0 = (4 shapes, 3 runs per chunk), 1 = (4, 1), 2 = (8, 1), 3 = (8, 2);
// 4 = (4, 3) and 5 = (8, 1) with the software-pipelined partner loop;
// 6 = (4 shapes) and 7 = (8 shapes) staged-triplet kernel (one CTA per
// atom, sf_staged.cuh) -- potentials it cannot serve run variant 0 / 5.
constexpr int kSFVariants = 8;
int sfDefaultVariant(SFParams const& P, int precision);
// Default SFLaunch::sortCats: the segment-wide item order by partner count
// (bit 2) for the product-form angular path whenever there are angular
// members; for the general angular paths categories by partner count
// (bit 0) and, with many angular members (long per-pair work), the
// balanced owner order (bit 1).
int sfDefaultSort(SFParams const& P);

// Atomic neural networks (forward + dE/dG) on the SIMT cores: FP64 (plain
// form) or FP32 (precision != PREC_FP64: the distilled student network).
struct NNLaunch
{
    int           n = 0;
    int           derivatives = 1;
    int           maxSF = 0;
    int           precision = PREC_FP64;  // type of weights, G and dE/dG
    int const*    elem = nullptr;
    void const*   weights = nullptr;  // blob, offsets in NNParams
    void const*   G = nullptr;
    double*       energy = nullptr;   // [n]
    void*         dEdG = nullptr;     // [n][maxSF]
    int const*    status = nullptr;
};

void launchNeuralNetworks(NNParams const& P, NNLaunch const& L,
                          cudaStream_t s);

// Atomic neural networks on the tensor cores (mixed form).  Per element the
// hidden layers run as 128-atom x width GEMMs (tcgen05.mma, BF16 operands
// in shared memory, FP32 accumulators in tensor memory); the single-output
// layer is a per-atom FP32 dot product.  Widths are padded to multiples of
// 16 with zero weights.
constexpr int kTcMaxHidden = kMaxLayers - 2;
constexpr int kTcRows = 128;              // atoms per tile (MMA M)

struct TcLayer
{
    int  in, out;        // true widths
    int  inP, outP;      // padded to multiples of 16
    int  act;            // activation of this layer's neurons
    int  w, wl;          // byte offsets of W (outP x inP, UMMA K-major), high
                         // and low BF16 parts, in the element's weight region
    int  wt, wtl;        // the same for W^T (inP x outP)
    int  b;              // float offset of the bias (outP) in the element's
                         // float region
    int  fp;             // tensor-memory column of this layer's f' values
    int  splitF, splitB; // operands of the forward (W) / backward (W^T) GEMM
                         // of this layer: 0 single BF16, 1 weights hi/lo
                         // (2 MMAs per K-step), 2 both hi/lo (3 MMAs)
};

struct TcNet
{
    int     hidden;               // number of hidden layers (>= 1)
    int     nin, ninP;            // input width (symmetry functions)
    int     outAct;               // output-neuron activation
    int     outW;                 // float offset of the output weights
    int     outB;                 // float offset of the output bias
    long    wOff;                 // byte offset of the weight region in blob
    int     wBytes;               // bytes of the weight region (16-multiple)
    long    fOff;                 // float offset of the float region in blob
    int     fCount;               // floats of the float region
    TcLayer layer[kTcMaxHidden];
};

struct TcNNParams
{
    int   numElements;
    int   maxP;                   // widest padded width (A tile columns)
    int   wMax;                   // bytes reserved for weights in smem
    int   fMax;                   // floats reserved for the float region
    int   split;                  // 1: some GEMM splits its activations
                                  // (the low operand tile is allocated)
    int   tmemCols;               // tensor-memory columns allocated per CTA
                                  // (accumulators, then the f' columns)
    int   smemBytes;              // dynamic shared memory per CTA
    TcNet net[kMaxElem];
};

struct TcNNLaunch
{
    int                n = 0;
    int                derivatives = 1;
    int                maxSF = 0;
    // Atoms of element e: atomsByElem[es.start[e] + k] for k < count_e, with
    // count_e = es.start[e + 1] - es.start[e], or listCount[e] (device) when
    // listCount is set (the teacher re-evaluating gated atoms).
    int const*         atomsByElem = nullptr;
    ElemStarts         es{};
    int const*         listCount = nullptr;
    int                grid = 0;
    unsigned char const* wblob = nullptr;  // BF16 weights (UMMA layout)
    float const*       fblob = nullptr;    // FP32 biases, output weights
    float const*       G = nullptr;        // [n][maxSF] scaled SFs
    double*            energy = nullptr;   // [n]
    float*             dEdG = nullptr;     // [n][maxSF]
    int*               status = nullptr;
};

void launchNeuralNetworksTC(TcNNParams const& P, TcNNLaunch const& L,
                            cudaStream_t s);
// Builds the tensor-core tables and blobs from the FP64 weight blob; false
// (with the reason) if a network does not fit the kernel.  split: 0 = single
// BF16 operands everywhere, 1 = hi/lo activations and weights in every
// GEMM, 2 = the same except the backward GEMMs of the hidden layers above
// the first, whose deltas stay single BF16 (their weights hi/lo).
bool tcBuild(NNParams const& nn, std::vector<double> const& blob, int split,
             TcNNParams& P, std::vector<unsigned char>& wblob,
             std::vector<float>& fblob, std::string& why);
// Resident CTAs per SM of the tensor-core NN kernel (shared and tensor
// memory limits).
int tcBlocksPerSM(TcNNParams const& P);

// Extrapolation test / student gate (kernels_gate.cu).
struct Range
{
    double lo, hi;    // allowed range of the unscaled symmetry function
};

struct EWLaunch
{
    int            n = 0;
    int            maxSF = 0;
    int            precision = PREC_FP64;   // type of G
    int            numSF[kMaxElem] = {};
    int const*     elem = nullptr;
    void const*    G = nullptr;             // [n][maxSF] scaled values
    SFScale const* scale = nullptr;         // [element][maxSF]
    Range const*   range = nullptr;         // [element][maxSF]
    int*           perAtom = nullptr;       // [n] warnings per atom, or null
    int*           list = nullptr;          // atoms with warnings, per
    int*           listCount = nullptr;     // element at listStart[e]
    int            listStart[kMaxElem] = {};
    int*           status = nullptr;
    int            countSlot = ST_EW_COUNT;  // status word that accumulates
};

void launchExtrapolationCheck(EWLaunch const& L, cudaStream_t s);

// Student training (kernels_student.cu).  The student network of element e
// has one hidden layer of hidden[e] tanh neurons and a linear output; its
// FP32 weights live in `blob` at the NNParams-style offsets below (W1 out x
// in, W1^T, b1, W2 (1 x H), W2^T, b2).
struct StudentLaunch
{
    int            n = 0;
    int            maxSF = 0;
    int            maxSlots = 0;
    int            numElements = 0;
    int            precision = PREC_FP64;     // type of G and dG/dr
    int            numSF[kMaxElem] = {};
    int            numSlots[kMaxElem][kMaxElem] = {};
    int            hidden[kMaxElem] = {};
    // Adam learning-rate factor per (element, input): 1 / sigma of the
    // input symmetry function (Adam on W1 for standardized inputs).
    float const*   lrScale = nullptr;         // [numElements][maxSF]
    long           woff1[kMaxElem] = {}, wtoff1[kMaxElem] = {};
    long           boff1[kMaxElem] = {};
    long           woff2[kMaxElem] = {}, wtoff2[kMaxElem] = {};
    long           boff2[kMaxElem] = {};
    int const*     elem = nullptr;
    int const*     nbrOff = nullptr;
    int const*     nbrIdx = nullptr;
    int const*     nbrCountElem = nullptr;
    int16_t const* slotSF = nullptr;
    int const*     atomsByElem = nullptr;
    ElemStarts     es{};
    int            blkBeg[kMaxElem + 1] = {}; // gradient blocks per element
    void const*    G = nullptr;
    void const*    dGdr = nullptr;
    double const*  Ei = nullptr;              // student atomic energies
    double const*  F = nullptr;               // student forces [n][3]
    double const*  labelE = nullptr;          // teacher atomic energies
    double const*  labelF = nullptr;          // teacher forces [n][3]
    int const*     batch = nullptr;           // batch atom indices
    int            batchSize = 0;
    double         wE = 1.0, wF = 1.0;        // loss weights
    double         eScale = 1.0;              // Ei units -> label units
    double         fScale = 1.0;              // chain-rule force -> F units
    float*         rE = nullptr;              // residuals (0 off the batch)
    float*         rF = nullptr;
    float*         u = nullptr;               // adjoint [n][maxSF]
    float*         blob = nullptr;            // student weights
    float*         m = nullptr;               // Adam moments (blob layout)
    float*         v = nullptr;
    float*         gpart = nullptr;           // [block][paramStride]
    float*         grad = nullptr;            // summed gradient (blob layout)
    int            paramStride = 0;
    double*        loss = nullptr;            // [2] sums of squared residuals
    float          lr = 1e-3f, beta1 = 0.9f, beta2 = 0.999f, epsAdam = 1e-8f;
    float          bc1 = 1.0f, bc2 = 1.0f;    // 1 - beta^t (bias correction)
};

struct RangeLaunch
{
    int            maxSF = 0;
    int            numElements = 0;
    int            precision = PREC_FP64;
    int            numSF[kMaxElem] = {};
    int const*     atomsByElem = nullptr;
    ElemStarts     es{};
    int            blkBeg[kMaxElem + 1] = {}; // 256-atom chunks per element
    void const*    G = nullptr;
    SFScale const* scale = nullptr;
    Range*         range = nullptr;           // [element][maxSF], min / max
};

std::size_t studentGradSmem(int maxNin, int maxH);
int studentGradBlocks(ElemStarts const& es, int numElements, int* blkBeg);
void launchStudentTrainStep(StudentLaunch const& L, std::size_t gradSmem,
                            int maxParams, cudaStream_t s);
void launchStudentRange(RangeLaunch const& L, cudaStream_t s);

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
    int            precision = PREC_FP64;  // type of the three inputs below
    void const*    dEdG = nullptr;
    void const*    dGdr = nullptr;
    double*        selfF = nullptr;   // [n][3]
    double*        pairF = nullptr;   // [entries][3]
    double*        F = nullptr;       // [n][3] output (physical units)
    double         forceScale = 1.0;  // divide by (convEnergy / convLength)
    int            gather = 1;        // 0: pair and self terms only
    int const*     status = nullptr;
};

void launchForces(ForceLaunch const& L, cudaStream_t s);
// dG/dr_i (self) of every atom into out [n][maxSF][3] (type of dGdr):
// minus the sum of its neighbor slots, per neighbor element in entry order
// (Atom::dGdr up to summation order).  Uses L's neighbor-list, slot-table
// and dGdr fields; not on the evaluation path.
void launchSelfDerivatives(ForceLaunch const& L, void* out, cudaStream_t s);

// Forces for an externally supplied neighbor list (an MD engine's local and
// ghost atoms, the InterfaceLammps::getForces scatter): thread per target
// m, F_m = [m local] selfF_m + sum of pairF over the entries pointing to m
// (revEntry[revOff[m] .. revOff[m + 1]), ascending: a fixed order).
struct TargetForceLaunch
{
    int           numLocal = 0;
    int           numTargets = 0;
    int const*    revOff = nullptr;
    int const*    revEntry = nullptr;
    double const* selfF = nullptr;
    double const* pairF = nullptr;
    double*       F = nullptr;          // [numTargets][3]
    double        forceScale = 1.0;
    int const*    status = nullptr;
};

void launchTargetForces(TargetForceLaunch const& L, cudaStream_t s);

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

// Per-structure energies of a batch: block per structure, fixed-order tree
// sum, then the conversion and energy offsets of one structure.
struct BatchEnergyLaunch
{
    int                numStructs = 0;
    int                numElements = 0;
    BatchStruct const* bs = nullptr;
    double const*      atomicEnergy = nullptr;
    double*            out = nullptr;            // [numStructs], physical
    double             convEnergy = 1.0;
    double             meanEnergy = 0.0;
    int                normalize = 0;
    double             offset[kMaxElem] = {};   // atomic energy offsets
    int const*         status = nullptr;
};

void launchEnergyBatch(BatchEnergyLaunch const& L, cudaStream_t s);

} // namespace n2p2b
