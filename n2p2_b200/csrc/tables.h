// Plain-old-data parameter tables shared by the host builder (context.cu) and
// the kernels.  The scalar parameters go to kernels by value as
// __grid_constant__ parameters; the symmetry-function group and member
// tables live in device memory (any size) and the kernel stages them into
// shared memory when they fit.
#pragma once

#include <cstdint>

namespace n2p2b
{

constexpr int kMaxElem      = 6;    // elements per potential on the device
constexpr int kMaxSF        = 4096; // symmetry functions per element
constexpr int kMaxLayers    = 8;    // NN layers incl. input and output
constexpr int kMaxWidth     = 512;  // NN layer width

// Core functions of the compact symmetry functions (CoreFunction::Type,
// libnnp/CoreFunction.h), as subtypes "p1".."p4" (optionally "a":
// asymmetric) and "e".
enum CompactCore
{
    CC_POLY1 = 1, CC_POLY2, CC_POLY3, CC_POLY4, CC_EXP
};

// Symmetry-function group (SymGrpExpRad / SymGrpExpAngn / SymGrpExpAngw).
struct DevGroup
{
    int    type;        // 2, 3, 9; weighted 12, 13 (e1 = e2 = -1: every
                        // element); compact 20, 21, 22 (rc = the members'
                        // largest rc, SymGrpBaseComp::rmax)
    int    e1, e2;      // neighbor elements (e2 == -1: radial)
    int    mbeg, mcnt;  // member range
    int    shapes;      // angular product form: members = runs x shapes
                        // (same (zeta, lambda) list per eta run, integer
                        // zeta, rs = 0); 0 = not of that form
    int    powBits;     // bits of the largest zeta - 1 of the members
                        // (branch-free integer powers when <= 4)
    int    cosSeries;   // 1: cosine cutoff with alpha = 0, evaluated for a
                        // pair distance as power series in (pi r / rc)^2
                        // (no square root, no sin/cos)
    double rc, rc2;     // cutoff radius and its square
    double rci, iw;     // CutoffFunction::rci, iw  (alpha-shifted inner cutoff)
    double rcinv;       // 1 / rc
    double a2;          // (pi / rc)^2 (cosSeries)
};

// One group member.  Angular members carry the SymGrpExpAngn::sortMembers
// derived factors; radial members use `factorNorm` for the scaling factor.
// Compact members (types 20-22) reuse the fields: eta, rs = radial support
// (rl, rc); lambda, zeta = angular support in radians; factorNorm = scaling
// factor; factorDeriv, zetaLambda = center and scale of the radial compact
// function; aCenter, aScale = those of the angular one
// (CompactFunction::setLeftRight); zetaInt = core function (CompactCore),
// useIntPow = asymmetric; calcExp = SymGrpCompAngn's calculateComp (the
// r_jk radial value is recomputed, not reused from the previous member);
// rsPositive = radial function id (first member of the group with the same
// rl, rc, core and asymmetry).
struct DevMember
{
    double  eta, rs, lambda, zeta;
    double  factorNorm;   // angular: 2^(1-zeta) * scalingFactor; radial: sf
    double  factorDeriv;  // 2 eta / zeta / lambda
    double  zetaLambda;   // zeta * lambda
    double  aCenter, aScale;  // compact angular function
    int16_t zetaInt;
    int16_t sf;           // element-local SF index (NN input index)
    uint8_t calcExp;      // first member of an (eta, rs) run
    uint8_t useIntPow;
    uint8_t rsPositive;
    uint8_t fillExp;      // first member of the element with its (eta, rs):
                          // fills the atom's exp table expIdx
    int16_t slot[kMaxElem];  // dG/dr slot per neighbor element, -1 = none
    int16_t expIdx;       // per-element index of the member's (eta, rs) run
};

struct SFParams
{
    int       numElements;
    int       cutoffType;      // CutoffType (global in n2p2)
    int       maxSlots;        // dG/dr slots per neighbor entry (stride)
    int       maxSF;           // SF stride of per-atom arrays
    int       maxExp;          // distinct angular (eta, rs) per element, max
    int       groupBeg[kMaxElem + 1];
    int       numSF[kMaxElem];
    int       numSlots[kMaxElem][kMaxElem];
    int       atomicNumber[kMaxElem];  // weights of types 12 and 13
    double    PI, PI_2, E, TANH_PRE;  // CutoffFunction constants, host-made
    int       numGroups;
    int       numMembers;
    int       stageTables;     // 1: kernels copy the tables to shared memory
    // Group / member tables: host copies (launch analysis on the host) and
    // device copies (kernels), same contents.
    DevGroup const*  groups;
    DevMember const* members;
    DevGroup const*  dGroups;
    DevMember const* dMembers;
};

// Final G transform per SF: G = Smin + b * (q * v - shift), with
// (Smin, b, shift) chosen so that all n2p2 scaling types come out
// exactly (SymFnc::scale): NONE -> (0, 1, 0), CENTER -> (0, 1, Gmean).
// q = factorNorm / scalingFactor for angular SFs (SymGrpExpAngn.cpp:396),
// 1 for radial.
struct SFScale
{
    double smin, b, shift, q;
};

// Neighbor-list geometry for one structure (all values in the units the
// kernels compute in, i.e. after normalization).
struct NLParams
{
    int    periodic;
    int    pbc[3];            // Structure::calculatePbcCopies
    int    ncell[3];          // cells per box vector (cell path) or 0
    int    nimg;              // (2 pbc0 + 1)(2 pbc1 + 1)(2 pbc2 + 1)
    double box[3][3];         // box[k] = k-th box vector
    double invbox[3][3];      // Structure::invbox rows
    double rc2;               // (max cutoff)^2, NL test dr.norm2() <= rc2
};

struct NNParams
{
    int    numElements;
    int    numLayers[kMaxElem];
    int    width[kMaxElem][kMaxLayers];
    int    act[kMaxElem][kMaxLayers];
    long   woff[kMaxElem][kMaxLayers];   // offset of W (out x in) in blob
    long   wtoff[kMaxElem][kMaxLayers];  // offset of W^T (in x out)
    long   boff[kMaxElem][kMaxLayers];   // offset of bias
    int    normalizeNeurons;
    int    maxWidth;
};

} // namespace n2p2b
