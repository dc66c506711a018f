// Host-side description of a 2G-HDNNP potential: input.nn settings, symmetry
// functions (types 2, 3, 9) sorted and grouped exactly as n2p2 does, the
// scaling read from scaling.data and the per-element atomic neural networks
// read from weights.%03zu.data.
//
// The ordering rules here fix the meaning of every index that crosses the
// boundary (NN input index = sorted SF index = scaling.data row, and the
// per-neighbor dG/dr slot tables), so they follow the reference exactly:
//   SF sort key      libnnp/SymFncExpRad.cpp:55-76, SymFncExpAngn.cpp:51-78
//   group criteria   libnnp/SymGrpExpRad.cpp (addMember), SymGrpExpAngn.cpp:68-99
//   group sort       libnnp/SymGrpExpAngn.cpp:48-66
//   member order     libnnp/SymGrpExpAngn.cpp:108-150
//   slot tables      libnnp/Element.cpp:289-311
//   scaling          libnnp/SymFnc.cpp:34-75,150-195; Mode.cpp:712-840
//   NN topology      libnnp/Mode.cpp:1158-1443
//   weight order     libnnp/NeuralNetwork.cpp:147-169
#pragma once

#include <cstddef>
#include <map>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "tables.h"

namespace n2p2b
{

// Cutoff function types, numbered as n2p2's `cutoff_type` keyword
// (libnnp/CutoffFunction.h enum CutoffType).
enum CutoffType
{
    CT_HARD = 0, CT_COS, CT_TANHU, CT_TANH, CT_EXP,
    CT_POLY1, CT_POLY2, CT_POLY3, CT_POLY4
};

// Symmetry function scaling (libnnp/SymFnc.h ScalingType).
enum ScalingType
{
    ST_NONE = 0, ST_SCALE, ST_CENTER, ST_SCALECENTER, ST_SCALESIGMA
};

// Activation functions, letters as in `global_activation_short`
// (libnnp/NeuralNetwork.cpp:1082-1091).
enum Activation
{
    AF_IDENTITY = 0, AF_TANH, AF_LOGISTIC, AF_SOFTPLUS, AF_RELU,
    AF_GAUSSIAN, AF_COS, AF_REVLOGISTIC, AF_EXP, AF_HARMONIC
};

inline bool isCompactType(int type)
{
    return type >= 20 && type <= 25;
}

// Element-weighted types (SymFncExpRadWeighted, SymFncExpAngnWeighted,
// SymFncCompRadWeighted, SymFncCompAngnWeighted, SymFncCompAngwWeighted):
// every neighbor element counts, weighted by its atomic number.
inline bool isWeightedType(int type)
{
    return type == 12 || type == 13 || type == 23 || type == 24
        || type == 25;
}

struct SymFnc
{
    int         type       = 0;   // 2 radial, 3 narrow angular, 9 wide
                                  // angular; 12 / 13 element-weighted
                                  // radial / narrow angular; 20 compact
                                  // radial, 21 / 22 compact narrow / wide
                                  // angular; 23 / 24 / 25 their
                                  // element-weighted forms
    int         ec         = 0;   // central element
    int         e1         = 0;   // neighbor element(s); e2 = -1 for radial
    int         e2         = -1;
    double      eta        = 0.0;
    double      rs         = 0.0;
    double      rc         = 0.0;
    double      zeta       = 0.0;
    double      lambda     = 0.0;
    int         zetaInt    = 0;
    bool        useIntegerPow = false;
    int         cutoffType = 0;
    double      cutoffAlpha = 0.0;
    // Compact types (SymFncBaseComp, SymFncBaseCompAng): radial support
    // (rl, rc), angular support in degrees, subtype and its core function.
    double      rl         = 0.0;
    double      angleLeft  = 0.0;
    double      angleRight = 0.0;
    std::string subtype;
    int         coreType   = 0;
    bool        asymmetric = false;
    double      convLength = 1.0;
    std::size_t lineNumber = 0;
    int         index      = 0;   // position in the element's sorted list
    std::vector<int> indexPerElement;  // dG/dr slot per neighbor element

    // Scaling (SymFnc::setScalingType).
    int    scalingType   = ST_NONE;
    double Smin = 0.0, Smax = 0.0;
    double Gmin = 0.0, Gmax = 0.0, Gmean = 0.0, Gsigma = 0.0;
    double scalingFactor = 1.0;

    bool   relevant(int ne) const
    {
        if (isWeightedType(type)) return true;
        return (type == 2 || type == 20) ? ne == e1
                                         : (ne == e1 || ne == e2);
    }
    double scale(double v) const;
    double unscale(double v) const;
};

bool sfLess(SymFnc const& a, SymFnc const& b);

struct SymGrp
{
    int              type = 0;
    int              ec = 0, e1 = 0, e2 = -1;
    double           rc = 0.0;
    int              cutoffType = 0;
    double           cutoffAlpha = 0.0;
    // Compact groups (SymGrpBaseComp): radial range of the members; rmin
    // stays 0 as in the reference (initialised to 0, then min'ed).
    double           rmin = 0.0, rmax = 0.0;
    std::vector<int> members;     // SF indices (element-local), member order
};

struct NeuralNet
{
    int              numLayers = 0;
    std::vector<int> neurons;      // per layer, layer 0 = inputs
    std::vector<int> activations;  // per layer
    bool             normalizeNeurons = false;
    // Per layer l >= 1: W[l] (out x in, row-major) and b[l].
    std::vector<std::vector<double>> W;
    std::vector<std::vector<double>> b;
    bool             hasWeights = false;
    int              numConnections() const;
    void             setConnections(std::vector<double> const& c);
};

struct Element
{
    std::string               symbol;
    int                       atomicNumber = 0;
    double                    atomicEnergyOffset = 0.0;
    std::vector<SymFnc>       sfs;
    std::vector<SymGrp>       groups;
    std::vector<std::vector<int>> sfTable;  // [neighbor element] -> SF index
    NeuralNet                 nn;
};

int         atomicNumberOf(std::string const& symbol);
std::string elementSymbolOf(int atomicNumber);

// Settings file (input.nn) as keyword -> list of (value, line number),
// following Settings::parseLines (libnnp/Settings.cpp:323-372).
class Settings
{
public:
    void loadFile(std::string const& fileName);
    void loadString(std::string const& text);
    bool exists(std::string const& key) const;
    std::string const& value(std::string const& key) const;
    std::vector<std::pair<std::string, std::size_t>>
         values(std::string const& key) const;

private:
    std::multimap<std::string, std::pair<std::string, std::size_t>> contents;
};

class Potential
{
public:
    // Mode::loadSettingsFile + Mode::setupGeneric
    // (normalization, elements, cutoff, SFs, slot tables, groups, NN).
    void loadSettingsFile(std::string const& fileName);
    void setupGeneric();
    // Mode::setupSymmetryFunctionScaling / ...ScalingNone.
    void setupSymmetryFunctionScaling(std::string const& fileName);
    void setupSymmetryFunctionScalingNone();
    // Mode::setupNeuralNetworkWeights for the short-range NN; `format` is
    // a printf pattern with one %zu / %03zu for the atomic number.
    void setupNeuralNetworkWeights(std::string const& format);

    Settings             settings;
    bool                 normalize = false;
    double               meanEnergy = 0.0;
    double               convEnergy = 1.0;
    double               convLength = 1.0;
    double               convCharge = 1.0;
    int                  cutoffType = CT_HARD;
    double               cutoffAlpha = 0.0;
    double               maxCutoffRadius = 0.0;
    int                  scalingType = ST_NONE;
    std::vector<Element> elements;
    bool                 hasScaling = false;

    int numElements() const { return (int)elements.size(); }
    int elementIndex(std::string const& symbol) const;
    int maxSymmetryFunctions() const;
    int maxSlots() const;

private:
    void setupNormalization();
    void setupElements();
    void setupCutoff();
    void setupSymmetryFunctions();
    void setupSymmetryFunctionMemory();
    void setupSymmetryFunctionGroups();
    void setupNeuralNetwork();
    void setGroupScaling();
};

} // namespace n2p2b
