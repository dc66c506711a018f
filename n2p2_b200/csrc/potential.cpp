// Host-side potential setup.  See potential.h for the reference rules each
// step follows.  Compiled with -ffp-contract=off so that every derived
// constant (unit conversion, scaling factors) is computed with the same
// IEEE operations as the reference's ISO C++ build.
#include "potential.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <limits>
#include <sstream>

namespace n2p2b
{

namespace
{

std::vector<std::string> splitWords(std::string const& s)
{
    std::vector<std::string> w;
    std::istringstream is(s);
    std::string t;
    while (is >> t) w.push_back(t);
    return w;
}

std::string joinWords(std::vector<std::string> const& w)
{
    std::string s;
    for (std::size_t i = 0; i < w.size(); ++i)
    {
        if (i) s += " ";
        s += w[i];
    }
    return s;
}

// Periodic table symbols by atomic number (1-based).
char const* const kSymbols[] = {
    "H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne",
    "Na", "Mg", "Al", "Si", "P",  "S",  "Cl", "Ar", "K",  "Ca",
    "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn",
    "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr",
    "Nb", "Mo", "Tc", "Ru", "Rh", "Pd", "Ag", "Cd", "In", "Sn",
    "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd",
    "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb",
    "Lu", "Hf", "Ta", "W",  "Re", "Os", "Ir", "Pt", "Au", "Hg",
    "Tl", "Pb", "Bi", "Po", "At", "Rn", "Fr", "Ra", "Ac", "Th",
    "Pa", "U",  "Np", "Pu", "Am", "Cm", "Bk", "Cf", "Es", "Fm",
    "Md", "No", "Lr", "Rf", "Db", "Sg", "Bh", "Hs", "Mt", "Ds",
    "Rg", "Cn", "Nh", "Fl", "Mc", "Lv", "Ts", "Og"};
int const kNumSymbols = (int)(sizeof(kSymbols) / sizeof(kSymbols[0]));

int activationFromLetter(std::string const& c)
{
    if (c == "l") return AF_IDENTITY;
    if (c == "t") return AF_TANH;
    if (c == "s") return AF_LOGISTIC;
    if (c == "p") return AF_SOFTPLUS;
    if (c == "r") return AF_RELU;
    if (c == "g") return AF_GAUSSIAN;
    if (c == "c") return AF_COS;
    if (c == "S") return AF_REVLOGISTIC;
    if (c == "e") return AF_EXP;
    if (c == "h") return AF_HARMONIC;
    throw std::runtime_error("ERROR: Unknown activation function \"" + c
                             + "\".\n");
}

// First column of every non-comment line (utility readColumnsFromFile).
std::vector<double> readFirstColumn(std::string const& fileName)
{
    std::ifstream f(fileName);
    if (!f.is_open())
    {
        throw std::runtime_error("ERROR: Could not open file: \"" + fileName
                                 + "\".\n");
    }
    std::vector<double> v;
    std::string line;
    while (std::getline(f, line))
    {
        if (!line.empty() && line[0] == '#') continue;
        std::vector<std::string> w = splitWords(line);
        if (w.empty()) continue;
        v.push_back(std::atof(w[0].c_str()));
    }
    return v;
}

} // namespace

int atomicNumberOf(std::string const& symbol)
{
    for (int i = 0; i < kNumSymbols; ++i)
    {
        if (symbol == kSymbols[i]) return i + 1;
    }
    throw std::runtime_error("ERROR: Unknown element symbol \"" + symbol
                             + "\".\n");
}

std::string elementSymbolOf(int atomicNumber)
{
    if (atomicNumber < 1 || atomicNumber > kNumSymbols)
    {
        throw std::runtime_error("ERROR: Atomic number out of range.\n");
    }
    return kSymbols[atomicNumber - 1];
}

double SymFnc::scale(double v) const
{
    switch (scalingType)
    {
    case ST_NONE:        return v;
    case ST_SCALE:       return Smin + scalingFactor * (v - Gmin);
    case ST_CENTER:      return v - Gmean;
    case ST_SCALECENTER: return Smin + scalingFactor * (v - Gmean);
    case ST_SCALESIGMA:  return Smin + scalingFactor * (v - Gmean);
    default:             return 0.0;
    }
}

double SymFnc::unscale(double v) const
{
    switch (scalingType)
    {
    case ST_NONE:        return v;
    case ST_SCALE:       return (v - Smin) / scalingFactor + Gmin;
    case ST_CENTER:      return v + Gmean;
    case ST_SCALECENTER: return (v - Smin) / scalingFactor + Gmean;
    case ST_SCALESIGMA:  return (v - Smin) / scalingFactor + Gmean;
    default:             return 0.0;
    }
}

// Strict weak order of n2p2's SymFnc::operator< for types 2, 3, 9
// (SymFncExpRad.cpp, SymFncExpAngn.cpp, SymFncExpAngw.cpp) and the compact
// types 20, 21, 22 (SymFncCompRad.cpp:55-74, SymFncCompAngn.cpp:52-74,
// SymFncCompAngw.cpp: subtype, elements, rc, rl, angles).
bool sfLess(SymFnc const& a, SymFnc const& b)
{
#define N2P2B_CMP(x) if (a.x < b.x) return true; if (a.x > b.x) return false;
    N2P2B_CMP(ec)
    N2P2B_CMP(type)
    if (isCompactType(a.type))
    {
        N2P2B_CMP(subtype)
        N2P2B_CMP(e1)
        if (a.type != 20 && a.type != 23)
        {
            N2P2B_CMP(e2)
        }
        N2P2B_CMP(rc)
        N2P2B_CMP(rl)
        if (a.type != 20 && a.type != 23)
        {
            N2P2B_CMP(angleLeft)
            N2P2B_CMP(angleRight)
        }
        return false;
    }
    N2P2B_CMP(cutoffType)
    N2P2B_CMP(cutoffAlpha)
    N2P2B_CMP(rc)
    N2P2B_CMP(eta)
    N2P2B_CMP(rs)
    if (a.type != 2)
    {
        N2P2B_CMP(zeta)
        N2P2B_CMP(lambda)
    }
    N2P2B_CMP(e1)
    if (a.type != 2)
    {
        N2P2B_CMP(e2)
    }
#undef N2P2B_CMP
    return false;
}

// SymGrp*::operator<; compact groups (SymGrpCompRad.cpp, SymGrpCompAngn.cpp,
// SymGrpCompAngw.cpp) compare elements only.
static bool grpLess(SymGrp const& a, SymGrp const& b)
{
#define N2P2B_CMP(x) if (a.x < b.x) return true; if (a.x > b.x) return false;
    N2P2B_CMP(ec)
    N2P2B_CMP(type)
    if (isCompactType(a.type))
    {
        N2P2B_CMP(e1)
        N2P2B_CMP(e2)
        return false;
    }
    N2P2B_CMP(cutoffType)
    N2P2B_CMP(cutoffAlpha)
    N2P2B_CMP(rc)
    N2P2B_CMP(e1)
    if (a.type != 2)
    {
        N2P2B_CMP(e2)
    }
#undef N2P2B_CMP
    return false;
}

int NeuralNet::numConnections() const
{
    int n = 0;
    for (int l = 1; l < numLayers; ++l)
    {
        n += neurons[l] * neurons[l - 1] + neurons[l];
    }
    return n;
}

// NeuralNetwork::setConnections (libnnp/NeuralNetwork.cpp:147-169): per layer,
// for each input j, for each neuron k: w[k][j]; then all biases.
void NeuralNet::setConnections(std::vector<double> const& c)
{
    if ((int)c.size() < numConnections())
    {
        throw std::runtime_error("ERROR: Too few neural network weights.\n");
    }
    W.assign(numLayers, std::vector<double>());
    b.assign(numLayers, std::vector<double>());
    std::size_t count = 0;
    for (int l = 1; l < numLayers; ++l)
    {
        int const nin = neurons[l - 1];
        int const nout = neurons[l];
        W[l].assign((std::size_t)nin * nout, 0.0);
        b[l].assign(nout, 0.0);
        for (int j = 0; j < nin; ++j)
        {
            for (int k = 0; k < nout; ++k)
            {
                W[l][(std::size_t)k * nin + j] = c[count++];
            }
        }
        for (int k = 0; k < nout; ++k) b[l][k] = c[count++];
    }
    hasWeights = true;
}

// -------------------------------------------------------------------------
// Settings
// -------------------------------------------------------------------------

void Settings::loadFile(std::string const& fileName)
{
    std::ifstream f(fileName);
    if (!f.is_open())
    {
        throw std::runtime_error("ERROR: Could not open file: \"" + fileName
                                 + "\".\n");
    }
    std::stringstream ss;
    ss << f.rdbuf();
    loadString(ss.str());
}

void Settings::loadString(std::string const& text)
{
    contents.clear();
    std::istringstream is(text);
    std::string line;
    std::size_t i = 0;
    for (; std::getline(is, line); ++i)
    {
        std::size_t p = line.find('#');
        if (p != std::string::npos) line.erase(p);
        p = line.find('!');
        if (p != std::string::npos) line.erase(p);
        std::vector<std::string> w = splitWords(line);
        if (w.empty()) continue;
        std::string key = w[0];
        w.erase(w.begin());
        contents.insert(std::make_pair(key, std::make_pair(joinWords(w), i)));
    }
}

bool Settings::exists(std::string const& key) const
{
    return contents.find(key) != contents.end();
}

std::string const& Settings::value(std::string const& key) const
{
    auto it = contents.find(key);
    if (it == contents.end())
    {
        throw std::runtime_error("ERROR: Keyword \"" + key
                                 + "\" not found.\n");
    }
    return it->second.first;
}

std::vector<std::pair<std::string, std::size_t>>
Settings::values(std::string const& key) const
{
    std::vector<std::pair<std::string, std::size_t>> v;
    auto r = contents.equal_range(key);
    for (auto it = r.first; it != r.second; ++it) v.push_back(it->second);
    return v;
}

// -------------------------------------------------------------------------
// Potential
// -------------------------------------------------------------------------

int Potential::elementIndex(std::string const& symbol) const
{
    for (std::size_t i = 0; i < elements.size(); ++i)
    {
        if (elements[i].symbol == symbol) return (int)i;
    }
    throw std::runtime_error("ERROR: Element \"" + symbol
                             + "\" is not part of the potential.\n");
}

int Potential::maxSymmetryFunctions() const
{
    int m = 0;
    for (auto const& e : elements) m = std::max(m, (int)e.sfs.size());
    return m;
}

int Potential::maxSlots() const
{
    int m = 0;
    for (auto const& e : elements)
        for (auto const& t : e.sfTable) m = std::max(m, (int)t.size());
    return m;
}

void Potential::loadSettingsFile(std::string const& fileName)
{
    settings.loadFile(fileName);
}

void Potential::setupGeneric()
{
    setupNormalization();
    setupElements();
    setupCutoff();
    setupSymmetryFunctions();
    setupSymmetryFunctionMemory();
    setupSymmetryFunctionGroups();
    setupNeuralNetwork();
}

// Mode::setupNormalization (libnnp/Mode.cpp:238-300).
void Potential::setupNormalization()
{
    bool const m = settings.exists("mean_energy");
    bool const e = settings.exists("conv_energy");
    bool const l = settings.exists("conv_length");
    if (m && e && l)
    {
        normalize = true;
        meanEnergy = std::atof(settings.value("mean_energy").c_str());
        convEnergy = std::atof(settings.value("conv_energy").c_str());
        convLength = std::atof(settings.value("conv_length").c_str());
        if (settings.exists("conv_charge"))
        {
            convCharge = std::atof(settings.value("conv_charge").c_str());
        }
    }
    else if (!m && !e && !l && !settings.exists("conv_charge"))
    {
        normalize = false;
    }
    else
    {
        throw std::runtime_error("ERROR: Incorrect usage of normalization"
                                 " keywords.\n");
    }
}

// Mode::setupElementMap + setupElements: elements sorted by atomic number
// (ElementMap::registerElements, libnnp/ElementMap.cpp:36-54).
void Potential::setupElements()
{
    if (settings.exists("nnp_type"))
    {
        std::string t = settings.value("nnp_type");
        if (t != "2" && t != "HDNNP_2G")
        {
            throw std::runtime_error("ERROR: Only 2G-HDNNPs (nnp_type 2) are "
                                     "supported on this path.\n");
        }
    }
    std::vector<std::string> syms = splitWords(settings.value("elements"));
    std::stable_sort(syms.begin(), syms.end(),
                     [](std::string const& a, std::string const& b)
                     { return atomicNumberOf(a) < atomicNumberOf(b); });
    int const n = std::atoi(settings.value("number_of_elements").c_str());
    if (n != (int)syms.size())
    {
        throw std::runtime_error("ERROR: Inconsistent number of elements.\n");
    }
    elements.clear();
    for (auto const& s : syms)
    {
        Element el;
        el.symbol = s;
        el.atomicNumber = atomicNumberOf(s);
        elements.push_back(el);
    }
    for (auto const& v : settings.values("atom_energy"))
    {
        std::vector<std::string> w = splitWords(v.first);
        elements.at(elementIndex(w.at(0))).atomicEnergyOffset =
            std::atof(w.at(1).c_str());
    }
}

// Mode::setupCutoff (libnnp/Mode.cpp:520-613).
void Potential::setupCutoff()
{
    std::vector<std::string> w = splitWords(settings.value("cutoff_type"));
    cutoffType = std::atoi(w.at(0).c_str());
    cutoffAlpha = 0.0;
    if (w.size() > 1)
    {
        cutoffAlpha = std::atof(w.at(1).c_str());
        if (0.0 < cutoffAlpha && cutoffAlpha >= 1.0)
        {
            throw std::invalid_argument("ERROR: 0 <= alpha < 1.0 is "
                                        "required.\n");
        }
    }
    if (cutoffType < CT_HARD || cutoffType > CT_POLY4)
    {
        throw std::invalid_argument("ERROR: Unknown cutoff type.\n");
    }
}

// SymFncBaseComp::setCompactFunction (libnnp/SymFncBaseComp.cpp:41-93):
// "p1".."p4" with an optional "a" (asymmetric), or "e".
static void setCompactSubtype(SymFnc& s)
{
    std::string const& t = s.subtype;
    if (t.size() < 1 || t.size() > 3)
        throw std::runtime_error("ERROR: Invalid compact function type "
                                 "specification: \"" + t + "\".\n");
    if (t.front() == 'p')
    {
        char const c = t.size() > 1 ? t.at(1) : '\0';
        if (c == '1') s.coreType = CC_POLY1;
        else if (c == '2') s.coreType = CC_POLY2;
        else if (c == '3') s.coreType = CC_POLY3;
        else if (c == '4') s.coreType = CC_POLY4;
        else
            throw std::runtime_error("ERROR: Invalid polynom type: \"" + t
                                     + "\".\n");
        if (t.size() == 3)
        {
            if (t.at(2) != 'a')
                throw std::runtime_error("ERROR: Invalid polynom specifier: "
                                         "\"" + t + "\".\n");
            s.asymmetric = true;
        }
    }
    else if (t.front() == 'e') s.coreType = CC_EXP;
    else
        throw std::runtime_error("ERROR: Unknown compact SF type: \"" + t
                                 + "\".\n");
}

// Mode::setupSymmetryFunctions (libnnp/Mode.cpp:615-690) with
// Element::addSymmetryFunction / sortSymmetryFunctions
// (libnnp/Element.cpp:82-166) and the parameter parsing of
// SymFncExpRad::setParameters / SymFncBaseExpAng::setParameters.
void Potential::setupSymmetryFunctions()
{
    int const ne = numElements();
    for (auto const& v : settings.values("symfunction_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        SymFnc s;
        s.ec = elementIndex(a.at(0));
        s.type = std::atoi(a.at(1).c_str());
        s.lineNumber = v.second;
        if (s.type == 2)
        {
            s.e1 = elementIndex(a.at(2));
            s.eta = std::atof(a.at(3).c_str());
            s.rs = std::atof(a.at(4).c_str());
            s.rc = std::atof(a.at(5).c_str());
        }
        else if (s.type == 3 || s.type == 9)
        {
            s.e1 = elementIndex(a.at(2));
            s.e2 = elementIndex(a.at(3));
            s.eta = std::atof(a.at(4).c_str());
            s.lambda = std::atof(a.at(5).c_str());
            s.zeta = std::atof(a.at(6).c_str());
            s.rc = std::atof(a.at(7).c_str());
            if (a.size() > 8) s.rs = std::atof(a.at(8).c_str());
            if (s.e1 > s.e2) std::swap(s.e1, s.e2);
            s.zetaInt = (int)std::round(s.zeta);
            s.useIntegerPow = std::fabs(s.zeta - s.zetaInt)
                              <= std::numeric_limits<double>::min();
        }
        else if (s.type == 12)
        {
            // SymFncExpRadWeighted::setParameters
            // (libnnp/SymFncExpRadWeighted.cpp:76-90): no element.
            s.e1 = -1;
            s.eta = std::atof(a.at(2).c_str());
            s.rs = std::atof(a.at(3).c_str());
            s.rc = std::atof(a.at(4).c_str());
        }
        else if (s.type == 13)
        {
            // SymFncExpAngnWeighted::setParameters
            // (libnnp/SymFncExpAngnWeighted.cpp:89-115).
            s.e1 = -1;
            s.e2 = -1;
            s.eta = std::atof(a.at(2).c_str());
            s.rs = std::atof(a.at(3).c_str());
            s.lambda = std::atof(a.at(4).c_str());
            s.zeta = std::atof(a.at(5).c_str());
            s.rc = std::atof(a.at(6).c_str());
            s.zetaInt = (int)std::round(s.zeta);
            s.useIntegerPow = std::fabs(s.zeta - s.zetaInt)
                              <= std::numeric_limits<double>::min();
        }
        else if (s.type == 20)
        {
            // SymFncCompRad::setParameters (libnnp/SymFncCompRad.cpp:84-113).
            s.e1 = elementIndex(a.at(2));
            s.rl = std::atof(a.at(3).c_str());
            s.rc = std::atof(a.at(4).c_str());
            s.subtype = a.at(5);
            if (s.rl > s.rc)
                throw std::runtime_error("ERROR: Lower radial boundary >= "
                                         "upper radial boundary.\n");
            setCompactSubtype(s);
        }
        else if (s.type == 23)
        {
            // SymFncCompRadWeighted::setParameters
            // (libnnp/SymFncCompRadWeighted.cpp:68-94): no element.
            s.e1 = -1;
            s.rl = std::atof(a.at(2).c_str());
            s.rc = std::atof(a.at(3).c_str());
            s.subtype = a.at(4);
            if (s.rl > s.rc)
                throw std::runtime_error("ERROR: Lower radial boundary >= "
                                         "upper radial boundary.\n");
            setCompactSubtype(s);
        }
        else if (s.type >= 21 && s.type <= 25)
        {
            // SymFncBaseCompAng::setParameters
            // (libnnp/SymFncBaseCompAng.cpp:48-115); the weighted forms
            // (SymFncBaseCompAngWeighted.cpp:46-100) have no elements.
            bool const w = (s.type == 24 || s.type == 25);
            int const o = w ? 0 : 2;
            s.e1 = w ? -1 : elementIndex(a.at(2));
            s.e2 = w ? -1 : elementIndex(a.at(3));
            s.rl = std::atof(a.at(2 + o).c_str());
            s.rc = std::atof(a.at(3 + o).c_str());
            s.angleLeft = std::atof(a.at(4 + o).c_str());
            s.angleRight = std::atof(a.at(5 + o).c_str());
            s.subtype = a.at(6 + o);
            if (s.e1 > s.e2) std::swap(s.e1, s.e2);
            if (s.rl > s.rc)
                throw std::runtime_error("ERROR: Lower radial boundary >= "
                                         "upper radial boundary.\n");
            setCompactSubtype(s);
            if (s.angleLeft >= s.angleRight)
                throw std::runtime_error("ERROR: Left angle boundary right "
                                         "of or equal to right angle "
                                         "boundary.\n");
            double const center = (s.angleLeft + s.angleRight) / 2.0;
            if ((s.angleLeft < 0.0 && center != 0.0)
                || (s.angleRight > 180.0 && center != 180.0))
                throw std::runtime_error("ERROR: Angle boundary out of "
                                         "[0,180] and center of angular "
                                         "function /= 0 or /= 180.\n");
            if (s.angleRight - s.angleLeft > 360.0)
                throw std::runtime_error("ERROR: Periodic symmetry function "
                                         "cannot spread over domain > 360 "
                                         "degrees\n");
        }
        else
        {
            throw std::runtime_error(
                "ERROR: Symmetry function type " + a.at(1)
                + " is not supported on this path (types 2, 3, 9, 12, 13, "
                  "20-25).\n");
        }
        elements.at(s.ec).sfs.push_back(s);
    }

    maxCutoffRadius = 0.0;
    for (auto& el : elements)
    {
        if (el.sfs.empty())
        {
            throw std::runtime_error("ERROR: Element " + el.symbol
                                     + " has no symmetry functions.\n");
        }
        if (normalize)
        {
            // SymFnc*::changeLengthUnit.
            for (auto& s : el.sfs)
            {
                s.convLength = convLength;
                s.eta /= convLength * convLength;
                s.rs *= convLength;
                s.rc *= convLength;
                s.rl *= convLength;
            }
        }
        std::sort(el.sfs.begin(), el.sfs.end(), sfLess);
        for (std::size_t i = 0; i < el.sfs.size(); ++i)
        {
            el.sfs[i].index = (int)i;
            el.sfs[i].cutoffType = cutoffType;
            el.sfs[i].cutoffAlpha = cutoffAlpha;
            el.sfs[i].indexPerElement.assign(ne, -1);
            maxCutoffRadius = std::max(maxCutoffRadius, el.sfs[i].rc);
        }
    }
}

// Element::setupSymmetryFunctionMemory (libnnp/Element.cpp:289-311).
void Potential::setupSymmetryFunctionMemory()
{
    int const ne = numElements();
    for (auto& el : elements)
    {
        el.sfTable.assign(ne, std::vector<int>());
        for (auto& s : el.sfs)
        {
            for (int i = 0; i < ne; ++i)
            {
                if (s.relevant(i))
                {
                    s.indexPerElement[i] = (int)el.sfTable[i].size();
                    el.sfTable[i].push_back(s.index);
                }
            }
        }
    }
}

// Element::setupSymmetryFunctionGroups (libnnp/Element.cpp:194-287).
void Potential::setupSymmetryFunctionGroups()
{
    for (auto& el : elements)
    {
        el.groups.clear();
        for (auto const& s : el.sfs)
        {
            bool const compact = isCompactType(s.type);
            bool const radial = (s.type == 2 || s.type == 12
                                 || s.type == 20 || s.type == 23);
            bool placed = false;
            for (auto& g : el.groups)
            {
                // SymGrp*::addMember: compact groups take every member of
                // their elements (SymGrpCompRad.cpp:60-85).
                if (g.type == s.type && g.ec == s.ec && g.e1 == s.e1
                    && (radial || g.e2 == s.e2)
                    && (compact || (g.cutoffType == s.cutoffType
                                    && g.cutoffAlpha == s.cutoffAlpha
                                    && g.rc == s.rc)))
                {
                    g.members.push_back(s.index);
                    if (compact) g.rmax = std::max(g.rmax, s.rc);
                    placed = true;
                    break;
                }
            }
            if (!placed)
            {
                SymGrp g;
                g.type = s.type;
                g.ec = s.ec;
                g.e1 = s.e1;
                g.e2 = radial ? -1 : s.e2;
                g.rc = s.rc;
                g.cutoffType = s.cutoffType;
                g.cutoffAlpha = s.cutoffAlpha;
                if (compact)
                {
                    g.rmin = 0.0;
                    g.rmax = s.rc;
                }
                g.members.push_back(s.index);
                el.groups.push_back(g);
            }
        }
        for (auto& g : el.groups)
            if (isCompactType(g.type)) g.rc = g.rmax;
        std::sort(el.groups.begin(), el.groups.end(), grpLess);
        for (auto& g : el.groups)
        {
            std::sort(g.members.begin(), g.members.end(),
                      [&el](int a, int b)
                      { return sfLess(el.sfs[a], el.sfs[b]); });
        }
    }
}

// Mode::setupNeuralNetwork (libnnp/Mode.cpp:1158-1443), short-range NN only.
void Potential::setupNeuralNetwork()
{
    int const ne = numElements();
    int globalHidden = 0;
    std::vector<int> numLayers(ne, 0);
    if (settings.exists("global_hidden_layers_short"))
    {
        globalHidden = std::atoi(settings.value(
            "global_hidden_layers_short").c_str());
        for (auto& n : numLayers) n = globalHidden + 2;
    }
    for (auto const& v : settings.values("element_hidden_layers_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        numLayers.at(elementIndex(a.at(0))) = std::atoi(a.at(1).c_str()) + 2;
    }
    for (int e = 0; e < ne; ++e)
    {
        if (numLayers[e] == 0)
        {
            throw std::runtime_error("ERROR: Number of neural network hidden "
                                     "layers unset for element "
                                     + elements[e].symbol + ".\n");
        }
    }
    std::vector<std::string> gNodes, gAct;
    if (settings.exists("global_nodes_short"))
    {
        gNodes = splitWords(settings.value("global_nodes_short"));
        if ((int)gNodes.size() != globalHidden)
        {
            throw std::runtime_error("ERROR: Inconsistent global NN topology"
                                     " keyword \"global_nodes_short\".\n");
        }
    }
    if (settings.exists("global_activation_short"))
    {
        gAct = splitWords(settings.value("global_activation_short"));
        if ((int)gAct.size() - 1 != globalHidden)
        {
            throw std::runtime_error("ERROR: Inconsistent global NN topology"
                                     " keyword \"global_activation_short\"."
                                     "\n");
        }
    }
    bool const normNodes = settings.exists("normalize_nodes");
    for (int e = 0; e < ne; ++e)
    {
        NeuralNet& nn = elements[e].nn;
        int const L = numLayers[e];
        nn.numLayers = L;
        nn.neurons.assign(L, 0);
        nn.activations.assign(L, -1);
        nn.neurons[0] = (int)elements[e].sfs.size();
        nn.activations[0] = AF_IDENTITY;
        nn.neurons[L - 1] = 1;
        nn.normalizeNeurons = normNodes;
        if (L != globalHidden + 2) continue;
        for (int j = 1; j < L; ++j)
        {
            if (j == L - 1 && !gAct.empty())
            {
                nn.activations[j] = activationFromLetter(gAct.at(L - 2));
            }
            else
            {
                if (!gNodes.empty())
                    nn.neurons[j] = std::atoi(gNodes.at(j - 1).c_str());
                if (!gAct.empty())
                    nn.activations[j] = activationFromLetter(gAct.at(j - 1));
            }
        }
    }
    for (auto const& v : settings.values("element_nodes_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        NeuralNet& nn = elements.at(elementIndex(a.at(0))).nn;
        if (nn.numLayers != (int)a.size() - 1 + 2)
        {
            throw std::runtime_error("ERROR: Inconsistent per-element NN "
                                     "topology keyword "
                                     "\"element_nodes_short\".\n");
        }
        for (int j = 1; j < nn.numLayers - 2; ++j)
        {
            nn.neurons[j] = std::atoi(a.at(j).c_str());
        }
    }
    for (auto const& v : settings.values("element_activation_short"))
    {
        std::vector<std::string> a = splitWords(v.first);
        NeuralNet& nn = elements.at(elementIndex(a.at(0))).nn;
        if (nn.numLayers != (int)a.size() - 1 + 1)
        {
            throw std::runtime_error("ERROR: Inconsistent per-element NN "
                                     "topology keyword "
                                     "\"element_activation_short\".\n");
        }
        for (int j = 1; j < nn.numLayers - 1; ++j)
        {
            nn.activations[j] = activationFromLetter(a.at(j));
        }
    }
    for (int e = 0; e < ne; ++e)
    {
        NeuralNet const& nn = elements[e].nn;
        for (int j = 0; j < nn.numLayers; ++j)
        {
            if (nn.neurons[j] == 0 || nn.activations[j] < 0)
            {
                throw std::runtime_error("ERROR: Neural network topology of "
                                         "element " + elements[e].symbol
                                         + " is incomplete.\n");
            }
        }
    }
}

// SymGrp*::setScalingFactors: the angular factorNorm carries the scaling
// factor; recomputed on the device-table side from SymFnc::scalingFactor.
void Potential::setGroupScaling()
{
    hasScaling = true;
}

void Potential::setupSymmetryFunctionScalingNone()
{
    scalingType = ST_NONE;
    for (auto& el : elements)
    {
        for (auto& s : el.sfs)
        {
            s.scalingType = ST_NONE;
            s.Gmin = s.Gmax = s.Gmean = s.Gsigma = 0.0;
            s.Smin = s.Smax = 0.0;
            s.scalingFactor = 1.0;
        }
    }
    setGroupScaling();
}

// Mode::setupSymmetryFunctionScaling (libnnp/Mode.cpp:712-840) and
// SymFnc::setScalingType (libnnp/SymFnc.cpp:34-75).
void Potential::setupSymmetryFunctionScaling(std::string const& fileName)
{
    bool const sc = settings.exists("scale_symmetry_functions");
    bool const ce = settings.exists("center_symmetry_functions");
    if (sc && !ce)                 scalingType = ST_SCALE;
    else if (!sc && ce)            scalingType = ST_CENTER;
    else if (sc && ce)             scalingType = ST_SCALECENTER;
    else if (settings.exists("scale_symmetry_functions_sigma"))
                                   scalingType = ST_SCALESIGMA;
    else                           scalingType = ST_NONE;

    double Smin = 0.0, Smax = 0.0;
    if (scalingType == ST_SCALE || scalingType == ST_SCALECENTER
        || scalingType == ST_SCALESIGMA)
    {
        Smin = settings.exists("scale_min_short")
             ? std::atof(settings.value("scale_min_short").c_str()) : 0.0;
        Smax = settings.exists("scale_max_short")
             ? std::atof(settings.value("scale_max_short").c_str()) : 1.0;
    }

    std::ifstream f(fileName);
    if (!f.is_open())
    {
        throw std::runtime_error("ERROR: Could not open file: \"" + fileName
                                 + "\".\n");
    }
    std::vector<std::string> lines;
    std::string line;
    while (std::getline(f, line))
    {
        if (line.empty())
        {
            throw std::runtime_error("ERROR: Empty line in scaling file.\n");
        }
        if (line[0] != '#') lines.push_back(line);
    }
    std::size_t pos = 0;
    for (auto& el : elements)
    {
        for (auto& s : el.sfs)
        {
            if (pos >= lines.size())
            {
                throw std::runtime_error("ERROR: Scaling file has too few "
                                         "lines.\n");
            }
            std::vector<std::string> w = splitWords(lines[pos++]);
            if (w.size() < 5)
            {
                throw std::runtime_error("ERROR: Malformed scaling line.\n");
            }
            if ((std::size_t)std::atoi(w[0].c_str()) != (std::size_t)s.ec + 1
                && (std::size_t)std::atoi(w[1].c_str())
                   != (std::size_t)s.index + 1)
            {
                throw std::runtime_error("ERROR: Inconsistent scaling "
                                         "statistics.\n");
            }
            s.scalingType = scalingType;
            s.Gmin = std::atof(w[2].c_str());
            s.Gmax = std::atof(w[3].c_str());
            s.Gmean = std::atof(w[4].c_str());
            if (w.size() > 5) s.Gsigma = std::atof(w[5].c_str());
            s.Smin = Smin;
            s.Smax = Smax;
            if (scalingType == ST_NONE || scalingType == ST_CENTER)
                s.scalingFactor = 1.0;
            else if (scalingType == ST_SCALE || scalingType == ST_SCALECENTER)
                s.scalingFactor = (Smax - Smin) / (s.Gmax - s.Gmin);
            else
                s.scalingFactor = (Smax - Smin) / s.Gsigma;
        }
    }
    setGroupScaling();
}

// Mode::readNeuralNetworkWeights (libnnp/Mode.cpp:2270-2289).
void Potential::setupNeuralNetworkWeights(std::string const& format)
{
    for (auto& el : elements)
    {
        char buf[4096];
        std::snprintf(buf, sizeof(buf), format.c_str(),
                      (std::size_t)el.atomicNumber);
        el.nn.setConnections(readFirstColumn(buf));
    }
}

} // namespace n2p2b
