// ORACLE / TEST INFRASTRUCTURE ONLY.
//
// A C-callable driver around the UNMODIFIED reference n2p2 library (libnnp),
// compiled from the reference sources by oracle/Makefile into
// oracle/_ref/libn2p2ref.so.  Only the test-suite, the smoke check and the
// CPU-baseline leg of bench.py load it; the product never does.
//
// Every entry point calls the reference's own public API in the order its own
// tools use it:
//   - setup:        Prediction::setup                 (libnnp/Prediction.cpp:34-46)
//   - structure:    Structure::readFromLines + remap  (libnnp/Structure.cpp:142-271)
//                   then removeEnergyOffset / toNormalizedUnits
//                   (libnnp/Prediction.cpp:48-63)
//   - evaluation:   Mode::evaluateNNP                 (libnnp/Mode.cpp:1967-2016)
//   - physical:     toPhysicalUnits + addEnergyOffset (libnnp/Prediction.cpp:65-76)
// The structure is handed to the reference as input.data text lines printed
// with 17 significant digits, which round-trips every double exactly, so the
// reference sees bit-identical coordinates.
#include "Prediction.h"
#include "Structure.h"
#include "Atom.h"
#include "SymFnc.h"
#include "SymFncBaseComp.h"
#include "SymFncBaseCompAng.h"
#include "SymFncBaseCompAngWeighted.h"
#include "SymFncBaseExpAng.h"
#include "SymFncCompRad.h"
#include "SymFncCompRadWeighted.h"
#include "SymFncExpAngnWeighted.h"
#include "SymFncExpRad.h"
#include "SymFncExpRadWeighted.h"
#include "utility.h"

#include <chrono>
#include <cstdio>
#include <cstring>
#include <exception>
#include <string>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

using namespace std;
using namespace nnp;

namespace
{

// Subclass only to read the protected setup state that the dumps need.
class OracleModel : public Prediction
{
public:
    bool   isNormalized() const { return normalize; }
    double meanE() const { return meanEnergy; }
    double convE() const { return convEnergy; }
    double convL() const { return convLength; }
    double convQ() const { return convCharge; }
    size_t numSF(size_t e) const { return elements.at(e).numSymmetryFunctions(); }
    size_t numElementsSetup() const { return elements.size(); }
    vector<vector<size_t>> const& sfTable(size_t e) const
    {
        return elements.at(e).getSymmetryFunctionTable();
    }
    SymFnc const& symmetryFunction(size_t e, size_t s) const
    {
        return elements.at(e).getSymmetryFunction(s);
    }
    void setupUnscaled()
    {
        initialize();
        loadSettingsFile(fileNameSettings);
        setupGeneric();
        setupSymmetryFunctionScalingNone();
    }
};

struct Handle
{
    OracleModel         model;
    vector<string>      lines;   // input.data lines of the loaded structure
    string              error;
    bool                unscaled = false;
};

string fmtLines(Handle& h, int n, double const* box9, double const* pos,
                int const* elem)
{
    vector<string>& L = h.lines;
    L.clear();
    L.push_back("begin");
    if (box9 != nullptr)
    {
        for (int k = 0; k < 3; ++k)
        {
            L.push_back(strpr("lattice %24.16E %24.16E %24.16E",
                              box9[3 * k + 0], box9[3 * k + 1],
                              box9[3 * k + 2]));
        }
    }
    for (int i = 0; i < n; ++i)
    {
        string sym = h.model.elementMap[(size_t)elem[i]];
        L.push_back(strpr("atom %24.16E %24.16E %24.16E %s 0.0 0.0 0.0 0.0 0.0",
                          pos[3 * i + 0], pos[3 * i + 1], pos[3 * i + 2],
                          sym.c_str()));
    }
    L.push_back("energy 0.0");
    L.push_back("charge 0.0");
    L.push_back("end");
    return "";
}

// Prediction::readStructureFromFile, but from the stored lines.
void readStructure(Handle& h)
{
    OracleModel& m = h.model;
    m.structure.reset();
    m.structure.setElementMap(m.elementMap);
    m.structure.readFromLines(h.lines);
    if (!h.unscaled)
    {
        m.removeEnergyOffset(m.structure);
        if (m.isNormalized())
        {
            m.structure.toNormalizedUnits(m.meanE(), m.convE(), m.convL(),
                                          m.convQ());
        }
    }
}

} // namespace

extern "C"
{

void* refh_create(char const* dir, int unscaled)
{
    Handle* h = new Handle();
    try
    {
        string d(dir);
        if (!d.empty() && d.back() != '/') d += "/";
        h->model.log.writeToStdout = false;
        h->model.fileNameSettings = d + "input.nn";
        h->model.fileNameScaling = d + "scaling.data";
        h->model.formatWeightsFilesShort = d + "weights.%03zu.data";
        h->model.formatWeightsFilesCharge = d + "weightse.%03zu.data";
        h->unscaled = (unscaled != 0);
        if (h->unscaled) h->model.setupUnscaled();
        else             h->model.setup();
        // The reference logs its low-neighbor-count warning from inside the
        // OpenMP loop over atoms (Mode::calculateSymmetryFunctionGroups,
        // libnnp/Mode.cpp:1598-1609), and Log::addLogEntry appends to a
        // shared std::vector (libnnp/Log.cpp): several threads warning at
        // once (a small open molecule, e.g. DMABN_SCAN) corrupt the heap.
        // A silent log stores nothing; the numbers are unaffected.
        h->model.log.silent = true;
    }
    catch (exception const& e)
    {
        fprintf(stderr, "refh_create: %s\n", e.what());
        delete h;
        return nullptr;
    }
    return h;
}

void refh_destroy(void* p) { delete static_cast<Handle*>(p); }

int refh_num_elements(void* p)
{
    return (int)static_cast<Handle*>(p)->model.numElementsSetup();
}

int refh_num_sf(void* p, int e)
{
    return (int)static_cast<Handle*>(p)->model.numSF((size_t)e);
}

// Number of dG/dr slots per neighbor of element ne for a central atom of
// element e (Element::setupSymmetryFunctionMemory, libnnp/Element.cpp:289-311).
int refh_num_slots(void* p, int e, int ne)
{
    return (int)static_cast<Handle*>(p)->model.sfTable((size_t)e)
           .at((size_t)ne).size();
}

double refh_max_cutoff(void* p)
{
    return static_cast<Handle*>(p)->model.getMaxCutoffRadius();
}

// Element::getSymmetryFunction(s) parameters: type, e1, e2 (-1 radial), eta,
// rs, rc, zeta, lambda, scaling factor, line number.
int refh_sf_params(void* p, int e, int s, double* out)
{
    Handle* h = static_cast<Handle*>(p);
    SymFnc const& f = h->model.symmetryFunction((size_t)e, (size_t)s);
    out[0] = (double)f.getType();
    out[5] = f.getRc();
    out[8] = f.getScalingFactor();
    out[9] = (double)f.getLineNumber();
    if (auto r = dynamic_cast<SymFncExpRad const*>(&f))
    {
        out[1] = (double)r->getE1();
        out[2] = -1.0;
        out[3] = r->getEta();
        out[4] = r->getRs();
        out[6] = 0.0;
        out[7] = 0.0;
        return 0;
    }
    if (auto a = dynamic_cast<SymFncBaseExpAng const*>(&f))
    {
        out[1] = (double)a->getE1();
        out[2] = (double)a->getE2();
        out[3] = a->getEta();
        out[4] = a->getRs();
        out[6] = a->getZeta();
        out[7] = a->getLambda();
        return 0;
    }
    if (auto w = dynamic_cast<SymFncExpRadWeighted const*>(&f))
    {
        out[1] = -1.0;
        out[2] = -1.0;
        out[3] = w->getEta();
        out[4] = w->getRs();
        out[6] = 0.0;
        out[7] = 0.0;
        return 0;
    }
    if (auto w = dynamic_cast<SymFncExpAngnWeighted const*>(&f))
    {
        out[1] = -1.0;
        out[2] = -1.0;
        out[3] = w->getEta();
        out[4] = w->getRs();
        out[6] = w->getZeta();
        out[7] = w->getLambda();
        return 0;
    }
    if (auto c = dynamic_cast<SymFncBaseComp const*>(&f))
    {
        // Compact types: rl, subtype rank in string order (e, p1, p1a, p2,
        // ...), rc; angles (degrees) for the angular ones.
        std::string const t = c->getSubtype();
        double rank = 0.0;
        if (t.size() >= 2 && t[0] == 'p')
            rank = 2.0 * (t[1] - '0') - 1.0 + (t.size() == 3 ? 1.0 : 0.0);
        out[3] = c->getRl();
        out[4] = rank;
        out[6] = 0.0;
        out[7] = 0.0;
        if (auto r = dynamic_cast<SymFncCompRad const*>(&f))
        {
            out[1] = (double)r->getE1();
            out[2] = -1.0;
            return 0;
        }
        if (auto a = dynamic_cast<SymFncBaseCompAng const*>(&f))
        {
            out[1] = (double)a->getE1();
            out[2] = (double)a->getE2();
            out[6] = a->getAngleLeft();
            out[7] = a->getAngleRight();
            return 0;
        }
        if (dynamic_cast<SymFncCompRadWeighted const*>(&f))
        {
            out[1] = -1.0;
            out[2] = -1.0;
            return 0;
        }
        if (auto a = dynamic_cast<SymFncBaseCompAngWeighted const*>(&f))
        {
            out[1] = -1.0;
            out[2] = -1.0;
            out[6] = a->getAngleLeft();
            out[7] = a->getAngleRight();
            return 0;
        }
    }
    return -1;
}

int refh_set_structure(void* p, int n, double const* box9, double const* pos,
                       int const* elem)
{
    Handle* h = static_cast<Handle*>(p);
    try
    {
        fmtLines(*h, n, box9, pos, elem);
        readStructure(*h);
    }
    catch (exception const& e)
    {
        fprintf(stderr, "refh_set_structure: %s\n", e.what());
        return -1;
    }
    return 0;
}

// Mode::evaluateNNP on the loaded structure, left in normalized units so that
// the intermediate dumps below compare against device buffers directly.
int refh_evaluate(void* p, int forces)
{
    Handle* h = static_cast<Handle*>(p);
    try
    {
        readStructure(*h);
        if (h->unscaled)
        {
            Structure& s = h->model.structure;
            s.calculateNeighborList(h->model.getMaxCutoffRadius(), false);
            h->model.calculateSymmetryFunctionGroups(s, forces != 0);
        }
        else
        {
            h->model.evaluateNNP(h->model.structure, forces != 0);
        }
    }
    catch (exception const& e)
    {
        fprintf(stderr, "refh_evaluate: %s\n", e.what());
        return -1;
    }
    return 0;
}

// Prediction::predict after refh_evaluate: physical units + energy offsets.
int refh_to_physical(void* p)
{
    Handle* h = static_cast<Handle*>(p);
    OracleModel& m = h->model;
    if (m.isNormalized())
    {
        m.structure.toPhysicalUnits(m.meanE(), m.convE(), m.convL(),
                                    m.convQ());
    }
    m.addEnergyOffset(m.structure, false);
    m.addEnergyOffset(m.structure, true);
    return 0;
}

int refh_num_atoms(void* p)
{
    return (int)static_cast<Handle*>(p)->model.structure.numAtoms;
}

double refh_energy(void* p)
{
    return static_cast<Handle*>(p)->model.structure.energy;
}

void refh_positions(void* p, double* out)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i)
        for (size_t k = 0; k < 3; ++k) out[3 * i + k] = s.atoms[i].r[k];
}

void refh_forces(void* p, double* out)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i)
        for (size_t k = 0; k < 3; ++k) out[3 * i + k] = s.atoms[i].f[k];
}

void refh_atomic_energies(void* p, double* out)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i) out[i] = s.atoms[i].energy;
}

void refh_neighbor_counts(void* p, long long* out)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i)
        out[i] = (long long)s.atoms[i].numNeighbors;
}

// Neighbor lists concatenated atom by atom in the reference's list order.
void refh_neighbors(void* p, long long* idx, double* dr, double* d)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    size_t e = 0;
    for (size_t i = 0; i < s.numAtoms; ++i)
    {
        for (auto const& n : s.atoms[i].neighbors)
        {
            idx[e] = (long long)n.index;
            for (size_t k = 0; k < 3; ++k) dr[3 * e + k] = n.dr[k];
            d[e] = n.d;
            ++e;
        }
    }
}

// G (as the NN sees it, i.e. scaled unless the handle is unscaled) and dE/dG,
// row-major [atom][sf] with row length `stride`.
void refh_G(void* p, double* out, int stride)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i)
        for (size_t k = 0; k < s.atoms[i].G.size(); ++k)
            out[i * stride + k] = s.atoms[i].G[k];
}

void refh_dEdG(void* p, double* out, int stride)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i)
        for (size_t k = 0; k < s.atoms[i].dEdG.size(); ++k)
            out[i * stride + k] = s.atoms[i].dEdG[k];
}

// Self derivatives dG_s/dr_i, [atom][sf][3] with `stride` SFs per atom.
void refh_dGdr_self(void* p, double* out, int stride)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    for (size_t i = 0; i < s.numAtoms; ++i)
        for (size_t k = 0; k < s.atoms[i].dGdr.size(); ++k)
            for (size_t c = 0; c < 3; ++c)
                out[(i * stride + k) * 3 + c] = s.atoms[i].dGdr[k][c];
}

// Neighbor-slot derivatives, [entry][slot][3] with `stride` slots per entry,
// entries in refh_neighbors order.
void refh_dGdr_nbr(void* p, double* out, int stride)
{
    Structure const& s = static_cast<Handle*>(p)->model.structure;
    size_t e = 0;
    for (size_t i = 0; i < s.numAtoms; ++i)
    {
        for (auto const& n : s.atoms[i].neighbors)
        {
            for (size_t k = 0; k < n.dGdr.size(); ++k)
                for (size_t c = 0; c < 3; ++c)
                    out[(e * stride + k) * 3 + c] = n.dGdr[k][c];
            ++e;
        }
    }
}

// Times the reference's prediction stages on the loaded structure with
// `threads` OpenMP threads (0 = library default), `reps` repetitions.
// Structure parsing is outside the timed region.  t_out[0..4] receive the
// summed seconds of: neighbor list, symmetry functions, atomic NNs, energy,
// forces (the calls Mode::evaluateNNP makes, libnnp/Mode.cpp:1967-2016).
int refh_time_stages(void* p, int threads, int reps, double* t_out)
{
    Handle* h = static_cast<Handle*>(p);
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    for (int k = 0; k < 5; ++k) t_out[k] = 0.0;
    try
    {
        for (int r = 0; r < reps; ++r)
        {
            readStructure(*h);
            Structure& s = h->model.structure;
            OracleModel& m = h->model;
            auto t0 = chrono::steady_clock::now();
            s.calculateNeighborList(m.getMaxCutoffRadius(), false);
            auto t1 = chrono::steady_clock::now();
            m.calculateSymmetryFunctionGroups(s, true);
            auto t2 = chrono::steady_clock::now();
            m.calculateAtomicNeuralNetworks(s, true);
            auto t3 = chrono::steady_clock::now();
            m.calculateEnergy(s);
            auto t4 = chrono::steady_clock::now();
            m.calculateForces(s);
            auto t5 = chrono::steady_clock::now();
            t_out[0] += chrono::duration<double>(t1 - t0).count();
            t_out[1] += chrono::duration<double>(t2 - t1).count();
            t_out[2] += chrono::duration<double>(t3 - t2).count();
            t_out[3] += chrono::duration<double>(t4 - t3).count();
            t_out[4] += chrono::duration<double>(t5 - t4).count();
        }
    }
    catch (exception const& e)
    {
        fprintf(stderr, "refh_time_stages: %s\n", e.what());
        return -1;
    }
    return 0;
}

// Mode::setupSymmetryFunctionStatistics (libnnp/Mode.cpp:1103-1137).
int refh_setup_statistics(void* p, int collect_statistics, int collect_ew,
                          int write_ew, int stop_on_ew)
{
    Handle* h = static_cast<Handle*>(p);
    h->model.setupSymmetryFunctionStatistics(collect_statistics != 0,
                                             collect_ew != 0, write_ew != 0,
                                             stop_on_ew != 0);
    return 0;
}

// Mode::getNumExtrapolationWarnings (libnnp/Mode.cpp:2166-2178).
long refh_num_extrapolation_warnings(void* p)
{
    return (long)static_cast<Handle*>(p)->model.getNumExtrapolationWarnings();
}

void refh_reset_extrapolation_warnings(void* p)
{
    static_cast<Handle*>(p)->model.resetExtrapolationWarnings();
}

int refh_max_threads()
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"
