/*
 * n2p2_b200.hpp -- C++ interface over the C-ABI of n2p2_b200.h, shaped like
 * the reference's own C++ classes so that existing callers change little:
 *
 *   n2p2b::Prediction      nnp::Prediction   (libnnp/Prediction.h:27-40)
 *   n2p2b::Structure       the fields of nnp::Structure that prediction
 *                          reads and writes (libnnp/Structure.h), with the
 *                          input.data reader/writer (Structure.cpp:142-271,
 *                          1474-1531)
 *   n2p2b::InterfaceLammps nnp::InterfaceLammps
 *                          (libnnpif/LAMMPS/InterfaceLammps.h:27-240)
 *
 * Errors come back as the exception types the reference throws:
 * std::invalid_argument (bad arguments), std::out_of_range (capacity,
 * extrapolation-warning stop), std::runtime_error (everything else).
 * Header-only; link with -ln2p2b200.
 */
#ifndef N2P2_B200_HPP
#define N2P2_B200_HPP

#include "n2p2_b200.h"

#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

namespace n2p2b
{

inline void check(n2p2b_context const* ctx, int rc)
{
    if (rc == N2P2B_OK) return;
    std::string msg = ctx ? n2p2b_last_error(ctx) : "";
    if (msg.empty()) msg = "n2p2_b200 error " + std::to_string(rc);
    if (rc == N2P2B_ERR_ARGUMENT) throw std::invalid_argument(msg);
    if (rc == N2P2B_ERR_CAPACITY || rc == N2P2B_ERR_EXTRAPOLATION)
        throw std::out_of_range(msg);
    throw std::runtime_error(msg);
}

// ---------------------------------------------------------------------------
// Structure (one configuration of input.data)
// ---------------------------------------------------------------------------
struct Structure
{
    std::string              comment;
    bool                     isPeriodic = false;
    double                   box[3][3] = {};
    std::vector<double>      r;          // numAtoms x 3
    std::vector<std::string> symbol;     // per atom, as in input.data
    std::vector<int32_t>     element;    // per atom, potential's index
    std::vector<double>      chargeRef;  // per atom
    std::vector<double>      fRef;       // numAtoms x 3
    std::vector<double>      f;          // numAtoms x 3 (prediction)
    std::vector<double>      atomEnergy; // per atom (prediction, physical,
                                         // no offsets)
    double                   energyRef = 0.0;
    double                   chargeRefTotal = 0.0;
    double                   energy = 0.0;
    std::size_t              index = 0;  // configuration index (0-based)

    std::size_t numAtoms() const { return symbol.size(); }

    // Structure::readFromLines for the configuration `which` (0-based) of
    // an input.data file.  Returns false if the file has fewer.
    bool readFromFile(std::string const& fileName, std::size_t which = 0)
    {
        std::ifstream in(fileName);
        if (!in.is_open())
            throw std::runtime_error("ERROR: Could not open file: \""
                                     + fileName + "\".\n");
        std::string line;
        std::size_t count = 0;
        bool inside = false;
        int nlat = 0;
        while (std::getline(in, line))
        {
            std::istringstream is(line);
            std::string key;
            if (!(is >> key)) continue;
            if (key == "begin")
            {
                inside = (count == which);
                if (inside)
                {
                    *this = Structure();
                    index = which;
                    nlat = 0;
                }
                continue;
            }
            if (key == "end")
            {
                if (inside)
                {
                    if (nlat != 0 && nlat != 3)
                        throw std::runtime_error("ERROR: Invalid number of "
                                                 "lattice vectors.\n");
                    isPeriodic = (nlat == 3);
                    return true;
                }
                ++count;
                continue;
            }
            if (!inside) continue;
            if (key == "comment")
            {
                std::size_t const p = line.find("comment");
                comment = line.substr(p + 7);
                std::size_t const q = comment.find_first_not_of(" \t");
                comment = q == std::string::npos ? "" : comment.substr(q);
            }
            else if (key == "lattice")
            {
                if (nlat >= 3)
                    throw std::runtime_error("ERROR: Too many lattice "
                                             "vectors.\n");
                is >> box[nlat][0] >> box[nlat][1] >> box[nlat][2];
                ++nlat;
            }
            else if (key == "atom")
            {
                double x, y, z, q, nn, fx, fy, fz;
                std::string sym;
                if (!(is >> x >> y >> z >> sym >> q >> nn >> fx >> fy >> fz))
                    throw std::runtime_error("ERROR: Bad atom line.\n");
                r.insert(r.end(), {x, y, z});
                symbol.push_back(sym);
                chargeRef.push_back(q);
                fRef.insert(fRef.end(), {fx, fy, fz});
            }
            else if (key == "energy") is >> energyRef;
            else if (key == "charge") is >> chargeRefTotal;
        }
        return false;
    }

    // Structure::writeToFile(file, false) (libnnp/Structure.cpp:1474-1531).
    void writeToFile(std::FILE* f) const
    {
        std::fprintf(f, "begin\ncomment %s\n", comment.c_str());
        if (isPeriodic)
            for (int i = 0; i < 3; ++i)
                std::fprintf(f, "lattice %24.16E %24.16E %24.16E\n",
                             box[i][0], box[i][1], box[i][2]);
        for (std::size_t i = 0; i < numAtoms(); ++i)
            std::fprintf(f, "atom %24.16E %24.16E %24.16E %2s %24.16E "
                            "%24.16E %24.16E %24.16E %24.16E\n",
                         r[3 * i], r[3 * i + 1], r[3 * i + 2],
                         symbol[i].c_str(), 0.0, 0.0, f_(i, 0), f_(i, 1),
                         f_(i, 2));
        std::fprintf(f, "energy %24.16E\ncharge %24.16E\nend\n", energy, 0.0);
    }

private:
    double f_(std::size_t i, int c) const
    {
        return f.empty() ? 0.0 : f[3 * i + c];
    }
};

// ---------------------------------------------------------------------------
// Mode / Prediction
// ---------------------------------------------------------------------------
class Mode
{
public:
    explicit Mode(int device = 0)
    {
        check(nullptr, n2p2b_create(device, &ctx_));
    }
    ~Mode()
    {
        if (ctx_) n2p2b_destroy(ctx_);
    }
    Mode(Mode const&) = delete;
    Mode& operator=(Mode const&) = delete;

    n2p2b_context* context() const { return ctx_; }

    void loadSettingsFile(std::string const& fileName = "input.nn")
    {
        check(ctx_, n2p2b_load_settings_file(ctx_, fileName.c_str()));
    }
    void setupGeneric() { check(ctx_, n2p2b_setup_generic(ctx_)); }
    void setupSymmetryFunctionScaling(std::string const& f = "scaling.data")
    {
        check(ctx_, n2p2b_setup_symmetry_function_scaling(ctx_, f.c_str()));
    }
    void setupNeuralNetworkWeights(std::string const& format
                                   = "weights.%03zu.data")
    {
        check(ctx_, n2p2b_setup_neural_network_weights(ctx_,
                                                        format.c_str()));
    }
    // The reference's form with one file-name format per network type
    // (libnnp/Mode.h): a 2G potential reads the "short" networks only.
    void setupNeuralNetworkWeights(
        std::map<std::string, std::string> const& formats)
    {
        auto const it = formats.find("short");
        setupNeuralNetworkWeights(it != formats.end() ? it->second
                                                      : "weights.%03zu.data");
    }
    void setupSymmetryFunctionStatistics(bool collectStatistics,
                                         bool collectExtrapolationWarnings,
                                         bool writeExtrapolationWarnings,
                                         bool stopOnExtrapolationWarnings)
    {
        check(ctx_, n2p2b_setup_symmetry_function_statistics(
                        ctx_, collectStatistics, collectExtrapolationWarnings,
                        writeExtrapolationWarnings,
                        stopOnExtrapolationWarnings));
    }
    std::size_t getNumExtrapolationWarnings() const
    {
        return (std::size_t)n2p2b_get_num_extrapolation_warnings(ctx_);
    }
    void resetExtrapolationWarnings()
    {
        check(ctx_, n2p2b_reset_extrapolation_warnings(ctx_));
    }
    double getMaxCutoffRadius() const
    {
        return n2p2b_max_cutoff_radius(ctx_);
    }
    std::size_t numElements() const
    {
        return (std::size_t)n2p2b_num_elements(ctx_);
    }
    std::string elementSymbol(int e) const
    {
        char buf[8];
        check(ctx_, n2p2b_element_symbol(ctx_, e, buf, sizeof(buf)));
        return buf;
    }
    int elementIndex(std::string const& symbol) const
    {
        return n2p2b_element_index(ctx_, symbol.c_str());
    }
    double atomicEnergyOffset(int e) const
    {
        return n2p2b_atomic_energy_offset(ctx_, e);
    }
    int atomicNumber(int e) const { return n2p2b_atomic_number(ctx_, e); }
    void setPrecision(int mode) { check(ctx_, n2p2b_set_precision(ctx_,
                                                                  mode)); }

    // Mode::initialize (libnnp/Mode.cpp:55) only writes the reference's
    // banner to its log; a context needs no such step.
    void initialize() {}
    // Mode::setupSymmetryFunctionGroups: setupGeneric builds the groups (as
    // the reference's setupGeneric does, libnnp/Mode.cpp:231), so a call
    // after it has nothing left to do.
    void setupSymmetryFunctionGroups() {}

    // Mode::evaluateNNP on a structure (its element indices are resolved
    // from the symbols), followed by Prediction::predict's unit conversion
    // and offsets; fills energy, f and atomEnergy.
    void evaluate(Structure& s, bool remap = true)
    {
        upload(s, remap);
        check(ctx_, n2p2b_evaluate(ctx_, 1));
        fetchAtomicEnergies(s);
        fetchEnergy(s);
        fetchForces(s);
    }

    // The evaluation steps of nnp::Mode (libnnp/Mode.h) on a structure.  The
    // reference's callers build the neighbor list first
    // (Structure::calculateNeighborList); calculateSymmetryFunctionGroups
    // uploads the structure and builds it.  Each step leaves its result in
    // the structure in the units Prediction::predict leaves there (physical
    // units; the energy with the atoms' offset energies).
    void calculateSymmetryFunctionGroups(Structure& s, bool derivatives,
                                         bool remap = true)
    {
        upload(s, remap);
        check(ctx_, n2p2b_calculate_neighbor_list(ctx_));
        check(ctx_, n2p2b_calculate_symmetry_function_groups(ctx_,
                                                             derivatives));
    }
    // Mode::calculateAtomicNeuralNetworks; id selects the network of a
    // 4G potential in the reference, and a 2G potential has only "short".
    void calculateAtomicNeuralNetworks(Structure& s, bool derivatives,
                                       std::string const& id = "")
    {
        if (!id.empty() && id != "short")
            throw std::invalid_argument("ERROR: Only the short-range network "
                                        "(2G) is available.\n");
        check(ctx_, n2p2b_calculate_atomic_neural_networks(ctx_,
                                                           derivatives));
        fetchAtomicEnergies(s);
    }
    void calculateEnergy(Structure& s) const
    {
        check(ctx_, n2p2b_calculate_energy(ctx_));
        fetchEnergy(s);
    }
    void calculateForces(Structure& s) const
    {
        check(ctx_, n2p2b_calculate_forces(ctx_));
        fetchForces(s);
    }
    // Mode::evaluateNNP (libnnp/Mode.cpp:1967-2016): neighbor list,
    // symmetry functions (derivatives with forces), networks (derivatives
    // with forces or dE/dG), energy, forces.
    void evaluateNNP(Structure& s, bool useForces = true, bool useDEdG = true,
                     bool remap = true)
    {
        useDEdG = useForces || useDEdG;
        if (useDEdG && !useForces)
        {
            calculateSymmetryFunctionGroups(s, false, remap);
            calculateAtomicNeuralNetworks(s, true);
            calculateEnergy(s);
            return;
        }
        upload(s, remap);
        check(ctx_, n2p2b_evaluate(ctx_, useForces ? 1 : 0));
        fetchAtomicEnergies(s);
        fetchEnergy(s);
        if (useForces) fetchForces(s);
    }

    // Mode::getEnergyOffset: sum of the atoms' offset energies.
    double getEnergyOffset(Structure const& s) const
    {
        double e = 0.0;
        for (int32_t el : s.element) e += atomicEnergyOffset(el);
        return e;
    }

protected:
    n2p2b_context* ctx_ = nullptr;

    // Uploads a structure: element indices from the symbols, positions and
    // box (wrapped into the cell with remap, as Structure::remap).
    void upload(Structure& s, bool remap)
    {
        std::size_t const n = s.numAtoms();
        s.element.resize(n);
        for (std::size_t i = 0; i < n; ++i)
        {
            int const e = elementIndex(s.symbol[i]);
            if (e < 0)
                throw std::runtime_error("ERROR: Element \"" + s.symbol[i]
                                         + "\" not in the potential.\n");
            s.element[i] = e;
        }
        check(ctx_, n2p2b_set_structure(ctx_, (int64_t)n,
                                        s.isPeriodic ? &s.box[0][0] : nullptr,
                                        s.r.data(), N2P2B_HOST,
                                        s.element.data(),
                                        remap ? N2P2B_REMAP : 0));
    }
    void fetchAtomicEnergies(Structure& s) const
    {
        s.atomEnergy.resize(s.numAtoms());
        check(ctx_, n2p2b_get_atomic_energies(ctx_, s.atomEnergy.data()));
    }
    void fetchEnergy(Structure& s) const
    {
        check(ctx_, n2p2b_get_energy(ctx_, &s.energy));
    }
    void fetchForces(Structure& s) const
    {
        s.f.resize(3 * s.numAtoms());
        check(ctx_, n2p2b_get_forces(ctx_, s.f.data(), N2P2B_HOST));
    }
};

class Prediction : public Mode
{
public:
    explicit Prediction(int device = 0) : Mode(device) {}

    std::string fileNameSettings = "input.nn";
    std::string fileNameScaling = "scaling.data";
    std::string formatWeightsFilesShort = "weights.%03zu.data";
    std::string formatWeightsFilesCharge = "weightse.%03zu.data"; // 4G only
    Structure   structure;

    // Prediction::setup (libnnp/Prediction.cpp:34-46).
    void setup()
    {
        loadSettingsFile(fileNameSettings);
        setupGeneric();
        setupSymmetryFunctionScaling(fileNameScaling);
        setupNeuralNetworkWeights(formatWeightsFilesShort);
        setupSymmetryFunctionStatistics(false, false, true, false);
    }
    // Prediction::readStructureFromFile (first configuration).
    void readStructureFromFile(std::string const& fileName = "input.data")
    {
        if (!structure.readFromFile(fileName, 0))
            throw std::runtime_error("ERROR: No configuration in \""
                                     + fileName + "\".\n");
    }
    // Prediction::predict (libnnp/Prediction.cpp:65-76).
    void predict() { evaluate(structure, true); }
};

// ---------------------------------------------------------------------------
// InterfaceLammps
// ---------------------------------------------------------------------------
class InterfaceLammps : public Mode
{
public:
    explicit InterfaceLammps(int device = 0) : Mode(device) {}

    // InterfaceLammps::initialize (libnnpif/LAMMPS/InterfaceLammps.cpp:
    // 51-255): potential directory, element map "type:symbol,..." (empty:
    // types 1..n map to the elements in order), extrapolation-warning
    // options, unit conversion factors, LAMMPS cutoff (checked against the
    // largest symmetry-function cutoff), number of LAMMPS types, MPI rank.
    void initialize(char const* const& directory, char const* const& emap,
                    bool showew, bool resetew, int showewsum, int maxew,
                    double cflength, double cfenergy, double lammpsCutoff,
                    int lammpsNtypes, int myRank)
    {
        std::string dir(directory);
        if (!dir.empty() && dir.back() != '/') dir += '/';
        showew_ = showew;
        resetew_ = resetew;
        maxew_ = maxew;
        cflength_ = cflength;
        cfenergy_ = cfenergy;
        myRank_ = myRank;
        (void)showewsum;
        loadSettingsFile(dir + "input.nn");
        setupGeneric();
        setupSymmetryFunctionScaling(dir + "scaling.data");
        // As the reference: warnings are collected (not written while the
        // symmetry functions are computed); writeExtrapolationWarnings
        // writes them.
        setupSymmetryFunctionStatistics(false, showew || showewsum > 0
                                                   || maxew >= 0,
                                        false, false);
        setupNeuralNetworkWeights(dir + "weights.%03zu.data");
        if (lammpsCutoff < getMaxCutoffRadiusLammps())
            throw std::runtime_error("ERROR: LAMMPS cutoff via pair_coeff "
                                     "keyword is smaller than maximum "
                                     "symmetry function cutoff.\n");
        typeToElement_.clear();
        std::string m(emap);
        if (m.empty())
        {
            if ((int)numElements() != lammpsNtypes)
                throw std::runtime_error("ERROR: No element mapping given "
                                         "and number of LAMMPS atom types "
                                         "and NNP elements does not "
                                         "match.\n");
            for (int t = 1; t <= lammpsNtypes; ++t) typeToElement_[t] = t - 1;
        }
        else
        {
            std::stringstream ss(m);
            std::string item;
            while (std::getline(ss, item, ','))
            {
                std::size_t const c = item.find(':');
                if (c == std::string::npos)
                    throw std::runtime_error("ERROR: Invalid element mapping "
                                             "string: \"" + item + "\".\n");
                int const t = std::stoi(item.substr(0, c));
                std::string sym = item.substr(c + 1);
                sym.erase(0, sym.find_first_not_of(" \t"));
                sym.erase(sym.find_last_not_of(" \t") + 1);
                if (t > lammpsNtypes)
                    throw std::runtime_error("ERROR: LAMMPS type not "
                                             "present.\n");
                int const e = elementIndex(sym);
                if (e < 0)
                    throw std::runtime_error("ERROR: Unknown element \"" + sym
                                             + "\".\n");
                typeToElement_[t] = e;
            }
        }
        initialized_ = true;
    }
    bool isInitialized() const { return initialized_; }

    // InterfaceLammps::setLocalAtoms: local atom types (LAMMPS, 1-based);
    // types without an element are ignored.
    void setLocalAtoms(int numAtomsLocal, int const* const atomType)
    {
        nlocal_ = numAtomsLocal;
        localIndex_.assign(numAtomsLocal, -1);
        elements_.clear();
        lammpsIndex_.clear();
        for (int i = 0; i < numAtomsLocal; ++i)
        {
            auto it = typeToElement_.find(atomType[i]);
            // Local atoms are force targets 0 .. n-1 in LAMMPS order, so
            // every local type must map to an element.
            if (it == typeToElement_.end())
                throw std::runtime_error("ERROR: Local atom of a LAMMPS type "
                                         "without an NNP element.\n");
            localIndex_[i] = (int)elements_.size();
            elements_.push_back(it->second);
            lammpsIndex_.push_back(i);
        }
        counts_.assign(elements_.size(), 0);
        index_.clear();
        nelem_.clear();
        dr_.clear();
        pending_.assign(elements_.size(), {});
        maxTarget_ = numAtomsLocal;
        finalized_ = false;
    }
    // InterfaceLammps::setLocalTags (InterfaceLammps.cpp:325-345): the
    // LAMMPS tags of the local atoms, the atom field of the warnings.
    void setLocalTags(int const* const atomTag)
    {
        tags_.assign(atomTag, atomTag + nlocal_);
    }
    void setLocalTags(int64_t const* const atomTag)
    {
        tags_.assign(atomTag, atomTag + nlocal_);
    }
    void allocateNeighborlists(int const* const numneigh)
    {
        for (int i = 0; i < nlocal_; ++i)
            if (localIndex_[i] >= 0)
                pending_[localIndex_[i]].reserve(numneigh[i]);
    }
    // InterfaceLammps::addNeighbor: neighbor j (LAMMPS index, local or
    // ghost) of local atom i, dx = x_i - x_j in LAMMPS units.
    void addNeighbor(int i, int j, int64_t tag, int type, double dx,
                     double dy, double dz, double d2)
    {
        (void)tag;
        (void)d2;
        auto it = typeToElement_.find(type);
        if (it == typeToElement_.end() || localIndex_.at(i) < 0) return;
        pending_[localIndex_[i]].push_back(
            Entry{j, it->second, dx * cflength_, dy * cflength_,
                  dz * cflength_});
        if (j + 1 > maxTarget_) maxTarget_ = j + 1;
        finalized_ = false;
    }
    // InterfaceLammps::finalizeNeighborList (InterfaceLammps.cpp:444-461):
    // the reference needs it only for 4G potentials, and the 2G pair style
    // never calls it (pair_hdnnp.cpp:81-120), so process() runs it itself
    // when neighbors were added since the last call.
    void finalizeNeighborList()
    {
        finalized_ = true;
        index_.clear();
        nelem_.clear();
        dr_.clear();
        for (std::size_t a = 0; a < pending_.size(); ++a)
        {
            counts_[a] = (int64_t)pending_[a].size();
            for (Entry const& e : pending_[a])
            {
                index_.push_back(e.j);
                nelem_.push_back(e.element);
                dr_.insert(dr_.end(), {e.dx, e.dy, e.dz});
            }
            pending_[a].clear();
        }
    }
    // InterfaceLammps::process (libnnpif/LAMMPS/InterfaceLammps.cpp:463-487)
    void process()
    {
        if (!finalized_) finalizeNeighborList();
        if (elements_.empty()) return;
        if (resetew_) resetExtrapolationWarnings();
        check(ctx_, n2p2b_set_neighbor_list(ctx_, (int64_t)elements_.size(),
                                            elements_.data(), counts_.data(),
                                            index_.data(), nelem_.data(),
                                            dr_.data(), maxTarget_));
        check(ctx_, n2p2b_evaluate(ctx_, 1));
        check(ctx_, n2p2b_get_energy(ctx_, &energy_));
        atomEnergy_.resize(elements_.size());
        check(ctx_, n2p2b_get_atomic_energies(ctx_, atomEnergy_.data()));
        forces_.resize(3 * (std::size_t)maxTarget_);
        check(ctx_, n2p2b_get_target_forces(ctx_, forces_.data()));
        if (showew_) collectExtrapolationWarnings();
    }
    double getEnergy() const { return energy_ / cfenergy_; }
    double getAtomicEnergy(int index) const
    {
        double meanE, convE, convL;
        int const norm = n2p2b_unit_conversion(ctx_, &meanE, &convE, &convL);
        return (atomEnergy_.at(index) + (norm ? meanE : 0.0)
                + atomicEnergyOffset(elements_[index])) / cfenergy_;
    }
    // InterfaceLammps::getForces: ADDS into the LAMMPS force array (local
    // and ghost atoms).
    void getForces(double* const* const& atomF) const
    {
        double const cf = cflength_ / cfenergy_;
        for (int m = 0; m < maxTarget_; ++m)
            for (int c = 0; c < 3; ++c)
                atomF[m][c] += forces_[3 * (std::size_t)m + c] * cf;
    }
    // Extrapolation-warning output (InterfaceLammps.cpp:638-776).  process()
    // records this rank's warnings per element and symmetry function (the
    // SymFncStatistics containers, SymFncStatistics.cpp:91-137: type, range,
    // and per warning the structure index, the atom's LAMMPS tag and the
    // value); the pair style moves other ranks' records to rank 0 through
    // the EW buffer (getEWBufferSize / fillEWBuffer / extractEWBuffer, a
    // plain byte layout of the same fields) and has rank 0 write them.
    long getEWBufferSize() const
    {
        long bs = 0;
        for (auto const& m : ewData_)
        {
            bs += 8;
            for (auto const& kv : m)
            {
                EWContainer const& d = kv.second;
                bs += 8 * 3 + 8 * 2 + 8 + (long)d.element.size() + 1;
                bs += (long)d.valueEW.size() * (8 + 8 + 8);
            }
        }
        return bs;
    }
    void fillEWBuffer(char* const& buf, int bs) const
    {
        std::size_t p = 0;
        auto put = [&](void const* v, std::size_t k) {
            if (p + k > (std::size_t)bs)
                throw std::out_of_range("ERROR: EW buffer too small.\n");
            std::memcpy(buf + p, v, k);
            p += k;
        };
        for (auto const& m : ewData_)
        {
            uint64_t const n = m.size();
            put(&n, 8);
            for (auto const& kv : m)
            {
                EWContainer const& d = kv.second;
                uint64_t const h[3] = {kv.first, d.valueEW.size(), d.type};
                put(h, sizeof(h));
                put(&d.gmin, 8);
                put(&d.gmax, 8);
                uint64_t const ts = d.element.size() + 1;
                put(&ts, 8);
                put(d.element.c_str(), ts);
                put(d.structureEW.data(), 8 * d.valueEW.size());
                put(d.atomEW.data(), 8 * d.valueEW.size());
                put(d.valueEW.data(), 8 * d.valueEW.size());
            }
        }
    }
    void extractEWBuffer(char const* const& buf, int bs)
    {
        std::size_t p = 0;
        auto get = [&](void* v, std::size_t k) {
            if (p + k > (std::size_t)bs)
                throw std::out_of_range("ERROR: EW buffer truncated.\n");
            std::memcpy(v, buf + p, k);
            p += k;
        };
        ewData_.resize(numElements());
        for (auto& m : ewData_)
        {
            uint64_t n = 0;
            get(&n, 8);
            for (uint64_t i = 0; i < n; ++i)
            {
                uint64_t h[3];
                get(h, sizeof(h));
                EWContainer& d = m[(std::size_t)h[0]];
                d.type = (std::size_t)h[2];
                get(&d.gmin, 8);
                get(&d.gmax, 8);
                uint64_t ts = 0;
                get(&ts, 8);
                std::string el(ts, '\0');
                get(&el[0], ts);
                d.element = el.c_str();
                std::size_t const c = d.valueEW.size(), k = (std::size_t)h[1];
                d.structureEW.resize(c + k);
                d.atomEW.resize(c + k);
                d.valueEW.resize(c + k);
                get(d.structureEW.data() + c, 8 * k);
                get(d.atomEW.data() + c, 8 * k);
                get(d.valueEW.data() + c, 8 * k);
            }
        }
    }
    // SymFncStatistics::getExtrapolationWarningLines for every element
    // (SymFncStatistics.cpp:112-137): element by element, symmetry function
    // by symmetry function, warnings in the order they were recorded.
    std::vector<std::string> getExtrapolationWarningLines() const
    {
        std::vector<std::string> vs;
        for (auto const& m : ewData_)
            for (auto const& kv : m)
            {
                EWContainer const& d = kv.second;
                for (std::size_t i = 0; i < d.valueEW.size(); ++i)
                {
                    char line[256];
                    std::snprintf(line, sizeof(line),
                                  "### NNP EXTRAPOLATION WARNING ### "
                                  "STRUCTURE: %6zu ATOM: %9zu ELEMENT: %2s "
                                  "SYMFUNC: %4zu TYPE: %2zu VALUE: %10.3E "
                                  "MIN: %10.3E MAX: %10.3E\n",
                                  (std::size_t)d.structureEW[i],
                                  (std::size_t)d.atomEW[i],
                                  d.element.c_str(), kv.first + 1, d.type,
                                  d.valueEW[i], d.gmin, d.gmax);
                    vs.push_back(line);
                }
            }
        return vs;
    }
    // InterfaceLammps::writeExtrapolationWarnings writes to the interface's
    // log; this class has none and writes to stderr (nnp::InterfaceLammps
    // in InterfaceLammps.h writes to its log).
    virtual void writeExtrapolationWarnings()
    {
        for (std::string const& l : getExtrapolationWarningLines())
            std::fputs(l.c_str(), stderr);
    }
    // SymFncStatistics::clear on every element: the records and the count.
    void clearExtrapolationWarnings()
    {
        ewData_.clear();
        resetExtrapolationWarnings();
    }
    virtual ~InterfaceLammps() = default;

    // InterfaceLammps::getMaxCutoffRadius (InterfaceLammps.cpp:489-493):
    // the largest symmetry-function cutoff in LAMMPS units (the pair style
    // checks its own cutoff against it, pair_hdnnp.cpp:245).
    double getMaxCutoffRadius() const { return getMaxCutoffRadiusLammps(); }
    double getMaxCutoffRadiusLammps() const
    {
        double meanE, convE, convL;
        n2p2b_unit_conversion(ctx_, &meanE, &convE, &convL);
        return Mode::getMaxCutoffRadius() / convL / cflength_;
    }

private:
    // The warnings of the last evaluation into the per-element records;
    // the atom field is the atom's LAMMPS tag (its local index + 1 when no
    // tags were set), the structure index 0.
    void collectExtrapolationWarnings()
    {
        int64_t cnt = 0;
        check(ctx_, n2p2b_get_extrapolation_warnings(ctx_, 0, nullptr, &cnt));
        if (cnt == 0) return;
        std::vector<n2p2b_extrapolation_warning> w((std::size_t)cnt);
        check(ctx_, n2p2b_get_extrapolation_warnings(ctx_, cnt, w.data(),
                                                     &cnt));
        ewData_.resize(numElements());
        for (n2p2b_extrapolation_warning const& x : w)
        {
            int const li = lammpsIndex_.at((std::size_t)x.atom);
            int64_t const tag = li < (int)tags_.size() ? tags_[li] : li + 1;
            EWContainer& d = ewData_[x.element][(std::size_t)x.sf];
            d.type = (std::size_t)x.type;
            d.gmin = x.gmin;
            d.gmax = x.gmax;
            d.element = elementSymbol(x.element);
            d.structureEW.push_back(0);
            d.atomEW.push_back((uint64_t)tag);
            d.valueEW.push_back(x.value);
        }
    }

    struct EWContainer
    {
        std::size_t           type = 0;
        double                gmin = 0.0, gmax = 0.0;
        std::string           element;
        std::vector<uint64_t> structureEW, atomEW;
        std::vector<double>   valueEW;
    };
    struct Entry
    {
        int    j;
        int    element;
        double dx, dy, dz;
    };
    std::vector<int64_t>                          tags_;
    std::vector<std::map<std::size_t, EWContainer>> ewData_;
    bool                            initialized_ = false;
    bool                            finalized_ = false;
    bool                            showew_ = false, resetew_ = false;
    int                             maxew_ = 0;  // enforced by the pair
                                                 // style (pair_hdnnp.cpp:
                                                 // 358-361), as for the
                                                 // reference
    double                          cflength_ = 1.0, cfenergy_ = 1.0;
    int                             myRank_ = 0;
    std::map<int, int>              typeToElement_;
    int                             nlocal_ = 0;
    int                             maxTarget_ = 0;
    std::vector<int>                localIndex_, lammpsIndex_;
    std::vector<int32_t>            elements_;
    std::vector<int64_t>            counts_, index_;
    std::vector<int32_t>            nelem_;
    std::vector<double>             dr_;
    std::vector<std::vector<Entry>> pending_;
    double                          energy_ = 0.0;
    std::vector<double>             atomEnergy_, forces_;
};

} // namespace n2p2b

#endif
