// nnp-predict: the reference's prediction tool (application/nnp-predict.cpp)
// on the GPU library.  Run in a directory holding input.data, input.nn,
// scaling.data and weights.%03zu.data; writes energy.out, nnatoms.out,
// nnforces.out, output.data and nnp-predict.log with the reference's data
// line formats.
#include "n2p2_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <exception>
#include <string>
#include <vector>

namespace
{

// Comment header in the layout of createFileHeader (libnnp/utility.cpp:
// 111-200): separator, title, column table, separator, column names.
void header(std::FILE* f, char const* title,
            std::vector<std::pair<int, std::pair<char const*, char const*>>>
                const& cols)
{
    std::string const sep(80, '#');
    std::fprintf(f, "%s\n# %s\n%s\n", sep.c_str(), title, sep.c_str());
    std::size_t w = 4;
    for (auto const& c : cols) w = std::max(w, std::string(c.second.first)
                                                   .size());
    std::fprintf(f, "# %-4s %-*s Description\n", "Col", (int)w, "Name");
    std::fprintf(f, "%s\n", sep.c_str());
    for (std::size_t i = 0; i < cols.size(); ++i)
        std::fprintf(f, "# %-4zu %-*s %s\n", i + 1, (int)w,
                     cols[i].second.first, cols[i].second.second);
    std::fprintf(f, "%s\n#", sep.c_str());
    for (auto const& c : cols)
        std::fprintf(f, " %*s", c.first - 1, c.second.first);
    std::fprintf(f, "\n%s\n", sep.c_str());
}

} // namespace

int main(int argc, char* argv[])
{
    if (argc != 2)
    {
        std::printf("USAGE: %s <info>\n"
                    "       <info> ... Write structure information for "
                    "debugging to \"structure.out (0/1)\" (not written by "
                    "this implementation).\n"
                    "       Execute in directory with these NNP files "
                    "present:\n"
                    "       - input.data (structure file)\n"
                    "       - input.nn (NNP settings)\n"
                    "       - scaling.data (symmetry function scaling data)\n"
                    "       - \"weights.%%03d.data\" (weights files)\n",
                    argv[0]);
        return 1;
    }
    std::FILE* log = std::fopen("nnp-predict.log", "w");
    try
    {
        int device = 0;
        if (char const* d = std::getenv("N2P2B_DEVICE")) device = std::atoi(d);
        n2p2b::Prediction p(device);
        p.setup();
        p.readStructureFromFile("input.data");
        n2p2b::Structure& s = p.structure;
        if (log)
            std::fprintf(log, "Structure contains %zu atoms.\n",
                         s.numAtoms());
        p.predict();
        double const offset = p.getEnergyOffset(s);
        if (log)
        {
            std::fprintf(log, "NNP         total energy: %16.8E\n", s.energy);
            std::fprintf(log, "\nNNP forces:\n");
            for (std::size_t i = 0; i < s.numAtoms(); ++i)
                std::fprintf(log, "%10zu %2s %16.8E %16.8E %16.8E\n", i + 1,
                             s.symbol[i].c_str(), s.f[3 * i],
                             s.f[3 * i + 1], s.f[3 * i + 2]);
        }
        std::FILE* f = std::fopen("energy.out", "w");
        header(f, "Energy comparison.",
               {{10, {"conf", "Configuration index (starting with 1)."}},
                {10, {"natoms", "Number of atoms in configuration."}},
                {24, {"Eref", "Reference potential energy."}},
                {24, {"Ennp", "Potential energy predicted by NNP."}},
                {24, {"Ediff", "Difference in energy per atom between "
                               "reference and NNP prediction."}},
                {24, {"E_offset", "Sum of atomic offset energies (included "
                                  "in column Ennp)."}}});
        std::fprintf(f, "%10zu %10zu %24.16E %24.16E %24.16E %24.16E\n",
                     s.index + 1, s.numAtoms(), s.energyRef, s.energy,
                     (s.energyRef - s.energy) / (double)s.numAtoms(), offset);
        std::fclose(f);
        f = std::fopen("nnatoms.out", "w");
        header(f, "Energy contributions calculated from NNP.",
               {{10, {"conf", "Configuration index (starting with 1)."}},
                {10, {"index", "Atom index (starting with 1)."}},
                {3, {"Z", "Nuclear charge of atom."}},
                {24, {"Qref", "Reference atomic charge."}},
                {24, {"Qnnp", "NNP atomic charge."}},
                {24, {"Eref_atom", "Reference atomic energy contribution."}},
                {24, {"Ennp_atom", "Atomic energy contribution (physical "
                                   "units, no mean or offset energy "
                                   "added)."}}});
        for (std::size_t i = 0; i < s.numAtoms(); ++i)
            std::fprintf(f, "%10zu %10zu %3d %24.16E %24.16E %24.16E "
                            "%24.16E\n",
                         s.index + 1, i + 1, p.atomicNumber(s.element[i]),
                         s.chargeRef[i], 0.0, 0.0, s.atomEnergy[i]);
        std::fclose(f);
        f = std::fopen("nnforces.out", "w");
        header(f, "Atomic force comparison (ordered by atom index).",
               {{10, {"conf", "Configuration index (starting with 1)."}},
                {10, {"index", "Atom index (starting with 1)."}},
                {24, {"fxRef", "Reference force in x direction."}},
                {24, {"fyRef", "Reference force in y direction."}},
                {24, {"fzRef", "Reference force in z direction."}},
                {24, {"fx", "Force in x direction."}},
                {24, {"fy", "Force in y direction."}},
                {24, {"fz", "Force in z direction."}}});
        for (std::size_t i = 0; i < s.numAtoms(); ++i)
            std::fprintf(f, "%10zu %10zu %24.16E %24.16E %24.16E %24.16E "
                            "%24.16E %24.16E\n",
                         s.index + 1, i + 1, s.fRef[3 * i], s.fRef[3 * i + 1],
                         s.fRef[3 * i + 2], s.f[3 * i], s.f[3 * i + 1],
                         s.f[3 * i + 2]);
        std::fclose(f);
        f = std::fopen("output.data", "w");
        s.writeToFile(f);
        std::fclose(f);
        if (log) std::fprintf(log, "Finished.\n");
    }
    catch (std::exception const& e)
    {
        std::fprintf(stderr, "%s", e.what());
        if (log) std::fprintf(log, "%s", e.what());
        if (log) std::fclose(log);
        return 2;
    }
    if (log) std::fclose(log);
    return 0;
}
