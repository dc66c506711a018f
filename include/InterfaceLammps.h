// Drop-in header for LAMMPS's pair_style hdnnp: the reference's
// src/libnnpif/LAMMPS/InterfaceLammps.h by name, class and member, so that
// the pair style (src/interface/LAMMPS/src/ML-HDNNP/pair_hdnnp.{h,cpp})
// compiles UNCHANGED against this library:
//
//   pair_hdnnp.h:32-34    namespace nnp { class InterfaceLammps; }
//   pair_hdnnp.cpp:34     #include "InterfaceLammps.h"
//   pair_hdnnp.cpp:67     new nnp::InterfaceLammps()
//   pair_hdnnp.cpp:235    interface->log.registerCFilePointer(&(lmp->screen))
//   pair_hdnnp.cpp:81-120, 230-364  the call set of n2p2b::InterfaceLammps
//
// nnp::InterfaceLammps is n2p2b::InterfaceLammps (include/n2p2_b200.hpp:
// every evaluation on the GPU through the C-ABI) plus the public `log`
// member of nnp::Mode (libnnp/Mode.h), an nnp::Log that writes its entries
// to the registered C file pointers (libnnp/Log.h: registerCFilePointer,
// writeToStdout, silent).
//
// Device: CUDA device 0, or the one named by the environment variable
// N2P2B_DEVICE (the reference's default constructor takes no arguments;
// one LAMMPS rank per GPU usually selects its GPU through
// CUDA_VISIBLE_DEVICES instead).
#ifndef N2P2_B200_INTERFACE_LAMMPS_H
#define N2P2_B200_INTERFACE_LAMMPS_H

#include "n2p2_b200.hpp"

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

namespace nnp
{

// The subset of nnp::Log (libnnp/Log.h) that its users touch: entries are
// kept in memory and copied to stdout (writeToStdout) and to every
// registered C file pointer / output stream; `silent` drops them.
class Log
{
public:
    bool writeToStdout = true;
    bool silent = false;

    Log& operator<<(std::string const& entry)
    {
        add(entry);
        return *this;
    }
    Log& operator<<(std::vector<std::string> const& entries)
    {
        for (std::string const& e : entries) add(e);
        return *this;
    }
    // The pointer is stored (not the FILE*): LAMMPS may reopen the file.
    void registerCFilePointer(FILE** const& filePointer)
    {
        cFiles_.push_back(filePointer);
    }
    void registerStreamPointer(std::ofstream* const& streamPointer)
    {
        streams_.push_back(streamPointer);
    }
    std::vector<std::string> getLog() const { return memory_; }

private:
    void add(std::string const& entry)
    {
        if (silent) return;
        memory_.push_back(entry);
        if (writeToStdout)
        {
            std::fputs(entry.c_str(), stdout);
            std::fflush(stdout);
        }
        for (FILE** f : cFiles_)
            if (f && *f)
            {
                std::fputs(entry.c_str(), *f);
                std::fflush(*f);
            }
        for (std::ofstream* s : streams_)
            if (s && s->is_open())
            {
                (*s) << entry;
                s->flush();
            }
    }

    std::vector<std::string>  memory_;
    std::vector<FILE**>       cFiles_;
    std::vector<std::ofstream*> streams_;
};

class InterfaceLammps : public n2p2b::InterfaceLammps
{
public:
    InterfaceLammps() : n2p2b::InterfaceLammps(deviceFromEnvironment()) {}

    // InterfaceLammps::initialize (libnnpif/LAMMPS/InterfaceLammps.cpp:
    // 51-255), with a short setup record written through `log` (the
    // reference writes its full setup protocol there).
    void initialize(char const* const& directory, char const* const& emap,
                    bool showew, bool resetew, int showewsum, int maxew,
                    double cflength, double cfenergy, double lammpsCutoff,
                    int lammpsNtypes, int myRank)
    {
        n2p2b::InterfaceLammps::initialize(directory, emap, showew, resetew,
                                           showewsum, maxew, cflength,
                                           cfenergy, lammpsCutoff,
                                           lammpsNtypes, myRank);
        char line[256];
        log << std::string("*** n2p2_b200: HDNNP prediction on the GPU "
                           "(nnp::InterfaceLammps drop-in) ***\n");
        std::snprintf(line, sizeof(line),
                      "Potential directory: %s, rank %d, element map "
                      "\"%s\"\n", directory, myRank, emap);
        log << std::string(line);
        for (std::size_t e = 0; e < numElements(); ++e)
        {
            std::snprintf(line, sizeof(line),
                          "Element %2zu: %-2s, %d symmetry functions\n", e,
                          elementSymbol((int)e).c_str(),
                          n2p2b_num_symmetry_functions(context(), (int)e));
            log << std::string(line);
        }
        std::snprintf(line, sizeof(line),
                      "Maximum symmetry function cutoff: %.6f (LAMMPS "
                      "units), pair_style cutoff %.6f\n",
                      getMaxCutoffRadiusLammps(), lammpsCutoff);
        log << std::string(line);
    }

    // InterfaceLammps::writeExtrapolationWarnings (InterfaceLammps.cpp:
    // 751-765): the recorded warnings' lines through the log.
    void writeExtrapolationWarnings() override
    {
        log << getExtrapolationWarningLines();
    }

    Log log;

private:
    static int deviceFromEnvironment()
    {
        char const* v = std::getenv("N2P2B_DEVICE");
        return v ? std::atoi(v) : 0;
    }
};

} // namespace nnp

#endif
