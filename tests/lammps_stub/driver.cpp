// TEST INFRASTRUCTURE: runs LAMMPS's pair_style hdnnp -- the reference's
// src/interface/LAMMPS/src/ML-HDNNP/pair_hdnnp.cpp, compiled unchanged
// against include/InterfaceLammps.h (nnp::InterfaceLammps of this library)
// and the single-rank LAMMPS stand-in headers of include/ here -- on one
// periodic structure, the way LAMMPS runs a pair style for one step:
//
//   pair_style hdnnp <cutoff> dir <potential> showew no|yes maxew 1000000000
//                    [cflength <a> cfenergy <b>]
//   pair_coeff * * <element symbols in input.nn order>
//   init_style (neighbor request, interface setup), compute(eflag, vflag)
//
// Atoms: the structure's atoms are the local atoms; every periodic image
// within the cutoff of the cell is a ghost atom; the full neighbor list of
// each local atom holds its local and ghost neighbors within the cutoff.
// After compute, the forces of the ghosts are added to their atoms (LAMMPS's
// reverse communication).  Positions are in LAMMPS units: the potential's
// length unit divided by cflength.
//
//   lammps_pair_hdnnp <potential dir> <input.data> [cflength cfenergy [showew]]
//
// Prints "energy E", "virial v0..v5", and "force i fx fy fz" / "eatom i e"
// per atom (LAMMPS units), plus "requests n flags f" of the neighbor
// request and "log <line>" for each line the interface wrote to the
// registered screen file.  With "showew" the pair style shows individual
// extrapolation warnings (atom tags = index + 1); the interface then runs
// process() once more and moves its warning records through the EW buffer
// (getEWBufferSize, fillEWBuffer, clearExtrapolationWarnings,
// extractEWBuffer), printing the lines it holds afterwards as
// "ewbuf <line>".
#include "pair_hdnnp.h"

#include "atom.h"
#include "citeme.h"
#include "comm.h"
#include "error.h"
#include "memory.h"
#include "neighbor.h"
#include "update.h"
#include "InterfaceLammps.h"
#include "n2p2_b200.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

using namespace LAMMPS_NS;

int main(int argc, char* argv[])
{
    if (argc != 3 && argc != 5 && argc != 6)
    {
        std::fprintf(stderr, "USAGE: %s <potential dir> <input.data> "
                             "[cflength cfenergy [showew]]\n", argv[0]);
        return 1;
    }
    std::string const cfl = argc >= 5 ? argv[3] : "1.0";
    std::string const cfe = argc >= 5 ? argv[4] : "1.0";
    bool const showew = argc == 6 && std::string(argv[5]) == "showew";
    double const cflength = std::atof(cfl.c_str());
    try
    {
        n2p2b::Structure s;
        if (!s.readFromFile(argv[2], 0) || !s.isPeriodic)
            throw std::runtime_error("need one periodic structure");
        std::vector<std::string> syms;
        {
            std::ifstream in(std::string(argv[1]) + "/input.nn");
            std::string line;
            while (std::getline(in, line))
            {
                std::istringstream is(line);
                std::string key, sym;
                if (!(is >> key) || key != "elements") continue;
                while (is >> sym && sym[0] != '#') syms.push_back(sym);
                break;
            }
        }
        int const n = (int)s.numAtoms();
        std::vector<int> type(n);
        for (int i = 0; i < n; ++i)
        {
            type[i] = 0;
            for (std::size_t k = 0; k < syms.size(); ++k)
                if (syms[k] == s.symbol[i]) type[i] = (int)k + 1;
            if (!type[i]) throw std::runtime_error("unknown element");
        }
        // LAMMPS units: lengths / cflength.
        std::vector<double> r(3 * (std::size_t)n);
        double b[3][3];
        for (int i = 0; i < 3 * n; ++i) r[i] = s.r[i] / cflength;
        for (int k = 0; k < 3; ++k)
            for (int c = 0; c < 3; ++c) b[k][c] = s.box[k][c] / cflength;
        // The pair style's cutoff: the potential's largest cutoff (read
        // back after init_style; a generous first guess for the ghosts).
        double const rcut = std::atof(std::getenv("LMP_CUTOFF")
                                      ? std::getenv("LMP_CUTOFF") : "12.0")
                          / cflength;
        double vol, cr[3][3];
        auto cross = [](double const* u, double const* v, double* w) {
            w[0] = u[1] * v[2] - u[2] * v[1];
            w[1] = u[2] * v[0] - u[0] * v[2];
            w[2] = u[0] * v[1] - u[1] * v[0];
        };
        cross(b[1], b[2], cr[0]);
        cross(b[2], b[0], cr[1]);
        cross(b[0], b[1], cr[2]);
        vol = std::fabs(b[0][0] * cr[0][0] + b[0][1] * cr[0][1]
                        + b[0][2] * cr[0][2]);
        int p[3];
        for (int k = 0; k < 3; ++k)
        {
            double const area = std::sqrt(cr[k][0] * cr[k][0]
                                          + cr[k][1] * cr[k][1]
                                          + cr[k][2] * cr[k][2]);
            p[k] = (int)std::ceil(rcut / (vol / area)) + 1;
        }
        std::map<std::tuple<int, int, int, int>, int> ghostOf;
        std::vector<int> owner;
        std::vector<std::vector<double>> gx;
        std::vector<std::vector<int>> nbr(n);
        double const rc2 = rcut * rcut;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int a = -p[0]; a <= p[0]; ++a)
                    for (int bb = -p[1]; bb <= p[1]; ++bb)
                        for (int cc = -p[2]; cc <= p[2]; ++cc)
                        {
                            if (i == j && !a && !bb && !cc) continue;
                            double xj[3], d2 = 0.0;
                            for (int k = 0; k < 3; ++k)
                            {
                                xj[k] = r[3 * j + k] + a * b[0][k]
                                      + bb * b[1][k] + cc * b[2][k];
                                double const d = r[3 * i + k] - xj[k];
                                d2 += d * d;
                            }
                            if (d2 > rc2) continue;
                            int idx = j;
                            if (a || bb || cc)
                            {
                                auto key = std::make_tuple(j, a, bb, cc);
                                auto it = ghostOf.find(key);
                                if (it == ghostOf.end())
                                {
                                    idx = n + (int)owner.size();
                                    ghostOf[key] = idx;
                                    owner.push_back(j);
                                    gx.push_back({xj[0], xj[1], xj[2]});
                                }
                                else idx = it->second;
                            }
                            nbr[i].push_back(idx);
                        }
        int const nall = n + (int)owner.size();

        LAMMPS lmp;
        Atom atom;
        Comm comm;
        Error error;
        Memory memory;
        Neighbor neighbor;
        Update update;
        CiteMe citeme;
        lmp.atom = &atom;
        lmp.comm = &comm;
        lmp.error = &error;
        lmp.memory = &memory;
        lmp.neighbor = &neighbor;
        lmp.update = &update;
        lmp.citeme = &citeme;
        lmp.screen = std::tmpfile();

        std::vector<double> xbuf(3 * (std::size_t)nall), fbuf(3 * (std::size_t)nall, 0.0);
        std::vector<double*> xp(nall), fp(nall);
        std::vector<int> typeAll(nall);
        std::vector<tagint> tag(nall);
        for (int m = 0; m < nall; ++m)
        {
            for (int k = 0; k < 3; ++k)
                xbuf[3 * (std::size_t)m + k] = m < n ? r[3 * m + k]
                                                     : gx[m - n][k];
            xp[m] = &xbuf[3 * (std::size_t)m];
            fp[m] = &fbuf[3 * (std::size_t)m];
            typeAll[m] = type[m < n ? m : owner[m - n]];
            tag[m] = (m < n ? m : owner[m - n]) + 1;
        }
        atom.nlocal = n;
        atom.nghost = nall - n;
        atom.ntypes = (int)syms.size();
        atom.x = xp.data();
        atom.f = fp.data();
        atom.type = typeAll.data();
        atom.tag = tag.data();

        NeighList list;
        std::vector<int> ilist(n), numneigh(n);
        std::vector<int*> firstneigh(n);
        for (int i = 0; i < n; ++i)
        {
            ilist[i] = i;
            numneigh[i] = (int)nbr[i].size();
            firstneigh[i] = nbr[i].data();
        }
        list.inum = n;
        list.ilist = ilist.data();
        list.numneigh = numneigh.data();
        list.firstneigh = firstneigh.data();

        // The pair style's interface member, for the EW buffer round trip.
        struct PairAccess : PairHDNNP
        {
            using PairHDNNP::PairHDNNP;
            nnp::InterfaceLammps* iface() { return interface; }
        };
        PairAccess pair(&lmp);
        std::string const rcs = std::to_string(rcut);
        std::vector<std::string> sa = {rcs, "dir", argv[1], "showew",
                                       showew ? "yes" : "no",
                                       "maxew", "1000000000", "cflength",
                                       cfl, "cfenergy", cfe};
        std::vector<char*> sv;
        for (auto& x : sa) sv.push_back(&x[0]);
        pair.settings((int)sv.size(), sv.data());
        std::vector<std::string> ca = {"*", "*"};
        for (auto const& sym : syms) ca.push_back(sym);
        std::vector<char*> cv;
        for (auto& x : ca) cv.push_back(&x[0]);
        pair.coeff((int)cv.size(), cv.data());
        pair.init_style();
        pair.list = &list;
        std::vector<double> eatom(nall, 0.0);
        pair.eatom = eatom.data();
        pair.compute(1 | 2, 1);
        for (int g = n; g < nall; ++g)
            for (int k = 0; k < 3; ++k) fp[owner[g - n]][k] += fp[g][k];
        std::printf("requests %d flags %d\n", neighbor.requests,
                    neighbor.lastFlags);
        std::printf("energy %.17g\n", pair.eng_vdwl);
        std::printf("virial %.17g %.17g %.17g %.17g %.17g %.17g\n",
                    pair.virial[0], pair.virial[1], pair.virial[2],
                    pair.virial[3], pair.virial[4], pair.virial[5]);
        for (int i = 0; i < n; ++i)
            std::printf("force %d %.17g %.17g %.17g\n", i, fp[i][0], fp[i][1],
                        fp[i][2]);
        for (int i = 0; i < n; ++i)
            std::printf("eatom %d %.17g\n", i, eatom[i]);
        std::rewind(lmp.screen);
        char line[512];
        while (std::fgets(line, sizeof(line), lmp.screen))
            std::printf("log %s", line);
        std::fclose(lmp.screen);
        if (showew)
        {
            nnp::InterfaceLammps* const in = pair.iface();
            in->process();
            long const bs = in->getEWBufferSize();
            std::vector<char> buf((std::size_t)bs + 1);
            char* const bp = buf.data();
            in->fillEWBuffer(bp, (int)bs);
            in->clearExtrapolationWarnings();
            char const* const cbp = buf.data();
            in->extractEWBuffer(cbp, (int)bs);
            for (std::string const& l : in->getExtrapolationWarningLines())
                std::printf("ewbuf %s", l.c_str());
            std::printf("ewbytes %ld\n", bs);
        }
    }
    catch (std::exception const& e)
    {
        std::fprintf(stderr, "%s\n", e.what());
        return 2;
    }
    return 0;
}
