// lammps-emulate: drives n2p2b::InterfaceLammps the way LAMMPS's
// pair_style hdnnp does (PairHDNNP::compute, interface/LAMMPS/src/ML-HDNNP/
// pair_hdnnp.cpp:81-120): local atoms plus ghost copies of their periodic
// images, a full neighbor list with dx = x_i - x_j per local atom, then
// process(), getEnergy() and getForces() into a force array over local and
// ghost atoms, and finally the reverse communication that adds every
// ghost's force to the atom it copies.  LAMMPS itself is not part of this
// project; the program stands in for it to exercise the interface.
//
//   lammps-emulate <potential directory> <input.data> [cflength cfenergy]
//
// Prints "energy E" and one "force i fx fy fz" line per atom (input units).
#include "n2p2_b200.hpp"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <exception>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <array>
#include <tuple>
#include <vector>

int main(int argc, char* argv[])
{
    if (argc != 3 && argc != 5)
    {
        std::fprintf(stderr, "USAGE: %s <potential dir> <input.data> "
                             "[cflength cfenergy]\n", argv[0]);
        return 1;
    }
    double const cflength = argc == 5 ? std::atof(argv[3]) : 1.0;
    double const cfenergy = argc == 5 ? std::atof(argv[4]) : 1.0;
    try
    {
        n2p2b::InterfaceLammps lmp;
        n2p2b::Structure s;
        if (!s.readFromFile(argv[2], 0))
            throw std::runtime_error("ERROR: no configuration\n");
        if (!s.isPeriodic)
            throw std::runtime_error("ERROR: the emulation needs a periodic "
                                     "box\n");
        // Types 1..n = the elements of input.nn's "elements" line, in that
        // order, given to the interface as an explicit element map.
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
        std::string emap;
        for (std::size_t k = 0; k < syms.size(); ++k)
            emap += (k ? "," : "") + std::to_string(k + 1) + ":" + syms[k];
        lmp.initialize(argv[1], emap.c_str(), false, false, 0, -1, cflength,
                       cfenergy, 1e300, (int)syms.size(), 0);
        int const n = (int)s.numAtoms();
        std::vector<int> type(n);
        for (int i = 0; i < n; ++i)
        {
            type[i] = 0;
            for (std::size_t k = 0; k < syms.size(); ++k)
                if (syms[k] == s.symbol[i]) type[i] = (int)k + 1;
            if (type[i] == 0)
                throw std::runtime_error("ERROR: unknown element\n");
        }
        double const rc = lmp.getMaxCutoffRadiusLammps();
        // Image range: enough copies along each box vector (widths).
        double const (*b)[3] = s.box;
        auto cross = [](double const* u, double const* v, double* w) {
            w[0] = u[1] * v[2] - u[2] * v[1];
            w[1] = u[2] * v[0] - u[0] * v[2];
            w[2] = u[0] * v[1] - u[1] * v[0];
        };
        double vol, c[3][3];
        cross(b[1], b[2], c[0]);
        cross(b[2], b[0], c[1]);
        cross(b[0], b[1], c[2]);
        vol = std::fabs(b[0][0] * c[0][0] + b[0][1] * c[0][1]
                        + b[0][2] * c[0][2]);
        int p[3];
        for (int k = 0; k < 3; ++k)
        {
            double const area = std::sqrt(c[k][0] * c[k][0]
                                          + c[k][1] * c[k][1]
                                          + c[k][2] * c[k][2]);
            p[k] = (int)std::ceil(rc / (vol / area)) + 1;
        }
        // Full neighbor list over local atoms and ghost images.
        std::map<std::tuple<int, int, int, int>, int> ghostOf;
        std::vector<int> owner;            // ghost -> local atom
        std::vector<std::vector<int>> nbr(n);
        std::vector<std::vector<std::array<double, 3>>> del(n);
        double const rc2 = rc * rc;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j)
                for (int a = -p[0]; a <= p[0]; ++a)
                    for (int bb = -p[1]; bb <= p[1]; ++bb)
                        for (int cc = -p[2]; cc <= p[2]; ++cc)
                        {
                            if (i == j && a == 0 && bb == 0 && cc == 0)
                                continue;
                            double d[3];
                            for (int k = 0; k < 3; ++k)
                                d[k] = s.r[3 * i + k]
                                     - (s.r[3 * j + k] + a * b[0][k]
                                        + bb * b[1][k] + cc * b[2][k]);
                            double const r2 = d[0] * d[0] + d[1] * d[1]
                                            + d[2] * d[2];
                            if (r2 > rc2) continue;
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
                                }
                                else idx = it->second;
                            }
                            nbr[i].push_back(idx);
                            del[i].push_back({d[0], d[1], d[2]});
                        }
        int const nall = n + (int)owner.size();
        std::vector<int> typeAll(nall);
        for (int m = 0; m < nall; ++m)
            typeAll[m] = type[m < n ? m : owner[m - n]];
        lmp.setLocalAtoms(n, type.data());
        std::vector<int> numneigh(n);
        for (int i = 0; i < n; ++i) numneigh[i] = (int)nbr[i].size();
        lmp.allocateNeighborlists(numneigh.data());
        for (int i = 0; i < n; ++i)
            for (std::size_t k = 0; k < nbr[i].size(); ++k)
            {
                auto const& d = del[i][k];
                lmp.addNeighbor(i, nbr[i][k], nbr[i][k] + 1,
                                typeAll[nbr[i][k]], d[0], d[1], d[2],
                                d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
            }
        lmp.finalizeNeighborList();
        lmp.process();
        std::vector<double> fbuf(3 * (std::size_t)nall, 0.0);
        std::vector<double*> f(nall);
        for (int m = 0; m < nall; ++m) f[m] = &fbuf[3 * (std::size_t)m];
        double* const* fp = f.data();
        lmp.getForces(fp);
        // Reverse communication: ghost forces back to their atoms.
        for (int g = n; g < nall; ++g)
            for (int k = 0; k < 3; ++k) f[owner[g - n]][k] += f[g][k];
        std::printf("energy %.17g\n", lmp.getEnergy());
        for (int i = 0; i < n; ++i)
            std::printf("force %d %.17g %.17g %.17g\n", i, f[i][0], f[i][1],
                        f[i][2]);
    }
    catch (std::exception const& e)
    {
        std::fprintf(stderr, "%s", e.what());
        return 2;
    }
    return 0;
}
