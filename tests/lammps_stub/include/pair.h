// TEST INFRASTRUCTURE: the base class of pair styles, with the members and
// energy/virial tallies that pair_style hdnnp uses.
#pragma once
#include "pointers.h"
#include "atom.h"
#include "neigh_list.h"
namespace LAMMPS_NS {
class Pair : protected Pointers {
 public:
  explicit Pair(LAMMPS* lmp) : Pointers(lmp) {}
  ~Pair() override = default;
  virtual void compute(int, int) = 0;
  virtual void settings(int, char**) {}
  virtual void coeff(int, char**) {}
  virtual void init_style() {}
  virtual double init_one(int, int) { return 0.0; }

  double eng_vdwl = 0.0, eng_coul = 0.0;
  double virial[6] = {0, 0, 0, 0, 0, 0};
  double* eatom = nullptr;
  NeighList* list = nullptr;
  int single_enable = 1, restartinfo = 1, one_coeff = 0, manybody_flag = 0;
  int unit_convert_flag = 0, reinitflag = 1;
  int allocated = 0;
  int** setflag = nullptr;
  double** cutsq = nullptr;
  int eflag_either = 0, eflag_global = 0, eflag_atom = 0;
  int vflag_either = 0, vflag_global = 0, vflag_fdotr = 0;

 protected:
  void ev_init(int eflag, int vflag)
  {
    eflag_either = eflag; eflag_global = eflag & 1; eflag_atom = (eflag & 2) ? 1 : 0;
    vflag_either = vflag; vflag_global = vflag & 1; vflag_fdotr = vflag_global;
    eng_vdwl = eng_coul = 0.0;
    for (double& v : virial) v = 0.0;
  }
  void ev_tally(int, int, int, int, double evdwl, double ecoul, double,
                double, double, double)
  {
    if (eflag_global) { eng_vdwl += evdwl; eng_coul += ecoul; }
  }
  // virial = sum over local and ghost atoms of x (x) f
  void virial_fdotr_compute()
  {
    int const nall = atom->nlocal + atom->nghost;
    for (int i = 0; i < nall; ++i) {
      double const* x = atom->x[i];
      double const* f = atom->f[i];
      virial[0] += f[0] * x[0]; virial[1] += f[1] * x[1]; virial[2] += f[2] * x[2];
      virial[3] += f[1] * x[0]; virial[4] += f[2] * x[0]; virial[5] += f[2] * x[1];
    }
  }
};
}
