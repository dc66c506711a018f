// TEST INFRASTRUCTURE: per-atom arrays (local atoms first, then ghosts).
#pragma once
#include "lmptype.h"
namespace LAMMPS_NS {
class Atom {
 public:
  int nlocal = 0, nghost = 0, ntypes = 0;
  double** x = nullptr;
  double** f = nullptr;
  int* type = nullptr;
  tagint* tag = nullptr;
};
}
