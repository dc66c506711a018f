// TEST INFRASTRUCTURE: the LAMMPS instance as seen by a pair style.
#pragma once
#include <cstdio>
#include "lmptype.h"
namespace LAMMPS_NS {
class Atom; class Comm; class Error; class Memory; class Neighbor;
class Update; class CiteMe;
class LAMMPS {
 public:
  Atom* atom = nullptr;
  Comm* comm = nullptr;
  Error* error = nullptr;
  Memory* memory = nullptr;
  Neighbor* neighbor = nullptr;
  Update* update = nullptr;
  CiteMe* citeme = nullptr;
  FILE* screen = nullptr;
  FILE* logfile = nullptr;
  MPI_Comm world = 0;
};
}
