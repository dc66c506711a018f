// TEST INFRASTRUCTURE: LAMMPS's Pointers base (references to the instance's
// members, as the real class holds them).
#pragma once
#include <string>
#include <vector>
#include "lammps.h"
#include "utils.h"   // LAMMPS's pointers.h brings utils:: into every class
namespace LAMMPS_NS {
class Pointers {
 public:
  explicit Pointers(LAMMPS* ptr)
      : lmp(ptr), atom(ptr->atom), comm(ptr->comm), error(ptr->error),
        memory(ptr->memory), neighbor(ptr->neighbor), update(ptr->update),
        world(ptr->world), screen(ptr->screen), logfile(ptr->logfile) {}
  virtual ~Pointers() = default;
 protected:
  LAMMPS* lmp;
  Atom*& atom;
  Comm*& comm;
  Error*& error;
  Memory*& memory;
  Neighbor*& neighbor;
  Update*& update;
  MPI_Comm& world;
  FILE*& screen;
  FILE*& logfile;
};
}
