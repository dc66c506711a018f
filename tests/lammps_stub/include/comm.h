// TEST INFRASTRUCTURE: one rank.
#pragma once
namespace LAMMPS_NS {
class Comm {
 public:
  int me = 0, nprocs = 1;
};
}
