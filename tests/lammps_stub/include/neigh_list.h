// TEST INFRASTRUCTURE: a full neighbor list.
#pragma once
#include "lmptype.h"
namespace LAMMPS_NS {
class NeighList {
 public:
  int inum = 0;
  int* ilist = nullptr;
  int* numneigh = nullptr;
  int** firstneigh = nullptr;
};
}
