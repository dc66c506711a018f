// TEST INFRASTRUCTURE: the time step counter.
#pragma once
#include "lmptype.h"
namespace LAMMPS_NS {
class Update {
 public:
  bigint ntimestep = 0;
};
}
