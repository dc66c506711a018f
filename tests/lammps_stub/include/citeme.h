// TEST INFRASTRUCTURE: citation records are counted, not printed.
#pragma once
namespace LAMMPS_NS {
class CiteMe {
 public:
  int count = 0;
  void add(const char*) { ++count; }
};
}
