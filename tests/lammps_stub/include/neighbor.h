// TEST INFRASTRUCTURE: neighbor requests are recorded, the list is built by
// the test driver.
#pragma once
namespace LAMMPS_NS {
namespace NeighConst { enum { REQ_DEFAULT = 0, REQ_FULL = 1 }; }
class Pair;
class NeighRequest {};
class Neighbor {
 public:
  int requests = 0, lastFlags = -1;
  NeighRequest* add_request(Pair*, int flags) { ++requests; lastFlags = flags; return &req; }
 private:
  NeighRequest req;
};
}
