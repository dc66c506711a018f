// TEST INFRASTRUCTURE: the LAMMPS utils functions a pair style calls.
#pragma once
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include "lammps.h"
namespace LAMMPS_NS {
namespace utils {
inline double numeric(const char*, int, const char* s, bool, LAMMPS*) { return std::atof(s); }
inline int inumeric(const char*, int, const char* s, bool, LAMMPS*) { return std::atoi(s); }
inline int logical(const char*, int, const char* s, bool, LAMMPS*)
{
  std::string v(s);
  if (v == "yes" || v == "on" || v == "true" || v == "1") return 1;
  if (v == "no" || v == "off" || v == "false" || v == "0") return 0;
  throw std::runtime_error("expected boolean: " + v);
}
inline char* strdup(const std::string& s)
{
  char* p = new char[s.size() + 1];
  std::memcpy(p, s.c_str(), s.size() + 1);
  return p;
}
template <typename... Args> void logmesg(LAMMPS* lmp, const std::string& fmt, Args&&...)
{
  if (lmp && lmp->screen) std::fputs(fmt.c_str(), lmp->screen);
}
}
}
