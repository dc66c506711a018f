// TEST INFRASTRUCTURE: LAMMPS errors become C++ exceptions.
#pragma once
#include <stdexcept>
#include <string>
namespace LAMMPS_NS {
class Error {
 public:
  [[noreturn]] void all(const std::string& file, int line, const std::string& msg)
  { throw std::runtime_error(file + ":" + std::to_string(line) + ": " + msg); }
  [[noreturn]] void one(const std::string& file, int line, const std::string& msg)
  { all(file, line, msg); }
};
}
