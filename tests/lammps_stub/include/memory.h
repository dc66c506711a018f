// TEST INFRASTRUCTURE: 2-D arrays as LAMMPS's Memory::create makes them
// (one contiguous block plus row pointers).
#pragma once
namespace LAMMPS_NS {
class Memory {
 public:
  template <typename T> T** create(T**& a, int n1, int n2, const char*)
  {
    T* data = new T[(size_t)n1 * n2]();
    a = new T*[n1];
    for (int i = 0; i < n1; ++i) a[i] = data + (size_t)i * n2;
    return a;
  }
  template <typename T> void destroy(T**& a)
  {
    if (a) { delete[] a[0]; delete[] a; }
    a = nullptr;
  }
};
}
