// TEST INFRASTRUCTURE: LAMMPS integer types (-DLAMMPS_SMALLBIG) and macros.
#pragma once
#include <cstdint>
#include "mpi.h"
namespace LAMMPS_NS {
typedef int tagint;
typedef int64_t bigint;
}
#define FLERR __FILE__, __LINE__
#define NEIGHMASK 0x1FFFFFFF
