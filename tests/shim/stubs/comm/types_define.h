// Stand-in for libcomm's comm/types_define.h (pkg libcomm v0.3.3, not vendored): the integer
// types and the process record the reference's headers name.
#pragma once
namespace comm {
typedef long _type_lattice_size;
typedef long _type_lattice_coord;
struct mpi_process {
  int own_rank = 0;
  int all_ranks = 1;
  int comm = 0;
};
}  // namespace comm
