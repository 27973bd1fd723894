// Stand-in for libcomm's comm/domain/colored_domain.h: the domain record the reference hands to
// gpu_prepare (the B200 shim serves one rank holding the whole periodic box and ignores it).
#pragma once
#include <comm/domain/region.hpp>
#include <comm/types_define.h>
namespace comm {
class ColoredDomain {
 public:
  _type_lattice_size lattice_size_ghost[3] = {0, 0, 0};
  Region<_type_lattice_size> local_sector_region[8];
};
}  // namespace comm
