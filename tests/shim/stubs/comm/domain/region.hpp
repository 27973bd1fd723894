// Stand-in for libcomm's comm/domain/region.hpp: an axis-aligned box of lattice cells.
#pragma once
namespace comm {
template <class T> struct Region {
  T x_low = 0, y_low = 0, z_low = 0, x_high = 0, y_high = 0, z_high = 0;
};
}  // namespace comm
