// Oracle test infrastructure: project-written stand-in for Cubism's
// BlockInfo as the reference uses it (Definitions.h:24-28): blockID,
// index[3], origin[3], h_gridpoint, ptrBlock and the cell-centre pos().
//
// Cell centres are origin + h*(i + 1/2) (implied by FishLibrary.cpp:346 and
// ShapeLibrary.h:27-29 which treat pos(0,0)/pos(BS-1,BS-1) as centres).
// The GPU path evaluates exactly this expression, so positions agree bitwise.
#pragma once
#include <array>

namespace cubism {

struct BlockInfo
{
  long long blockID = 0;
  int index[3] = {0, 0, 0};
  double origin[3] = {0, 0, 0};
  double h = 0, h_gridpoint = 0;
  void* ptrBlock = nullptr;

  template <typename T>
  inline void pos(T p[2], const int ix, const int iy) const {
    p[0] = (T)(origin[0] + h_gridpoint * (ix + 0.5));
    p[1] = (T)(origin[1] + h_gridpoint * (iy + 0.5));
  }
  template <typename T>
  inline std::array<T, 2> pos(const int ix, const int iy) const {
    std::array<T, 2> p;
    pos(p.data(), ix, iy);
    return p;
  }
};

} // namespace cubism
