// Oracle test infrastructure: project-written stand-in for Cubism's uniform
// block Grid as the reference uses it (SimulationData.cpp:17-32):
// Grid(bpdx, bpdy, bpdz, maxextent), getBlocksInfo(), getBlocksPerDimension(),
// getH().  h = maxextent / max(bpdx*BS, bpdy*BS); block b = bx + bpdx*by.
#pragma once
#include <algorithm>
#include <cstdlib>
#include <vector>
#include "BlockInfo.h"

namespace cubism {

template <typename TBlock, template <typename X> class allocator = std::allocator>
class Grid
{
  std::vector<TBlock*> blocks;
  std::vector<BlockInfo> infos;
  int nb[3] = {0, 0, 0};
  double h = 0;
 public:
  using Block = TBlock;
  Grid(const int bpdx, const int bpdy, const int bpdz, const double maxextent)
  {
    nb[0] = bpdx; nb[1] = bpdy; nb[2] = bpdz;
    h = maxextent / std::max(bpdx * TBlock::sizeX, bpdy * TBlock::sizeY);
    for (int by = 0; by < bpdy; by++)
    for (int bx = 0; bx < bpdx; bx++) {
      // blocks and elements delete their copy constructors and so have no
      // default constructor: storage is raw, zero-filled memory
      TBlock* b = static_cast<TBlock*>(std::calloc(1, sizeof(TBlock)));
      blocks.push_back(b);
      BlockInfo I;
      I.blockID = bx + (long long)bpdx * by;
      I.index[0] = bx; I.index[1] = by; I.index[2] = 0;
      I.origin[0] = (double)(bx * TBlock::sizeX) * h;
      I.origin[1] = (double)(by * TBlock::sizeY) * h;
      I.h = h; I.h_gridpoint = h;
      I.ptrBlock = b;
      infos.push_back(I);
    }
  }
  ~Grid() { for (auto b : blocks) std::free(b); }
  std::vector<BlockInfo>& getBlocksInfo() { return infos; }
  const std::vector<BlockInfo>& getBlocksInfo() const { return infos; }
  int getBlocksPerDimension(const int d) const { return nb[d]; }
  double getH() const { return h; }
  TBlock* block(int bx, int by) const { return blocks[bx + nb[0] * by]; }
};

} // namespace cubism
