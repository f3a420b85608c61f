// Oracle test infrastructure: project-written stand-in for Cubism's BlockLab,
// the per-block ghost-cell loader the reference's operators go through
// (Definitions.h:112-170 derives BlockLabOpen from it).
//
// What the reference relies on:
//  - prepare(grid, stenBeg, stenEnd, tensorial) sizes a cache of
//    (BS + stenEnd - stenBeg - 1)^2 elements;
//  - load(info) copies the block and the ghost cells of its neighbours; cells
//    outside the domain are then filled by the subclass hook _apply_bc()
//    (BlockLabOpen copies the first/last interior row: zero gradient);
//  - m_cacheBlock->Access(ix,iy,iz) with indices shifted by -stenBeg;
//  - m_stencilStart/End, NX/NY (blocks per dimension), read(ix,iy,iz).
// Corner ghosts are copied from diagonal neighbours only for tensorial labs.
#pragma once
#include <cstdlib>
#include <vector>
#include "BlockInfo.h"
#include "Grid.h"

namespace cubism {

template <typename TElement>
struct LabCache
{
  int sx = 0, sy = 0;
  TElement* data = nullptr;  // raw storage: elements have no default constructor
  void resize(int nx, int ny) {
    std::free(data);
    sx = nx; sy = ny;
    data = static_cast<TElement*>(std::calloc((size_t)nx * ny, sizeof(TElement)));
  }
  ~LabCache() { std::free(data); }
  TElement& Access(int ix, int iy, int iz = 0) { (void)iz; return data[ix + sx * iy]; }
  const TElement& Access(int ix, int iy, int iz = 0) const { (void)iz; return data[ix + sx * iy]; }
};

template <typename BlockType, template <typename X> class allocator = std::allocator>
class BlockLab
{
 public:
  using ElementType = typename BlockType::ElementType;
 protected:
  LabCache<ElementType>* m_cacheBlock = nullptr;
  int m_stencilStart[3] = {0, 0, 0};
  int m_stencilEnd[3] = {1, 1, 1};
  bool istensorial = false;
  int NX = 0, NY = 0;
  const Grid<BlockType, allocator>* m_grid = nullptr;
 public:
  BlockLab() { m_cacheBlock = new LabCache<ElementType>(); }
  virtual ~BlockLab() { delete m_cacheBlock; }
  BlockLab(const BlockLab&) = delete;
  BlockLab& operator=(const BlockLab&) = delete;

  template <typename TGrid>
  void prepare(TGrid& grid, const int stenBeg[3], const int stenEnd[3], const int tensorial)
  {
    m_grid = &grid;
    for (int i = 0; i < 3; i++) { m_stencilStart[i] = stenBeg[i]; m_stencilEnd[i] = stenEnd[i]; }
    istensorial = tensorial != 0;
    NX = grid.getBlocksPerDimension(0);
    NY = grid.getBlocksPerDimension(1);
    m_cacheBlock->resize(BlockType::sizeX + stenEnd[0] - stenBeg[0] - 1,
                         BlockType::sizeY + stenEnd[1] - stenBeg[1] - 1);
  }

  virtual void _apply_bc(const BlockInfo& info, const double t = 0) { (void)info; (void)t; }

  void load(const BlockInfo& info, const double t = 0)
  {
    const int BX = BlockType::sizeX, BY = BlockType::sizeY;
    const int bx = info.index[0], by = info.index[1];
    const int s0 = m_stencilStart[0], s1 = m_stencilStart[1];
    const int e0 = BX + m_stencilEnd[0] - 1, e1 = BY + m_stencilEnd[1] - 1;
    for (int iy = s1; iy < e1; iy++)
    for (int ix = s0; ix < e0; ix++) {
      const bool outX = ix < 0 || ix >= BX, outY = iy < 0 || iy >= BY;
      if (outX && outY && !istensorial) continue;  // corners of a cross lab
      int nbx = bx, nby = by, lx = ix, ly = iy;
      if (ix < 0) { nbx--; lx += BX; } else if (ix >= BX) { nbx++; lx -= BX; }
      if (iy < 0) { nby--; ly += BY; } else if (iy >= BY) { nby++; ly -= BY; }
      if (nbx < 0 || nbx >= NX || nby < 0 || nby >= NY) continue;  // set by BC
      const BlockType& B = *m_grid->block(nbx, nby);
      m_cacheBlock->Access(ix - s0, iy - s1) = B(lx, ly);
    }
    _apply_bc(info, t);
  }

  const ElementType& read(const int ix, const int iy, const int iz = 0) const {
    (void)iz;
    return m_cacheBlock->Access(ix - m_stencilStart[0], iy - m_stencilStart[1]);
  }
};

} // namespace cubism
