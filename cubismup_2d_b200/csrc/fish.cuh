// Fish obstacle support shared by obstacles.cu and fish.cu.
#pragma once
#include "internal.cuh"

namespace cup2d {

struct Ctx;

struct FishSegPtrs { const Segment* seg[MAX_SHAPES]; };
FishSegPtrs fish_seg_ptrs(const Ctx& c);
void fish_setup_kernels();
void launch_fish_midline(Ctx& c, int k, cudaStream_t stream, int mode);
void launch_fish_kinematics(Ctx& c, int k);
void launch_fish_raster(Ctx& c, int k);

// AreaSegment::isIntersectingWithAABB (FishLibrary.cpp:344-401) against the
// block whose first/last cell centres are (start, end).
__device__ __forceinline__ bool segment_hits_block(const Segment& S, const double start[2],
                                                   const double end[2], const double safe)
{
  const double AABB_w[2] = {(end[0] - start[0]) / 2 + safe, (end[1] - start[1]) / 2 + safe};
  const double AABB_c[2] = {(end[0] + start[0]) / 2, (end[1] + start[1]) / 2};
  const double AABB_box[2][2] = {{AABB_c[0] - AABB_w[0], AABB_c[0] + AABB_w[0]},
                                 {AABB_c[1] - AABB_w[1], AABB_c[1] + AABB_w[1]}};
  const double il00 = fmax(S.boxLab[0][0], AABB_box[0][0]), il01 = fmin(S.boxLab[0][1], AABB_box[0][1]);
  const double il10 = fmax(S.boxLab[1][0], AABB_box[1][0]), il11 = fmin(S.boxLab[1][1], AABB_box[1][1]);
  if (il01 - il00 < 0 || il11 - il10 < 0) return false;
  const double widthXbox[2] = {AABB_w[0] * S.normalI[0], AABB_w[0] * S.normalJ[0]};
  const double widthYbox[2] = {AABB_w[1] * S.normalI[1], AABB_w[1] * S.normalJ[1]};
  const double boxBox[2][2] = {
      {AABB_c[0] - widthXbox[0] - widthYbox[0], AABB_c[0] + widthXbox[0] + widthYbox[0]},
      {AABB_c[1] - widthXbox[1] - widthYbox[1], AABB_c[1] + widthXbox[1] + widthYbox[1]}};
  const double if00 = fmax(boxBox[0][0], S.boxObj[0][0]), if01 = fmin(boxBox[0][1], S.boxObj[0][1]);
  const double if10 = fmax(boxBox[1][0], S.boxObj[1][0]), if11 = fmin(boxBox[1][1], S.boxObj[1][1]);
  if (if01 - if00 < 0 || if11 - if10 < 0) return false;
  return true;
}

// Fish::create step 6 (Fish.cpp:158-173): does any segment intersect block?
__device__ __forceinline__ bool fish_block_touching(const GridDesc& g, const Segment* seg, int nseg,
                                                    int bx, int by)
{
  const double start[2] = {cell_x(g, bx, 0), cell_y(g, by, 0)};
  const double end[2] = {cell_x(g, bx, BS - 1), cell_y(g, by, BS - 1)};
  for (int s = 0; s < nseg; s++)
    if (segment_hits_block(seg[s], start, end, 2 * g.h)) return true;
  return false;
}

} // namespace cup2d
