// Fish obstacle support shared by obstacles.cu and fish.cu.
#pragma once
#include "internal.cuh"

namespace cup2d {

struct Ctx;

cudaError_t fish_setup_kernels();          // dynamic shared-memory limits
cudaError_t fish_width_cubes(const FishArrays& F, cudaStream_t st);   // F.w3 from F.width
bool fish_fits_on_chip(int Nm, int nseg, int device);   // staged arrays within the opt-in limit
void launch_fish_midline(Ctx& c, int k, cudaStream_t stream, int mode);
void launch_fish_place(Ctx& c, int k);
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

__device__ __forceinline__ void clip_rect(const GridDesc& g, int& bx0, int& bx1, int& by0, int& by1) {
  bx0 = bx0 < 0 ? 0 : bx0; by0 = by0 < 0 ? 0 : by0;
  bx1 = bx1 > g.bpdx - 1 ? g.bpdx - 1 : bx1; by1 = by1 > g.bpdy - 1 ? g.bpdy - 1 : by1;
}

// Ordered tile selection: the blocks of the rectangle [bx0, bx1] x [by0, by1]
// (clipped to the grid) for which touch(bx, by) holds, in increasing block
// index (the order of obstacleBlocks[blockID]), become t.tiles[0..n) with
// t.slot[b]; n goes to *ntilesOut, overflow of the capacity raises
// ST_CAPACITY.  touch(q, bx, by) gets the candidate's row-major index q in
// the clipped rectangle (clip_rect).  Called by a whole 1D CTA whose size
// is a multiple of 32.
template <class Touch>
__device__ void select_tiles(const GridDesc& g, ObstTiles t, int bx0, int bx1, int by0, int by1,
                             Touch touch, int* ntilesOut, int* status)
{
  __shared__ int wcnt[32];
  __shared__ int base;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  clip_rect(g, bx0, bx1, by0, by1);
  const int W = bx1 - bx0 + 1, H = by1 - by0 + 1, n = (W > 0 && H > 0) ? W * H : 0;
  if (tid == 0) base = 0;
  __syncthreads();
  for (int q0 = 0; q0 < n; q0 += blockDim.x) {
    const int q = q0 + tid;
    int b = -1;
    bool f = false;
    if (q < n) {
      const int by = by0 + q / W, bx = bx0 + q % W;
      b = by * g.bpdx + bx;
      f = touch(q, bx, by);
    }
    const unsigned m = __ballot_sync(0xffffffffu, f);
    if (lane == 0) wcnt[wid] = __popc(m);
    __syncthreads();
    int off = 0, tot = 0;
    for (int w = 0; w < nw; w++) { if (w < wid) off += wcnt[w]; tot += wcnt[w]; }
    const int pos = base + off + __popc(m & ((1u << lane) - 1u));
    if (f) {
      if (pos < t.capacity) { t.tiles[pos] = b; t.slot[b] = pos; }
      else atomicOr(status, ST_CAPACITY);
    }
    __syncthreads();
    if (tid == 0) base += tot;
    __syncthreads();
  }
  if (tid == 0) *ntilesOut = base < t.capacity ? base : t.capacity;
}

// Block index range whose cells' AABB, widened by `safe`, can overlap
// [lo, hi] along one axis (one block of margin on each side).
__device__ __forceinline__ void block_range(double lo, double hi, double h, double safe, int& b0, int& b1) {
  if (!(lo <= hi)) { b0 = 1; b1 = 0; return; }            // empty (also for NaN)
  const double bw = BS * h;
  b0 = (int)floor(fmax((lo - safe) / bw, -2.0)) - 1;
  b1 = (int)floor(fmin((hi + safe) / bw, 1e8)) + 1;
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
