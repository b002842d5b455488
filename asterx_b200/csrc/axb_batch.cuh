// Batched launches over the boxes of a level.
//
// A batched launch runs one kernel body over the tiles (CTA-sized work
// items) of every box of a batch.  The tiles of box b are items
// [prefix[b], prefix[b+1]) of a flat list; the tile's block index inside
// its box is unflattened from the box's own grid, so every body sees exactly
// the block indices its single-box launch would give it and the results are
// bit-identical to one launch per box.  The grid is persistent: each CTA
// draws chunks of items from an atomic work counter, and copies the per-box
// argument block
// into shared memory when it moves on to the next box.
#pragma once

#include <type_traits>

#include "axb_common.cuh"

namespace axb {

struct TileTable {
  const long long *prefix; // nbox + 1 entries
  const uint3 *grid;       // per-box grid of the single-box launch
  int nbox;
  long long total;
};

// box of a flat item index (prefix is non-decreasing, prefix[0] = 0)
AXB_D int tile_box(const TileTable &t, long long item) {
  int lo = 0, hi = t.nbox - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(t.prefix + mid) <= item)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

AXB_D uint3 tile_bid(const uint3 g, long long local) {
  uint3 b;
  b.x = unsigned(local % g.x);
  local /= g.x;
  b.y = unsigned(local % g.y);
  b.z = unsigned(local / g.y);
  return b;
}

// Items are handed out in chunks of this many by an atomic counter, so CTAs
// that drew cheap tiles (small boxes) take more of them.
constexpr int BATCH_CHUNK = 4;

// Run f(args_of_box, block_index) over the items this CTA draws from the
// work counter `ctr` (zeroed before the launch).  The loop ends when the
// counter passes the item count; it never waits on other CTAs.
template <class Args, class F>
AXB_D void batch_loop(const Args *__restrict__ args, const TileTable &t,
                      unsigned long long *ctr, F &&f) {
  __shared__ __align__(16) unsigned char raw[sizeof(Args)];
  __shared__ long long s_base;
  Args &a = *reinterpret_cast<Args *>(raw);
  const int nthreads = blockDim.x * blockDim.y * blockDim.z;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  int cur = -1;
  for (;;) {
    __syncthreads();
    if (tid == 0)
      s_base = (long long)atomicAdd(ctr, (unsigned long long)BATCH_CHUNK);
    __syncthreads();
    const long long base = s_base;
    if (base >= t.total) // CTA-uniform
      break;
    const long long last = min(base + BATCH_CHUNK, t.total);
    for (long long item = base; item < last; ++item) {
      const int bx = tile_box(t, item);
      if (bx != cur) {
        __syncthreads();
        const unsigned *src = reinterpret_cast<const unsigned *>(args + bx);
        unsigned *dst = reinterpret_cast<unsigned *>(raw);
        for (int q = tid; q < int(sizeof(Args) / 4); q += nthreads)
          dst[q] = __ldg(src + q);
        __syncthreads();
        cur = bx;
      }
      const uint3 bid = tile_bid(t.grid[bx], item - __ldg(t.prefix + bx));
      if constexpr (std::is_invocable_v<F &, const Args &, uint3, int>)
        f(a, bid, bx); // bodies that need the box index
      else
        f(a, bid);
    }
  }
}

} // namespace axb
