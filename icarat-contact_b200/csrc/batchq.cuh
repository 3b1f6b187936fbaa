// batchq.cuh -- the work queue of a batched launch: many problems' launches
// of one kernel run by one grid of persistent CTAs.
//
// A batched launch is a table of per-problem launch records and a map of
// items (record, block of that record's own grid) in record order.  The CTAs
// take chunks of items from an atomic counter (one item each while a launch
// fits in one wave); an item runs that
// block of that problem's launch.  A problem whose solve has stopped has
// nothing to do in any of its blocks, so the CTA that meets one of its items
// skips the rest of that record's items in its chunk at once and moves the
// counter past the record's last item: a converged problem costs a few
// counter steps, not a block launch (or a chunk) each.  The last CTA to
// leave resets the counters for the next launch on the stream.
#pragma once
#include <algorithm>

#include "icb_internal.hpp"

namespace icb
{
/// a block's coordinates and its grid's extent: blockIdx / gridDim of a
/// launch of its own, or the block's place in one grid of a batched launch
struct Blk
{
  unsigned x, y, z, gx, gy, gz;
};
__device__ __forceinline__ Blk this_block()
{
  return Blk{blockIdx.x, blockIdx.y, blockIdx.z, gridDim.x, gridDim.y, gridDim.z};
}

struct BatchQueue
{
  unsigned *next = nullptr; ///< items handed out
  unsigned *done = nullptr; ///< CTAs that have left
  int items = 0;
  int chunk = 1; ///< items a CTA takes at a time (queue_chunk)
};
/// items per chunk: 1 while every item gets a CTA of its own in one wave
/// (small launches stay fully parallel), more for launches many waves long,
/// so a converged problem's items are skipped several at a time
inline int queue_chunk(int items, int capacity)
{
  return std::max(1, std::min(16, items / std::max(1, 2 * capacity)));
}

/// nb(rec): blocks of a record's own grid; skip(rec): the record's blocks
/// have nothing to do (read by one thread, the same for the whole record
/// while any of its blocks is pending); run(rec, b, fresh): block b of the
/// record, fresh when the CTA's previous item was of another record (what
/// a body stages per record in shared memory survives until then)
template <class Rec, class Nb, class Skip, class Run>
__device__ __forceinline__ void batch_queue(const Rec *__restrict__ D, const int2 *__restrict__ map,
                                            const BatchQueue &q, Nb nb, Skip skip, Run run)
{
  __shared__ int base, jump;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0;
  for(;;)
  {
    if(lead)
      base = int(atomicAdd(q.next, unsigned(q.chunk)));
    __syncthreads();
    const int b0 = base;
    __syncthreads();
    if(b0 >= q.items)
      break;
    const int b1 = min(b0 + q.chunk, q.items);
    int running = -1; // the record of the last item run: not skipped
    for(int it = b0; it < b1;)
    {
      const int2 m = map[it];
      const Rec &r = D[m.x];
      // a record found running stays so while any of its items is pending
      const bool fresh = m.x != running;
      if(fresh)
      {
        if(lead)
        {
          jump = skip(r) ? nb(r) - m.y : 0;
          // the record's items are contiguous in the map: move the queue
          // past its last one, so no CTA takes another chunk of it (chunks
          // already taken skip it here)
          if(jump > 0)
            atomicMax(q.next, unsigned(it + jump));
        }
        __syncthreads();
        const int j = jump;
        __syncthreads();
        if(j > 0)
        {
          it += j;
          continue;
        }
        running = m.x;
      }
      run(r, m.y, fresh);
      __syncthreads(); // the bodies' shared memory is reused by the next item
      ++it;
    }
  }
  if(lead)
  {
    __threadfence();
    const unsigned g = gridDim.x * gridDim.y * gridDim.z;
    if(atomicAdd(q.done, 1u) == g - 1)
    {
      *q.next = 0u;
      *q.done = 0u;
    }
  }
}

/// CTAs of a persistent batched launch (the kernel's residency on every SM,
/// no more than the chunks there are); sets q.chunk
inline int queue_grid(const void *kern, int threads, int smem, BatchQueue &q)
{
  int per = 0;
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess ||
     per < 1)
  {
    (void)cudaGetLastError();
    per = 1;
  }
  const int cap = per * num_sms();
  q.chunk = queue_chunk(q.items, cap);
  const int chunks = (q.items + q.chunk - 1) / q.chunk;
  return std::max(1, std::min(cap, chunks));
}
} // namespace icb
