// batchq.cuh -- the work queue of a batched launch: many problems' launches
// of one kernel run by one grid of persistent CTAs.
//
// A batched launch is a table of per-problem launch records and a map of
// items (record, block of that record's own grid) in record order.  The CTAs
// take chunks of kQueueChunk items from an atomic counter; an item runs that
// block of that problem's launch.  A problem whose solve has stopped has
// nothing to do in any of its blocks, so the CTA that meets one of its items
// skips the rest of that record's items in its chunk at once: converged
// problems cost a counter step, not a block launch each.  The last CTA to
// leave resets the counters for the next launch on the stream.
#pragma once
#include "icb_internal.hpp"

namespace icb
{
struct BatchQueue
{
  unsigned *next = nullptr; ///< items handed out
  unsigned *done = nullptr; ///< CTAs that have left
  int items = 0;
};
constexpr int kQueueChunk = 4;

/// nb(rec): blocks of a record's own grid; skip(rec): the record's blocks
/// have nothing to do (read by one thread, the same for the whole record
/// while any of its blocks is pending); run(rec, b): block b of the record
template <class Rec, class Nb, class Skip, class Run>
__device__ __forceinline__ void batch_queue(const Rec *__restrict__ D, const int2 *__restrict__ map,
                                            const BatchQueue &q, Nb nb, Skip skip, Run run)
{
  __shared__ int base, jump;
  const bool lead = threadIdx.x == 0 && threadIdx.y == 0 && threadIdx.z == 0;
  for(;;)
  {
    if(lead)
      base = int(atomicAdd(q.next, unsigned(kQueueChunk)));
    __syncthreads();
    const int b0 = base;
    __syncthreads();
    if(b0 >= q.items)
      break;
    const int b1 = min(b0 + kQueueChunk, q.items);
    for(int it = b0; it < b1;)
    {
      const int2 m = map[it];
      const Rec &r = D[m.x];
      if(lead)
        jump = skip(r) ? nb(r) - m.y : 0;
      __syncthreads();
      const int j = jump;
      __syncthreads();
      if(j > 0)
      {
        it += j;
        continue;
      }
      run(r, m.y);
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

/// CTAs of a persistent batched launch: the kernel's residency on every SM,
/// no more than the chunks there are
inline int queue_grid(const void *kern, int threads, int smem, int items)
{
  int per = 0;
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, threads, smem) != cudaSuccess ||
     per < 1)
  {
    (void)cudaGetLastError();
    per = 1;
  }
  const int chunks = (items + kQueueChunk - 1) / kQueueChunk;
  return std::max(1, std::min(per * num_sms(), chunks));
}
} // namespace icb
