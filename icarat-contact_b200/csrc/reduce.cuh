// reduce.cuh -- deterministic grid-wide reductions without a second launch.
//
// Every block reduces its values (warp shuffles, then shared memory) and
// writes them to red.partials[block]; the block that finishes last (atomic
// ticket) sums all partials in block order and hands the totals to a
// finisher functor run by its thread 0.  The summation order depends only on
// the launch shape, so results are bitwise reproducible run to run.
#pragma once
#include "icb_internal.hpp"

namespace icb
{

/// the ticket of the last-block pattern: an atomic add with acquire-release
/// semantics at GPU scope, which orders this thread's partial stores before
/// the ticket (release) and, for the last block, the other blocks' partials
/// before its reads (acquire) -- without a full sequentially consistent fence
__device__ __forceinline__ unsigned ticket_acq_rel(unsigned *counter)
{
  unsigned t;
  asm volatile("atom.acq_rel.gpu.add.u32 %0, [%1], 1;"
               : "=r"(t)
               : "l"(counter)
               : "memory");
  return t;
}

__device__ __forceinline__ double warp_sum_d(double v)
{
#pragma unroll
  for(int o = 16; o > 0; o >>= 1)
    v += __shfl_down_sync(0xffffffffu, v, o);
  return v;
}

/// the reduction of block `bid` of `nb` blocks: a batched launch that runs
/// several independent grids passes each block's index and count within its
/// own grid, so every grid reduces exactly as its own launch would
template <int NV, class Fin>
__device__ __forceinline__ void block_reduce_at(double (&v)[NV], const RedScratch &red, Fin fin,
                                                int bid, int nb)
{
  __shared__ double sw[32][NV];
  __shared__ int last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const int nw = (nth + 31) >> 5;
#pragma unroll
  for(int k = 0; k < NV; k++)
    v[k] = warp_sum_d(v[k]);
  if((tid & 31) == 0)
#pragma unroll
    for(int k = 0; k < NV; k++)
      sw[tid >> 5][k] = v[k];
  __syncthreads();
  if(tid == 0)
  {
#pragma unroll
    for(int k = 0; k < NV; k++)
    {
      double s = 0.0;
      for(int w = 0; w < nw; w++)
        s += sw[w][k];
      red.partials[(long long)bid * NV + k] = s;
    }
    const unsigned t = ticket_acq_rel(red.counter);
    last = (t == unsigned(nb - 1));
  }
  __syncthreads();
  if(!last)
    return;
  __threadfence();
  double s[NV];
#pragma unroll
  for(int k = 0; k < NV; k++)
    s[k] = 0.0;
  for(int b = tid; b < nb; b += nth)
#pragma unroll
    for(int k = 0; k < NV; k++)
      s[k] += __ldcg(red.partials + (long long)b * NV + k);
#pragma unroll
  for(int k = 0; k < NV; k++)
    s[k] = warp_sum_d(s[k]);
  __syncthreads();
  if((tid & 31) == 0)
#pragma unroll
    for(int k = 0; k < NV; k++)
      sw[tid >> 5][k] = s[k];
  __syncthreads();
  if(tid == 0)
  {
    double tot[NV];
#pragma unroll
    for(int k = 0; k < NV; k++)
    {
      tot[k] = 0.0;
      for(int w = 0; w < nw; w++)
        tot[k] += sw[w][k];
    }
    *red.counter = 0u;
    fin(tot);
  }
}

/// The finish of a sum whose partials sit at slots fixed by the work, not by
/// the block that computed them (so the launch may be cut into any number of
/// blocks): each block calls it once, after its threads stored their slots;
/// the last of the nb blocks to arrive sums slots [0, nslots) in a fixed order
/// (thread t takes t, t + blockDim, ...; then the warps in order) and hands
/// the total to fin.  `wrote`: this thread stored slots (it fences them).
template <class Fin>
__device__ __forceinline__ void slots_reduce_finish(const RedScratch &red, long long nslots,
                                                    int nb, bool wrote, Fin fin)
{
  __shared__ double sw[32];
  __shared__ int last;
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nth = blockDim.x * blockDim.y * blockDim.z;
  const int nw = (nth + 31) >> 5;
  if(wrote)
    __threadfence();
  __syncthreads();
  if(tid == 0)
    last = ticket_acq_rel(red.counter) == unsigned(nb - 1);
  __syncthreads();
  if(!last)
    return;
  __threadfence();
  double s = 0.0;
  for(long long k = tid; k < nslots; k += nth)
    s += __ldcg(red.partials + k);
  s = warp_sum_d(s);
  if((tid & 31) == 0)
    sw[tid >> 5] = s;
  __syncthreads();
  if(tid == 0)
  {
    double tot = 0.0;
    for(int w = 0; w < nw; w++)
      tot += sw[w];
    *red.counter = 0u;
    fin(&tot);
  }
}

template <int NV, class Fin>
__device__ __forceinline__ void block_reduce(double (&v)[NV], const RedScratch &red,
                                             Fin fin)
{
  block_reduce_at<NV>(v, red, fin, blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z),
                      gridDim.x * gridDim.y * gridDim.z);
}

struct FinStore
{
  double *out;
  __device__ void operator()(const double *t) const { *out = t[0]; }
};

} // namespace icb
