// operator_tc.cu -- the FP32 Hex8 element operator with the element
// contraction on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// Same decomposition as k_matvec_h8 (operator.cu): a CTA of 32x8 threads owns
// a 31x7 tile of output nodes and marches up a chunk of z planes, one thread
// per element column, bottom-corner values and top-corner contributions kept
// in registers.  Per element layer the 256 elements of the CTA form two
// 128-row MMA tiles:
//   A (128 x 24, K-major, TF32): row m = the element's 8 corner
//     displacements x 3 components, written by its thread into shared memory
//     in the SWIZZLE_128B K-major layout (16-byte chunk c of row m stored at
//     chunk c ^ (m & 7) of the row's 128-byte line);
//   B (32 x 24, K-major): the unit element matrix K0 (rows 24..31 zero);
//   D (128 x 32, FP32) in tensor memory: D[m][n] = (K0 u_m)[n].
// One thread issues the 2 x 3 tcgen05.mma (K = 8 each) and commits them to an
// mbarrier; every thread then reads its element's 24 results back with one
// tcgen05.ld (lane m = its element), scales by E_e and continues exactly as
// the CUDA-core kernel.  Every mbarrier wait is bounded: on timeout the CTA
// records the event in g_tc_timeouts, stops, frees its tensor memory and
// returns.
//
// TF32 keeps 10 mantissa bits of every operand, so this operator is used for
// the FP32 multigrid V-cycle under the FP64 Krylov iteration (ICB_MIXED),
// never for a residual the outer iteration relies on.
#include <algorithm>

#include "icb_internal.hpp"
#include "reduce.cuh"

namespace icb
{
__device__ unsigned g_tc_timeouts = 0;

namespace
{
constexpr int TX = 32, TY = 8;
constexpr unsigned kSpinLimit = 1u << 22; // try_wait polls before a CTA gives up

__device__ __forceinline__ constexpr int lnodeTc(int a, int b) { return (a ^ b) + 2 * b; }

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

/// K-major SWIZZLE_128B shared-memory matrix descriptor: rows of 128 bytes,
/// 8-row swizzle atoms 1024 bytes apart (SBO), version 1 (tcgen05)
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
  uint64_t d = 0;
  d |= uint64_t((saddr >> 4) & 0x3FFFu);
  d |= uint64_t(1) << 16;          // leading byte offset (unused for swizzled K-major)
  d |= uint64_t(1024 >> 4) << 32;  // stride byte offset: next 8-row group
  d |= uint64_t(1) << 46;          // descriptor version
  d |= uint64_t(2) << 61;          // SWIZZLE_128B
  return d;
}

/// instruction descriptor: kind::tf32, D FP32, A/B TF32, both K-major,
/// N = 32, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((32u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t accumulate)
{
  asm volatile("{\n\t.reg .pred p;\n\t"
               "setp.ne.b32 p, %4, 0;\n\t"
               "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
               :
               : "r"(dtmem), "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar)
{
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity)
{
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}\n"
               : "=r"(ok)
               : "r"(mbar), "r"(parity)
               : "memory");
  return ok != 0;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v)
{
  uint32_t r[32];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                 "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                 "=r"(r[30]), "=r"(r[31])
               : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for(int i = 0; i < 24; i++)
    v[i] = __uint_as_float(r[i]);
}

template <int MODE>
__device__ __forceinline__ float epilogueTc(float Au, float uself, long long i, const Epi<float> &ep)
{
  if(MODE == OP_APPLY)
    return Au;
  float r = __ldg(ep.b + i) - Au;
  if(MODE == OP_RESIDUAL)
    return r;
  if(MODE == OP_JACOBI)
    return uself + ep.omega * __ldg(ep.dinv + i) * r;
  float dn = ep.c2 * __ldg(ep.dinv + i) * r;
  if(ep.c1 != 0.f)
    dn += ep.c1 * ep.d[i];
  ep.d[i] = dn;
  return uself + dn;
}

template <bool DOT, int MODE>
__global__ void __launch_bounds__(TX *TY)
    k_matvec_h8_tc(const KMat<float, 24> K, const Dims d, const int zchunk,
                   const float *__restrict__ E, const float *__restrict__ u,
                   float *__restrict__ y, const uint8_t *__restrict__ fix, RedScratch red,
                   double *dotOut, const KState *gate, const int gateConv, const Epi<float> ep)
{
  if(gate && (gate->stop || (gateConv && gate->conv)))
    return;
  __shared__ __align__(1024) float sA[2][128 * 32]; // two 128-row A tiles, 128-byte rows
  __shared__ __align__(1024) float sBm[32 * 32];    // K0 as a 32-row K-major B tile
  __shared__ float sX[2][3][TY][TX];                // y-neighbour exchange
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t tmemBase;

  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = lx + TX * ly;
  // ---- set-up: B tile, mbarrier, tensor memory
  for(int i = tid; i < 32 * 32; i += TX * TY)
  {
    int n = i >> 5, k = i & 31; // logical B[n][k]
    float v = (n < 24 && k < 24) ? K.k[n * 24 + k] : 0.f;
    int chunk = k >> 2, w = k & 3;
    sBm[n * 32 + (((chunk ^ (n & 7)) << 2) | w)] = v;
  }
  if(tid == 0)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if(ly == 0)
  {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 64;" ::"r"(
                     smem_u32(&tmemBase))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmemBase;
  const uint32_t mbarA = smem_u32(&mbar);
  const int tile = ly >> 2;                  // rows 0-3 -> tile 0, rows 4-7 -> tile 1
  const int m = ((ly & 3) << 5) | lx;        // TMEM lane / A row of this element
  float *rowA = &sA[tile][m * 32];
  const uint32_t taddr = tmem + (uint32_t(32 * (ly & 3)) << 16) + uint32_t(32 * tile);

  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TY - 1);
  const int ei = X0 - 1 + lx, ej = Y0 - 1 + ly;
  const int Z0 = blockIdx.z * zchunk;
  const int Z1 = min(Z0 + zchunk, d.sz) - 1;
  const bool col = ei >= 0 && ei < d.nx && ej >= 0 && ej < d.ny;
  const long long sxy = (long long)d.sx * d.sy;
  const long long ld = d.ld;
  const long long nb = col ? (long long)ei + (long long)ej * d.sx : 0;
  const long long qoff[4] = {0, 1, 1 + (long long)d.sx, (long long)d.sx};

  float ub[3][4], ut[3][4], carry[3][4];
#pragma unroll
  for(int c = 0; c < 3; c++)
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      carry[c][q] = 0.f;
      ub[c][q] = 0.f;
    }
  if(col && Z0 - 1 >= 0)
  {
    long long base = nb + (long long)(Z0 - 1) * sxy;
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int q = 0; q < 4; q++)
        ub[c][q] = __ldg(u + c * ld + base + qoff[q]);
  }
  double dot = 0.0;
  uint32_t parity = 0;
  bool failed = false;
  for(int ek = Z0 - 1; ek <= Z1; ++ek)
  {
    const bool lay = col && ek >= 0 && ek < d.nz;
    const bool topok = col && ek + 1 >= 0 && ek + 1 <= d.nz;
    if(topok)
    {
      long long base = nb + (long long)(ek + 1) * sxy;
#pragma unroll
      for(int c = 0; c < 3; c++)
#pragma unroll
        for(int q = 0; q < 4; q++)
          ut[c][q] = __ldg(u + c * ld + base + qoff[q]);
    }
    else
    {
#pragma unroll
      for(int c = 0; c < 3; c++)
#pragma unroll
        for(int q = 0; q < 4; q++)
          ut[c][q] = 0.f;
    }
    const float Ee = lay ? __ldg(E + (long long)ei + (long long)ej * d.nx +
                                 (long long)ek * d.nx * d.ny)
                         : 0.f;
    // ---- A row: K index = local node * 3 + component, 6 chunks of 4
    {
      float v[24];
#pragma unroll
      for(int q = 0; q < 4; q++)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          v[q * 3 + c] = ub[c][q];
          v[12 + q * 3 + c] = ut[c][q];
        }
#pragma unroll
      for(int ch = 0; ch < 6; ch++)
      {
        float4 f4 = make_float4(v[4 * ch], v[4 * ch + 1], v[4 * ch + 2], v[4 * ch + 3]);
        *reinterpret_cast<float4 *>(rowA + ((ch ^ (m & 7)) << 2)) = f4;
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if(tid == 0)
    {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
      for(int t = 0; t < 2; t++)
#pragma unroll
        for(int k = 0; k < 3; k++)
          mma_tf32(tmem + uint32_t(32 * t), sw128_desc(smem_u32(&sA[t][0]) + 32u * k),
                   sw128_desc(smem_u32(&sBm[0]) + 32u * k), k > 0 ? 1u : 0u);
      tc_commit(mbarA);
    }
    // ---- wait for the MMAs (bounded)
    bool ok = false;
    for(unsigned spin = 0; spin < kSpinLimit; spin++)
      if((ok = mbar_try_wait(mbarA, parity)))
        break;
    parity ^= 1u;
    if(__syncthreads_or(!ok))
    {
      if(tid == 0)
        atomicAdd(&g_tc_timeouts, 1u);
      failed = true;
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    float f[24];
    tmem_ld32(taddr, f);
    // rows of the bottom corners: complete the column contribution to plane ek
    float acc[3][4];
#pragma unroll
    for(int q = 0; q < 4; q++)
#pragma unroll
      for(int c = 0; c < 3; c++)
        acc[c][q] = fmaf(Ee, f[q * 3 + c], carry[c][q]);
    if(ek >= Z0)
    {
      float A[3];
      const int buf = ek & 1;
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        A[c] = acc[c][lnodeTc(1, 1)] + __shfl_down_sync(0xffffffffu, acc[c][lnodeTc(0, 1)], 1);
        sX[buf][c][ly][lx] =
            acc[c][lnodeTc(1, 0)] + __shfl_down_sync(0xffffffffu, acc[c][lnodeTc(0, 0)], 1);
      }
      __syncthreads();
      const int ni = ei + 1, nj = ej + 1;
      if(lx < TX - 1 && ly < TY - 1 && ni < d.sx && nj < d.sy)
      {
        const long long node = (long long)ni + (long long)nj * d.sx + (long long)ek * sxy;
        const unsigned fx = __ldg(fix + node);
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          float o = A[c] + sX[buf][c][ly + 1][lx];
          if((fx >> c) & 1u)
            o = 0.f;
          float us = 0.f;
          if(DOT || MODE >= OP_JACOBI)
            us = __ldg(u + c * ld + node);
          if(DOT)
            dot += double(us) * double(o);
          y[c * ld + node] = epilogueTc<MODE>(o, us, c * ld + node, ep);
        }
      }
    }
#pragma unroll
    for(int q = 0; q < 4; q++)
#pragma unroll
      for(int c = 0; c < 3; c++)
        carry[c][q] = Ee * f[12 + q * 3 + c];
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int q = 0; q < 4; q++)
        ub[c][q] = ut[c][q];
  }
  // ---- release tensor memory (also after a timeout)
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if(ly == 0)
  {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 64;" ::"r"(tmem) : "memory");
  }
  if(DOT && !failed)
  {
    double v[1] = {dot};
    block_reduce<1>(v, red, FinStore{dotOut});
  }
}

template <int MODE>
void launch_tc_mode(const Dims &d, const float *K, const float *E, const float *u, float *y,
                    const uint8_t *fix, cudaStream_t s, const OpExtras<float> &x)
{
  KMat<float, 24> km;
  std::copy(K, K + 576, km.k);
  const int target = num_sms() * 4;
  int bx = (d.sx + TX - 2) / (TX - 1), by = (d.sy + TY - 2) / (TY - 1);
  int bz = std::max(1, std::min(d.sz, (target + bx * by - 1) / (bx * by)));
  int zchunk = (d.sz + bz - 1) / bz;
  bz = (d.sz + zchunk - 1) / zchunk;
  dim3 grid(bx, by, bz), block(TX, TY);
  RedScratch red = x.dotRed ? *x.dotRed : RedScratch{};
  Epi<float> ep{x.b, x.dinv, float(x.omega), x.d, float(x.c1), float(x.c2)};
  if(x.dotRed)
  {
    ICB_REQUIRE(bx * by * bz <= red.maxBlocks, "reduction scratch too small");
    k_matvec_h8_tc<true, MODE><<<grid, block, 0, s>>>(km, d, zchunk, E, u, y, fix, red, x.dotOut,
                                                      x.gate, x.gateConv, ep);
  }
  else
    k_matvec_h8_tc<false, MODE><<<grid, block, 0, s>>>(km, d, zchunk, E, u, y, fix, red, x.dotOut,
                                                       x.gate, x.gateConv, ep);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
} // namespace

void launch_op_tc(const Dims &d, const float *K, const float *E, const float *u, float *y,
                  const uint8_t *fix, cudaStream_t s, const OpExtras<float> &x)
{
  ICB_REQUIRE(d.dim == 3, "the tensor-core operator is for Hex8 grids");
  if(x.mode == OP_APPLY)
    launch_tc_mode<OP_APPLY>(d, K, E, u, y, fix, s, x);
  else if(x.mode == OP_RESIDUAL)
    launch_tc_mode<OP_RESIDUAL>(d, K, E, u, y, fix, s, x);
  else if(x.mode == OP_JACOBI)
    launch_tc_mode<OP_JACOBI>(d, K, E, u, y, fix, s, x);
  else
    launch_tc_mode<OP_CHEB>(d, K, E, u, y, fix, s, x);
}

unsigned tc_timeouts()
{
  unsigned h = 0;
  cudaMemcpyFromSymbol(&h, g_tc_timeouts, sizeof(unsigned));
  return h;
}

} // namespace icb
