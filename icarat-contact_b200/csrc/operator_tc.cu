// operator_tc.cu -- the FP32 Hex8 element operator with the element
// contraction on the 5th-generation tensor cores (tcgen05, kind::tf32).
//
// Same decomposition as k_matvec_h8 (operator.cu), with smaller tiles: a CTA
// of 32x4 threads owns a 31x3 tile of output nodes and marches up a chunk of z
// planes, one thread per element column, bottom-corner values and top-corner
// contributions kept in registers (4 such CTAs run per SM: more independent
// layer chains than 2 CTAs of 32x8, measured 5 % faster at 384x128x128).  Per
// element layer the 128 elements of the CTA form one 128-row MMA tile:
//   A (128 x 24, K-major, TF32): row m = the element's 8 corner
//     displacements x 3 components, written by its thread into shared memory
//     in the SWIZZLE_128B K-major layout (16-byte chunk c of row m stored at
//     chunk c ^ (m & 7) of the row's 128-byte line);
//   B (32 x 24, K-major): the unit element matrix K0 (rows 24..31 zero);
//   D (128 x 32, FP32) in tensor memory: D[m][n] = (K0 u_m)[n].
// One thread issues the 3 tcgen05.mma (K = 8 each) and commits them to an
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
#include <atomic>

#include "icb_internal.hpp"
#include "reduce.cuh"

namespace icb
{
__device__ unsigned g_tc_timeouts = 0;

namespace
{
constexpr int TX = 32, TY = 4, TY1 = TY + 1;
constexpr int kTiles = TY / 4;                                 // 128-row MMA tiles per layer
constexpr int kTmemCols = kTiles * 32 > 32 ? kTiles * 32 : 32; // power of 2, >= 32
constexpr unsigned kSpinLimit = 1u << 22; // default try_wait polls before a CTA gives up

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
  __syncwarp(); // .sync.aligned: the whole warp executes the load together
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
               "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
               "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
               "tcgen05.wait::ld.sync.aligned;\n"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                 "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]),
                 "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                 "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
                 "=r"(r[30]), "=r"(r[31])
               : "r"(taddr)
               : "memory");
#pragma unroll
  for(int i = 0; i < 24; i++)
    v[i] = __uint_as_float(r[i]);
}

/// bounded wait on an mbarrier phase; false when `limit` polls ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint32_t mbar, uint32_t parity, unsigned limit)
{
  for(unsigned spin = 0; spin < limit; spin++)
    if(mbar_try_wait(mbar, parity))
      return true;
  return false;
}

__device__ __forceinline__ void cp_async4(uint32_t dst, const float *src)
{
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait()
{
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- staged node planes ------------------------------------------------------
// A CTA's element tile (32 x TY element columns) touches a 33 x (TY + 1)
// block of nodes in every z plane: 3 components x (TY + 1) rows x 33 nodes
// per plane.  All the CTA's threads copy a plane into a ring of kStages shared-memory slots with
// 4-byte cp.async copies (a warp copies 32 consecutive nodes of a row, so its
// copies coalesce), kStages - 2 planes ahead of the plane the tile reads.
// Nodes outside the grid are not copied and never read.
constexpr int kStages = 4;
constexpr int kRow = TX + 1;              // nodes per staged row
constexpr int kPlaneF = 3 * TY1 * kRow;
constexpr int kBlocksPerSm = 4;

struct TcSmem
{
  float A[kTiles][128 * 32]; // 128-row A tiles (SWIZZLE_128B, K-major)
  float B[32 * 32];          // K0, 32-row K-major B tile
  float P[kStages][kPlaneF]; // staged node planes
  float X[2][3][TY][TX];     // y-neighbour exchange
  unsigned long long mbarMma;
  uint32_t tmemBase;
};

/// the work items of the persistent operator: (tile x, tile y, z chunk)
struct TcWork
{
  int bx, by, bz, zchunk, items;
  unsigned spin; ///< polls of an MMA wait before the CTA gives up (icb option tc_spin_limit)
  __device__ __forceinline__ void item(int it, int &X0, int &Y0, int &Z0, int &Z1, const Dims &d) const
  {
    int tx = it % bx, r = it / bx;
    int ty = r % by, tz = r / by;
    X0 = tx * (TX - 1);
    Y0 = ty * (TY - 1);
    Z0 = tz * zchunk;
    Z1 = min(Z0 + zchunk, d.sz) - 1;
  }
};

/// the plane cursor: planes are staged in order across this CTA's items
/// (item blockIdx.x, blockIdx.x + gridDim.x, ...; an item of T layers has
/// planes z = Z0 - 1 ... Z1 + 1)
struct PlaneCursor
{
  int it, r;
  long long g;           // global index of the plane, its ring slot is g % kStages
  int X0, Y0, Z0, Z1;    // the item's geometry
  __device__ __forceinline__ void start(int item, const TcWork &W, const Dims &d)
  {
    it = item;
    r = 0;
    if(it < W.items)
      W.item(it, X0, Y0, Z0, Z1, d);
  }
};

/// this thread's share of a staged plane: node column lx of the staged rows
/// R = ly + 8 s (s = 0..3, R < 27; row R is component R / 9, node row R % 9),
/// plus column 32 for the lx == 0 threads.  Offsets inside one SoA vector
/// are 32-bit (the host checks 3 ld < 2^31).
__device__ __forceinline__ void stage_plane(TcSmem &S, const PlaneCursor &pc, const TcWork &W,
                                            const Dims &d, const float *__restrict__ u, int lx,
                                            int ly)
{
  if(pc.it >= W.items)
    return;
  const int k = pc.Z0 - 1 + pc.r;
  if(k < 0 || k > d.nz)
    return;
  const int i = pc.X0 - 1 + lx;
  const bool iok = i >= 0 && i <= d.nx, i2ok = lx == 0 && pc.X0 + TX - 1 <= d.nx;
  const int ld = int(d.ld);
  const int base = k * d.sx * d.sy + (pc.Y0 - 1) * d.sx + i;
  const uint32_t dst = smem_u32(S.P[pc.g % kStages]) + uint32_t(lx) * 4u;
#pragma unroll
  for(int s = 0; s < 4; s++)
  {
    const int R = ly + TY * s;
    if(R >= 3 * TY1)
      break;
    const int c = R / TY1, jj = R - c * TY1;
    const int j = pc.Y0 - 1 + jj;
    if(j < 0 || j > d.ny)
      continue;
    const uint32_t drow = dst + uint32_t(R * kRow) * 4u;
    const int off = c * ld + jj * d.sx + base;
    if(iok)
      cp_async4(drow, u + off);
    if(i2ok)
      cp_async4(drow + uint32_t(TX) * 4u, u + off + TX);
  }
}

__device__ __forceinline__ void advance(PlaneCursor &pc, const TcWork &W, const Dims &d)
{
  pc.g++;
  if(++pc.r > pc.Z1 - pc.Z0 + 2)
    pc.start(pc.it + gridDim.x, W, d);
}

/// one layer's operands besides the staged displacements
template <bool DOT, int MODE> struct LayerOps
{
  float Ee = 0.f;
  unsigned fx = 0;
  float us[3] = {0.f, 0.f, 0.f}; // halo columns only
  float bb[3] = {0.f, 0.f, 0.f}, dv[3] = {0.f, 0.f, 0.f}, dp[3] = {0.f, 0.f, 0.f};
  __device__ __forceinline__ void load(bool lay, const float *__restrict__ E, long long e, bool outp,
                                       const uint8_t *__restrict__ fix,
                                       const float *__restrict__ u, const float *y,
                                       const Epi<float> &ep, long long node, long long ld,
                                       bool col)
  {
    Ee = lay ? __ldg(E + e) : 0.f;
    if(!outp)
      return;
    fx = __ldg(fix + node);
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      if((DOT || MODE >= OP_JACOBI) && !col)
        us[c] = __ldg(u + c * ld + node);
      if(MODE != OP_APPLY)
        bb[c] = __ldg(ep.b + c * ld + node);
      if(MODE >= OP_JACOBI)
        dv[c] = __ldg(ep.dinv + c * ld + node);
      if(MODE == OP_CHEB && ep.c1 != 0.f)
        dp[c] = y[c * ld + node]; // the previous iterate (y is written after)
    }
  }
};

template <bool DOT, int MODE>
__global__ void __launch_bounds__(TX *TY, kBlocksPerSm)
    k_matvec_h8_tc(const KMat<float, 24> K, const Dims d, const TcWork W,
                   const float *__restrict__ E, const float *__restrict__ u,
                   float *__restrict__ y, const uint8_t *__restrict__ fix, RedScratch red,
                   double *dotOut, const KState *gate, const int gateConv, const Epi<float> ep)
{
  if(gate && (gate->stop || (gateConv && gate->conv)))
    return;
  extern __shared__ __align__(1024) unsigned char smraw[];
  // the swizzled A and B tiles need 1024-byte aligned shared addresses
  TcSmem &S = *reinterpret_cast<TcSmem *>(smraw + ((1024u - (smem_u32(smraw) & 1023u)) & 1023u));

  const int lx = threadIdx.x, ly = threadIdx.y;
  const int tid = lx + TX * ly;
  // ---- set-up: B tile, barrier, tensor memory, the first planes
  for(int i = tid; i < 32 * 32; i += TX * TY)
  {
    int n = i >> 5, k = i & 31; // logical B[n][k]
    float v = (n < 24 && k < 24) ? K.k[n * 24 + k] : 0.f;
    int chunk = k >> 2, w = k & 3;
    S.B[n * 32 + (((chunk ^ (n & 7)) << 2) | w)] = v;
  }
  if(tid == 0)
  {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.mbarMma)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if(ly == 0)
  {
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(&S.tmemBase)),
                 "n"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  // planes 0 .. kStages - 2 in flight; plane 0 complete before the barrier
  PlaneCursor pc;
  pc.g = 0;
  pc.start(blockIdx.x, W, d);
#pragma unroll
  for(int s = 0; s < kStages - 1; s++)
  {
    stage_plane(S, pc, W, d, u, lx, ly);
    cp_async_commit();
    advance(pc, W, d);
  }
  cp_async_wait<kStages - 2>();
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = S.tmemBase;
  const uint32_t mbarA = smem_u32(&S.mbarMma);
  const int tile = ly >> 2;           // element rows 4t .. 4t+3 form MMA tile t
  const int m = ((ly & 3) << 5) | lx; // TMEM lane / A row of this element
  float *rowA = &S.A[tile][m * 32];
  const uint32_t taddr = tmem + (uint32_t(32 * (ly & 3)) << 16) + uint32_t(32 * tile);
  const long long sxy = (long long)d.sx * d.sy;
  const long long ld = d.ld;

  // Every plane read is one step: read plane `cons` (made complete and
  // visible by the previous step's barrier), stage plane cons + kStages - 1
  // into the slot of plane cons - 1, wait for this thread's copies of plane
  // cons + 1, barrier.
  long long cons = 0;
  auto step_stage = [&]() {
    stage_plane(S, pc, W, d, u, lx, ly);
    cp_async_commit();
    advance(pc, W, d);
    cp_async_wait<kStages - 2>();
    cons++;
  };

  double dot = 0.0;
  uint32_t parity = 0;
  bool failed = false;
  for(int it = blockIdx.x; it < W.items && !failed; it += gridDim.x)
  {
    int X0, Y0, Z0, Z1;
    W.item(it, X0, Y0, Z0, Z1, d);
    const int ei = X0 - 1 + lx, ej = Y0 - 1 + ly;
    const bool col = ei >= 0 && ei < d.nx && ej >= 0 && ej < d.ny;
    // node (ei + a, ej + h) of a staged plane, component c
    auto at = [&](const float *plane, int c, int h, int a) {
      return plane[(c * TY1 + ly + h) * kRow + lx + a];
    };

    float ub[3][4], carry[3][4];
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int q = 0; q < 4; q++)
      {
        carry[c][q] = 0.f;
        ub[c][q] = 0.f;
      }
    // plane 0 of the item (z = Z0 - 1) seeds the bottom corners
    {
      const float *pl = S.P[cons % kStages];
      if(col && Z0 - 1 >= 0)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          // corners q: 0 (i,j) 1 (i+1,j) 2 (i+1,j+1) 3 (i,j+1)
          ub[c][0] = at(pl, c, 0, 0);
          ub[c][1] = at(pl, c, 0, 1);
          ub[c][2] = at(pl, c, 1, 1);
          ub[c][3] = at(pl, c, 1, 0);
        }
      step_stage();
      __syncthreads();
    }
    // per-layer operands are loaded one layer ahead (the element modulus, the
    // output node's Dirichlet bits and the smoother's vectors); u at the
    // output node is the column's own bottom corner 2 (ub[c][2]) except in
    // the halo columns outside the grid, which load it
    const int ni = ei + 1, nj = ej + 1;
    const bool outCol = lx < TX - 1 && ly < TY - 1 && ni < d.sx && nj < d.sy;
    const long long eBase = (long long)ei + (long long)ej * d.nx;
    const long long nxy = (long long)d.nx * d.ny;
    const long long nBase = (long long)ni + (long long)nj * d.sx;
    LayerOps<DOT, MODE> cur, nxt;
    cur.load(col && Z0 - 1 >= 0 && Z0 - 1 < d.nz, E, eBase + (long long)(Z0 - 1) * nxy, false, fix,
             u, y, ep, nBase, ld, col);
    for(int ek = Z0 - 1; ek <= Z1; ++ek)
    {
      const int kt = ek + 1;
      const bool topok = col && kt <= d.nz;
      const bool outp = ek >= Z0 && outCol;
      const long long node = nBase + (long long)ek * sxy;
      if(ek + 1 <= Z1)
        nxt.load(col && ek + 1 < d.nz, E, eBase + (long long)(ek + 1) * nxy, outCol, fix, u, y, ep,
                 nBase + (long long)(ek + 1) * sxy, ld, col);
      const float Ee = cur.Ee;
      // ---- top corners from the staged plane
      float ut[3][4];
      {
        const float *pl = S.P[cons % kStages];
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          ut[c][0] = topok ? at(pl, c, 0, 0) : 0.f;
          ut[c][1] = topok ? at(pl, c, 0, 1) : 0.f;
          ut[c][2] = topok ? at(pl, c, 1, 1) : 0.f;
          ut[c][3] = topok ? at(pl, c, 1, 0) : 0.f;
        }
      }
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
      step_stage();
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      // one thread issues the six MMAs of this layer
      if(tid == 0)
      {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
#pragma unroll
        for(int t = 0; t < kTiles; t++)
#pragma unroll
          for(int k = 0; k < 3; k++)
            mma_tf32(tmem + uint32_t(32 * t), sw128_desc(smem_u32(&S.A[t][0]) + 32u * k),
                     sw128_desc(smem_u32(&S.B[0]) + 32u * k), k > 0 ? 1u : 0u);
        tc_commit(mbarA);
      }
      // one thread waits for the MMAs; the barrier hands the result to all
      bool ok = true;
      if(tid == 0)
      {
        ok = mbar_wait_bounded(mbarA, parity, W.spin);
        // a CTA that gives up still lets the MMAs it issued finish (again
        // bounded) before it releases the tensor memory they write
        if(!ok)
          mbar_wait_bounded(mbarA, parity, kSpinLimit);
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      }
      parity ^= 1u;
      if(__syncthreads_or(!ok))
      {
        failed = true;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      float f[24];
      tmem_ld32(taddr, f);
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
          S.X[buf][c][ly][lx] =
              acc[c][lnodeTc(1, 0)] + __shfl_down_sync(0xffffffffu, acc[c][lnodeTc(0, 0)], 1);
        }
        __syncthreads();
        if(outp)
        {
#pragma unroll
          for(int c = 0; c < 3; c++)
          {
            float o = A[c] + S.X[buf][c][ly + 1][lx];
            if((cur.fx >> c) & 1u)
              o = 0.f;
            const float us = col ? ub[c][2] : cur.us[c];
            if(DOT)
              dot += double(us) * double(o);
            float outv = o;
            if(MODE == OP_RESIDUAL)
              outv = cur.bb[c] - o;
            else if(MODE == OP_JACOBI)
              outv = us + ep.omega * cur.dv[c] * (cur.bb[c] - o);
            else if(MODE == OP_CHEB)
            {
              float dn = ep.c2 * cur.dv[c] * (cur.bb[c] - o);
              if(ep.c1 != 0.f)
                dn += ep.c1 * (us - cur.dp[c]);
              outv = us + dn;
            }
            y[c * ld + node] = outv;
          }
        }
      }
#pragma unroll
      for(int q = 0; q < 4; q++)
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          carry[c][q] = Ee * f[12 + q * 3 + c];
          ub[c][q] = ut[c][q];
        }
      cur = nxt;
    }
  }
  // copies still in flight land before the shared memory is released
  cp_async_wait<0>();
  if(failed && tid == 0)
    atomicAdd(&g_tc_timeouts, 1u);
  // ---- release tensor memory (also after a timeout)
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if(ly == 0)
  {
    __syncwarp();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "n"(kTmemCols)
                 : "memory");
  }
  if(DOT)
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
  auto kern = x.dotRed ? k_matvec_h8_tc<true, MODE> : k_matvec_h8_tc<false, MODE>;
  // the shared-memory opt-in is a per-device attribute: set it on every call
  // (same value from every thread, so concurrent launches never see less)
  const int smem = int(sizeof(TcSmem)) + 1024;
  ICB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  ICB_REQUIRE(3 * d.ld < (1LL << 31), "grid too large for the tensor-core operator's 32-bit offsets");
  TcWork w;
  w.bx = (d.sx + TX - 2) / (TX - 1);
  w.by = (d.sy + TY - 2) / (TY - 1);
  const int slots = num_sms() * kBlocksPerSm;
  // about four z chunks per resident CTA, chunks of at least 4 layers
  const int wantBz = std::max(1, (4 * slots + w.bx * w.by - 1) / (w.bx * w.by));
  w.zchunk = std::max(4, (d.sz + wantBz - 1) / wantBz);
  w.bz = (d.sz + w.zchunk - 1) / w.zchunk;
  w.items = w.bx * w.by * w.bz;
  w.spin = tc_spin_limit();
  const int grid = std::min(w.items, slots);
  RedScratch red = x.dotRed ? *x.dotRed : RedScratch{};
  Epi<float> ep{x.b, x.dinv, float(x.omega), float(x.c1), float(x.c2)};
  if(x.dotRed)
    ICB_REQUIRE(grid <= red.maxBlocks, "reduction scratch too small");
  kern<<<grid, dim3(TX, TY), smem, s>>>(km, d, w, E, u, y, fix, red, x.dotOut, x.gate,
                                         x.gateConv, ep);
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

static std::atomic<unsigned> g_tc_spin{kSpinLimit};
unsigned tc_spin_limit() { return g_tc_spin.load(); }
void set_tc_spin_limit(unsigned polls) { g_tc_spin = polls; }

unsigned tc_timeouts()
{
  unsigned h = 0;
  cudaMemcpyFromSymbol(&h, g_tc_timeouts, sizeof(unsigned));
  return h;
}

} // namespace icb
