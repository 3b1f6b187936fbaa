// operator.cu -- matrix-free element-by-element stiffness operator on the
// structured Q4 / Hex8 grids, its diagonal, SIMP moduli and sensitivities.
//
// Replaces the assembled path of ICARAT: LinearElastic::makeKeFint
// (src/problem/elasticity.cpp:210-254) + assembling()
// (src/misc/assembling.hpp:17-38) + SparseMatrix::setFromTriplets
// (src/analysis/linear.hpp:155-161) + Eigen's SpMV inside ConjugateGradient.
// On a uniform grid Ke = E(rho_e) K0, so K(rho) u = sum_e E_e K0 u_e; nothing
// is assembled.
//
// Layout in HBM: displacement-like vectors are SoA, one plane per component,
// node index n = i + j*sx + k*sx*sy (MeshIcarat numbering), component c at
// c*ld + n.  Constrained DOFs are masked by a per-node bit mask (bit c set:
// component c fixed), so the operator acts on the free space exactly as the
// eliminated numeq system of assembling() does.
//
// Hex8 kernel: a CTA owns a 31x7 tile of output nodes in x-y and marches up a
// chunk of z planes.  Each thread owns one element column (the tile's
// elements plus a one-element halo on the low side), keeps the 4 bottom
// corner displacements of its current element in registers (they are the top
// corners of the element below) and carries the element's top-corner
// contributions up to the next plane in registers, so the vertical sharing
// needs no memory at all.  The four columns around a node are summed with one
// warp shuffle (x) and one shared-memory exchange (y).  No atomics, no
// colouring, deterministic results.
#include "icb_internal.hpp"
#include "batchq.cuh"
#include "reduce.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <mutex>
#include <unordered_map>
#include <type_traits>

namespace icb
{
namespace
{
constexpr int TX = 32; // threads along x (one warp)
constexpr int TY3 = 8; // warps along y (3D)
constexpr int TY2 = 4; // warps per CTA (2D: independent x strips)

/// local node index of the corner with offsets (a,b) in a plane (meshBox order)
__host__ __device__ constexpr int lnode(int a, int b) { return (a ^ b) + 2 * b; }

/// fused output stage: y = Au (OP_APPLY), b - Au (OP_RESIDUAL), a damped
/// Jacobi sweep u + w D^-1 (b - Au) (OP_JACOBI) or a three-term Chebyshev
/// step (OP_CHEB, which reads the previous iterate from y at this DOF before
/// overwriting it); Au is already 0 on constrained DOFs and so are b and D^-1.
template <typename T, int MODE>
__device__ __forceinline__ T epilogue(T Au, T uself, long long i, const Epi<T> &ep, const T *y)
{
  if(MODE == OP_APPLY)
    return Au;
  T r = __ldg(ep.b + i) - Au;
  if(MODE == OP_RESIDUAL)
    return r;
  if(MODE == OP_JACOBI)
    return uself + ep.omega * __ldg(ep.dinv + i) * r;
  T dn = ep.c2 * __ldg(ep.dinv + i) * r;
  if(ep.c1 != T(0))
    dn += ep.c1 * (uself - y[i]);
  return uself + dn;
}

/// upper triangle of the symmetric 24x24 K0, row-major (300 doubles).  The
/// full FP64 matrix (4608 bytes) is past the 4 KB of kernel parameters that
/// live in the constant bank; packed, every entry stays a constant operand of
/// its FMA instead of a value the kernel must load into a register.
struct KSym24
{
  double k[300];
};
__host__ __device__ constexpr int symIdx(int r, int c)
{
  return r <= c ? r * 24 - r * (r - 1) / 2 + (c - r) : c * 24 - c * (c - 1) / 2 + (r - c);
}
template <typename T>
__device__ __forceinline__ T kget(const KMat<T, 24> &K, int r, int c)
{
  return K.k[r * 24 + c];
}
__device__ __forceinline__ double kget(const KSym24 &K, int r, int c) { return K.k[symIdx(r, c)]; }

// ----------------------------------------------------------------- Hex8 ----
template <typename T, typename KT, int TYK, bool DOT, int MODE>
__global__ void __launch_bounds__(TX *TYK)
    k_matvec_h8(const KT K, const Dims d, const int zchunk,
                const T *__restrict__ E, const T *__restrict__ u, T *__restrict__ y,
                const uint8_t *__restrict__ fix, RedScratch red, double *dotOut,
                const KState *gate, const int gateConv, const Epi<T> ep)
{
  if(gate && (gate->stop || (gateConv && gate->conv)))
    return;
  __shared__ T sB[2][3][TYK][TX];
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TYK - 1);
  const int ei = X0 - 1 + lx, ej = Y0 - 1 + ly;
  const int Z0 = blockIdx.z * zchunk;
  const int Z1 = min(Z0 + zchunk, d.sz) - 1;
  const bool col = ei >= 0 && ei < d.nx && ej >= 0 && ej < d.ny;
  const long long sxy = (long long)d.sx * d.sy;
  const long long ld = d.ld;
  const long long nb = col ? (long long)ei + (long long)ej * d.sx : 0;
  // corner q (lnode order) -> node offset within a plane
  const long long qoff[4] = {0, 1, 1 + (long long)d.sx, (long long)d.sx};

  T ub[3][4], ut[3][4], carry[3][4];
#pragma unroll
  for(int c = 0; c < 3; c++)
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      carry[c][q] = T(0);
      ub[c][q] = T(0);
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
          ut[c][q] = T(0);
    }
    const T Ee = lay ? __ldg(E + (long long)ei + (long long)ej * d.nx +
                             (long long)ek * d.nx * d.ny)
                     : T(0);
    // rows of the bottom corners: complete the column contribution to plane ek
    T acc[3][4];
#pragma unroll
    for(int q = 0; q < 4; q++)
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const int row = q * 3 + c;
        T s = T(0);
#pragma unroll
        for(int q2 = 0; q2 < 4; q2++)
#pragma unroll
          for(int c2 = 0; c2 < 3; c2++)
            s = fma(kget(K, row, q2 * 3 + c2), ub[c2][q2], s);
#pragma unroll
        for(int q2 = 0; q2 < 4; q2++)
#pragma unroll
          for(int c2 = 0; c2 < 3; c2++)
            s = fma(kget(K, row, 12 + q2 * 3 + c2), ut[c2][q2], s);
        acc[c][q] = fma(Ee, s, carry[c][q]);
      }
    if(ek >= Z0)
    {
      T A[3];
      const int buf = ek & 1;
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        A[c] = acc[c][lnode(1, 1)] + __shfl_down_sync(0xffffffffu, acc[c][lnode(0, 1)], 1);
        sB[buf][c][ly][lx] =
            acc[c][lnode(1, 0)] + __shfl_down_sync(0xffffffffu, acc[c][lnode(0, 0)], 1);
      }
      __syncthreads();
      const int ni = ei + 1, nj = ej + 1;
      if(lx < TX - 1 && ly < TYK - 1 && ni < d.sx && nj < d.sy)
      {
        const long long node = (long long)ni + (long long)nj * d.sx + (long long)ek * sxy;
        const unsigned f = __ldg(fix + node);
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          T o = A[c] + sB[buf][c][ly + 1][lx];
          if((f >> c) & 1u)
            o = T(0);
          // the node's own input value: read it here, the thread owning this
          // node may be a halo column (i = 0 or j = 0) with no element
          T us = T(0);
          if(DOT || MODE >= OP_JACOBI)
            us = __ldg(u + c * ld + node);
          if(DOT)
            dot += double(us) * double(o);
          y[c * ld + node] = epilogue<T, MODE>(o, us, c * ld + node, ep, y);
        }
      }
    }
    // rows of the top corners: carried to plane ek+1
#pragma unroll
    for(int q = 0; q < 4; q++)
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const int row = 12 + q * 3 + c;
        T s = T(0);
#pragma unroll
        for(int q2 = 0; q2 < 4; q2++)
#pragma unroll
          for(int c2 = 0; c2 < 3; c2++)
            s = fma(kget(K, row, q2 * 3 + c2), ub[c2][q2], s);
#pragma unroll
        for(int q2 = 0; q2 < 4; q2++)
#pragma unroll
          for(int c2 = 0; c2 < 3; c2++)
            s = fma(kget(K, row, 12 + q2 * 3 + c2), ut[c2][q2], s);
        carry[c][q] = Ee * s;
      }
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int q = 0; q < 4; q++)
        ub[c][q] = ut[c][q];
  }
  if(DOT)
  {
    double v[1] = {dot};
    block_reduce<1>(v, red, FinStore{dotOut});
  }
}

// ------------------------------------------------ Hex8, corner-mode form ----
// The 8 corners of a box element are the vertices of a unit cube, so the
// 8-point Hadamard transform  h_s = sum_a (-1)^(s.o_a) u_a  (s, o_a in {0,1}^3)
// takes a component's corner values to the element's corner modes: the mean,
// the three first differences, the three mixed second differences and the
// xyz twist.  For an isotropic material on a box (every Hex8 element of the
// structured grids) K0 is block-diagonal in that basis: the 24 x 24 matrix
// Kt = H K0 H / 64 (H = H8 (x) I3, DOF s*3+c) has 45 nonzeros in 11 dense
// blocks -- {e_xx, e_yy, e_zz}, the three shear pairs, four blocks of mixed
// second differences and the three twist modes; the rigid translations (s = 0)
// are its null rows.  So  K0 u = H (Kt (H u))  costs two butterflies and 45
// FMAs instead of 576.  The host builds Kt from K0 and checks that every entry
// outside the blocks vanishes (to rounding); an element matrix that fails the
// check runs on the dense kernel above.
//
// The marching column shares the butterflies between layers: the x-y half of
// the transform is applied once per node plane (the top plane of element k is
// the bottom plane of element k+1), and the top-face result is carried up in
// x-y mode form, where the next element's bottom-face result is added to it
// before the one inverse x-y butterfly per plane.
constexpr int kModalNnz = 45;
template <typename T> struct KModal
{
  T v[kModalNnz]; ///< Kt entries, block by block, row-major within a block
};
/// the 11 blocks of Kt (modal DOF s*3+c), listed by their modal DOFs
struct ModalBlocks
{
  int n[11];
  int dof[11][3];
};
__host__ __device__ constexpr ModalBlocks modal_blocks()
{
  return ModalBlocks{{3, 2, 2, 2, 2, 2, 3, 2, 1, 1, 1},
                     {{3, 7, 14},
                      {4, 6, 0},
                      {5, 12, 0},
                      {8, 13, 0},
                      {9, 20, 0},
                      {10, 17, 0},
                      {11, 16, 18},
                      {15, 19, 0},
                      {21, 0, 0},
                      {22, 0, 0},
                      {23, 0, 0}}};
}

/// yh = Kt uh, block B onwards (OFF: offset of block B in K.v); every index
/// is a compile-time constant, so uh and yh stay in registers
template <int B, int OFF, typename T>
__device__ __forceinline__ void modal_blocks_apply(const KModal<T> &K, const T (&uh)[24],
                                                   T (&yh)[24])
{
  if constexpr(B < 11)
  {
    constexpr ModalBlocks MB = modal_blocks();
    constexpr int n = MB.n[B];
    constexpr int a = MB.dof[B][0], b = MB.dof[B][1], c = MB.dof[B][2];
    if constexpr(n == 1)
      yh[a] = K.v[OFF] * uh[a];
    else if constexpr(n == 2)
    {
      yh[a] = fma(K.v[OFF + 1], uh[b], K.v[OFF] * uh[a]);
      yh[b] = fma(K.v[OFF + 3], uh[b], K.v[OFF + 2] * uh[a]);
    }
    else
    {
      yh[a] = fma(K.v[OFF + 2], uh[c], fma(K.v[OFF + 1], uh[b], K.v[OFF] * uh[a]));
      yh[b] = fma(K.v[OFF + 5], uh[c], fma(K.v[OFF + 4], uh[b], K.v[OFF + 3] * uh[a]));
      yh[c] = fma(K.v[OFF + 8], uh[c], fma(K.v[OFF + 7], uh[b], K.v[OFF + 6] * uh[a]));
    }
    modal_blocks_apply<B + 1, OFF + n * n>(K, uh, yh);
  }
}

/// x-y half of the transform on one plane, corners in lnode order
/// (q0 (0,0), q1 (1,0), q2 (1,1), q3 (0,1)) -> modes h[sx + 2 sy]
template <typename T> __device__ __forceinline__ void plane_modes(const T u[4], T h[4])
{
  const T a = u[0] + u[1], b = u[0] - u[1], c = u[3] + u[2], e = u[3] - u[2];
  h[0] = a + c;
  h[1] = b + e;
  h[2] = a - c;
  h[3] = b - e;
}
/// its inverse up to a factor 4 (the factors of both butterflies, 64 in all,
/// are folded into Kt): modes -> corners
template <typename T> __device__ __forceinline__ void plane_corners(const T h[4], T u[4])
{
  const T p = h[0] + h[2], m = h[0] - h[2], r = h[1] + h[3], n = h[1] - h[3];
  u[0] = p + r;
  u[1] = p - r;
  u[2] = m - n;
  u[3] = m + n;
}

/// the epilogue's per-node inputs (the node's own value, b, D^-1, the
/// previous Chebyshev iterate), loaded ahead of their use
template <typename T> struct EpiIn
{
  T b[3], dinv[3], d[3], us[3];
};

/// dynamic shared memory of k_matvec_h8m: the carry, and for FP64 the
/// bottom plane's modes (12 values per thread each)
template <typename T, int TYK> constexpr int h8m_smem_bytes()
{
  return int(sizeof(T)) * 12 * TYK * TX * (sizeof(T) == 8 ? 2 : 1);
}

/// Each layer issues the loads of the next layer's top plane and modulus
/// ahead of its own element work, so the arithmetic covers their latency.
/// The carried top-face result lives in shared memory (each thread its own
/// 12 values), which keeps the registers for the prefetched plane.
template <typename T, int TYK, bool DOT, int MODE, int MINB>
__global__ void __launch_bounds__(TX *TYK, MINB)
    k_matvec_h8m(const KModal<T> K, const Dims d, const int zchunk,
                 const T *__restrict__ E, const T *__restrict__ u, T *__restrict__ y,
                 const uint8_t *__restrict__ fix, RedScratch red, double *dotOut,
                 const KState *gate, const int gateConv, const Epi<T> ep)
{
  if(gate && (gate->stop || (gateConv && gate->conv)))
    return;
  // FP64 also keeps the bottom plane's modes in shared memory (kSmemModes);
  // carry and modes take h8m_smem_bytes of dynamic shared memory
  constexpr bool kSmemModes = sizeof(T) == 8;
  extern __shared__ __align__(16) unsigned char h8m_dyn[];
  auto sC = reinterpret_cast<T(*)[TYK][TX]>(h8m_dyn);
  auto sH = reinterpret_cast<T(*)[TYK][TX]>(h8m_dyn + sizeof(T) * 12 * TYK * TX);
  __shared__ T sB[2][3][TYK][TX];
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (TYK - 1);
  const int ei = X0 - 1 + lx, ej = Y0 - 1 + ly;
  const int Z0 = blockIdx.z * zchunk;
  const int Z1 = min(Z0 + zchunk, d.sz) - 1;
  const bool col = ei >= 0 && ei < d.nx && ej >= 0 && ej < d.ny;
  const long long sxy = (long long)d.sx * d.sy, exy = (long long)d.nx * d.ny;
  const long long ld = d.ld;
  // component c of this column's corner q in node plane k: u[c*ld + nb + qoff[q] + k*sxy]
  const long long nb = col ? (long long)ei + (long long)ej * d.sx : 0;
  const long long qoff[4] = {0, 1, 1 + (long long)d.sx, (long long)d.sx};
  const long long eb = col ? (long long)ei + (long long)ej * d.nx : 0;
  auto load_plane = [&](int k, T (&v)[3][4]) {
    const bool ok = col && k >= 0 && k <= d.nz;
    const T *p = u + nb + (long long)k * sxy;
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int q = 0; q < 4; q++)
        v[c][q] = ok ? __ldg(p + c * ld + qoff[q]) : T(0);
  };
  auto load_E = [&](int k) {
    return col && k >= 0 && k < d.nz ? __ldg(E + eb + (long long)k * exy) : T(0);
  };

  // the bottom plane's x-y modes; the top-face result carried up (sC)
  T bh[3][4], nxt[3][4];
  {
    T v[3][4];
    load_plane(Z0 - 1, v);
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      plane_modes(v[c], bh[c]);
#pragma unroll
      for(int q = 0; q < 4; q++)
      {
        sC[c * 4 + q][ly][lx] = T(0);
        if(kSmemModes)
          sH[c * 4 + q][ly][lx] = bh[c][q];
      }
    }
  }
  load_plane(Z0, nxt);
  T Enxt = load_E(Z0 - 1);
  double dot = 0.0;
  for(int ek = Z0 - 1; ek <= Z1; ++ek)
  {
    T th[3][4];
#pragma unroll
    for(int c = 0; c < 3; c++)
      plane_modes(nxt[c], th[c]);
    const T Ee = Enxt;
    // next layer's inputs: FP32 at the top of the layer, FP64 after the
    // element product (its registers are the limit)
    constexpr bool kLateNext = sizeof(T) == 8;
    if(!kLateNext)
    {
      load_plane(ek + 2, nxt);
      Enxt = load_E(ek + 1);
    }
    const bool out = ek >= Z0;
    const int ni = ei + 1, nj = ej + 1;
    const bool own = out && lx < TX - 1 && ly < TYK - 1 && ni < d.sx && nj < d.sy;
    const long long node = (long long)ni + (long long)nj * d.sx + (long long)ek * sxy;
    unsigned f = 0;
    EpiIn<T> in;
    auto load_in = [&]() {
      if(own)
      {
        f = __ldg(fix + node);
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          if(DOT || MODE >= OP_JACOBI)
            in.us[c] = __ldg(u + c * ld + node);
          if(MODE != OP_APPLY)
            in.b[c] = __ldg(ep.b + c * ld + node);
          if(MODE >= OP_JACOBI)
            in.dinv[c] = __ldg(ep.dinv + c * ld + node);
          if(MODE == OP_CHEB)
            in.d[c] = ep.c1 != T(0) ? y[c * ld + node] : T(0); // the previous iterate
        }
      }
    };
    // FP32: before the element work; FP64: after it, where the registers
    // of the element work are free again (the exchange barrier covers part
    // of the latency)
    constexpr bool kEarly = sizeof(T) == 4;
    if(kEarly)
      load_in();
    // element modes: z butterfly of the two planes' x-y modes
    T uh[24], yh[24];
#pragma unroll
    for(int s = 0; s < 4; s++)
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const T b = kSmemModes ? sH[c * 4 + s][ly][lx] : bh[c][s];
        uh[s * 3 + c] = b + th[c][s];
        uh[(s + 4) * 3 + c] = b - th[c][s];
        if(kSmemModes)
          sH[c * 4 + s][ly][lx] = th[c][s];
      }
    yh[0] = yh[1] = yh[2] = T(0); // rigid translations
    modal_blocks_apply<0, 0>(K, uh, yh);
    if(kLateNext)
    {
      load_plane(ek + 2, nxt);
      Enxt = load_E(ek + 1);
    }
    // inverse z butterfly: bottom face completes plane ek, top face is carried
    T acc[3][4];
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      T hb[4];
#pragma unroll
      for(int s = 0; s < 4; s++)
      {
        hb[s] = fma(Ee, yh[s * 3 + c] + yh[(s + 4) * 3 + c], sC[c * 4 + s][ly][lx]);
        sC[c * 4 + s][ly][lx] = Ee * (yh[s * 3 + c] - yh[(s + 4) * 3 + c]);
      }
      plane_corners(hb, acc[c]);
    }
    if(!kSmemModes)
#pragma unroll
      for(int c = 0; c < 3; c++)
#pragma unroll
        for(int q = 0; q < 4; q++)
          bh[c][q] = th[c][q];
    if(!kEarly)
      load_in();
    if(out)
    {
      T A[3];
      const int buf = ek & 1;
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        A[c] = acc[c][lnode(1, 1)] + __shfl_down_sync(0xffffffffu, acc[c][lnode(0, 1)], 1);
        sB[buf][c][ly][lx] =
            acc[c][lnode(1, 0)] + __shfl_down_sync(0xffffffffu, acc[c][lnode(0, 0)], 1);
      }
      __syncthreads();
      if(own)
      {
#pragma unroll
        for(int c = 0; c < 3; c++)
        {
          T o = A[c] + sB[buf][c][ly + 1][lx];
          if((f >> c) & 1u)
            o = T(0);
          const T us = in.us[c];
          if(DOT)
            dot += double(us) * double(o);
          const long long i = c * ld + node;
          T w;
          if(MODE == OP_APPLY)
            w = o;
          else
          {
            const T r = in.b[c] - o;
            if(MODE == OP_RESIDUAL)
              w = r;
            else if(MODE == OP_JACOBI)
              w = us + ep.omega * in.dinv[c] * r;
            else
            {
              T dn = ep.c2 * in.dinv[c] * r;
              if(ep.c1 != T(0))
                dn += ep.c1 * (us - in.d[c]);
              w = us + dn;
            }
          }
          y[i] = w;
        }
      }
    }
  }
  if(DOT)
  {
    double v[1] = {dot};
    block_reduce<1>(v, red, FinStore{dotOut});
  }
}

// ------------------------------------------------- Hex8, paired rows ----
// The FP32 corner-mode operator with two element rows per thread.  A CTA of
// 32 x TW threads owns a 31 x (2 TW - 1) tile of output nodes (one element of
// halo on the low side of each axis) and marches up a chunk of z planes, as
// k_matvec_h8m does; thread (lx, ly) owns element rows j = Y0 - 1 + 2 ly and
// j + 1 of element column i = X0 - 1 + lx.  The two elements run in lockstep
// as the two lanes of packed FP32 pairs (add / sub / mul / fma .f32x2): the
// x-y butterflies, the z butterfly and the modulus scaling of both elements
// are one packed instruction each, while the 45 block products stay scalar
// (their coefficients are constant-bank operands).  The node row between the
// two elements is summed inside the thread, so only one node row per two
// element rows goes through shared memory to the warp below.
template <typename T> struct PairOps;
template <> struct PairOps<float>
{
  using P = float2;
  static __device__ __forceinline__ P add(P a, P b) { return __fadd2_rn(a, b); }
  static __device__ __forceinline__ P mul(P a, P b) { return __fmul2_rn(a, b); }
  static __device__ __forceinline__ P fma(P a, P b, P c) { return __ffma2_rn(a, b, c); }
  static __device__ __forceinline__ P sub(P a, P b)
  {
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(r)
        : "l"(*reinterpret_cast<unsigned long long *>(&a)),
          "l"(*reinterpret_cast<unsigned long long *>(&b)));
    return *reinterpret_cast<P *>(&r);
  }
};

constexpr int kPairWarps = 4;     // warps of k_matvec_h8p (two element rows each)
constexpr int kPairMinBlocks = 3;
constexpr int kPairPrefetch = 4;  // planes the L2 prefetch runs ahead of the loads
template <typename T, int TW, bool DOT, int MODE, int MINB>
__global__ void __launch_bounds__(TX *TW, MINB)
    k_matvec_h8p(const KModal<T> K, const Dims d, const int zchunk, const T *__restrict__ E,
                 const T *__restrict__ u, T *__restrict__ y, const uint8_t *__restrict__ fix,
                 RedScratch red, double *dotOut, const KState *gate, const int gateConv,
                 const Epi<T> ep)
{
  using O = PairOps<T>;
  using P = typename O::P;
  if(gate && (gate->stop || (gateConv && gate->conv)))
    return;
  __shared__ T sB[2][3][TW][TX];
  const int lx = threadIdx.x, ly = threadIdx.y;
  const int X0 = blockIdx.x * (TX - 1), Y0 = blockIdx.y * (2 * TW - 1);
  const int ei = X0 - 1 + lx, ej = Y0 - 1 + 2 * ly;
  const int Z0 = blockIdx.z * zchunk;
  const int Z1 = min(Z0 + zchunk, d.sz) - 1;
  const long long sxy = (long long)d.sx * d.sy, exy = (long long)d.nx * d.ny;
  const long long ld = d.ld;
  // nodes (ei + a, ej + r), r = 0, 1, 2, a = 0, 1, and the two elements
  bool nok[3][2];
#pragma unroll
  for(int r = 0; r < 3; r++)
#pragma unroll
    for(int a = 0; a < 2; a++)
      nok[r][a] = ei + a >= 0 && ei + a < d.sx && ej + r >= 0 && ej + r < d.sy;
  const bool ecol = ei >= 0 && ei < d.nx;
  const bool eok0 = ecol && ej >= 0 && ej < d.ny, eok1 = ecol && ej + 1 >= 0 && ej + 1 < d.ny;
  // element (ei, ej) of layer 0 and node (ei, ej) of plane 0 (either may lie
  // outside the grid: every access below is guarded by the flags above)
  const long long eb = (long long)ei + (long long)ej * d.nx;
  const long long nb = (long long)ei + (long long)ej * d.sx;
  auto ldn = [&](int k, int c, int r, int a) -> T {
    return (nok[r][a] && k >= 0 && k <= d.nz)
               ? __ldg(u + c * ld + nb + (long long)r * d.sx + a + (long long)k * sxy)
               : T(0);
  };
  // plane k as pairs over the row pairs (j, j + 1) and (j + 1, j + 2)
  auto load_plane = [&](int k, P (&lo)[3][2], P (&hi)[3][2]) {
#pragma unroll
    for(int c = 0; c < 3; c++)
#pragma unroll
      for(int a = 0; a < 2; a++)
      {
        lo[c][a].x = ldn(k, c, 0, a);
        lo[c][a].y = ldn(k, c, 1, a);
        hi[c][a].x = lo[c][a].y;
        hi[c][a].y = ldn(k, c, 2, a);
      }
  };
  auto load_E = [&](int k) -> P {
    P e;
    const bool kok = k >= 0 && k < d.nz;
    e.x = (eok0 && kok) ? __ldg(E + eb + (long long)k * exy) : T(0);
    e.y = (eok1 && kok) ? __ldg(E + eb + d.nx + (long long)k * exy) : T(0);
    return e;
  };
  // x-y modes of a plane for both elements: h[c][sx + 2 sy]
  auto modes = [&](const P (&lo)[3][2], const P (&hi)[3][2], P (&h)[3][4]) {
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      const P sl = O::add(lo[c][0], lo[c][1]), dl = O::sub(lo[c][0], lo[c][1]);
      const P sh = O::add(hi[c][0], hi[c][1]), dh = O::sub(hi[c][0], hi[c][1]);
      h[c][0] = O::add(sl, sh);
      h[c][1] = O::add(dl, dh);
      h[c][2] = O::sub(sl, sh);
      h[c][3] = O::sub(dl, dh);
    }
  };

  // the carried top-face result lives in shared memory (each thread its own
  // 12 pairs), the next plane is loaded at the top of its layer from L2 (the
  // prefetch below runs kPairPrefetch planes ahead): both keep the registers
  // under the 168 of three 128-thread CTAs per SM
  __shared__ P sC[12][TW][TX];
  P bh[3][4];
  {
    P lo[3][2], hi[3][2];
    load_plane(Z0 - 1, lo, hi);
    modes(lo, hi, bh);
#pragma unroll
    for(int q = 0; q < 12; q++)
      sC[q][ly][lx] = P{T(0), T(0)};
  }
  P Enxt = load_E(Z0 - 1);
  // L2 prefetch, kPairPrefetch planes ahead of the plane loads: lane
  // l < 18 takes component l / 6, row l / 2 % 3 and half-row l % 2 of the
  // warp's three node rows, lanes 18..21 the two element rows' moduli, so one
  // instruction per warp and layer keeps the plane loads L2 hits
  long long pfOff = -1;
  long long pfStep = sxy;
  bool pfE = false;
  {
    const int x0 = min(max(X0 - 1 + 32 * (lx & 1), 0), d.nx);
    if(lx < 18)
    {
      const int c = lx / 6, r = (lx >> 1) % 3;
      const int row = ej + r;
      if(row >= 0 && row < d.sy)
        pfOff = c * ld + x0 + (long long)row * d.sx;
    }
    else if(lx < 22)
    {
      const int row = ej + ((lx - 18) >> 1);
      if(row >= 0 && row < d.ny)
      {
        pfOff = min(x0, d.nx - 1) + (long long)row * d.nx;
        pfStep = exy;
        pfE = true;
      }
    }
  }
  const int ni = ei + 1;
  const bool ocol = lx < TX - 1 && ni < d.sx;
  const bool own1 = ocol && ej + 1 >= 0 && ej + 1 < d.sy;
  const bool own2 = ocol && ly < TW - 1 && ej + 2 < d.sy;
  const long long nodeb = (long long)ni + (long long)(ej + 1) * d.sx; // row j + 1, plane 0
  double dot = 0.0;
  for(int ek = Z0 - 1; ek <= Z1; ++ek)
  {
    P th[3][4];
    {
      P lo[3][2], hi[3][2];
      load_plane(ek + 1, lo, hi);
      modes(lo, hi, th);
    }
    const P Ee = Enxt;
    Enxt = load_E(ek + 1);
    {
      const int kp = ek + 1 + kPairPrefetch; // plane (layer for the moduli)
      if(pfOff >= 0 && kp <= (pfE ? d.nz - 1 : d.nz))
      {
        const T *a = (pfE ? E : u) + pfOff + (long long)kp * pfStep;
        asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
      }
    }
    const bool out = ek >= Z0;
    // the epilogue's inputs at the two output nodes of plane ek
    const long long node1 = nodeb + (long long)ek * sxy, node2 = node1 + d.sx;
    unsigned f1 = 0, f2 = 0;
    T us1[3] = {T(0), T(0), T(0)}, us2[3] = {T(0), T(0), T(0)};
    T b1[3], b2[3], dv1[3], dv2[3], pv1[3], pv2[3];
    if(out)
    {
      if(own1)
        f1 = __ldg(fix + node1);
      if(own2)
        f2 = __ldg(fix + node2);
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const long long i1 = c * ld + node1, i2 = c * ld + node2;
        if(DOT || MODE >= OP_JACOBI)
        {
          us1[c] = own1 ? __ldg(u + i1) : T(0);
          us2[c] = own2 ? __ldg(u + i2) : T(0);
        }
        if(MODE != OP_APPLY)
        {
          b1[c] = own1 ? __ldg(ep.b + i1) : T(0);
          b2[c] = own2 ? __ldg(ep.b + i2) : T(0);
        }
        if(MODE >= OP_JACOBI)
        {
          dv1[c] = own1 ? __ldg(ep.dinv + i1) : T(0);
          dv2[c] = own2 ? __ldg(ep.dinv + i2) : T(0);
        }
        if(MODE == OP_CHEB)
        {
          pv1[c] = (own1 && ep.c1 != T(0)) ? y[i1] : T(0);
          pv2[c] = (own2 && ep.c1 != T(0)) ? y[i2] : T(0);
        }
      }
    }
    // element modes (z butterfly) and the 11 blocks, lane by lane
    T ux[24], uy[24], yx[24], yy[24];
#pragma unroll
    for(int q = 0; q < 4; q++)
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        const P sp = O::add(bh[c][q], th[c][q]), sm = O::sub(bh[c][q], th[c][q]);
        ux[q * 3 + c] = sp.x;
        uy[q * 3 + c] = sp.y;
        ux[(q + 4) * 3 + c] = sm.x;
        uy[(q + 4) * 3 + c] = sm.y;
        bh[c][q] = th[c][q];
      }
    yx[0] = yx[1] = yx[2] = T(0); // rigid translations
    yy[0] = yy[1] = yy[2] = T(0);
    modal_blocks_apply<0, 0>(K, ux, yx);
    modal_blocks_apply<0, 0>(K, uy, yy);
    // inverse z butterfly with the moduli: the bottom face completes plane
    // ek, the top face is carried up
    T o0[3], o1[3], o2[3]; // x-summed rows j, j + 1, j + 2 of plane ek
    const int buf = ek & 1;
#pragma unroll
    for(int c = 0; c < 3; c++)
    {
      P hb[4];
#pragma unroll
      for(int q = 0; q < 4; q++)
      {
        const P a = P{yx[q * 3 + c], yy[q * 3 + c]}, b = P{yx[(q + 4) * 3 + c], yy[(q + 4) * 3 + c]};
        hb[q] = O::fma(Ee, O::add(a, b), sC[c * 4 + q][ly][lx]);
        sC[c * 4 + q][ly][lx] = O::mul(Ee, O::sub(a, b));
      }
      // inverse x-y butterfly: y stage packed, the shared middle row summed
      // before its x stage
      const P pp = O::add(hb[0], hb[2]), mm = O::sub(hb[0], hb[2]);
      const P rr = O::add(hb[1], hb[3]), nn = O::sub(hb[1], hb[3]);
      const T pm = mm.x + pp.y, rn = nn.x + rr.y;
      // corner a = 0 of each row goes to the lane on the left
      const T l0 = pp.x + rr.x, r0v = pp.x - rr.x;
      const T l1 = pm + rn, r1v = pm - rn;
      const T l2 = mm.y + nn.y, r2v = mm.y - nn.y;
      o0[c] = r0v + __shfl_down_sync(0xffffffffu, l0, 1);
      o1[c] = r1v + __shfl_down_sync(0xffffffffu, l1, 1);
      o2[c] = r2v + __shfl_down_sync(0xffffffffu, l2, 1);
    }
    if(out)
    {
#pragma unroll
      for(int c = 0; c < 3; c++)
        sB[buf][c][ly][lx] = o0[c];
      __syncthreads();
#pragma unroll
      for(int c = 0; c < 3; c++)
      {
        T v1 = ((f1 >> c) & 1u) ? T(0) : o1[c];
        T v2 = o2[c] + (ly < TW - 1 ? sB[buf][c][ly + 1][lx] : T(0));
        if((f2 >> c) & 1u)
          v2 = T(0);
        if(DOT)
          dot += double(us1[c]) * double(v1) + double(us2[c]) * double(v2);
        T w1 = v1, w2 = v2;
        if(MODE != OP_APPLY)
        {
          const T q1 = b1[c] - v1, q2 = b2[c] - v2;
          if(MODE == OP_RESIDUAL)
          {
            w1 = q1;
            w2 = q2;
          }
          else if(MODE == OP_JACOBI)
          {
            w1 = us1[c] + ep.omega * dv1[c] * q1;
            w2 = us2[c] + ep.omega * dv2[c] * q2;
          }
          else
          {
            T d1 = ep.c2 * dv1[c] * q1, d2 = ep.c2 * dv2[c] * q2;
            if(ep.c1 != T(0))
            {
              d1 += ep.c1 * (us1[c] - pv1[c]);
              d2 += ep.c1 * (us2[c] - pv2[c]);
            }
            w1 = us1[c] + d1;
            w2 = us2[c] + d2;
          }
        }
        if(own1)
          y[c * ld + node1] = w1;
        if(own2)
          y[c * ld + node2] = w2;
      }
    }
  }
  if(DOT)
  {
    double v[1] = {dot};
    block_reduce<1>(v, red, FinStore{dotOut});
  }
}

// ------------------------------------------------------------------- Q4 ----
/// the Q4 operator for block (bxi, byi) of a (bx, by) grid: the body of
/// k_matvec_q4 and of its batched form k_matvec_q4_batch
/// The Q4 operator over one block's columns and element rows.  Each row's
/// loads (the next node row, the element modulus, and the inputs of this
/// row's fused update) are issued one row ahead of, or before, the element
/// work that consumes them, so their latency overlaps arithmetic; the
/// arithmetic is the same, in the same order.
template <typename T, bool DOT, int MODE>
__device__ __forceinline__ void q4_body(const KMat<T, 8> &K, const Dims &d, const int ychunk,
                                        const T *__restrict__ E, const T *__restrict__ u,
                                        T *__restrict__ y, const uint8_t *__restrict__ fix,
                                        const RedScratch &red, double *dotOut,
                                        const KState *gate, const int gateConv, const Epi<T> &ep,
                                        int bxi, int byi, int nbx, int nby)
{
  if(gate && (gate->stop || (gateConv && gate->conv)))
    return;
  const int lx = threadIdx.x, w = threadIdx.y;
  const int X0 = (bxi * TY2 + w) * (TX - 1);
  const int ei = X0 - 1 + lx;
  const int Y0 = byi * ychunk;
  const int Y1 = min(Y0 + ychunk, d.sy) - 1;
  const bool col = ei >= 0 && ei < d.nx;
  const long long ld = d.ld;
  T ub[2][2], ut[2][2], un[2][2], carry[2][2];
#pragma unroll
  for(int c = 0; c < 2; c++)
#pragma unroll
    for(int a = 0; a < 2; a++)
    {
      carry[c][a] = T(0);
      ub[c][a] = T(0);
    }
  if(col && Y0 - 1 >= 0)
  {
    long long base = ei + (long long)(Y0 - 1) * d.sx;
#pragma unroll
    for(int c = 0; c < 2; c++)
#pragma unroll
      for(int a = 0; a < 2; a++)
        ub[c][a] = __ldg(u + c * ld + base + a);
  }
  // the top node row and the modulus of element row ej
  auto load_row = [&](int ej, T(&v)[2][2], T &Ev) {
    const bool topok = col && ej + 1 >= 0 && ej + 1 <= d.ny;
#pragma unroll
    for(int c = 0; c < 2; c++)
#pragma unroll
      for(int a = 0; a < 2; a++)
        v[c][a] = topok ? __ldg(u + c * ld + ei + (long long)(ej + 1) * d.sx + a) : T(0);
    const bool lay = col && ej >= 0 && ej < d.ny;
    Ev = lay ? __ldg(E + (long long)ei + (long long)ej * d.nx) : T(0);
  };
  T En;
  load_row(Y0 - 1, un, En);
  const int ni = ei + 1;
  const bool ownCol = lx < TX - 1 && ni < d.sx && X0 < d.sx;
  // the fused dot: one slot per (node row, warp strip), the warp's sum over
  // its strip of that row, so the total does not depend on how the rows are
  // cut into blocks
  const int strips = nbx * TY2, strip = bxi * TY2 + w;
  // the inputs of the update of row ej's output node (FP32: loaded a row
  // ahead, with the next node row; the previous iterate in y is read before
  // this thread, its only writer, overwrites it)
  auto load_inp = [&](int ej, unsigned &f, T(&us)[2], T(&bv)[2], T(&dv)[2], T(&yp)[2]) {
    f = 0;
#pragma unroll
    for(int c = 0; c < 2; c++)
      us[c] = bv[c] = dv[c] = yp[c] = T(0);
    if(ej >= Y0 && ej <= Y1 && ownCol)
    {
      const long long node = (long long)ni + (long long)ej * d.sx;
      f = __ldg(fix + node);
#pragma unroll
      for(int c = 0; c < 2; c++)
      {
        const long long i = c * ld + node;
        if(DOT || MODE >= OP_JACOBI)
          us[c] = __ldg(u + i); // node i = 0 belongs to a halo column
        if(MODE != OP_APPLY)
          bv[c] = __ldg(ep.b + i);
        if(MODE >= OP_JACOBI)
          dv[c] = __ldg(ep.dinv + i);
        if(MODE == OP_CHEB && ep.c1 != T(0))
          yp[c] = y[i];
      }
    }
  };
  constexpr bool kAhead = sizeof(T) == 4;
  unsigned nf = 0;
  T nus[2], nbv[2], ndv[2], nyp[2];
  if(kAhead)
    load_inp(Y0 - 1, nf, nus, nbv, ndv, nyp);
  for(int ej = Y0 - 1; ej <= Y1; ++ej)
  {
#pragma unroll
    for(int c = 0; c < 2; c++)
#pragma unroll
      for(int a = 0; a < 2; a++)
        ut[c][a] = un[c][a];
    const T Ee = En;
    // this row's output node and the inputs of its update
    const bool own = ej >= Y0 && ownCol;
    const long long node = (long long)ni + (long long)ej * d.sx;
    unsigned f;
    T us[2], bv[2], dv[2], yp[2];
    if(kAhead)
    {
      f = nf;
#pragma unroll
      for(int c = 0; c < 2; c++)
      {
        us[c] = nus[c];
        bv[c] = nbv[c];
        dv[c] = ndv[c];
        yp[c] = nyp[c];
      }
    }
    if(ej < Y1)
    {
      load_row(ej + 1, un, En);
      if(kAhead)
        load_inp(ej + 1, nf, nus, nbv, ndv, nyp);
    }
    if(!kAhead)
      load_inp(ej, f, us, bv, dv, yp);
    // element vector in local order: n0=(0,0) n1=(1,0) n2=(1,1) n3=(0,1)
    T ue[8];
#pragma unroll
    for(int c = 0; c < 2; c++)
    {
      ue[0 * 2 + c] = ub[c][0];
      ue[1 * 2 + c] = ub[c][1];
      ue[2 * 2 + c] = ut[c][1];
      ue[3 * 2 + c] = ut[c][0];
    }
    T acc[2][2];
#pragma unroll
    for(int a = 0; a < 2; a++)
#pragma unroll
      for(int c = 0; c < 2; c++)
      {
        const int row = lnode(a, 0) * 2 + c;
        T s = T(0);
#pragma unroll
        for(int j = 0; j < 8; j++)
          s = fma(K.k[row * 8 + j], ue[j], s);
        acc[c][a] = fma(Ee, s, carry[c][a]);
      }
    if(ej >= Y0)
    {
      T o[2];
#pragma unroll
      for(int c = 0; c < 2; c++)
        o[c] = acc[c][1] + __shfl_down_sync(0xffffffffu, acc[c][0], 1);
      double dot = 0.0;
      if(own)
      {
#pragma unroll
        for(int c = 0; c < 2; c++)
        {
          T v = ((f >> c) & 1u) ? T(0) : o[c];
          if(DOT)
            dot += double(us[c]) * double(v);
          // the fused update (epilogue's arithmetic, inputs loaded above)
          T out;
          if(MODE == OP_APPLY)
            out = v;
          else
          {
            T r = bv[c] - v;
            if(MODE == OP_RESIDUAL)
              out = r;
            else if(MODE == OP_JACOBI)
              out = us[c] + ep.omega * dv[c] * r;
            else
            {
              T dn = ep.c2 * dv[c] * r;
              if(ep.c1 != T(0))
                dn += ep.c1 * (us[c] - yp[c]);
              out = us[c] + dn;
            }
          }
          y[c * ld + node] = out;
        }
      }
      if(DOT)
      {
        dot = warp_sum_d(dot);
        if(lx == 0)
          red.partials[(long long)ej * strips + strip] = dot;
      }
    }
#pragma unroll
    for(int a = 0; a < 2; a++)
#pragma unroll
      for(int c = 0; c < 2; c++)
      {
        const int row = lnode(a, 1) * 2 + c;
        T s = T(0);
#pragma unroll
        for(int j = 0; j < 8; j++)
          s = fma(K.k[row * 8 + j], ue[j], s);
        carry[c][a] = Ee * s;
      }
#pragma unroll
    for(int c = 0; c < 2; c++)
#pragma unroll
      for(int a = 0; a < 2; a++)
        ub[c][a] = ut[c][a];
  }
  if(DOT)
    slots_reduce_finish(red, (long long)d.sy * strips, nbx * nby, lx == 0 && Y0 <= Y1,
                        FinStore{dotOut});
}

template <typename T, bool DOT, int MODE>
__global__ void __launch_bounds__(TX *TY2)
    k_matvec_q4(const KMat<T, 8> K, const Dims d, const int ychunk,
                const T *__restrict__ E, const T *__restrict__ u, T *__restrict__ y,
                const uint8_t *__restrict__ fix, RedScratch red, double *dotOut,
                const KState *gate, const int gateConv, const Epi<T> ep)
{
  q4_body<T, DOT, MODE>(K, d, ychunk, E, u, y, fix, red, dotOut, gate, gateConv, ep, blockIdx.x,
                        blockIdx.y, gridDim.x, gridDim.y);
}

/// many Q4 operator launches in one: block b runs block map[b].y of the
/// launch described by D[map[b].x], with that launch's grid, so each
/// problem's result (and its fused dot product) is bitwise that of its own
/// launch.  UK: every launch has the same element matrix, passed as the
/// kernel parameter Ku (constant-bank FMA operands, as in the per-problem
/// kernel); otherwise each record's matrix is staged in shared memory.
template <typename T, bool DOT, int MODE, bool UK>
__global__ void __launch_bounds__(TX *TY2, sizeof(T) == 4 ? 8 : 4)
    k_matvec_q4_batch(const Q4Launch<T> *__restrict__ D, const int2 *__restrict__ map,
                      BatchQueue bq, const KMat<T, 8> Ku)
{
  batch_queue(
      D, map, bq, [](const Q4Launch<T> &q) { return q.bx * q.by; },
      [](const Q4Launch<T> &q) {
        return q.gate && (q.gate->stop || (q.gateConv && q.gate->conv));
      },
      [&](const Q4Launch<T> &q, int b, bool fresh) {
        if constexpr(UK)
        {
          (void)fresh;
          q4_body<T, DOT, MODE>(Ku, q.d, q.ychunk, q.E, q.u, q.y, q.fix, q.red, q.dotOut, q.gate,
                                q.gateConv, q.ep, b % q.bx, b / q.bx, q.bx, q.by);
        }
        else
        {
          // the element matrix in shared memory: in registers it would take
          // 64 (FP32) or 128 (FP64) of them and a quarter of the occupancy;
          // staged once per run of items of one record (the queue's barrier
          // after each item protects it until every thread is done)
          __shared__ KMat<T, 8> sK;
          if(fresh)
          {
            const int t = threadIdx.x + blockDim.x * threadIdx.y;
            if(t < 64)
              sK.k[t] = q.K.k[t];
            __syncthreads();
          }
          q4_body<T, DOT, MODE>(sK, q.d, q.ychunk, q.E, q.u, q.y, q.fix, q.red, q.dotOut,
                                q.gate, q.gateConv, q.ep, b % q.bx, b / q.bx, q.bx, q.by);
        }
      });
}

// ------------------------------------------------------------ diagonal ----
/// the diagonal of K(E) and its Eigen-rule inverse for the nodes of block bx
/// (the body of k_diag and of its batched form); KM holds the element matrix
template <typename T, int DIM, class KM>
__device__ __forceinline__ void diag_b(const KM &K, const Dims &d, const T *__restrict__ E,
                                       const uint8_t *__restrict__ fix, T *__restrict__ invdiag,
                                       T *__restrict__ diag, unsigned bx)
{
  long long n = bx * (long long)blockDim.x + threadIdx.x;
  if(n >= d.nnode)
    return;
  const int nd = DIM == 2 ? 8 : 24;
  long long sxy = (long long)d.sx * d.sy;
  int i = int(n % d.sx), j = int((n / d.sx) % d.sy), k = DIM == 3 ? int(n / sxy) : 0;
  double s[3] = {0, 0, 0};
  for(int dk = (DIM == 3 ? -1 : 0); dk <= 0; dk++)
    for(int dj = -1; dj <= 0; dj++)
      for(int di = -1; di <= 0; di++)
      {
        int ei = i + di, ej = j + dj, ek = k + dk;
        if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (DIM == 3 && ek >= d.nz))
          continue;
        long long e = ei + (long long)ej * d.nx + (long long)ek * d.nx * d.ny;
        int l = lnode(-di, -dj) + (DIM == 3 ? 4 * (-dk) : 0);
        double Ee = E[e];
        for(int c = 0; c < DIM; c++)
          s[c] += Ee * double(K.k[(l * DIM + c) * nd + l * DIM + c]);
      }
  unsigned f = fix[n];
  for(int c = 0; c < DIM; c++)
  {
    bool fx = (f >> c) & 1u;
    if(diag)
      diag[c * d.ld + n] = fx ? T(0) : T(s[c]);
    // Eigen's DiagonalPreconditioner: 1 where the diagonal is 0
    invdiag[c * d.ld + n] = fx ? T(0) : (s[c] != 0.0 ? T(1.0 / s[c]) : T(1));
  }
}
template <typename T, int DIM>
__global__ void k_diag(const KMat<T, 24> K, const Dims d, const T *__restrict__ E,
                       const uint8_t *__restrict__ fix, T *__restrict__ invdiag,
                       T *__restrict__ diag)
{
  diag_b<T, DIM>(K, d, E, fix, invdiag, diag, blockIdx.x);
}

/// many 2D diagonal launches in one (block b runs block map[b].y of launch
/// D[map[b].x], 256 threads, its own grid of blocks_for(nnode, 256))
template <typename T>
__global__ void k_diag2_batch(const Diag2Launch<T> *__restrict__ D, const int2 *__restrict__ map,
                              BatchQueue bq)
{
  batch_queue(
      D, map, bq, [](const Diag2Launch<T> &q) { return int((q.d.nnode + 255) / 256); },
      [](const Diag2Launch<T> &) { return false; },
      [](const Diag2Launch<T> &q, int b, bool) {
        diag_b<T, 2>(q.K, q.d, q.E, q.fix, q.invdiag, nullptr, unsigned(b));
      });
}

__global__ void k_gather_free(long long numeq, const long long *__restrict__ idx,
                              const double *__restrict__ soa, double *__restrict__ out)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < numeq)
    out[i] = soa[idx[i]];
}
__global__ void k_scatter_free(long long numeq, const long long *__restrict__ idx,
                               const double *__restrict__ in, double *__restrict__ soa)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < numeq)
    soa[idx[i]] = in[i];
}

/// SIMP of src/problem/elasticity.hpp:15-22
__global__ void k_simp(long long n, double y1, double y2, double p,
                       const double *__restrict__ rho, double *__restrict__ E,
                       float *__restrict__ Ef)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i >= n)
    return;
  double s = rho[i], v;
  if(y2 - y1 >= 0.0)
    v = (1.0 - pow(s, p)) * y1 + pow(s, p) * y2;
  else
    v = pow(1.0 - s, p) * y1 + (1.0 - pow(1.0 - s, p)) * y2;
  E[i] = v;
  if(Ef)
    Ef[i] = float(v);
}

/// sensitivity() of opt_macro_oc.cpp:182-207 / opt_mma_Helmholtz.cpp:173-205:
/// dc_e = -(E'/E) u_e^T (E K0) u_e, u from the node values with |u| < 1e-15
/// zeroed as divideValIntoNode does.
template <int DIM>
__global__ void k_sensitivity(const KMat<double, 24> K, const Dims d, double y1, double y2,
                              double p, const double *__restrict__ rho,
                              const double *__restrict__ u, double *__restrict__ dc)
{
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= d.nel)
    return;
  constexpr int NE = DIM == 2 ? 4 : 8, ND = NE * DIM;
  int ei = int(e % d.nx), ej = int((e / d.nx) % d.ny);
  int ek = DIM == 3 ? int(e / ((long long)d.nx * d.ny)) : 0;
  long long base = ei + (long long)ej * d.sx + (long long)ek * d.sx * d.sy;
  long long sxy = (long long)d.sx * d.sy;
  double ue[ND];
#pragma unroll
  for(int l = 0; l < NE; l++)
  {
    int q = l & 3, top = l >> 2;
    long long off = (q == 1 || q == 2 ? 1 : 0) + (q >= 2 ? (long long)d.sx : 0) + top * sxy;
#pragma unroll
    for(int c = 0; c < DIM; c++)
    {
      double v = u[c * d.ld + base + off];
      ue[l * DIM + c] = fabs(v) < 1.0e-15 ? 0.0 : v;
    }
  }
  double s = rho[e], young, dyoung;
  if(y2 >= y1)
  {
    young = (1.0 - pow(s, p)) * y1 + pow(s, p) * y2;
    dyoung = p * pow(s, p - 1.0) * (y2 - y1);
  }
  else
  {
    young = pow(1.0 - s, p) * y1 + (1.0 - pow(1.0 - s, p)) * y2;
    dyoung = (y2 - y1) * p * pow(1.0 - s, p - 1.0);
  }
  double q = 0.0;
#pragma unroll
  for(int i = 0; i < ND; i++)
  {
    double t = 0.0;
#pragma unroll
    for(int j = 0; j < ND; j++)
      t = fma(young * K.k[i * ND + j], ue[j], t);
    q = fma(ue[i], t, q);
  }
  dc[e] = -(dyoung / young) * q;
}

/// the same sensitivity for a Hex8 element in the corner-mode form:
/// u_e^T K0 u_e = (H u_e)^T Kt (H u_e), 45 multiply-adds instead of 576; one
/// thread per element on a 3D launch (x along threads, y and z along the grid)
__global__ void k_sensitivity_h8m(const KModal<double> K, const Dims d, double y1, double y2,
                                  double p, const double *__restrict__ rho,
                                  const double *__restrict__ u, double *__restrict__ dc)
{
  const int ei = blockIdx.x * blockDim.x + threadIdx.x, ej = blockIdx.y, ek = blockIdx.z;
  if(ei >= d.nx)
    return;
  const long long e = ei + (long long)ej * d.nx + (long long)ek * d.nx * d.ny;
  const long long sxy = (long long)d.sx * d.sy;
  const long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
  const long long qoff[4] = {0, 1, 1 + (long long)d.sx, (long long)d.sx};
  double uh[24], yh[24];
#pragma unroll
  for(int c = 0; c < 3; c++)
  {
    double vb[4], vt[4], hb[4], ht[4];
#pragma unroll
    for(int q = 0; q < 4; q++)
    {
      // node values with |u| < 1e-15 zeroed, as divideValIntoNode leaves them
      const double b = u[c * d.ld + base + qoff[q]], t = u[c * d.ld + base + qoff[q] + sxy];
      vb[q] = fabs(b) < 1.0e-15 ? 0.0 : b;
      vt[q] = fabs(t) < 1.0e-15 ? 0.0 : t;
    }
    plane_modes(vb, hb);
    plane_modes(vt, ht);
#pragma unroll
    for(int s = 0; s < 4; s++)
    {
      uh[s * 3 + c] = hb[s] + ht[s];
      uh[(s + 4) * 3 + c] = hb[s] - ht[s];
    }
  }
  yh[0] = yh[1] = yh[2] = 0.0;
  modal_blocks_apply<0, 0>(K, uh, yh);
  double q = 0.0;
#pragma unroll
  for(int r = 3; r < 24; r++)
    q = fma(uh[r], yh[r], q);
  const double s = rho[e];
  double young, dyoung;
  if(y2 >= y1)
  {
    young = (1.0 - pow(s, p)) * y1 + pow(s, p) * y2;
    dyoung = p * pow(s, p - 1.0) * (y2 - y1);
  }
  else
  {
    young = pow(1.0 - s, p) * y1 + (1.0 - pow(1.0 - s, p)) * y2;
    dyoung = (y2 - y1) * p * pow(1.0 - s, p - 1.0);
  }
  dc[e] = -(dyoung / young) * (young * q);
}

inline unsigned blocks_for(long long n, int bs) { return unsigned((n + bs - 1) / bs); }
} // namespace

Dims make_dims(int dim, int nx, int ny, int nz)
{
  Dims d;
  d.dim = dim;
  d.nx = nx;
  d.ny = ny;
  d.nz = dim == 3 ? nz : 1;
  d.sx = nx + 1;
  d.sy = ny + 1;
  d.sz = dim == 3 ? nz + 1 : 1;
  d.nnode = (long long)d.sx * d.sy * d.sz;
  d.nel = (long long)d.nx * d.ny * d.nz;
  d.ld = (d.nnode + 63) / 64 * 64;
  return d;
}

int num_sms()
{
  // thread-safe one-time query (worker threads of the batch runner and the
  // server call it concurrently)
  static const int n = [] {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    return v > 0 ? v : 148;
  }();
  return n;
}

/// CTAs of a kernel resident at once on the device (occupancy queried once
/// per kernel)
static int resident_ctas(const void *kern, int threads, int smem)
{
  static std::mutex mu;
  // keyed by kernel and device: the shared-memory opt-in is per device
  static std::unordered_map<const void *, int> memo[64];
  int dev = 0;
  ICB_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  auto &m = memo[dev & 63];
  auto it = m.find(kern);
  if(it != m.end())
    return it->second;
  // static + dynamic shared memory past 48 KB needs the opt-in
  if(smem > 0)
    ICB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
  int n = 0;
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, smem) != cudaSuccess || n < 1)
  {
    (void)cudaGetLastError();
    n = 1;
  }
  return m[kern] = n * num_sms();
}

/// z planes per CTA of the Hex8 kernels: `tiles` x-y tiles, `resident` CTAs
/// in flight.  A CTA marches zchunk + 1 element layers (the layer below its
/// chunk is recomputed), and the launch takes ceil(CTAs / resident) rounds,
/// so the split minimises rounds x (zchunk + 1).
static int h8_zchunk(const Dims &d, long long tiles, int resident)
{
  int best = d.sz;
  long long bestCost = -1;
  for(int bz = 1; bz <= d.sz; bz++)
  {
    const int zc = (d.sz + bz - 1) / bz;
    const long long n = tiles * ((d.sz + zc - 1) / zc);
    const long long cost = (n + resident - 1) / resident * (zc + 1);
    if(bestCost < 0 || cost < bestCost)
    {
      bestCost = cost;
      best = zc;
    }
  }
  return best;
}

void q4_grid(const Dims &d, int &bx, int &by, int &ychunk)
{
  const int target = num_sms() * 4;
  const int strips = (d.sx + TX - 2) / (TX - 1);
  bx = (strips + TY2 - 1) / TY2;
  by = std::max(1, std::min(d.sy, (target + bx - 1) / bx));
  ychunk = (d.sy + by - 1) / by;
  by = (d.sy + ychunk - 1) / ychunk;
}

int matvec_blocks(const Dims &d)
{
  if(d.dim == 3)
  {
    // the largest CTA count h8_zchunk picks for any occupancy of 1..8 CTAs/SM,
    // for the one-row tiles (31 x 7 nodes) and the paired ones (31 x 15)
    const long long bx = (d.sx + TX - 2) / (TX - 1);
    long long most = 0;
    for(int rows : {TY3 - 1, 2 * kPairWarps - 1})
    {
      const long long tiles = bx * ((d.sy + rows - 1) / rows);
      for(int k = 1; k <= 8; k++)
      {
        const int zc = h8_zchunk(d, tiles, k * num_sms());
        most = std::max(most, tiles * ((d.sz + zc - 1) / zc));
      }
    }
    return int(most);
  }
  int bx, by, ychunk;
  q4_grid(d, bx, by, ychunk);
  // the fused dot's slots (a node row per warp strip) and the blocks
  return std::max(bx * by, q4_dot_slots(d));
}

static std::atomic<bool> g_hex8_modal{true}; // read by every launching thread
static std::atomic<bool> g_hex8_pair{false}; // FP32: two element rows per thread

/// Kt = H K0 H / 64 on the 11 blocks of the corner-mode form.  False when an
/// entry outside the blocks is above rounding (|Kt_rc| > tol max |Kt|, tol
/// 1e-12 for an FP64 K0, 1e-5 for its FP32 copy).
template <typename T> static bool modal_form(const T *K, KModal<T> &m)
{
  auto sign = [](int s, int a) {
    const int q = a & 3;
    const int o = ((q == 1 || q == 2) ? 1 : 0) | (q >= 2 ? 2 : 0) | ((a >> 2) << 2);
    return (__builtin_popcount(unsigned(s & o)) & 1) ? -1.0 : 1.0;
  };
  double hk[24][24], kt[24][24];
  for(int r = 0; r < 24; r++)
    for(int c = 0; c < 24; c++)
    {
      double v = 0.0;
      for(int a = 0; a < 8; a++)
        v += sign(r / 3, a) * double(K[(a * 3 + r % 3) * 24 + c]);
      hk[r][c] = v;
    }
  double big = 0.0;
  for(int r = 0; r < 24; r++)
    for(int c = 0; c < 24; c++)
    {
      double v = 0.0;
      for(int b = 0; b < 8; b++)
        v += hk[r][b * 3 + c % 3] * sign(c / 3, b);
      kt[r][c] = v / 64.0;
      big = std::max(big, std::fabs(kt[r][c]));
    }
  constexpr ModalBlocks MB = modal_blocks();
  bool in[24][24] = {};
  int k = 0;
  for(int b = 0; b < 11; b++)
    for(int i = 0; i < MB.n[b]; i++)
      for(int j = 0; j < MB.n[b]; j++, k++)
      {
        in[MB.dof[b][i]][MB.dof[b][j]] = true;
        m.v[k] = T(kt[MB.dof[b][i]][MB.dof[b][j]]);
      }
  const double tol = sizeof(T) == 8 ? 1e-12 : 1e-5;
  for(int r = 0; r < 24; r++)
    for(int c = 0; c < 24; c++)
      if(!in[r][c] && std::fabs(kt[r][c]) > tol * big)
        return false;
  return big > 0.0;
}

/// modal_form with a small per-thread cache keyed by K0's entries (the
/// multigrid levels each have their own K0; launchers run on several host
/// threads in the batch runner and the server)
template <typename T> static bool modal_form_cached(const T *K, KModal<T> &m)
{
  struct Entry
  {
    T K[576];
    KModal<T> m;
    bool ok = false, used = false;
  };
  thread_local Entry cache[8];
  thread_local int next = 0;
  for(Entry &e : cache)
    if(e.used && std::equal(K, K + 576, e.K))
    {
      m = e.m;
      return e.ok;
    }
  Entry &e = cache[next];
  next = (next + 1) % 8;
  std::copy(K, K + 576, e.K);
  e.used = true;
  e.ok = modal_form(K, e.m);
  m = e.m;
  return e.ok;
}

template <typename T, int MODE>
static void launch_op_mode(const Dims &d, const T *K, const T *E, const T *u, T *y,
                           const uint8_t *fix, cudaStream_t s, const OpExtras<T> &x)
{
  RedScratch red = x.dotRed ? *x.dotRed : RedScratch{};
  const int target = num_sms() * 4;
  Epi<T> ep{x.b, x.dinv, T(x.omega), T(x.c1), T(x.c2)};
  if(d.dim == 3)
  {
    // 8 element rows per tile for FP64 and FP32 (16-row FP64 tiles were
    // measured: faster at 384x128x128, slower at 192x64x64)
    constexpr int TYK = TY3;
    const int bx = (d.sx + TX - 2) / (TX - 1), by = (d.sy + TYK - 2) / (TYK - 1);
    auto run = [&](auto kern, const auto &kp, int smem) {
      const int zchunk =
          h8_zchunk(d, (long long)bx * by, resident_ctas((const void *)kern, TX * TYK, smem));
      const int bz = (d.sz + zchunk - 1) / zchunk;
      if(x.dotRed)
        ICB_REQUIRE((long long)bx * by * bz <= red.maxBlocks, "reduction scratch too small");
      kern<<<dim3(bx, by, bz), dim3(TX, TYK), smem, s>>>(kp, d, zchunk, E, u, y, fix, red,
                                                         x.dotOut, x.gate, x.gateConv, ep);
    };
    KModal<T> kmod;
    if constexpr(std::is_same<T, float>::value)
    {
      if(g_hex8_pair && g_hex8_modal && modal_form_cached(K, kmod))
      {
        // two element rows per thread (k_matvec_h8p): a 31 x 15 node tile
        constexpr int TW = kPairWarps;
        const int bxp = (d.sx + TX - 2) / (TX - 1);
        const int byp = (d.sy + 2 * TW - 2) / (2 * TW - 1);
        auto kern = x.dotRed ? k_matvec_h8p<T, TW, true, MODE, kPairMinBlocks>
                             : k_matvec_h8p<T, TW, false, MODE, kPairMinBlocks>;
        const int zchunk =
            h8_zchunk(d, (long long)bxp * byp, resident_ctas((const void *)kern, TX * TW, 0));
        const int bz = (d.sz + zchunk - 1) / zchunk;
        if(x.dotRed)
          ICB_REQUIRE((long long)bxp * byp * bz <= red.maxBlocks, "reduction scratch too small");
        kern<<<dim3(bxp, byp, bz), dim3(TX, TW), 0, s>>>(kmod, d, zchunk, E, u, y, fix, red,
                                                          x.dotOut, x.gate, x.gateConv, ep);
        ICB_CUDA(cudaGetLastError());
        count_launch();
        return;
      }
    }
    if(g_hex8_modal && modal_form_cached(K, kmod))
    {
      // 3 (FP32) CTAs of 256 threads per SM; FP64 2 with the fused dot and 1
      // without (no register cap short of the kernel's own: the FP64 V-cycle
      // took 58.3 against 59.4 ms at 384x128x128, the dot-fused form was
      // unchanged).  The carry (and for FP64 the bottom plane's modes) live
      // in shared memory: FP64 with both in registers spills, and the
      // dot-fused FP64 Jacobi-PCG on halfmbb3d 192x64x64 took 208 ms against
      // 172 ms for 2374 iterations
      constexpr int MB = sizeof(T) == 8 ? 2 : 3, MBnodot = sizeof(T) == 8 ? 1 : 3;
      if(x.dotRed)
        run(k_matvec_h8m<T, TYK, true, MODE, MB>, kmod, h8m_smem_bytes<T, TYK>());
      else
        run(k_matvec_h8m<T, TYK, false, MODE, MBnodot>, kmod, h8m_smem_bytes<T, TYK>());
    }
    else if constexpr(std::is_same<T, double>::value)
    {
      KSym24 ks;
      for(int r = 0; r < 24; r++)
        for(int c = r; c < 24; c++)
          ks.k[symIdx(r, c)] = K[r * 24 + c];
      if(x.dotRed)
        run(k_matvec_h8<T, KSym24, TYK, true, MODE>, ks, 0);
      else
        run(k_matvec_h8<T, KSym24, TYK, false, MODE>, ks, 0);
    }
    else
    {
      KMat<T, 24> km;
      std::copy(K, K + 576, km.k);
      if(x.dotRed)
        run(k_matvec_h8<T, KMat<T, 24>, TYK, true, MODE>, km, 0);
      else
        run(k_matvec_h8<T, KMat<T, 24>, TYK, false, MODE>, km, 0);
    }
  }
  else
  {
    KMat<T, 8> km;
    std::copy(K, K + 64, km.k);
    int bx, by, ychunk;
    q4_grid(d, bx, by, ychunk);
    (void)target;
    dim3 grid(bx, by), block(TX, TY2);
    if(x.dotRed)
    {
      ICB_REQUIRE(q4_dot_slots(d) <= red.maxBlocks, "reduction scratch too small");
      k_matvec_q4<T, true, MODE><<<grid, block, 0, s>>>(km, d, ychunk, E, u, y, fix, red,
                                                        x.dotOut, x.gate, x.gateConv, ep);
    }
    else
      k_matvec_q4<T, false, MODE><<<grid, block, 0, s>>>(km, d, ychunk, E, u, y, fix, red,
                                                         x.dotOut, x.gate, x.gateConv, ep);
  }
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

template <typename T, bool UK> static const void *q4_batch_kernel_uk(int mode, bool dot)
{
  if(mode == OP_APPLY)
    return dot ? (const void *)k_matvec_q4_batch<T, true, OP_APPLY, UK>
               : (const void *)k_matvec_q4_batch<T, false, OP_APPLY, UK>;
  if(mode == OP_RESIDUAL)
    return (const void *)k_matvec_q4_batch<T, false, OP_RESIDUAL, UK>;
  if(mode == OP_CHEB)
    return (const void *)k_matvec_q4_batch<T, false, OP_CHEB, UK>;
  throw Error{ICB_ERR_BAD_ARG, "batched Q4 operator: unsupported mode"};
}
template <typename T> static const void *q4_batch_kernel(int mode, bool dot, bool uk)
{
  return uk ? q4_batch_kernel_uk<T, true>(mode, dot) : q4_batch_kernel_uk<T, false>(mode, dot);
}
template <typename T> int q4_batch_grid(int mode, bool dot, bool uk, BatchQueue &q)
{
  return queue_grid(q4_batch_kernel<T>(mode, dot, uk), TX * TY2, 0, q);
}
template int q4_batch_grid<double>(int, bool, bool, BatchQueue &);
template int q4_batch_grid<float>(int, bool, bool, BatchQueue &);
int q4_block_warps() { return TY2; }
int q4_dot_slots(const Dims &d)
{
  int bx, by, ychunk;
  q4_grid(d, bx, by, ychunk);
  const long long n = (long long)bx * TY2 * d.sy;
  ICB_REQUIRE(n < (1LL << 31), "grid too large for the Q4 operator's dot");
  return int(n);
}
template <typename T> long long q4_batch_capacity_warps(int mode, bool dot, bool uk)
{
  BatchQueue q{nullptr, nullptr, 1 << 30};
  return (long long)q4_batch_grid<T>(mode, dot, uk, q) * TY2;
}
template long long q4_batch_capacity_warps<double>(int, bool, bool);
template long long q4_batch_capacity_warps<float>(int, bool, bool);

template <typename T>
void launch_q4_batch(const Q4Launch<T> *D, const int2 *map, const BatchQueue &q, int grid,
                     int mode, bool dot, const KMat<T, 8> *uniformK, cudaStream_t s)
{
  if(q.items <= 0)
    return;
  const dim3 block(TX, TY2);
  KMat<T, 8> K{};
  if(uniformK)
    K = *uniformK;
  auto go = [&](auto kern) { kern<<<grid, block, 0, s>>>(D, map, q, K); };
  auto pick = [&](auto uk) {
    constexpr bool U = decltype(uk)::value;
    if(mode == OP_APPLY)
      dot ? go(k_matvec_q4_batch<T, true, OP_APPLY, U>)
          : go(k_matvec_q4_batch<T, false, OP_APPLY, U>);
    else if(mode == OP_RESIDUAL)
      go(k_matvec_q4_batch<T, false, OP_RESIDUAL, U>);
    else if(mode == OP_CHEB)
      go(k_matvec_q4_batch<T, false, OP_CHEB, U>);
    else
      throw Error{ICB_ERR_BAD_ARG, "batched Q4 operator: unsupported mode"};
  };
  if(uniformK)
    pick(std::true_type{});
  else
    pick(std::false_type{});
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
template <typename T>
void launch_diag2_batch(const Diag2Launch<T> *D, const int2 *map, const BatchQueue &q,
                        cudaStream_t s)
{
  if(q.items <= 0)
    return;
  BatchQueue qq = q;
  const int grid = queue_grid((const void *)k_diag2_batch<T>, 256, 0, qq);
  k_diag2_batch<T><<<grid, 256, 0, s>>>(D, map, qq);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
template void launch_diag2_batch<double>(const Diag2Launch<double> *, const int2 *,
                                         const BatchQueue &, cudaStream_t);
template void launch_diag2_batch<float>(const Diag2Launch<float> *, const int2 *,
                                        const BatchQueue &, cudaStream_t);
template void launch_q4_batch<double>(const Q4Launch<double> *, const int2 *,
                                      const BatchQueue &, int, int, bool,
                                      const KMat<double, 8> *, cudaStream_t);
template void launch_q4_batch<float>(const Q4Launch<float> *, const int2 *, const BatchQueue &,
                                     int, int, bool, const KMat<float, 8> *, cudaStream_t);

static std::atomic<bool> g_tc_operator{false};
bool tc_operator_enabled() { return g_tc_operator; }
void set_tc_operator(bool on) { g_tc_operator = on; }
bool hex8_modal_enabled() { return g_hex8_modal; }
void set_hex8_modal(bool on) { g_hex8_modal = on; }
bool hex8_pair_enabled() { return g_hex8_pair; }
void set_hex8_pair(bool on) { g_hex8_pair = on; }

template <typename T>
void launch_op(const Dims &d, const T *K, const T *E, const T *u, T *y, const uint8_t *fix,
               cudaStream_t s, const OpExtras<T> &x)
{
  if constexpr(sizeof(T) == 4)
  {
    if(d.dim == 3 && g_tc_operator && !x.cudaCores)
    {
      launch_op_tc(d, K, E, u, y, fix, s, x);
      return;
    }
  }
  if(x.mode == OP_APPLY)
    launch_op_mode<T, OP_APPLY>(d, K, E, u, y, fix, s, x);
  else if(x.mode == OP_RESIDUAL)
    launch_op_mode<T, OP_RESIDUAL>(d, K, E, u, y, fix, s, x);
  else if(x.mode == OP_JACOBI)
    launch_op_mode<T, OP_JACOBI>(d, K, E, u, y, fix, s, x);
  else
    launch_op_mode<T, OP_CHEB>(d, K, E, u, y, fix, s, x);
}
template void launch_op<double>(const Dims &, const double *, const double *, const double *,
                                double *, const uint8_t *, cudaStream_t,
                                const OpExtras<double> &);
template void launch_op<float>(const Dims &, const float *, const float *, const float *,
                               float *, const uint8_t *, cudaStream_t, const OpExtras<float> &);

template <typename T>
void launch_matvec(const Dims &d, const T *K, const T *E, const T *u, T *y,
                   const uint8_t *fix, cudaStream_t s, RedScratch *dotRed, double *dotOut,
                   const KState *gate)
{
  OpExtras<T> x;
  x.dotRed = dotRed;
  x.dotOut = dotOut;
  x.gate = gate;
  launch_op<T>(d, K, E, u, y, fix, s, x);
}
template void launch_matvec<double>(const Dims &, const double *, const double *,
                                    const double *, double *, const uint8_t *, cudaStream_t,
                                    RedScratch *, double *, const KState *);
template void launch_matvec<float>(const Dims &, const float *, const float *, const float *,
                                   float *, const uint8_t *, cudaStream_t, RedScratch *,
                                   double *, const KState *);

template <typename T>
void launch_diag(const Dims &d, const T *K, const T *E, const uint8_t *fix, T *invdiag,
                 T *diag, cudaStream_t s)
{
  KMat<T, 24> km;
  int nd = d.dim == 2 ? 8 : 24;
  std::copy(K, K + nd * nd, km.k);
  if(d.dim == 3)
    k_diag<T, 3><<<blocks_for(d.nnode, 256), 256, 0, s>>>(km, d, E, fix, invdiag, diag);
  else
    k_diag<T, 2><<<blocks_for(d.nnode, 256), 256, 0, s>>>(km, d, E, fix, invdiag, diag);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
template void launch_diag<double>(const Dims &, const double *, const double *,
                                  const uint8_t *, double *, double *, cudaStream_t);
template void launch_diag<float>(const Dims &, const float *, const float *, const uint8_t *,
                                 float *, float *, cudaStream_t);

void launch_gather_free(const Dims &d, const long long *freeIdx, long long numeq,
                        const double *soa, double *numeqv, cudaStream_t s)
{
  (void)d;
  if(numeq)
  {
    k_gather_free<<<blocks_for(numeq, 256), 256, 0, s>>>(numeq, freeIdx, soa, numeqv);
    count_launch();
  }
  ICB_CUDA(cudaGetLastError());
}
void launch_scatter_free(const Dims &d, const long long *freeIdx, long long numeq,
                         const double *numeqv, double *soa, cudaStream_t s)
{
  (void)d;
  if(numeq)
  {
    k_scatter_free<<<blocks_for(numeq, 256), 256, 0, s>>>(numeq, freeIdx, numeqv, soa);
    count_launch();
  }
  ICB_CUDA(cudaGetLastError());
}
void launch_simp(long long n, double y1, double y2, double p, const double *rho, double *E,
                 float *Ef, cudaStream_t s)
{
  k_simp<<<blocks_for(n, 256), 256, 0, s>>>(n, y1, y2, p, rho, E, Ef);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
void launch_sensitivity(const Dims &d, const double *K, double y1, double y2, double p,
                        const double *rho, const double *u, double *dc, cudaStream_t s)
{
  KMat<double, 24> km;
  int nd = d.dim == 2 ? 8 : 24;
  std::copy(K, K + nd * nd, km.k);
  KModal<double> kmod;
  if(d.dim == 3 && g_hex8_modal && d.ny <= 65535 && d.nz <= 65535 && modal_form_cached(K, kmod))
    k_sensitivity_h8m<<<dim3(unsigned((d.nx + 127) / 128), unsigned(d.ny), unsigned(d.nz)), 128,
                        0, s>>>(kmod, d, y1, y2, p, rho, u, dc);
  else if(d.dim == 3)
    k_sensitivity<3><<<blocks_for(d.nel, 128), 128, 0, s>>>(km, d, y1, y2, p, rho, u, dc);
  else
    k_sensitivity<2><<<blocks_for(d.nel, 128), 128, 0, s>>>(km, d, y1, y2, p, rho, u, dc);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

} // namespace icb
