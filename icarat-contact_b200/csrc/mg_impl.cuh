// mg_impl.cuh -- the multigrid kernels and hierarchy types shared by the
// per-problem solves (mg.cu) and the batched solve of many problems
// (mgbatch.cu); see mg.cu for the design.
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>

#include "batchq.cuh"
#include "graphloop.hpp"
#include "loopcache.hpp"
#include "mg.hpp"
#include "reduce.cuh"

namespace icb
{
namespace
{
constexpr int VB = 256;
/// blocks of a vector kernel over n entries: at least four entries per
/// thread, at most eight blocks per SM (a batched launch runs each block as
/// one work item, so small problems do not split into many tiny ones)
constexpr int kVecPerThread = 4;
inline int vblocks(long long n)
{
  return int(std::max<long long>(
      1, std::min<long long>((n + VB * kVecPerThread - 1) / (VB * kVecPerThread),
                             num_sms() * 8LL)));
}
inline unsigned nblocks(long long n, int bs) { return unsigned((n + bs - 1) / bs); }
/// transfer kernels: kTB threads along x, one grid row per (y, z) node line
constexpr int kTB = 128;
inline dim3 grid3(const Dims &d)
{
  ICB_REQUIRE(d.sy <= 65535 && d.sz <= 65535, "grid too large for the transfer launch");
  return dim3(unsigned((d.sx + kTB - 1) / kTB), unsigned(d.sy), unsigned(d.sz));
}
__device__ __forceinline__ bool gated(const KState *g)
{
  return g && (g->stop || g->conv);
}
/// The vector kernels walk their grid-stride loop (i, i + s, i + 2s, ...) in
/// groups of kGroup iterations: the operands of a group are loaded before any
/// of its iterations is processed, so a thread has kGroup loads in flight per
/// operand instead of one; the iterations (and the order of every sum) are
/// those of the plain loop.
constexpr int kGroup = 4;

// ------------------------------------------------------- grid transfer ----
/// coarse modulus = sum of the children's E over the number of child slots
/// (2 per halved axis, 1 per kept one; slots outside the fine grid add 0)
template <typename T>
__device__ __forceinline__ void coarsen_E_b(Dims df, Dims dc, int3 sh, const T *__restrict__ Ef,
                            T *__restrict__ Ec, const Blk &B)
{
  long long e = B.x * (long long)blockDim.x + threadIdx.x;
  if(e >= dc.nel)
    return;
  int ci = int(e % dc.nx), cj = int((e / dc.nx) % dc.ny), ck = int(e / ((long long)dc.nx * dc.ny));
  double s = 0.0;
  const int nk = df.dim == 3 ? 1 << sh.z : 1;
  for(int c = 0; c < nk; c++)
    for(int b = 0; b < (1 << sh.y); b++)
      for(int a = 0; a < (1 << sh.x); a++)
      {
        int i = (ci << sh.x) + a, j = (cj << sh.y) + b, k = (ck << sh.z) + c;
        if(i < df.nx && j < df.ny && (df.dim == 2 || k < df.nz))
          s += double(Ef[i + (long long)j * df.nx + (long long)k * df.nx * df.ny]);
      }
  Ec[e] = T(s / double((1 << sh.x) * (1 << sh.y) * nk));
}
template <typename T>
__global__ void k_coarsen_E(Dims df, Dims dc, int3 sh, const T *__restrict__ Ef,
                            T *__restrict__ Ec)
{
  coarsen_E_b<T>(df, dc, sh, Ef, Ec, this_block());
}

/// b_c = R r_f (R = P^T), constrained coarse DOFs zeroed.  One thread per
/// coarse node (x along threads, y and z along the grid, so no index
/// division): along a halved axis the 1-D weights of the fine neighbours
/// 2I-1, 2I, 2I+1 are 1/2, 1, 1/2 (those inside the fine grid), along a kept
/// axis (shift 0) the fine node I alone has weight 1; applied row by row.
template <typename T>
__device__ __forceinline__ void restrict_b(Dims df, Dims dc, int3 sh, const T *__restrict__ rf,
                           T *__restrict__ bc, const uint8_t *__restrict__ fixc,
                           const KState *gate, const Blk &B)
{
  if(gated(gate))
    return;
  const int I = B.x * blockDim.x + threadIdx.x, J = B.y, K = B.z;
  if(I >= dc.sx)
    return;
  const long long fsxy = (long long)df.sx * df.sy;
  const int kr = df.dim == 3 ? sh.z : 0;
  const T h = T(0.5);
  T s[3] = {T(0), T(0), T(0)};
  for(int dk = -kr; dk <= kr; dk++)
  {
    const int k = (K << sh.z) + dk;
    if(k < 0 || k >= df.sz)
      continue;
    T sk[3] = {T(0), T(0), T(0)};
    for(int dj = -sh.y; dj <= sh.y; dj++)
    {
      const int j = (J << sh.y) + dj;
      if(j < 0 || j >= df.sy)
        continue;
      const long long row = (long long)j * df.sx + (long long)k * fsxy;
      const int i = I << sh.x;
      const bool lo = sh.x && i - 1 >= 0, mid = i < df.sx, hi = sh.x && i + 1 < df.sx;
#pragma unroll
      for(int c = 0; c < 3; c++)
        if(c < df.dim)
        {
          const T *r = rf + c * df.ld + row;
          const T v = (mid ? r[i] : T(0)) + h * ((lo ? r[i - 1] : T(0)) + (hi ? r[i + 1] : T(0)));
          sk[c] = dj ? fma(h, v, sk[c]) : sk[c] + v;
        }
    }
#pragma unroll
    for(int c = 0; c < 3; c++)
      s[c] = dk ? fma(h, sk[c], s[c]) : s[c] + sk[c];
  }
  const long long n = I + (long long)J * dc.sx + (long long)K * dc.sx * dc.sy;
  const unsigned fx = fixc[n];
#pragma unroll
  for(int c = 0; c < 3; c++)
    if(c < dc.dim)
      bc[c * dc.ld + n] = ((fx >> c) & 1u) ? T(0) : s[c];
}
template <typename T>
__global__ void k_restrict(Dims df, Dims dc, int3 sh, const T *__restrict__ rf,
                           T *__restrict__ bc, const uint8_t *__restrict__ fixc,
                           const KState *gate)
{
  restrict_b<T>(df, dc, sh, rf, bc, fixc, gate, this_block());
}

/// x_f += P x_c, constrained fine DOFs untouched (they stay 0).  One thread
/// per fine node of kProlongRows node rows (x along threads, a group of rows
/// and z along the grid): the trilinear interpolant as three nested
/// midpoints; an even index on a halved axis, and every index on a kept one,
/// takes the same coarse node twice, which the midpoint returns exactly.  The
/// thread loads its rows' fine values and flags first and then the coarse
/// values, so the loads of all its rows are in flight together.
constexpr int kProlongRows = 4;
template <typename T>
__device__ __forceinline__ void prolong_rows_b(const Dims &df, const Dims &dc, const int3 &sh,
                                               const T *__restrict__ xc, T *__restrict__ xf,
                                               const uint8_t *__restrict__ fixf, int i, int j0,
                                               int k)
{
  if(i >= df.sx)
    return;
  constexpr int R = kProlongRows;
  const long long fsxy = (long long)df.sx * df.sy;
  T old[R][3];
  unsigned fx[R];
#pragma unroll
  for(int r = 0; r < R; r++)
  {
    const int j = j0 + r;
    const long long n = i + (long long)j * df.sx + (long long)k * fsxy;
    fx[r] = j < df.sy ? unsigned(fixf[n]) : 7u; // a row past the grid: nothing to do
#pragma unroll
    for(int c = 0; c < 3; c++)
      old[r][c] = c < df.dim && !((fx[r] >> c) & 1u) ? xf[c * df.ld + n] : T(0);
  }
  const int I0 = i >> sh.x, I1 = (i + sh.x) >> sh.x;
  const int K0 = k >> sh.z, K1 = df.dim == 3 ? (k + sh.z) >> sh.z : K0;
  const long long csxy = (long long)dc.sx * dc.sy;
  const T h = T(0.5);
#pragma unroll
  for(int r = 0; r < R; r++)
  {
    const int j = j0 + r;
    const int J0 = j >> sh.y, J1 = (j + sh.y) >> sh.y;
    const long long r00 = (long long)J0 * dc.sx + K0 * csxy, r10 = (long long)J1 * dc.sx + K0 * csxy;
    const long long r01 = (long long)J0 * dc.sx + K1 * csxy, r11 = (long long)J1 * dc.sx + K1 * csxy;
    const long long n = i + (long long)j * df.sx + (long long)k * fsxy;
#pragma unroll
    for(int c = 0; c < 3; c++)
      if(c < df.dim && !((fx[r] >> c) & 1u))
      {
        const T *x = xc + c * dc.ld;
        const T a = h * (x[r00 + I0] + x[r00 + I1]), b = h * (x[r10 + I0] + x[r10 + I1]);
        const T a2 = h * (x[r01 + I0] + x[r01 + I1]), b2 = h * (x[r11 + I0] + x[r11 + I1]);
        xf[c * df.ld + n] = old[r][c] + h * (h * (a + b) + h * (a2 + b2));
      }
  }
}
/// rows of a prolongation launch block: kProlongRows node rows each
inline unsigned prolong_row_blocks(const Dims &d)
{
  return unsigned((d.sy + kProlongRows - 1) / kProlongRows);
}
template <typename T>
__global__ void k_prolong_add(Dims df, Dims dc, int3 sh, const T *__restrict__ xc,
                              T *__restrict__ xf, const uint8_t *__restrict__ fixf,
                              const KState *gate)
{
  if(gated(gate))
    return;
  prolong_rows_b<T>(df, dc, sh, xc, xf, fixf, blockIdx.x * blockDim.x + threadIdx.x,
                    blockIdx.y * kProlongRows, blockIdx.z);
}

/// first smoothing step from a zero guess: x = c D^-1 b, x0 = 0
template <typename T>
__device__ __forceinline__ void jacobi0_b(long long n, T c, const T *__restrict__ dinv,
                          const T *__restrict__ b, T *__restrict__ x, T *__restrict__ x0,
                          const KState *gate, const Blk &B)
{
  if(gated(gate))
    return;
  const long long st = (long long)B.gx * blockDim.x;
  for(long long i0 = B.x * (long long)blockDim.x + threadIdx.x; i0 < n; i0 += kGroup * st)
  {
    T dv[kGroup], bv[kGroup];
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * st;
      dv[g] = i < n ? dinv[i] : T(0);
      bv[g] = i < n ? b[i] : T(0);
    }
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * st;
      if(i < n)
      {
        x[i] = c * dv[g] * bv[g];
        x0[i] = T(0); // the iterate before x, for the next three-term step
      }
    }
  }
}
template <typename T>
__global__ void k_jacobi0(long long n, T c, const T *__restrict__ dinv,
                          const T *__restrict__ b, T *__restrict__ x, T *__restrict__ x0,
                          const KState *gate)
{
  jacobi0_b<T>(n, c, dinv, b, x, x0, gate, this_block());
}

// --------------------------------------------------------- coarse level ----
/// Dense coarse matrix, row by row: the thread of free DOF (node n, c) adds
/// the rows of its <= 8 elements in element order.  Each row has one writer,
/// so the sums are deterministic (no atomics).
template <typename T>
__device__ __forceinline__ void dense_assemble_b(Dims d, KMat<double, 24> K, const T *__restrict__ E,
                                 const int *__restrict__ dense, int n, double *A, const Blk &B)
{
  long long t = B.x * (long long)blockDim.x + threadIdx.x;
  if(t >= (long long)d.nnode * d.dim)
    return;
  const int c = int(t % d.dim);
  const long long nd = t / d.dim;
  const int row = dense[c * d.ld + nd];
  if(row < 0)
    return;
  const int ne = d.dim == 2 ? 4 : 8, ndof = ne * d.dim;
  const long long sxy = (long long)d.sx * d.sy;
  const int i = int(nd % d.sx), j = int((nd / d.sx) % d.sy), k = d.dim == 3 ? int(nd / sxy) : 0;
  double *Arow = A + (long long)row * n;
  for(int dk = (d.dim == 3 ? -1 : 0); dk <= 0; dk++)
    for(int dj = -1; dj <= 0; dj++)
      for(int di = -1; di <= 0; di++)
      {
        int ei = i + di, ej = j + dj, ek = k + dk;
        if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (d.dim == 3 && ek >= d.nz))
          continue;
        const int a = ((-di) ^ (-dj)) + 2 * (-dj) + (d.dim == 3 ? 4 * (-dk) : 0);
        const double Ee = double(E[ei + (long long)ej * d.nx + (long long)ek * d.nx * d.ny]);
        const long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
        for(int l = 0; l < ne; l++)
        {
          int q = l & 3, top = l >> 2;
          long long node = base + ((q == 1 || q == 2) ? 1 : 0) + (q >= 2 ? d.sx : 0) + top * sxy;
          for(int c2 = 0; c2 < d.dim; c2++)
          {
            int col = dense[c2 * d.ld + node];
            if(col >= 0)
              Arow[col] += Ee * K.k[(a * d.dim + c) * ndof + l * d.dim + c2];
          }
        }
      }
}
template <typename T>
__global__ void k_dense_assemble(Dims d, KMat<double, 24> K, const T *__restrict__ E,
                                 const int *__restrict__ dense, int n, double *A)
{
  dense_assemble_b<T>(d, K, E, dense, n, A, this_block());
}

/// In-place Gauss-Jordan inversion of the SPD coarse matrix (no pivoting is
/// needed for SPD).  One CTA; a non-positive pivot is recorded in *status
/// and replaced by a tiny positive value so the preconditioner stays usable.
/// SMEM: the matrix is worked on in shared memory (n^2 doubles, n <=
/// kInvSmemMax) and copied back once; otherwise in place in global memory
/// (L2-resident).  Warp w updates rows w, w + 32, ..., its lanes the columns.
constexpr int kInvSmemMax = 160;
template <bool SMEM>
__device__ __forceinline__ void invert_spd_b(int n, double *Ag, int *status)
{
  extern __shared__ double sA[];
  __shared__ double rowk[1024];
  __shared__ double colk[1024];
  __shared__ double piv;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int warp = tid >> 5, lane = tid & 31, nwarp = nth >> 5;
  double *A = SMEM ? sA : Ag;
  if(SMEM)
  {
    for(int t = tid; t < n * n; t += nth)
      sA[t] = Ag[t];
    __syncthreads();
  }
  double dmax = 0.0;
  for(int i = 0; i < n; i++)
    dmax = fmax(dmax, A[(long long)i * n + i]);
  for(int k = 0; k < n; k++)
  {
    if(tid == 0)
    {
      double p = A[(long long)k * n + k];
      if(!(p > 1e-14 * dmax))
      {
        status[0] = k + 1;
        p = fmax(1e-14 * dmax, DBL_MIN);
      }
      piv = p;
    }
    __syncthreads();
    const double p = piv;
    for(int j = tid; j < n; j += nth)
    {
      rowk[j] = (j == k ? 1.0 : A[(long long)k * n + j]) / p;
      colk[j] = A[(long long)j * n + k];
    }
    __syncthreads();
    for(int i = warp; i < n; i += nwarp)
    {
      double *Ai = A + (long long)i * n;
      const double f = colk[i];
      if(i == k)
        for(int j = lane; j < n; j += 32)
          Ai[j] = rowk[j];
      else
        for(int j = lane; j < n; j += 32)
          Ai[j] = (j == k ? 0.0 : Ai[j]) - f * rowk[j];
    }
    __syncthreads();
  }
  if(SMEM)
    for(int t = tid; t < n * n; t += nth)
      Ag[t] = sA[t];
}
template <bool SMEM>
__global__ void __launch_bounds__(1024) k_invert_spd(int n, double *Ag, int *status)
{
  invert_spd_b<SMEM>(n, Ag, status);
}

/// x_c = A^-1 b_c over the free coarse DOFs (warp per row)
template <typename T>
__device__ __forceinline__ void dense_apply_b(int n, const double *__restrict__ Ainv,
                              const long long *__restrict__ soa, const T *__restrict__ b,
                              T *__restrict__ x, const KState *gate, const Blk &B)
{
  if(gated(gate))
    return;
  extern __shared__ double sb[];
  for(int j = threadIdx.x; j < n; j += blockDim.x)
    sb[j] = double(b[soa[j]]);
  __syncthreads();
  int warp = (B.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  int nw = (B.gx * blockDim.x) >> 5;
  for(int i = warp; i < n; i += nw)
  {
    double s = 0.0;
    for(int j = lane; j < n; j += 32)
      s += Ainv[(long long)i * n + j] * sb[j];
    s = warp_sum_d(s);
    if(lane == 0)
      x[soa[i]] = T(s);
  }
}
template <typename T>
__global__ void k_dense_apply(int n, const double *__restrict__ Ainv,
                              const long long *__restrict__ soa, const T *__restrict__ b,
                              T *__restrict__ x, const KState *gate)
{
  dense_apply_b<T>(n, Ainv, soa, b, x, gate, this_block());
}

template <typename T>
__device__ __forceinline__ void fill_b(long long n, T v, T *__restrict__ x, const Blk &B)
{
  for(long long i = B.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)B.gx * blockDim.x)
    x[i] = v;
}
template <typename T>
__global__ void k_fill(long long n, T v, T *__restrict__ x)
{
  fill_b<T>(n, v, x, this_block());
}

// ------------------------------------------------------------- MG-PCG ------
// Flexible (Polak-Ribiere) CG in precision TK preconditioned by a V-cycle in
// precision TP.  TK = TP = double is the FP64 GMG path; TK = double,
// TP = float is the mixed path: FP64 iterate, residual, operator and
// reductions, FP32 multigrid.  The precision casts are fused into the Krylov
// kernels (rP = TP(r) written by the residual update, z read as TP).
struct FinInitMg
{
  KState *st;
  double tol;
  int maxit;
  __device__ void operator()(const double *t) const
  {
    st->bb = t[0];
    st->rr = t[0];
    st->tol = tol;
    st->thr = fmax(tol * tol * t[0], DBL_MIN);
    st->iter = 0;
    st->pad = 0;
    st->matvecs = 0;
    st->maxit = maxit;
    st->conv = 0;
    st->alpha = st->beta = 0.0;
    st->status = ICB_OK;
    st->stop = 0;
    if(!isfinite(t[0]))
    {
      st->status = ICB_ERR_NAN;
      st->stop = 1;
    }
    else if(t[0] == 0.0 || t[0] < st->thr)
      st->stop = 1;
  }
};

template <typename TK, typename TP>
__device__ __forceinline__ void mg_init_b(long long n, const TK *__restrict__ b, TK *__restrict__ x,
                          TK *__restrict__ r, TP *__restrict__ rP, RedScratch red, KState *st,
                          double tol, int maxit, const Blk &B)
{
  double v[1] = {0.0};
  const long long sd = (long long)B.gx * blockDim.x;
  for(long long i0 = B.x * (long long)blockDim.x + threadIdx.x; i0 < n; i0 += kGroup * sd)
  {
    TK bv[kGroup];
#pragma unroll
    for(int g = 0; g < kGroup; g++)
      bv[g] = i0 + g * sd < n ? b[i0 + g * sd] : TK(0);
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * sd;
      if(i < n)
      {
        const TK bi = bv[g];
        r[i] = bi;
        if(rP)
          rP[i] = TP(bi);
        x[i] = TK(0);
        v[0] += double(bi) * double(bi);
      }
    }
  }
  block_reduce_at<1>(v, red, FinInitMg{st, tol, maxit}, int(B.x), int(B.gx));
}
template <typename TK, typename TP>
__global__ void k_mg_init(long long n, const TK *__restrict__ b, TK *__restrict__ x,
                          TK *__restrict__ r, TP *__restrict__ rP, RedScratch red, KState *st,
                          double tol, int maxit)
{
  mg_init_b<TK, TP>(n, b, x, r, rP, red, st, tol, maxit, this_block());
}

struct FinRz0
{
  KState *st;
  __device__ void operator()(const double *t) const
  {
    st->rz = t[0];
    if(!isfinite(t[0]) || !(t[0] > 0.0))
    {
      st->status = isfinite(t[0]) ? ICB_ERR_BREAKDOWN : ICB_ERR_NAN;
      st->stop = 1;
    }
  }
};

/// p = z; rz = r.z
template <typename TK, typename TP>
__device__ __forceinline__ void mg_init2_b(long long n, const TK *__restrict__ r, const TP *__restrict__ z,
                           TK *__restrict__ p, RedScratch red, KState *st, const Blk &B)
{
  if(st->stop)
    return;
  double v[1] = {0.0};
  const long long sd = (long long)B.gx * blockDim.x;
  for(long long i0 = B.x * (long long)blockDim.x + threadIdx.x; i0 < n; i0 += kGroup * sd)
  {
    TP zv[kGroup];
    TK rv[kGroup];
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * sd;
      zv[g] = i < n ? z[i] : TP(0);
      rv[g] = i < n ? r[i] : TK(0);
    }
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * sd;
      if(i < n)
      {
        TK zi = TK(zv[g]);
        p[i] = zi;
        v[0] += double(rv[g]) * double(zi);
      }
    }
  }
  block_reduce_at<1>(v, red, FinRz0{st}, int(B.x), int(B.gx));
}
template <typename TK, typename TP>
__global__ void k_mg_init2(long long n, const TK *__restrict__ r, const TP *__restrict__ z,
                           TK *__restrict__ p, RedScratch red, KState *st)
{
  mg_init2_b<TK, TP>(n, r, z, p, red, st, this_block());
}

struct FinRmg
{
  KState *st;
  double pq, alpha;
  bool bad;
  __device__ void operator()(const double *t) const
  {
    st->matvecs++;
    if(bad)
    {
      st->status = ICB_ERR_BREAKDOWN;
      st->stop = 1;
      return;
    }
    st->pq = pq;
    st->alpha = alpha;
    st->rr = t[0];
    st->rzo = t[1];
    if(!isfinite(t[0]))
    {
      st->status = ICB_ERR_NAN;
      st->stop = 1;
    }
    else if(t[0] < st->thr)
      st->conv = 1;
  }
};

/// r -= alpha q (and rP = TP(r)); sums r.r and r.z_old (z still holds the
/// previous preconditioned residual) for the flexible beta
template <typename TK, typename TP>
__device__ __forceinline__ void mg_r_b(long long n, TK *__restrict__ r, TP *__restrict__ rP,
                       const TK *__restrict__ q, const TP *__restrict__ zold,
                       const double *__restrict__ pq, RedScratch red, KState *st, const Blk &B)
{
  if(st->stop)
    return;
  const double pqv = *pq;
  const double alpha = st->rz / pqv;
  const bool bad = !(pqv > 0.0) || !isfinite(alpha);
  double v[2] = {0.0, 0.0};
  if(!bad)
  {
    const TK a = TK(alpha);
    const long long sd = (long long)B.gx * blockDim.x;
    for(long long i0 = B.x * (long long)blockDim.x + threadIdx.x; i0 < n; i0 += kGroup * sd)
    {
      TK rv[kGroup], qv[kGroup];
      TP zv[kGroup];
#pragma unroll
      for(int g = 0; g < kGroup; g++)
      {
        const long long i = i0 + g * sd;
        rv[g] = i < n ? r[i] : TK(0);
        qv[g] = i < n ? q[i] : TK(0);
        zv[g] = i < n ? zold[i] : TP(0);
      }
#pragma unroll
      for(int g = 0; g < kGroup; g++)
      {
        const long long i = i0 + g * sd;
        if(i < n)
        {
          TK ri = rv[g] - a * qv[g];
          r[i] = ri;
          if(rP)
            rP[i] = TP(ri);
          v[0] += double(ri) * double(ri);
          v[1] += double(ri) * double(zv[g]);
        }
      }
    }
  }
  block_reduce_at<2>(v, red, FinRmg{st, pqv, alpha, bad}, int(B.x), int(B.gx));
}
template <typename TK, typename TP>
__global__ void k_mg_r(long long n, TK *__restrict__ r, TP *__restrict__ rP,
                       const TK *__restrict__ q, const TP *__restrict__ zold,
                       const double *__restrict__ pq, RedScratch red, KState *st)
{
  mg_r_b<TK, TP>(n, r, rP, q, zold, pq, red, st, this_block());
}

struct FinRz
{
  KState *st;
  __device__ void operator()(const double *t) const
  {
    if(!isfinite(t[0]))
    {
      st->status = ICB_ERR_NAN;
      st->stop = 1;
      return;
    }
    // Polak-Ribiere (flexible CG): tolerates a V-cycle that is only
    // symmetric up to rounding, and a preconditioner in lower precision
    st->beta = (t[0] - st->rzo) / st->rz;
    st->rz = t[0];
  }
};

template <typename TK, typename TP>
__device__ __forceinline__ void mg_rz_b(long long n, const TK *__restrict__ r, const TP *__restrict__ z,
                        RedScratch red, KState *st, const Blk &B)
{
  if(st->stop || st->conv)
    return;
  double v[1] = {0.0};
  const long long sd = (long long)B.gx * blockDim.x;
  for(long long i0 = B.x * (long long)blockDim.x + threadIdx.x; i0 < n; i0 += kGroup * sd)
  {
    TK rv[kGroup];
    TP zv[kGroup];
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * sd;
      rv[g] = i < n ? r[i] : TK(0);
      zv[g] = i < n ? z[i] : TP(0);
    }
#pragma unroll
    for(int g = 0; g < kGroup; g++)
      if(i0 + g * sd < n)
        v[0] += double(rv[g]) * double(zv[g]);
  }
  block_reduce_at<1>(v, red, FinRz{st}, int(B.x), int(B.gx));
}
template <typename TK, typename TP>
__global__ void k_mg_rz(long long n, const TK *__restrict__ r, const TP *__restrict__ z,
                        RedScratch red, KState *st)
{
  mg_rz_b<TK, TP>(n, r, z, red, st, this_block());
}

struct FinXPmg
{
  KState *st;
  LoopCtl L;
  __device__ void operator()(const double *) const
  {
    if(st->conv)
      st->stop = 1;
    else
    {
      st->iter++;
      if(st->iter >= st->maxit)
      {
        st->status = ICB_ERR_MAXITER;
        st->stop = 1;
      }
    }
    loop_end_krylov(L, st);
  }
};

/// the last kernel of an iteration; inside the solve graph it also decides
/// whether the device runs the next one
template <typename TK, typename TP>
__device__ __forceinline__ void mg_xp_b(long long n, TK *__restrict__ x, TK *__restrict__ p,
                        const TP *__restrict__ z, RedScratch red, KState *st, LoopCtl L, const Blk &B)
{
  if(st->stop)
  {
    if(B.x == 0 && threadIdx.x == 0)
      loop_stop(L);
    return;
  }
  const TK a = TK(st->alpha), bt = TK(st->beta);
  const bool conv = st->conv;
  const long long sd = (long long)B.gx * blockDim.x;
  for(long long i0 = B.x * (long long)blockDim.x + threadIdx.x; i0 < n; i0 += kGroup * sd)
  {
    TK pv[kGroup], xv[kGroup];
    TP zv[kGroup];
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * sd;
      pv[g] = i < n ? p[i] : TK(0);
      xv[g] = i < n ? x[i] : TK(0);
      zv[g] = i < n && !conv ? z[i] : TP(0);
    }
#pragma unroll
    for(int g = 0; g < kGroup; g++)
    {
      const long long i = i0 + g * sd;
      if(i < n)
      {
        const TK pi = pv[g];
        x[i] = xv[g] + a * pi;
        if(!conv)
          p[i] = TK(zv[g]) + bt * pi;
      }
    }
  }
  double v[1] = {0.0};
  block_reduce_at<1>(v, red, FinXPmg{st, L}, int(B.x), int(B.gx));
}
template <typename TK, typename TP>
__global__ void k_mg_xp(long long n, TK *__restrict__ x, TK *__restrict__ p,
                        const TP *__restrict__ z, RedScratch red, KState *st, LoopCtl L)
{
  mg_xp_b<TK, TP>(n, x, p, z, red, st, L, this_block());
}
} // namespace

// ============================================================ hierarchy ====
/// lambda_max(diag(K0)^-1 K0) by power iteration on D^-1/2 K0 D^-1/2 (host)
template <typename T> double element_lmax(int dim, const T *K)
{
  const int nd = dim == 2 ? 8 : 24;
  std::vector<double> M(nd * nd), v(nd, 1.0), w(nd);
  for(int i = 0; i < nd; i++)
    for(int j = 0; j < nd; j++)
      M[i * nd + j] = double(K[i * nd + j]) / std::sqrt(double(K[i * nd + i]) * double(K[j * nd + j]));
  for(int i = 0; i < nd; i++)
    v[i] = 1.0 + 0.1 * i;
  double lam = 0.0;
  for(int it = 0; it < 2000; it++)
  {
    double nn = 0.0;
    for(int i = 0; i < nd; i++)
    {
      double s = 0.0;
      for(int j = 0; j < nd; j++)
        s += M[i * nd + j] * v[j];
      w[i] = s;
      nn += s * s;
    }
    nn = std::sqrt(nn);
    lam = nn;
    for(int i = 0; i < nd; i++)
      v[i] = w[i] / nn;
  }
  return lam * 1.02;
}

template <typename T> struct Level
{
  Dims d;
  /// coarsening from the next finer level, per axis: 1 halves the element
  /// count (ceil), 0 keeps an axis that is one element thick
  int3 sh = make_int3(1, 1, 1);
  double h[3];
  T K[576]; ///< unit element matrix of this level (passed by value)
  DevBuf<T> Eown;
  const T *E = nullptr;
  DevBuf<uint8_t> fixOwn;
  const uint8_t *fix = nullptr;
  DevBuf<T> dinv, x, b, r, t;
};

/// Flexible CG in TK with a TP V-cycle (see the kernels above).
template <typename TK, typename TP> struct MgPcg
{
  std::vector<Level<TP>> lv;
  int nu = 2;
  /// Chebyshev interval [lmax/10, lmax] for D^-1 K; lmax is the element
  /// bound lambda_max(diag(K0)^-1 K0), which holds for any moduli E because
  /// x^T K x / x^T D x is a weighted mean of the element quotients.
  double lmax = 4.0;
  std::vector<double> cc1, cc2; ///< per-step Chebyshev coefficients
  // Krylov operator (fine level in TK)
  TK Kk[576];
  const TK *Ek = nullptr;
  // coarsest dense system
  int nc = 0;
  DevBuf<long long> cSoa;
  DevBuf<int> cDense;
  DevBuf<double> cA;
  DevBuf<int> cStatus;
  // Krylov vectors (fine level)
  long long n = 0;
  DevBuf<TK> r, p, q;
  DevBuf<TP> rP, z;
  DevBuf<KState> st;
  DevBuf<double> partials, dots;
  DevBuf<unsigned> counter;
  RedScratch red;
  KState *hst = nullptr;
  WhileGraph loop; ///< one FCG iteration, repeated on the device until stop
  GraphKey key;    ///< what `loop` bakes in besides this object's own buffers

  ~MgPcg()
  {
    if(hst)
      cudaFreeHost(hst);
  }

  static constexpr bool same() { return sizeof(TK) == sizeof(TP); }
  TP *rin() { return same() ? (TP *)r.p : rP.p; }

  /// level dims, element matrices and Dirichlet masks (host), device buffers
  void build(const HostSetup &hs, const TK *Kkrylov, const TK *Ekrylov, const TP *Kfine,
             const TP *Efine, const uint8_t *fixFine, int coarseDofs, int smooth,
             cudaStream_t s)
  {
    // all device initialisation goes to the solve's stream (the blocking
    // copies and memsets run on the legacy stream, which the library's
    // non-blocking streams do not wait for); host staging is synchronised
    // before it goes out of scope
    nu = smooth > 0 ? smooth : 2;
    lmax = element_lmax(hs.desc.dim, Kfine);
    bool shapeChanged = false;
    std::copy(Kkrylov, Kkrylov + 576, Kk);
    Ek = Ekrylov;
    Level<TP> L0;
    L0.d = hs.dims;
    std::memcpy(L0.h, hs.h, sizeof(L0.h));
    std::copy(Kfine, Kfine + 576, L0.K);
    L0.E = Efine;
    L0.fix = fixFine;
    lv.clear();
    lv.push_back(std::move(L0));
    std::vector<uint8_t> fm(hs.dims.nnode, 0);
    for(long long nd = 0; nd < hs.dims.nnode; nd++)
      for(int c = 0; c < hs.desc.dim; c++)
        if(hs.fixed[nd * hs.desc.dim + c])
          fm[nd] |= uint8_t(1u << c);
    const int dim = hs.desc.dim;
    // default: coarsen until the grid has <= 160 DOFs, so the coarsest
    // matrix is inverted in shared memory (600 DOFs cost 14.6 ms a density)
    const int cd = coarseDofs > 0 ? coarseDofs : kInvSmemMax;
    while(true)
    {
      const Dims &f = lv.back().d;
      long long dofs = f.nnode * dim;
      // semi-coarsening: an axis one element thick is kept, the others halve
      const int3 sh = make_int3(f.nx >= 2, f.ny >= 2, dim == 3 && f.nz >= 2);
      if(dofs <= cd || !(sh.x || sh.y || sh.z))
        break;
      Level<TP> c;
      c.sh = sh;
      c.d = make_dims(dim, sh.x ? (f.nx + 1) / 2 : f.nx, sh.y ? (f.ny + 1) / 2 : f.ny,
                      dim == 3 ? (sh.z ? (f.nz + 1) / 2 : f.nz) : 1);
      const int shk[3] = {sh.x, sh.y, sh.z};
      for(int k = 0; k < 3; k++)
        c.h[k] = shk[k] ? 2.0 * lv.back().h[k] : lv.back().h[k];
      double Kd[576];
      unit_stiffness(dim, hs.desc.state, hs.desc.poisson, c.h, Kd);
      for(int i = 0; i < 576; i++)
        c.K[i] = TP(Kd[i]);
      // the elements change shape when some axes halve and others do not;
      // the smoother's bound must then hold for this level's K0 too
      if(sh.x != sh.y || (dim == 3 && sh.y != sh.z))
        shapeChanged = true;
      if(shapeChanged)
        lmax = std::max(lmax, element_lmax(dim, c.K));
      // coarse mask: a coarse DOF is constrained when a constrained fine DOF
      // interpolates from it (P(i, I) != 0); for constraints on even grid
      // lines this is the fine DOF at the same point, a constraint at an odd
      // index (a point support between coarse nodes) constrains the coarse
      // neighbours so the coarse operator never loses it.
      std::vector<uint8_t> cm(c.d.nnode, 0);
      for(long long nd = 0; nd < f.nnode; nd++)
      {
        if(!fm[nd])
          continue;
        long long i = nd % f.sx, j = (nd / f.sx) % f.sy, k = nd / ((long long)f.sx * f.sy);
        long long I0 = i >> sh.x, I1 = (i + sh.x) >> sh.x, J0 = j >> sh.y,
                  J1 = (j + sh.y) >> sh.y, K0 = k >> sh.z, K1 = dim == 3 ? (k + sh.z) >> sh.z : 0;
        for(long long K = K0; K <= K1; K++)
          for(long long J = J0; J <= J1; J++)
            for(long long I = I0; I <= I1; I++)
              cm[I + J * c.d.sx + K * (long long)c.d.sx * c.d.sy] |= fm[nd];
      }
      c.fixOwn.alloc(c.d.nnode);
      ICB_CUDA(cudaMemcpyAsync(c.fixOwn.p, cm.data(), cm.size(), cudaMemcpyHostToDevice, s));
      ICB_CUDA(cudaStreamSynchronize(s));
      c.fix = c.fixOwn.p;
      c.Eown.alloc(c.d.nel);
      c.E = c.Eown.p;
      fm.swap(cm);
      lv.push_back(std::move(c));
    }
    // Chebyshev coefficients of steps 0..nu-1 (Saad, Iterative Methods for
    // Sparse Linear Systems, 2nd ed., Alg. 12.1) on [lmax/10, lmax]
    {
      double a = lmax / 10.0, b = lmax, theta = 0.5 * (b + a), delta = 0.5 * (b - a);
      double sigma = theta / delta, rho0 = 1.0 / sigma;
      cc1.assign(nu, 0.0);
      cc2.assign(nu, 0.0);
      cc2[0] = 1.0 / theta;
      for(int k = 1; k < nu; k++)
      {
        double rho1 = 1.0 / (2.0 * sigma - rho0);
        cc1[k] = rho1 * rho0;
        cc2[k] = 2.0 * rho1 / delta;
        rho0 = rho1;
      }
    }
    for(size_t l = 0; l < lv.size(); l++)
    {
      long long m = (long long)dim * lv[l].d.ld;
      lv[l].dinv.alloc(m);
      lv[l].r.alloc(m);
      lv[l].t.alloc(m);
      if(l > 0)
      {
        lv[l].x.alloc(m);
        lv[l].b.alloc(m);
      }
      for(DevBuf<TP> *v : {&lv[l].dinv, &lv[l].r, &lv[l].t, &lv[l].x, &lv[l].b})
        if(v->p)
          ICB_CUDA(cudaMemsetAsync(v->p, 0, v->bytes(), s));
    }
    // coarsest dense index map
    const Level<TP> &C = lv.back();
    std::vector<uint8_t> cmask(C.d.nnode);
    ICB_CUDA(cudaMemcpyAsync(cmask.data(), C.fix, C.d.nnode, cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    std::vector<int> dense((size_t)dim * C.d.ld, -1);
    std::vector<long long> soa;
    for(long long nd = 0; nd < C.d.nnode; nd++)
      for(int c = 0; c < dim; c++)
        if(!((cmask[nd] >> c) & 1u))
        {
          dense[c * C.d.ld + nd] = int(soa.size());
          soa.push_back(c * C.d.ld + nd);
        }
    nc = int(soa.size());
    if(nc > 1024)
      throw Error{ICB_ERR_BAD_ARG, "coarsest grid too large for the dense solve (>1024 DOFs)"};
    cSoa.alloc(std::max(nc, 1));
    cDense.alloc(dense.size());
    if(nc)
      ICB_CUDA(cudaMemcpyAsync(cSoa.p, soa.data(), sizeof(long long) * nc, cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaMemcpyAsync(cDense.p, dense.data(), sizeof(int) * dense.size(),
                             cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    cA.alloc((size_t)std::max(nc, 1) * std::max(nc, 1));
    cStatus.alloc(1);
    n = (long long)dim * lv[0].d.ld;
    for(DevBuf<TK> *v : {&r, &p, &q})
    {
      v->alloc(n);
      ICB_CUDA(cudaMemsetAsync(v->p, 0, v->bytes(), s));
    }
    z.alloc(n);
    ICB_CUDA(cudaMemsetAsync(z.p, 0, z.bytes(), s));
    if(!same())
    {
      rP.alloc(n);
      ICB_CUDA(cudaMemsetAsync(rP.p, 0, rP.bytes(), s));
    }
    st.alloc(1);
    int mb = reduction_blocks(lv[0].d);
    partials.alloc((size_t)mb * 2);
    dots.alloc(4);
    counter.alloc(1);
    ICB_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), s));
    red = RedScratch{partials.p, counter.p, mb};
    ICB_CUDA(cudaMallocHost(&hst, sizeof(KState)));
  }

  /// per density: coarse moduli, diagonals, coarse inverse
  void refresh(cudaStream_t s)
  {
    for(size_t l = 1; l < lv.size(); l++)
    {
      k_coarsen_E<TP><<<nblocks(lv[l].d.nel, 256), 256, 0, s>>>(lv[l - 1].d, lv[l].d, lv[l].sh,
                                                                lv[l - 1].E, lv[l].Eown.p);
      count_launch();
    }
    for(auto &L : lv)
      launch_diag<TP>(L.d, L.K, L.E, L.fix, L.dinv.p, nullptr, s);
    const Level<TP> &C = lv.back();
    if(nc)
    {
      ICB_CUDA(cudaMemsetAsync(cA.p, 0, sizeof(double) * (size_t)nc * nc, s));
      ICB_CUDA(cudaMemsetAsync(cStatus.p, 0, sizeof(int), s));
      KMat<double, 24> kd;
      for(int i = 0; i < 576; i++)
        kd.k[i] = double(C.K[i]);
      k_dense_assemble<TP><<<nblocks(C.d.nnode * C.d.dim, 128), 128, 0, s>>>(C.d, kd, C.E,
                                                                            cDense.p, nc, cA.p);
      if(nc <= kInvSmemMax)
      {
        // the shared-memory opt-in is a per-device function attribute shared by
        // every host thread: always set it to the largest size, so threads of
        // the batch runner never shrink it under one another's launch
        ICB_CUDA(cudaFuncSetAttribute(k_invert_spd<true>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      int(sizeof(double)) * kInvSmemMax * kInvSmemMax));
        k_invert_spd<true><<<1, 1024, int(sizeof(double)) * nc * nc, s>>>(nc, cA.p, cStatus.p);
      }
      else
        k_invert_spd<false><<<1, 1024, 0, s>>>(nc, cA.p, cStatus.p);
      count_launch(2);
    }
    ICB_CUDA(cudaGetLastError());
  }

  void coarseSolve(const TP *b, TP *x, cudaStream_t s, const KState *gate)
  {
    const Level<TP> &C = lv.back();
    long long m = (long long)C.d.dim * C.d.ld;
    k_fill<TP><<<vblocks(m), VB, 0, s>>>(m, TP(0), x);
    count_launch();
    if(nc)
    {
      k_dense_apply<TP><<<8, 256, sizeof(double) * nc, s>>>(nc, cA.p, cSoa.p, b, x, gate);
      count_launch();
    }
  }

  /// out = V-cycle(b) on level l
  void level(size_t l, const TP *b, TP *out, cudaStream_t s, const KState *gate)
  {
    Level<TP> &L = lv[l];
    if(l + 1 == lv.size())
    {
      coarseSolve(b, out, s, gate);
      return;
    }
    long long m = (long long)L.d.dim * L.d.ld;
    // step 0 from zero, then 2nu-1 operator steps: an odd number of
    // ping-pongs ends in out
    TP *cur = L.t.p, *oth = out;
    k_jacobi0<TP><<<vblocks(m), VB, 0, s>>>(m, TP(cc2[0]), L.dinv.p, b, cur, oth, gate);
    count_launch();
    OpExtras<TP> ch;
    ch.mode = OP_CHEB;
    ch.b = b;
    ch.dinv = L.dinv.p;
    ch.gate = gate;
    ch.gateConv = 1;
    for(int k = 1; k < nu; k++)
    {
      ch.c1 = cc1[k];
      ch.c2 = cc2[k];
      launch_op<TP>(L.d, L.K, L.E, cur, oth, L.fix, s, ch);
      std::swap(cur, oth);
    }
    OpExtras<TP> res;
    res.mode = OP_RESIDUAL;
    res.b = b;
    res.gate = gate;
    res.gateConv = 1;
    launch_op<TP>(L.d, L.K, L.E, cur, L.r.p, L.fix, s, res);
    Level<TP> &Cn = lv[l + 1];
    k_restrict<TP><<<grid3(Cn.d), kTB, 0, s>>>(L.d, Cn.d, Cn.sh, L.r.p, Cn.b.p, Cn.fix, gate);
    count_launch();
    level(l + 1, Cn.b.p, Cn.x.p, s, gate);
    dim3 gp = grid3(L.d);
    gp.y = prolong_row_blocks(L.d);
    k_prolong_add<TP><<<gp, kTB, 0, s>>>(L.d, Cn.d, Cn.sh, Cn.x.p, cur, L.fix, gate);
    count_launch();
    for(int k = 0; k < nu; k++)
    {
      ch.c1 = cc1[k];
      ch.c2 = cc2[k];
      launch_op<TP>(L.d, L.K, L.E, cur, oth, L.fix, s, ch);
      std::swap(cur, oth);
    }
    if(cur != out)
      ICB_CUDA(cudaMemcpyAsync(out, cur, sizeof(TP) * m, cudaMemcpyDeviceToDevice, s));
  }

  void iteration(TK *x, cudaStream_t s, const LoopCtl &L)
  {
    const Dims &d = lv[0].d;
    int nb = vblocks(n);
    OpExtras<TK> a;
    a.dotRed = &red;
    a.dotOut = dots.p;
    a.gate = st.p;
    launch_op<TK>(d, Kk, Ek, p.p, q.p, lv[0].fix, s, a);
    k_mg_r<TK, TP><<<nb, VB, 0, s>>>(n, r.p, same() ? nullptr : rP.p, q.p, z.p, dots.p, red, st.p);
    level(0, rin(), z.p, s, st.p);
    k_mg_rz<TK, TP><<<nb, VB, 0, s>>>(n, r.p, z.p, red, st.p);
    k_mg_xp<TK, TP><<<nb, VB, 0, s>>>(n, x, p.p, z.p, red, st.p, L);
    count_launch(3);
  }

  int solve(const TK *b, TK *x, double tol, int maxit, cudaStream_t s, icb_solve_info *info)
  {
    int nb = vblocks(n);
    k_mg_init<TK, TP><<<nb, VB, 0, s>>>(n, b, x, r.p, same() ? nullptr : rP.p, red, st.p, tol,
                                         maxit);
    count_launch();
    level(0, rin(), z.p, s, nullptr);
    k_mg_init2<TK, TP><<<nb, VB, 0, s>>>(n, r.p, z.p, p.p, red, st.p);
    count_launch();
    ICB_CUDA(cudaGetLastError());
    return iterate(x, maxit, s, info);
  }

  /// the iteration graph for iterates x on stream s (built when anything it
  /// bakes in changed)
  void prepareLoop(TK *x, cudaStream_t s)
  {
    GraphKey k;
    k.add(x).add(Ek).add(lv[0].E).add((const void *)s).add((long long)kernel_switches());
    const bool dev = device_loops_enabled();
    if(loop.exec == nullptr || loop.device != dev || k != key)
    {
      const long long before = thread_launch_count();
      loop.build([&](cudaStream_t cs, const LoopCtl &L) { iteration(x, cs, L); }, dev, 8);
      count_launch(before - thread_launch_count()); // recorded, not launched
      key = k;
    }
  }
  /// device form: the iterations until the solve stops as one launch on s,
  /// and the final state copied to hst (valid once s is synchronised)
  void launchLoop(cudaStream_t s)
  {
    loop.launch(s);
    ICB_CUDA(cudaMemcpyAsync(hst, st.p, sizeof(KState), cudaMemcpyDeviceToHost, s));
  }

  /// the FCG iterations from the current state until the solve stops: the
  /// rest of a solve that solve() or a batched solve of many problems began
  /// (the same kernels per iteration, so the same iterates)
  int iterate(TK *x, int maxit, cudaStream_t s, icb_solve_info *info)
  {
    prepareLoop(x, s);
    if(loop.device)
    {
      // the whole solve: one launch, one wait
      launchLoop(s);
      ICB_CUDA(cudaStreamSynchronize(s));
      count_launch((long long)hst->pad * loop.graphNodes);
    }
    else
    {
      long long launched = 0;
      for(;;)
      {
        ICB_CUDA(cudaMemcpyAsync(hst, st.p, sizeof(KState), cudaMemcpyDeviceToHost, s));
        ICB_CUDA(cudaStreamSynchronize(s));
        if(hst->stop || launched > (long long)maxit + loop.batch)
          break;
        loop.launch(s);
        launched += loop.batch;
        count_launch(loop.graphNodes);
      }
    }
    if(info)
    {
      info->iters = hst->iter;
      info->matvecs = hst->matvecs;
      info->relres = hst->bb > 0 ? std::sqrt(hst->rr / hst->bb) : 0.0;
      info->status = hst->status;
    }
    return hst->status;
  }
};

/// the multigrid and mixed-precision solvers of one problem
struct Mixed
{
  int coarseDofs = -1, smooth = -1;
  std::unique_ptr<MgPcg<double, double>> mg64;
  std::unique_ptr<MgPcg<double, float>> mgmx;
  // defect correction: FP32 GMG-PCG inside an FP64 residual loop
  std::unique_ptr<MgPcg<float, float>> mg32;
  DevBuf<double> r64;
  DevBuf<float> r32, d32;
};
/// the problem's solvers, dropped and rebuilt when the multigrid options
/// (smoothing degree, coarsest size) change (mg.cu)
Mixed &mixed_of(icb_problem p, const icb_solve_opts &o);

} // namespace icb
