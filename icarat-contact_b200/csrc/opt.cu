// opt.cu -- density filter, threshold projection, OC and MMA updates on the
// device.
//
// * Cone filter: Filter<E,N>::densityFilter (src/optimization/filter.hpp:
//   102-151).  The neighbour set of ICARAT's O(N^2) preNeighbour scan
//   (filter.hpp:191-234) is, on a uniform grid, the set of integer element
//   offsets with |offset * h| <= r; it is built once on the host, in
//   increasing element-index order (the order preNeighbour lists them, so the
//   sums are taken in ICARAT's order), and the per-element weight sums aa
//   (dfilters_ds) are computed once on the device.
// * Threshold: Filter::threshold / thresholdDerivative (filter.hpp:153-185),
//   fused into the forward filter.
// * OC: OC::UpdateVariables (src/optimization/opt-solver/OCSolver.hpp:20-68)
//   with the volume callback of opt_macro_oc.cpp:155-164 (re-filter and
//   re-threshold the candidate).  A bisection step is two kernels: every
//   element's candidate once, then the filter stencil over the stored
//   candidates with the threshold and the volume reduction, whose last block
//   runs the bisection logic; a whole update is one CUDA graph with early
//   exit.  Many problems' updates run as batched launches (OcBatch).
// * MMA: Svanberg's MMA with ICARAT's MMASolver parameters
//   (MMASolver.cpp:41-55), m = 1: GenSub as one element pass, the dual
//   interior-point iteration as one fused pass per Newton step (x(lambda),
//   the dual gradient and Hessian sums) whose last block runs SolveDIP's
//   scalar logic (MMASolver.cpp:88-154, 214-344) as a state machine.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <vector>

#include "graphloop.hpp"
#include "opt.hpp"
#include "batchq.cuh"
#include "reduce.cuh"

namespace icb
{
namespace
{
constexpr int VB = 256;
inline int vblocks(long long n)
{
  return int(std::max<long long>(1, std::min<long long>((n + VB - 1) / VB, num_sms() * 8LL)));
}

/// element e's grid coordinates (the cone filter's grids hold fewer than
/// 2^31 elements: 32-bit division)
__device__ __forceinline__ void elemIJK(const Dims &d, long long e, int &i, int &j, int &k)
{
  const unsigned ue = unsigned(e), t = ue / unsigned(d.nx);
  i = int(ue - t * unsigned(d.nx));
  j = int(t % unsigned(d.ny));
  k = int(t / unsigned(d.ny));
}

/// f(w_t, f_t) for the stencil's neighbours of element (i, j, k) = e that lie
/// in the grid, in the stencil's order; nb[t] = (di, dj, dk, linear offset)
template <class F>
__device__ __forceinline__ void cone_each(const Dims &d, int i, int j, int k, long long e,
                                          const int4 *__restrict__ nb,
                                          const double *__restrict__ w, int nnb, F f)
{
  for(int t = 0; t < nnb; t++)
  {
    const int4 o = __ldg(nb + t);
    if(unsigned(i + o.x) >= unsigned(d.nx) || unsigned(j + o.y) >= unsigned(d.ny) ||
       unsigned(k + o.z) >= unsigned(d.nz))
      continue;
    f(__ldg(w + t), e + o.w);
  }
}

__device__ __forceinline__ double thresh(double x, double beta, double T)
{
  return 0.5 * (tanh(T * beta) + tanh(beta * (x - T))) / tanh(T * beta);
}
/// thresh with tanh(T beta) given (the same value thresh computes)
__device__ __forceinline__ double thresh_tb(double x, double beta, double T, double tb)
{
  return 0.5 * (tb + tanh(beta * (x - T))) / tb;
}
__device__ __forceinline__ double thresh_d(double x, double beta, double T)
{
  double t = tanh(beta * (x - T));
  return (0.5 * (beta * (1.0 - t * t)) / tanh(T * beta)); // pow(t, 2.0)
}

// ---------------------------------------------------------------- cone ----
__global__ void k_cone_aa(Dims d, const int4 *__restrict__ nb, const double *__restrict__ w,
                          int nnb, double *__restrict__ aa)
{
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= d.nel)
    return;
  int i, j, k;
  elemIJK(d, e, i, j, k);
  double s = 0.0;
  cone_each(d, i, j, k, e, nb, w, nnb, [&](double wt, long long) { s += wt; });
  aa[e] = s;
}

/// forward: out = sum w x / aa (+ threshold and its derivative when beta > 0)
/// adjoint: out = sum w g / aa_j
template <bool SENS>
__global__ void k_cone(Dims d, const int4 *__restrict__ nb, const double *__restrict__ w,
                       int nnb, const double *__restrict__ aa, const double *__restrict__ in,
                       double *__restrict__ out, double beta, double T,
                       double *__restrict__ xhat, double *__restrict__ dxhat)
{
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= d.nel)
    return;
  int i, j, k;
  elemIJK(d, e, i, j, k);
  double s = 0.0;
  cone_each(d, i, j, k, e, nb, w, nnb, [&](double wt, long long f) {
    if(SENS)
      s += wt * in[f] / aa[f];
    else
      s += wt * in[f];
  });
  double v = SENS ? s : s / aa[e];
  out[e] = v;
  if(!SENS && xhat)
  {
    xhat[e] = beta > 0.0 ? thresh(v, beta, T) : v;
    dxhat[e] = beta > 0.0 ? thresh_d(v, beta, T) : 1.0;
  }
}

__global__ void k_threshold(long long n, const double *__restrict__ x, double beta, double T,
                            double *__restrict__ xh, double *__restrict__ dxh)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i >= n)
    return;
  if(xh)
    xh[i] = thresh(x[i], beta, T);
  if(dxh)
    dxh[i] = thresh_d(x[i], beta, T);
}

// ------------------------------------------------------------------ OC ----
__device__ __forceinline__ double oc_candidate(double x, double df, double dg, double lam,
                                               double eta, double move, double xmin,
                                               double xmax)
{
  // OCSolver's pow(B, eta): for the usual eta = 0.5 the square root, which is
  // that power correctly rounded (the stencil kernel evaluates this for every
  // neighbour of every element on each bisection step)
  const double b = fmax(0.0, -df / (dg * lam));
  double v = (eta == 0.5 ? sqrt(b) : pow(b, eta)) * x;
  double lo = fmax(xmin, (1.0 - move) * x), hi = fmin(xmax, (1.0 + move) * x);
  if(v < lo)
    v = lo;
  else if(v > hi)
    v = hi;
  return v;
}

struct FinOc
{
  OcState *st;
  LoopCtl L;
  __device__ void operator()(const double *t) const
  {
    // the lambda just evaluated, before the bisection moves it
    st->lastLam = st->lam;
    // OCSolver.hpp:52-60: lambda goes up while the candidate's volume exceeds g
    if(t[0] - st->g > 0.0)
      st->l0 = st->lam;
    else
      st->l1 = st->lam;
    st->counter++;
    st->vol = t[0];
    if(!((st->l1 - st->l0) / (st->l1 + st->l0) > st->lambdaeps && st->maxiter > st->counter))
      st->done = 1;
    else
      st->lam = 0.5 * (st->l1 + st->l0);
    // inside the update graph: repeat while not done (at most maxiter + 1
    // passes, counted in pad)
    if(L.on)
    {
      if(++st->pad > st->maxiter)
        st->done = 1;
      cudaGraphSetConditional(L.h, st->done ? 0u : 1u);
    }
  }
};

/// the first half of a filtered bisection step: every element's candidate
/// x+(lambda) at st->lam, once, into xc (the stencil then sums stored
/// values instead of re-evaluating the candidate, with its division and
/// square root, for every neighbour); block B of its grid
__device__ __forceinline__ void oc_cand_b(long long nel, const double *__restrict__ x,
                                          const double *__restrict__ df,
                                          const double *__restrict__ dg,
                                          const double *__restrict__ xmin,
                                          const double *__restrict__ xmax, const OcParams &P,
                                          const OcState *st, double *__restrict__ xc,
                                          const Blk &B)
{
  if(st->done)
    return;
  const double lam = st->lam;
  for(long long e = B.x * (long long)blockDim.x + threadIdx.x; e < nel;
      e += (long long)B.gx * blockDim.x)
    xc[e] = oc_candidate(x[e], df[e], dg[e], lam, P.eta, P.move, xmin[e], xmax[e]);
}
/// the candidates of elements [base, base + VB * kCandPerThread) (the
/// batched launch's work item: no reduction, so any cut of the elements
/// gives the same values); each thread's loads in groups of four
constexpr int kCandPerThread = 8;
__device__ __forceinline__ void oc_cand_chunk(long long nel, const double *__restrict__ x,
                                              const double *__restrict__ df,
                                              const double *__restrict__ dg,
                                              const double *__restrict__ xmin,
                                              const double *__restrict__ xmax, const OcParams &P,
                                              const OcState *st, double *__restrict__ xc,
                                              long long base)
{
  if(st->done)
    return;
  const double lam = st->lam;
  constexpr int G = 4;
  for(int k0 = 0; k0 < kCandPerThread; k0 += G)
  {
    double xv[G], fv[G], gv[G], lo[G], hi[G];
#pragma unroll
    for(int g = 0; g < G; g++)
    {
      const long long e = base + threadIdx.x + (long long)(k0 + g) * VB;
      const bool in = e < nel;
      xv[g] = in ? x[e] : 0.0;
      fv[g] = in ? df[e] : 0.0;
      gv[g] = in ? dg[e] : 1.0;
      lo[g] = in ? xmin[e] : 0.0;
      hi[g] = in ? xmax[e] : 0.0;
    }
#pragma unroll
    for(int g = 0; g < G; g++)
    {
      const long long e = base + threadIdx.x + (long long)(k0 + g) * VB;
      if(e < nel)
        xc[e] = oc_candidate(xv[g], fv[g], gv[g], lam, P.eta, P.move, lo[g], hi[g]);
    }
  }
}
__global__ void k_oc_cand(long long nel, const double *__restrict__ x,
                          const double *__restrict__ df, const double *__restrict__ dg,
                          const double *__restrict__ xmin, const double *__restrict__ xmax,
                          OcParams P, const OcState *st, double *__restrict__ xc)
{
  oc_cand_b(nel, x, df, dg, xmin, xmax, P, st, xc, this_block());
}

/// one bisection step: volume of threshold(filter(x+(lambda))) at st->lam,
/// block B of its grid (the body of k_oc_step and of the batched step).
/// With the filter the candidates come from xc (oc_cand_b of this step);
/// the sum over the stencil takes the same values in the same order as
/// evaluating each neighbour's candidate in place.
__device__ __forceinline__ void oc_step_b(const Dims &d, const int4 *__restrict__ nb,
                                          const double *__restrict__ w, int nnb,
                                          const double *__restrict__ aa,
                                          const double *__restrict__ x,
                                          const double *__restrict__ df,
                                          const double *__restrict__ dg,
                                          const double *__restrict__ xmin,
                                          const double *__restrict__ xmax,
                                          const double *__restrict__ vol,
                                          const double *__restrict__ xc, const OcParams &P,
                                          const RedScratch &red, OcState *st, const LoopCtl &L,
                                          const Blk &B)
{
  if(st->done)
  {
    if(B.x == 0 && threadIdx.x == 0)
      loop_stop(L);
    return;
  }
  const double lam = st->lam, tb = st->tanhTb;
  double v[1] = {0.0};
  for(long long e = B.x * (long long)blockDim.x + threadIdx.x; e < d.nel;
      e += (long long)B.gx * blockDim.x)
  {
    double xf;
    if(P.useFilter)
    {
      int i, j, k;
      elemIJK(d, e, i, j, k);
      double s = 0.0;
      cone_each(d, i, j, k, e, nb, w, nnb, [&](double wt, long long f) { s += wt * xc[f]; });
      xf = s / aa[e];
    }
    else
      xf = oc_candidate(x[e], df[e], dg[e], lam, P.eta, P.move, xmin[e], xmax[e]);
    double xh = P.beta > 0.0 ? thresh_tb(xf, P.beta, P.T, tb) : xf;
    v[0] += xh * vol[e];
  }
  block_reduce_at<1>(v, red, FinOc{st, L}, int(B.x), int(B.gx));
}
__global__ void k_oc_step(Dims d, const int4 *__restrict__ nb, const double *__restrict__ w,
                          int nnb, const double *__restrict__ aa, const double *__restrict__ x,
                          const double *__restrict__ df, const double *__restrict__ dg,
                          const double *__restrict__ xmin, const double *__restrict__ xmax,
                          const double *__restrict__ vol, const double *__restrict__ xc,
                          OcParams P, RedScratch red, OcState *st, LoopCtl L)
{
  oc_step_b(d, nb, w, nnb, aa, x, df, dg, xmin, xmax, vol, xc, P, red, st, L, this_block());
}

/// The filtered bisection step on a 2D grid, one kOcTW x kOcTH tile of
/// elements per block (256 threads, four rows each): the tile's candidates
/// with a halo of (hx, hy) elements are staged in shared memory (zero outside
/// the grid, which adds exactly nothing) with the stencil as shared-memory
/// offsets, so each neighbour costs a shared load and an FMA instead of
/// bounds checks and a dependent global load.  Each element sums its
/// neighbours in the stencil's order, as oc_step_b does; the tile of block
/// B.x is (B.x mod ntx, B.x div ntx).
constexpr int kOcTW = 32, kOcTH = 32, kOcHalo = 8;
__host__ __device__ constexpr int oc_tile_smem(int hx, int hy, int nnb)
{
  return 8 * ((kOcTW + 2 * hx) * (kOcTH + 2 * hy) + nnb) + 4 * nnb;
}
__device__ __forceinline__ void oc_step_tile_b(const Dims &d, int hx, int hy, unsigned ntx,
                                               const int4 *__restrict__ nb,
                                               const double *__restrict__ w, int nnb,
                                               const double *__restrict__ aa,
                                               const double *__restrict__ vol,
                                               const double *__restrict__ xc, const OcParams &P,
                                               const RedScratch &red, OcState *st,
                                               const LoopCtl &L, const Blk &B,
                                               unsigned char *smem)
{
  if(st->done)
  {
    if(B.x == 0 && threadIdx.x == 0)
      loop_stop(L);
    return;
  }
  const double tb = st->tanhTb;
  const int TWP = kOcTW + 2 * hx, THP = kOcTH + 2 * hy;
  double *tile = reinterpret_cast<double *>(smem);
  double *sw = tile + TWP * THP;
  int *so = reinterpret_cast<int *>(sw + nnb);
  const int x0 = int(B.x % ntx) * kOcTW, y0 = int(B.x / ntx) * kOcTH;
  // every load of the tile in flight before the first shared store
  constexpr int kPer = ((kOcTW + 2 * kOcHalo) * (kOcTH + 2 * kOcHalo) + VB - 1) / VB;
  double tv[kPer];
#pragma unroll
  for(int k = 0; k < kPer; k++)
  {
    const int q = threadIdx.x + k * VB;
    const int ty = q / TWP, tx = q - ty * TWP;
    const int i = x0 - hx + tx, j = y0 - hy + ty;
    tv[k] = q < TWP * THP && unsigned(i) < unsigned(d.nx) && unsigned(j) < unsigned(d.ny)
                ? __ldg(xc + i + (long long)j * d.nx)
                : 0.0;
  }
  // the stencil table (at most (2 kOcHalo + 1)^2 entries, two per thread) and
  // this thread's four elements' weight sums and volumes, in the same round
  constexpr int kTab = ((2 * kOcHalo + 1) * (2 * kOcHalo + 1) + VB - 1) / VB;
  int4 tn[kTab];
  double twv[kTab];
#pragma unroll
  for(int k = 0; k < kTab; k++)
  {
    const int t = threadIdx.x + k * VB;
    tn[k] = t < nnb ? __ldg(nb + t) : make_int4(0, 0, 0, 0);
    twv[k] = t < nnb ? __ldg(w + t) : 0.0;
  }
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  constexpr int kRows = kOcTH / 8;
  double aav[kRows], volv[kRows];
#pragma unroll
  for(int k = 0; k < kRows; k++)
  {
    const int i = x0 + tx, j = y0 + ty + 8 * k;
    const bool in = i < d.nx && j < d.ny;
    const long long e = i + (long long)j * d.nx;
    aav[k] = in ? aa[e] : 1.0;
    volv[k] = in ? vol[e] : 0.0;
  }
#pragma unroll
  for(int k = 0; k < kPer; k++)
  {
    const int q = threadIdx.x + k * VB;
    if(q < TWP * THP)
      tile[q] = tv[k];
  }
#pragma unroll
  for(int k = 0; k < kTab; k++)
  {
    const int t = threadIdx.x + k * VB;
    if(t < nnb)
    {
      so[t] = tn[k].y * TWP + tn[k].x;
      sw[t] = twv[k];
    }
  }
  __syncthreads();
  const double *c0 = tile + (ty + hy) * TWP + tx + hx;
  const int rs = 8 * TWP;
  double acc[kRows];
#pragma unroll
  for(int k = 0; k < kRows; k++)
    acc[k] = 0.0;
  for(int t = 0; t < nnb; t++)
  {
    const double wt = sw[t];
    const double *c = c0 + so[t];
#pragma unroll
    for(int k = 0; k < kRows; k++)
      acc[k] += wt * c[k * rs];
  }
  double v[1] = {0.0};
#pragma unroll
  for(int k = 0; k < kRows; k++)
  {
    const int i = x0 + tx, j = y0 + ty + 8 * k;
    if(i < d.nx && j < d.ny)
    {
      const double xf = acc[k] / aav[k];
      const double xh = P.beta > 0.0 ? thresh_tb(xf, P.beta, P.T, tb) : xf;
      v[0] += xh * volv[k];
    }
  }
  block_reduce_at<1>(v, red, FinOc{st, L}, int(B.x), int(B.gx));
}
__global__ void __launch_bounds__(VB)
    k_oc_step_tile(Dims d, int hx, int hy, unsigned ntx, const int4 *__restrict__ nb,
                   const double *__restrict__ w, int nnb, const double *__restrict__ aa,
                   const double *__restrict__ vol, const double *__restrict__ xc, OcParams P,
                   RedScratch red, OcState *st, LoopCtl L)
{
  extern __shared__ __align__(16) unsigned char oc_tile_dyn[];
  oc_step_tile_b(d, hx, hy, ntx, nb, w, nnb, aa, vol, xc, P, red, st, L, this_block(),
                 oc_tile_dyn);
}

__device__ __forceinline__ void oc_init_b(OcState *st, double g, const OcParams &P)
{
  // the threshold's constant tanh(T beta), once per update
  st->tanhTb = P.beta > 0.0 ? tanh(P.T * P.beta) : 0.0;
  st->l0 = 0.0;
  st->l1 = 1.0e4;
  st->lambdaeps = 1.0e-5;
  st->maxiter = 100;
  st->counter = 0;
  st->pad = 0;
  st->g = g;
  st->done = 0;
  st->vol = 0.0;
  // the first lambda of the bisection (OCSolver.hpp:33)
  st->lam = 0.5 * (st->l1 + st->l0);
  if(!((st->l1 - st->l0) / (st->l1 + st->l0) > st->lambdaeps && st->maxiter > st->counter))
    st->done = 1;
}
__global__ void k_oc_init(OcState *st, double g, OcParams P) { oc_init_b(st, g, P); }

/// x = x+(lambda of the last bisection step): OCSolver.hpp keeps the last
/// evaluated candidate, not the midpoint of the final bracket
__global__ void k_oc_final(long long n, double *__restrict__ x, const double *__restrict__ df,
                           const double *__restrict__ dg, const double *__restrict__ xmin,
                           const double *__restrict__ xmax, OcParams P, const OcState *st)
{
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= n)
    return;
  // the last evaluated lambda is the one whose result set l0 or l1 last
  double lam = st->lastLam;
  x[e] = oc_candidate(x[e], df[e], dg[e], lam, P.eta, P.move, xmin[e], xmax[e]);
}

// ----------------------------------------------------------------- MMA ----
/// GenSub (MMASolver.cpp:400-512) for m = 1: asymptotes, move bounds, p0,
/// q0, p, q; the constraint constant b = -g + sum(p/(U-x) + q/(x-L)) is
/// reduced into st->b by the finisher.
struct FinGenSub
{
  MmaState *st;
  __device__ void operator()(const double *t) const { st->b = -st->g + t[0]; }
};

__global__ void k_mma_gensub(long long n, MmaVec V, const double *__restrict__ x,
                             const double *__restrict__ dfdx, const double *__restrict__ dgdx,
                             const double *__restrict__ xmin, const double *__restrict__ xmax,
                             MmaParams P, int iter, RedScratch red, MmaState *st)
{
  double v[1] = {0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    double xv = x[i], range = xmax[i] - xmin[i];
    double lo, up;
    if(iter < 3)
    {
      lo = xv - P.asyminit * range;
      up = xv + P.asyminit * range;
    }
    else
    {
      double o1 = V.xold1[i], o2 = V.xold2[i];
      double zzz = (xv - o1) * (o1 - o2);
      double gam = zzz < 0.0 ? P.asymdec : (zzz > 0.0 ? P.asyminc : 1.0);
      lo = xv - gam * (o1 - V.low[i]);
      up = xv + gam * (V.upp[i] - o1);
      double xmami = fmax(P.xmamieps, range);
      lo = fmax(lo, xv - 100.0 * xmami);
      lo = fmin(lo, xv - 1.0e-5 * xmami);
      up = fmax(up, xv + 1.0e-5 * xmami);
      up = fmin(up, xv + 100.0 * xmami);
      double xmi = xmin[i] - 1.0e-6, xma = xmax[i] + 1.0e-6;
      if(xv < xmi)
      {
        lo = xv - (xma - xv) / 0.9;
        up = xv + (xma - xv) / 0.9;
      }
      if(xv > xma)
      {
        lo = xv - (xv - xmi) / 0.9;
        up = xv + (xv - xmi) / 0.9;
      }
    }
    V.low[i] = lo;
    V.upp[i] = up;
    double al = fmax(xmin[i], lo + P.albefa * (xv - lo));
    al = fmax(al, xv - P.move * range);
    al = fmin(al, xmax[i]);
    double be = fmin(xmax[i], up - P.albefa * (up - xv));
    be = fmin(be, xv + P.move * range);
    be = fmax(be, xmin[i]);
    V.alpha[i] = al;
    V.beta[i] = be;
    double inv = 1.0 / fmax(P.xmamieps, range);
    double u2 = (up - xv) * (up - xv), l2 = (xv - lo) * (xv - lo); // pow(d, 2.0)
    double df = dfdx[i], dg = dgdx[i];
    double pq = 0.001 * fabs(df) + P.raa0 * inv;
    V.p0[i] = u2 * (fmax(0.0, df) + pq);
    V.q0[i] = l2 * (fmax(0.0, -df) + pq);
    double pqg = 0.001 * fabs(dg) + P.raa0 * inv;
    double pij = u2 * (fmax(0.0, dg) + pqg), qij = l2 * (fmax(0.0, -dg) + pqg);
    V.pij[i] = pij;
    V.qij[i] = qij;
    v[0] += pij / (up - xv) + qij / (xv - lo);
    // xold2 = xold1; xold1 = x (Update, MMASolver.cpp:74-75)
    V.xold2[i] = V.xold1[i];
    V.xold1[i] = xv;
  }
  block_reduce<1>(v, red, FinGenSub{st});
}

/// SolveDIP's scalar logic for m = 1, run by the last block of each pass
/// with the sums S_g = sum(p/(U-x)+q/(x-L)) and S_h = sum(PQ^2 df2) taken at
/// the current lambda.
struct FinDip
{
  MmaState *st;
  MmaParams P;
  __device__ void newton(double Sg, double Sh) const
  {
    // XYZofLAMBDA clamps lambda (MMASolver.cpp:365-368); y = max(0, lam - c)
    double lam = fmax(st->lam, 0.0), mu = st->mu, epsi = st->epsi;
    double y = fmax(0.0, lam - P.c);
    st->loop++;
    double grad = -st->b - P.a * st->z - y + Sg;
    grad = -1.0 * grad - epsi / lam;
    // DualHess (MMASolver.cpp:238-344)
    double hess = Sh;
    if(lam > P.c)
      hess += -1.0;
    hess += -mu / lam;
    double corr = 1e-4 * hess;
    if(-1.0 * corr < 1.0e-7)
      corr = -1.0e-7;
    hess += corr;
    double s0 = grad / hess;
    double s1 = -mu + epsi / lam - s0 * mu / lam;
    // DualLineSearch (MMASolver.cpp:214-236)
    double theta = 1.005;
    if(theta < -1.01 * s0 / lam)
      theta = -1.01 * s0 / lam;
    if(theta < -1.01 * s1 / mu)
      theta = -1.01 * s1 / mu;
    theta = 1.0 / theta;
    st->lam = lam + theta * s0;
    st->mu = mu + theta * s1;
  }
  __device__ void operator()(const double *t) const
  {
    const double Sg = t[0], Sh = t[1];
    st->passes++;
    if(st->phase == 0)
    {
      // first pass of an update: outer loop 1, inner loop 1 at lambda = c/2
      st->outloop = 1;
      st->loop = 0;
      newton(Sg, Sh);
      st->phase = 1;
      return;
    }
    // phase 1: sums at the lambda after a Newton step: KKT residual
    double lam = fmax(st->lam, 0.0);
    st->lam = lam;
    double y = fmax(0.0, lam - P.c);
    double r0 = -st->b - P.a * st->z - y + st->mu + Sg;
    double r1 = st->mu * lam - st->epsi;
    st->err = fmax(fabs(r0), fabs(r1));
    // inner loop continues with the sums already at this lambda
    if(st->err > 0.9 * st->epsi && st->loop < 100)
    {
      newton(Sg, Sh);
      return;
    }
    // inner loop over: next outer loops until one runs an inner iteration
    for(;;)
    {
      st->epsi *= 0.1;
      if(!(st->epsi > P.epsimin && st->outloop < 100))
      {
        st->done = 1;
        return;
      }
      st->outloop++;
      st->loop = 0;
      if(st->err > 0.9 * st->epsi)
      {
        newton(Sg, Sh);
        return;
      }
    }
  }
};

/// one pass at the current lambda: x(lambda) (XYZofLAMBDA), S_g (DualGrad)
/// and S_h (DualHess) with ICARAT's expressions
__global__ void k_mma_pass(long long n, MmaVec V, double *__restrict__ x, MmaParams P,
                           RedScratch red, MmaState *st)
{
  if(st->done)
    return;
  const double lam = fmax(st->lam, 0.0);
  double v[2] = {0.0, 0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    double low = V.low[i], upp = V.upp[i];
    double pl = V.p0[i] + V.pij[i] * lam, ql = V.q0[i] + V.qij[i] * lam;
    double sp = sqrt(pl), sq = sqrt(ql);
    double xp = (sp * low + sq * upp) / (sp + sq);
    double xi = xp;
    if(xi < V.alpha[i])
      xi = V.alpha[i];
    if(xi > V.beta[i])
      xi = V.beta[i];
    x[i] = xi;
    // MMASolver's pow(d, 2.0) and pow(d, 3.0) as products (the square is the
    // correctly rounded pow; the cube is within an ulp of it)
    const double du = upp - xi, dl = xi - low, du2 = du * du, dl2 = dl * dl;
    v[0] += V.pij[i] / du + V.qij[i] / dl;
    double PQ = V.pij[i] / du2 - V.qij[i] / dl2;
    double df2 = -1.0 / (2.0 * pl / (du2 * du) + 2.0 * ql / (dl2 * dl));
    if(xp < V.alpha[i] || xp > V.beta[i])
      df2 = 0.0;
    v[1] += PQ * df2 * PQ;
  }
  block_reduce<2>(v, red, FinDip{st, P});
}

__global__ void k_mma_dip_init(MmaState *st, MmaParams P)
{
  st->lam = P.c / 2.0;
  st->mu = 1.0;
  st->epsi = 1.0;
  st->err = 1.0;
  st->outloop = 0;
  st->loop = 0;
  st->phase = 0;
  st->done = !(st->epsi > P.epsimin);
  st->passes = 0;
  st->z = 0.0; // z = max(0, 10 (lam a - 1)) with a = 0
}
/// GenSub of GCMMA (GCMMASolver.cpp:432-508 with asymp, 546-596): the
/// asymptotes only in an outer update (then xold shifts), bounds without the
/// final clamps, p/q with raa0 for the objective and raa for the constraint;
/// the finisher stores r0 = f0x - S0, r = g - S1 and b = -r.
struct FinGcSub
{
  MmaState *st;
  __device__ void operator()(const double *t) const
  {
    st->r0 = st->f0x - t[0];
    st->rr = st->g - t[1];
    st->b = -st->rr;
  }
};

__global__ void k_gc_gensub(long long n, MmaVec V, const double *__restrict__ x,
                            const double *__restrict__ df0dx, const double *__restrict__ dfdx,
                            const double *__restrict__ xmin, const double *__restrict__ xmax,
                            MmaParams P, double raa0, double raa, int outerIter, int asymp,
                            RedScratch red, MmaState *st)
{
  double v[2] = {0.0, 0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    const double xv = x[i], range = xmax[i] - xmin[i];
    double lo = V.low[i], up = V.upp[i];
    if(asymp)
    {
      if(outerIter < 3)
      {
        lo = xv - P.asyminit * range;
        up = xv + P.asyminit * range;
      }
      else
      {
        const double o1 = V.xold1[i], o2 = V.xold2[i];
        const double zzz = (xv - o1) * (o1 - o2);
        const double gam = zzz < 0.0 ? P.asymdec : (zzz > 0.0 ? P.asyminc : 1.0);
        lo = xv - gam * (o1 - lo);
        up = xv + gam * (up - o1);
        const double xmami = fmax(P.xmamieps, range);
        lo = fmax(lo, xv - 100.0 * xmami);
        lo = fmin(lo, xv - 1.0e-5 * xmami);
        up = fmax(up, xv + 1.0e-5 * xmami);
        up = fmin(up, xv + 100.0 * xmami);
        const double xmi = xmin[i] - 1.0e-6, xma = xmax[i] + 1.0e-6;
        if(xv < xmi)
        {
          lo = xv - (xma - xv) / 0.9;
          up = xv + (xma - xv) / 0.9;
        }
        if(xv > xma)
        {
          lo = xv - (xv - xmi) / 0.9;
          up = xv + (xv - xmi) / 0.9;
        }
      }
      V.low[i] = lo;
      V.upp[i] = up;
    }
    V.alpha[i] = fmax(fmax(xmin[i], lo + P.albefa * (xv - lo)), xv - P.move * range);
    V.beta[i] = fmin(fmin(xmax[i], up - P.albefa * (up - xv)), xv + P.move * range);
    const double uxinv = 1.0 / (up - xv), xlinv = 1.0 / (xv - lo);
    const double inv = 1.0 / fmax(P.xmamieps, range);
    const double u2 = (up - xv) * (up - xv), l2 = (xv - lo) * (xv - lo); // pow(d, 2.0)
    const double df = df0dx[i], dg = dfdx[i];
    const double pq = 0.001 * fabs(df) + raa0 * inv;
    const double p0 = u2 * (fmax(0.0, df) + pq), q0 = l2 * (fmax(0.0, -df) + pq);
    V.p0[i] = p0;
    V.q0[i] = q0;
    const double pqg = 0.001 * fabs(dg) + raa * inv;
    const double pij = u2 * (fmax(0.0, dg) + pqg), qij = l2 * (fmax(0.0, -dg) + pqg);
    V.pij[i] = pij;
    V.qij[i] = qij;
    v[0] += p0 * uxinv + q0 * xlinv;
    v[1] += pij * uxinv + qij * xlinv;
    if(asymp)
    {
      V.xold2[i] = V.xold1[i];
      V.xold1[i] = xv;
    }
  }
  block_reduce<2>(v, red, FinGcSub{st});
}

/// ComputeApprox (GCMMASolver.cpp:598-621)
struct FinGcApprox
{
  MmaState *st;
  __device__ void operator()(const double *t) const
  {
    st->f0app = t[0] + st->r0;
    st->fapp = t[1] + st->rr;
  }
};
__global__ void k_gc_approx(long long n, MmaVec V, const double *__restrict__ xm, RedScratch red,
                            MmaState *st)
{
  double v[2] = {0.0, 0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    const double uxinv = 1.0 / (V.upp[i] - xm[i]), xlinv = 1.0 / (xm[i] - V.low[i]);
    v[0] += V.p0[i] * uxinv + V.q0[i] * xlinv;
    v[1] += V.pij[i] * uxinv + V.qij[i] * xlinv;
  }
  block_reduce<2>(v, red, FinGcApprox{st});
}

/// the raacof sum of RaaUpdate (GCMMASolver.cpp:513-523)
struct FinRaacof
{
  MmaState *st;
  __device__ void operator()(const double *t) const { st->raacof = t[0]; }
};
__global__ void k_gc_raacof(long long n, MmaVec V, const double *__restrict__ xm,
                            const double *__restrict__ xv, const double *__restrict__ xmin,
                            const double *__restrict__ xmax, MmaParams P, RedScratch red,
                            MmaState *st)
{
  double v[1] = {0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    const double xmami = fmax(P.xmamieps, xmax[i] - xmin[i]);
    const double xxux = (xm[i] - xv[i]) / (V.upp[i] - xm[i]);
    const double xxxl = (xm[i] - xv[i]) / (xm[i] - V.low[i]);
    v[0] += xxux * xxxl * ((V.upp[i] - V.low[i]) / xmami);
  }
  block_reduce<1>(v, red, FinRaacof{st});
}

} // namespace

// =============================================================== Cone =====
ConeFilter::ConeFilter(const Dims &dims, const double *h, double radius, cudaStream_t s)
    : d(dims), r(radius)
{
  if(!(radius > 0.0))
    throw Error{ICB_ERR_BAD_ARG, "filter radius must be > 0"};
  int R[3];
  for(int a = 0; a < 3; a++)
    R[a] = int(std::floor(radius / h[a])) + 1;
  if(d.dim == 2)
    R[2] = 0;
  std::vector<int> off;
  std::vector<double> w;
  for(int dk = -R[2]; dk <= R[2]; dk++)
    for(int dj = -R[1]; dj <= R[1]; dj++)
      for(int di = -R[0]; di <= R[0]; di++)
      {
        double dx = di * h[0], dy = dj * h[1], dz = dk * h[2];
        double dist = std::sqrt(dx * dx + dy * dy + (d.dim == 3 ? dz * dz : 0.0));
        if(dist <= radius)
        {
          off.push_back(di);
          off.push_back(dj);
          off.push_back(dk);
          w.push_back(radius - dist);
        }
      }
  nnb = int(w.size());
  // (di, dj, dk, linear offset) per neighbour; the kernels index elements in
  // 32 bits
  ICB_REQUIRE(d.nel < (1LL << 31), "grid too large for the cone filter");
  std::vector<int4> nb4(nnb);
  for(int t = 0; t < nnb; t++)
  {
    const long long lo = off[3 * t] + (long long)off[3 * t + 1] * d.nx +
                         (long long)off[3 * t + 2] * d.nx * d.ny;
    ICB_REQUIRE(lo > -(1LL << 31) && lo < (1LL << 31), "filter stencil too large");
    nb4[t] = make_int4(off[3 * t], off[3 * t + 1], off[3 * t + 2], int(lo));
    hx = std::max(hx, std::abs(off[3 * t]));
    hy = std::max(hy, std::abs(off[3 * t + 1]));
  }
  offs.alloc(std::max(nnb, 1));
  wts.alloc(w.size());
  ICB_CUDA(cudaMemcpyAsync(offs.p, nb4.data(), sizeof(int4) * nnb, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(wts.p, w.data(), sizeof(double) * w.size(), cudaMemcpyHostToDevice, s));
  aa.alloc(d.nel);
  k_cone_aa<<<unsigned((d.nel + 255) / 256), 256, 0, s>>>(d, offs.p, wts.p, nnb, aa.p);
  ICB_CUDA(cudaGetLastError());
  count_launch();
  ICB_CUDA(cudaStreamSynchronize(s)); // off / w are host temporaries
}

void ConeFilter::forward(const double *in, double *out, double beta, double T, double *xhat,
                         double *dxhat, cudaStream_t s) const
{
  k_cone<false><<<unsigned((d.nel + 255) / 256), 256, 0, s>>>(d, offs.p, wts.p, nnb, aa.p, in, out,
                                                             beta, T, xhat, dxhat);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

void ConeFilter::adjoint(const double *in, double *out, cudaStream_t s) const
{
  k_cone<true><<<unsigned((d.nel + 255) / 256), 256, 0, s>>>(d, offs.p, wts.p, nnb, aa.p, in, out,
                                                            0.0, 0.5, nullptr, nullptr);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

void launch_threshold(long long n, const double *x, double beta, double T, double *xh,
                      double *dxh, cudaStream_t s)
{
  k_threshold<<<unsigned((n + 255) / 256), 256, 0, s>>>(n, x, beta, T, xh, dxh);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

// ================================================================= OC =====
namespace
{
/// the form of a problem's bisection step: 2D grids with a cone filter whose
/// halo fits kOcHalo take the tiled kernel (one block per tile), the rest the
/// element-strided one (vblocks)
struct OcTiling
{
  bool tiled = false;
  int hx = 0, hy = 0, smem = 0, blocks = 0;
  unsigned ntx = 0;
};
OcTiling oc_tiling(const Dims &d, const ConeFilter *cone)
{
  OcTiling t;
  if(!cone || d.dim != 2 || cone->hx > kOcHalo || cone->hy > kOcHalo)
    return t;
  t.tiled = true;
  t.hx = cone->hx;
  t.hy = cone->hy;
  t.smem = oc_tile_smem(t.hx, t.hy, cone->nnb);
  t.ntx = unsigned((d.nx + kOcTW - 1) / kOcTW);
  t.blocks = int(t.ntx) * ((d.ny + kOcTH - 1) / kOcTH);
  return t;
}
} // namespace

OcUpdater::OcUpdater(const Dims &dims, cudaStream_t s) : d(dims)
{
  st.alloc(1);
  // enough partials for either form of the step: the element-strided grid
  // and the 2D tiles
  const long long tiles =
      d.dim == 2 ? ((d.nx + kOcTW - 1) / kOcTW) * (long long)((d.ny + kOcTH - 1) / kOcTH) : 0;
  ICB_REQUIRE(tiles < (1LL << 31), "grid too large for the OC update");
  const int nb = std::max(vblocks(d.nel), int(tiles));
  partials.alloc(nb);
  counter.alloc(1);
  ICB_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), s));
  red = RedScratch{partials.p, counter.p, nb};
  cand.alloc(std::max<long long>(d.nel, 1));
  ICB_CUDA(cudaMallocHost(&hst, sizeof(OcState)));
}
OcUpdater::~OcUpdater()
{
  if(hst)
    cudaFreeHost(hst);
}

int OcUpdater::update(const ConeFilter *cone, double *x, const double *df, const double *dg,
                      double g, const double *xmin, const double *xmax, const double *vol,
                      const OcParams &P, cudaStream_t s)
{
  launch(cone, x, df, dg, g, xmin, xmax, vol, P, s);
  ICB_CUDA(cudaStreamSynchronize(s));
  return finish();
}

int OcUpdater::finish()
{
  count_launch(1 + (loop.device ? (long long)hst->pad : 1) * loop.graphNodes);
  return hst->counter;
}

void OcUpdater::launch(const ConeFilter *cone, double *x, const double *df, const double *dg,
                       double g, const double *xmin, const double *xmax, const double *vol,
                       const OcParams &P, cudaStream_t s)
{
  const int nb = vblocks(d.nel);
  k_oc_init<<<1, 1, 0, s>>>(st.p, g, P);
  count_launch();
  const int4 *off = cone ? cone->offs.p : nullptr;
  const double *w = cone ? cone->wts.p : nullptr;
  const double *aa = cone ? cone->aa.p : nullptr;
  int nnb = cone ? cone->nnb : 0;
  OcParams Pp = P;
  Pp.useFilter = cone != nullptr;
  const OcTiling tl = oc_tiling(d, cone);
  const int sb = tl.tiled ? tl.blocks : nb;
  // graph of the bisection: one step as the body of a conditional WHILE node
  // that the device repeats until done (at most maxiter = 100 steps), rebuilt
  // when anything it bakes in changes -- the stencil's device buffers and
  // size included, never the filter object's host address (a filter rebuilt
  // for another radius can reuse it while its old buffers are freed)
  const bool dev = device_loops_enabled();
  GraphKey k;
  k.add(off).add(w).add(aa).add((long long)nnb).add(x).add(df).add(dg).add(xmin).add(xmax);
  k.add(vol).add(cand.p).add((const void *)s).addBytes(Pp).add((long long)kernel_switches());
  if(loop.exec == nullptr || loop.device != dev || k != key)
  {
    // host form: all of ICARAT's 100 steps in one launch, gated after done
    loop.build(
        [&](cudaStream_t cs, const LoopCtl &L) {
          if(Pp.useFilter)
            k_oc_cand<<<nb, VB, 0, cs>>>(d.nel, x, df, dg, xmin, xmax, Pp, st.p, cand.p);
          if(tl.tiled)
            k_oc_step_tile<<<sb, VB, tl.smem, cs>>>(d, tl.hx, tl.hy, tl.ntx, off, w, nnb, aa, vol,
                                                    cand.p, Pp, red, st.p, L);
          else
            k_oc_step<<<sb, VB, 0, cs>>>(d, off, w, nnb, aa, x, df, dg, xmin, xmax, vol, cand.p,
                                         Pp, red, st.p, L);
        },
        dev, 100);
    key = k;
  }
  loop.launch(s);
  k_oc_final<<<unsigned((d.nel + 255) / 256), 256, 0, s>>>(d.nel, x, df, dg, xmin, xmax, Pp, st.p);
  ICB_CUDA(cudaGetLastError());
  ICB_CUDA(cudaMemcpyAsync(hst, st.p, sizeof(OcState), cudaMemcpyDeviceToHost, s));
}

// ========================================================== OC batch =====
struct OcBatch::Rec
{
  Dims d;
  unsigned gx;  ///< blocks of the problem's own step launch (tiles or vblocks(nel))
  unsigned gxc; ///< work items of its candidates (VB * kCandPerThread elements each)
  int tiled, hx, hy;
  unsigned ntx;
  const int4 *off;
  const double *w;
  int nnb;
  const double *aa;
  double *x;
  const double *df, *dg, *xmin, *xmax, *vol;
  double *xc; ///< the candidates of the step (the problem's OcUpdater::cand)
  OcParams P;
  RedScratch red;
  OcState *st;
  double g;
};

namespace
{
constexpr int kOcStepsPerLaunch = 8;

__global__ void k_oc_init_batch(const OcBatch::Rec *__restrict__ R, int n)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i < n)
    oc_init_b(R[i].st, R[i].g, R[i].P);
}
__global__ void __launch_bounds__(VB, 4)
    k_oc_cand_batch(const OcBatch::Rec *__restrict__ R, const int2 *__restrict__ map, BatchQueue q)
{
  batch_queue(
      R, map, q, [](const OcBatch::Rec &r) { return int(r.gxc); },
      [](const OcBatch::Rec &r) { return r.st->done != 0 || !r.P.useFilter; },
      [](const OcBatch::Rec &r, int b, bool) {
        oc_cand_chunk(r.d.nel, r.x, r.df, r.dg, r.xmin, r.xmax, r.P, r.st, r.xc,
                      (long long)b * VB * kCandPerThread);
      });
}
__global__ void __launch_bounds__(VB, 4)
    k_oc_step_batch(const OcBatch::Rec *__restrict__ R, const int2 *__restrict__ map, BatchQueue q)
{
  extern __shared__ __align__(16) unsigned char oc_batch_dyn[];
  batch_queue(
      R, map, q, [](const OcBatch::Rec &r) { return int(r.gx); },
      [](const OcBatch::Rec &r) { return r.st->done != 0; },
      [](const OcBatch::Rec &r, int b, bool) {
        const Blk B{unsigned(b), 0, 0, r.gx, 1, 1};
        if(r.tiled)
          oc_step_tile_b(r.d, r.hx, r.hy, r.ntx, r.off, r.w, r.nnb, r.aa, r.vol, r.xc, r.P, r.red,
                         r.st, LoopCtl{}, B, oc_batch_dyn);
        else
          oc_step_b(r.d, r.off, r.w, r.nnb, r.aa, r.x, r.df, r.dg, r.xmin, r.xmax, r.vol, r.xc,
                    r.P, r.red, r.st, LoopCtl{}, B);
      });
}
__global__ void __launch_bounds__(256)
    k_oc_final_batch(const OcBatch::Rec *__restrict__ R, const int2 *__restrict__ map, BatchQueue q)
{
  batch_queue(
      R, map, q, [](const OcBatch::Rec &r) { return int((r.d.nel + 255) / 256); },
      [](const OcBatch::Rec &) { return false; },
      [](const OcBatch::Rec &r, int b, bool) {
        const long long e = b * 256LL + threadIdx.x;
        if(e < r.d.nel)
          r.x[e] = oc_candidate(r.x[e], r.df[e], r.dg[e], r.st->lastLam, r.P.eta, r.P.move,
                                r.xmin[e], r.xmax[e]);
      });
}
/// every problem's state into one array, and the count of updates not done
__global__ void k_oc_gather(const OcBatch::Rec *__restrict__ R, int n, OcState *out, int *notDone)
{
  __shared__ int c;
  if(threadIdx.x == 0)
    c = 0;
  __syncthreads();
  int mine = 0;
  for(int i = threadIdx.x; i < n; i += blockDim.x)
  {
    out[i] = *R[i].st;
    mine += R[i].st->done ? 0 : 1;
  }
  atomicAdd(&c, mine);
  __syncthreads();
  if(threadIdx.x == 0)
    *notDone = c;
}
} // namespace

OcBatch::~OcBatch()
{
  if(exec)
    cudaGraphExecDestroy(exec);
  if(hst)
    cudaFreeHost(hst);
  if(hNotDone)
    cudaFreeHost(hNotDone);
}

void OcBatch::build(const std::vector<OcBatchItem> &items, cudaStream_t s)
{
  n = int(items.size());
  recsHost.assign(sizeof(Rec) * std::max(n, 1), 0);
  Rec *R = reinterpret_cast<Rec *>(recsHost.data());
  std::vector<int2> ms, mc, mf;
  smemStep = 0;
  for(int i = 0; i < n; i++)
  {
    const OcBatchItem &it = items[i];
    Rec &r = R[i];
    r.d = it.oc->d;
    const OcTiling tl = oc_tiling(r.d, it.cone);
    r.gxc = unsigned((r.d.nel + VB * kCandPerThread - 1) / (VB * kCandPerThread));
    r.gx = tl.tiled ? unsigned(tl.blocks) : r.gxc;
    r.tiled = tl.tiled;
    r.hx = tl.hx;
    r.hy = tl.hy;
    r.ntx = tl.ntx;
    smemStep = std::max(smemStep, tl.smem);
    r.off = it.cone ? it.cone->offs.p : nullptr;
    r.w = it.cone ? it.cone->wts.p : nullptr;
    r.nnb = it.cone ? it.cone->nnb : 0;
    r.aa = it.cone ? it.cone->aa.p : nullptr;
    r.x = it.x;
    r.df = it.df;
    r.dg = it.dg;
    r.xmin = it.xmin;
    r.xmax = it.xmax;
    r.vol = it.vol;
    r.xc = it.oc->cand.p;
    r.red = it.oc->red;
    r.st = it.oc->st.p;
    for(unsigned b = 0; b < r.gx; b++)
      ms.push_back(make_int2(i, int(b)));
    for(unsigned b = 0; b < r.gxc; b++)
      mc.push_back(make_int2(i, int(b)));
    for(long long b = 0; b < (r.d.nel + 255) / 256; b++)
      mf.push_back(make_int2(i, int(b)));
  }
  recs.alloc(recsHost.size());
  mapStep.alloc(std::max<size_t>(ms.size(), 1));
  mapCand.alloc(std::max<size_t>(mc.size(), 1));
  if(!mc.empty())
    ICB_CUDA(cudaMemcpyAsync(mapCand.p, mc.data(), sizeof(int2) * mc.size(), cudaMemcpyHostToDevice, s));
  mapFinal.alloc(std::max<size_t>(mf.size(), 1));
  if(!ms.empty())
    ICB_CUDA(cudaMemcpyAsync(mapStep.p, ms.data(), sizeof(int2) * ms.size(), cudaMemcpyHostToDevice, s));
  if(!mf.empty())
    ICB_CUDA(cudaMemcpyAsync(mapFinal.p, mf.data(), sizeof(int2) * mf.size(), cudaMemcpyHostToDevice, s));
  if(!qc.p)
  {
    qc.alloc(2);
    ICB_CUDA(cudaMemsetAsync(qc.p, 0, 2 * sizeof(unsigned), s));
  }
  states.alloc(std::max(n, 1));
  notDone.alloc(1);
  if(hst)
    cudaFreeHost(hst);
  ICB_CUDA(cudaMallocHost(&hst, sizeof(OcState) * std::max(n, 1)));
  if(!hNotDone)
    ICB_CUDA(cudaMallocHost(&hNotDone, sizeof(int)));
  BatchQueue qs{qc.p, qc.p + 1, int(ms.size())}, qf{qc.p, qc.p + 1, int(mf.size())};
  BatchQueue qa{qc.p, qc.p + 1, int(mc.size())};
  itemsStep = qs.items;
  itemsFinal = qf.items;
  gridCand = queue_grid((const void *)k_oc_cand_batch, VB, 0, qa);
  chunkCand = qa.chunk;
  gridStep = queue_grid((const void *)k_oc_step_batch, VB, smemStep, qs);
  chunkStep = qs.chunk;
  gridFinal = queue_grid((const void *)k_oc_final_batch, 256, 0, qf);
  chunkFinal = qf.chunk;
  ICB_CUDA(cudaStreamSynchronize(s));
  // kOcStepsPerLaunch bisection steps of every problem and the done count
  if(exec)
    cudaGraphExecDestroy(exec);
  exec = nullptr;
  cudaStream_t cs;
  ICB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t gr = nullptr;
  ICB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  const Rec *Rd = reinterpret_cast<const Rec *>(recs.p);
  for(int k = 0; k < kOcStepsPerLaunch; k++)
  {
    k_oc_cand_batch<<<gridCand, VB, 0, cs>>>(Rd, mapCand.p, qa);
    k_oc_step_batch<<<gridStep, VB, smemStep, cs>>>(Rd, mapStep.p, qs);
  }
  k_oc_gather<<<1, 256, 0, cs>>>(Rd, n, states.p, notDone.p);
  ICB_CUDA(cudaMemcpyAsync(hNotDone, notDone.p, sizeof(int), cudaMemcpyDeviceToHost, cs));
  ICB_CUDA(cudaStreamEndCapture(cs, &gr));
  ICB_CUDA(cudaGraphInstantiate(&exec, gr, 0));
  cudaGraphDestroy(gr);
  cudaStreamDestroy(cs);
}

void OcBatch::update(const std::vector<double> &g, const std::vector<OcParams> &P, cudaStream_t s)
{
  if(n == 0)
    return;
  Rec *R = reinterpret_cast<Rec *>(recsHost.data());
  for(int i = 0; i < n; i++)
  {
    R[i].g = g[i];
    R[i].P = P[i];
    R[i].P.useFilter = R[i].off != nullptr;
  }
  ICB_CUDA(cudaMemcpyAsync(recs.p, recsHost.data(), recsHost.size(), cudaMemcpyHostToDevice, s));
  const Rec *Rd = reinterpret_cast<const Rec *>(recs.p);
  k_oc_init_batch<<<(n + 127) / 128, 128, 0, s>>>(Rd, n);
  ICB_CUDA(cudaGetLastError());
  count_launch();
  // at most ICARAT's 100 bisection steps (the updates stop themselves)
  for(int steps = 0; steps <= 100; steps += kOcStepsPerLaunch)
  {
    ICB_CUDA(cudaGraphLaunch(exec, s));
    count_launch(2 * kOcStepsPerLaunch + 1);
    ICB_CUDA(cudaStreamSynchronize(s));
    if(*hNotDone == 0)
      break;
  }
  BatchQueue qf{qc.p, qc.p + 1, itemsFinal, chunkFinal};
  k_oc_final_batch<<<gridFinal, 256, 0, s>>>(Rd, mapFinal.p, qf);
  ICB_CUDA(cudaGetLastError());
  k_oc_gather<<<1, 256, 0, s>>>(Rd, n, states.p, notDone.p);
  count_launch(2);
  ICB_CUDA(cudaMemcpyAsync(hst, states.p, sizeof(OcState) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
}

// ================================================================ MMA =====
MmaUpdater::MmaUpdater(long long nvar, cudaStream_t s) : n(nvar)
{
  for(DevBuf<double> *b : {&low, &upp, &alpha, &beta, &p0, &q0, &pij, &qij, &xold1, &xold2})
    b->alloc(n);
  st.alloc(1);
  int nb = vblocks(n);
  partials.alloc((size_t)nb * 2);
  counter.alloc(1);
  red = RedScratch{partials.p, counter.p, nb};
  ICB_CUDA(cudaMallocHost(&hst, sizeof(MmaState)));
  P.epsimin = std::sqrt(double(n + 1)) * 1e-9;
  reset(s);
}
void MmaUpdater::reset(cudaStream_t s)
{
  iter = 0;
  for(DevBuf<double> *b : {&low, &upp, &alpha, &beta, &p0, &q0, &pij, &qij, &xold1, &xold2})
    ICB_CUDA(cudaMemsetAsync(b->p, 0, b->bytes(), s));
  ICB_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), s));
}
MmaUpdater::~MmaUpdater()
{
  if(exec)
    cudaGraphExecDestroy(exec);
  if(hst)
    cudaFreeHost(hst);
}

int MmaUpdater::update(double *x, const double *dfdx, double g, const double *dgdx,
                       const double *xmin, const double *xmax, cudaStream_t s)
{
  iter++;
  MmaVec V{low.p, upp.p, alpha.p, beta.p, p0.p, q0.p, pij.p, qij.p, xold1.p, xold2.p};
  const int nb = vblocks(n);
  // the constraint value for GenSub's b
  ICB_CUDA(cudaMemcpyAsync(&st.p->g, &g, sizeof(double), cudaMemcpyHostToDevice, s));
  k_mma_gensub<<<nb, VB, 0, s>>>(n, V, x, dfdx, dgdx, xmin, xmax, P, iter, red, st.p);
  count_launch();
  return solveDual(x, s);
}

int MmaUpdater::solveDual(double *x, cudaStream_t s)
{
  MmaVec V{low.p, upp.p, alpha.p, beta.p, p0.p, q0.p, pij.p, qij.p, xold1.p, xold2.p};
  const int nb = vblocks(n);
  k_mma_dip_init<<<1, 1, 0, s>>>(st.p, P);
  count_launch();
  // the batch graph bakes in x, the stream and the parameters by value
  GraphKey k;
  k.add(x).add((const void *)s).addBytes(P);
  const int batch = 32;
  if(exec == nullptr || k != key)
  {
    if(exec)
      cudaGraphExecDestroy(exec);
    exec = nullptr;
    cudaStream_t cs;
    ICB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t gr;
    ICB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    for(int it = 0; it < batch; it++)
      k_mma_pass<<<nb, VB, 0, cs>>>(n, V, x, P, red, st.p);
    ICB_CUDA(cudaStreamEndCapture(cs, &gr));
    ICB_CUDA(cudaGraphInstantiate(&exec, gr, 0));
    cudaGraphDestroy(gr);
    cudaStreamDestroy(cs);
    key = k;
  }
  // SolveDIP needs at most 100 x 100 Newton steps; each pass is one step
  for(int launches = 0; launches < 10000 / batch + 1; launches++)
  {
    ICB_CUDA(cudaGraphLaunch(exec, s));
    count_launch(batch);
    ICB_CUDA(cudaMemcpyAsync(hst, st.p, sizeof(MmaState), cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    if(hst->done)
      break;
  }
  return hst->passes;
}

// ============================================================== GCMMA =====
GcmmaUpdater::GcmmaUpdater(long long nvar, cudaStream_t s) : core(nvar, s)
{
  core.P.c = 1000.0; // GCMMASolver(n, m, a = 0, c = 1000, d = 0)
}

void GcmmaUpdater::subproblem(const double *xval, double f0x, const double *df0dx, double fx,
                              const double *dfdx, const double *xmin, const double *xmax,
                              bool asymp, cudaStream_t s)
{
  MmaVec V{core.low.p, core.upp.p, core.alpha.p, core.beta.p, core.p0.p,
           core.q0.p,  core.pij.p, core.qij.p,   core.xold1.p, core.xold2.p};
  double gf[2] = {fx, f0x};
  ICB_CUDA(cudaMemcpyAsync(&core.st.p->g, &gf[0], sizeof(double), cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(&core.st.p->f0x, &gf[1], sizeof(double), cudaMemcpyHostToDevice, s));
  k_gc_gensub<<<vblocks(core.n), VB, 0, s>>>(core.n, V, xval, df0dx, dfdx, xmin, xmax, core.P,
                                              raa0, raa, outerIter, asymp ? 1 : 0, core.red,
                                              core.st.p);
  count_launch();
  ICB_CUDA(cudaStreamSynchronize(s)); // gf is a host temporary
}

void GcmmaUpdater::approx(const double *xmma, cudaStream_t s)
{
  MmaVec V{core.low.p, core.upp.p, core.alpha.p, core.beta.p, core.p0.p,
           core.q0.p,  core.pij.p, core.qij.p,   core.xold1.p, core.xold2.p};
  k_gc_approx<<<vblocks(core.n), VB, 0, s>>>(core.n, V, xmma, core.red, core.st.p);
  count_launch();
  ICB_CUDA(cudaMemcpyAsync(core.hst, core.st.p, sizeof(MmaState), cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  f0app = core.hst->f0app;
  fapp = core.hst->fapp;
}

void GcmmaUpdater::outer(double *xmma, const double *xval, double f0x, const double *df0dx,
                         double fx, const double *dfdx, const double *xmin, const double *xmax,
                         cudaStream_t s)
{
  // Asymp (GCMMASolver.cpp:432-508): iteration count, raa shrink
  outerIter++;
  raa0 = std::max(1e-6, 0.1 * raa0);
  raa = std::max(1e-6, 0.1 * raa);
  subproblem(xval, f0x, df0dx, fx, dfdx, xmin, xmax, true, s);
  core.solveDual(xmma, s);
  approx(xmma, s);
}

void GcmmaUpdater::inner(double *xmma, double f0xnew, double fxnew, const double *xval, double f0x,
                         const double *df0dx, double fx, const double *dfdx, const double *xmin,
                         const double *xmax, cudaStream_t s)
{
  // RaaUpdate (GCMMASolver.cpp:510-544)
  MmaVec V{core.low.p, core.upp.p, core.alpha.p, core.beta.p, core.p0.p,
           core.q0.p,  core.pij.p, core.qij.p,   core.xold1.p, core.xold2.p};
  k_gc_raacof<<<vblocks(core.n), VB, 0, s>>>(core.n, V, xmma, xval, xmin, xmax, core.P, core.red,
                                              core.st.p);
  count_launch();
  ICB_CUDA(cudaMemcpyAsync(core.hst, core.st.p, sizeof(MmaState), cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  const double raacof = std::max(1e-12, core.hst->raacof);
  const double eps = core.P.epsimin;
  if(f0xnew > f0app + 0.5 * eps)
    raa0 = std::min(1.1 * (raa0 + (f0xnew - f0app) / raacof), 10.0 * raa0);
  if(fxnew > fapp + 0.5 * eps)
    raa = std::min(1.1 * (raa + (fxnew - fapp) / raacof), 10.0 * raa);
  subproblem(xval, f0x, df0dx, fx, dfdx, xmin, xmax, false, s);
  core.solveDual(xmma, s);
  approx(xmma, s);
}

} // namespace icb
