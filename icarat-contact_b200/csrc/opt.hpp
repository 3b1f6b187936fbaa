// opt.hpp -- density filter, threshold, OC and MMA on the device.
#pragma once
#include <cstring>

#include "icb_internal.hpp"

namespace icb
{

/// Filter<E,N> (src/optimization/filter.hpp:17-57) on a structured grid
struct ConeFilter
{
  Dims d;
  double r;
  int nnb = 0;           ///< neighbours in the stencil
  DevBuf<int> offs;      ///< (di,dj,dk) per neighbour, element-index order
  DevBuf<double> wts;    ///< r - distance
  DevBuf<double> aa;     ///< sum of weights per element (dfilters_ds)

  ConeFilter(const Dims &dims, const double *h, double radius, cudaStream_t s);
  /// densityFilter(x, false); with beta > 0 also the threshold projection and
  /// its derivative (threshold / thresholdDerivative with T) into xhat/dxhat
  void forward(const double *in, double *out, double beta, double T, double *xhat,
               double *dxhat, cudaStream_t s) const;
  /// densityFilter(g, true): sum_j w_ij g_j / aa_j
  void adjoint(const double *in, double *out, cudaStream_t s) const;
};

void launch_threshold(long long n, const double *x, double beta, double T, double *xh,
                      double *dxh, cudaStream_t s);

struct OcParams
{
  double eta = 0.5;   ///< iota
  double move = 0.15; ///< movelimit
  double beta = 0.0;  ///< threshold sharpness in the volume callback (0: none)
  double T = 0.5;
  int useFilter = 1;
  int pad = 0;
};
struct OcState
{
  double l0, l1, lam, lastLam, lambdaeps, g, vol;
  int counter, maxiter, done, pad;
};

/// OC::UpdateVariables with the filtered-and-thresholded volume callback
struct OcUpdater
{
  Dims d;
  DevBuf<OcState> st;
  DevBuf<double> partials;
  DevBuf<unsigned> counter;
  RedScratch red;
  OcState *hst = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *key[9] = {};
  OcParams keyP;

  OcUpdater(const Dims &dims, cudaStream_t s);
  ~OcUpdater();
  /// x <- the OC update; returns the number of bisection steps
  int update(const ConeFilter *cone, double *x, const double *df, const double *dg, double g,
             const double *xmin, const double *xmax, const double *vol, const OcParams &P,
             cudaStream_t s);
};

/// ICARAT's MMASolver parameters (MMASolver.cpp:41-55)
struct MmaParams
{
  double move = 0.15, albefa = 0.2, asyminit = 0.2, asymdec = 0.7, asyminc = 1.2;
  double raa0 = 1e-5, xmamieps = 1e-5, epsimin = 1e-9;
  double a = 0.0, c = 1e5;
};
struct MmaVec
{
  double *low, *upp, *alpha, *beta, *p0, *q0, *pij, *qij, *xold1, *xold2;
};
struct MmaState
{
  double g, b, z, lam, mu, epsi, err;
  int outloop, loop, phase, done, passes, pad;
};

/// MMASolver (MMASolver.hpp:62-117) for one constraint
struct MmaUpdater
{
  long long n;
  int iter = 0;
  MmaParams P;
  DevBuf<double> low, upp, alpha, beta, p0, q0, pij, qij, xold1, xold2;
  DevBuf<MmaState> st;
  DevBuf<double> partials;
  DevBuf<unsigned> counter;
  RedScratch red;
  MmaState *hst = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void *key[3] = {};

  MmaUpdater(long long nvar, cudaStream_t s);
  ~MmaUpdater();
  /// MMASolver::Update(x, dfdx, &g, dgdx, xmin, xmax); returns the dual passes
  int update(double *x, const double *dfdx, double g, const double *dgdx, const double *xmin,
             const double *xmax, cudaStream_t s);
};

} // namespace icb
