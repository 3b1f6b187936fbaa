// opt.hpp -- density filter, threshold, OC and MMA on the device.
#pragma once
#include <cstring>

#include "graphloop.hpp"
#include "icb_internal.hpp"

namespace icb
{

/// Filter<E,N> (src/optimization/filter.hpp:17-57) on a structured grid
struct ConeFilter
{
  Dims d;
  double r;
  int nnb = 0;           ///< neighbours in the stencil
  int hx = 0, hy = 0;    ///< the stencil's largest |di|, |dj|
  DevBuf<int4> offs;     ///< (di,dj,dk, linear offset) per neighbour, element-index order
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
  double tanhTb; ///< tanh(T beta) of the update's threshold
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
  DevBuf<double> cand; ///< the candidates x+(lambda) of the current step
  OcState *hst = nullptr;
  WhileGraph loop; ///< one bisection step, repeated on the device until done
  GraphKey key;     ///< what `loop` bakes in

  OcUpdater(const Dims &dims, cudaStream_t s);
  ~OcUpdater();
  /// x <- the OC update; returns the number of bisection steps
  int update(const ConeFilter *cone, double *x, const double *df, const double *dg, double g,
             const double *xmin, const double *xmax, const double *vol, const OcParams &P,
             cudaStream_t s);
  /// update() in two halves: launch queues the update on s; finish, once s
  /// has been synchronised, returns the number of bisection steps
  void launch(const ConeFilter *cone, double *x, const double *df, const double *dg, double g,
              const double *xmin, const double *xmax, const double *vol, const OcParams &P,
              cudaStream_t s);
  int finish();
};

/// one problem's OC update in a batch: the operands of OcUpdater::update
struct OcBatchItem
{
  const ConeFilter *cone;
  OcUpdater *oc;
  double *x;
  const double *df, *dg, *xmin, *xmax, *vol;
};
/// The OC updates of many problems as batched launches (opt.cu): the init,
/// every bisection step and the final candidate each launched once for all
/// problems through the work queue; each problem's blocks run exactly its own
/// update's blocks, so its design is bitwise that of OcUpdater::update.
struct OcBatch
{
  struct Rec; ///< one problem's step launch (opt.cu)
  int n = 0;
  std::vector<unsigned char> recsHost; ///< n records
  DevBuf<unsigned char> recs;
  DevBuf<int2> mapStep, mapCand, mapFinal;
  int smemStep = 0; ///< dynamic shared memory of the step launch (tiled problems)
  DevBuf<unsigned> qc;
  DevBuf<OcState> states;
  DevBuf<int> notDone;
  OcState *hst = nullptr;
  int *hNotDone = nullptr;
  int gridCand = 0, gridStep = 0, gridFinal = 0, chunkCand = 1, chunkStep = 1, chunkFinal = 1,
      itemsStep = 0, itemsFinal = 0;
  cudaGraphExec_t exec = nullptr; ///< kStepsPerLaunch steps and the done count
  OcBatch() = default;
  OcBatch(const OcBatch &) = delete;
  OcBatch &operator=(const OcBatch &) = delete;
  ~OcBatch();
  void build(const std::vector<OcBatchItem> &items, cudaStream_t s);
  /// the updates with constraint values g[i] and parameters P[i]; returns
  /// when every update is done (x updated, states in hst)
  void update(const std::vector<double> &g, const std::vector<OcParams> &P, cudaStream_t s);
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
  // GCMMA: objective at xval, constant terms, approximations at xmma, raacof
  double f0x, r0, rr, f0app, fapp, raacof;
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
  GraphKey key; ///< what `exec` bakes in

  MmaUpdater(long long nvar, cudaStream_t s);
  ~MmaUpdater();
  /// back to the state of a new solver (iteration 0, zero history)
  void reset(cudaStream_t s);
  /// MMASolver::Update(x, dfdx, &g, dgdx, xmin, xmax); returns the dual passes
  int update(double *x, const double *dfdx, double g, const double *dgdx, const double *xmin,
             const double *xmax, cudaStream_t s);
  /// SolveDIP on the subproblem set up last: x <- x(lambda*); returns the passes
  int solveDual(double *x, cudaStream_t s);
};

/// GCMMASolver (GCMMASolver.hpp:60-90, GCMMASolver.cpp:41-661) for one
/// constraint: the MMA subproblem and dual of MmaUpdater with GCMMA's
/// adaptive raa0 / raa, constant terms and approximation values
struct GcmmaUpdater
{
  MmaUpdater core;
  double raa0 = 1.0, raa = 1.0; ///< GCMMASolver.cpp:51
  int outerIter = 0;
  double f0app = 0.0, fapp = 0.0; ///< approximations at the last xmma

  GcmmaUpdater(long long nvar, cudaStream_t s);
  /// back to the state of a new solver
  void reset(cudaStream_t s)
  {
    core.reset(s);
    raa0 = raa = 1.0;
    outerIter = 0;
    f0app = fapp = 0.0;
  }
  /// OuterUpdate (GCMMASolver.cpp:66-89)
  void outer(double *xmma, const double *xval, double f0x, const double *df0dx, double fx,
             const double *dfdx, const double *xmin, const double *xmax, cudaStream_t s);
  /// InnerUpdate (GCMMASolver.cpp:91-112)
  void inner(double *xmma, double f0xnew, double fxnew, const double *xval, double f0x,
             const double *df0dx, double fx, const double *dfdx, const double *xmin,
             const double *xmax, cudaStream_t s);
  /// ConCheck (GCMMASolver.cpp:114-128)
  bool concheck(double f0xnew, double fxnew) const
  {
    return !(f0app + core.P.epsimin < f0xnew) && !(fapp + core.P.epsimin < fxnew);
  }

private:
  void subproblem(const double *xval, double f0x, const double *df0dx, double fx,
                  const double *dfdx, const double *xmin, const double *xmax, bool asymp,
                  cudaStream_t s);
  void approx(const double *xmma, cudaStream_t s);
};

} // namespace icb
