// krylov.hpp -- preconditioned conjugate gradients on the device.
#pragma once
#include <functional>

#include "graphloop.hpp"
#include "icb_internal.hpp"

namespace icb
{

/// Jacobi-preconditioned CG with the semantics of Eigen 3.4's
/// ConjugateGradient<SparseMatrix, Lower|Upper, DiagonalPreconditioner> as
/// called by Solvers::EigenCG (src/analysis/solver/solvers.cpp:64-92):
/// x0 = 0, stop when ||r||^2 < max(tol^2 ||b||^2, DBL_MIN), the iteration
/// count excludes the converging iteration.  Every scalar stays on the device;
/// the host only polls the stop flag once per batch of iterations, and a
/// batch is one CUDA-graph launch.
template <typename T> struct JacobiPcg
{
  Dims d;
  long long n = 0; ///< vector length (dim * ld)
  DevBuf<T> r, p, q;
  DevBuf<KState> st;
  DevBuf<double> partials, dots;
  DevBuf<unsigned> counter;
  RedScratch red;
  KState *hst = nullptr; ///< pinned mirror
  WhileGraph loop; ///< host form: 16 iterations per launch
  GraphKey graphKey; ///< what `loop` bakes in besides this object's own buffers

  JacobiPcg(const Dims &dims, cudaStream_t s);
  ~JacobiPcg();
  /// solve K(E) x = b; K: host pointer to the unit element matrix of this
  /// level (captured by value into the batch graph: keep it stable).
  int solve(const T *K, const T *E, const uint8_t *fix, const T *invdiag, const T *b, T *x,
            double tol, int maxit, cudaStream_t s, icb_solve_info *info);
  /// the same iteration with any operator: `op(stream)` must compute q = A p
  /// on this object's p/q buffers and store p.q in dots[0] through `red`;
  /// opKey* identify the operator's operands for the graph cache.
  int solveOp(const std::function<void(cudaStream_t)> &op, const void *opKey0,
              const void *opKey1, const void *opKey2, const T *invdiag, const T *b, T *x,
              double tol, int maxit, cudaStream_t s, icb_solve_info *info);
};

/// Jacobi-PCG (FP64) on caller-supplied buffers, no graph, no allocation:
/// r, p, q are SoA vectors of dim*ld entries, dotOut one double, st one
/// device KState, red a reduction scratch with >= reduction_blocks(d) slots.
int pcg_run_external(const Dims &d, const double *K, const double *E, const uint8_t *fix,
                     const double *invdiag, const double *b, double *x, double *r, double *p,
                     double *q, double *dotOut, KState *st, RedScratch red, double tol,
                     int maxit, cudaStream_t s, KState *hostState);

/// partial-sum slots a reduction over this grid's vectors or operator needs
int reduction_blocks(const Dims &d);

// vector helpers (krylov.cu)
void launch_axpy_sub(long long n, const double *b, const double *Ku, double *r,
                     cudaStream_t s); ///< r = b - Ku
void launch_add(long long n, const double *a, const double *b, double *out, cudaStream_t s);
double device_dot(long long n, const double *a, const double *b, RedScratch &red,
                  double *scratch, cudaStream_t s);

} // namespace icb
