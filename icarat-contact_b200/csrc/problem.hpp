// problem.hpp -- device-side state of one structured SIMP problem.
#pragma once
#include <memory>

#include "krylov.hpp"
#include "setup.hpp"

struct icb_ctx_s
{
  int device = 0;
  cudaStream_t stream = nullptr;
  int refs = 0; ///< the handle plus one per live problem (not thread-safe)
};

namespace icb
{
struct Mixed;     // multigrid / mixed-precision machinery (mg.cu)
struct LoopCache; // work space of the app loops (loopcache.hpp)
}

/// One LinearAnalysis-equivalent: mesh, BCs, loads and the device arrays the
/// solve and the sensitivity need (src/analysis/linear.hpp:15-41 holds the
/// same things by reference: FEM, element, node, Force, Value).
struct icb_problem_s
{
  icb_ctx ctx = nullptr;
  std::unique_ptr<icb::HostSetup> hs;
  icb::Dims d;
  long long nsoa = 0; ///< dim * ld
  double K0[576];     ///< unit element matrix (this level)
  float K0f[576];
  // device arrays
  icb::DevBuf<uint8_t> fix;   ///< per-node Dirichlet bit mask
  icb::DevBuf<uint8_t> fixNone; ///< all-zero mask (operator over every DOF, lazy)
  icb::DevBuf<double> f;      ///< load, SoA, zero on constrained DOFs
  icb::DevBuf<double> uD;     ///< Dirichlet values, SoA (empty if all zero)
  icb::DevBuf<double> u;      ///< displacement, SoA, Dirichlet values included
  icb::DevBuf<double> x;      ///< free part of the displacement (PCG unknown)
  icb::DevBuf<double> b;      ///< right-hand side fres
  icb::DevBuf<double> work;   ///< scratch SoA vector
  icb::DevBuf<double> work2;  ///< second scratch SoA vector (lazy)
  icb::DevBuf<double> rho;    ///< physical densities
  icb::DevBuf<double> E;      ///< SIMP moduli
  icb::DevBuf<float> Ef;      ///< SIMP moduli (FP32 copy for the mixed path)
  icb::DevBuf<double> dinv;   ///< inverse diagonal (0 on constrained DOFs)
  icb::DevBuf<double> dc;     ///< sensitivities
  icb::DevBuf<long long> freeIdx; ///< SoA index of each numeq DOF
  icb::DevBuf<double> numeqBuf;   ///< numeq staging
  icb::DevBuf<double> scal;       ///< small device scalars
  icb::DevBuf<double> redPart;
  icb::DevBuf<unsigned> redCnt;
  icb::RedScratch red;
  std::unique_ptr<icb::JacobiPcg<double>> pcg;
  std::unique_ptr<icb::Mixed> mixed;
  std::unique_ptr<icb::LoopCache> loops; ///< filters, updaters, vectors of the app loops
  bool hasDirichletValues = false;
  bool hasDensity = false;
  bool solved = false;
  bool diagValid = false;
  icb_solve_info last{};

  cudaStream_t stream() const { return ctx->stream; }
  icb_problem_s();
  ~icb_problem_s(); ///< defined where icb::Mixed and icb::LoopCache are complete (mg.cu)
};
