// helm.hpp -- Helmholtz PDE filter (FilterHelmholtz) on the device.
#pragma once
#include <memory>

#include "krylov.hpp"

namespace icb
{

struct HelmFilter
{
  Dims d;
  double radius;
  int ne = 8;
  KMat<double, 8> K; ///< M + re^2 K_grad of one element (ne x ne)
  double nint = 0.0; ///< int N_a over an element (the same for every node)
  double h[3] = {1.0, 1.0, 1.0}; ///< element edge lengths
  std::unique_ptr<JacobiPcg<double>> pcg;
  DevBuf<double> dinv, rhs, phi;

  HelmFilter(const Dims &dims, const double *h, double R, cudaStream_t s);
  /// densityFilter(in, "Eigen_CG", 0, sens): element values in -> out
  int apply(const double *in, double *out, bool sens, double tol, cudaStream_t s,
            icb_solve_info *info);
};

} // namespace icb
