// setup.hpp -- host-side set-up of a structured SIMP problem.
#pragma once
#include <vector>

#include "icb_internal.hpp"

namespace icb
{

void lame_constants(int state, double nu, double &lam, double &mu);
/// unit-modulus element stiffness (E = 1) of a box element with sides h,
/// (d*ne)^2 row-major, DOFs node-major with interleaved components
void unit_stiffness(int dim, int state, double nu, const double *h, double *K);
/// heat element matrix int grad N^T D grad N over the box element (the
/// Gauss sum of LinearHeat::makeKeFint, heat.cpp:67-111, done exactly), for a
/// dim x dim conductivity D; ne x ne row-major
void heat_element(int dim, const double *h, const double *D, double *K);
/// Helmholtz filter element matrix (M + re^2 K_grad, re = R/(2 sqrt 3)) and
/// the load integrals int N_a of FilterHelmholtz::makeKeFint
/// (src/optimization/filter_helm.hpp:178-222)
void helmholtz_element(int dim, const double *h, double R, double *Ke, double *Nint);

struct Traction
{
  double val[3];
  double range[6];
};

/// Everything ICARAT sets up on the host before the first solve
/// (opt_mma_Helmholtz.cpp:30-64): mesh, Dirichlet flags, countDOF, loads.
struct HostSetup
{
  icb_grid_desc desc;
  Dims dims;
  int dofnp = 0; ///< DOFs per node: dim (elasticity) or 1 (heat)
  double h[3];
  long long neq = 0, numeq = 0;
  std::vector<unsigned char> fixed; ///< neq
  std::vector<double> dval;         ///< neq
  std::vector<double> nodal;        ///< neq nodal loads
  std::vector<Traction> tractions;
  std::vector<int> dof;             ///< neq, countDOF numbering
  std::vector<double> fext;         ///< numeq, Force::fext_org
  double K0[576];
  double volume = 0.0;
  bool finalized = false;

  explicit HostSetup(const icb_grid_desc &g);
  void nodeX(long long n, double x[3]) const;
  void elemNodes(long long e, long long nd[8]) const;
  void dirichletBox(const int *flag, const double *val, const double *range);
  void dirichletMask(const unsigned char *f, const double *v);
  void tractionBox(const double *val, const double *range);
  void nodalLoad(long long node, const double *f);
  void finalize();
};

} // namespace icb
