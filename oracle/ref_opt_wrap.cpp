// ref_opt_wrap.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points around ICARAT's own OC and MMA updates so that tests can run
// the reference code itself.  This file is compiled together with ICARAT's
// src/optimization/opt-solver/MMASolver.cpp and OCSolver.hpp, read in place
// from the ICARAT source tree by oracle/Makefile, into oracle/_ref/ (never
// committed).  Nothing of ICARAT's source is copied here.
//
// OCSolver.hpp uses std::max/pow/cerr without including their headers, so
// they are included before it.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <iostream>
#include <vector>

#include "MMASolver.hpp"
#include "OCSolver.hpp"

extern "C" {

typedef double (*ref_volume_cb)(const double *xkp1, void *ud);

/// icarat::OC::UpdateVariables (OCSolver.hpp:20-68) with the volume
/// callback supplied by the caller; movelimit as OC::setMoveLimit.
void ref_oc_update(int n, double *x, const double *dfdx, double g,
                   const double *dgdx, const double *xmin, const double *xmax,
                   double movelimit, ref_volume_cb cb, void *ud)
{
  icarat::OC oc(n);
  oc.setMoveLimit(movelimit);
  std::vector<double> xk(x, x + n), df(dfdx, dfdx + n), dg(dgdx, dgdx + n),
      lo(xmin, xmin + n), hi(xmax, xmax + n);
  oc.UpdateVariables(xk, df, g, dg, lo, hi,
                     [&](std::vector<double> &xkp1) { return cb(xkp1.data(), ud); });
  std::copy(xk.begin(), xk.end(), x);
}

/// icarat::MMASolver (MMASolver.hpp:67-78, MMASolver.cpp:41-82)
void *ref_mma_create(int n, int m)
{
  return new icarat::MMASolver(n, m);
}
void ref_mma_update(void *h, double *x, const double *dfdx, const double *gx,
                    const double *dgdx, const double *xmin, const double *xmax)
{
  static_cast<icarat::MMASolver *>(h)->Update(x, dfdx, gx, dgdx, xmin, xmax);
}
void ref_mma_free(void *h) { delete static_cast<icarat::MMASolver *>(h); }
}
