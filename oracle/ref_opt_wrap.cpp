// ref_opt_wrap.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points around ICARAT's own OC, MMA and GCMMA updates so that tests can run
// the reference code itself.  This file is compiled together with ICARAT's
// src/optimization/opt-solver/MMASolver.cpp, GCMMASolver.cpp and OCSolver.hpp, read in place
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

#include "GCMMASolver.hpp"
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

/// icarat::GCMMASolver (GCMMASolver.hpp:60-90): OuterUpdate, InnerUpdate,
/// ConCheck with the default a = 0, c = 1000, d = 0
void *ref_gcmma_create(int n, int m) { return new icarat::GCMMASolver(n, m); }
void ref_gcmma_outer(void *h, double *xmma, const double *xval, double f0x, const double *df0dx,
                     const double *fx, const double *dfdx, const double *xmin, const double *xmax)
{
  static_cast<icarat::GCMMASolver *>(h)->OuterUpdate(xmma, xval, f0x, df0dx, fx, dfdx, xmin, xmax);
}
void ref_gcmma_inner(void *h, double *xmma, double f0xnew, const double *fxnew, const double *xval,
                     double f0x, const double *df0dx, const double *fx, const double *dfdx,
                     const double *xmin, const double *xmax)
{
  static_cast<icarat::GCMMASolver *>(h)->InnerUpdate(xmma, f0xnew, fxnew, xval, f0x, df0dx, fx,
                                                      dfdx, xmin, xmax);
}
int ref_gcmma_concheck(void *h, double f0xnew, const double *fxnew)
{
  return static_cast<icarat::GCMMASolver *>(h)->ConCheck(f0xnew, fxnew) ? 1 : 0;
}
void ref_gcmma_free(void *h) { delete static_cast<icarat::GCMMASolver *>(h); }
}
