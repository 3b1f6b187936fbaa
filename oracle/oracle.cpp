// oracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A plain C++17 + OpenMP restatement, on the CPU, of ICARAT's linear-elastic
// SIMP analysis-and-sensitivity step.  It is the checker for the CUDA library
// and the timed CPU baseline; it is never linked into the product library and
// the product never calls it.  Only tests/, __graft_entry__.smoke() and the
// cpu_baseline / --impl reference legs of bench.py load it.
//
// Parity status: the FEM solve is unpinned by reference-run outputs (ICARAT's
// solve needs Eigen 3.4 + toml11, absent here, and ICARAT ships no test
// vectors).  It is pinned instead by (a) published closed-form element
// stiffness matrices and independent quadratures (elastic and heat), (b) a
// direct sparse factorisation of the same assembled matrix, (c) the
// reference's own finite-difference sensitivity procedure, (d) properties the
// reference's filters have by construction (constants kept, sensitivity map =
// transpose).  The OC, MMA and GCMMA updates are pinned against ICARAT's own
// OCSolver.hpp / MMASolver.cpp / GCMMASolver.cpp compiled from source into
// oracle/_ref.
//
// Every function names the ICARAT source (path inside the ICARAT project,
// file:line) whose behaviour it restates.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <map>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

/// Structured box problem (src/io/mesh_icarat.hpp:69-128 `[mesh]` keys and
/// src/problem/elasticity.cpp:19-32 `[material]` keys).
struct OrcGrid
{
  int dim;       ///< 2 or 3
  int nx, ny, nz; ///< `division`
  double lx, ly, lz; ///< `length`
  int state;     ///< 0 plane_stress, 1 plane_strain, 2 3D
  double young1; ///< young[0]
  double young2; ///< young[1]
  double nu;     ///< poisson
  double penal;  ///< penalty
};
}

namespace
{
/// DOFs per node: dim for elasticity, 1 for heat conduction (state 3)
inline int dofnp(const OrcGrid &g) { return g.state == 3 ? 1 : g.dim; }

inline int64_t numnp(const OrcGrid &g)
{
  return g.dim == 2 ? int64_t(g.nx + 1) * (g.ny + 1)
                    : int64_t(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
}
inline int64_t nelx(const OrcGrid &g)
{
  return g.dim == 2 ? int64_t(g.nx) * g.ny : int64_t(g.nx) * g.ny * g.nz;
}
inline int nen(const OrcGrid &g) { return g.dim == 2 ? 4 : 8; }
inline double hx(const OrcGrid &g) { return g.lx / g.nx; }
inline double hy(const OrcGrid &g) { return g.ly / g.ny; }
inline double hz(const OrcGrid &g) { return g.dim == 3 ? g.lz / g.nz : 1.0; }

/// node coordinate as MeshIcarat::meshBox writes it (mesh_icarat.hpp:328-337,
/// 443-456): x = (length/division) * index.
inline void nodeX(const OrcGrid &g, int64_t n, double x[3])
{
  int64_t sx = g.nx + 1, sy = g.ny + 1;
  int64_t i = n % sx, j = (n / sx) % sy, k = n / (sx * sy);
  x[0] = (g.lx / g.nx) * i;
  x[1] = (g.ly / g.ny) * j;
  x[2] = g.dim == 3 ? (g.lz / g.nz) * k : 0.0;
}

/// element connectivity (mesh_icarat.hpp:340-354 quad4, 459-493 hexa8).
inline void elemNodes(const OrcGrid &g, int64_t e, int64_t *nd)
{
  int64_t sx = g.nx + 1;
  if(g.dim == 2)
  {
    int64_t j = e % g.nx, i = e / g.nx;
    int64_t b = i * sx + j;
    nd[0] = b;
    nd[1] = b + 1;
    nd[2] = b + 1 + sx;
    nd[3] = b + sx;
  }
  else
  {
    int64_t sxy = sx * (g.ny + 1);
    int64_t k = e % g.nx, j = (e / g.nx) % g.ny, i = e / (int64_t(g.nx) * g.ny);
    int64_t b = sxy * i + sx * j + k;
    nd[0] = b;
    nd[1] = b + 1;
    nd[2] = b + 1 + sx;
    nd[3] = b + sx;
    for(int q = 0; q < 4; q++)
      nd[4 + q] = nd[q] + sxy;
  }
}

/// natural coordinates of the local nodes (shape_function.cpp:97-118, 403-447)
const double kQ4r[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
const double kH8r[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                           {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};

/// D matrix of Elastic::De (elasticity.cpp:34-98), row-major voigt x voigt.
void makeDe(const OrcGrid &g, double E, double *D)
{
  double nu = g.nu;
  if(g.dim == 2)
  {
    for(int i = 0; i < 9; i++)
      D[i] = 0.0;
    if(g.state == 0)
    {
      D[0] = 1.0;
      D[1] = nu;
      D[4] = 1.0;
      D[8] = 0.5 * (1.0 - nu);
      D[3] = D[1];
      double s = E / (1.0 - nu * nu);
      for(int i = 0; i < 9; i++)
        D[i] *= s;
    }
    else
    {
      D[0] = 1.0;
      D[1] = nu / (1.0 - nu);
      D[4] = 1.0;
      D[8] = (1.0 - 2.0 * nu) / (2.0 * (1.0 - nu));
      D[3] = D[1];
      double s = E * ((1.0 - nu) / ((1.0 - 2.0 * nu) * (1.0 + nu)));
      for(int i = 0; i < 9; i++)
        D[i] *= s;
    }
  }
  else
  {
    for(int i = 0; i < 36; i++)
      D[i] = 0.0;
    double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = E / (2 * (1.0 + nu));
    for(int a = 0; a < 3; a++)
      for(int b = 0; b < 3; b++)
        D[a * 6 + b] = (a == b) ? lam + 2 * mu : lam;
    D[3 * 6 + 3] = mu;
    D[4 * 6 + 4] = mu;
    D[5 * 6 + 5] = mu;
  }
}

/// Gauss rule of Gauss4Square / Gauss8Cubic (gauss_integration.cpp:72-…,
/// 268-289): points +-1/sqrt(3), weights 1, listed in local-node order.
int gaussPoints(const OrcGrid &g, double pts[8][3])
{
  double a = 1.0 / std::sqrt(3.0);
  int n = nen(g);
  for(int q = 0; q < n; q++)
    for(int c = 0; c < g.dim; c++)
      pts[q][c] = a * (g.dim == 2 ? kQ4r[q][c] : kH8r[q][c]);
  return n;
}

/// dN/dX (dim x nen, row-major) and det(J)*w at one Gauss point for the
/// reference element at the origin (bmatrix.hpp:28-87 / 90-162).
double shapeGrad(const OrcGrid &g, const double *r, double *dNdX, double *N)
{
  int n = nen(g), d = g.dim;
  double dNdr[3][8];
  for(int a = 0; a < n; a++)
  {
    if(d == 2)
    {
      double ra = kQ4r[a][0], sa = kQ4r[a][1];
      N[a] = 0.25 * (1.0 + ra * r[0]) * (1.0 + sa * r[1]);
      dNdr[0][a] = 0.25 * ra * (1.0 + sa * r[1]);
      dNdr[1][a] = 0.25 * sa * (1.0 + ra * r[0]);
    }
    else
    {
      double ra = kH8r[a][0], sa = kH8r[a][1], ta = kH8r[a][2];
      N[a] = 0.125 * (1.0 + ra * r[0]) * (1.0 + sa * r[1]) * (1.0 + ta * r[2]);
      dNdr[0][a] = 0.125 * ra * (1.0 + sa * r[1]) * (1.0 + ta * r[2]);
      dNdr[1][a] = 0.125 * sa * (1.0 + ra * r[0]) * (1.0 + ta * r[2]);
      dNdr[2][a] = 0.125 * ta * (1.0 + ra * r[0]) * (1.0 + sa * r[1]);
    }
  }
  // X of the element: corners at 0 / h along each axis
  double h[3] = {hx(g), hy(g), hz(g)};
  double J[3][3] = {{0}};
  for(int i = 0; i < d; i++)
    for(int j = 0; j < d; j++)
    {
      double s = 0.0;
      for(int a = 0; a < n; a++)
      {
        double xa = (d == 2 ? kQ4r[a][j] : kH8r[a][j]) > 0 ? h[j] : 0.0;
        s += dNdr[i][a] * xa;
      }
      J[i][j] = s;
    }
  double det, inv[3][3];
  if(d == 2)
  {
    det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    inv[0][0] = J[1][1] / det;
    inv[0][1] = -J[0][1] / det;
    inv[1][0] = -J[1][0] / det;
    inv[1][1] = J[0][0] / det;
  }
  else
  {
    det = J[0][0] * (J[1][1] * J[2][2] - J[1][2] * J[2][1]) -
          J[0][1] * (J[1][0] * J[2][2] - J[1][2] * J[2][0]) +
          J[0][2] * (J[1][0] * J[2][1] - J[1][1] * J[2][0]);
    inv[0][0] = (J[1][1] * J[2][2] - J[1][2] * J[2][1]) / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][0] = (J[1][2] * J[2][0] - J[1][0] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][0] = (J[1][0] * J[2][1] - J[1][1] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  }
  for(int i = 0; i < d; i++)
    for(int a = 0; a < n; a++)
    {
      double s = 0.0;
      for(int k = 0; k < d; k++)
        s += inv[i][k] * dNdr[k][a];
      dNdX[i * n + a] = s;
    }
  return det; // Gauss weight is 1 for every point
}

/// structural B matrix (bmatrix.hpp:62-69, 125-140), voigt x (d*nen)
void makeB(const OrcGrid &g, const double *dNdX, double *B)
{
  int n = nen(g), d = g.dim, nd = d * n, v = d == 2 ? 3 : 6;
  for(int i = 0; i < v * nd; i++)
    B[i] = 0.0;
  for(int a = 0; a < n; a++)
  {
    double gx = dNdX[0 * n + a], gy = dNdX[1 * n + a];
    if(d == 2)
    {
      B[0 * nd + 2 * a] = gx;
      B[1 * nd + 2 * a + 1] = gy;
      B[2 * nd + 2 * a] = gy;
      B[2 * nd + 2 * a + 1] = gx;
    }
    else
    {
      double gz = dNdX[2 * n + a];
      B[0 * nd + 3 * a] = gx;
      B[1 * nd + 3 * a + 1] = gy;
      B[2 * nd + 3 * a + 2] = gz;
      B[3 * nd + 3 * a] = gy;
      B[3 * nd + 3 * a + 1] = gx;
      B[4 * nd + 3 * a + 1] = gz;
      B[4 * nd + 3 * a + 2] = gy;
      B[5 * nd + 3 * a] = gz;
      B[5 * nd + 3 * a + 2] = gx;
    }
  }
}

/// SIMP of elasticity.hpp:15-22
inline double simp(double y1, double y2, double s, double p)
{
  if(y2 - y1 >= 0.0)
    return (1.0 - std::pow(s, p)) * y1 + std::pow(s, p) * y2;
  return std::pow(1.0 - s, p) * y1 + (1.0 - std::pow(1.0 - s, p)) * y2;
}

struct Csr
{
  int64_t n = 0;
  std::vector<int64_t> rowptr;
  std::vector<int> col;
  std::vector<double> val;
  std::vector<double> diag;
};

void spmv(const Csr &A, const double *x, double *y)
{
#pragma omp parallel for schedule(static)
  for(int64_t r = 0; r < A.n; r++)
  {
    double s = 0.0;
    for(int64_t p = A.rowptr[r]; p < A.rowptr[r + 1]; p++)
      s += A.val[p] * x[A.col[p]];
    y[r] = s;
  }
}

double dot(int64_t n, const double *a, const double *b)
{
  double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
  for(int64_t i = 0; i < n; i++)
    s += a[i] * b[i];
  return s;
}

/// Jacobi-preconditioned CG with the semantics of Eigen 3.4's
/// ConjugateGradient<..., Lower|Upper, DiagonalPreconditioner> as called by
/// Solvers::EigenCG (src/analysis/solver/solvers.cpp:64-92): x0 = 0, stop when
/// ||r||^2 < tol^2 ||b||^2, iteration count excludes the final check,
/// inverse diagonal = 1 where the diagonal is 0.
int pcgCsr(const Csr &A, const double *b, double *x, double tol, int maxit,
           int *iters, double *relres, int *matvecs)
{
  int64_t n = A.n;
  std::vector<double> r(b, b + n), z(n), p(n), q(n), inv(n);
  for(int64_t i = 0; i < n; i++)
  {
    x[i] = 0.0;
    inv[i] = A.diag[i] != 0.0 ? 1.0 / A.diag[i] : 1.0;
  }
  double rhs2 = dot(n, b, b);
  *matvecs = 0;
  if(rhs2 == 0.0)
  {
    *iters = 0;
    *relres = 0.0;
    return 0;
  }
  double thr = std::max(tol * tol * rhs2, std::numeric_limits<double>::min());
  double r2 = rhs2;
  if(r2 < thr)
  {
    *iters = 0;
    *relres = std::sqrt(r2 / rhs2);
    return 0;
  }
  for(int64_t i = 0; i < n; i++)
    p[i] = inv[i] * r[i];
  double absNew = dot(n, r.data(), p.data());
  int it = 0;
  while(it < maxit)
  {
    spmv(A, p.data(), q.data());
    (*matvecs)++;
    double alpha = absNew / dot(n, p.data(), q.data());
#pragma omp parallel for schedule(static)
    for(int64_t i = 0; i < n; i++)
    {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
    }
    r2 = dot(n, r.data(), r.data());
    if(r2 < thr)
      break;
#pragma omp parallel for schedule(static)
    for(int64_t i = 0; i < n; i++)
      z[i] = inv[i] * r[i];
    double absOld = absNew;
    absNew = dot(n, r.data(), z.data());
    double beta = absNew / absOld;
#pragma omp parallel for schedule(static)
    for(int64_t i = 0; i < n; i++)
      p[i] = z[i] + beta * p[i];
    it++;
  }
  *iters = it;
  *relres = std::sqrt(r2 / rhs2);
  return r2 < thr ? 0 : 1;
}

/// grid index helpers
inline void nodeIJK(const OrcGrid &g, int64_t n, int &i, int &j, int &k)
{
  int64_t sx = g.nx + 1, sy = g.ny + 1;
  i = int(n % sx);
  j = int((n / sx) % sy);
  k = int(n / (sx * sy));
}
/// local index of the node at corner (a,b,c) of an element (meshBox order)
inline int localIdx(int dim, int a, int b, int c)
{
  static const int l2[2][2] = {{0, 3}, {1, 2}}; // [a][b]
  int l = l2[a][b];
  return dim == 2 ? l : l + 4 * c;
}

/// Assemble K(rho) over free DOFs in `dof` numbering: the result of
/// LinearAnalysis::assemblingK (src/analysis/linear.hpp:117-166) with
/// LinearElastic::makeKeFint (src/problem/elasticity.cpp:210-254) and the
/// elimination of constrained DOFs in assembling()
/// (src/misc/assembling.hpp:17-38).  Rows are built directly from the
/// structured stencil instead of a triplet sort (setFromTriplets sums
/// duplicates, so the entries are the same sums).
void assemble(const OrcGrid &g, const int *dof, int64_t numeq,
              const double *Eel, const double *K0, int scalarDofs, Csr &A)
{
  int d = scalarDofs ? 1 : g.dim;
  int n = nen(g), nd = d * n;
  int64_t nn = numnp(g);
  int sx = g.nx + 1, sy = g.ny + 1;
  int nzn = g.dim == 3 ? g.nz + 1 : 1;
  A.n = numeq;
  A.rowptr.assign(numeq + 1, 0);
  A.diag.assign(numeq, 0.0);
  auto nodeAt = [&](int i, int j, int k) -> int64_t {
    return int64_t(i) + int64_t(j) * sx + int64_t(k) * sx * sy;
  };
  // pass 1: counts
#pragma omp parallel for schedule(dynamic, 256)
  for(int64_t nd0 = 0; nd0 < nn; nd0++)
  {
    int i, j, k;
    nodeIJK(g, nd0, i, j, k);
    int cnt = 0;
    for(int dk = (g.dim == 3 ? -1 : 0); dk <= (g.dim == 3 ? 1 : 0); dk++)
      for(int dj = -1; dj <= 1; dj++)
        for(int di = -1; di <= 1; di++)
        {
          int mi = i + di, mj = j + dj, mk = k + dk;
          if(mi < 0 || mi >= sx || mj < 0 || mj >= sy || mk < 0 || mk >= nzn)
            continue;
          int64_t m = nodeAt(mi, mj, mk);
          for(int c2 = 0; c2 < d; c2++)
            if(dof[m * d + c2] < numeq)
              cnt++;
        }
    for(int c = 0; c < d; c++)
      if(dof[nd0 * d + c] < numeq)
        A.rowptr[dof[nd0 * d + c] + 1] = cnt;
  }
  for(int64_t r = 0; r < numeq; r++)
    A.rowptr[r + 1] += A.rowptr[r];
  A.col.resize(A.rowptr[numeq]);
  A.val.resize(A.rowptr[numeq]);
  // pass 2: values
#pragma omp parallel for schedule(dynamic, 256)
  for(int64_t nd0 = 0; nd0 < nn; nd0++)
  {
    int i, j, k;
    nodeIJK(g, nd0, i, j, k);
    for(int c = 0; c < d; c++)
    {
      int row = dof[nd0 * d + c];
      if(row >= numeq)
        continue;
      int64_t p = A.rowptr[row];
      for(int dk = (g.dim == 3 ? -1 : 0); dk <= (g.dim == 3 ? 1 : 0); dk++)
        for(int dj = -1; dj <= 1; dj++)
          for(int di = -1; di <= 1; di++)
          {
            int mi = i + di, mj = j + dj, mk = k + dk;
            if(mi < 0 || mi >= sx || mj < 0 || mj >= sy || mk < 0 || mk >= nzn)
              continue;
            int64_t m = nodeAt(mi, mj, mk);
            for(int c2 = 0; c2 < d; c2++)
            {
              int colj = dof[m * d + c2];
              if(colj >= numeq)
                continue;
              // elements containing both nodes, in element-index order
              double s = 0.0;
              for(int ek = (g.dim == 3 ? std::max(k, mk) - 1 : 0);
                  ek <= (g.dim == 3 ? std::min(k, mk) : 0); ek++)
                for(int ej = std::max(j, mj) - 1; ej <= std::min(j, mj); ej++)
                  for(int ei = std::max(i, mi) - 1; ei <= std::min(i, mi); ei++)
                  {
                    if(ei < 0 || ej < 0 || ek < 0 || ei >= g.nx || ej >= g.ny ||
                       (g.dim == 3 && ek >= g.nz))
                      continue;
                    int64_t e = g.dim == 2
                                    ? int64_t(ej) * g.nx + ei
                                    : (int64_t(ek) * g.ny + ej) * g.nx + ei;
                    int ln = localIdx(g.dim, i - ei, j - ej, k - ek);
                    int lm = localIdx(g.dim, mi - ei, mj - ej, mk - ek);
                    s += Eel[e] * K0[(ln * d + c) * nd + lm * d + c2];
                  }
              A.col[p] = colj;
              A.val[p] = s;
              if(colj == row)
                A.diag[row] = s;
              p++;
            }
          }
    }
  }
}

void unitK0(const OrcGrid &g, double *K0)
{
  int n = nen(g), d = g.dim, nd = n * d, v = d == 2 ? 3 : 6;
  double D[36], pts[8][3], dNdX[24], N[8], B[6 * 24];
  makeDe(g, 1.0, D);
  for(int i = 0; i < nd * nd; i++)
    K0[i] = 0.0;
  int nq = gaussPoints(g, pts);
  for(int q = 0; q < nq; q++)
  {
    double jac = shapeGrad(g, pts[q], dNdX, N);
    makeB(g, dNdX, B);
    // K += B^T D B jac
    double DB[6 * 24];
    for(int a = 0; a < v; a++)
      for(int j = 0; j < nd; j++)
      {
        double s = 0.0;
        for(int b = 0; b < v; b++)
          s += D[a * v + b] * B[b * nd + j];
        DB[a * nd + j] = s;
      }
    for(int i = 0; i < nd; i++)
      for(int j = 0; j < nd; j++)
      {
        double s = 0.0;
        for(int a = 0; a < v; a++)
          s += B[a * nd + i] * DB[a * nd + j];
        K0[i * nd + j] += s * jac;
      }
  }
}

/// Helmholtz element matrix and load integral of FilterHelmholtz::makeKeFint
/// (src/optimization/filter_helm.hpp:178-222): Ke = sum (N N^T + re^2 B^T B)
/// jac with re = R / (2 sqrt 3); Nint = sum N jac.
void helmKe(const OrcGrid &g, double R, double *Ke, double *Nint, double *Nq)
{
  int n = nen(g), d = g.dim;
  double pts[8][3], dNdX[24], N[8];
  double re2 = std::pow(R / (2 * std::sqrt(3.0)), 2);
  for(int i = 0; i < n * n; i++)
    Ke[i] = 0.0;
  for(int i = 0; i < n; i++)
    Nint[i] = 0.0;
  int nq = gaussPoints(g, pts);
  for(int q = 0; q < nq; q++)
  {
    double jac = shapeGrad(g, pts[q], dNdX, N);
    for(int a = 0; a < n; a++)
    {
      Nq[q * n + a] = N[a];
      for(int b = 0; b < n; b++)
      {
        double s = 0.0;
        for(int c = 0; c < d; c++)
          s += dNdX[c * n + a] * re2 * dNdX[c * n + b];
        Ke[a * n + b] += (N[a] * N[b] + s) * jac;
      }
      Nint[a] += N[a] * jac;
    }
  }
}

struct Cone
{
  OrcGrid g;
  double r;
  std::vector<int> off;    // neighbour offsets (di,dj,dk) triples
  std::vector<double> w;   // r - dist
  std::vector<double> aa;  // cached sum of weights (dfilters_ds)
};

} // namespace

extern "C" {

int64_t orc_numnp(const OrcGrid *g) { return numnp(*g); }
int64_t orc_nelx(const OrcGrid *g) { return nelx(*g); }

/// unit-modulus element stiffness K0 (E = 1): Ke of makeKeFint divided by E
void orc_K0(const OrcGrid *g, double *K0) { unitK0(*g, K0); }

/// element volume = sum of Gauss jac (elasticity.cpp:249)
double orc_element_volume(const OrcGrid *g)
{
  double pts[8][3], dNdX[24], N[8], v = 0.0;
  int nq = gaussPoints(*g, pts);
  for(int q = 0; q < nq; q++)
    v += shapeGrad(*g, pts[q], dNdX, N);
  return v;
}

/// BCIcarat::input_dirich (src/io/boundary_condition_icarat.hpp:68-127):
/// every node inside the box widened by 1e-7 gets the flags/values.
/// `fixed`, `dval`: neq, node-major interleaved.
void orc_dirichlet_box(const OrcGrid *g, const int *flag, const double *val,
                       const double *range, uint8_t *fixed, double *dval)
{
  double tol = 1.0e-7;
  double lo[3] = {range[0] - tol, range[2] - tol, range[4] - tol};
  double hi[3] = {range[1] + tol, range[3] + tol, range[5] + tol};
  int64_t nn = numnp(*g);
  int d = g->dim, nd = dofnp(*g);
  for(int64_t n = 0; n < nn; n++)
  {
    double x[3];
    nodeX(*g, n, x);
    bool in = true;
    for(int c = 0; c < d; c++)
      in = in && x[c] >= lo[c] && x[c] <= hi[c];
    if(!in)
      continue;
    // setDirichValue (boundary_condition_base.hpp:17-33): copies flag & value
    for(int c = 0; c < nd; c++)
    {
      fixed[n * nd + c] = uint8_t(flag[c] != 0);
      dval[n * nd + c] = val[c];
    }
  }
}

/// countDOF (src/io/boundary_condition_base.hpp:35-88): free DOFs numbered
/// node by node, constrained DOFs after them.  Returns numeq.
int64_t orc_count_dof(const OrcGrid *g, const uint8_t *fixed, int *dof)
{
  int64_t nn = numnp(*g);
  int d = dofnp(*g);
  int64_t cnt = 0;
  for(int64_t n = 0; n < nn; n++)
    for(int c = 0; c < d; c++)
      if(!fixed[n * d + c])
        dof[n * d + c] = int(cnt++);
  int64_t cc = cnt;
  for(int64_t n = 0; n < nn; n++)
    for(int c = 0; c < d; c++)
      if(fixed[n * d + c])
        dof[n * d + c] = int(cc++);
  return cnt;
}

/// BCIcarat::generateLoadMain + SurfaceLoad::judgeLine/generate for quad4 and
/// hexa8 (boundary_condition_icarat.hpp:300-385,
/// boundary_condition_base.cpp:16-86, 143-180, 182-378): an element side is
/// loaded when the `numnode`-th of its nodes (local order) falls in the box;
/// the side is picked from that local index exactly as judgeLine does; the
/// constant traction is integrated with the 2-point / 2x2 Gauss rule, which
/// on a straight edge / flat rectangle gives val * L / 2 (val * A / 4) per
/// side node.  Adds into `fext` (numeq).
void orc_traction_box(const OrcGrid *g, const double *val, const double *range,
                      const int *dof, int64_t numeq, double *fext)
{
  double tol = 1.0e-7;
  double lo[3] = {range[0] - tol, range[2] - tol, range[4] - tol};
  double hi[3] = {range[1] + tol, range[3] + tol, range[5] + tol};
  int d = g->dim, ne = nen(*g), numnode = d == 2 ? 2 : 4;
  int64_t ne_tot = nelx(*g);
  static const int q4side[5][2] = {{0, 0}, {0, 1}, {1, 2}, {2, 3}, {3, 0}};
  static const int h8side[7][4] = {{0, 0, 0, 0}, {0, 1, 2, 3}, {3, 0, 4, 7},
                                   {0, 1, 5, 4}, {1, 2, 6, 5}, {2, 3, 7, 6},
                                   {4, 5, 6, 7}};
  for(int64_t e = 0; e < ne_tot; e++)
  {
    int64_t nd[8];
    elemNodes(*g, e, nd);
    int counter = 0;
    int hit[8];
    for(int k = 0; k < ne; k++)
    {
      double x[3];
      nodeX(*g, nd[k], x);
      bool in = true;
      for(int c = 0; c < d; c++)
        in = in && lo[c] <= x[c] && x[c] <= hi[c];
      if(!in)
        continue;
      hit[counter++] = k;
      if(counter != numnode)
        continue;
      int side;
      if(d == 2)
      {
        if(k == 1)
          side = 1;
        else if(k == 2)
          side = 2;
        else
          side = (hit[1] - hit[0] == 1) ? 3 : 4;
      }
      else
      {
        if(k == 3)
          side = 1;
        else if(k == 5)
          side = 3;
        else if(k == 6)
          side = 4;
        else if(hit[2] - hit[1] == 1)
          side = 2;
        else if(hit[1] - hit[0] == 1)
          side = 5;
        else
          side = 6;
      }
      // measure of the side from its node coordinates (Gauss-integrated jac)
      double share;
      if(d == 2)
      {
        double xa[3], xb[3];
        nodeX(*g, nd[q4side[side][0]], xa);
        nodeX(*g, nd[q4side[side][1]], xb);
        double L = std::sqrt(std::pow(xb[0] - xa[0], 2) + std::pow(xb[1] - xa[1], 2));
        share = 0.5 * L; // sum over 2 points of N * (L/2)
        for(int s = 0; s < 2; s++)
          for(int c = 0; c < dofnp(*g); c++)
          {
            int dd = dof[nd[q4side[side][s]] * dofnp(*g) + c];
            if(dd < numeq)
              fext[dd] += share * val[c];
          }
      }
      else
      {
        double X[4][3];
        for(int s = 0; s < 4; s++)
          nodeX(*g, nd[h8side[side][s]], X[s]);
        // bilinear quad: |dX/dr x dX/ds| at the 4 Gauss points
        double a = 1.0 / std::sqrt(3.0);
        double gp[4][2] = {{-a, -a}, {a, -a}, {-a, a}, {a, a}};
        double fe[4] = {0, 0, 0, 0};
        for(int q = 0; q < 4; q++)
        {
          double r = gp[q][0], t = gp[q][1];
          double Nq[4] = {0.25 * (1 - r) * (1 - t), 0.25 * (1 + r) * (1 - t),
                          0.25 * (1 + r) * (1 + t), 0.25 * (1 - r) * (1 + t)};
          double dr[4] = {-0.25 * (1 - t), 0.25 * (1 - t), 0.25 * (1 + t),
                          -0.25 * (1 + t)};
          double ds[4] = {-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r),
                          0.25 * (1 - r)};
          double t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
          for(int s = 0; s < 4; s++)
            for(int c = 0; c < 3; c++)
            {
              t1[c] += dr[s] * X[s][c];
              t2[c] += ds[s] * X[s][c];
            }
          double cx = t1[1] * t2[2] - t1[2] * t2[1];
          double cy = t1[2] * t2[0] - t1[0] * t2[2];
          double cz = t1[0] * t2[1] - t1[1] * t2[0];
          double jac = std::sqrt(cx * cx + cy * cy + cz * cz);
          for(int s = 0; s < 4; s++)
            fe[s] += Nq[s] * jac;
        }
        for(int s = 0; s < 4; s++)
          for(int c = 0; c < dofnp(*g); c++)
          {
            int dd = dof[nd[h8side[side][s]] * dofnp(*g) + c];
            if(dd < numeq)
              fext[dd] += fe[s] * val[c];
          }
      }
    }
  }
}

/// Young's modulus of every element via SIMP (elasticity.hpp:15-22)
void orc_simp(const OrcGrid *g, const double *rho, double *E)
{
  int64_t n = nelx(*g);
#pragma omp parallel for
  for(int64_t e = 0; e < n; e++)
    E[e] = simp(g->young1, g->young2, rho[e], g->penal);
}

// ------------------------------------------------------------------ CSR ----
void *orc_csr_assemble(const OrcGrid *g, const int *dof, int64_t numeq,
                       const double *rho)
{
  Csr *A = new Csr;
  std::vector<double> K0(24 * 24), E(nelx(*g));
  unitK0(*g, K0.data());
  orc_simp(g, rho, E.data());
  assemble(*g, dof, numeq, E.data(), K0.data(), 0, *A);
  return A;
}
void orc_csr_free(void *h) { delete static_cast<Csr *>(h); }
int64_t orc_csr_nnz(void *h) { return static_cast<Csr *>(h)->rowptr.back(); }
void orc_csr_export(void *h, int64_t *rowptr, int *col, double *val)
{
  Csr *A = static_cast<Csr *>(h);
  std::memcpy(rowptr, A->rowptr.data(), sizeof(int64_t) * (A->n + 1));
  std::memcpy(col, A->col.data(), sizeof(int) * A->col.size());
  std::memcpy(val, A->val.data(), sizeof(double) * A->val.size());
}
void orc_csr_spmv(void *h, const double *x, double *y)
{
  spmv(*static_cast<Csr *>(h), x, y);
}
int orc_csr_pcg(void *h, const double *b, double *x, double tol, int maxit,
                int *iters, double *relres, int *matvecs)
{
  return pcgCsr(*static_cast<Csr *>(h), b, x, tol, maxit, iters, relres,
                matvecs);
}
/// timing helper for the CPU baseline: run exactly `nit` Jacobi-PCG
/// iterations (no convergence exit) and return the final relative residual.
double orc_csr_pcg_fixed(void *h, const double *b, double *x, int nit)
{
  int it, mv;
  double rr;
  pcgCsr(*static_cast<Csr *>(h), b, x, 0.0, nit, &it, &rr, &mv);
  return rr;
}

/// LinearAnalysis::solve (src/analysis/linear.hpp:54-104) with the
/// Eigen_CG solver: Dirichlet values into the nodes, fint from the assembled
/// element forces, fres = fext - fint, Jacobi-PCG on K_ff, then
/// divideValIntoNode (src/analysis/analysis_utility.hpp:8-31) which zeroes
/// |v| < 1e-15.  Outputs value.val (numeq), node values (neq) and the
/// compliance value.val . fext (opt_macro_oc.cpp:110).
int orc_linear_solve(const OrcGrid *g, const uint8_t *fixed, const double *dval,
                     const int *dof, int64_t numeq, const double *fext,
                     const double *rho, double tol, int maxit, double *u,
                     double *nodeval, double *compliance, int *iters,
                     double *relres, int *matvecs)
{
  int d = g->dim, ne = nen(*g), nd = d * ne;
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<double> K0(24 * 24), E(nel);
  unitK0(*g, K0.data());
  orc_simp(g, rho, E.data());
  Csr A;
  assemble(*g, dof, numeq, E.data(), K0.data(), 0, A);
  // fint from the Dirichlet values (fe = Ke * disp, free rows only)
  std::vector<double> fres(fext, fext + numeq);
  bool anyD = false;
  for(int64_t i = 0; i < nn * d; i++)
    if(fixed[i] && dval[i] != 0.0)
      anyD = true;
  if(anyD)
  {
    std::vector<double> fint(numeq, 0.0);
    for(int64_t e = 0; e < nel; e++)
    {
      int64_t ndn[8];
      elemNodes(*g, e, ndn);
      double ue[24];
      for(int a = 0; a < ne; a++)
        for(int c = 0; c < d; c++)
        {
          int64_t gi = ndn[a] * d + c;
          ue[a * d + c] = fixed[gi] ? dval[gi] : 0.0;
        }
      for(int a = 0; a < ne; a++)
        for(int c = 0; c < d; c++)
        {
          int r = dof[ndn[a] * d + c];
          if(r >= numeq)
            continue;
          double s = 0.0;
          for(int j = 0; j < nd; j++)
            s += E[e] * K0[(a * d + c) * nd + j] * ue[j];
          fint[r] += s;
        }
    }
    for(int64_t i = 0; i < numeq; i++)
      fres[i] -= fint[i];
  }
  int rc = pcgCsr(A, fres.data(), u, tol, maxit, iters, relres, matvecs);
  for(int64_t n = 0; n < nn; n++)
    for(int c = 0; c < d; c++)
    {
      int64_t gi = n * d + c;
      double v = dof[gi] >= numeq ? dval[gi] : u[dof[gi]];
      if(std::fabs(v) < 1.0e-15)
        v = 0.0;
      nodeval[gi] = v;
    }
  *compliance = dot(numeq, u, fext);
  return rc;
}

/// element sensitivity of the apps' sensitivity() (opt_macro_oc.cpp:182-207,
/// opt_mma_Helmholtz.cpp:173-205): dc_e = -(E'/E) u_e^T Ke u_e with
/// Ke = E K0, u_e from the node values.
void orc_sensitivity(const OrcGrid *g, const double *rho, const double *nodeval,
                     double *dc)
{
  int d = g->dim, ne = nen(*g), nd = d * ne;
  int64_t nel = nelx(*g);
  std::vector<double> K0(24 * 24);
  unitK0(*g, K0.data());
  double y1 = g->young1, y2 = g->young2, p = g->penal;
#pragma omp parallel for schedule(static)
  for(int64_t e = 0; e < nel; e++)
  {
    double s = rho[e], young, dyoung;
    if(y2 >= y1)
    {
      young = (1.0 - std::pow(s, p)) * y1 + std::pow(s, p) * y2;
      dyoung = p * std::pow(s, p - 1.0) * (y2 - y1);
    }
    else
    {
      young = std::pow(1.0 - s, p) * y1 + (1.0 - std::pow(1.0 - s, p)) * y2;
      dyoung = (y2 - y1) * p * std::pow(1.0 - s, p - 1.0);
    }
    int64_t ndn[8];
    elemNodes(*g, e, ndn);
    double ue[24];
    for(int a = 0; a < ne; a++)
      for(int c = 0; c < d; c++)
        ue[a * d + c] = nodeval[ndn[a] * d + c];
    double q = 0.0;
    for(int i = 0; i < nd; i++)
    {
      double t = 0.0;
      for(int j = 0; j < nd; j++)
        t += young * K0[i * nd + j] * ue[j];
      q += ue[i] * t;
    }
    dc[e] = -(dyoung / young) * q;
  }
}

// -------------------------------------------------------------- filters ----
/// Filter<E,N> (src/optimization/filter.hpp:59-66, 191-234).  Neighbour sets
/// are built from integer element offsets with |offset * h| <= r, which on a
/// uniform grid is the set the O(N^2) preNeighbour scan finds; offsets are
/// kept in increasing element-index order, the order preNeighbour lists them.
void *orc_cone_create(const OrcGrid *g, double r)
{
  Cone *c = new Cone;
  c->g = *g;
  c->r = r;
  double h[3] = {hx(*g), hy(*g), hz(*g)};
  int R[3];
  for(int a = 0; a < 3; a++)
    R[a] = int(std::floor(r / h[a])) + 1;
  if(g->dim == 2)
    R[2] = 0;
  for(int dk = -R[2]; dk <= R[2]; dk++)
    for(int dj = -R[1]; dj <= R[1]; dj++)
      for(int di = -R[0]; di <= R[0]; di++)
      {
        double dx = di * h[0], dy = dj * h[1], dz = dk * h[2];
        double dist = std::sqrt(dx * dx + dy * dy + (g->dim == 3 ? dz * dz : 0.0));
        if(dist <= r)
        {
          c->off.push_back(di);
          c->off.push_back(dj);
          c->off.push_back(dk);
          c->w.push_back(r - dist);
        }
      }
  c->aa.assign(nelx(*g), 0.0);
  return c;
}
void orc_cone_free(void *h) { delete static_cast<Cone *>(h); }
int orc_cone_size(void *h) { return int(static_cast<Cone *>(h)->w.size()); }

/// Filter::densityFilter (filter.hpp:102-151): isSens = 0 forward (caches
/// aa), isSens = 1 adjoint sum w g_j / aa_j.
int orc_cone_apply(void *h, const double *in, double *out, int isSens)
{
  Cone *c = static_cast<Cone *>(h);
  const OrcGrid &g = c->g;
  int64_t nel = nelx(g);
  int nnb = int(c->w.size());
  int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
  for(int64_t e = 0; e < nel; e++)
  {
    int i = int(e % g.nx), j, k;
    if(g.dim == 2)
    {
      j = int(e / g.nx);
      k = 0;
    }
    else
    {
      j = int((e / g.nx) % g.ny);
      k = int(e / (int64_t(g.nx) * g.ny));
    }
    double aa = 0.0, bb = 0.0;
    for(int t = 0; t < nnb; t++)
    {
      int ii = i + c->off[3 * t], jj = j + c->off[3 * t + 1], kk = k + c->off[3 * t + 2];
      if(ii < 0 || jj < 0 || kk < 0 || ii >= g.nx || jj >= g.ny ||
         (g.dim == 3 && kk >= g.nz))
        continue;
      int64_t f = g.dim == 2 ? int64_t(jj) * g.nx + ii
                             : (int64_t(kk) * g.ny + jj) * g.nx + ii;
      double w = c->w[t];
      if(!isSens)
      {
        aa += w;
        bb += w * in[f];
      }
      else
        bb += w * in[f] / c->aa[f];
    }
    if(!isSens)
    {
      if(aa < 1.0e-10)
        bad = 1;
      out[e] = bb / aa;
      c->aa[e] = aa;
    }
    else
      out[e] = bb;
  }
  return bad;
}

/// O(N^2) neighbour scan exactly as preNeighbour (filter.hpp:191-234), for
/// checking the stencil on small grids.  Writes per element the neighbour
/// count; returns the total.
int64_t orc_cone_bruteforce_counts(const OrcGrid *g, double r, int *counts)
{
  int64_t nel = nelx(*g);
  int ne = nen(*g), d = g->dim;
  std::vector<double> cen(nel * 3, 0.0);
  for(int64_t e = 0; e < nel; e++)
  {
    int64_t nd[8];
    elemNodes(*g, e, nd);
    for(int c = 0; c < d; c++)
      for(int a = 0; a < ne; a++)
      {
        double x[3];
        nodeX(*g, nd[a], x);
        cen[e * 3 + c] += x[c] / ne;
      }
  }
  int64_t tot = 0;
  for(int64_t e = 0; e < nel; e++)
  {
    int cnt = 0;
    for(int64_t f = 0; f < nel; f++)
    {
      double s = 0.0;
      for(int c = 0; c < d; c++)
        s += std::pow(cen[e * 3 + c] - cen[f * 3 + c], 2);
      if(std::sqrt(s) <= r)
        cnt++;
    }
    counts[e] = cnt;
    tot += cnt;
  }
  return tot;
}

/// Filter::threshold / thresholdDerivative (filter.hpp:153-185)
void orc_threshold(int64_t n, const double *x, double beta, double T,
                   double *out)
{
  for(int64_t i = 0; i < n; i++)
    out[i] = 0.5 * (std::tanh(T * beta) + std::tanh(beta * (x[i] - T))) /
             std::tanh(T * beta);
}
void orc_threshold_deriv(int64_t n, const double *x, double beta, double T,
                         double *out)
{
  for(int64_t i = 0; i < n; i++)
    out[i] = (0.5 * (beta * (1.0 - std::pow(std::tanh(beta * (x[i] - T)), 2.0))) /
              std::tanh(T * beta));
}

/// FilterHelmholtz::densityFilter (src/optimization/filter_helm.hpp:75-137,
/// 178-256): assemble (M + re^2 K_grad) over all nodes, rhs = sum_e x_e
/// int N (divided by ipmax when sensFlag), Jacobi-PCG ("Eigen_CG", default
/// tol), element value = sum_ip N(ip) . phi_e (divided by ipmax unless
/// sensFlag).
int orc_helmholtz(const OrcGrid *g, double R, const double *in, double *out,
                  int sensFlag, double tol, int *iters)
{
  OrcGrid gs = *g;
  int ne = nen(gs);
  int64_t nn = numnp(gs), nel = nelx(gs);
  double Ke[64], Nint[8], Nq[64];
  helmKe(gs, R, Ke, Nint, Nq);
  std::vector<int> dof(nn);
  for(int64_t i = 0; i < nn; i++)
    dof[i] = int(i);
  std::vector<double> ones(nel, 1.0);
  Csr A;
  assemble(gs, dof.data(), nn, ones.data(), Ke, 1, A);
  std::vector<double> rhs(nn, 0.0), phi(nn, 0.0);
  for(int64_t e = 0; e < nel; e++)
  {
    int64_t nd[8];
    elemNodes(gs, e, nd);
    for(int a = 0; a < ne; a++)
    {
      double fe = in[e] * Nint[a];
      if(sensFlag)
        fe = fe / ne;
      rhs[nd[a]] += fe;
    }
  }
  int it, mv;
  double rr;
  int rc = pcgCsr(A, rhs.data(), phi.data(), tol, 10000, &it, &rr, &mv);
  if(iters)
    *iters = it;
#pragma omp parallel for schedule(static)
  for(int64_t e = 0; e < nel; e++)
  {
    int64_t nd[8];
    elemNodes(gs, e, nd);
    double s = 0.0;
    for(int q = 0; q < ne; q++)
    {
      double t = 0.0;
      for(int a = 0; a < ne; a++)
        t += Nq[q * ne + a] * phi[nd[a]];
      s += t;
    }
    out[e] = sensFlag ? s : s / ne;
  }
  return rc;
}

// ------------------------------------------------------------------- OC ----
typedef double (*orc_volume_cb)(const double *xkp1, void *ud);

/// OC::UpdateVariables (src/optimization/opt-solver/OCSolver.hpp:20-68):
/// bisection on lambda in [0, 1e4] until (l1-l0)/(l1+l0) <= 1e-5 or 100
/// steps; x+ = x * max(0, -df/(dg lambda))^0.5 clamped by the move limit and
/// the bounds; lambda goes up while gkp1(x+) - g > 0.
int orc_oc_update(int64_t n, double *x, const double *dfdx, double g,
                  const double *dgdx, const double *xmin, const double *xmax,
                  double movelimit, orc_volume_cb gkp1, void *ud)
{
  double l0 = 0.0, l1 = 1.0e4, lam;
  std::vector<double> xn(n);
  int counter = 0;
  while((l1 - l0) / (l1 + l0) > 1.0e-5 && counter < 100)
  {
    lam = 0.5 * (l1 + l0);
#pragma omp parallel for schedule(static)
    for(int64_t i = 0; i < n; i++)
    {
      double v = std::pow(std::max(0.0, -dfdx[i] / (dgdx[i] * lam)), 0.5) * x[i];
      double lo = std::max(xmin[i], (1.0 - movelimit) * x[i]);
      double hi = std::min(xmax[i], (1.0 + movelimit) * x[i]);
      if(v < lo)
        v = lo;
      else if(v > hi)
        v = hi;
      xn[i] = v;
    }
    if(gkp1(xn.data(), ud) - g > 0.0)
      l0 = lam;
    else
      l1 = lam;
    counter++;
  }
  std::copy(xn.begin(), xn.end(), x);
  return counter;
}

// ------------------------------------------------------------------ MMA ----
/// Svanberg's MMA subproblem solved in the dual by a primal-dual interior
/// point iteration, with the parameters ICARAT sets in MMASolver's
/// constructor (src/optimization/opt-solver/MMASolver.cpp:41-55): move 0.15,
/// albefa 0.2, asyminit 0.2, asymdec 0.7, asyminc 1.2, raa0 1e-5, c = 1e5,
/// a = d = 0, epsimin = sqrt(n+m) 1e-9; asymptote update as GenSub
/// (:400-512); dual Newton steps, line search and stopping as SolveDIP
/// (:88-154).  Written here from the published method for m constraints.
struct Mma
{
  int64_t n;
  int m, iter = 0;
  double move = 0.15, albefa = 0.2, asyminit = 0.2, asymdec = 0.7,
         asyminc = 1.2, raa0 = 1e-5, xmamieps = 1e-5, epsimin;
  std::vector<double> a, c, low, upp, alpha, beta, p0, q0, pij, qij, b,
      xold1, xold2, lam, mu, y, grad, hess, s;
  double z = 0.0;
  // GCMMA only: constraint raa, constant terms and approximation values
  std::vector<double> raa, r, fapp;
  double r0 = 0.0, f0app = 0.0;
  int dualCap = 100; // outer-loop cap of the dual (none in GCMMA: 1 << 30)
};

void *orc_mma_create(int64_t n, int m, double a, double c, double d)
{
  (void)d;
  Mma *M = new Mma;
  M->n = n;
  M->m = m;
  M->epsimin = std::sqrt(double(n + m)) * 1e-9;
  M->a.assign(m, a);
  M->c.assign(m, c);
  for(auto *v : {&M->low, &M->upp, &M->alpha, &M->beta, &M->p0, &M->q0,
                 &M->xold1, &M->xold2})
    v->assign(n, 0.0);
  M->pij.assign(n * m, 0.0);
  M->qij.assign(n * m, 0.0);
  for(auto *v : {&M->b, &M->lam, &M->mu, &M->y, &M->grad})
    v->assign(m, 0.0);
  M->hess.assign(m * m, 0.0);
  M->s.assign(2 * m, 0.0);
  return M;
}
void orc_mma_free(void *h) { delete static_cast<Mma *>(h); }

namespace
{
void mmaPrimal(Mma &M, double *x)
{
  double lamai = 0.0;
  for(int j = 0; j < M.m; j++)
  {
    if(M.lam[j] < 0.0)
      M.lam[j] = 0.0;
    M.y[j] = std::max(0.0, M.lam[j] - M.c[j]);
    lamai += M.lam[j] * M.a[j];
  }
  M.z = std::max(0.0, 10.0 * (lamai - 1.0));
  for(int64_t i = 0; i < M.n; i++)
  {
    double pl = M.p0[i], ql = M.q0[i];
    for(int j = 0; j < M.m; j++)
    {
      pl += M.pij[i * M.m + j] * M.lam[j];
      ql += M.qij[i * M.m + j] * M.lam[j];
    }
    double sp = std::sqrt(pl), sq = std::sqrt(ql);
    double xi = (sp * M.low[i] + sq * M.upp[i]) / (sp + sq);
    xi = std::min(std::max(xi, M.alpha[i]), M.beta[i]);
    x[i] = xi;
  }
}
void mmaDualGrad(Mma &M, const double *x, std::vector<double> &g)
{
  for(int j = 0; j < M.m; j++)
  {
    double s = -M.b[j] - M.a[j] * M.z - M.y[j];
    for(int64_t i = 0; i < M.n; i++)
      s += M.pij[i * M.m + j] / (M.upp[i] - x[i]) +
           M.qij[i * M.m + j] / (x[i] - M.low[i]);
    g[j] = s;
  }
}
} // namespace

namespace
{
/// SolveDIP (MMASolver.cpp:88-154; GCMMASolver.cpp:128-200): the dual of the
/// subproblem by a primal-dual interior point iteration, x <- x(lambda)
void mmaDual(Mma &M, double *x)
{
  int64_t n = M.n;
  int m = M.m;
  for(int j = 0; j < m; j++)
  {
    M.lam[j] = M.c[j] / 2.0;
    M.mu[j] = 1.0;
  }
  double epsi = 1.0, err = 1.0;
  int outer = 0;
  std::vector<double> df2(n), PQ(n * m);
  while(epsi > M.epsimin && outer < M.dualCap)
  {
    outer++;
    int inner = 0;
    while(err > 0.9 * epsi && inner < 100)
    {
      inner++;
      mmaPrimal(M, x);
      mmaDualGrad(M, x, M.grad);
      for(int j = 0; j < m; j++)
        M.grad[j] = -1.0 * M.grad[j] - epsi / M.lam[j];
      // dual Hessian
      for(int64_t i = 0; i < n; i++)
      {
        double pl = M.p0[i], ql = M.q0[i];
        for(int j = 0; j < m; j++)
        {
          pl += M.pij[i * m + j] * M.lam[j];
          ql += M.qij[i * m + j] * M.lam[j];
          PQ[i * m + j] = M.pij[i * m + j] / std::pow(M.upp[i] - x[i], 2.0) -
                          M.qij[i * m + j] / std::pow(x[i] - M.low[i], 2.0);
        }
        double v = -1.0 / (2.0 * pl / std::pow(M.upp[i] - x[i], 3.0) +
                           2.0 * ql / std::pow(x[i] - M.low[i], 3.0));
        double xp = (std::sqrt(pl) * M.low[i] + std::sqrt(ql) * M.upp[i]) /
                    (std::sqrt(pl) + std::sqrt(ql));
        if(xp < M.alpha[i] || xp > M.beta[i])
          v = 0.0;
        df2[i] = v;
      }
      for(int r = 0; r < m; r++)
        for(int c = 0; c < m; c++)
        {
          double s = 0.0;
          for(int64_t i = 0; i < n; i++)
            s += PQ[i * m + r] * df2[i] * PQ[i * m + c];
          M.hess[r * m + c] = s;
        }
      double lamai = 0.0;
      for(int j = 0; j < m; j++)
      {
        if(M.lam[j] < 0.0)
          M.lam[j] = 0.0;
        lamai += M.lam[j] * M.a[j];
        if(M.lam[j] > M.c[j])
          M.hess[j * m + j] += -1.0;
        M.hess[j * m + j] += -M.mu[j] / M.lam[j];
      }
      if(lamai > 0.0)
        for(int r = 0; r < m; r++)
          for(int c = 0; c < m; c++)
            M.hess[r * m + c] += -10.0 * M.a[r] * M.a[c];
      double tr = 0.0;
      for(int j = 0; j < m; j++)
        tr += M.hess[j * m + j];
      double corr = 1e-4 * tr / m;
      if(-1.0 * corr < 1.0e-7)
        corr = -1.0e-7;
      for(int j = 0; j < m; j++)
        M.hess[j * m + j] += corr;
      // Newton step: solve hess * s = grad (LU without pivoting)
      if(m == 1)
        M.s[0] = M.grad[0] / M.hess[0];
      else
      {
        std::vector<double> K(M.hess), rhs(M.grad);
        for(int k = 0; k < m - 1; k++)
          for(int r = k + 1; r < m; r++)
          {
            K[r * m + k] /= K[k * m + k];
            for(int c = k + 1; c < m; c++)
              K[r * m + c] -= K[r * m + k] * K[k * m + c];
          }
        for(int r = 1; r < m; r++)
          for(int c = 0; c < r; c++)
            rhs[r] -= K[r * m + c] * rhs[c];
        for(int r = m - 1; r >= 0; r--)
        {
          double t = rhs[r];
          for(int c = r + 1; c < m; c++)
            t -= K[r * m + c] * rhs[c];
          rhs[r] = t / K[r * m + r];
        }
        for(int j = 0; j < m; j++)
          M.s[j] = rhs[j];
      }
      for(int j = 0; j < m; j++)
        M.s[m + j] = -M.mu[j] + epsi / M.lam[j] - M.s[j] * M.mu[j] / M.lam[j];
      // line search keeping lam, mu > 0
      double theta = 1.005;
      for(int j = 0; j < m; j++)
      {
        theta = std::max(theta, -1.01 * M.s[j] / M.lam[j]);
        theta = std::max(theta, -1.01 * M.s[m + j] / M.mu[j]);
      }
      theta = 1.0 / theta;
      for(int j = 0; j < m; j++)
      {
        M.lam[j] += theta * M.s[j];
        M.mu[j] += theta * M.s[m + j];
      }
      mmaPrimal(M, x);
      // KKT residual
      std::vector<double> gr(m);
      mmaDualGrad(M, x, gr);
      err = 0.0;
      for(int j = 0; j < m; j++)
      {
        double r1 = gr[j] + M.mu[j];
        double r2 = M.mu[j] * M.lam[j] - epsi;
        err = std::max(err, std::max(std::fabs(r1), std::fabs(r2)));
      }
    }
    epsi *= 0.1;
  }
}
} // namespace

void orc_mma_update(void *h, double *x, const double *dfdx, const double *gx,
                    const double *dgdx, const double *xmin, const double *xmax)
{
  Mma &M = *static_cast<Mma *>(h);
  int64_t n = M.n;
  int m = M.m;
  M.iter++;
  // asymptotes
  for(int64_t i = 0; i < n; i++)
  {
    double range = xmax[i] - xmin[i];
    if(M.iter < 3)
    {
      M.low[i] = x[i] - M.asyminit * range;
      M.upp[i] = x[i] + M.asyminit * range;
      continue;
    }
    double t = (x[i] - M.xold1[i]) * (M.xold1[i] - M.xold2[i]);
    double gam = t < 0.0 ? M.asymdec : (t > 0.0 ? M.asyminc : 1.0);
    double lo = x[i] - gam * (M.xold1[i] - M.low[i]);
    double up = x[i] + gam * (M.upp[i] - M.xold1[i]);
    double xmami = std::max(M.xmamieps, range);
    lo = std::min(std::max(lo, x[i] - 100.0 * xmami), x[i] - 1.0e-5 * xmami);
    up = std::min(std::max(up, x[i] + 1.0e-5 * xmami), x[i] + 100.0 * xmami);
    double xmi = xmin[i] - 1.0e-6, xma = xmax[i] + 1.0e-6;
    if(x[i] < xmi)
    {
      lo = x[i] - (xma - x[i]) / 0.9;
      up = x[i] + (xma - x[i]) / 0.9;
    }
    if(x[i] > xma)
    {
      lo = x[i] - (x[i] - xmi) / 0.9;
      up = x[i] + (x[i] - xmi) / 0.9;
    }
    M.low[i] = lo;
    M.upp[i] = up;
  }
  // bounds and approximation coefficients
  for(int64_t i = 0; i < n; i++)
  {
    double range = xmax[i] - xmin[i];
    double al = std::max(xmin[i], M.low[i] + M.albefa * (x[i] - M.low[i]));
    al = std::min(std::max(al, x[i] - M.move * range), xmax[i]);
    double be = std::min(xmax[i], M.upp[i] - M.albefa * (M.upp[i] - x[i]));
    be = std::max(std::min(be, x[i] + M.move * range), xmin[i]);
    M.alpha[i] = al;
    M.beta[i] = be;
    double inv = 1.0 / std::max(M.xmamieps, range);
    double u2 = std::pow(M.upp[i] - x[i], 2.0), l2 = std::pow(x[i] - M.low[i], 2.0);
    double pq = 0.001 * std::fabs(dfdx[i]) + M.raa0 * inv;
    M.p0[i] = u2 * (std::max(0.0, dfdx[i]) + pq);
    M.q0[i] = l2 * (std::max(0.0, -dfdx[i]) + pq);
    for(int j = 0; j < m; j++)
    {
      double gg = dgdx[i * m + j];
      double pqj = 0.001 * std::fabs(gg) + M.raa0 * inv;
      M.pij[i * m + j] = u2 * (std::max(0.0, gg) + pqj);
      M.qij[i * m + j] = l2 * (std::max(0.0, -gg) + pqj);
    }
  }
  for(int j = 0; j < m; j++)
  {
    double s = -gx[j];
    for(int64_t i = 0; i < n; i++)
      s += M.pij[i * m + j] / (M.upp[i] - x[i]) +
           M.qij[i * m + j] / (x[i] - M.low[i]);
    M.b[j] = s;
  }
  M.xold2 = M.xold1;
  std::copy(x, x + n, M.xold1.begin());

  mmaDual(M, x);
}

// ---------------------------------------------------------------- loops ----
/// The optimisation loop of opt-macro-oc (opt_macro_oc.cpp:84-172) on a
/// structured grid with a cone filter of radius `rfil`, without I/O and with
/// a fixed number of steps: filter, threshold (beta = min(2^(step/40), 16)
/// when `use_beta`, else beta skipped), solve, compliance, V0 at step 1,
/// sensitivities times the threshold derivative, adjoint filter, OC update
/// whose volume callback re-filters and re-thresholds.  Writes the
/// compliance of every step into `hist` and the final design into `x`.
struct OcCtx
{
  void *cone;
  double beta;
  bool use_beta;
  int64_t nel;
  double vol;
  std::vector<double> tmp, tmp2;
};
static double ocVolume(const double *xk, void *ud)
{
  OcCtx *c = static_cast<OcCtx *>(ud);
  orc_cone_apply(c->cone, xk, c->tmp.data(), 0);
  if(c->use_beta)
    orc_threshold(c->nel, c->tmp.data(), c->beta, 0.5, c->tmp2.data());
  else
    c->tmp2 = c->tmp;
  double g = 0.0;
  for(int64_t i = 0; i < c->nel; i++)
    g += c->tmp2[i] * c->vol;
  return g;
}

int orc_oc_loop(const OrcGrid *g, const uint8_t *fixed, const double *dval,
                const double *fext, const double *rho0, int nsteps,
                double rfil, double movelimit, int use_beta, double tol,
                double *hist, double *x, int *iters_total)
{
  int d = g->dim;
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<int> dof(nn * d);
  int64_t numeq = orc_count_dof(g, fixed, dof.data());
  std::vector<double> u(numeq), nodeval(nn * d), xf(nel), xt(nel), dxt(nel),
      dc(nel), dv(nel), xmin(nel, 1.0e-4), xmax(nel, 1.0);
  std::copy(rho0, rho0 + nel, x);
  void *cone = orc_cone_create(g, rfil);
  double vol = orc_element_volume(g);
  OcCtx ctx{cone, 1.0, use_beta != 0, nel, vol, std::vector<double>(nel),
            std::vector<double>(nel)};
  double V0 = 0.0;
  *iters_total = 0;
  for(int step = 1; step <= nsteps; step++)
  {
    orc_cone_apply(cone, x, xf.data(), 0);
    double beta = std::min(std::pow(2, (int)(step / 40)), 16.0);
    if(use_beta)
    {
      orc_threshold(nel, xf.data(), beta, 0.5, xt.data());
      orc_threshold_deriv(nel, xf.data(), beta, 0.5, dxt.data());
    }
    else
    {
      xt = xf;
      std::fill(dxt.begin(), dxt.end(), 1.0);
    }
    double comp;
    int it, mv;
    double rr;
    orc_linear_solve(g, fixed, dval, dof.data(), numeq, fext, xt.data(), tol,
                     100000, u.data(), nodeval.data(), &comp, &it, &rr, &mv);
    *iters_total += mv;
    hist[step - 1] = comp;
    if(step == 1)
    {
      V0 = 0.0;
      for(int64_t i = 0; i < nel; i++)
        V0 += xt[i] * vol;
    }
    orc_sensitivity(g, xt.data(), nodeval.data(), dc.data());
    for(int64_t i = 0; i < nel; i++)
    {
      dc[i] *= dxt[i];
      dv[i] = vol * dxt[i];
    }
    std::vector<double> t1(nel), t2(nel);
    orc_cone_apply(cone, dc.data(), t1.data(), 1);
    orc_cone_apply(cone, dv.data(), t2.data(), 1);
    // the forward-filter cache must be that of x (it is: the adjoint reads aa)
    ctx.beta = beta;
    orc_oc_update(nel, x, t1.data(), V0, t2.data(), xmin.data(), xmax.data(),
                  movelimit, ocVolume, &ctx);
  }
  orc_cone_free(cone);
  return 0;
}

/// The optimisation loop of opt-mma-HelmholtzFilter
/// (opt_mma_Helmholtz.cpp:81-163) without I/O: Helmholtz filter (radius
/// `R`), threshold, solve, V0 at step 1 (or the given `Vref` when > 0),
/// constraint sum x v / V0 - 1 (0 at step 1 as in the app), sensitivities
/// times the threshold derivative, adjoint Helmholtz filters, MMA update.
int orc_mma_loop(const OrcGrid *g, const uint8_t *fixed, const double *dval,
                 const double *fext, const double *rho0, int nsteps, double R,
                 double Vref, double tol, double *hist, double *x)
{
  int d = g->dim;
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<int> dof(nn * d);
  int64_t numeq = orc_count_dof(g, fixed, dof.data());
  std::vector<double> u(numeq), nodeval(nn * d), xf(nel), xt(nel), dxt(nel),
      dc(nel), dv(nel), xmin(nel, 1.0e-4), xmax(nel, 1.0), t1(nel), t2(nel);
  std::copy(rho0, rho0 + nel, x);
  double vol = orc_element_volume(g);
  void *mma = orc_mma_create(nel, 1, 0.0, 1e5, 0.0);
  double V0 = Vref;
  for(int step = 1; step <= nsteps; step++)
  {
    int it;
    orc_helmholtz(g, R, x, xf.data(), 0, 1e-10, &it);
    double beta = std::min(std::pow(2, (int)(step / 40)), 16.0);
    orc_threshold(nel, xf.data(), beta, 0.5, xt.data());
    double comp, rr;
    int mv;
    orc_linear_solve(g, fixed, dval, dof.data(), numeq, fext, xt.data(), tol,
                     100000, u.data(), nodeval.data(), &comp, &it, &rr, &mv);
    double gval = 0.0;
    if(step == 1 && Vref <= 0.0)
    {
      V0 = 0.0;
      for(int64_t i = 0; i < nel; i++)
        V0 += xt[i] * vol;
    }
    else
    {
      for(int64_t i = 0; i < nel; i++)
        gval += xt[i] * vol / V0;
      gval -= 1;
    }
    hist[step - 1] = comp;
    orc_sensitivity(g, xt.data(), nodeval.data(), dc.data());
    orc_threshold_deriv(nel, xf.data(), beta, 0.5, dxt.data());
    for(int64_t i = 0; i < nel; i++)
    {
      dc[i] *= dxt[i];
      dv[i] = vol / V0 * dxt[i];
    }
    orc_helmholtz(g, R, dc.data(), t1.data(), 1, 1e-10, &it);
    orc_helmholtz(g, R, dv.data(), t2.data(), 1, 1e-10, &it);
    orc_mma_update(mma, x, t1.data(), &gval, t2.data(), xmin.data(),
                   xmax.data());
  }
  orc_mma_free(mma);
  return 0;
}


// ------------------------------------------------------ stress, reactions ----
/// Elastic::makeMisesStress (elasticity.cpp:165-208): the element stress is
/// the Gauss-point average of D(E(rho)) B u_e and the von Mises value is
/// sqrt(s^T V s) with V = [[1,-.5,0],[-.5,1,0],[0,0,3]] in 2D (for plane
/// strain too, as the reference does) and the 6x6 counterpart in 3D.
/// stress (nel x voigt) may be NULL.
void orc_von_mises(const OrcGrid *g, const double *rho, const double *nodeval, double *mises,
                   double *stress)
{
  int d = g->dim, ne = nen(*g), nd = d * ne, v = d == 2 ? 3 : 6;
  int64_t nel = nelx(*g);
  double pts[8][3];
  int nq = gaussPoints(*g, pts);
  std::vector<double> Bq(size_t(nq) * v * nd);
  for(int q = 0; q < nq; q++)
  {
    double dNdX[24], N[8];
    shapeGrad(*g, pts[q], dNdX, N);
    makeB(*g, dNdX, &Bq[size_t(q) * v * nd]);
  }
  const double fac = 1.0 / nq;
#pragma omp parallel for schedule(static)
  for(int64_t e = 0; e < nel; e++)
  {
    double D[36];
    makeDe(*g, simp(g->young1, g->young2, rho[e], g->penal), D);
    int64_t ndn[8];
    elemNodes(*g, e, ndn);
    double ue[24];
    for(int a = 0; a < ne; a++)
      for(int c = 0; c < d; c++)
        ue[a * d + c] = nodeval[ndn[a] * d + c];
    double sig[6] = {0, 0, 0, 0, 0, 0};
    for(int q = 0; q < nq; q++)
    {
      const double *B = &Bq[size_t(q) * v * nd];
      double eps[6];
      for(int r = 0; r < v; r++)
      {
        double t = 0.0;
        for(int j = 0; j < nd; j++)
          t += B[r * nd + j] * ue[j];
        eps[r] = t;
      }
      for(int r = 0; r < v; r++)
      {
        double t = 0.0;
        for(int c = 0; c < v; c++)
          t += D[r * v + c] * eps[c];
        sig[r] += t * fac;
      }
    }
    double m2;
    if(d == 2)
      m2 = sig[0] * sig[0] + sig[1] * sig[1] - sig[0] * sig[1] + 3.0 * sig[2] * sig[2];
    else
      m2 = sig[0] * sig[0] + sig[1] * sig[1] + sig[2] * sig[2] - sig[0] * sig[1] -
           sig[1] * sig[2] - sig[0] * sig[2] +
           3.0 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5]);
    mises[e] = std::sqrt(m2);
    if(stress)
      for(int r = 0; r < v; r++)
        stress[e * v + r] = sig[r];
  }
}

/// The reaction of LinearAnalysis::assemblingK (linear.hpp:117-162,
/// assembling.hpp:79-84) as divideReactionIntoNode stores it
/// (analysis_utility.hpp:34-51): the internal force sum_e Ke u_e at every
/// DOF, node-major (neq), entries below 1e-15 in magnitude set to 0.
void orc_reactions(const OrcGrid *g, const double *rho, const double *nodeval, double *react)
{
  int d = g->dim, ne = nen(*g), nd = d * ne;
  int64_t nel = nelx(*g), neq = numnp(*g) * d;
  std::vector<double> K0(24 * 24);
  unitK0(*g, K0.data());
  std::fill(react, react + neq, 0.0);
  for(int64_t e = 0; e < nel; e++)
  {
    double E = simp(g->young1, g->young2, rho[e], g->penal);
    int64_t ndn[8];
    elemNodes(*g, e, ndn);
    double ue[24];
    for(int a = 0; a < ne; a++)
      for(int c = 0; c < d; c++)
        ue[a * d + c] = nodeval[ndn[a] * d + c];
    for(int i = 0; i < nd; i++)
    {
      double t = 0.0;
      for(int j = 0; j < nd; j++)
        t += K0[i * nd + j] * ue[j];
      react[ndn[i / d] * d + i % d] += E * t;
    }
  }
  for(int64_t i = 0; i < neq; i++)
    if(std::fabs(react[i]) < 1.0e-15)
      react[i] = 0.0;
}

/// The optimisation loop of opt-macro-mma-nondesign
/// (opt_macro_mma_nondesign.cpp:82-178) without I/O: cone filter (radius
/// rfil), threshold, solve, V0 over the elements flagged in `volset` (all when
/// NULL) at step 1, constraint sum_volset x v / V0 - 1 (0 at step 1),
/// sensitivities dv = v / V0 times the threshold derivative, adjoint cone
/// filter, sensitivities of the `nondesign` elements set to 0, MMA update.
int orc_mma_cone_loop(const OrcGrid *g, const uint8_t *fixed, const double *dval,
                      const double *fext, const double *rho0, int nsteps, double rfil,
                      const uint8_t *nondesign, const uint8_t *volset, double tol, double *hist,
                      double *x)
{
  int d = g->dim;
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<int> dof(nn * d);
  int64_t numeq = orc_count_dof(g, fixed, dof.data());
  std::vector<double> u(numeq), nodeval(nn * d), xf(nel), xt(nel), dxt(nel), dc(nel), dv(nel),
      xmin(nel, 1.0e-4), xmax(nel, 1.0), t1(nel), t2(nel);
  std::copy(rho0, rho0 + nel, x);
  double vol = orc_element_volume(g);
  void *mma = orc_mma_create(nel, 1, 0.0, 1e5, 0.0);
  void *cone = orc_cone_create(g, rfil);
  double V0 = 0.0;
  for(int step = 1; step <= nsteps; step++)
  {
    orc_cone_apply(cone, x, xf.data(), 0);
    double beta = std::min(std::pow(2, (int)(step / 40)), 16.0);
    orc_threshold(nel, xf.data(), beta, 0.5, xt.data());
    orc_threshold_deriv(nel, xf.data(), beta, 0.5, dxt.data());
    double comp, rr;
    int it, mv;
    orc_linear_solve(g, fixed, dval, dof.data(), numeq, fext, xt.data(), tol, 100000, u.data(),
                     nodeval.data(), &comp, &it, &rr, &mv);
    double gval = 0.0, vs = 0.0;
    for(int64_t i = 0; i < nel; i++)
      if(!volset || volset[i])
        vs += xt[i] * vol;
    if(step == 1)
      V0 = vs;
    else
      gval = vs / V0 - 1.0;
    hist[step - 1] = comp;
    orc_sensitivity(g, xt.data(), nodeval.data(), dc.data());
    for(int64_t i = 0; i < nel; i++)
    {
      dc[i] *= dxt[i];
      dv[i] = vol / V0 * dxt[i];
    }
    orc_cone_apply(cone, dc.data(), t1.data(), 1);
    orc_cone_apply(cone, dv.data(), t2.data(), 1);
    if(nondesign)
      for(int64_t i = 0; i < nel; i++)
        if(nondesign[i])
        {
          t1[i] = 0.0;
          t2[i] = 0.0;
        }
    orc_mma_update(mma, x, t1.data(), &gval, t2.data(), xmin.data(), xmax.data());
  }
  orc_cone_free(cone);
  orc_mma_free(mma);
  return 0;
}

// ---------------------------------------------------------------- GCMMA ----
/// GCMMA, the globally convergent MMA with conservative inner iterations, as
/// GCMMASolver sets it up (src/optimization/opt-solver/GCMMASolver.cpp:41-58):
/// raa0 = raa_j = 1 at start, raa0eps = raaeps = 1e-6, xmamieps 1e-5,
/// epsimin sqrt(n+m) 1e-9, move 0.15, albefa 0.2, asymptotes 0.2 / 0.7 /
/// 1.2, c = 1000 by default; the dual has no outer-loop cap.  Outer update
/// (:66-89): asymptotes and raa shrink (:432-508), subproblem (:546-596),
/// xold shift, dual, approximation values (:598-621).  Inner update
/// (:91-112): raa growth from the non-conservative misfit (:510-544), then
/// the same subproblem, dual and approximation.  Written from Svanberg's
/// published method with these constants.
void *orc_gcmma_create(int64_t n, int m, double a, double c, double d)
{
  Mma *M = static_cast<Mma *>(orc_mma_create(n, m, a, c, d));
  M->raa0 = 1.0;
  M->raa.assign(m, 1.0);
  M->r.assign(m, 0.0);
  M->fapp.assign(m, 0.0);
  M->dualCap = 1 << 30;
  return M;
}
void orc_gcmma_free(void *h) { delete static_cast<Mma *>(h); }

namespace
{
void gcAsymp(Mma &M, const double *x, const double *xmin, const double *xmax)
{
  M.iter++;
  for(int64_t i = 0; i < M.n; i++)
  {
    double range = xmax[i] - xmin[i];
    if(M.iter < 3)
    {
      M.low[i] = x[i] - M.asyminit * range;
      M.upp[i] = x[i] + M.asyminit * range;
      continue;
    }
    double t = (x[i] - M.xold1[i]) * (M.xold1[i] - M.xold2[i]);
    double gam = t < 0.0 ? M.asymdec : (t > 0.0 ? M.asyminc : 1.0);
    double lo = x[i] - gam * (M.xold1[i] - M.low[i]);
    double up = x[i] + gam * (M.upp[i] - M.xold1[i]);
    double xmami = std::max(M.xmamieps, range);
    lo = std::min(std::max(lo, x[i] - 100.0 * xmami), x[i] - 1.0e-5 * xmami);
    up = std::min(std::max(up, x[i] + 1.0e-5 * xmami), x[i] + 100.0 * xmami);
    double xmi = xmin[i] - 1.0e-6, xma = xmax[i] + 1.0e-6;
    if(x[i] < xmi)
    {
      lo = x[i] - (xma - x[i]) / 0.9;
      up = x[i] + (xma - x[i]) / 0.9;
    }
    if(x[i] > xma)
    {
      lo = x[i] - (x[i] - xmi) / 0.9;
      up = x[i] + (x[i] - xmi) / 0.9;
    }
    M.low[i] = lo;
    M.upp[i] = up;
  }
  M.raa0 = std::max(1e-6, 0.1 * M.raa0);
  for(int j = 0; j < M.m; j++)
    M.raa[j] = std::max(1e-6, 0.1 * M.raa[j]);
}

void gcSub(Mma &M, const double *x, double f0x, const double *df0dx, const double *fx,
           const double *dfdx, const double *xmin, const double *xmax)
{
  int m = M.m;
  double r0 = 0.0;
  std::vector<double> r(m, 0.0);
  for(int64_t i = 0; i < M.n; i++)
  {
    double range = xmax[i] - xmin[i];
    double al = std::max(xmin[i], M.low[i] + M.albefa * (x[i] - M.low[i]));
    M.alpha[i] = std::max(al, x[i] - M.move * range);
    double be = std::min(xmax[i], M.upp[i] - M.albefa * (M.upp[i] - x[i]));
    M.beta[i] = std::min(be, x[i] + M.move * range);
    double uxinv = 1.0 / (M.upp[i] - x[i]), xlinv = 1.0 / (x[i] - M.low[i]);
    double inv = 1.0 / std::max(M.xmamieps, range);
    double u2 = std::pow(M.upp[i] - x[i], 2.0), l2 = std::pow(x[i] - M.low[i], 2.0);
    double pq = 0.001 * std::fabs(df0dx[i]) + M.raa0 * inv;
    M.p0[i] = u2 * (std::max(0.0, df0dx[i]) + pq);
    M.q0[i] = l2 * (std::max(0.0, -df0dx[i]) + pq);
    r0 += M.p0[i] * uxinv + M.q0[i] * xlinv;
    for(int j = 0; j < m; j++)
    {
      double gg = dfdx[i * m + j];
      double pqj = 0.001 * std::fabs(gg) + M.raa[j] * inv;
      M.pij[i * m + j] = u2 * (std::max(0.0, gg) + pqj);
      M.qij[i * m + j] = l2 * (std::max(0.0, -gg) + pqj);
      r[j] += M.pij[i * m + j] * uxinv + M.qij[i * m + j] * xlinv;
    }
  }
  M.r0 = f0x - r0;
  for(int j = 0; j < m; j++)
  {
    M.r[j] = fx[j] - r[j];
    M.b[j] = -M.r[j];
  }
}

void gcApprox(Mma &M, const double *xmma)
{
  double f0 = 0.0;
  std::vector<double> f(M.m, 0.0);
  for(int64_t i = 0; i < M.n; i++)
  {
    double uxinv = 1.0 / (M.upp[i] - xmma[i]), xlinv = 1.0 / (xmma[i] - M.low[i]);
    f0 += M.p0[i] * uxinv + M.q0[i] * xlinv;
    for(int j = 0; j < M.m; j++)
      f[j] += M.pij[i * M.m + j] * uxinv + M.qij[i * M.m + j] * xlinv;
  }
  M.f0app = f0 + M.r0;
  for(int j = 0; j < M.m; j++)
    M.fapp[j] = f[j] + M.r[j];
}
} // namespace

void orc_gcmma_outer(void *h, double *xmma, const double *xval, double f0x, const double *df0dx,
                     const double *fx, const double *dfdx, const double *xmin, const double *xmax)
{
  Mma &M = *static_cast<Mma *>(h);
  gcAsymp(M, xval, xmin, xmax);
  gcSub(M, xval, f0x, df0dx, fx, dfdx, xmin, xmax);
  M.xold2 = M.xold1;
  std::copy(xval, xval + M.n, M.xold1.begin());
  std::copy(xval, xval + M.n, xmma);
  mmaDual(M, xmma);
  gcApprox(M, xmma);
}

void orc_gcmma_inner(void *h, double *xmma, double f0xnew, const double *fxnew, const double *xval,
                     double f0x, const double *df0dx, const double *fx, const double *dfdx,
                     const double *xmin, const double *xmax)
{
  Mma &M = *static_cast<Mma *>(h);
  double raacof = 0.0;
  for(int64_t i = 0; i < M.n; i++)
  {
    double xmami = std::max(M.xmamieps, xmax[i] - xmin[i]);
    double xxux = (xmma[i] - xval[i]) / (M.upp[i] - xmma[i]);
    double xxxl = (xmma[i] - xval[i]) / (xmma[i] - M.low[i]);
    raacof += xxux * xxxl * ((M.upp[i] - M.low[i]) / xmami);
  }
  raacof = std::max(1e-12, raacof);
  if(f0xnew > M.f0app + 0.5 * M.epsimin)
    M.raa0 = std::min(1.1 * (M.raa0 + (f0xnew - M.f0app) / raacof), 10.0 * M.raa0);
  for(int j = 0; j < M.m; j++)
    if(fxnew[j] > M.fapp[j] + 0.5 * M.epsimin)
      M.raa[j] = std::min(1.1 * (M.raa[j] + (fxnew[j] - M.fapp[j]) / raacof), 10.0 * M.raa[j]);
  gcSub(M, xval, f0x, df0dx, fx, dfdx, xmin, xmax);
  std::copy(xval, xval + M.n, xmma);
  mmaDual(M, xmma);
  gcApprox(M, xmma);
}

/// ConCheck (GCMMASolver.cpp:114-128): 1 when the approximations at xmma
/// are conservative for the new values
int orc_gcmma_concheck(void *h, double f0xnew, const double *fxnew)
{
  Mma &M = *static_cast<Mma *>(h);
  if(M.f0app + M.epsimin < f0xnew)
    return 0;
  for(int j = 0; j < M.m; j++)
    if(M.fapp[j] + M.epsimin < fxnew[j])
      return 0;
  return 1;
}

/// The optimisation loop of opt_macro_gcmma.cpp (:83-238) without I/O: cone
/// filter (radius rfil), threshold with beta = min(int(max((step - 100) / 40,
/// 1)), 8), solve, V0 at step 1, constraint sum x v - V0 (not normalised),
/// sensitivities times the threshold derivative (dv = v), adjoint filter,
/// GCMMA outer update, evaluation at the candidate, at most 15 inner updates
/// until the approximation is conservative.  hist[step] is the compliance of
/// the step's design; inner[step] the number of inner iterations.
int orc_gcmma_loop(const OrcGrid *g, const uint8_t *fixed, const double *dval, const double *fext,
                   const double *rho0, int nsteps, double rfil, double tol, double *hist, int *inner,
                   double *x)
{
  int d = g->dim;
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<int> dof(nn * d);
  int64_t numeq = orc_count_dof(g, fixed, dof.data());
  std::vector<double> u(numeq), nodeval(nn * d), xf(nel), xt(nel), dxt(nel), dc(nel), dv(nel),
      xmin(nel, 1.0e-4), xmax(nel, 1.0), t1(nel), t2(nel), xnew(nel);
  std::copy(rho0, rho0 + nel, x);
  double vol = orc_element_volume(g);
  void *gc = orc_gcmma_create(nel, 1, 0.0, 1000.0, 0.0);
  void *cone = orc_cone_create(g, rfil);
  double V0 = 0.0;
  auto evaluate = [&](const double *xx, double beta, double &f, double &gv) {
    orc_cone_apply(cone, xx, xf.data(), 0);
    orc_threshold(nel, xf.data(), beta, 0.5, xt.data());
    double rr;
    int it, mv;
    orc_linear_solve(g, fixed, dval, dof.data(), numeq, fext, xt.data(), tol, 100000, u.data(),
                     nodeval.data(), &f, &it, &rr, &mv);
    double vs = 0.0;
    for(int64_t i = 0; i < nel; i++)
      vs += xt[i] * vol;
    gv = vs;
  };
  for(int step = 1; step <= nsteps; step++)
  {
    int btmp = int(std::max((step - 100) / 40.0, 1.0));
    double beta = std::min(double(btmp), 8.0);
    double f, vs;
    evaluate(x, beta, f, vs);
    orc_threshold_deriv(nel, xf.data(), beta, 0.5, dxt.data());
    if(step == 1)
      V0 = vs;
    double gv = vs - V0;
    hist[step - 1] = f;
    orc_sensitivity(g, xt.data(), nodeval.data(), dc.data());
    for(int64_t i = 0; i < nel; i++)
    {
      dc[i] *= dxt[i];
      dv[i] = vol * dxt[i];
    }
    orc_cone_apply(cone, dc.data(), t1.data(), 1);
    orc_cone_apply(cone, dv.data(), t2.data(), 1);
    orc_gcmma_outer(gc, xnew.data(), x, f, t1.data(), &gv, t2.data(), xmin.data(), xmax.data());
    double fn, vn;
    evaluate(xnew.data(), beta, fn, vn);
    double gn = vn - V0;
    int k = 0;
    for(; !orc_gcmma_concheck(gc, fn, &gn) && k < 15; k++)
    {
      orc_gcmma_inner(gc, xnew.data(), fn, &gn, x, f, t1.data(), &gv, t2.data(), xmin.data(),
                      xmax.data());
      evaluate(xnew.data(), beta, fn, vn);
      gn = vn - V0;
    }
    if(inner)
      inner[step - 1] = k;
    std::copy(xnew.begin(), xnew.end(), x);
  }
  orc_cone_free(cone);
  orc_gcmma_free(gc);
  return 0;
}

// ----------------------------------------------------------------- heat ----
namespace
{
/// conductivity tensor from ICARAT's [xx, yy, zz, xy, yz, xz] (heat.cpp:31-51;
/// the 3D branch of the reference assigns De1_ twice, overwriting material
/// 1 with material 2 and leaving De2_ unset: here each material gets its own
/// tensor, the evident intent)
void condTensor(int dim, const double *c, double *D)
{
  if(dim == 2)
  {
    D[0] = c[0];
    D[1] = c[3];
    D[2] = c[3];
    D[3] = c[1];
  }
  else
  {
    const double v[9] = {c[0], c[3], c[5], c[3], c[1], c[4], c[5], c[4], c[2]};
    for(int i = 0; i < 9; i++)
      D[i] = v[i];
  }
}

/// LinearHeat::makeKeFint (heat.cpp:67-111) for a conductivity D: Ke =
/// sum over the Gauss points of B^T D B jac, B = dN/dX
void heatKe(const OrcGrid &g, const double *D, double *Ke)
{
  int ne = nen(g), d = g.dim;
  for(int i = 0; i < ne * ne; i++)
    Ke[i] = 0.0;
  double pts[8][3];
  int nq = gaussPoints(g, pts);
  for(int q = 0; q < nq; q++)
  {
    double dNdX[24], N[8];
    double jac = shapeGrad(g, pts[q], dNdX, N);
    for(int a = 0; a < ne; a++)
      for(int b = 0; b < ne; b++)
      {
        double t = 0.0;
        for(int i = 0; i < d; i++)
          for(int j = 0; j < d; j++)
            t += dNdX[i * ne + a] * D[i * d + j] * dNdX[j * ne + b];
        Ke[a * ne + b] += t * jac;
      }
  }
}
} // namespace

/// the element matrices K1, K2 of the two materials (ne x ne each)
void orc_heat_Ke(const OrcGrid *g, const double *cond1, const double *cond2, double *K1, double *K2)
{
  double D1[9], D2[9];
  condTensor(g->dim, cond1, D1);
  condTensor(g->dim, cond2, D2);
  heatKe(*g, D1, K1);
  heatKe(*g, D2, K2);
}

/// LinearAnalysis<LinearHeat, Node>::solve with Eigen_CG on the assembled
/// free-DOF matrix of Ke(rho) = rho^p K1 + (1 - rho^p) K2 (heat.cpp:53-64):
/// fres = fext - K_fd u_d, Jacobi-PCG from 0 to tol; nodeval[nnode] gets the
/// temperatures (Dirichlet values included, |T| < 1e-15 set to 0) and
/// *objective the app's u^T K u over the free DOFs (opt_heat.cpp:116).
int orc_heat_solve(const OrcGrid *g, const double *cond1, const double *cond2, const uint8_t *fixed,
                   const double *dval, const double *fext, const double *rho, double tol,
                   double *nodeval, double *objective, int *iters)
{
  int ne = nen(*g);
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<int> dof(nn);
  int64_t numeq = orc_count_dof(g, fixed, dof.data());
  std::vector<double> K1(ne * ne), K2(ne * ne);
  orc_heat_Ke(g, cond1, cond2, K1.data(), K2.data());
  std::vector<std::map<int, double>> rows(numeq);
  std::vector<double> b(fext, fext + numeq);
  for(int64_t e = 0; e < nel; e++)
  {
    double a = std::pow(rho[e], g->penal);
    int64_t nd[8];
    elemNodes(*g, e, nd);
    for(int i = 0; i < ne; i++)
    {
      int di = dof[nd[i]];
      if(di >= numeq)
        continue;
      for(int j = 0; j < ne; j++)
      {
        double k = a * K1[i * ne + j] + (1.0 - a) * K2[i * ne + j];
        int dj = dof[nd[j]];
        if(dj < numeq)
          rows[di][dj] += k;
        else
          b[di] -= k * dval[nd[j]];
      }
    }
  }
  Csr A;
  A.n = numeq;
  A.rowptr.assign(numeq + 1, 0);
  A.diag.assign(numeq, 0.0);
  for(int64_t r = 0; r < numeq; r++)
  {
    A.rowptr[r + 1] = A.rowptr[r] + int64_t(rows[r].size());
    for(auto &kv : rows[r])
    {
      A.col.push_back(kv.first);
      A.val.push_back(kv.second);
      if(kv.first == r)
        A.diag[r] = kv.second;
    }
  }
  std::vector<double> u(numeq);
  double rr;
  int mv;
  int rc = pcgCsr(A, b.data(), u.data(), tol, 100000, iters, &rr, &mv);
  std::vector<double> Ku(numeq);
  spmv(A, u.data(), Ku.data());
  *objective = dot(numeq, u.data(), Ku.data());
  for(int64_t n = 0; n < nn; n++)
  {
    double v = dof[n] < numeq ? u[dof[n]] : dval[n];
    nodeval[n] = std::fabs(v) < 1.0e-15 ? 0.0 : v;
  }
  return rc;
}

/// the heat app's sensitivity (opt_heat.cpp:155-190) without the threshold
/// factor: dc_e = -u_e^T (p rho^(p-1) (K1 - K2)) u_e
void orc_heat_sensitivity(const OrcGrid *g, const double *cond1, const double *cond2,
                          const double *rho, const double *nodeval, double *dc)
{
  int ne = nen(*g);
  int64_t nel = nelx(*g);
  std::vector<double> K1(ne * ne), K2(ne * ne);
  orc_heat_Ke(g, cond1, cond2, K1.data(), K2.data());
  for(int64_t e = 0; e < nel; e++)
  {
    double dk = g->penal * std::pow(rho[e], g->penal - 1.0);
    int64_t nd[8];
    elemNodes(*g, e, nd);
    double q = 0.0;
    for(int i = 0; i < ne; i++)
      for(int j = 0; j < ne; j++)
        q += nodeval[nd[i]] * dk * (K1[i * ne + j] - K2[i * ne + j]) * nodeval[nd[j]];
    dc[e] = -q;
  }
}

/// The opt-heat loop (opt_heat.cpp:79-151) without I/O: Helmholtz filter of
/// radius R, threshold (beta = min(2^(step/40), 16)), solve, V0 at step 1,
/// objective u^T K u, constraint sum x v - V0, sensitivities times the
/// threshold derivative (dv = derivative * v), adjoint Helmholtz filters, MMA.
int orc_heat_loop(const OrcGrid *g, const double *cond1, const double *cond2, const uint8_t *fixed,
                  const double *dval, const double *fext, const double *rho0, int nsteps, double R,
                  double tol, double *hist, double *x)
{
  int64_t nn = numnp(*g), nel = nelx(*g);
  std::vector<double> nodeval(nn), xf(nel), xt(nel), dxt(nel), dc(nel), dv(nel),
      xmin(nel, 1.0e-4), xmax(nel, 1.0), t1(nel), t2(nel);
  std::copy(rho0, rho0 + nel, x);
  double vol = orc_element_volume(g);
  void *mma = orc_mma_create(nel, 1, 0.0, 1e5, 0.0);
  double V0 = 0.0;
  for(int step = 1; step <= nsteps; step++)
  {
    int it;
    orc_helmholtz(g, R, x, xf.data(), 0, 1e-10, &it);
    double beta = std::min(std::pow(2, (int)(step / 40)), 16.0);
    orc_threshold(nel, xf.data(), beta, 0.5, xt.data());
    double obj;
    orc_heat_solve(g, cond1, cond2, fixed, dval, fext, xt.data(), tol, nodeval.data(), &obj, &it);
    double vs = 0.0;
    for(int64_t i = 0; i < nel; i++)
      vs += xt[i] * vol;
    if(step == 1)
      V0 = vs;
    double gval = vs - V0;
    hist[step - 1] = obj;
    orc_threshold_deriv(nel, xf.data(), beta, 0.5, dxt.data());
    orc_heat_sensitivity(g, cond1, cond2, xt.data(), nodeval.data(), dc.data());
    for(int64_t i = 0; i < nel; i++)
    {
      dc[i] *= dxt[i];
      dv[i] = dxt[i] * vol;
    }
    orc_helmholtz(g, R, dc.data(), t1.data(), 1, 1e-10, &it);
    orc_helmholtz(g, R, dv.data(), t2.data(), 1, 1e-10, &it);
    orc_mma_update(mma, x, t1.data(), &gval, t2.data(), xmin.data(), xmax.data());
  }
  orc_mma_free(mma);
  return 0;
}

// ------------------------------------------------- matrix-free CPU sample ----
/// Jacobi-PCG iterations with a matrix-free element-by-element operator on
/// the host cores (OpenMP over nodes: every node gathers the rows of its <= 8
/// elements, so no two threads write one entry), on full-grid node-major
/// vectors with constrained DOFs held at 0.  For grids whose assembled
/// matrix does not fit in host memory this is the CPU path that can run; it
/// is timed over `nit` iterations from x = 0 with b = the load `fneq` (neq).
/// Returns the seconds of the iterations (set-up excluded); *rr the final
/// ||r||^2.
double orc_ebe_pcg_time(const OrcGrid *g, const uint8_t *fixed, const double *rho,
                        const double *fneq, int nit, double *rr)
{
  const int d = g->dim, ne = nen(*g), nd = d * ne;
  const int64_t nn = numnp(*g), neq = nn * d;
  const int64_t sx = g->nx + 1, sy = g->ny + 1, nx = g->nx, ny = g->ny,
                nz = d == 3 ? g->nz : 1;
  std::vector<double> K0(24 * 24), E(nelx(*g));
  unitK0(*g, K0.data());
  for(int64_t e = 0; e < nelx(*g); e++)
    E[e] = simp(g->young1, g->young2, rho[e], g->penal);
  auto apply = [&](const double *u, double *y) {
#pragma omp parallel for schedule(static)
    for(int64_t n = 0; n < nn; n++)
    {
      const int64_t i = n % sx, j = (n / sx) % sy, k = d == 3 ? n / (sx * sy) : 0;
      double acc[3] = {0, 0, 0};
      for(int dk = (d == 3 ? -1 : 0); dk <= 0; dk++)
        for(int dj = -1; dj <= 0; dj++)
          for(int di = -1; di <= 0; di++)
          {
            const int64_t ei = i + di, ej = j + dj, ek = k + dk;
            if(ei < 0 || ej < 0 || ek < 0 || ei >= nx || ej >= ny || ek >= nz)
              continue;
            const int64_t e = ei + ej * nx + ek * nx * ny;
            int64_t nd8[8];
            elemNodes(*g, e, nd8);
            int ln = 0;
            for(int a = 0; a < ne; a++)
              if(nd8[a] == n)
                ln = a;
            for(int c = 0; c < d; c++)
            {
              double s = 0.0;
              const double *row = &K0[size_t(ln * d + c) * nd];
              for(int b = 0; b < ne; b++)
                for(int c2 = 0; c2 < d; c2++)
                  s += row[b * d + c2] * u[nd8[b] * d + c2];
              acc[c] += E[e] * s;
            }
          }
      for(int c = 0; c < d; c++)
        y[n * d + c] = fixed[n * d + c] ? 0.0 : acc[c];
    }
  };
  std::vector<double> x(neq, 0.0), r(neq), z(neq), p(neq), q(neq), inv(neq, 1.0), ones(neq, 0.0);
  // inverse diagonal from e_i probes would cost neq operator rows; use the
  // per-node diagonal of the element sums
#pragma omp parallel for schedule(static)
  for(int64_t n = 0; n < nn; n++)
  {
    const int64_t i = n % sx, j = (n / sx) % sy, k = d == 3 ? n / (sx * sy) : 0;
    for(int c = 0; c < d; c++)
    {
      double s = 0.0;
      for(int dk = (d == 3 ? -1 : 0); dk <= 0; dk++)
        for(int dj = -1; dj <= 0; dj++)
          for(int di = -1; di <= 0; di++)
          {
            const int64_t ei = i + di, ej = j + dj, ek = k + dk;
            if(ei < 0 || ej < 0 || ek < 0 || ei >= nx || ej >= ny || ek >= nz)
              continue;
            const int64_t e = ei + ej * nx + ek * nx * ny;
            int64_t nd8[8];
            elemNodes(*g, e, nd8);
            for(int a = 0; a < ne; a++)
              if(nd8[a] == n)
                s += E[e] * K0[size_t(a * d + c) * nd + a * d + c];
          }
      inv[n * d + c] = (fixed[n * d + c] || s == 0.0) ? 1.0 : 1.0 / s;
    }
  }
  for(int64_t i = 0; i < neq; i++)
    r[i] = fixed[i] ? 0.0 : fneq[i];
  auto t0 = std::chrono::steady_clock::now();
  for(int64_t i = 0; i < neq; i++)
    p[i] = inv[i] * r[i];
  double absNew = dot(neq, r.data(), p.data()), r2 = 0.0;
  for(int it = 0; it < nit; it++)
  {
    apply(p.data(), q.data());
    const double alpha = absNew / dot(neq, p.data(), q.data());
#pragma omp parallel for schedule(static)
    for(int64_t i = 0; i < neq; i++)
    {
      x[i] += alpha * p[i];
      r[i] -= alpha * q[i];
      z[i] = inv[i] * r[i];
    }
    r2 = dot(neq, r.data(), r.data());
    const double absOld = absNew;
    absNew = dot(neq, r.data(), z.data());
    const double beta = absNew / absOld;
#pragma omp parallel for schedule(static)
    for(int64_t i = 0; i < neq; i++)
      p[i] = z[i] + beta * p[i];
  }
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if(rr)
    *rr = r2;
  return sec;
}

int orc_num_threads()
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

} // extern "C"
