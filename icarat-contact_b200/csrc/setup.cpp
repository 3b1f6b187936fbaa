// setup.cpp -- host-side set-up of a structured SIMP problem: element
// matrices, Dirichlet boxes, DOF numbering and consistent loads.
//
// Element matrices are built in closed form from 1-D integrals of the
// (bi/tri)linear Lagrange basis, which is what the 2x2(x2) Gauss rule of
// Bmatrix::make + LinearElastic::makeKeFint (src/basis/bmatrix.hpp:28-162,
// src/problem/elasticity.cpp:210-254) integrates exactly on a box element.
#include <cmath>
#include <stdexcept>

#include "setup.hpp"

namespace icb
{
namespace
{
/// 1-D integrals on [0,h] of L0 = 1 - x/h, L1 = x/h:
/// M = int La Lb, S = int La' Lb', G = int La' Lb
inline double M1(int a, int b, double h) { return h / 6.0 * (a == b ? 2.0 : 1.0); }
inline double S1(int a, int b, double h) { return (a == b ? 1.0 : -1.0) / h; }
inline double G1(int a, double) { return a ? 0.5 : -0.5; }

/// corner offsets of local node l (meshBox order, bottom face then top face)
inline void corner(int l, int o[3])
{
  int q = l & 3;
  o[0] = (q == 1 || q == 2) ? 1 : 0;
  o[1] = q >= 2 ? 1 : 0;
  o[2] = l >> 2;
}

/// int dN_a/dx_i dN_b/dx_j dV over the box element
double gradInt(int dim, const double *h, int a, int b, int i, int j)
{
  int oa[3], ob[3];
  corner(a, oa);
  corner(b, ob);
  double v = 1.0;
  for(int k = 0; k < dim; k++)
  {
    if(k == i && k == j)
      v *= S1(oa[k], ob[k], h[k]);
    else if(k == i)
      v *= G1(oa[k], h[k]);
    else if(k == j)
      v *= G1(ob[k], h[k]);
    else
      v *= M1(oa[k], ob[k], h[k]);
  }
  return v;
}
} // namespace

/// Lame-type constants of Elastic::De (src/problem/elasticity.cpp:34-98) at
/// E = 1: plane stress uses lambda* = nu/(1-nu^2).
void lame_constants(int state, double nu, double &lam, double &mu)
{
  mu = 1.0 / (2.0 * (1.0 + nu));
  if(state == ICB_PLANE_STRESS)
    lam = nu / (1.0 - nu * nu);
  else
    lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

void heat_element(int dim, const double *h, const double *D, double *K)
{
  int ne = dim == 2 ? 4 : 8;
  for(int a = 0; a < ne; a++)
    for(int b = 0; b < ne; b++)
    {
      double v = 0.0;
      for(int i = 0; i < dim; i++)
        for(int j = 0; j < dim; j++)
          v += D[i * dim + j] * gradInt(dim, h, a, b, i, j);
      K[a * ne + b] = v;
    }
}

void unit_stiffness(int dim, int state, double nu, const double *h, double *K)
{
  double lam, mu;
  lame_constants(state, nu, lam, mu);
  int ne = dim == 2 ? 4 : 8, nd = ne * dim;
  for(int a = 0; a < ne; a++)
    for(int c = 0; c < dim; c++)
      for(int b = 0; b < ne; b++)
        for(int e = 0; e < dim; e++)
        {
          double v = lam * gradInt(dim, h, a, b, c, e) + mu * gradInt(dim, h, a, b, e, c);
          if(c == e)
            for(int k = 0; k < dim; k++)
              v += mu * gradInt(dim, h, a, b, k, k);
          K[(a * dim + c) * nd + b * dim + e] = v;
        }
}

void helmholtz_element(int dim, const double *h, double R, double *Ke, double *Nint)
{
  int ne = dim == 2 ? 4 : 8;
  double re2 = std::pow(R / (2.0 * std::sqrt(3.0)), 2);
  double vol = 1.0;
  for(int k = 0; k < dim; k++)
    vol *= h[k];
  for(int a = 0; a < ne; a++)
  {
    Nint[a] = vol / ne;
    for(int b = 0; b < ne; b++)
    {
      int oa[3], ob[3];
      corner(a, oa);
      corner(b, ob);
      double m = 1.0;
      for(int k = 0; k < dim; k++)
        m *= M1(oa[k], ob[k], h[k]);
      double s = 0.0;
      for(int k = 0; k < dim; k++)
        s += gradInt(dim, h, a, b, k, k);
      Ke[a * ne + b] = m + re2 * s;
    }
  }
}

// ------------------------------------------------------------- HostSetup --
HostSetup::HostSetup(const icb_grid_desc &g) : desc(g)
{
  if(g.dim != 2 && g.dim != 3)
    throw Error{ICB_ERR_BAD_ARG, "dim must be 2 or 3"};
  if(g.nx < 1 || g.ny < 1 || (g.dim == 3 && g.nz < 1))
    throw Error{ICB_ERR_BAD_ARG, "division must be >= 1"};
  if(!(g.lx > 0 && g.ly > 0 && (g.dim == 2 || g.lz > 0)))
    throw Error{ICB_ERR_BAD_ARG, "length must be > 0"};
  const bool heat = g.state == ICB_HEAT;
  if(!heat && g.dim == 3 && g.state != ICB_3D)
    throw Error{ICB_ERR_BAD_ARG, "3D problems need state ICB_3D"};
  if(!heat && g.dim == 2 && g.state != ICB_PLANE_STRESS && g.state != ICB_PLANE_STRAIN)
    throw Error{ICB_ERR_BAD_ARG, "2D problems need plane_stress or plane_strain"};
  if(!heat && !(g.poisson > -1.0 && g.poisson < 0.5))
    throw Error{ICB_ERR_BAD_ARG, "poisson out of range"};
  dofnp = heat ? 1 : g.dim; // mesh_icarat.hpp:77 (probTypeToDofnpVoigt)
  dims = make_dims(g.dim, g.nx, g.ny, g.dim == 3 ? g.nz : 1);
  h[0] = g.lx / g.nx;
  h[1] = g.ly / g.ny;
  h[2] = g.dim == 3 ? g.lz / g.nz : 1.0;
  neq = dims.nnode * dofnp;
  fixed.assign(neq, 0);
  dval.assign(neq, 0.0);
  nodal.assign(neq, 0.0);
  for(double &k : K0)
    k = 0.0;
  if(!heat)
    unit_stiffness(g.dim, g.state, g.poisson, h, K0);
  volume = h[0] * h[1] * (g.dim == 3 ? h[2] : 1.0);
}

void HostSetup::nodeX(long long n, double x[3]) const
{
  long long sx = dims.sx, sy = dims.sy;
  long long i = n % sx, j = (n / sx) % sy, k = n / (sx * sy);
  // MeshIcarat::meshBox coordinates (mesh_icarat.hpp:328-337, 443-456)
  x[0] = (desc.lx / desc.nx) * double(i);
  x[1] = (desc.ly / desc.ny) * double(j);
  x[2] = desc.dim == 3 ? (desc.lz / desc.nz) * double(k) : 0.0;
}

void HostSetup::elemNodes(long long e, long long nd[8]) const
{
  long long sx = dims.sx, sxy = (long long)dims.sx * dims.sy;
  long long i = e % dims.nx, j = (e / dims.nx) % dims.ny, k = e / ((long long)dims.nx * dims.ny);
  long long b = i + j * sx + (desc.dim == 3 ? k * sxy : 0);
  nd[0] = b;
  nd[1] = b + 1;
  nd[2] = b + 1 + sx;
  nd[3] = b + sx;
  if(desc.dim == 3)
    for(int q = 0; q < 4; q++)
      nd[4 + q] = nd[q] + sxy;
}

void HostSetup::dirichletBox(const int *flag, const double *val, const double *range)
{
  if(finalized)
    throw Error{ICB_ERR_STATE, "boundary conditions are frozen after icb_finalize"};
  const double tol = 1.0e-7; // boundary_condition_icarat.hpp:73
  double lo[3] = {range[0] - tol, range[2] - tol, range[4] - tol};
  double hi[3] = {range[1] + tol, range[3] + tol, range[5] + tol};
  const int d = desc.dim, nd = dofnp;
  for(long long n = 0; n < dims.nnode; n++)
  {
    double x[3];
    nodeX(n, x);
    bool in = true;
    for(int c = 0; c < d; c++)
      in = in && x[c] >= lo[c] && x[c] <= hi[c];
    if(!in)
      continue;
    for(int c = 0; c < nd; c++)
    {
      fixed[n * nd + c] = flag[c] != 0;
      dval[n * nd + c] = val[c];
    }
  }
}

void HostSetup::dirichletMask(const unsigned char *f, const double *v)
{
  if(finalized)
    throw Error{ICB_ERR_STATE, "boundary conditions are frozen after icb_finalize"};
  for(long long i = 0; i < neq; i++)
  {
    fixed[i] = f[i] != 0;
    dval[i] = v ? v[i] : 0.0;
  }
}

void HostSetup::tractionBox(const double *val, const double *range)
{
  if(finalized)
    throw Error{ICB_ERR_STATE, "loads are frozen after icb_finalize"};
  Traction t;
  for(int c = 0; c < 3; c++)
    t.val[c] = val[c];
  for(int c = 0; c < 6; c++)
    t.range[c] = range[c];
  tractions.push_back(t);
}

void HostSetup::nodalLoad(long long node, const double *f)
{
  if(finalized)
    throw Error{ICB_ERR_STATE, "loads are frozen after icb_finalize"};
  if(node < 0 || node >= dims.nnode)
    throw Error{ICB_ERR_BAD_ARG, "node index out of range"};
  for(int c = 0; c < dofnp; c++)
    nodal[node * dofnp + c] += f[c];
}

/// countDOF (boundary_condition_base.hpp:35-88) then the loads: nodal loads
/// on free DOFs, and each traction box as generateLoadMain /
/// SurfaceLoad::generate do it (boundary_condition_icarat.hpp:300-385,
/// boundary_condition_base.cpp:16-86, 143-180).
void HostSetup::finalize()
{
  int d = desc.dim;
  dof.assign(neq, 0);
  long long cnt = 0;
  for(long long i = 0; i < neq; i++)
    if(!fixed[i])
      dof[i] = int(cnt++);
  numeq = cnt;
  for(long long i = 0; i < neq; i++)
    if(fixed[i])
      dof[i] = int(cnt++);
  fext.assign(numeq, 0.0);
  for(long long i = 0; i < neq; i++)
    if(!fixed[i])
      fext[dof[i]] += nodal[i];

  static const int q4side[5][2] = {{0, 0}, {0, 1}, {1, 2}, {2, 3}, {3, 0}};
  static const int h8side[7][4] = {{0, 0, 0, 0}, {0, 1, 2, 3}, {3, 0, 4, 7}, {0, 1, 5, 4},
                                   {1, 2, 6, 5}, {2, 3, 7, 6}, {4, 5, 6, 7}};
  const int ne = d == 2 ? 4 : 8, numnode = d == 2 ? 2 : 4;
  for(const Traction &t : tractions)
  {
    const double tol = 1.0e-7;
    double lo[3] = {t.range[0] - tol, t.range[2] - tol, t.range[4] - tol};
    double hi[3] = {t.range[1] + tol, t.range[3] + tol, t.range[5] + tol};
    for(long long e = 0; e < dims.nel; e++)
    {
      long long nd[8];
      elemNodes(e, nd);
      int hit[8], counter = 0;
      for(int k = 0; k < ne; k++)
      {
        double x[3];
        nodeX(nd[k], x);
        bool in = true;
        for(int c = 0; c < d; c++)
          in = in && lo[c] <= x[c] && x[c] <= hi[c];
        if(!in)
          continue;
        hit[counter++] = k;
        if(counter != numnode)
          continue;
        // SurfaceLoad::judgeLine: the side from the local index of the
        // numnode-th hit (boundary_condition_base.cpp:31-76)
        int side;
        if(d == 2)
          side = k == 1 ? 1 : k == 2 ? 2 : (hit[1] - hit[0] == 1 ? 3 : 4);
        else
          side = k == 3 ? 1
                 : k == 5 ? 3
                 : k == 6 ? 4
                 : hit[2] - hit[1] == 1 ? 2
                 : hit[1] - hit[0] == 1 ? 5
                                       : 6;
        // consistent load of a constant traction on the straight side:
        // length/2 per end node (line2, 2 Gauss points) or the Gauss-
        // integrated bilinear-quad share per corner (quad4, 2x2 points)
        int ns = d == 2 ? 2 : 4;
        double share[4];
        long long sn[4];
        for(int s = 0; s < ns; s++)
          sn[s] = nd[d == 2 ? q4side[side][s] : h8side[side][s]];
        if(d == 2)
        {
          double xa[3], xb[3];
          nodeX(sn[0], xa);
          nodeX(sn[1], xb);
          double L = std::sqrt((xb[0] - xa[0]) * (xb[0] - xa[0]) + (xb[1] - xa[1]) * (xb[1] - xa[1]));
          share[0] = share[1] = 0.5 * L;
        }
        else
        {
          double X[4][3];
          for(int s = 0; s < 4; s++)
            nodeX(sn[s], X[s]);
          const double g = 1.0 / std::sqrt(3.0);
          const double gp[4][2] = {{-g, -g}, {g, -g}, {-g, g}, {g, g}};
          for(int s = 0; s < 4; s++)
            share[s] = 0.0;
          for(int q = 0; q < 4; q++)
          {
            double r = gp[q][0], tt = gp[q][1];
            double N[4] = {0.25 * (1 - r) * (1 - tt), 0.25 * (1 + r) * (1 - tt),
                           0.25 * (1 + r) * (1 + tt), 0.25 * (1 - r) * (1 + tt)};
            double dr[4] = {-0.25 * (1 - tt), 0.25 * (1 - tt), 0.25 * (1 + tt), -0.25 * (1 + tt)};
            double ds[4] = {-0.25 * (1 - r), -0.25 * (1 + r), 0.25 * (1 + r), 0.25 * (1 - r)};
            double t1[3] = {0, 0, 0}, t2[3] = {0, 0, 0};
            for(int s = 0; s < 4; s++)
              for(int c = 0; c < 3; c++)
              {
                t1[c] += dr[s] * X[s][c];
                t2[c] += ds[s] * X[s][c];
              }
            double cx = t1[1] * t2[2] - t1[2] * t2[1], cy = t1[2] * t2[0] - t1[0] * t2[2],
                   cz = t1[0] * t2[1] - t1[1] * t2[0];
            double jac = std::sqrt(cx * cx + cy * cy + cz * cz);
            for(int s = 0; s < 4; s++)
              share[s] += N[s] * jac;
          }
        }
        for(int s = 0; s < ns; s++)
          for(int c = 0; c < dofnp; c++)
          {
            long long gi = sn[s] * dofnp + c;
            if(!fixed[gi])
              fext[dof[gi]] += share[s] * t.val[c];
          }
      }
    }
  }
  finalized = true;
}

} // namespace icb
