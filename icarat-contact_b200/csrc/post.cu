// post.cu -- results a TO app writes out after a solve: element stresses
// with their von Mises value, and the nodal reactions.
//
// Elastic::makeMisesStress (src/problem/elasticity.cpp:165-208) averages
// D(E(rho)) B u_e over the element's Gauss points.  On a box element B is
// linear in each natural coordinate, so that average is B at the element
// centre, where dN_a/dx_i = +-1 / (h_i 2^(d-1)) (sign: the side of node a in
// direction i).  The von Mises value is sqrt(s^T V s) with ICARAT's V: in 2D
// s_xx^2 + s_yy^2 - s_xx s_yy + 3 t_xy^2 for plane stress and plane strain
// alike, in 3D the usual six-component form.
#include <cmath>

#include "icb_internal.hpp"
#include "problem.hpp"
#include "setup.hpp"

namespace icb
{
namespace
{
struct MisesParams
{
  double g[3];     ///< 1 / (h_i 2^(d-1))
  double lam, mu;  ///< D at E = 1 (lame_constants)
  double y1, y2, p; ///< SIMP
};

template <int DIM>
__global__ void k_von_mises(const MisesParams P, const Dims d, const double *__restrict__ rho,
                            const double *__restrict__ u, double *__restrict__ mises,
                            double *__restrict__ stress)
{
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= d.nel)
    return;
  constexpr int NE = DIM == 2 ? 4 : 8, V = DIM == 2 ? 3 : 6;
  const int ei = int(e % d.nx), ej = int((e / d.nx) % d.ny);
  const int ek = DIM == 3 ? int(e / ((long long)d.nx * d.ny)) : 0;
  const long long sxy = (long long)d.sx * d.sy;
  const long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
  // grad u at the centre: du_c/dx_i = sum_a G_a,i u_a,c
  double gu[3][3] = {{0, 0, 0}, {0, 0, 0}, {0, 0, 0}};
#pragma unroll
  for(int l = 0; l < NE; l++)
  {
    const int q = l & 3, top = l >> 2;
    const int ox = (q == 1 || q == 2) ? 1 : 0, oy = q >= 2 ? 1 : 0;
    const long long node = base + ox + (long long)oy * d.sx + top * sxy;
    const double G[3] = {ox ? P.g[0] : -P.g[0], oy ? P.g[1] : -P.g[1],
                         top ? P.g[2] : -P.g[2]};
#pragma unroll
    for(int c = 0; c < DIM; c++)
    {
      double v = u[c * d.ld + node];
      v = fabs(v) < 1.0e-15 ? 0.0 : v; // node[].val as divideValIntoNode leaves it
#pragma unroll
      for(int i = 0; i < DIM; i++)
        gu[c][i] = fma(G[i], v, gu[c][i]);
    }
  }
  const double s = rho[e];
  const double E = P.y2 >= P.y1 ? (1.0 - pow(s, P.p)) * P.y1 + pow(s, P.p) * P.y2
                                : pow(1.0 - s, P.p) * P.y1 + (1.0 - pow(1.0 - s, P.p)) * P.y2;
  const double lam = E * P.lam, mu = E * P.mu;
  double sig[V], m2;
  if(DIM == 2)
  {
    const double exx = gu[0][0], eyy = gu[1][1], gxy = gu[0][1] + gu[1][0];
    sig[0] = (lam + 2.0 * mu) * exx + lam * eyy;
    sig[1] = lam * exx + (lam + 2.0 * mu) * eyy;
    sig[2] = mu * gxy;
    m2 = sig[0] * sig[0] + sig[1] * sig[1] - sig[0] * sig[1] + 3.0 * sig[2] * sig[2];
  }
  else
  {
    const double tr = gu[0][0] + gu[1][1] + gu[2][2];
    sig[0] = lam * tr + 2.0 * mu * gu[0][0];
    sig[1] = lam * tr + 2.0 * mu * gu[1][1];
    sig[2] = lam * tr + 2.0 * mu * gu[2][2];
    sig[3] = mu * (gu[0][1] + gu[1][0]);
    sig[4] = mu * (gu[1][2] + gu[2][1]);
    sig[5] = mu * (gu[2][0] + gu[0][2]);
    m2 = sig[0] * sig[0] + sig[1] * sig[1] + sig[2] * sig[2] - sig[0] * sig[1] -
         sig[1] * sig[2] - sig[0] * sig[2] +
         3.0 * (sig[3] * sig[3] + sig[4] * sig[4] + sig[5] * sig[5]);
  }
  mises[e] = sqrt(m2);
  if(stress)
#pragma unroll
    for(int r = 0; r < V; r++)
      stress[e * V + r] = sig[r];
}

/// SoA (c * ld + n) -> node-major (n * dim + c) with ICARAT's zeroing of
/// |r| < 1e-15 (analysis_utility.hpp:47-49)
__global__ void k_soa_to_nodes(const Dims d, const double *__restrict__ a, double *__restrict__ out)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i >= d.nnode * d.dim)
    return;
  const long long n = i / d.dim;
  const int c = int(i - n * d.dim);
  const double v = a[c * d.ld + n];
  out[i] = fabs(v) < 1.0e-15 ? 0.0 : v;
}
} // namespace

void launch_von_mises(const icb_problem_s &p, double *mises, double *stress, cudaStream_t s)
{
  const Dims &d = p.d;
  const icb_grid_desc &g = p.hs->desc;
  MisesParams P{};
  const double two = d.dim == 2 ? 2.0 : 4.0;
  for(int i = 0; i < 3; i++)
    P.g[i] = i < d.dim ? 1.0 / (p.hs->h[i] * two) : 0.0;
  lame_constants(g.state, g.poisson, P.lam, P.mu);
  P.y1 = g.young1;
  P.y2 = g.young2;
  P.p = g.penalty;
  const unsigned nb = unsigned((d.nel + 127) / 128);
  if(d.dim == 3)
    k_von_mises<3><<<nb, 128, 0, s>>>(P, d, p.rho.p, p.u.p, mises, stress);
  else
    k_von_mises<2><<<nb, 128, 0, s>>>(P, d, p.rho.p, p.u.p, mises, stress);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

void launch_reactions(icb_problem_s &p, double *out, cudaStream_t s)
{
  const Dims &d = p.d;
  if(!p.work2.p)
    p.work2.alloc(p.nsoa);
  if(!p.fixNone.p)
  {
    p.fixNone.alloc(d.nnode);
    ICB_CUDA(cudaMemsetAsync(p.fixNone.p, 0, d.nnode, s));
  }
  // the operator without the Dirichlet mask: K_full u at every DOF
  launch_matvec<double>(d, p.K0, p.E.p, p.u.p, p.work2.p, p.fixNone.p, s);
  const long long n = d.nnode * d.dim;
  k_soa_to_nodes<<<unsigned((n + 255) / 256), 256, 0, s>>>(d, p.work2.p, out);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

} // namespace icb
