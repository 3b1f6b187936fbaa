// helm.cu -- Helmholtz PDE filter on the device.
//
// FilterHelmholtz::densityFilter (src/optimization/filter_helm.hpp:75-137,
// 178-256): (M + re^2 K_grad) phi = F with re = R / (2 sqrt 3), assembled
// over all nodes without constraints, solved with the Eigen_CG semantics
// (Jacobi-PCG, x0 = 0, Solvers' default tolerance 1e-10); the element value
// is the Gauss average of N.phi.  On a box element sum_q N_a(q) = 1 for every
// node a, so the Gauss average is the mean of the element's nodal values and
// the load integral int N_a is V/ne.  The adjoint (sensFlag) divides the
// load by ne instead and sums instead of averaging, exactly as ICARAT does.
// The operator is matrix-free: a node gathers its <= 8 elements' rows of the
// 4x4 / 8x8 element matrix.
#include <algorithm>
#include <cmath>

#include "helm.hpp"
#include "reduce.cuh"
#include "setup.hpp"

namespace icb
{
namespace
{
constexpr int VB = 256;
inline int vblocks(long long n)
{
  return int(std::max<long long>(1, std::min<long long>((n + VB - 1) / VB, num_sms() * 8LL)));
}

__device__ __forceinline__ int lnode(int a, int b) { return (a ^ b) + 2 * b; }

template <int DIM, bool DOT>
__global__ void k_helm_apply(KMat<double, 8> K, Dims d, const double *__restrict__ u,
                             double *__restrict__ y, RedScratch red, double *dotOut,
                             const KState *gate)
{
  if(gate && gate->stop)
    return;
  double dot = 0.0;
  const long long sxy = (long long)d.sx * d.sy;
  constexpr int NE = DIM == 2 ? 4 : 8;
  for(long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < d.nnode;
      n += (long long)gridDim.x * blockDim.x)
  {
    int i = int(n % d.sx), j = int((n / d.sx) % d.sy), k = DIM == 3 ? int(n / sxy) : 0;
    double s = 0.0;
    for(int dk = (DIM == 3 ? -1 : 0); dk <= 0; dk++)
      for(int dj = -1; dj <= 0; dj++)
        for(int di = -1; di <= 0; di++)
        {
          int ei = i + di, ej = j + dj, ek = k + dk;
          if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (DIM == 3 && ek >= d.nz))
            continue;
          int ln = lnode(-di, -dj) + (DIM == 3 ? 4 * (-dk) : 0);
          long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
#pragma unroll
          for(int lm = 0; lm < NE; lm++)
          {
            int q = lm & 3, top = lm >> 2;
            long long m = base + ((q == 1 || q == 2) ? 1 : 0) + (q >= 2 ? d.sx : 0) + top * sxy;
            s += K.k[ln * NE + lm] * u[m];
          }
        }
    y[n] = s;
    if(DOT)
      dot += u[n] * s;
  }
  if(DOT)
  {
    double v[1] = {dot};
    block_reduce<1>(v, red, FinStore{dotOut});
  }
}

template <int DIM>
__global__ void k_helm_diag(KMat<double, 8> K, Dims d, double *__restrict__ dinv)
{
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(n >= d.nnode)
    return;
  constexpr int NE = DIM == 2 ? 4 : 8;
  const long long sxy = (long long)d.sx * d.sy;
  int i = int(n % d.sx), j = int((n / d.sx) % d.sy), k = DIM == 3 ? int(n / sxy) : 0;
  double s = 0.0;
  for(int dk = (DIM == 3 ? -1 : 0); dk <= 0; dk++)
    for(int dj = -1; dj <= 0; dj++)
      for(int di = -1; di <= 0; di++)
      {
        int ei = i + di, ej = j + dj, ek = k + dk;
        if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (DIM == 3 && ek >= d.nz))
          continue;
        int ln = lnode(-di, -dj) + (DIM == 3 ? 4 * (-dk) : 0);
        s += K.k[ln * NE + ln];
      }
  dinv[n] = s != 0.0 ? 1.0 / s : 1.0;
}

/// F_n = sum over the node's elements of x_e int N (/ ne for the adjoint)
template <int DIM>
__global__ void k_helm_rhs(Dims d, const double *__restrict__ x, double w, double *__restrict__ F)
{
  long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(n >= d.ld)
    return;
  if(n >= d.nnode)
  {
    F[n] = 0.0;
    return;
  }
  const long long sxy = (long long)d.sx * d.sy;
  int i = int(n % d.sx), j = int((n / d.sx) % d.sy), k = DIM == 3 ? int(n / sxy) : 0;
  double s = 0.0;
  for(int dk = (DIM == 3 ? -1 : 0); dk <= 0; dk++)
    for(int dj = -1; dj <= 0; dj++)
      for(int di = -1; di <= 0; di++)
      {
        int ei = i + di, ej = j + dj, ek = k + dk;
        if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (DIM == 3 && ek >= d.nz))
          continue;
        s += x[ei + (long long)ej * d.nx + (long long)ek * d.nx * d.ny];
      }
  F[n] = s * w;
}

/// element value: w * sum of the element's nodal values
template <int DIM>
__global__ void k_helm_out(Dims d, const double *__restrict__ phi, double w, double *__restrict__ out)
{
  long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= d.nel)
    return;
  int ei = int(e % d.nx), ej = int((e / d.nx) % d.ny), ek = int(e / ((long long)d.nx * d.ny));
  const long long sxy = (long long)d.sx * d.sy;
  long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
  double s = phi[base] + phi[base + 1] + phi[base + 1 + d.sx] + phi[base + d.sx];
  if(DIM == 3)
    s += phi[base + sxy] + phi[base + 1 + sxy] + phi[base + 1 + d.sx + sxy] + phi[base + d.sx + sxy];
  out[e] = w * s;
}
} // namespace

HelmFilter::HelmFilter(const Dims &dims, const double *h, double R, cudaStream_t s)
    : d(dims), radius(R)
{
  if(!(R > 0.0))
    throw Error{ICB_ERR_BAD_ARG, "Helmholtz filter radius must be > 0"};
  double Ke[64], Nint[8];
  helmholtz_element(d.dim, h, R, Ke, Nint);
  ne = d.dim == 2 ? 4 : 8;
  for(int i = 0; i < ne * ne; i++)
    K.k[i] = Ke[i];
  nint = Nint[0];
  Dims sd = d;
  sd.dim = 1; // a scalar field on the same nodes: vectors of ld entries
  pcg = std::make_unique<JacobiPcg<double>>(sd, s);
  dinv.alloc(d.ld);
  rhs.alloc(d.ld);
  phi.alloc(d.ld);
  ICB_CUDA(cudaMemsetAsync(dinv.p, 0, dinv.bytes(), s));
  ICB_CUDA(cudaMemsetAsync(rhs.p, 0, rhs.bytes(), s));
  ICB_CUDA(cudaMemsetAsync(phi.p, 0, phi.bytes(), s));
  unsigned nb = unsigned((d.nnode + 255) / 256);
  if(d.dim == 3)
    k_helm_diag<3><<<nb, 256, 0, s>>>(K, d, dinv.p);
  else
    k_helm_diag<2><<<nb, 256, 0, s>>>(K, d, dinv.p);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

int HelmFilter::apply(const double *in, double *out, bool sens, double tol, cudaStream_t s,
                      icb_solve_info *info)
{
  unsigned nbn = unsigned((d.ld + 255) / 256), nbe = unsigned((d.nel + 255) / 256);
  double wr = sens ? nint / ne : nint;
  if(d.dim == 3)
    k_helm_rhs<3><<<nbn, 256, 0, s>>>(d, in, wr, rhs.p);
  else
    k_helm_rhs<2><<<nbn, 256, 0, s>>>(d, in, wr, rhs.p);
  count_launch();
  JacobiPcg<double> &P = *pcg;
  const Dims dd = d;
  const KMat<double, 8> KK = K;
  double *pp = P.p.p, *qp = P.q.p, *dp = P.dots.p;
  KState *sp = P.st.p;
  RedScratch *rp = &P.red;
  const int nb = vblocks(d.nnode);
  auto op = [=](cudaStream_t cs) {
    if(dd.dim == 3)
      k_helm_apply<3, true><<<nb, VB, 0, cs>>>(KK, dd, pp, qp, *rp, dp, sp);
    else
      k_helm_apply<2, true><<<nb, VB, 0, cs>>>(KK, dd, pp, qp, *rp, dp, sp);
    count_launch();
  };
  int st = P.solveOp(op, this, nullptr, nullptr, dinv.p, rhs.p, phi.p, tol, 10000, s, info);
  double wo = sens ? 1.0 : 1.0 / ne;
  if(d.dim == 3)
    k_helm_out<3><<<nbe, 256, 0, s>>>(d, phi.p, wo, out);
  else
    k_helm_out<2><<<nbe, 256, 0, s>>>(d, phi.p, wo, out);
  ICB_CUDA(cudaGetLastError());
  count_launch();
  return st;
}

} // namespace icb
