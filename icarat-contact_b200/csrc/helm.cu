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

/// 1-D assembled mass and stiffness stencils of one axis: off-diagonals h/6
/// and -1/h, diagonal h/3 and 1/h per element beside the node
struct HelmAxis
{
  double mo, mh, so, sh;
};
struct HelmTensor
{
  HelmAxis a[3];
  double re2;
};

/// The 3D Helmholtz operator as a tensor-product stencil.  On the box grid
/// the assembled M + re^2 K_grad is Mx.My.Mz + re^2 (Sx.My.Mz + Mx.Sy.Mz +
/// Mx.My.Sz) with the 1-D assembled mass / stiffness matrices of each axis
/// (boundary nodes have half the diagonal), so per node
///   y = Mz o H + re^2 Sz o G,  G = My o (Mx o u),
///   H = G + re^2 (My o (Sx o u) + Sy o (Mx o u)),
/// where "o" applies the 3-point 1-D stencil along that axis.  A CTA owns a
/// 32 x 8 node tile and marches up a chunk of z planes: each plane (with a
/// one-node halo, zero outside the grid) goes through shared memory once,
/// the in-plane sums G and H are formed there, and a 3-plane window of them
/// in registers gives the output one plane behind.  No index division, no
/// element loop; results equal the element gather up to summation order.
constexpr int HTX = 32, HTY = 8;
template <bool DOT>
__global__ void __launch_bounds__(HTX *HTY)
    k_helm_apply3(const HelmTensor C, const Dims d, const int zchunk,
                  const double *__restrict__ u, double *__restrict__ y, RedScratch red,
                  double *dotOut, const KState *gate)
{
  if(gate && gate->stop)
    return;
  constexpr int NX = HTX + 2, NY = HTY + 2, NP = NX * NY, NT = HTX * HTY;
  __shared__ double sP[2][NY][NX];
  const int lx = threadIdx.x, ly = threadIdx.y, tid = ly * HTX + lx;
  const int X0 = blockIdx.x * HTX, Y0 = blockIdx.y * HTY;
  const int i = X0 + lx, j = Y0 + ly;
  const int Z0 = blockIdx.z * zchunk, Z1 = min(Z0 + zchunk, d.sz) - 1;
  const long long sxy = (long long)d.sx * d.sy;
  // this thread's (at most two) values of each staged plane
  long long off[2];
  bool ok[2];
#pragma unroll
  for(int t = 0; t < 2; t++)
  {
    const int q = tid + t * NT;
    const int gi = X0 - 1 + q % NX, gj = Y0 - 1 + q / NX;
    ok[t] = q < NP && gi >= 0 && gi < d.sx && gj >= 0 && gj < d.sy;
    off[t] = ok[t] ? gi + (long long)gj * d.sx : 0;
  }
  auto fetch = [&](int k, double (&v)[2]) {
    const bool kin = k >= 0 && k < d.sz;
#pragma unroll
    for(int t = 0; t < 2; t++)
      v[t] = kin && ok[t] ? __ldg(u + off[t] + k * sxy) : 0.0;
  };
  // in-plane diagonals at this node (half per element beside it)
  const HelmAxis &ax = C.a[0], &ay = C.a[1], &az = C.a[2];
  const double mdx = (i > 0 ? ax.mh : 0.0) + (i < d.sx - 1 ? ax.mh : 0.0);
  const double sdx = (i > 0 ? ax.sh : 0.0) + (i < d.sx - 1 ? ax.sh : 0.0);
  const double mdy = (j > 0 ? ay.mh : 0.0) + (j < d.sy - 1 ? ay.mh : 0.0);
  const double sdy = (j > 0 ? ay.sh : 0.0) + (j < d.sy - 1 ? ay.sh : 0.0);
  const bool own = i < d.sx && j < d.sy;
  // window: G, H of planes k-2 and k-1 (the plane output at step k), and
  // u at this node of plane k-1 (for the fused dot product)
  double Gm = 0.0, Hm = 0.0, G0 = 0.0, H0 = 0.0, U0 = 0.0;
  double dot = 0.0;
  // plane k's values (v) and plane k+1's (w) are in flight: loads are issued
  // two planes ahead of their use
  double v[2], w[2];
  fetch(Z0 - 1, v);
  fetch(Z0, w);
  for(int k = Z0 - 1; k <= Z1 + 1; ++k)
  {
    const int b = k & 1;
#pragma unroll
    for(int t = 0; t < 2; t++)
    {
      if(tid + t * NT < NP)
        (&sP[b][0][0])[tid + t * NT] = v[t];
      v[t] = w[t];
    }
    __syncthreads();
    if(k + 2 <= Z1 + 1)
      fetch(k + 2, w);
    // in-plane sums of plane k at this node
    double mx[3], sx[3];
#pragma unroll
    for(int r = 0; r < 3; r++)
    {
      const double c = sP[b][ly + r][lx + 1], e = sP[b][ly + r][lx] + sP[b][ly + r][lx + 2];
      mx[r] = fma(mdx, c, ax.mo * e);
      sx[r] = fma(sdx, c, ax.so * e);
    }
    const double U1 = sP[b][ly + 1][lx + 1];
    const double G1 = fma(mdy, mx[1], ay.mo * (mx[0] + mx[2]));
    const double H1 =
        G1 + C.re2 * (fma(mdy, sx[1], ay.mo * (sx[0] + sx[2])) + fma(sdy, mx[1], ay.so * (mx[0] + mx[2])));
    // plane k-1 is complete: output it
    const int ko = k - 1;
    if(ko >= Z0 && ko <= Z1 && own)
    {
      const double mdz = (ko > 0 ? az.mh : 0.0) + (ko < d.sz - 1 ? az.mh : 0.0);
      const double sdz = (ko > 0 ? az.sh : 0.0) + (ko < d.sz - 1 ? az.sh : 0.0);
      const double out = fma(mdz, H0, az.mo * (Hm + H1)) +
                         C.re2 * fma(sdz, G0, az.so * (Gm + G1));
      const long long n = i + (long long)j * d.sx + ko * sxy;
      y[n] = out;
      if(DOT)
        dot += U0 * out;
    }
    Gm = G0;
    Hm = H0;
    G0 = G1;
    H0 = H1;
    U0 = U1;
  }
  if(DOT)
  {
    double vv[1] = {dot};
    block_reduce<1>(vv, red, FinStore{dotOut});
  }
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
  for(int k = 0; k < d.dim; k++)
    this->h[k] = h[k];
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
  // 3D: the tensor-product stencil kernel, z split so that the CTAs fill
  // the GPU about four times over within the reduction scratch
  HelmTensor T{};
  T.re2 = std::pow(radius / (2.0 * std::sqrt(3.0)), 2);
  for(int k = 0; k < 3; k++)
  {
    const double hk = k < d.dim ? h[k] : 1.0;
    T.a[k] = HelmAxis{hk / 6.0, hk / 3.0, -1.0 / hk, 1.0 / hk};
  }
  const int tx = (d.sx + HTX - 1) / HTX, ty = (d.sy + HTY - 1) / HTY;
  const long long tiles = (long long)tx * ty;
  // planes per CTA: fewest rounds x (planes + 2) for the CTAs resident at once
  // (a CTA also stages the planes just below and above its chunk), within the
  // reduction scratch
  int per = 0;
  if(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_helm_apply3<true>, HTX * HTY, 0) !=
         cudaSuccess ||
     per < 1)
  {
    (void)cudaGetLastError();
    per = 1;
  }
  const long long resident = (long long)per * num_sms();
  int zc = d.sz;
  long long best = -1;
  for(int bzt = 1; bzt <= d.sz; bzt++)
  {
    const int z = (d.sz + bzt - 1) / bzt;
    const long long nb3 = tiles * ((d.sz + z - 1) / z);
    if(nb3 > P.red.maxBlocks)
      break;
    const long long cost = (nb3 + resident - 1) / resident * (z + 2);
    if(best < 0 || cost < best)
    {
      best = cost;
      zc = z;
    }
  }
  int bz = (d.sz + zc - 1) / zc;
  const bool tensor = d.dim == 3 && tiles * bz <= P.red.maxBlocks;
  const dim3 tgrid(tx, ty, bz), tblock(HTX, HTY);
  auto op = [=](cudaStream_t cs) {
    if(tensor)
      k_helm_apply3<true><<<tgrid, tblock, 0, cs>>>(T, dd, zc, pp, qp, *rp, dp, sp);
    else if(dd.dim == 3)
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
