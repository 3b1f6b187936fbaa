// heat.cu -- steady heat conduction with SIMP conductivity on the device
// (ICARAT's LinearHeat, src/problem/heat.{hpp,cpp}, and the opt-heat app,
// opt-heat/opt_heat.cpp).
//
// One temperature per node.  The element matrix is
//   Ke(rho) = rho^p K1 + (1 - rho^p) K2,  K_m = int grad N^T D_m grad N,
// D_m the conductivity tensor of material m (heat.cpp:53-64).  The operator
// is matrix-free: a node gathers its <= 8 elements' rows of K1 and K2, each
// weighted by the element's rho^p or 1 - rho^p.  Constrained temperatures
// are eliminated as in elasticity (fres = f - K_fd T_d, rows and columns of
// constrained nodes dropped).  The solve is the Eigen_CG drop-in Jacobi-PCG.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>
#include <memory>

#include "helm.hpp"
#include "krylov.hpp"
#include "opt.hpp"
#include "problem.hpp"
#include "reduce.cuh"
#include "setup.hpp"

using namespace icb;

struct icb_heat_s
{
  icb_ctx ctx = nullptr;
  icb_heat_desc desc{};
  std::unique_ptr<HostSetup> hs;
  Dims d;
  KMat<double, 8> K1{}, K2{};
  DevBuf<uint8_t> fix;
  DevBuf<double> a, f, uD, u, x, b, dinv, work, dc;
  std::unique_ptr<JacobiPcg<double>> pcg;
  bool finalized = false, hasDensity = false, solved = false;
  cudaStream_t stream() const { return ctx->stream; }
};

namespace
{
constexpr int VB = 256;
inline int vblocks(long long n)
{
  return int(std::max<long long>(1, std::min<long long>((n + VB - 1) / VB, num_sms() * 8LL)));
}

__device__ __forceinline__ int lnodeH(int a, int b) { return (a ^ b) + 2 * b; }

/// y_n = sum over the node's elements of (a_e K1 + (1 - a_e) K2) u_e rows,
/// 0 on constrained nodes; with DOT the partial of u . y
template <int DIM, bool DOT>
__global__ void k_heat_apply(KMat<double, 8> K1, KMat<double, 8> K2, Dims d,
                             const double *__restrict__ a, const uint8_t *__restrict__ fix,
                             const double *__restrict__ u, double *__restrict__ y,
                             RedScratch red, double *dotOut, const KState *gate)
{
  if(gate && gate->stop)
    return;
  double dot = 0.0;
  const long long sxy = (long long)d.sx * d.sy;
  constexpr int NE = DIM == 2 ? 4 : 8;
  for(long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x; n < d.nnode;
      n += (long long)gridDim.x * blockDim.x)
  {
    double s = 0.0;
    if(!fix[n])
    {
      const int i = int(n % d.sx), j = int((n / d.sx) % d.sy), k = DIM == 3 ? int(n / sxy) : 0;
      for(int dk = (DIM == 3 ? -1 : 0); dk <= 0; dk++)
        for(int dj = -1; dj <= 0; dj++)
          for(int di = -1; di <= 0; di++)
          {
            const int ei = i + di, ej = j + dj, ek = k + dk;
            if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (DIM == 3 && ek >= d.nz))
              continue;
            const int ln = lnodeH(-di, -dj) + (DIM == 3 ? 4 * (-dk) : 0);
            const long long e = ei + (long long)ej * d.nx + (long long)ek * d.nx * d.ny;
            const double w1 = a[e], w2 = 1.0 - w1;
            const long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
#pragma unroll
            for(int lm = 0; lm < NE; lm++)
            {
              const int q = lm & 3, top = lm >> 2;
              const long long m = base + ((q == 1 || q == 2) ? 1 : 0) + (q >= 2 ? d.sx : 0) + top * sxy;
              s += (w1 * K1.k[ln * NE + lm] + w2 * K2.k[ln * NE + lm]) * u[m];
            }
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

/// inverse diagonal of the free rows (1 on constrained nodes and where 0)
template <int DIM>
__global__ void k_heat_dinv(KMat<double, 8> K1, KMat<double, 8> K2, Dims d,
                            const double *__restrict__ a, const uint8_t *__restrict__ fix,
                            double *__restrict__ dinv)
{
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(n >= d.ld)
    return;
  if(n >= d.nnode || fix[n])
  {
    dinv[n] = n < d.nnode ? 1.0 : 0.0;
    return;
  }
  constexpr int NE = DIM == 2 ? 4 : 8;
  const long long sxy = (long long)d.sx * d.sy;
  const int i = int(n % d.sx), j = int((n / d.sx) % d.sy), k = DIM == 3 ? int(n / sxy) : 0;
  double s = 0.0;
  for(int dk = (DIM == 3 ? -1 : 0); dk <= 0; dk++)
    for(int dj = -1; dj <= 0; dj++)
      for(int di = -1; di <= 0; di++)
      {
        const int ei = i + di, ej = j + dj, ek = k + dk;
        if(ei < 0 || ej < 0 || ek < 0 || ei >= d.nx || ej >= d.ny || (DIM == 3 && ek >= d.nz))
          continue;
        const int ln = lnodeH(-di, -dj) + (DIM == 3 ? 4 * (-dk) : 0);
        const double w1 = a[ei + (long long)ej * d.nx + (long long)ek * d.nx * d.ny];
        s += w1 * K1.k[ln * NE + ln] + (1.0 - w1) * K2.k[ln * NE + ln];
      }
  dinv[n] = s != 0.0 ? 1.0 / s : 1.0;
}

__global__ void k_heat_simp(long long n, const double *__restrict__ rho, double p,
                            double *__restrict__ a)
{
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e < n)
    a[e] = pow(rho[e], p);
}

/// b = f - y on free nodes, 0 on constrained ones (y = K_fd T_d)
__global__ void k_heat_rhs(Dims d, const uint8_t *__restrict__ fix, const double *__restrict__ f,
                           const double *__restrict__ y, double *__restrict__ b)
{
  const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(n >= d.ld)
    return;
  b[n] = (n < d.nnode && !fix[n]) ? f[n] - y[n] : 0.0;
}

/// dc_e = -u_e^T (p rho^(p-1) (K1 - K2)) u_e (opt_heat.cpp:155-190 without
/// the threshold factor); u_e as node[].val leaves it (|T| < 1e-15 -> 0)
template <int DIM>
__global__ void k_heat_sens(KMat<double, 8> K1, KMat<double, 8> K2, Dims d,
                            const double *__restrict__ rho, double p,
                            const double *__restrict__ u, double *__restrict__ dc)
{
  const long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(e >= d.nel)
    return;
  constexpr int NE = DIM == 2 ? 4 : 8;
  const int ei = int(e % d.nx), ej = int((e / d.nx) % d.ny);
  const int ek = DIM == 3 ? int(e / ((long long)d.nx * d.ny)) : 0;
  const long long sxy = (long long)d.sx * d.sy;
  const long long base = ei + (long long)ej * d.sx + (long long)ek * sxy;
  double ue[NE];
#pragma unroll
  for(int l = 0; l < NE; l++)
  {
    const int q = l & 3, top = l >> 2;
    const double v = u[base + ((q == 1 || q == 2) ? 1 : 0) + (q >= 2 ? d.sx : 0) + top * sxy];
    ue[l] = fabs(v) < 1.0e-15 ? 0.0 : v;
  }
  double s = 0.0;
#pragma unroll
  for(int i = 0; i < NE; i++)
  {
    double t = 0.0;
#pragma unroll
    for(int j = 0; j < NE; j++)
      t += (K1.k[i * NE + j] - K2.k[i * NE + j]) * ue[j];
    s += ue[i] * t;
  }
  dc[e] = -p * pow(rho[e], p - 1.0) * s;
}

void condTensor(int dim, const double *c, double *D)
{
  if(dim == 2)
  {
    D[0] = c[0];
    D[1] = c[3];
    D[2] = c[3];
    D[3] = c[1];
    return;
  }
  const double v[9] = {c[0], c[3], c[5], c[3], c[1], c[4], c[5], c[4], c[2]};
  for(int i = 0; i < 9; i++)
    D[i] = v[i];
}

unsigned nb256(long long n) { return unsigned((n + 255) / 256); }

void heatOp(const icb_heat_s &H, const double *u, double *y, RedScratch red, double *dotOut,
            const KState *gate, cudaStream_t s)
{
  const int nb = vblocks(H.d.nnode);
  if(H.desc.dim == 3) // H.d.dim is 1: one value per node
  {
    if(dotOut)
      k_heat_apply<3, true><<<nb, VB, 0, s>>>(H.K1, H.K2, H.d, H.a.p, H.fix.p, u, y, red, dotOut, gate);
    else
      k_heat_apply<3, false><<<nb, VB, 0, s>>>(H.K1, H.K2, H.d, H.a.p, H.fix.p, u, y, red, dotOut, gate);
  }
  else
  {
    if(dotOut)
      k_heat_apply<2, true><<<nb, VB, 0, s>>>(H.K1, H.K2, H.d, H.a.p, H.fix.p, u, y, red, dotOut, gate);
    else
      k_heat_apply<2, false><<<nb, VB, 0, s>>>(H.K1, H.K2, H.d, H.a.p, H.fix.p, u, y, red, dotOut, gate);
  }
  count_launch();
}

void needH(icb_heat h, bool final)
{
  if(!h)
    throw Error{ICB_ERR_BAD_ARG, "NULL heat problem"};
  if(final && !h->finalized)
    throw Error{ICB_ERR_STATE, "call icb_heat_finalize first"};
}

void solveHeat(icb_heat_s &H, const icb_solve_opts *opts, icb_solve_info *info)
{
  NvtxRange range("heat solve");
  cudaStream_t s = H.stream();
  const Dims &d = H.d;
  const double tol = opts ? opts->tol : 1e-10;
  const int maxit = opts ? opts->maxit : 10000;
  if(opts && (opts->precision != ICB_FP64 || opts->precond != ICB_PRECOND_JACOBI))
    throw Error{ICB_ERR_BAD_ARG, "heat problems solve with FP64 Jacobi-PCG"};
  // fres = f - K_fd T_d (LinearAnalysis::solve with fint of the Dirichlet values)
  heatOp(H, H.uD.p, H.work.p, RedScratch{}, nullptr, nullptr, s);
  k_heat_rhs<<<nb256(d.ld), 256, 0, s>>>(d, H.fix.p, H.f.p, H.work.p, H.b.p);
  if(H.desc.dim == 3)
    k_heat_dinv<3><<<nb256(d.ld), 256, 0, s>>>(H.K1, H.K2, d, H.a.p, H.fix.p, H.dinv.p);
  else
    k_heat_dinv<2><<<nb256(d.ld), 256, 0, s>>>(H.K1, H.K2, d, H.a.p, H.fix.p, H.dinv.p);
  count_launch(2);
  ICB_CUDA(cudaGetLastError());
  JacobiPcg<double> &P = *H.pcg;
  double *pp = P.p.p, *qp = P.q.p, *dp = P.dots.p;
  KState *sp = P.st.p;
  RedScratch *rp = &P.red;
  const icb_heat_s *hp = &H;
  auto op = [=](cudaStream_t cs) { heatOp(*hp, pp, qp, *rp, dp, sp, cs); };
  icb_solve_info inf{};
  int st = P.solveOp(op, &H, H.a.p, nullptr, H.dinv.p, H.b.p, H.x.p, tol, maxit, s, &inf);
  launch_add(d.ld, H.x.p, H.uD.p, H.u.p, s);
  ICB_CUDA(cudaStreamSynchronize(s));
  H.solved = true;
  if(info)
    *info = inf;
  if(st != ICB_OK && st != ICB_ERR_MAXITER)
    throw Error{st, "heat solve failed"};
  if(info)
    info->status = st;
}

double heatObjective(icb_heat_s &H)
{
  // u_f^T K_ff u_f (opt_heat.cpp:116): the operator on the free part x
  cudaStream_t s = H.stream();
  JacobiPcg<double> &P = *H.pcg;
  heatOp(H, H.x.p, H.work.p, P.red, P.dots.p, nullptr, s);
  double v;
  ICB_CUDA(cudaMemcpyAsync(&v, P.dots.p, sizeof(double), cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  // the DOT variant sums x . (K x) over all nodes; x is 0 on constrained ones
  return v;
}

void heatSensDevice(icb_heat_s &H, const double *rho, double *dc, cudaStream_t s)
{
  if(H.desc.dim == 3)
    k_heat_sens<3><<<nb256(H.d.nel), 256, 0, s>>>(H.K1, H.K2, H.d, rho, H.desc.penalty, H.u.p, dc);
  else
    k_heat_sens<2><<<nb256(H.d.nel), 256, 0, s>>>(H.K1, H.K2, H.d, rho, H.desc.penalty, H.u.p, dc);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}

__global__ void k_mul(long long n, double *__restrict__ a, const double *__restrict__ m, double s)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < n)
    a[i] = s * a[i] * m[i];
}
__global__ void k_fill(long long n, double v, double *__restrict__ a)
{
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < n)
    a[i] = v;
}
} // namespace

extern "C" {

int icb_heat_create(icb_ctx ctx, const icb_heat_desc *desc, icb_heat *out)
{
  ICB_API_BEGIN
  if(!ctx || !desc || !out)
    throw Error{ICB_ERR_BAD_ARG, "NULL argument"};
  if(desc->cond1[0] < desc->cond2[0])
    throw Error{ICB_ERR_BAD_ARG, "the thermal conductivity of material 1 must not be below that "
                                 "of material 2 (heat.cpp:56-61)"};
  ICB_CUDA(cudaSetDevice(ctx->device));
  auto H = std::make_unique<icb_heat_s>();
  H->ctx = ctx;
  H->desc = *desc;
  icb_grid_desc g{};
  g.dim = desc->dim;
  g.nx = desc->nx;
  g.ny = desc->ny;
  g.nz = desc->dim == 3 ? desc->nz : 1;
  g.lx = desc->lx;
  g.ly = desc->ly;
  g.lz = desc->dim == 3 ? desc->lz : 1.0;
  g.state = ICB_HEAT;
  g.young1 = 0.0;
  g.young2 = 1.0;
  g.poisson = 0.0;
  g.penalty = desc->penalty;
  H->hs = std::make_unique<HostSetup>(g);
  H->d = H->hs->dims;
  H->d.dim = 1; // one component per node: vectors of ld entries
  double D1[9], D2[9], k1[64], k2[64];
  condTensor(desc->dim, desc->cond1, D1);
  condTensor(desc->dim, desc->cond2, D2);
  heat_element(desc->dim, H->hs->h, D1, k1);
  heat_element(desc->dim, H->hs->h, D2, k2);
  const int ne = desc->dim == 2 ? 4 : 8;
  for(int i = 0; i < ne * ne; i++)
  {
    H->K1.k[i] = k1[i];
    H->K2.k[i] = k2[i];
  }
  ctx->refs++;
  *out = H.release();
  ICB_API_END
}

int icb_heat_destroy(icb_heat h)
{
  ICB_API_BEGIN
  if(!h)
    return ICB_OK;
  icb_ctx c = h->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete h;
  icb_ctx_destroy(c);
  ICB_API_END
}

int icb_heat_dirichlet_box(icb_heat h, int flag, double val, const double *range)
{
  ICB_API_BEGIN
  needH(h, false);
  if(!range)
    throw Error{ICB_ERR_BAD_ARG, "NULL range"};
  const int f[6] = {flag, 0, 0, 0, 0, 0};
  const double v[6] = {val, 0, 0, 0, 0, 0};
  h->hs->dirichletBox(f, v, range);
  ICB_API_END
}

int icb_heat_flux_box(icb_heat h, double q, const double *range)
{
  ICB_API_BEGIN
  needH(h, false);
  if(!range)
    throw Error{ICB_ERR_BAD_ARG, "NULL range"};
  const double v[3] = {q, 0, 0};
  h->hs->tractionBox(v, range);
  ICB_API_END
}

int icb_heat_nodal_source(icb_heat h, long long node, double q)
{
  ICB_API_BEGIN
  needH(h, false);
  h->hs->nodalLoad(node, &q);
  ICB_API_END
}

int icb_heat_finalize(icb_heat h, long long *numeq)
{
  ICB_API_BEGIN
  needH(h, false);
  if(h->finalized)
    throw Error{ICB_ERR_STATE, "icb_heat_finalize called twice"};
  ICB_CUDA(cudaSetDevice(h->ctx->device));
  HostSetup &hs = *h->hs;
  hs.finalize();
  const Dims &d = h->d;
  cudaStream_t s = h->stream();
  std::vector<uint8_t> mask(d.nnode);
  std::vector<double> f(d.ld, 0.0), ud(d.ld, 0.0);
  for(long long n = 0; n < d.nnode; n++)
  {
    mask[n] = hs.fixed[n] ? 1 : 0;
    if(hs.fixed[n])
      ud[n] = hs.dval[n];
    else
      f[n] = hs.fext[hs.dof[n]];
  }
  h->fix.alloc(d.nnode);
  for(DevBuf<double> *b : {&h->f, &h->uD, &h->u, &h->x, &h->b, &h->dinv, &h->work})
  {
    b->alloc(d.ld);
    ICB_CUDA(cudaMemsetAsync(b->p, 0, b->bytes(), s));
  }
  h->a.alloc(d.nel);
  h->dc.alloc(d.nel);
  ICB_CUDA(cudaMemcpyAsync(h->fix.p, mask.data(), d.nnode, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->f.p, f.data(), sizeof(double) * d.ld, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->uD.p, ud.data(), sizeof(double) * d.ld, cudaMemcpyHostToDevice, s));
  h->pcg = std::make_unique<JacobiPcg<double>>(d, s);
  ICB_CUDA(cudaStreamSynchronize(s));
  h->finalized = true;
  if(numeq)
    *numeq = hs.numeq;
  ICB_API_END
}

int icb_heat_set_density(icb_heat h, const double *rho)
{
  ICB_API_BEGIN
  needH(h, true);
  if(!rho)
    throw Error{ICB_ERR_BAD_ARG, "NULL rho"};
  ICB_CUDA(cudaSetDevice(h->ctx->device));
  cudaStream_t s = h->stream();
  const long long n = h->d.nel;
  ICB_CUDA(cudaMemcpyAsync(h->dc.p, rho, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_heat_simp<<<nb256(n), 256, 0, s>>>(n, h->dc.p, h->desc.penalty, h->a.p);
  count_launch();
  ICB_CUDA(cudaStreamSynchronize(s));
  h->hasDensity = true;
  ICB_API_END
}

int icb_heat_solve(icb_heat h, const icb_solve_opts *opts, icb_solve_info *info)
{
  ICB_API_BEGIN
  needH(h, true);
  if(!h->hasDensity)
    throw Error{ICB_ERR_STATE, "set the density first"};
  ICB_CUDA(cudaSetDevice(h->ctx->device));
  icb_solve_info inf{};
  solveHeat(*h, opts, &inf);
  if(info)
    *info = inf;
  if(inf.status != ICB_OK)
    return inf.status;
  ICB_API_END
}

int icb_heat_get_temperature(icb_heat h, double *nodeval)
{
  ICB_API_BEGIN
  needH(h, true);
  if(!nodeval)
    throw Error{ICB_ERR_BAD_ARG, "NULL argument"};
  if(!h->solved)
    throw Error{ICB_ERR_STATE, "solve first"};
  cudaStream_t s = h->stream();
  std::vector<double> t(h->d.ld);
  ICB_CUDA(cudaMemcpyAsync(t.data(), h->u.p, sizeof(double) * h->d.ld, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  for(long long n = 0; n < h->d.nnode; n++)
    nodeval[n] = std::fabs(t[n]) < 1.0e-15 ? 0.0 : t[n];
  ICB_API_END
}

int icb_heat_objective(icb_heat h, double *f)
{
  ICB_API_BEGIN
  needH(h, true);
  if(!f)
    throw Error{ICB_ERR_BAD_ARG, "NULL argument"};
  if(!h->solved)
    throw Error{ICB_ERR_STATE, "solve first"};
  *f = heatObjective(*h);
  ICB_API_END
}

int icb_heat_sensitivity(icb_heat h, const double *rho, double *dc, double *dv)
{
  ICB_API_BEGIN
  needH(h, true);
  if(!rho || !dc)
    throw Error{ICB_ERR_BAD_ARG, "NULL argument"};
  if(!h->solved)
    throw Error{ICB_ERR_STATE, "solve first (and pass the density of the solve)"};
  cudaStream_t s = h->stream();
  const long long n = h->d.nel;
  DevBuf<double> r(n), out(n);
  ICB_CUDA(cudaMemcpyAsync(r.p, rho, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  heatSensDevice(*h, r.p, out.p, s);
  ICB_CUDA(cudaMemcpyAsync(dc, out.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  if(dv)
    for(long long e = 0; e < n; e++)
      dv[e] = h->hs->volume;
  ICB_API_END
}

/// The opt-heat loop (opt_heat.cpp:79-151) on the device: Helmholtz filter,
/// threshold, solve, V0 at step 1, objective u^T K u, constraint
/// sum x v - V0, sensitivities times the threshold derivative, adjoint
/// Helmholtz filters, MMA (c = 1e5).  hist[step] = the objective.
int icb_run_heat(icb_heat h, const icb_loop_opts *o, const double *rho0, double *hist, double *xout)
{
  ICB_API_BEGIN
  needH(h, true);
  if(!o || !rho0 || !hist || o->nsteps <= 0 || !(o->filter_radius > 0.0))
    throw Error{ICB_ERR_BAD_ARG, "bad loop options"};
  ICB_CUDA(cudaSetDevice(h->ctx->device));
  cudaStream_t s = h->stream();
  const long long n = h->d.nel;
  const double vol = h->hs->volume;
  Dims fd = h->hs->dims; // the filter works on the element / node grid
  HelmFilter helm(fd, h->hs->h, o->filter_radius, s);
  MmaUpdater mma(n, s);
  DevBuf<double> x(n), xf(n), xh(n), dxh(n), dc(n), dv(n), dcf(n), dvf(n), lo(n), hi(n);
  ICB_CUDA(cudaMemcpyAsync(x.p, rho0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_fill<<<nb256(n), 256, 0, s>>>(n, 1.0e-4, lo.p);
  k_fill<<<nb256(n), 256, 0, s>>>(n, 1.0, hi.p);
  count_launch(2);
  icb_solve_opts so = o->solve;
  so.precision = ICB_FP64;
  so.precond = ICB_PRECOND_JACOBI;
  double V0 = 0.0;
  auto filt = [&](const double *in, double *out, bool sens) {
    icb_solve_info hi_{};
    int rc = helm.apply(in, out, sens, 1e-10, s, &hi_);
    if(rc)
      throw Error{rc, "Helmholtz filter solve did not converge"};
  };
  // the apps' Optimize::isConvergence stop rule (conv_eps > 0) and step
  // reports (on_step: design, temperature, no stress)
  double fold = 0.0;
  std::vector<double> hostRho, hostT, hostU;
  for(int step = 1; step <= o->nsteps; step++)
  {
    auto t0 = std::chrono::steady_clock::now();
    NvtxRange stepRange("heat step");
    filt(x.p, xf.p, false);
    const double beta = std::min(std::pow(2.0, (int)(step / 40)), 16.0);
    launch_threshold(n, xf.p, beta, 0.5, xh.p, dxh.p, s);
    k_heat_simp<<<nb256(n), 256, 0, s>>>(n, xh.p, h->desc.penalty, h->a.p);
    count_launch();
    h->hasDensity = true;
    icb_solve_info inf{};
    solveHeat(*h, &so, &inf);
    if(inf.status != ICB_OK)
      return inf.status;
    hist[step - 1] = heatObjective(*h);
    if(o->on_step)
    {
      hostRho.resize(n);
      hostU.resize(h->d.ld);
      hostT.resize(h->d.nnode);
      ICB_CUDA(cudaMemcpyAsync(hostRho.data(), xh.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
      ICB_CUDA(cudaMemcpyAsync(hostU.data(), h->u.p, sizeof(double) * h->d.ld,
                               cudaMemcpyDeviceToHost, s));
      ICB_CUDA(cudaStreamSynchronize(s));
      for(long long nd = 0; nd < h->d.nnode; nd++)
        hostT[nd] = std::fabs(hostU[nd]) < 1.0e-15 ? 0.0 : hostU[nd];
      o->on_step(o->step_user, step, hist[step - 1], hostRho.data(), hostT.data(), nullptr);
    }
    if(o->steps_done)
      *o->steps_done = step;
    bool last = false;
    if(o->conv_eps > 0.0)
    {
      last = std::fabs(fold - hist[step - 1]) / hist[step - 1] < o->conv_eps &&
             step > o->conv_min_steps;
      fold = hist[step - 1];
    }
    const double vs = device_dot(n, xh.p, hi.p, h->pcg->red, h->pcg->dots.p, s) * vol; // hi = 1
    if(step == 1)
      V0 = vs;
    const double g = vs - V0;
    heatSensDevice(*h, xh.p, dc.p, s);
    k_mul<<<nb256(n), 256, 0, s>>>(n, dc.p, dxh.p, 1.0);
    ICB_CUDA(cudaMemcpyAsync(dv.p, dxh.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_fill<<<nb256(n), 256, 0, s>>>(n, vol, dcf.p);
    k_mul<<<nb256(n), 256, 0, s>>>(n, dv.p, dcf.p, 1.0);
    count_launch(3);
    filt(dc.p, dcf.p, true);
    filt(dv.p, dvf.p, true);
    mma.update(x.p, dcf.p, g, dvf.p, lo.p, hi.p, s);
    ICB_CUDA(cudaStreamSynchronize(s));
    if(o->iter_seconds)
      o->iter_seconds[step - 1] =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if(last)
      break;
  }
  if(xout)
    ICB_CUDA(cudaMemcpyAsync(xout, x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

} // extern "C"
