// toapi.cu -- C entry points of the optimisation side: cone and Helmholtz
// filters, threshold, OC and MMA updates, and the two ICARAT app loops run
// end to end on the device (opt_macro_oc.cpp:84-172,
// opt_mma_Helmholtz.cpp:81-163).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "helm.hpp"
#include "loopcache.hpp"
#include "mg.hpp"
#include "opt.hpp"
#include "problem.hpp"
#include "reduce.cuh"

using namespace icb;

struct icb_cone_s
{
  icb_problem p;
  std::unique_ptr<ConeFilter> f;
  DevBuf<double> a, b; ///< staging for the host-pointer entry points
};
struct icb_helm_s
{
  icb_problem p;
  std::unique_ptr<HelmFilter> f;
  DevBuf<double> a, b;
  double tol = 1e-10;
};
struct icb_mma_s
{
  icb_ctx ctx;
  std::unique_ptr<MmaUpdater> m;
  DevBuf<double> x, df, dg, lo, hi;
};
struct icb_gcmma_s
{
  icb_ctx ctx;
  std::unique_ptr<GcmmaUpdater> g;
  DevBuf<double> xm, xv, df, dg, lo, hi;
};

namespace icb
{
void launch_sum(icb_problem p, const double *a, long long n, double *out);
}

namespace
{

void need(bool c, const char *m)
{
  if(!c)
    throw Error{ICB_ERR_BAD_ARG, m};
}
void needFinal(icb_problem p)
{
  if(!p)
    throw Error{ICB_ERR_BAD_ARG, "NULL problem"};
  if(!p->hs->finalized)
    throw Error{ICB_ERR_STATE, "problem not finalized"};
}

__global__ void k_scale_mul(long long n, double *__restrict__ a, const double *__restrict__ m,
                            double s)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < n)
    a[i] = s * a[i] * m[i];
}
__global__ void k_fill_d(long long n, double v, double *__restrict__ a)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < n)
    a[i] = v;
}
__global__ void k_sum(long long n, const double *__restrict__ a, RedScratch red, double *out)
{
  double v[1] = {0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    v[0] += a[i];
  block_reduce<1>(v, red, FinStore{out});
}
unsigned nb256(long long n) { return unsigned((n + 255) / 256); }
__global__ void k_sum_masked(long long n, const double *__restrict__ a,
                             const uint8_t *__restrict__ m, RedScratch red, double *out)
{
  double v[1] = {0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    if(m[i])
      v[0] += a[i];
  block_reduce<1>(v, red, FinStore{out});
}
__global__ void k_zero_masked(long long n, const uint8_t *__restrict__ m, double *__restrict__ a,
                              double *__restrict__ b)
{
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if(i < n && m[i])
  {
    a[i] = 0.0;
    b[i] = 0.0;
  }
}

double deviceSum(icb_problem p, const double *a, long long n)
{
  launch_sum(p, a, n, p->scal.p + 8);
  double h;
  ICB_CUDA(cudaMemcpyAsync(&h, p->scal.p + 8, sizeof(double), cudaMemcpyDeviceToHost, p->stream()));
  ICB_CUDA(cudaStreamSynchronize(p->stream()));
  return h;
}

/// sum of a over the flagged elements (all when m is NULL)
double deviceSumMasked(icb_problem p, const double *a, const uint8_t *m, long long n)
{
  if(!m)
    return deviceSum(p, a, n);
  int nb = int(std::min<long long>(nb256(n), (long long)p->red.maxBlocks));
  k_sum_masked<<<nb, 256, 0, p->stream()>>>(n, a, m, p->red, p->scal.p + 8);
  ICB_CUDA(cudaGetLastError());
  count_launch();
  double h;
  ICB_CUDA(cudaMemcpyAsync(&h, p->scal.p + 8, sizeof(double), cudaMemcpyDeviceToHost, p->stream()));
  ICB_CUDA(cudaStreamSynchronize(p->stream()));
  return h;
}

/// the per-step callback of a device loop: host copies of the physical
/// density, the node values and the von Mises stresses
struct StepReport
{
  std::vector<double> rho, nodeval, mises;
  void operator()(icb_problem p, const icb_loop_opts *o, int step, double comp,
                  const double *rhoDev)
  {
    if(!o->on_step)
      return;
    const long long nel = p->d.nel, neq = p->d.nnode * p->d.dim;
    rho.resize(nel);
    nodeval.resize(neq);
    mises.resize(nel);
    cudaStream_t s = p->stream();
    ICB_CUDA(cudaMemcpyAsync(rho.data(), rhoDev, sizeof(double) * nel, cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    int rc = icb_get_node_values(p, nodeval.data());
    if(rc == ICB_OK)
      rc = icb_von_mises(p, mises.data(), nullptr);
    if(rc != ICB_OK)
      throw Error{rc, "step report failed"};
    o->on_step(o->step_user, step, comp, rho.data(), nodeval.data(), mises.data());
  }
};

/// Optimize::isConvergence (optimize.hpp) as the loops apply it: `done` once
/// |f_old - f| / f < eps after step minstep; every step reports steps_done
struct StopRule
{
  double fold = 0.0;
  bool check(const icb_loop_opts *o, int step, double f)
  {
    if(o->steps_done)
      *o->steps_done = step;
    if(!(o->conv_eps > 0.0))
      return false;
    const bool done = std::fabs(fold - f) / f < o->conv_eps && step > o->conv_min_steps;
    fold = f;
    return done;
  }
};

/// the state a loop carries from step to step, as written into a checkpoint:
/// this header, the design x[nel], then for MMA low, upp, xold1, xold2 [nel]
struct LoopCkpt
{
  unsigned long long magic;
  int kind, step;
  long long nel;
  double V0, fold;
  int mmaIter, pad;
};
constexpr unsigned long long kCkptMagic = 0x69636231636b7074ull; // "icb1ckpt"
long long ckptBytes(long long nel, int kind) { return icb::loop_checkpoint_bytes(nel, kind); }
/// the header of a resume blob, checked against this run
const LoopCkpt &ckptRead(const void *blob, int kind, long long nel, int nsteps)
{
  const LoopCkpt &h = *static_cast<const LoopCkpt *>(blob);
  need(h.magic == kCkptMagic && h.kind == kind && h.nel == nel,
       "resume blob does not belong to this loop kind and grid");
  need(h.step >= 1 && h.step < nsteps, "resume step outside 1 .. nsteps - 1");
  return h;
}
/// copy n doubles of the blob's payload (after the header) at offset k * nel
void ckptToDev(const void *blob, long long k, long long nel, double *dst, cudaStream_t s)
{
  const double *src =
      reinterpret_cast<const double *>(static_cast<const char *>(blob) + sizeof(LoopCkpt)) + k * nel;
  ICB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * nel, cudaMemcpyHostToDevice, s));
}
void ckptFromDev(void *blob, long long k, long long nel, const double *src, cudaStream_t s)
{
  double *dst = reinterpret_cast<double *>(static_cast<char *>(blob) + sizeof(LoopCkpt)) + k * nel;
  ICB_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * nel, cudaMemcpyDeviceToHost, s));
}

void toDev(DevBuf<double> &b, const double *h, long long n, cudaStream_t s)
{
  if((long long)b.n < n)
    b.alloc(n);
  ICB_CUDA(cudaMemcpyAsync(b.p, h, sizeof(double) * n, cudaMemcpyHostToDevice, s));
}
} // namespace

namespace icb
{
long long loop_checkpoint_bytes(long long nel, int kind)
{
  return (long long)sizeof(LoopCkpt) + (long long)sizeof(double) * nel * (kind == ICB_JOB_MMA ? 5 : 1);
}
/// the problem's loop work space, created on first use
LoopCache &loop_cache(icb_problem p)
{
  if(!p->loops)
    p->loops = std::make_unique<LoopCache>();
  return *p->loops;
}
void launch_fill(long long n, double v, double *a, cudaStream_t s)
{
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, v, a);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
void launch_scale_mul(long long n, double *a, const double *m, double sc, cudaStream_t s)
{
  k_scale_mul<<<nb256(n), 256, 0, s>>>(n, a, m, sc);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
void launch_sum(icb_problem p, const double *a, long long n, double *out)
{
  int nb = int(std::min<long long>(nb256(n), (long long)p->red.maxBlocks));
  k_sum<<<nb, 256, 0, p->stream()>>>(n, a, p->red, out);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
} // namespace icb

extern "C" {

// ----------------------------------------------------------------- cone ----
int icb_cone_create(icb_problem p, double radius, icb_cone *out)
{
  ICB_API_BEGIN
  need(out != nullptr, "out is NULL");
  needFinal(p);
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  auto c = std::make_unique<icb_cone_s>();
  c->p = p;
  c->f = std::make_unique<ConeFilter>(p->d, p->hs->h, radius, p->stream());
  ICB_CUDA(cudaStreamSynchronize(p->stream()));
  *out = c.release();
  ICB_API_END
}

int icb_cone_destroy(icb_cone c)
{
  ICB_API_BEGIN
  delete c;
  ICB_API_END
}

int icb_cone_filter_device(icb_cone c, const double *in, double *out, int isSens)
{
  ICB_API_BEGIN
  need(c && in && out, "NULL argument");
  ICB_CUDA(cudaSetDevice(c->p->ctx->device));
  if(isSens)
    c->f->adjoint(in, out, c->p->stream());
  else
    c->f->forward(in, out, 0.0, 0.5, nullptr, nullptr, c->p->stream());
  ICB_API_END
}

int icb_cone_filter(icb_cone c, const double *in, double *out, int isSens)
{
  ICB_API_BEGIN
  need(c && in && out, "NULL argument");
  long long n = c->p->d.nel;
  cudaStream_t s = c->p->stream();
  ICB_CUDA(cudaSetDevice(c->p->ctx->device));
  toDev(c->a, in, n, s);
  if((long long)c->b.n < n)
    c->b.alloc(n);
  if(isSens)
    c->f->adjoint(c->a.p, c->b.p, s);
  else
    c->f->forward(c->a.p, c->b.p, 0.0, 0.5, nullptr, nullptr, s);
  ICB_CUDA(cudaMemcpyAsync(out, c->b.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_threshold(icb_ctx ctx, long long n, const double *x, double beta, double T, double *xhat,
                  double *dxhat)
{
  ICB_API_BEGIN
  need(ctx && x && n >= 0, "bad argument");
  need(beta > 0.0, "beta must be > 0");
  ICB_CUDA(cudaSetDevice(ctx->device));
  cudaStream_t s = ctx->stream;
  DevBuf<double> a(n), b(n), c(n);
  ICB_CUDA(cudaMemcpyAsync(a.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  launch_threshold(n, a.p, beta, T, b.p, c.p, s);
  if(xhat)
    ICB_CUDA(cudaMemcpyAsync(xhat, b.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  if(dxhat)
    ICB_CUDA(cudaMemcpyAsync(dxhat, c.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

// ------------------------------------------------------------ Helmholtz ----
int icb_helm_create(icb_problem p, double radius, icb_helm *out)
{
  ICB_API_BEGIN
  need(out != nullptr, "out is NULL");
  needFinal(p);
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  auto h = std::make_unique<icb_helm_s>();
  h->p = p;
  h->f = std::make_unique<HelmFilter>(p->d, p->hs->h, radius, p->stream());
  ICB_CUDA(cudaStreamSynchronize(p->stream()));
  *out = h.release();
  ICB_API_END
}

int icb_helm_destroy(icb_helm h)
{
  ICB_API_BEGIN
  delete h;
  ICB_API_END
}

int icb_helm_filter(icb_helm h, const double *in, double *out, int sensFlag)
{
  ICB_API_BEGIN
  need(h && in && out, "NULL argument");
  long long n = h->p->d.nel;
  cudaStream_t s = h->p->stream();
  ICB_CUDA(cudaSetDevice(h->p->ctx->device));
  toDev(h->a, in, n, s);
  if((long long)h->b.n < n)
    h->b.alloc(n);
  icb_solve_info inf{};
  int st = h->f->apply(h->a.p, h->b.p, sensFlag != 0, h->tol, s, &inf);
  ICB_CUDA(cudaMemcpyAsync(out, h->b.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  if(st != ICB_OK)
    throw Error{st, "Helmholtz filter solve did not converge"};
  ICB_API_END
}

// ------------------------------------------------------------------- OC ----
int icb_oc_update(icb_problem p, icb_cone cone, double *x, const double *dfdx, double g,
                  const double *dgdx, const double *xmin, const double *xmax, double movelimit,
                  double beta, double T, int *steps)
{
  ICB_API_BEGIN
  needFinal(p);
  need(x && dfdx && dgdx && xmin && xmax, "NULL argument");
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  cudaStream_t s = p->stream();
  long long n = p->d.nel;
  DevBuf<double> X(n), DF(n), DG(n), LO(n), HI(n), V(n);
  ICB_CUDA(cudaMemcpyAsync(X.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(DF.p, dfdx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(DG.p, dgdx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(LO.p, xmin, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(HI.p, xmax, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, p->hs->volume, V.p);
  count_launch();
  OcUpdater oc(p->d, s);
  OcParams P;
  P.move = movelimit;
  P.beta = beta;
  P.T = T;
  int k = oc.update(cone ? cone->f.get() : nullptr, X.p, DF.p, DG.p, g, LO.p, HI.p, V.p, P, s);
  ICB_CUDA(cudaMemcpyAsync(x, X.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  if(steps)
    *steps = k;
  ICB_API_END
}

// ------------------------------------------------------------------ MMA ----
int icb_mma_create(icb_ctx ctx, long long n, int m, icb_mma *out)
{
  ICB_API_BEGIN
  need(ctx && out && n > 0, "bad argument");
  need(m == 1, "the device MMA supports one constraint (m = 1)");
  ICB_CUDA(cudaSetDevice(ctx->device));
  auto h = std::make_unique<icb_mma_s>();
  h->ctx = ctx;
  h->m = std::make_unique<MmaUpdater>(n, ctx->stream);
  for(DevBuf<double> *b : {&h->x, &h->df, &h->dg, &h->lo, &h->hi})
    b->alloc(n);
  *out = h.release();
  ICB_API_END
}

int icb_mma_destroy(icb_mma h)
{
  ICB_API_BEGIN
  delete h;
  ICB_API_END
}

int icb_mma_update(icb_mma h, double *x, const double *dfdx, const double *gx,
                   const double *dgdx, const double *xmin, const double *xmax)
{
  ICB_API_BEGIN
  need(h && x && dfdx && gx && dgdx && xmin && xmax, "NULL argument");
  ICB_CUDA(cudaSetDevice(h->ctx->device));
  cudaStream_t s = h->ctx->stream;
  long long n = h->m->n;
  ICB_CUDA(cudaMemcpyAsync(h->x.p, x, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->df.p, dfdx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->dg.p, dgdx, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->lo.p, xmin, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->hi.p, xmax, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  h->m->update(h->x.p, h->df.p, gx[0], h->dg.p, h->lo.p, h->hi.p, s);
  ICB_CUDA(cudaMemcpyAsync(x, h->x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

// --------------------------------------------------------------- GCMMA ----
int icb_gcmma_create(icb_ctx ctx, long long n, int m, icb_gcmma *out)
{
  ICB_API_BEGIN
  need(ctx && out && n > 0, "bad argument");
  need(m == 1, "the device GCMMA supports one constraint (m = 1)");
  ICB_CUDA(cudaSetDevice(ctx->device));
  auto h = std::make_unique<icb_gcmma_s>();
  h->ctx = ctx;
  h->g = std::make_unique<GcmmaUpdater>(n, ctx->stream);
  for(DevBuf<double> *b : {&h->xm, &h->xv, &h->df, &h->dg, &h->lo, &h->hi})
    b->alloc(n);
  ICB_CUDA(cudaStreamSynchronize(ctx->stream));
  *out = h.release();
  ICB_API_END
}

int icb_gcmma_destroy(icb_gcmma h)
{
  ICB_API_BEGIN
  delete h;
  ICB_API_END
}

namespace
{
void gcmmaUpload(icb_gcmma h, const double *xval, const double *df0dx, const double *dfdx,
                 const double *xmin, const double *xmax)
{
  need(h && xval && df0dx && dfdx && xmin && xmax, "NULL argument");
  ICB_CUDA(cudaSetDevice(h->ctx->device));
  cudaStream_t s = h->ctx->stream;
  const size_t b = sizeof(double) * h->g->core.n;
  ICB_CUDA(cudaMemcpyAsync(h->xv.p, xval, b, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->df.p, df0dx, b, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->dg.p, dfdx, b, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->lo.p, xmin, b, cudaMemcpyHostToDevice, s));
  ICB_CUDA(cudaMemcpyAsync(h->hi.p, xmax, b, cudaMemcpyHostToDevice, s));
}
} // namespace

int icb_gcmma_outer(icb_gcmma h, double *xmma, const double *xval, double f0x,
                    const double *df0dx, const double *fx, const double *dfdx, const double *xmin,
                    const double *xmax)
{
  ICB_API_BEGIN
  need(xmma && fx, "NULL argument");
  gcmmaUpload(h, xval, df0dx, dfdx, xmin, xmax);
  cudaStream_t s = h->ctx->stream;
  h->g->outer(h->xm.p, h->xv.p, f0x, h->df.p, fx[0], h->dg.p, h->lo.p, h->hi.p, s);
  ICB_CUDA(cudaMemcpyAsync(xmma, h->xm.p, sizeof(double) * h->g->core.n, cudaMemcpyDeviceToHost,
                           s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_gcmma_inner(icb_gcmma h, double *xmma, double f0xnew, const double *fxnew,
                    const double *xval, double f0x, const double *df0dx, const double *fx,
                    const double *dfdx, const double *xmin, const double *xmax)
{
  ICB_API_BEGIN
  need(xmma && fxnew && fx, "NULL argument");
  gcmmaUpload(h, xval, df0dx, dfdx, xmin, xmax);
  cudaStream_t s = h->ctx->stream;
  const size_t b = sizeof(double) * h->g->core.n;
  ICB_CUDA(cudaMemcpyAsync(h->xm.p, xmma, b, cudaMemcpyHostToDevice, s));
  h->g->inner(h->xm.p, f0xnew, fxnew[0], h->xv.p, f0x, h->df.p, fx[0], h->dg.p, h->lo.p, h->hi.p,
              s);
  ICB_CUDA(cudaMemcpyAsync(xmma, h->xm.p, b, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_gcmma_concheck(icb_gcmma h, double f0xnew, const double *fxnew, int *conservative)
{
  ICB_API_BEGIN
  need(h && fxnew && conservative, "NULL argument");
  *conservative = h->g->concheck(f0xnew, fxnew[0]) ? 1 : 0;
  ICB_API_END
}

// ---------------------------------------------------------------- loops ----
/// The opt-macro-oc loop (opt_macro_oc.cpp:84-172) on the device, without
/// I/O and with a fixed number of steps.  hist[step] = compliance.
int icb_run_oc(icb_problem p, const icb_loop_opts *o, const double *rho0, double *hist,
               double *xout)
{
  ICB_API_BEGIN
  needFinal(p);
  need(o && (rho0 || o->resume) && hist, "NULL argument");
  need(o->nsteps > 0 && o->filter_radius > 0.0, "bad loop options");
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  cudaStream_t s = p->stream();
  const long long n = p->d.nel;
  const double vol = p->hs->volume;
  LoopCache &LC = loop_cache(p);
  ConeFilter &cone = LC.coneFilter(p->d, p->hs->h, o->filter_radius, s);
  OcUpdater &oc = LC.ocUpdater(p->d, s);
  DevBuf<double> &x = LC.buf(0, n), &xf = LC.buf(1, n), &xh = LC.buf(2, n), &dxh = LC.buf(3, n),
                 &dc = LC.buf(4, n), &dv = LC.buf(5, n), &dcf = LC.buf(6, n), &dvf = LC.buf(7, n),
                 &lo = LC.buf(8, n), &hi = LC.buf(9, n), &V = LC.buf(10, n);
  double V0 = 0.0;
  StopRule stop;
  int first = 1;
  if(o->resume)
  {
    const LoopCkpt &h = ckptRead(o->resume, ICB_JOB_OC, n, o->nsteps);
    ckptToDev(o->resume, 0, n, x.p, s);
    V0 = h.V0;
    stop.fold = h.fold;
    first = h.step + 1;
  }
  else
    ICB_CUDA(cudaMemcpyAsync(x.p, rho0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, 1.0e-4, lo.p);
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, 1.0, hi.p);
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, vol, V.p);
  count_launch(3);
  icb_solve_opts so = o->solve;
  StepReport report;
  OcParams P;
  P.move = o->move_limit;
  int done = first - 1;
  for(int step = first; step <= o->nsteps; step++)
  {
    auto t0 = std::chrono::steady_clock::now();
    NvtxRange stepRange("oc step");
    const double beta = o->use_threshold ? std::min(std::pow(2.0, (int)(step / 40)), 16.0) : 0.0;
    cone.forward(x.p, xf.p, beta, 0.5, xh.p, dxh.p, s); // beta 0: xh = xf, dxh = 1
    int rc = icb_set_density_device(p, xh.p);
    if(rc)
      return rc;
    rc = icb_solve(p, &so, nullptr);
    if(rc)
      return rc;
    rc = icb_compliance(p, &hist[step - 1]);
    if(rc)
      return rc;
    report(p, o, step, hist[step - 1], xh.p);
    const bool last = stop.check(o, step, hist[step - 1]);
    if(step == 1)
      V0 = deviceSum(p, xh.p, n) * vol;
    const double *dcd = icb_sensitivity_device(p);
    if(!dcd)
      throw Error{ICB_ERR_STATE, "sensitivity failed"};
    ICB_CUDA(cudaMemcpyAsync(dc.p, dcd, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_scale_mul<<<nb256(n), 256, 0, s>>>(n, dc.p, dxh.p, 1.0);
    ICB_CUDA(cudaMemcpyAsync(dv.p, V.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_scale_mul<<<nb256(n), 256, 0, s>>>(n, dv.p, dxh.p, 1.0);
    count_launch(2);
    cone.adjoint(dc.p, dcf.p, s);
    cone.adjoint(dv.p, dvf.p, s);
    P.beta = beta;
    {
      NvtxRange r("oc update");
      oc.update(&cone, x.p, dcf.p, dvf.p, V0, lo.p, hi.p, V.p, P, s);
    }
    if(o->iter_seconds)
      o->iter_seconds[step - 1] =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    done = step;
    if(last)
      break;
  }
  if(xout)
    ICB_CUDA(cudaMemcpyAsync(xout, x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  if(o->checkpoint)
  {
    LoopCkpt h{kCkptMagic, ICB_JOB_OC, done, n, V0, stop.fold, 0, 0};
    std::memcpy(o->checkpoint, &h, sizeof h);
    ckptFromDev(o->checkpoint, 0, n, x.p, s);
  }
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

/// The opt-mma-HelmholtzFilter loop (opt_mma_Helmholtz.cpp:81-163) on the
/// device: Helmholtz filter, threshold, solve, constraint sum x v / V0 - 1
/// (0 at step 1 unless o->volume_ref > 0, then V0 = volume_ref), MMA.
int icb_run_mma(icb_problem p, const icb_loop_opts *o, const double *rho0, double *hist,
                double *xout)
{
  ICB_API_BEGIN
  needFinal(p);
  need(o && (rho0 || o->resume) && hist, "NULL argument");
  need(o->nsteps > 0 && o->filter_radius > 0.0, "bad loop options");
  need(o->filter_type == ICB_FILTER_HELMHOLTZ || o->filter_type == ICB_FILTER_CONE,
       "unknown filter_type");
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  cudaStream_t s = p->stream();
  const long long n = p->d.nel;
  const double vol = p->hs->volume;
  const bool cone = o->filter_type == ICB_FILTER_CONE;
  LoopCache &LC = loop_cache(p);
  HelmFilter *helm = nullptr;
  ConeFilter *cf = nullptr;
  if(cone)
    cf = &LC.coneFilter(p->d, p->hs->h, o->filter_radius, s);
  else
    helm = &LC.helmholtz(p->d, p->hs->h, o->filter_radius, s);
  MmaUpdater &mma = LC.mmaUpdater(n, s);
  DevBuf<double> &x = LC.buf(0, n), &xf = LC.buf(1, n), &xh = LC.buf(2, n), &dxh = LC.buf(3, n),
                 &dc = LC.buf(4, n), &dv = LC.buf(5, n), &dcf = LC.buf(6, n), &dvf = LC.buf(7, n),
                 &lo = LC.buf(8, n), &hi = LC.buf(9, n);
  DevBuf<uint8_t> nd(o->nondesign ? n : 0), vs(o->volume_set ? n : 0);
  if(o->nondesign)
    ICB_CUDA(cudaMemcpyAsync(nd.p, o->nondesign, n, cudaMemcpyHostToDevice, s));
  if(o->volume_set)
    ICB_CUDA(cudaMemcpyAsync(vs.p, o->volume_set, n, cudaMemcpyHostToDevice, s));
  double V0 = o->volume_ref;
  StopRule stop;
  int first = 1;
  if(o->resume)
  {
    const LoopCkpt &h = ckptRead(o->resume, ICB_JOB_MMA, n, o->nsteps);
    ckptToDev(o->resume, 0, n, x.p, s);
    ckptToDev(o->resume, 1, n, mma.low.p, s);
    ckptToDev(o->resume, 2, n, mma.upp.p, s);
    ckptToDev(o->resume, 3, n, mma.xold1.p, s);
    ckptToDev(o->resume, 4, n, mma.xold2.p, s);
    mma.iter = h.mmaIter;
    V0 = h.V0;
    stop.fold = h.fold;
    first = h.step + 1;
  }
  else
    ICB_CUDA(cudaMemcpyAsync(x.p, rho0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, 1.0e-4, lo.p);
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, 1.0, hi.p);
  count_launch(2);
  icb_solve_opts so = o->solve;
  StepReport report;
  auto filt = [&](const double *in, double *out, bool sens) {
    NvtxRange r(sens ? "filter (sensitivities)" : "filter");
    if(cone)
    {
      if(sens)
        cf->adjoint(in, out, s);
      else
        cf->forward(in, out, 0.0, 0.5, nullptr, nullptr, s);
      return;
    }
    icb_solve_info hi_{};
    int rc = helm->apply(in, out, sens, 1e-10, s, &hi_);
    if(rc)
      throw Error{rc, "Helmholtz filter solve did not converge"};
  };
  int done = first - 1;
  for(int step = first; step <= o->nsteps; step++)
  {
    auto t0 = std::chrono::steady_clock::now();
    NvtxRange stepRange("mma step");
    filt(x.p, xf.p, false);
    const double beta = std::min(std::pow(2.0, (int)(step / 40)), 16.0);
    launch_threshold(n, xf.p, beta, 0.5, xh.p, dxh.p, s);
    int rc = icb_set_density_device(p, xh.p);
    if(rc)
      return rc;
    rc = icb_solve(p, &so, nullptr);
    if(rc)
      return rc;
    double g = 0.0;
    const double vsum = deviceSumMasked(p, xh.p, o->volume_set ? vs.p : nullptr, n) * vol;
    if(step == 1 && o->volume_ref <= 0.0)
      V0 = vsum;
    else
      g = vsum / V0 - 1.0;
    rc = icb_compliance(p, &hist[step - 1]);
    if(rc)
      return rc;
    report(p, o, step, hist[step - 1], xh.p);
    const bool last = stop.check(o, step, hist[step - 1]);
    const double *dcd = icb_sensitivity_device(p);
    if(!dcd)
      throw Error{ICB_ERR_STATE, "sensitivity failed"};
    ICB_CUDA(cudaMemcpyAsync(dc.p, dcd, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_scale_mul<<<nb256(n), 256, 0, s>>>(n, dc.p, dxh.p, 1.0);
    k_fill_d<<<nb256(n), 256, 0, s>>>(n, vol / V0, dv.p);
    k_scale_mul<<<nb256(n), 256, 0, s>>>(n, dv.p, dxh.p, 1.0);
    count_launch(3);
    filt(dc.p, dcf.p, true);
    filt(dv.p, dvf.p, true);
    if(o->nondesign)
    {
      k_zero_masked<<<nb256(n), 256, 0, s>>>(n, nd.p, dcf.p, dvf.p);
      count_launch();
    }
    {
      NvtxRange r("mma update");
      mma.update(x.p, dcf.p, g, dvf.p, lo.p, hi.p, s);
    }
    ICB_CUDA(cudaStreamSynchronize(s));
    if(o->iter_seconds)
      o->iter_seconds[step - 1] =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    done = step;
    if(last)
      break;
  }
  if(xout)
    ICB_CUDA(cudaMemcpyAsync(xout, x.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  if(o->checkpoint)
  {
    LoopCkpt h{kCkptMagic, ICB_JOB_MMA, done, n, V0, stop.fold, mma.iter, 0};
    std::memcpy(o->checkpoint, &h, sizeof h);
    ckptFromDev(o->checkpoint, 0, n, x.p, s);
    ckptFromDev(o->checkpoint, 1, n, mma.low.p, s);
    ckptFromDev(o->checkpoint, 2, n, mma.upp.p, s);
    ckptFromDev(o->checkpoint, 3, n, mma.xold1.p, s);
    ckptFromDev(o->checkpoint, 4, n, mma.xold2.p, s);
  }
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

long long icb_loop_checkpoint_bytes(icb_problem p, int kind)
{
  if(!p || !p->hs || (kind != ICB_JOB_OC && kind != ICB_JOB_MMA))
    return -1;
  return ckptBytes(p->d.nel, kind);
}

/// The opt_macro_gcmma loop (opt_macro_gcmma.cpp:83-238) on the device:
/// cone filter, threshold with beta = min(int(max((step - 100) / 40, 1)), 8),
/// solve, V0 at step 1, constraint sum x v - V0, sensitivities times the
/// threshold derivative (dv = v), adjoint filter, GCMMA outer update,
/// evaluation of the candidate, at most 15 inner updates until ConCheck.
int icb_run_gcmma(icb_problem p, const icb_loop_opts *o, const double *rho0, double *hist,
                  int *inner, double *xout)
{
  ICB_API_BEGIN
  needFinal(p);
  need(o && rho0 && hist, "NULL argument");
  need(o->nsteps > 0 && o->filter_radius > 0.0, "bad loop options");
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  cudaStream_t s = p->stream();
  const long long n = p->d.nel;
  const double vol = p->hs->volume;
  LoopCache &LC = loop_cache(p);
  ConeFilter &cone = LC.coneFilter(p->d, p->hs->h, o->filter_radius, s);
  GcmmaUpdater &gc = LC.gcmmaUpdater(n, s);
  DevBuf<double> &x = LC.buf(0, n), &xnew = LC.buf(1, n), &xf = LC.buf(2, n), &xh = LC.buf(3, n),
                 &dxh = LC.buf(4, n), &dc = LC.buf(5, n), &dv = LC.buf(6, n), &dcf = LC.buf(7, n),
                 &dvf = LC.buf(8, n), &lo = LC.buf(9, n), &hi = LC.buf(10, n), &V = LC.buf(11, n);
  ICB_CUDA(cudaMemcpyAsync(x.p, rho0, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, 1.0e-4, lo.p);
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, 1.0, hi.p);
  k_fill_d<<<nb256(n), 256, 0, s>>>(n, vol, V.p);
  count_launch(3);
  icb_solve_opts so = o->solve;
  double V0 = 0.0;
  StepReport report;
  // filter, threshold and solve at xx: compliance and sum x v
  auto evaluate = [&](const double *xx, double beta, double &f, double &vs) {
    cone.forward(xx, xf.p, beta, 0.5, xh.p, dxh.p, s);
    int rc = icb_set_density_device(p, xh.p);
    if(rc == ICB_OK)
      rc = icb_solve(p, &so, nullptr);
    if(rc == ICB_OK)
      rc = icb_compliance(p, &f);
    if(rc)
      throw Error{rc, icb_last_error()};
    vs = deviceSum(p, xh.p, n) * vol;
  };
  StopRule stop;
  for(int step = 1; step <= o->nsteps; step++)
  {
    auto t0 = std::chrono::steady_clock::now();
    NvtxRange stepRange("gcmma step");
    const int btmp = int(std::max((step - 100) / 40.0, 1.0));
    const double beta = std::min(double(btmp), 8.0);
    double f, vs;
    evaluate(x.p, beta, f, vs);
    hist[step - 1] = f;
    report(p, o, step, f, xh.p);
    const bool last = stop.check(o, step, f);
    if(step == 1)
      V0 = vs;
    const double g = vs - V0;
    const double *dcd = icb_sensitivity_device(p);
    if(!dcd)
      throw Error{ICB_ERR_STATE, "sensitivity failed"};
    ICB_CUDA(cudaMemcpyAsync(dc.p, dcd, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_scale_mul<<<nb256(n), 256, 0, s>>>(n, dc.p, dxh.p, 1.0);
    ICB_CUDA(cudaMemcpyAsync(dv.p, V.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    k_scale_mul<<<nb256(n), 256, 0, s>>>(n, dv.p, dxh.p, 1.0);
    count_launch(2);
    cone.adjoint(dc.p, dcf.p, s);
    cone.adjoint(dv.p, dvf.p, s);
    {
      NvtxRange r("gcmma outer update");
      gc.outer(xnew.p, x.p, f, dcf.p, g, dvf.p, lo.p, hi.p, s);
    }
    double fn, vn;
    evaluate(xnew.p, beta, fn, vn);
    int k = 0;
    for(; !gc.concheck(fn, vn - V0) && k < 15; k++)
    {
      {
        NvtxRange r("gcmma inner update");
        gc.inner(xnew.p, fn, vn - V0, x.p, f, dcf.p, g, dvf.p, lo.p, hi.p, s);
      }
      evaluate(xnew.p, beta, fn, vn);
    }
    if(inner)
      inner[step - 1] = k;
    ICB_CUDA(cudaMemcpyAsync(x.p, xnew.p, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
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
