// capi.cpp -- the extern "C" boundary of libicarat_b200.so.
//
// Each entry point maps one ICARAT call (cited in include/icarat_b200.h) onto
// the device implementation, converts C++ exceptions into status codes and
// never lets one cross the C ABI.  Where ICARAT calls exit(1) on bad input
// (solvers.cpp:57-61, elasticity.cpp:64-67, filter.hpp:126-130) this library
// returns ICB_ERR_BAD_ARG with a message instead.
#include <cmath>
#include <cstring>
#include <string>

#include "graphloop.hpp"
#include "mg.hpp"
#include "problem.hpp"

using namespace icb;

#include <atomic>

namespace icb
{
static thread_local std::string g_err;
static std::atomic<long long> g_launches{0};
void set_error(const std::string &m) { g_err = m; }
static thread_local long long t_launches = 0;
void count_launch(long long n)
{
  g_launches += n;
  t_launches += n;
}
long long thread_launch_count() { return t_launches; }
} // namespace icb

namespace
{
void need(bool c, const char *m)
{
  if(!c)
    throw Error{ICB_ERR_BAD_ARG, m};
}
void needState(bool c, const char *m)
{
  if(!c)
    throw Error{ICB_ERR_STATE, m};
}
void setDevice(icb_problem p) { ICB_CUDA(cudaSetDevice(p->ctx->device)); }

/// neq host array (node-major interleaved) -> SoA device layout
std::vector<double> toSoa(const Dims &d, const std::vector<double> &v)
{
  std::vector<double> o((size_t)d.dim * d.ld, 0.0);
  for(long long n = 0; n < d.nnode; n++)
    for(int c = 0; c < d.dim; c++)
      o[c * d.ld + n] = v[n * d.dim + c];
  return o;
}

void ensureDiag(icb_problem p)
{
  if(!p->diagValid)
  {
    launch_diag<double>(p->d, p->K0, p->E.p, p->fix.p, p->dinv.p, nullptr, p->stream());
    p->diagValid = true;
  }
}
} // namespace

extern "C" {

const char *icb_last_error(void) { return icb::g_err.c_str(); }
const char *icb_version(void) { return "icarat-b200 0.1 (sm_100a)"; }

int icb_ctx_create(int device, icb_ctx *out)
{
  ICB_API_BEGIN
  need(out != nullptr, "out is NULL");
  int n = 0;
  ICB_CUDA(cudaGetDeviceCount(&n));
  need(device >= 0 && device < n, "no such CUDA device");
  ICB_CUDA(cudaSetDevice(device));
  // the no-alloc solve's static scratch gets its device memory here, when
  // its module loads, not in the middle of a caller's solve
  noalloc_prepare_current_device();
  auto *c = new icb_ctx_s;
  c->device = device;
  c->refs = 1;
  cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
  if(e != cudaSuccess)
  {
    delete c;
    ICB_CUDA(e);
  }
  *out = c;
  ICB_API_END
}

namespace
{
/// drop one reference; the context (stream) goes when the last holder does
void ctxRelease(icb_ctx ctx)
{
  if(--ctx->refs > 0)
    return;
  cudaSetDevice(ctx->device);
  cudaStreamSynchronize(ctx->stream);
  cudaStreamDestroy(ctx->stream);
  delete ctx;
}
} // namespace

int icb_ctx_destroy(icb_ctx ctx)
{
  ICB_API_BEGIN
  if(!ctx)
    return ICB_OK;
  ctxRelease(ctx);
  ICB_API_END
}

void *icb_ctx_stream(icb_ctx ctx) { return ctx ? (void *)ctx->stream : nullptr; }

int icb_ctx_synchronize(icb_ctx ctx)
{
  ICB_API_BEGIN
  need(ctx != nullptr, "ctx is NULL");
  ICB_CUDA(cudaStreamSynchronize(ctx->stream));
  ICB_API_END
}

int icb_problem_create(icb_ctx ctx, const icb_grid_desc *desc, icb_problem *out)
{
  ICB_API_BEGIN
  need(ctx && desc && out, "NULL argument");
  need(desc->state != ICB_HEAT, "heat conduction problems are created with icb_heat_create");
  auto p = std::make_unique<icb_problem_s>();
  p->ctx = ctx;
  p->hs = std::make_unique<HostSetup>(*desc);
  ctx->refs++;
  p->d = p->hs->dims;
  p->nsoa = (long long)p->d.dim * p->d.ld;
  std::memcpy(p->K0, p->hs->K0, sizeof(p->K0));
  for(int i = 0; i < 576; i++)
    p->K0f[i] = float(p->K0[i]);
  *out = p.release();
  ICB_API_END
}

int icb_problem_destroy(icb_problem p)
{
  ICB_API_BEGIN
  if(!p)
    return ICB_OK;
  icb_ctx c = p->ctx;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  delete p;
  ctxRelease(c);
  ICB_API_END
}

int icb_dirichlet_box(icb_problem p, const int *flag, const double *val, const double *range)
{
  ICB_API_BEGIN
  need(p && flag && val && range, "NULL argument");
  p->hs->dirichletBox(flag, val, range);
  ICB_API_END
}

int icb_dirichlet_mask(icb_problem p, const unsigned char *fixed, const double *val)
{
  ICB_API_BEGIN
  need(p && fixed, "NULL argument");
  p->hs->dirichletMask(fixed, val);
  ICB_API_END
}

int icb_traction_box(icb_problem p, const double *val, const double *range)
{
  ICB_API_BEGIN
  need(p && val && range, "NULL argument");
  p->hs->tractionBox(val, range);
  ICB_API_END
}

int icb_nodal_load(icb_problem p, long long node, const double *f)
{
  ICB_API_BEGIN
  need(p && f, "NULL argument");
  p->hs->nodalLoad(node, f);
  ICB_API_END
}

int icb_finalize(icb_problem p, long long *numeq)
{
  ICB_API_BEGIN
  need(p != nullptr, "NULL problem");
  needState(!p->hs->finalized, "icb_finalize called twice");
  setDevice(p);
  HostSetup &hs = *p->hs;
  hs.finalize();
  const Dims &d = p->d;
  cudaStream_t s = p->stream();
  // Dirichlet bit mask per node, loads and Dirichlet values in SoA
  std::vector<uint8_t> mask(d.nnode, 0);
  std::vector<double> fneq(hs.neq, 0.0), dv(hs.neq, 0.0);
  std::vector<long long> fidx(hs.numeq);
  bool anyD = false;
  for(long long n = 0; n < d.nnode; n++)
    for(int c = 0; c < d.dim; c++)
    {
      long long gi = n * d.dim + c;
      if(hs.fixed[gi])
      {
        mask[n] |= uint8_t(1u << c);
        dv[gi] = hs.dval[gi];
        anyD = anyD || hs.dval[gi] != 0.0;
      }
      else
      {
        fneq[gi] = hs.fext[hs.dof[gi]];
        fidx[hs.dof[gi]] = c * d.ld + n;
      }
    }
  p->fix.alloc(d.nnode);
  ICB_CUDA(cudaMemcpyAsync(p->fix.p, mask.data(), d.nnode, cudaMemcpyHostToDevice, s));
  std::vector<double> fs = toSoa(d, fneq);
  p->f.alloc(p->nsoa);
  ICB_CUDA(cudaMemcpyAsync(p->f.p, fs.data(), sizeof(double) * p->nsoa, cudaMemcpyHostToDevice, s));
  p->hasDirichletValues = anyD;
  if(anyD)
  {
    std::vector<double> ds = toSoa(d, dv);
    p->uD.alloc(p->nsoa);
    ICB_CUDA(cudaMemcpyAsync(p->uD.p, ds.data(), sizeof(double) * p->nsoa,
                             cudaMemcpyHostToDevice, s));
  }
  p->freeIdx.alloc(std::max<long long>(hs.numeq, 1));
  if(hs.numeq)
    ICB_CUDA(cudaMemcpyAsync(p->freeIdx.p, fidx.data(), sizeof(long long) * hs.numeq,
                             cudaMemcpyHostToDevice, s));
  for(auto *b : {&p->u, &p->x, &p->b, &p->work, &p->dinv})
  {
    b->alloc(p->nsoa);
    ICB_CUDA(cudaMemsetAsync(b->p, 0, b->bytes(), s));
  }
  p->rho.alloc(d.nel);
  p->E.alloc(d.nel);
  p->Ef.alloc(d.nel);
  p->dc.alloc(d.nel);
  p->numeqBuf.alloc(std::max<long long>(hs.numeq, 1));
  p->scal.alloc(16);
  int mb = reduction_blocks(d);
  p->redPart.alloc((size_t)mb * 4);
  p->redCnt.alloc(1);
  ICB_CUDA(cudaMemsetAsync(p->redCnt.p, 0, sizeof(unsigned), s));
  p->red = RedScratch{p->redPart.p, p->redCnt.p, mb};
  p->pcg = std::make_unique<JacobiPcg<double>>(d, s);
  ICB_CUDA(cudaStreamSynchronize(s));
  if(numeq)
    *numeq = hs.numeq;
  ICB_API_END
}

int icb_count_dof(icb_problem p, int *dof, long long *numeq)
{
  ICB_API_BEGIN
  need(p && numeq, "NULL argument");
  const HostSetup &hs = *p->hs;
  long long cnt = 0;
  for(long long i = 0; i < hs.neq; i++)
    cnt += hs.fixed[i] ? 0 : 1;
  *numeq = cnt;
  if(dof)
  {
    long long f = 0, c = cnt;
    for(long long i = 0; i < hs.neq; i++)
      dof[i] = int(hs.fixed[i] ? c++ : f++);
  }
  ICB_API_END
}

int icb_get_dof_map(icb_problem p, int *dof)
{
  ICB_API_BEGIN
  need(p && dof, "NULL argument");
  needState(p->hs->finalized, "call icb_finalize first");
  std::memcpy(dof, p->hs->dof.data(), sizeof(int) * p->hs->neq);
  ICB_API_END
}

int icb_get_load(icb_problem p, double *fext)
{
  ICB_API_BEGIN
  need(p && fext, "NULL argument");
  needState(p->hs->finalized, "call icb_finalize first");
  std::memcpy(fext, p->hs->fext.data(), sizeof(double) * p->hs->numeq);
  ICB_API_END
}

int icb_problem_sizes(icb_problem p, long long *nel, long long *nnode, long long *neq,
                      long long *numeq)
{
  ICB_API_BEGIN
  need(p != nullptr, "NULL problem");
  if(nel)
    *nel = p->d.nel;
  if(nnode)
    *nnode = p->d.nnode;
  if(neq)
    *neq = p->hs->neq;
  if(numeq)
    *numeq = p->hs->finalized ? p->hs->numeq : -1;
  ICB_API_END
}

int icb_get_K0(icb_problem p, double *K0)
{
  ICB_API_BEGIN
  need(p && K0, "NULL argument");
  int nd = p->d.dim == 2 ? 8 : 24;
  std::memcpy(K0, p->K0, sizeof(double) * nd * nd);
  ICB_API_END
}

int icb_element_volume(icb_problem p, double *v)
{
  ICB_API_BEGIN
  need(p && v, "NULL argument");
  *v = p->hs->volume;
  ICB_API_END
}

int icb_set_density_device(icb_problem p, const double *rho_dev)
{
  ICB_API_BEGIN
  need(p && rho_dev, "NULL argument");
  needState(p->hs->finalized, "call icb_finalize first");
  setDevice(p);
  const icb_grid_desc &g = p->hs->desc;
  if(rho_dev != p->rho.p)
    ICB_CUDA(cudaMemcpyAsync(p->rho.p, rho_dev, sizeof(double) * p->d.nel,
                             cudaMemcpyDeviceToDevice, p->stream()));
  launch_simp(p->d.nel, g.young1, g.young2, g.penalty, p->rho.p, p->E.p, p->Ef.p, p->stream());
  p->hasDensity = true;
  p->diagValid = false;
  p->solved = false;
  ICB_API_END
}

int icb_set_density(icb_problem p, const double *rho)
{
  ICB_API_BEGIN
  need(p && rho, "NULL argument");
  needState(p->hs->finalized, "call icb_finalize first");
  setDevice(p);
  ICB_CUDA(cudaMemcpyAsync(p->rho.p, rho, sizeof(double) * p->d.nel, cudaMemcpyHostToDevice,
                           p->stream()));
  int rc = icb_set_density_device(p, p->rho.p);
  if(rc)
    return rc;
  ICB_CUDA(cudaStreamSynchronize(p->stream()));
  ICB_API_END
}

int icb_solve(icb_problem p, const icb_solve_opts *opts, icb_solve_info *info)
{
  ICB_API_BEGIN
  need(p != nullptr, "NULL problem");
  needState(p->hasDensity, "set the density first");
  setDevice(p);
  icb_solve_opts o{ICB_FP64, ICB_PRECOND_JACOBI, 1.0e-10, 10000, 0.0, 0, 0};
  if(opts)
    o = *opts;
  need(o.tol >= 0.0 && o.maxit > 0, "bad tolerance / iteration limit");
  need(o.precision == ICB_FP64 || o.precision == ICB_MIXED || o.precision == ICB_MIXED_REFINE,
       "unknown precision");
  need(o.inner_tol >= 0.0 && o.inner_tol < 1.0, "inner_tol must be in [0, 1)");
  need(o.precond == ICB_PRECOND_JACOBI || o.precond == ICB_PRECOND_GMG, "unknown preconditioner");
  NvtxRange range("icb_solve");
  cudaStream_t s = p->stream();
  // fres = fext - fint(u_D) (linear.hpp:74-80)
  const double *bptr = p->f.p;
  if(p->hasDirichletValues)
  {
    launch_matvec<double>(p->d, p->K0, p->E.p, p->uD.p, p->work.p, p->fix.p, s);
    launch_axpy_sub(p->nsoa, p->f.p, p->work.p, p->b.p, s);
    bptr = p->b.p;
  }
  icb_solve_info inf{};
  int st;
  if(o.precision == ICB_FP64 && o.precond == ICB_PRECOND_JACOBI)
  {
    ensureDiag(p);
    st = p->pcg->solve(p->K0, p->E.p, p->fix.p, p->dinv.p, bptr, p->x.p, o.tol, o.maxit, s, &inf);
  }
  else
  {
    st = solve_multigrid(p, o, bptr, &inf);
  }
  // u = x + u_D ; true residual in FP64
  if(p->hasDirichletValues)
    launch_add(p->nsoa, p->x.p, p->uD.p, p->u.p, s);
  else
    ICB_CUDA(cudaMemcpyAsync(p->u.p, p->x.p, sizeof(double) * p->nsoa, cudaMemcpyDeviceToDevice, s));
  launch_matvec<double>(p->d, p->K0, p->E.p, p->x.p, p->work.p, p->fix.p, s);
  launch_axpy_sub(p->nsoa, bptr, p->work.p, p->work.p, s);
  double rr = device_dot(p->nsoa, p->work.p, p->work.p, p->red, p->scal.p, s);
  double bb = device_dot(p->nsoa, bptr, bptr, p->red, p->scal.p + 1, s);
  inf.true_relres = bb > 0 ? std::sqrt(rr / bb) : 0.0;
  inf.status = st;
  p->last = inf;
  p->solved = true;
  if(info)
    *info = inf;
  if(st != ICB_OK)
  {
    set_error(st == ICB_ERR_MAXITER     ? "iteration limit reached"
              : st == ICB_ERR_BREAKDOWN ? "CG breakdown (p.Kp <= 0)"
              : st == ICB_ERR_TIMEOUT   ? "a tensor-core operator wait timed out inside the V-cycle"
                                        : "non-finite values in the solve");
    return st;
  }
  ICB_API_END
}

int icb_get_displacement(icb_problem p, double *u)
{
  ICB_API_BEGIN
  need(p && u, "NULL argument");
  needState(p->solved, "solve first");
  setDevice(p);
  cudaStream_t s = p->stream();
  long long ne = p->hs->numeq;
  launch_gather_free(p->d, p->freeIdx.p, ne, p->x.p, p->numeqBuf.p, s);
  ICB_CUDA(cudaMemcpyAsync(u, p->numeqBuf.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_get_node_values(icb_problem p, double *nodeval)
{
  ICB_API_BEGIN
  need(p && nodeval, "NULL argument");
  needState(p->solved, "solve first");
  setDevice(p);
  std::vector<double> h(p->nsoa);
  ICB_CUDA(cudaMemcpyAsync(h.data(), p->u.p, sizeof(double) * p->nsoa, cudaMemcpyDeviceToHost,
                           p->stream()));
  ICB_CUDA(cudaStreamSynchronize(p->stream()));
  const Dims &d = p->d;
  for(long long n = 0; n < d.nnode; n++)
    for(int c = 0; c < d.dim; c++)
    {
      double v = h[c * d.ld + n];
      nodeval[n * d.dim + c] = std::fabs(v) < 1.0e-15 ? 0.0 : v; // analysis_utility.hpp:27-28
    }
  ICB_API_END
}

int icb_compliance(icb_problem p, double *c)
{
  ICB_API_BEGIN
  need(p && c, "NULL argument");
  needState(p->solved, "solve first");
  setDevice(p);
  *c = device_dot(p->nsoa, p->x.p, p->f.p, p->red, p->scal.p + 2, p->stream());
  ICB_API_END
}

int icb_sensitivity(icb_problem p, double *dc, double *dv)
{
  ICB_API_BEGIN
  need(p && dc, "NULL argument");
  needState(p->solved, "solve first");
  setDevice(p);
  const icb_grid_desc &g = p->hs->desc;
  cudaStream_t s = p->stream();
  launch_sensitivity(p->d, p->K0, g.young1, g.young2, g.penalty, p->rho.p, p->u.p, p->dc.p, s);
  ICB_CUDA(cudaMemcpyAsync(dc, p->dc.p, sizeof(double) * p->d.nel, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  if(dv)
    for(long long e = 0; e < p->d.nel; e++)
      dv[e] = p->hs->volume;
  ICB_API_END
}

const double *icb_sensitivity_device(icb_problem p)
{
  if(!p || !p->solved)
  {
    set_error(p ? "solve first" : "NULL problem");
    return nullptr;
  }
  try
  {
    setDevice(p);
    const icb_grid_desc &g = p->hs->desc;
    launch_sensitivity(p->d, p->K0, g.young1, g.young2, g.penalty, p->rho.p, p->u.p, p->dc.p,
                       p->stream());
  }
  catch(const Error &e)
  {
    set_error(e.msg);
    return nullptr;
  }
  catch(const std::exception &e)
  {
    set_error(e.what());
    return nullptr;
  }
  return p->dc.p;
}

int icb_von_mises(icb_problem p, double *mises, double *stress)
{
  ICB_API_BEGIN
  need(p && mises, "NULL argument");
  needState(p->solved, "solve first");
  setDevice(p);
  cudaStream_t s = p->stream();
  const long long nel = p->d.nel;
  const int v = p->d.dim == 2 ? 3 : 6;
  DevBuf<double> m(nel), st(stress ? nel * v : 0);
  launch_von_mises(*p, m.p, stress ? st.p : nullptr, s);
  ICB_CUDA(cudaMemcpyAsync(mises, m.p, sizeof(double) * nel, cudaMemcpyDeviceToHost, s));
  if(stress)
    ICB_CUDA(cudaMemcpyAsync(stress, st.p, sizeof(double) * nel * v, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_reactions(icb_problem p, double *reaction)
{
  ICB_API_BEGIN
  need(p && reaction, "NULL argument");
  needState(p->solved, "solve first");
  setDevice(p);
  cudaStream_t s = p->stream();
  const long long n = p->d.nnode * p->d.dim;
  DevBuf<double> r(n);
  launch_reactions(*p, r.p, s);
  ICB_CUDA(cudaMemcpyAsync(reaction, r.p, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_matvec(icb_problem p, const double *x, double *y)
{
  ICB_API_BEGIN
  need(p && x && y, "NULL argument");
  needState(p->hasDensity, "set the density first");
  setDevice(p);
  cudaStream_t s = p->stream();
  long long ne = p->hs->numeq;
  ICB_CUDA(cudaMemsetAsync(p->work.p, 0, sizeof(double) * p->nsoa, s));
  ICB_CUDA(cudaMemcpyAsync(p->numeqBuf.p, x, sizeof(double) * ne, cudaMemcpyHostToDevice, s));
  launch_scatter_free(p->d, p->freeIdx.p, ne, p->numeqBuf.p, p->work.p, s);
  if(!p->work2.p)
    p->work2.alloc(p->nsoa);
  launch_matvec<double>(p->d, p->K0, p->E.p, p->work.p, p->work2.p, p->fix.p, s);
  launch_gather_free(p->d, p->freeIdx.p, ne, p->work2.p, p->numeqBuf.p, s);
  ICB_CUDA(cudaMemcpyAsync(y, p->numeqBuf.p, sizeof(double) * ne, cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

int icb_diagonal(icb_problem p, double *dg)
{
  ICB_API_BEGIN
  need(p && dg, "NULL argument");
  needState(p->hasDensity, "set the density first");
  setDevice(p);
  cudaStream_t s = p->stream();
  launch_diag<double>(p->d, p->K0, p->E.p, p->fix.p, p->dinv.p, p->work.p, s);
  p->diagValid = true;
  launch_gather_free(p->d, p->freeIdx.p, p->hs->numeq, p->work.p, p->numeqBuf.p, s);
  ICB_CUDA(cudaMemcpyAsync(dg, p->numeqBuf.p, sizeof(double) * p->hs->numeq,
                           cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  ICB_API_END
}

} // extern "C"

extern "C" {

long long icb_soa_length(icb_problem p) { return p ? p->nsoa : -1; }

long long icb_launch_count(void) { return icb::g_launches.load(); }

int icb_set_option(const char *name, long long value)
{
  ICB_API_BEGIN
  need(name != nullptr, "NULL name");
  std::string n(name);
  if(n == "tc_operator")
    set_tc_operator(value != 0);
  else if(n == "hex8_modal")
    set_hex8_modal(value != 0);
  else if(n == "device_loops")
    set_device_loops(value != 0);
  else if(n == "hex8_pair")
    set_hex8_pair(value != 0);
  else if(n == "batch_fused")
    set_batch_fused(value != 0);
  else if(n == "batch_handoff")
  {
    need(value >= 0 && value <= 1000000, "batch_handoff must be in [0, 1e6]");
    set_batch_handoff(int(value));
  }
  else if(n == "tc_spin_limit")
  {
    need(value >= 0 && value <= 0x7fffffffLL, "tc_spin_limit must be in [0, 2^31)");
    set_tc_spin_limit(unsigned(value));
  }
  else
    need(false, "unknown option");
  ICB_API_END
}

long long icb_get_option(const char *name)
{
  if(!name)
    return -1;
  std::string n(name);
  if(n == "tc_operator")
    return tc_operator_enabled() ? 1 : 0;
  if(n == "hex8_modal")
    return hex8_modal_enabled() ? 1 : 0;
  if(n == "device_loops")
    return device_loops_enabled() ? 1 : 0;
  if(n == "hex8_pair")
    return hex8_pair_enabled() ? 1 : 0;
  if(n == "batch_fused")
    return batch_fused_enabled() ? 1 : 0;
  if(n == "batch_handoff")
    return batch_handoff();
  if(n == "fused_batch_iters")
    return fused_iterations(0);
  if(n == "fused_problem_iters")
    return fused_iterations(1);
  if(n.rfind("fused_phase_us_", 0) == 0 && n.size() == 16)
    return (long long)(1e6 * fused_phase_seconds(n[15] - '0'));
  if(n.rfind("fused_active_us_", 0) == 0 && n.size() == 17)
    return (long long)(1e6 * fused_active_seconds(n[16] - '0'));
  if(n.rfind("fused_active_launches_", 0) == 0 && n.size() == 23)
    return fused_active_launches(n[22] - '0');
  if(n == "tc_timeouts")
    return (long long)tc_timeouts();
  if(n == "tc_spin_limit")
    return (long long)tc_spin_limit();
  return -1;
}

int icb_operator_apply_device(icb_problem p, int precision, const void *x, void *y)
{
  ICB_API_BEGIN
  need(p && x && y, "NULL argument");
  needState(p->hasDensity, "set the density first");
  setDevice(p);
  if(precision == ICB_FP64)
    launch_matvec<double>(p->d, p->K0, p->E.p, (const double *)x, (double *)y, p->fix.p,
                          p->stream());
  else if(precision == ICB_MIXED)
  {
    // the FP32 CUDA-core kernel, whatever the tensor-core switch says (the
    // process-wide switch is left alone: other threads may be solving)
    OpExtras<float> ex;
    ex.cudaCores = 1;
    launch_op<float>(p->d, p->K0f, p->Ef.p, (const float *)x, (float *)y, p->fix.p,
                     p->stream(), ex);
  }
  else if(precision == ICB_TF32)
  {
    // a tensor-core wait that gave up leaves its CTA's tile of y unwritten:
    // report it as ICB_ERR_TIMEOUT instead of returning a wrong product
    const unsigned t0 = tc_timeouts();
    OpExtras<float> ex;
    launch_op_tc(p->d, p->K0f, p->Ef.p, (const float *)x, (float *)y, p->fix.p, p->stream(), ex);
    ICB_CUDA(cudaStreamSynchronize(p->stream()));
    if(tc_timeouts() != t0)
      throw Error{ICB_ERR_TIMEOUT, "a tensor-core operator wait timed out; y is incomplete"};
  }
  else
    need(false, "unknown precision");
  ICB_API_END
}

int icb_smoother_apply_device(icb_problem p, int precision, const void *u, void *y,
                              const void *b, const void *dinv, double c1, double c2)
{
  ICB_API_BEGIN
  need(p && u && y && b && dinv, "NULL argument");
  needState(p->hasDensity, "set the density first");
  need(u != y, "u and y must be different vectors");
  setDevice(p);
  if(precision == ICB_FP64)
  {
    OpExtras<double> ex;
    ex.mode = OP_CHEB;
    ex.b = (const double *)b;
    ex.dinv = (const double *)dinv;
    ex.c1 = c1;
    ex.c2 = c2;
    ex.cudaCores = 1;
    launch_op<double>(p->d, p->K0, p->E.p, (const double *)u, (double *)y, p->fix.p,
                      p->stream(), ex);
  }
  else if(precision == ICB_MIXED)
  {
    OpExtras<float> ex;
    ex.mode = OP_CHEB;
    ex.b = (const float *)b;
    ex.dinv = (const float *)dinv;
    ex.c1 = c1;
    ex.c2 = c2;
    ex.cudaCores = 1;
    launch_op<float>(p->d, p->K0f, p->Ef.p, (const float *)u, (float *)y, p->fix.p,
                     p->stream(), ex);
  }
  else
    need(false, "unknown precision");
  ICB_API_END
}

} // extern "C"
