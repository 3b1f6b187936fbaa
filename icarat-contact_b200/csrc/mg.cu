// mg.cu -- geometric multigrid preconditioner on the structured grid
// hierarchy and the multigrid-preconditioned flexible CG, in FP64 throughout
// (ICB_FP64) or with an FP32 V-cycle under the FP64 Krylov iteration
// (ICB_MIXED: FP64 iterate, residual, operator and reductions; FP32
// smoother, transfers and coarse apply; FP64 coarse factorisation).
//
// FP32 inner solves inside FP64 defect correction were tried first: with
// SIMP contrast (E from 1e-6 to 1 and Emin = 1e-9) the FP32 operator loses
// p.Kp to cancellation once the search directions are smooth, and the inner
// CG breaks down; keeping the Krylov recurrence in FP64 and only the
// preconditioner in FP32 converges like the FP64 solve.
//
// ICARAT has no multigrid (its iterative path is Eigen's Jacobi CG,
// src/analysis/solver/solvers.cpp:64-92); this is the B200 replacement of
// that solve for large grids.  Design:
//  * levels by 2:1 coarsening of the element grid (ceil for odd counts: the
//    last coarse element then sticks out of the domain, and its modulus sums
//    the children that exist over all its child slots), coarse moduli = mean
//    of the children's E, coarse element matrix = K0 of the 2h element
//    (rediscretisation; equal to the Galerkin product for constant
//    coefficients).  An axis that is one element thick is kept while the
//    others halve (semi-coarsening), so thin and high-aspect grids still
//    reach a small coarsest system; the coarse elements then change shape
//    and the smoother's eigenvalue bound covers every level's K0;
//  * transfer: (bi/tri)linear prolongation P, restriction R = P^T;
//    constrained DOFs are masked on every level (a coarse DOF is constrained
//    when a constrained fine DOF interpolates from it);
//  * smoother: Chebyshev polynomial in D^-1 K of degree nu on
//    [lmax/10, lmax], one fused operator kernel per step (three-term form),
//    before and after the coarse correction; the first pre-smoothing step
//    starts from zero and needs no operator;
//  * coarsest level (<= 160 DOFs by default): dense FP64 inverse built on
//    the device (one CTA, Gauss-Jordan in shared memory), applied as a
//    dense product.
// The whole V-cycle is a fixed kernel sequence, so one PCG iteration with
// its V-cycle is captured as the body of a CUDA graph's conditional WHILE
// node, which the device repeats until the stop flag is set.
#include "mg_impl.cuh"

namespace icb
{
// ============================================================== Mixed ======
/// r32 = float(s * r64): the outer residual, scaled to unit norm, as the
/// right-hand side of the FP32 inner solve
__global__ void k_dc_to_f32(long long n, const double *__restrict__ r, double sc,
                            float *__restrict__ r32)
{
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    r32[i] = float(sc * r[i]);
}
/// x += w * d (the FP32 correction accumulated into the FP64 iterate)
__global__ void k_dc_update(long long n, double *__restrict__ x, const float *__restrict__ d,
                            double w)
{
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    x[i] += w * double(d[i]);
}


/// FP64 iterative refinement (defect correction) around an all-FP32
/// multigrid PCG: r = b - K x in FP64, the correction K d = r solved in FP32
/// (Krylov vectors, operator, V-cycle; scalars reduced in FP64) to a relative
/// tolerance, x += d in FP64, until ||r|| <= tol ||b|| measured in FP64.  FP64
/// work per outer step: one operator application and three vector passes.
static int solve_refine(icb_problem p, Mixed &M, const icb_solve_opts &o, const double *b,
                        icb_solve_info &inf)
{
  cudaStream_t s = p->stream();
  const HostSetup &hs = *p->hs;
  if(!M.mg32)
  {
    M.mg32 = std::make_unique<MgPcg<float, float>>();
    M.mg32->build(hs, p->K0f, p->Ef.p, p->K0f, p->Ef.p, p->fix.p, o.mg_coarse_dofs, o.mg_smooth,
                  s);
    M.r64.alloc(p->nsoa);
    M.r32.alloc(p->nsoa);
    M.d32.alloc(p->nsoa);
    ICB_CUDA(cudaMemsetAsync(M.r32.p, 0, M.r32.bytes(), s));
    ICB_CUDA(cudaMemsetAsync(M.d32.p, 0, M.d32.bytes(), s));
  }
  M.mg32->refresh(s);
  const long long n = p->nsoa;
  const int nb = vblocks(n);
  double *x = p->x.p, *r = M.r64.p;
  ICB_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, s));
  ICB_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
  const double bb = device_dot(n, b, b, p->red, p->scal.p, s);
  const double thr = std::max(o.tol * o.tol * bb, DBL_MIN);
  // inner relative tolerance: the requested one (inner_tol), else 1e-4; the
  // last outer step only solves as far as the outer tolerance needs
  const double eta = o.inner_tol > 0.0 ? o.inner_tol : 1e-4;
  double rr = bb;
  int iters = 0, matvecs = 0, outer = 0, status = ICB_OK;
  if(!std::isfinite(bb))
    status = ICB_ERR_NAN;
  while(status == ICB_OK && bb > 0.0 && rr >= thr)
  {
    if(iters >= o.maxit || outer >= 100)
    {
      status = ICB_ERR_MAXITER;
      break;
    }
    outer++;
    const double sc = 1.0 / std::sqrt(rr);
    k_dc_to_f32<<<nb, VB, 0, s>>>(n, r, sc, M.r32.p);
    count_launch();
    const double need = 0.5 * std::sqrt(thr / rr);
    icb_solve_info ii{};
    int st = M.mg32->solve(M.r32.p, M.d32.p, std::min(0.5, std::max(eta, need)),
                           o.maxit - iters, s, &ii);
    iters += ii.iters;
    matvecs += ii.matvecs;
    if(st == ICB_ERR_NAN || (st != ICB_OK && ii.iters == 0))
    {
      status = st == ICB_ERR_MAXITER ? ICB_ERR_MAXITER : st;
      break;
    }
    // a breakdown or the iteration cap of the inner solve still leaves a
    // usable correction; the FP64 residual below judges it
    k_dc_update<<<nb, VB, 0, s>>>(n, x, M.d32.p, 1.0 / sc);
    count_launch();
    OpExtras<double> ex;
    ex.mode = OP_RESIDUAL;
    ex.b = b;
    launch_op<double>(p->d, p->K0, p->E.p, x, r, p->fix.p, s, ex);
    const double rn = device_dot(n, r, r, p->red, p->scal.p, s);
    if(!std::isfinite(rn))
      status = ICB_ERR_NAN;
    else if(rn >= rr && st != ICB_OK)
      status = st; // the inner solve failed and the correction did not help
    rr = rn;
  }
  inf.iters = iters;
  inf.matvecs = matvecs + outer;
  inf.outer = outer;
  inf.relres = bb > 0.0 ? std::sqrt(rr / bb) : 0.0;
  return status;
}

Mixed &mixed_of(icb_problem p, const icb_solve_opts &o)
{
  if(!p->mixed)
    p->mixed = std::make_unique<Mixed>();
  Mixed &M = *p->mixed;
  if(M.coarseDofs != o.mg_coarse_dofs || M.smooth != o.mg_smooth)
  {
    M.mg64.reset();
    M.mgmx.reset();
    M.mg32.reset();
    M.coarseDofs = o.mg_coarse_dofs;
    M.smooth = o.mg_smooth;
  }
  return M;
}

int solve_multigrid(icb_problem p, const icb_solve_opts &o, const double *b, icb_solve_info *info)
{
  cudaStream_t s = p->stream();
  const HostSetup &hs = *p->hs;
  Mixed &M = mixed_of(p, o);
  cudaEvent_t e0, e1;
  ICB_CUDA(cudaEventCreate(&e0));
  ICB_CUDA(cudaEventCreate(&e1));
  ICB_CUDA(cudaEventRecord(e0, s));
  // the FP32 V-cycle may run on the tensor cores: count their timed-out waits
  const bool tc = o.precision != ICB_FP64 && tc_operator_enabled();
  const unsigned tc0 = tc ? tc_timeouts() : 0u;
  int status;
  icb_solve_info inf{};
  if(o.precision == ICB_MIXED_REFINE)
    status = solve_refine(p, M, o, b, inf);
  else if(o.precision == ICB_FP64)
  {
    if(!M.mg64)
    {
      M.mg64 = std::make_unique<MgPcg<double, double>>();
      M.mg64->build(hs, p->K0, p->E.p, p->K0, p->E.p, p->fix.p, o.mg_coarse_dofs, o.mg_smooth, s);
    }
    M.mg64->refresh(s);
    status = M.mg64->solve(b, p->x.p, o.tol, o.maxit, s, &inf);
  }
  else
  {
    if(!M.mgmx)
    {
      M.mgmx = std::make_unique<MgPcg<double, float>>();
      M.mgmx->build(hs, p->K0, p->E.p, p->K0f, p->Ef.p, p->fix.p, o.mg_coarse_dofs, o.mg_smooth,
                    s);
    }
    M.mgmx->refresh(s);
    status = M.mgmx->solve(b, p->x.p, o.tol, o.maxit, s, &inf);
  }
  if(o.precision != ICB_MIXED_REFINE)
    inf.outer = 1;
  // a CTA whose tensor-core wait gave up left its tile of a V-cycle operator
  // product unwritten: the solve is not trusted, whatever it converged to
  if(tc && tc_timeouts() != tc0)
  {
    status = ICB_ERR_TIMEOUT;
    set_error("a tensor-core operator wait timed out inside the V-cycle");
  }
  ICB_CUDA(cudaEventRecord(e1, s));
  ICB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  inf.seconds = ms * 1e-3;
  inf.status = status;
  if(info)
    *info = inf;
  return status;
}

} // namespace icb

icb_problem_s::icb_problem_s() = default;
icb_problem_s::~icb_problem_s() = default;
