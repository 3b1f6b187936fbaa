/*
 * icarat_b200.h -- C ABI of the B200-native SIMP analysis-and-sensitivity
 * library (libicarat_b200.so).
 *
 * Plain C: opaque handles, plain pointers and sizes, int status codes
 * (0 = ok, negative = error; icb_last_error() gives the message).  Every
 * entry point names the ICARAT interface it replaces (path inside the ICARAT
 * project, file:line).  Arrays follow ICARAT's layouts:
 *   - element arrays: element index of MeshIcarat::meshBox
 *     (src/io/mesh_icarat.hpp:340-354 quad4, 459-493 hexa8);
 *   - "neq" arrays: node-major, components interleaved (node*dim + c);
 *   - "numeq" arrays: free DOFs in countDOF order
 *     (src/io/boundary_condition_base.hpp:35-88), i.e. Value::val / Force.
 * Host-pointer entry points copy through pinned staging; *_device entry points
 * take device pointers on the context's device and stream.
 */
#ifndef ICARAT_B200_H
#define ICARAT_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ICB_OK 0
#define ICB_ERR_BAD_ARG (-1)
#define ICB_ERR_OOM (-2)
#define ICB_ERR_BREAKDOWN (-3)
#define ICB_ERR_MAXITER (-4)
#define ICB_ERR_TIMEOUT (-5)
#define ICB_ERR_NAN (-6)
#define ICB_ERR_CUDA (-7)
#define ICB_ERR_STATE (-8)
#define ICB_ERR_REJECTED (-9)

/* ---- enums ------------------------------------------------------------- */
#define ICB_PLANE_STRESS 0
#define ICB_PLANE_STRAIN 1
#define ICB_3D 2
#define ICB_HEAT 3 /* icb_heat problems: scalar heat conduction, one DOF per node */

#define ICB_FP64 0  /* plain FP64 path: the drop-in for Solvers "Eigen_CG"   */
#define ICB_MIXED 1 /* FP64 Krylov + operator, FP32 multigrid preconditioner */
#define ICB_TF32 2  /* icb_operator_apply_device only: tensor-core FP32 operator */
/* FP64 defect correction around an FP32 GMG-PCG: FP32 Krylov vectors, operator
 * and V-cycle; FP64 residual, iterate and reductions */
#define ICB_MIXED_REFINE 3

#define ICB_PRECOND_JACOBI 0 /* DiagonalPreconditioner (solvers.cpp:64-92)  */
#define ICB_PRECOND_GMG 1    /* geometric multigrid V-cycle                 */

typedef struct icb_ctx_s *icb_ctx;
typedef struct icb_problem_s *icb_problem;
typedef struct icb_cone_s *icb_cone;
typedef struct icb_helm_s *icb_helm;
typedef struct icb_mma_s *icb_mma;
typedef struct icb_gcmma_s *icb_gcmma;

/* Structured box problem: the `[mesh]` keys of MeshIcarat::setParameter
 * (src/io/mesh_icarat.hpp:69-128) and the `[material]` keys of
 * Elastic::setParameter (src/problem/elasticity.cpp:19-32). */
typedef struct
{
  int dim;           /* 2 (quad4) or 3 (hexa8)                             */
  int nx, ny, nz;    /* division                                           */
  double lx, ly, lz; /* length                                             */
  int state;         /* ICB_PLANE_STRESS | ICB_PLANE_STRAIN | ICB_3D       */
  double young1;     /* young[0]  (E of rho = 0 when young[1] >= young[0]) */
  double young2;     /* young[1]                                           */
  double poisson;
  double penalty;
} icb_grid_desc;

typedef struct
{
  int precision;  /* ICB_FP64 | ICB_MIXED                                   */
  int precond;    /* ICB_PRECOND_JACOBI | ICB_PRECOND_GMG                   */
  double tol;     /* relative residual ||r||/||f|| (Solvers tol_, 1e-10)    */
  int maxit;      /* Solvers maxIter_ (10000)                               */
  double inner_tol; /* ICB_MIXED_REFINE: relative tolerance of each FP32 inner solve (0 = 1e-4) */
  int mg_smooth;  /* GMG: Chebyshev smoothing steps before and after (0 = 2) */
  int mg_coarse_dofs; /* GMG: coarsen while the grid has more DOFs (0 = 160, at most 1024) */
} icb_solve_opts;

typedef struct
{
  int iters;          /* Krylov iterations (Eigen's count: the converging one excluded) */
  int matvecs;        /* fine-level operator applications in the Krylov loop(s) */
  int outer;          /* Krylov cycles (1; ICB_MIXED_REFINE: refinement steps) */
  double relres;      /* ||r||/||f|| as the solver tracked it               */
  double true_relres; /* ||f - K u|| / ||f|| recomputed in FP64             */
  double seconds;     /* device time of the solve                           */
  int status;         /* ICB_OK, ICB_ERR_MAXITER, ICB_ERR_BREAKDOWN, ...    */
} icb_solve_info;

/* the message of this thread's last failed call (ICARAT prints it to
 * std::cerr before exit(1), e.g. solvers.cpp:57-61) */
const char *icb_last_error(void);
const char *icb_version(void);

/* ---- context ----------------------------------------------------------- */
/* No counterpart in ICARAT (one problem per process, no device): a context is
 * one CUDA device and one stream; problems created on it share the stream. */
int icb_ctx_create(int device, icb_ctx *out);
int icb_ctx_destroy(icb_ctx ctx);
/* cudaStream_t the library launches on (for events / interop) */
void *icb_ctx_stream(icb_ctx ctx);
int icb_ctx_synchronize(icb_ctx ctx);

/* ---- problem set-up ---------------------------------------------------- */
/* MeshIcarat(fem, config).setParameter + generate + LinearElastic
 * setParameter for every element (opt_mma_Helmholtz.cpp:31-50). */
int icb_problem_create(icb_ctx ctx, const icb_grid_desc *desc, icb_problem *out);
int icb_problem_destroy(icb_problem p);
/* BCIcarat::input_dirich (src/io/boundary_condition_icarat.hpp:68-127):
 * flag[6], val[6], range[6] = {xmin,xmax,ymin,ymax,zmin,zmax}, tol 1e-7. */
int icb_dirichlet_box(icb_problem p, const int *flag, const double *val,
                      const double *range);
/* setDirichValue for every node at once (boundary_condition_base.hpp:18-33):
 * per-DOF Dirichlet flags (neq bytes) and values (neq, or NULL for 0) */
int icb_dirichlet_mask(icb_problem p, const unsigned char *fixed, const double *val);
/* BCIcarat::input_neumann / generateLoadMain / SurfaceLoad::generate
 * (boundary_condition_icarat.hpp:253-396, boundary_condition_base.cpp:143-180):
 * constant traction val[3] on element sides selected by the box range[6]. */
int icb_traction_box(icb_problem p, const double *val, const double *range);
/* nodal point load (extension: ICARAT's TOML cannot express point/line loads) */
int icb_nodal_load(icb_problem p, long long node, const double *f);
/* BCIcarat::makeDOF -> countDOF (boundary_condition_base.hpp:35-88), load
 * assembly into Force::fext_org, upload to the device.  Returns numeq. */
int icb_finalize(icb_problem p, long long *numeq);
/* BCIcarat::makeDOF -> countDOF (boundary_condition_base.hpp:35-88) on the
 * Dirichlet flags set so far, without freezing the problem: numeq and, when
 * dof is not NULL, the neq-entry numbering.  Lets a caller follow ICARAT's
 * order (makeDOF, then Force(numeq), then input_neumann, then icb_finalize). */
int icb_count_dof(icb_problem p, int *dof, long long *numeq);
/* node[i].dof[j] of countDOF, neq ints */
int icb_get_dof_map(icb_problem p, int *dof);
/* Force::fext_org (numeq) */
int icb_get_load(icb_problem p, double *fext);
/* sizes: nelx, numnp, neq, numeq */
int icb_problem_sizes(icb_problem p, long long *nel, long long *nnode, long long *neq,
                      long long *numeq);
/* unit-modulus element matrix K0 (Ke of LinearElastic::makeKeFint,
 * elasticity.cpp:210-254, with E = 1), (d*ne)^2 row-major */
int icb_get_K0(icb_problem p, double *K0);
/* the element volume (one value: every element of the box grid has it),
 * the sum of Gauss jac of elasticity.cpp:249 */
int icb_element_volume(icb_problem p, double *v);

/* ---- analysis ---------------------------------------------------------- */
/* Elastic::setDesignS for every element (elasticity.hpp:55): the physical
 * (filtered, thresholded) density the stiffness uses. */
int icb_set_density(icb_problem p, const double *rho);
int icb_set_density_device(icb_problem p, const double *rho_dev);
/* LinearAnalysis::solve(solvName, log) (src/analysis/linear.hpp:54-104)
 * with Solvers::solve (src/analysis/solver/solvers.cpp:28-92): Dirichlet
 * values, fres = fext - fint, K(rho) u = fres from u0 = 0 to
 * ||r|| < tol ||fres||.  opts may be NULL (FP64, Jacobi, tol 1e-10). */
int icb_solve(icb_problem p, const icb_solve_opts *opts, icb_solve_info *info);
/* Value::val (numeq) */
int icb_get_displacement(icb_problem p, double *u);
/* node[].val after divideValIntoNode (analysis_utility.hpp:8-31), neq */
int icb_get_node_values(icb_problem p, double *nodeval);
/* value.val . force.fext (opt_macro_oc.cpp:110) */
int icb_compliance(icb_problem p, double *c);
/* sensitivity() of the apps (opt_macro_oc.cpp:182-207,
 * opt_mma_Helmholtz.cpp:173-205): dc_e = -(E'/E) u_e^T Ke u_e; dv_e = v_e
 * (dv may be NULL). */
int icb_sensitivity(icb_problem p, double *dc, double *dv);
/* the same dc on the device (nel doubles, valid until the problem is
 * destroyed or the next sensitivity call); NULL on failure, with the reason in
 * icb_last_error */
const double *icb_sensitivity_device(icb_problem p);
/* Elastic::makeMisesStress (src/problem/elasticity.cpp:165-208) for every
 * element of the last solve: mises[nel] and, when stress is not NULL, the
 * element stress stress[nel * voigt] (voigt order [xx, yy, xy] in 2D,
 * [xx, yy, zz, xy, yz, zx] in 3D), both from the physical density. */
int icb_von_mises(icb_problem p, double *mises, double *stress);
/* node[].reaction after LinearAnalysis::solve (linear.hpp:89-91,
 * assembling.hpp:79-84, analysis_utility.hpp:34-51): the internal force
 * sum_e Ke u_e at every DOF, node-major (neq), |r| < 1e-15 set to 0.  At a
 * free DOF it equals the load; at a constrained DOF it is the reaction. */
int icb_reactions(icb_problem p, double *reaction);
/* K(rho) x over free DOFs (numeq in, numeq out): the product globalK * x of
 * the assembled LinearAnalysis::K() (linear.hpp:31), matrix-free. */
int icb_matvec(icb_problem p, const double *x, double *y);
/* the diagonal of K(rho) over free DOFs (numeq) */
int icb_diagonal(icb_problem p, double *d);

/* ---- filters, projection and design updates ----------------------------- */
/* Filter<E,N>(fem, element, node, radius) (src/optimization/filter.hpp:17-66):
 * neighbour stencil |offset * h| <= radius and the weight sums, on the device */
int icb_cone_create(icb_problem p, double radius, icb_cone *out);
int icb_cone_destroy(icb_cone c);
/* Filter::densityFilter(in, isSens) (filter.hpp:102-151): element arrays */
int icb_cone_filter(icb_cone c, const double *in, double *out, int isSens);
int icb_cone_filter_device(icb_cone c, const double *in, double *out, int isSens);
/* Filter::threshold / thresholdDerivative (filter.hpp:153-185); either output
 * may be NULL */
int icb_threshold(icb_ctx ctx, long long n, const double *x, double beta, double T,
                  double *xhat, double *dxhat);
/* FilterHelmholtz<E,N>(fem, element, node, R) and densityFilter(in,
 * "Eigen_CG", 0, sensFlag) (src/optimization/filter_helm.hpp:28-137) */
int icb_helm_create(icb_problem p, double radius, icb_helm *out);
int icb_helm_destroy(icb_helm h);
int icb_helm_filter(icb_helm h, const double *in, double *out, int sensFlag);
/* OC::UpdateVariables(x, dfdx, g, dgdx, xmin, xmax, gkp1) with setMoveLimit
 * (src/optimization/opt-solver/OCSolver.hpp:20-70); gkp1 is the volume callback
 * of opt_macro_oc.cpp:155-164: sum of threshold(filter(x+)) * v over elements
 * (cone may be NULL: no filter; beta <= 0: no threshold).  steps: bisections. */
int icb_oc_update(icb_problem p, icb_cone cone, double *x, const double *dfdx, double g,
                  const double *dgdx, const double *xmin, const double *xmax,
                  double movelimit, double beta, double T, int *steps);
/* MMASolver(n, m) and Update(x, dfdx, gx, dgdx, xmin, xmax)
 * (src/optimization/opt-solver/MMASolver.hpp:67-78); m must be 1 */
int icb_mma_create(icb_ctx ctx, long long n, int m, icb_mma *out);
int icb_mma_destroy(icb_mma h);
int icb_mma_update(icb_mma h, double *x, const double *dfdx, const double *gx,
                   const double *dgdx, const double *xmin, const double *xmax);
/* GCMMASolver(n, m) (src/optimization/opt-solver/GCMMASolver.hpp:60-90) with
 * a = 0, c = 1000, d = 0; m must be 1.  OuterUpdate (GCMMASolver.cpp:66-89),
 * InnerUpdate (:91-112) and ConCheck (:114-128) as the GCMMA app calls them
 * (opt_macro_gcmma.cpp:153-212). */
int icb_gcmma_create(icb_ctx ctx, long long n, int m, icb_gcmma *out);
int icb_gcmma_destroy(icb_gcmma h);
int icb_gcmma_outer(icb_gcmma h, double *xmma, const double *xval, double f0x,
                    const double *df0dx, const double *fx, const double *dfdx, const double *xmin,
                    const double *xmax);
int icb_gcmma_inner(icb_gcmma h, double *xmma, double f0xnew, const double *fxnew,
                    const double *xval, double f0x, const double *df0dx, const double *fx,
                    const double *dfdx, const double *xmin, const double *xmax);
/* *conservative = 1 when the approximations at the last xmma bound f0xnew, fxnew */
int icb_gcmma_concheck(icb_gcmma h, double f0xnew, const double *fxnew, int *conservative);

/* ---- the ICARAT app loops on the device ----------------------------------- */
#define ICB_FILTER_HELMHOLTZ 0 /* FilterHelmholtz (filter_helm.hpp)              */
#define ICB_FILTER_CONE 1      /* Filter (filter.hpp)                            */

/* Per-step results of a device loop, for the apps' output() (res<step>.vtk,
 * function.csv): host arrays valid during the call.  rho_phys[nel] is the
 * physical (filtered, thresholded) density, nodeval[neq] node[].val,
 * mises[nel] the element von Mises stress. */
typedef void (*icb_step_cb)(void *user, int step, double compliance, const double *rho_phys,
                            const double *nodeval, const double *mises);

typedef struct
{
  int nsteps;           /* optimisation steps (fixed count, no I/O)          */
  double filter_radius; /* cone radius (icb_run_oc) or Helmholtz R (icb_run_mma) */
  double move_limit;    /* OC move limit (0.15 in OCSolver.hpp:78)           */
  int use_threshold;    /* beta = min(2^(step/40), 16) projection (icb_run_oc) */
  double volume_ref;    /* icb_run_mma: V0 of the constraint (<= 0: step-1 volume) */
  icb_solve_opts solve; /* the structural solve of every step                */
  double *iter_seconds; /* optional [nsteps]: wall time of every step (or NULL) */
  int filter_type;      /* icb_run_mma: ICB_FILTER_HELMHOLTZ (0) or ICB_FILTER_CONE */
  /* icb_run_mma, opt-macro-mma-nondesign (opt_macro_mma_nondesign.cpp:120-166):
   * nel flags; flagged elements get zero objective and constraint
   * sensitivities after the filter (NULL: none) */
  const unsigned char *nondesign;
  /* icb_run_mma: nel flags of the elements summed into V0 and the volume
   * constraint (the app's design IDs; NULL: every element) */
  const unsigned char *volume_set;
  icb_step_cb on_step;  /* optional, called after every step's solve      */
  void *step_user;      /* passed to on_step                               */
  /* optional stop rule of the apps' Optimize::isConvergence(eps, minstep)
   * (opt_heat.cpp:121, opt_mma_Helmholtz.cpp:128): once a step's objective
   * differs from the previous step's by less than conv_eps (relative) and
   * step > conv_min_steps, that step's update is completed and the loop
   * ends.  conv_eps <= 0: all nsteps run.  steps_done (may be NULL) receives
   * the number of steps run (icb_server ignores it). */
  double conv_eps;
  int conv_min_steps;
  int *steps_done;
  /* checkpoint and resume (icb_run_oc, icb_run_mma; no counterpart in ICARAT,
   * whose apps only write res<step>.vtk): a run given `checkpoint` (may be
   * NULL) writes there, after its last step, the state the loop carries from
   * step to step -- the design, V0, the stop rule's last objective and for MMA
   * the iteration count, asymptotes and the two previous designs, in
   * icb_loop_checkpoint_bytes(p, kind) bytes.  A run given `resume` (may be
   * NULL) takes that state and continues with the step after the recorded
   * one (rho0 is then ignored; nsteps is still the number of the last step),
   * so a run stopped and resumed, on this problem or another of the same
   * grid, repeats the uninterrupted run bitwise.  hist[step - 1] is written
   * for the steps this call runs.  The job server copies `resume` with the
   * job and ignores `checkpoint`. */
  const void *resume;
  void *checkpoint;
} icb_loop_opts;
/* bytes of a checkpoint of icb_run_oc (kind ICB_JOB_OC) or icb_run_mma
 * (ICB_JOB_MMA) on this problem; < 0 on a bad argument */
long long icb_loop_checkpoint_bytes(icb_problem p, int kind);
/* opt-macro-oc/opt_macro_oc.cpp:84-172: cone filter, threshold, solve,
 * compliance, V0 at step 1, sensitivities, adjoint filter, OC; hist[nsteps]
 * receives the compliance of every step, xout (nel, may be NULL) the design. */
int icb_run_oc(icb_problem p, const icb_loop_opts *o, const double *rho0, double *hist,
               double *xout);
/* opt-mma-HelmholtzFilter/opt_mma_Helmholtz.cpp:81-163: Helmholtz filter,
 * threshold, solve, volume constraint, sensitivities, adjoint filters, MMA. */
int icb_run_mma(icb_problem p, const icb_loop_opts *o, const double *rho0, double *hist,
                double *xout);

/* opt-macro-gcmma (opt_macro_gcmma.cpp:83-238): cone filter of radius
 * filter_radius, threshold beta = min(int(max((step - 100) / 40, 1)), 8),
 * solve, constraint sum x v - V0, GCMMA outer update and up to 15 inner
 * updates per step, each with a full evaluation.  hist[step] is the
 * compliance of the step's design, inner[step] (may be NULL) its inner
 * iterations. */
int icb_run_gcmma(icb_problem p, const icb_loop_opts *o, const double *rho0, double *hist,
                  int *inner, double *xout);

/* ---- heat conduction (LinearHeat, opt-heat) ------------------------------ */
typedef struct icb_heat_s *icb_heat;
/* src/problem/heat.{hpp,cpp}: a structured box of quad4 / hexa8 elements with
 * one temperature per node; conductivities of the two materials as ICARAT's
 * [material] conductivity rows [xx, yy, zz, xy, yz, xz]; SIMP
 * De = rho^p D1 + (1 - rho^p) D2 (heat.cpp:53-64), cond1[0] >= cond2[0]. */
typedef struct
{
  int dim, nx, ny, nz;
  double lx, ly, lz;
  double cond1[6], cond2[6];
  double penalty;
} icb_heat_desc;
/* MeshIcarat setParameter + generate and Heat::setParameter (heat.cpp:18-51)
 * for every element of the box */
int icb_heat_create(icb_ctx ctx, const icb_heat_desc *desc, icb_heat *out);
int icb_heat_destroy(icb_heat h);
/* BCIcarat::input_dirich (boundary_condition_icarat.hpp:68-127) with dofnp 1:
 * fixed temperature `val` where flag != 0 in the box */
int icb_heat_dirichlet_box(icb_heat h, int flag, double val, const double *range);
/* BCIcarat::input_neumann (boundary_condition_icarat.hpp:253-396) with dofnp
 * 1: constant flux q on the element sides of the box */
int icb_heat_flux_box(icb_heat h, double q, const double *range);
/* nodal heat source (extension, like icb_nodal_load) */
int icb_heat_nodal_source(icb_heat h, long long node, double q);
/* makeDOF -> countDOF (boundary_condition_base.hpp:35-88), upload; numeq */
int icb_heat_finalize(icb_heat h, long long *numeq);
/* Heat::setDesign for every element (heat.hpp:35), host array of nel */
int icb_heat_set_density(icb_heat h, const double *rho);
/* LinearAnalysis<LinearHeat>::solve with Eigen_CG: FP64 Jacobi-PCG (opts NULL:
 * tol 1e-10, 10000 iterations) */
int icb_heat_solve(icb_heat h, const icb_solve_opts *opts, icb_solve_info *info);
/* node[].val[0] after divideValIntoNode (analysis_utility.hpp:8-31), nnode */
int icb_heat_get_temperature(icb_heat h, double *nodeval);
/* the app's objective u^T K u over the free DOFs (opt_heat.cpp:116) */
int icb_heat_objective(icb_heat h, double *f);
/* opt_heat.cpp:155-190 without the threshold factor: dc_e = -u_e^T
 * (p rho^(p-1) (K1 - K2)) u_e at the density rho of the solve; dv_e = v_e */
int icb_heat_sensitivity(icb_heat h, const double *rho, double *dc, double *dv);
/* the opt-heat loop (opt_heat.cpp:79-151): Helmholtz filter (filter_radius),
 * threshold, solve, objective, constraint sum x v - V0, MMA; hist[step] is
 * the objective; on_step receives the thresholded design, the temperatures
 * (nnode) and no stress (NULL) */
int icb_run_heat(icb_heat h, const icb_loop_opts *o, const double *rho0, double *hist,
                 double *xout);

/* ---- many runs on one GPU: batch runner and job server ------------------- */
/* No counterpart in ICARAT (one problem per process).  Runs are independent
 * icb_problems; give each one its own icb_ctx (stream) so their kernels
 * overlap.  Results do not depend on what else runs. */
#define ICB_JOB_OC 0  /* icb_run_oc: cone filter + OC (opt_macro_oc)              */
#define ICB_JOB_MMA 1 /* icb_run_mma: Helmholtz filter + MMA (opt_mma_Helmholtz) */
/* run n app loops with nworkers host threads; kinds may be NULL (all OC),
 * xout may be NULL; status[n] (may be NULL) gets each run's status */
int icb_run_batch(int n, const icb_problem *probs, const int *kinds, const icb_loop_opts *opts,
                  const double *const *rho0, double *const *hist, double *const *xout,
                  int nworkers, int *status);

typedef struct icb_server_s *icb_server;
#define ICB_JOB_QUEUED 0
#define ICB_JOB_RUNNING 1
#define ICB_JOB_DONE 2
#define ICB_JOB_CANCELLED 3
typedef struct
{
  icb_grid_desc grid;
  int kind;                   /* ICB_JOB_OC | ICB_JOB_MMA                       */
  icb_loop_opts loop;         /* iter_seconds is ignored (the server keeps them) */
  const unsigned char *fixed; /* neq Dirichlet flags (node-major, interleaved)   */
  const double *load;         /* neq nodal loads                                 */
  const double *rho0;         /* nel initial design                              */
} icb_job_desc;
typedef struct
{
  int state, status;
  double submit_s, start_s, end_s; /* seconds since the server was created */
  long long bytes;                 /* device footprint the job was admitted with */
  int nsteps;
} icb_job_info;
/* estimated device bytes of one run (what admission charges against the budget) */
long long icb_job_footprint(const icb_grid_desc *g, int kind);
/* a server with `slots` workers (one stream each) and an HBM budget: a queued
 * job starts as soon as a worker is free and its footprint fits what the
 * running jobs leave of the budget (the first queued job that fits) */
int icb_server_create(int device, long long budget_bytes, int slots, icb_server *out);
/* copies the job's arrays; ICB_ERR_REJECTED when it can never fit the budget */
int icb_server_submit(icb_server s, const icb_job_desc *job, long long *id);
/* waits up to timeout_s (< 0: forever) for the job; ICB_ERR_TIMEOUT if still running */
int icb_server_wait(icb_server s, long long id, double timeout_s, icb_job_info *info);
/* hist[nsteps], x[nel], iter_seconds[nsteps] (any may be NULL) of a finished job */
int icb_server_result(icb_server s, long long id, double *hist, double *x, double *iter_seconds);
/* cancels a job that has not started (ICB_ERR_STATE otherwise) */
int icb_server_cancel(icb_server s, long long id);
/* drops a finished job's record and results */
int icb_server_forget(icb_server s, long long id);
/* cancels queued jobs, waits for running ones, joins the workers */
int icb_server_destroy(icb_server s);

/* ---- device-level access (benchmarks, interop) --------------------------- */
/* length of one SoA field vector on the device (dim * padded node count):
 * component c of node n sits at c*ld + n, n in MeshIcarat numbering */
long long icb_soa_length(icb_problem p);
/* y = K(rho) x on device SoA vectors of icb_soa_length() entries; precision
 * ICB_FP64 (double*), ICB_MIXED (float*, CUDA cores) or ICB_TF32 (float*,
 * tensor cores, Hex8 only); one operator launch on the context's stream, no
 * synchronisation.  Constrained rows of y are 0. */
int icb_operator_apply_device(icb_problem p, int precision, const void *x, void *y);
/* One Chebyshev smoothing step of the multigrid V-cycle as the library runs it:
 * the operator with its fused update, y <- u + c2 D^-1 (b - K u) + c1 (u - y)
 * (y holds the previous iterate on entry; with c1 = 0 it is not read).  Device
 * SoA vectors of icb_soa_length() entries, double* for ICB_FP64, float* for
 * ICB_MIXED (the FP32 CUDA-core kernel); dinv is the inverse diagonal (0 on
 * constrained DOFs).  One launch on the context's stream, no
 * synchronisation; u and y must differ. */
int icb_smoother_apply_device(icb_problem p, int precision, const void *u, void *y,
                              const void *b, const void *dinv, double c1, double c2);
/* number of kernels this library has launched in the process (graph nodes
 * counted one by one) */
long long icb_launch_count(void);
/* process-wide switches: "tc_operator" (1: the FP32 Hex8 operator inside the
 * ICB_MIXED V-cycle runs on the tcgen05 tensor cores in TF32; 0: CUDA
 * cores); "hex8_modal" (1, the default: CUDA-core Hex8 operators apply K0 in
 * the element's corner-mode basis, 45 multiply-adds per element instead of
 * 576; 0: the dense 24 x 24 product); "device_loops" (1, the default: the
 * multigrid PCG and the OC bisection run their iterations in a CUDA graph's
 * conditional WHILE node, one launch and one host wait each; 0: batches of
 * iterations polled from the host, for profilers that cannot follow
 * conditional graph nodes).  icb_get_option also reports "tc_timeouts"
 * (tensor-core waits that gave up; 0 in a healthy run) and
 * "fused_phase_us_0" .. "fused_phase_us_4" (wall microseconds of the last
 * fused icb_run_batch: building its batched launches, per-design filter and
 * moduli launches, the batched multigrid set-up and solves, compliance /
 * sensitivities / adjoint filters, OC updates with the step's wait),
 * "fused_batch_iters" and "fused_problem_iters" (its solves' iterations: of
 * the batch, and summed over the designs), "fused_active_us_0" .. "_2" and
 * "fused_active_launches_0" .. "_2" (its solves' graph launches, wall
 * microseconds and count, by the share of the batch still iterating when
 * each started: more than a half, more than an eighth, at most an eighth).
 * Further switches: "hex8_pair" (FP32 Hex8 operator with two element rows per
 * thread), "tc_spin_limit" (polls of a tensor-core wait before it gives up),
 * "batch_fused" (icb_run_batch advances qualifying 2D OC batches together),
 * "batch_handoff" (a fused batch's solves hand the designs still iterating to
 * their own solve loops once at most this many are left; 0, the default: an
 * eighth of the batch, at most 32).
 * Unknown names: ICB_ERR_BAD_ARG / -1. */
int icb_set_option(const char *name, long long value);
long long icb_get_option(const char *name);

/* ---- solve without device allocation ------------------------------------ */
/* No counterpart in ICARAT.  For callers that cannot allocate device memory
 * when they solve: hosts that give all GPU memory to their own pool and treat
 * any allocation from outside it as a failure, and real-time or serving loops
 * that must not stall on the allocator or hit out-of-memory mid-request.
 * The same FP64 Jacobi-PCG as icb_solve with ICB_FP64 / ICB_PRECOND_JACOBI
 * (Eigen_CG semantics), on caller-provided device SoA vectors: b_dev holds
 * the right-hand side, x_dev receives the solution; both have
 * icb_soa_length(p) doubles.  b_dev is read on the unknowns only: its
 * constrained slots and the SoA padding past each component's last node are
 * ignored, whatever they hold.  Both must be ready on the context's stream
 * (icb_ctx_stream) when the call is made.  Scratch comes from a 32 MiB static
 * device array that every GPU loading this library holds until exit; problems
 * with icb_soa_length(p) > icb_noalloc_max_soa() are rejected with
 * ICB_ERR_BAD_ARG.  The call allocates nothing: icb_ctx_create looks up the
 * array's device address on its device, which is also when CUDA loads the
 * module holding it and maps its memory, so create the context before the
 * host's pool takes the rest of the GPU.  All calls share the array: calls
 * that overlap on the GPU race, so serialise them.  info->true_relres is -1
 * (not recomputed). */
int icb_solve_noalloc(icb_problem p, const double *b_dev, double *x_dev, double tol, int maxit,
                      icb_solve_info *info);
/* largest icb_soa_length() icb_solve_noalloc accepts */
long long icb_noalloc_max_soa(void);

#ifdef __cplusplus
}
#endif
#endif
