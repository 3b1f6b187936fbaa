// icb_internal.hpp -- shared declarations of the B200 SIMP library.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/icarat_b200.h"
#include <nvtx3/nvToolsExt.h>

namespace icb
{

// ---------------------------------------------------------------- errors --
void set_error(const std::string &msg);
/// add to the process-wide count of kernel launches (icb_launch_count)
void count_launch(long long n = 1);
/// this host thread's share of that count (to undo launches recorded by a capture)
long long thread_launch_count();
struct Error
{
  int code;
  std::string msg;
};
#define ICB_CUDA(call)                                                          \
  do                                                                            \
  {                                                                             \
    cudaError_t e__ = (call);                                                   \
    if(e__ != cudaSuccess)                                                      \
      throw ::icb::Error{e__ == cudaErrorMemoryAllocation ? ICB_ERR_OOM          \
                                                          : ICB_ERR_CUDA,       \
                         std::string(#call) + ": " + cudaGetErrorString(e__)};  \
  } while(0)
#define ICB_REQUIRE(cond, msg)                                                  \
  do                                                                            \
  {                                                                             \
    if(!(cond))                                                                 \
      throw ::icb::Error{ICB_ERR_BAD_ARG, msg};                                 \
  } while(0)
/// the body of every extern "C" entry point: no C++ exception crosses the C
/// ABI; an Error returns its code, a failed host allocation ICB_ERR_OOM, any
/// other exception ICB_ERR_STATE, each with its message in icb_last_error
#define ICB_API_BEGIN try {
#define ICB_API_END                                                             \
  }                                                                             \
  catch(const ::icb::Error &e)                                                  \
  {                                                                             \
    ::icb::set_error(e.msg);                                                    \
    return e.code;                                                              \
  }                                                                             \
  catch(const std::bad_alloc &)                                                 \
  {                                                                             \
    ::icb::set_error("host allocation failed");                                 \
    return ICB_ERR_OOM;                                                         \
  }                                                                             \
  catch(const std::exception &e)                                                \
  {                                                                             \
    ::icb::set_error(e.what());                                                 \
    return ICB_ERR_STATE;                                                       \
  }                                                                             \
  return ICB_OK;

/// a named NVTX range over a host scope (the solve, a loop step and its
/// phases), so Nsight timelines show where the launches of each phase come
/// from; with no profiler attached the calls return at once
struct NvtxRange
{
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

// ---------------------------------------------------------- device memory --
template <typename T> struct DevBuf
{
  T *p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  explicit DevBuf(size_t cnt) { alloc(cnt); }
  DevBuf(const DevBuf &) = delete;
  DevBuf &operator=(const DevBuf &) = delete;
  DevBuf(DevBuf &&o) noexcept : p(o.p), n(o.n) { o.p = nullptr, o.n = 0; }
  DevBuf &operator=(DevBuf &&o) noexcept
  {
    release();
    p = o.p;
    n = o.n;
    o.p = nullptr;
    o.n = 0;
    return *this;
  }
  ~DevBuf() { release(); }
  void alloc(size_t cnt)
  {
    release();
    if(cnt)
      ICB_CUDA(cudaMalloc(&p, cnt * sizeof(T)));
    n = cnt;
  }
  void release()
  {
    if(p)
      cudaFree(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

// ------------------------------------------------------------- geometry --
/// one structured grid (a multigrid level): elements nx*ny(*nz), nodes sx*sy(*sz)
struct Dims
{
  int dim = 3;
  int nx = 0, ny = 0, nz = 1;
  int sx = 0, sy = 0, sz = 1;
  long long nnode = 0, nel = 0;
  long long ld = 0; ///< SoA stride of one displacement component (padded nnode)
};
Dims make_dims(int dim, int nx, int ny, int nz);

/// unit element matrix passed by value to kernels (lives in the constant bank)
template <typename T, int N> struct KMat
{
  T k[N * N];
};

/// reduction scratch: per-block partials + a completion counter.  The block
/// that finishes last sums the partials in block order (deterministic).
struct RedScratch
{
  double *partials = nullptr; ///< [maxBlocks * nvals]
  unsigned *counter = nullptr;
  int maxBlocks = 0;
};

/// device-resident Krylov state (all scalars stay on the GPU between launches)
struct KState
{
  double bb;     ///< ||b||^2
  double thr;    ///< max(tol^2 ||b||^2, DBL_MIN)
  double rz;     ///< r.z of the current iterate
  double rr;     ///< r.r
  double pq;     ///< p.Ap
  double alpha, beta;
  double rzo; ///< r_{k+1}.z_k (flexible CG: Polak-Ribiere beta)
  double tol;
  int iter;      ///< completed iterations (Eigen's count)
  int matvecs;
  int maxit;
  int conv;      ///< converged in the current iteration (x still to update)
  int stop;      ///< no further work: converged, maxit or breakdown
  int status;    ///< ICB_OK, ICB_ERR_MAXITER, ICB_ERR_BREAKDOWN, ICB_ERR_NAN
  int pad;
};

// -------------------------------------------------------------- kernels --
int num_sms();

/// output stage of the element operator
enum OpMode
{
  OP_APPLY = 0,    ///< y = K u
  OP_RESIDUAL = 1, ///< y = b - K u
  OP_JACOBI = 2,   ///< y = u + omega D^-1 (b - K u)
  /// Chebyshev step in three-term form: y = u + c1 (u - y_in) + c2 D^-1 (b - K u),
  /// y_in the previous iterate that y holds on entry (not read when c1 = 0)
  OP_CHEB = 3
};
template <typename T> struct Epi
{
  const T *b;
  const T *dinv;
  T omega;
  T c1, c2;
};
template <typename T> struct OpExtras
{
  int mode = OP_APPLY;
  const T *b = nullptr;
  const T *dinv = nullptr;
  double omega = 0.0;
  double c1 = 0.0, c2 = 0.0;
  RedScratch *dotRed = nullptr; ///< fused u.y reduction (OP_APPLY) into *dotOut
  double *dotOut = nullptr;
  const KState *gate = nullptr; ///< skip when gate->stop (or gate->conv if gateConv)
  int gateConv = 0;
  int cudaCores = 0; ///< 1: the CUDA-core kernel, whatever the tensor-core switch says
};
/// the OC loops of many 2D problems advanced together with batched solves
/// (mgbatch.cu): whether a batch qualifies, and the run (status / message per
/// problem)
bool oc_fused_eligible(int n, icb_problem_s *const *probs, const int *kinds,
                       const icb_loop_opts *opts);
void run_oc_fused(int n, icb_problem_s *const *probs, const icb_loop_opts *opts,
                  const double *const *rho0, double *const *hist, double *const *xout, int *status,
                  std::vector<std::string> &err);
/// wall seconds of phase k of the last fused run (mgbatch.cu)
double fused_phase_seconds(int k);
/// iterations of the last fused run: k = 0 the batch's, 1 the problems' sum
long long fused_iterations(int k);
/// the batched solves' graph launches of the last fused run, binned by the
/// share of the batch still iterating (k = 0: > 1/2, 1: > 1/8, 2: <= 1/8):
/// wall seconds and launches
void fused_active_record(int active, int n, double seconds);
/// designs left when a fused batch hands them to their own solve loops
/// (option batch_handoff; 0: an eighth of the batch, at most 32)
int batch_handoff();
void set_batch_handoff(int k);
double fused_active_seconds(int k);
long long fused_active_launches(int k);
/// whether icb_run_batch uses the fused loop when a batch qualifies (option
/// batch_fused, default on)
bool batch_fused_enabled();
void set_batch_fused(bool on);
/// bytes of an app-loop checkpoint (toapi.cu) for nel elements and a job kind
long long loop_checkpoint_bytes(long long nel, int kind);
/// look up the no-alloc solve's static scratch on the current device
/// (noalloc.cu; called by icb_ctx_create)
void noalloc_prepare_current_device();
/// one Q4 operator launch as data, for the batched launch that runs many of
/// them at once (k_matvec_q4_batch): the element matrix by value, the grid of
/// its own launch (q4_grid) and every argument of k_matvec_q4
template <typename T> struct Q4Launch
{
  KMat<T, 8> K;
  Dims d;
  int ychunk, bx, by, gateConv;
  const T *E, *u;
  T *y;
  const uint8_t *fix;
  RedScratch red;
  double *dotOut;
  const KState *gate;
  Epi<T> ep;
};
/// one 2D diagonal launch (k_diag) as data: its own grid is
/// blocks_for(d.nnode, 256) blocks of 256 threads
template <typename T> struct Diag2Launch
{
  KMat<T, 8> K;
  Dims d;
  const T *E;
  const uint8_t *fix;
  T *invdiag;
};
struct BatchQueue;
template <typename T>
void launch_diag2_batch(const Diag2Launch<T> *D, const int2 *map, const BatchQueue &q,
                        cudaStream_t s);
/// the launch grid of the Q4 operator on d: (bx, by) blocks, ychunk rows each
void q4_grid(const Dims &d, int &bx, int &by, int &ychunk);
/// n Q4 operator launches of one mode as one persistent kernel: D (device, n
/// entries), map (device, one (launch, block) item per block of each
/// launch's own grid) and the work queue over those items (batchq.cuh)
template <typename T>
void launch_q4_batch(const Q4Launch<T> *D, const int2 *map, const BatchQueue &q, int grid,
                     int mode, bool dot, const KMat<T, 8> *uniformK, cudaStream_t s);
/// CTAs of that persistent launch (by the kernel's occupancy), found once when
/// the launch is built, outside any stream capture
template <typename T> int q4_batch_grid(int mode, bool dot, bool uniformK, BatchQueue &q);
/// warps of one block of the Q4 operator, and the resident warps of its
/// batched launch on the whole GPU
int q4_block_warps();
/// reduction slots of the Q4 operator's fused dot (a node row per warp strip)
int q4_dot_slots(const Dims &d);
template <typename T> long long q4_batch_capacity_warps(int mode, bool dot, bool uniformK);

/// tensor-core (tcgen05, TF32) Hex8 operator (operator_tc.cu)
void launch_op_tc(const Dims &d, const float *K, const float *E, const float *u, float *y,
                  const uint8_t *fix, cudaStream_t s, const OpExtras<float> &x);
unsigned tc_timeouts();
/// polls of a tensor-core MMA wait before a CTA gives up, counts a timeout
/// and returns (process-wide; default 2^22)
unsigned tc_spin_limit();
void set_tc_spin_limit(unsigned polls);
/// whether FP32 Hex8 operator launches use the tensor-core kernel
bool tc_operator_enabled();
void set_tc_operator(bool on);
/// whether Hex8 operator launches use the corner-mode kernel when K0 allows it
bool hex8_modal_enabled();
void set_hex8_modal(bool on);
/// whether FP32 corner-mode Hex8 launches run two element rows per thread
bool hex8_pair_enabled();
void set_hex8_pair(bool on);

/// K: HOST pointer to the unit element matrix ((d*ne)^2 entries); it is
/// passed by value, so the kernel's FMAs take it from the constant bank.
template <typename T>
void launch_op(const Dims &d, const T *K, const T *E, const T *u, T *y, const uint8_t *fix,
               cudaStream_t s, const OpExtras<T> &x);

// post-processing (post.cu); icb_problem_s is defined in problem.hpp
void launch_von_mises(const icb_problem_s &p, double *mises, double *stress, cudaStream_t s);
void launch_reactions(icb_problem_s &p, double *out, cudaStream_t s);

// operators (operator.cu): every launcher takes the element matrix as a HOST
// pointer and passes it by value.
template <typename T>
void launch_matvec(const Dims &d, const T *K, const T *E, const T *u, T *y,
                   const uint8_t *fix, cudaStream_t s, RedScratch *dotRed = nullptr,
                   double *dotOut = nullptr, const KState *gate = nullptr);
template <typename T>
void launch_diag(const Dims &d, const T *K, const T *E, const uint8_t *fix, T *invdiag,
                 T *diag, cudaStream_t s);
void launch_gather_free(const Dims &d, const long long *freeIdx, long long numeq,
                        const double *soa, double *numeqv, cudaStream_t s);
void launch_scatter_free(const Dims &d, const long long *freeIdx, long long numeq,
                         const double *numeqv, double *soa, cudaStream_t s);
void launch_simp(long long n, double y1, double y2, double p, const double *rho,
                 double *E, float *Ef, cudaStream_t s);
void launch_sensitivity(const Dims &d, const double *K, double y1, double y2, double p,
                        const double *rho, const double *u, double *dc, cudaStream_t s);

// reductions / vector kernels (krylov.cu)
void launch_dot(long long n, const double *a, const double *b, RedScratch &red,
                double *out, cudaStream_t s);
void launch_axpby(long long n, double a, const double *x, double b, double *y,
                  cudaStream_t s);

} // namespace icb
