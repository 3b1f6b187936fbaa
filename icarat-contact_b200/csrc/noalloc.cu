// noalloc.cu -- icb_solve_noalloc: the FP64 Jacobi-PCG solve for callers
// that must not allocate device memory.
//
// Some callers cannot call cudaMalloc at the point where they need a solve:
// hosts that hand the whole GPU memory to their own pool up front and treat
// any allocation from outside it as a failure, and real-time or serving loops
// that must not risk an allocator stall or an out-of-memory error in the
// middle of a request.  For them this entry point
// takes its scratch (three Krylov vectors, the reduction partials, the
// completion counter and the device-side solver state) from one file-scope
// device array instead of allocating it.
//
// Limits and rules (also in include/icarat_b200.h):
//  * the array holds kNoAllocBytes (32 MiB) on every GPU that loads this
//    library, until the process exits;
//  * problems whose SoA field length (icb_soa_length) exceeds
//    kNoAllocMaxSoa are rejected with ICB_ERR_BAD_ARG;
//  * the array's device address is looked up with cudaGetSymbolAddress (in
//    host code the array's name is a host-side stand-in, not a device
//    address) once per device when icb_ctx_create opens a context on it.
//    That lookup also makes CUDA load this module (CUDA and torch load
//    modules lazily), which is when the array gets its device memory, so a
//    host that gives the rest of the GPU to its own pool afterwards still
//    finds the array in place, and no solve call maps or allocates anything;
//  * every call shares the array: calls that overlap on the GPU (different
//    streams, or several host threads) race and must be serialised by the
//    caller.  Each call clears what has to start at zero (the completion
//    counter and the q vector) and initialises the rest itself.
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>

#include "problem.hpp"
#include "krylov.hpp"

namespace
{
constexpr size_t kNoAllocBytes = size_t(32) << 20;
constexpr int kNoAllocMaxBlocks = 32768;
constexpr size_t align256(size_t v) { return (v + 255) & ~size_t(255); }
// layout: [KState][counter][pq][partials: 2*kNoAllocMaxBlocks][r][p][q]
constexpr size_t kOffState = 0;
constexpr size_t kOffCounter = align256(kOffState + sizeof(icb::KState));
constexpr size_t kOffDot = align256(kOffCounter + sizeof(unsigned));
constexpr size_t kOffPartials = align256(kOffDot + 4 * sizeof(double));
constexpr size_t kOffVectors = align256(kOffPartials + 2 * kNoAllocMaxBlocks * sizeof(double));
/// largest SoA length (dim * padded node count) three FP64 vectors can hold
constexpr long long kNoAllocMaxSoa =
    (long long)((kNoAllocBytes - kOffVectors) / (3 * sizeof(double)) / 64 * 64);

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

constexpr int kMaxDevices = 64;
static std::atomic<void *> g_scratch_ptr[kMaxDevices] = {};

/// device address of the scratch array on the current device, looked up on
/// the first call for that device (icb_ctx_create makes that call)
unsigned char *scratchOnCurrentDevice()
{
  int dev = 0;
  ICB_CUDA(cudaGetDevice(&dev));
  if(dev < 0 || dev >= kMaxDevices)
    throw icb::Error{ICB_ERR_BAD_ARG, "device ordinal out of range for the no-alloc solve"};
  void *ptr = g_scratch_ptr[dev].load();
  if(!ptr)
  {
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if(e != cudaSuccess || !ptr)
      throw icb::Error{ICB_ERR_CUDA, std::string("cudaGetSymbolAddress(no-alloc scratch): ") +
                                         cudaGetErrorString(e)};
    g_scratch_ptr[dev].store(ptr);
  }
  return static_cast<unsigned char *>(ptr);
}
} // namespace

namespace icb
{
/// look up the no-alloc scratch on the current device now, at context
/// creation, so the module holding it is loaded before any solve
void noalloc_prepare_current_device() { (void)scratchOnCurrentDevice(); }
} // namespace icb

extern "C" {

long long icb_noalloc_max_soa(void) { return kNoAllocMaxSoa; }

int icb_solve_noalloc(icb_problem p, const double *b_dev, double *x_dev, double tol, int maxit,
                      icb_solve_info *info)
{
  ICB_API_BEGIN
  if(!p || !b_dev || !x_dev)
    throw icb::Error{ICB_ERR_BAD_ARG, "NULL argument"};
  if(!p->hasDensity)
    throw icb::Error{ICB_ERR_STATE, "set the density first"};
  if(!(tol >= 0.0) || maxit <= 0)
    throw icb::Error{ICB_ERR_BAD_ARG, "bad tolerance / iteration limit"};
  if(p->nsoa > kNoAllocMaxSoa)
    throw icb::Error{ICB_ERR_BAD_ARG,
                     "problem too large for icb_solve_noalloc: SoA length " +
                         std::to_string(p->nsoa) + " exceeds the static scratch limit " +
                         std::to_string(kNoAllocMaxSoa)};
  if(icb::reduction_blocks(p->d) > kNoAllocMaxBlocks)
    throw icb::Error{ICB_ERR_BAD_ARG, "grid needs more reduction slots than the no-alloc scratch has"};
  ICB_CUDA(cudaSetDevice(p->ctx->device));
  unsigned char *base = scratchOnCurrentDevice();
  cudaStream_t s = p->stream();
  auto t0 = std::chrono::steady_clock::now();
  // what must start at zero: the completion counter, and q, whose padding
  // slots (past the last node of each component) the operator never writes
  // but the residual update reads; the array keeps the previous call's
  // contents, so both are cleared on every call.  r, p, x and the state are
  // written in full before they are read.
  ICB_CUDA(cudaMemsetAsync(base + kOffCounter, 0, sizeof(unsigned), s));
  icb::KState *st = reinterpret_cast<icb::KState *>(base + kOffState);
  double *dot = reinterpret_cast<double *>(base + kOffDot);
  icb::RedScratch red{reinterpret_cast<double *>(base + kOffPartials),
                      reinterpret_cast<unsigned *>(base + kOffCounter), kNoAllocMaxBlocks};
  double *r = reinterpret_cast<double *>(base + kOffVectors);
  double *pv = r + p->nsoa;
  double *q = pv + p->nsoa;
  ICB_CUDA(cudaMemsetAsync(q, 0, sizeof(double) * p->nsoa, s));
  // the inverse diagonal goes to the problem's own (already allocated) array
  icb::launch_diag<double>(p->d, p->K0, p->E.p, p->fix.p, p->dinv.p, nullptr, s);
  icb::KState hs; // pageable host copy: no pinned allocation
  int status = icb::pcg_run_external(p->d, p->K0, p->E.p, p->fix.p, p->dinv.p, b_dev, x_dev,
                                     r, pv, q, dot, st, red, tol, maxit, s, &hs);
  double sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if(info)
  {
    std::memset(info, 0, sizeof(*info));
    info->iters = hs.iter;
    info->matvecs = hs.matvecs;
    info->outer = 1;
    info->relres = hs.bb > 0 ? std::sqrt(hs.rr / hs.bb) : 0.0;
    info->true_relres = -1.0; // not recomputed: that would need a fourth vector
    info->seconds = sec;
    info->status = status;
  }
  if(status != ICB_OK)
    icb::set_error(status == ICB_ERR_MAXITER ? "iteration limit reached"
                                             : "CG breakdown or non-finite values");
  return status;
  ICB_API_END
}

} // extern "C"
