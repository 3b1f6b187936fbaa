// loopcache.hpp -- the work space of the app loops (icb_run_oc, icb_run_mma,
// icb_run_gcmma), kept with the problem.  A loop needs a dozen element-sized
// vectors, a filter and an updater; allocating and freeing them on every run
// cost 0.2-0.7 s of cudaMalloc / cudaFree stalls on a 19M-DOF problem whose
// multigrid hierarchies already hold several GB, so repeated runs on one
// problem (a design study, a served job re-run) reuse them instead.  Freed
// with the problem.
#pragma once
#include <memory>
#include <vector>

#include "helm.hpp"
#include "icb_internal.hpp"
#include "opt.hpp"
#include "problem.hpp"

namespace icb
{
struct LoopCache
{
  std::vector<std::unique_ptr<DevBuf<double>>> bufs;
  std::unique_ptr<HelmFilter> helm;
  std::unique_ptr<ConeFilter> cone;
  std::unique_ptr<OcUpdater> oc;
  std::unique_ptr<MmaUpdater> mma;
  std::unique_ptr<GcmmaUpdater> gcmma;

  /// work vector k with at least n entries (contents undefined)
  DevBuf<double> &buf(size_t k, size_t n)
  {
    while(bufs.size() <= k)
      bufs.push_back(std::make_unique<DevBuf<double>>());
    if(bufs[k]->n < n)
      bufs[k]->alloc(n);
    return *bufs[k];
  }
  HelmFilter &helmholtz(const Dims &d, const double *h, double R, cudaStream_t s)
  {
    if(!helm || helm->radius != R)
    {
      helm.reset();
      helm = std::make_unique<HelmFilter>(d, h, R, s);
    }
    return *helm;
  }
  ConeFilter &coneFilter(const Dims &d, const double *h, double R, cudaStream_t s)
  {
    if(!cone || cone->r != R)
    {
      cone.reset();
      cone = std::make_unique<ConeFilter>(d, h, R, s);
    }
    return *cone;
  }
  OcUpdater &ocUpdater(const Dims &d, cudaStream_t s)
  {
    if(!oc)
      oc = std::make_unique<OcUpdater>(d, s);
    return *oc;
  }
  /// a fresh MMA solver state (iteration 0) for a new run
  MmaUpdater &mmaUpdater(long long n, cudaStream_t s)
  {
    if(!mma)
      mma = std::make_unique<MmaUpdater>(n, s);
    else
      mma->reset(s);
    return *mma;
  }
  GcmmaUpdater &gcmmaUpdater(long long n, cudaStream_t s)
  {
    if(!gcmma)
      gcmma = std::make_unique<GcmmaUpdater>(n, s);
    else
      gcmma->reset(s);
    return *gcmma;
  }
};
/// the problem's loop work space, created on first use (toapi.cu)
LoopCache &loop_cache(icb_problem p);
/// a[i] = v; a[i] *= sc * m[i]; *out = sum of a (p's reduction scratch), all
/// asynchronous on the given stream / the problem's stream (toapi.cu)
void launch_fill(long long n, double v, double *a, cudaStream_t s);
void launch_scale_mul(long long n, double *a, const double *m, double sc, cudaStream_t s);
void launch_sum(icb_problem p, const double *a, long long n, double *out);
} // namespace icb
