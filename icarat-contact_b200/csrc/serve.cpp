// serve.cpp -- many independent topology-optimisation runs on one GPU:
// the batch runner (icb_run_batch) and the continuous-batching job server
// (icb_server_*).  No counterpart in ICARAT, which runs one problem per
// process (linear.hpp:15-41 holds its state by reference).
//
// Design: every run is an ordinary icb_problem on its own CUDA stream; a pool
// of host workers drives the runs through icb_run_oc / icb_run_mma, so the
// kernels of different runs overlap on the device (each run's solver batches
// are CUDA graphs, its host waits are per-stream).  The server admits a
// queued job as soon as a worker slot is free and the job's estimated device
// footprint fits in what is left of the HBM budget (first job in queue order
// that fits: small jobs may pass a large one that is waiting for memory), so
// jobs arriving while others are running join them immediately.  Every run is
// deterministic and independent of the others: its results are the same
// alone and in any mix.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <system_error>
#include <thread>
#include <vector>

#include "problem.hpp"

using namespace icb;

namespace
{
using Clock = std::chrono::steady_clock;

int runOne(icb_problem p, int kind, const icb_loop_opts &o, const double *rho0, double *hist,
           double *x)
{
  return kind == ICB_JOB_MMA ? icb_run_mma(p, &o, rho0, hist, x) : icb_run_oc(p, &o, rho0, hist, x);
}
} // namespace

// ================================================================= jobs ====
struct Job
{
  long long id = 0;
  icb_grid_desc grid{};
  int kind = ICB_JOB_OC;
  icb_loop_opts loop{};
  std::vector<unsigned char> fixed, nondesign, volumeSet;
  std::vector<double> load, rho0, hist, x, iters;
  std::vector<char> resumeBlob; ///< the checkpoint a resumed job starts from
  long long bytes = 0;
  int state = ICB_JOB_QUEUED;
  int status = ICB_OK;
  std::string error;
  double submit = 0, start = 0, end = 0;
};

struct icb_server_s
{
  int device = 0;
  long long budget = 0, inUse = 0;
  int slots = 1;
  std::mutex mu;
  std::condition_variable cv;     ///< queue / shutdown changes (workers wait)
  std::condition_variable doneCv; ///< job completions (waiters)
  std::deque<std::shared_ptr<Job>> queue;
  std::map<long long, std::shared_ptr<Job>> jobs;
  std::vector<std::thread> workers;
  bool stopping = false;
  long long nextId = 1;
  Clock::time_point t0 = Clock::now();

  double now() const { return std::chrono::duration<double>(Clock::now() - t0).count(); }

  /// next job that fits the remaining budget (queue order), or null
  std::shared_ptr<Job> takeFitting()
  {
    for(auto it = queue.begin(); it != queue.end(); ++it)
      if(inUse + (*it)->bytes <= budget)
      {
        auto j = *it;
        queue.erase(it);
        return j;
      }
    return nullptr;
  }

  void worker()
  {
    // a worker without a context still takes jobs and fails them with the
    // context's error, so no admitted job waits for ever
    icb_ctx ctx = nullptr;
    const int ctxStatus = icb_ctx_create(device, &ctx);
    const std::string ctxError = ctxStatus == ICB_OK ? "" : icb_last_error();
    for(;;)
    {
      std::shared_ptr<Job> j;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return stopping || (j = takeFitting()) != nullptr; });
        if(!j)
          break; // stopping and nothing admissible
        inUse += j->bytes;
        j->state = ICB_JOB_RUNNING;
        j->start = now();
      }
      int st = ctxStatus;
      icb_problem p = nullptr;
      if(st == ICB_OK)
        st = icb_problem_create(ctx, &j->grid, &p);
      if(st == ICB_OK)
        st = icb_dirichlet_mask(p, j->fixed.data(), nullptr);
      if(st == ICB_OK)
      {
        const int dim = j->grid.dim;
        long long nnode = (long long)j->load.size() / dim;
        for(long long n = 0; n < nnode && st == ICB_OK; n++)
        {
          bool any = false;
          for(int c = 0; c < dim; c++)
            any = any || j->load[n * dim + c] != 0.0;
          if(any)
            st = icb_nodal_load(p, n, &j->load[n * dim]);
        }
      }
      long long numeq = 0;
      if(st == ICB_OK)
        st = icb_finalize(p, &numeq);
      if(st == ICB_OK)
      {
        icb_loop_opts o = j->loop;
        o.iter_seconds = j->iters.data();
        st = runOne(p, j->kind, o, j->rho0.empty() ? nullptr : j->rho0.data(), j->hist.data(),
                    j->x.data());
      }
      std::string err = st == ICB_OK ? "" : ctxStatus != ICB_OK ? ctxError : icb_last_error();
      icb_problem_destroy(p);
      {
        std::lock_guard<std::mutex> lk(mu);
        inUse -= j->bytes;
        j->status = st;
        j->error = err;
        j->state = ICB_JOB_DONE;
        j->end = now();
      }
      doneCv.notify_all();
      cv.notify_all(); // memory was released: a waiting job may fit now
    }
    icb_ctx_destroy(ctx);
  }
};

namespace
{
/// cancels the queued jobs, lets the running ones finish and joins the workers
void stopAll(icb_server_s &s)
{
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stopping = true;
    for(auto &j : s.queue)
    {
      j->state = ICB_JOB_CANCELLED;
      j->status = ICB_ERR_STATE;
      j->error = "server stopped";
    }
    s.queue.clear();
  }
  s.cv.notify_all();
  s.doneCv.notify_all();
  for(auto &t : s.workers)
    t.join();
}
} // namespace

extern "C" {

long long icb_job_footprint(const icb_grid_desc *g, int kind)
{
  if(!g || (g->dim != 2 && g->dim != 3))
    return -1;
  Dims d = make_dims(g->dim, g->nx, g->ny, g->dim == 3 ? g->nz : 1);
  long long nsoa = (long long)d.dim * d.ld;
  // problem vectors (8 FP64 fields) + Jacobi/Krylov (5 FP64 + 2 FP32) + the
  // multigrid hierarchy (<= 8/7 of 6 FP32 fields) + per-element arrays of the
  // problem and the loop (~20 FP64) + filters, graphs and scratch
  long long b = nsoa * (8 * 13 + 4 * 2) + (long long)(nsoa * 8.0 / 7.0) * 4 * 6 +
                d.nel * 8 * 20 + d.nnode * 8 * (kind == ICB_JOB_MMA ? 8 : 1) + (48ll << 20);
  return b;
}

int icb_server_create(int device, long long budget_bytes, int slots, icb_server *out)
{
  ICB_API_BEGIN
  if(!out || slots < 1 || budget_bytes <= 0)
    throw Error{ICB_ERR_BAD_ARG, "bad server arguments"};
  auto s = std::make_unique<icb_server_s>();
  s->device = device;
  s->budget = budget_bytes;
  s->slots = slots;
  try
  {
    for(int i = 0; i < slots; i++)
    {
      icb_server_s *raw = s.get();
      s->workers.emplace_back([raw] { raw->worker(); });
    }
  }
  catch(...)
  {
    // a thread that could not start: stop and join the ones that did
    stopAll(*s);
    throw;
  }
  *out = s.release();
  ICB_API_END
}

int icb_server_submit(icb_server s, const icb_job_desc *jd, long long *id)
{
  ICB_API_BEGIN
  if(!s || !jd || !jd->fixed || !jd->load || !(jd->rho0 || jd->loop.resume) ||
     jd->loop.nsteps <= 0)
    throw Error{ICB_ERR_BAD_ARG, "bad job"};
  if(jd->kind != ICB_JOB_OC && jd->kind != ICB_JOB_MMA)
    throw Error{ICB_ERR_BAD_ARG, "job kind must be ICB_JOB_OC or ICB_JOB_MMA"};
  const icb_grid_desc &g = jd->grid;
  if((g.dim != 2 && g.dim != 3) || g.nx < 1 || g.ny < 1 || (g.dim == 3 && g.nz < 1))
    throw Error{ICB_ERR_BAD_ARG, "bad grid"};
  auto j = std::make_shared<Job>();
  j->grid = g;
  j->kind = jd->kind;
  j->loop = jd->loop;
  j->loop.iter_seconds = nullptr;
  j->loop.steps_done = nullptr; // the caller's memory is not written later
  j->loop.checkpoint = nullptr;
  Dims d = make_dims(g.dim, g.nx, g.ny, g.dim == 3 ? g.nz : 1);
  long long neq = d.nnode * g.dim;
  j->fixed.assign(jd->fixed, jd->fixed + neq);
  j->load.assign(jd->load, jd->load + neq);
  if(jd->rho0)
    j->rho0.assign(jd->rho0, jd->rho0 + d.nel);
  // the element masks are copied like the other arrays; on_step (if set) is
  // called on the worker thread that runs the job
  if(jd->loop.nondesign)
  {
    j->nondesign.assign(jd->loop.nondesign, jd->loop.nondesign + d.nel);
    j->loop.nondesign = j->nondesign.data();
  }
  if(jd->loop.volume_set)
  {
    j->volumeSet.assign(jd->loop.volume_set, jd->loop.volume_set + d.nel);
    j->loop.volume_set = j->volumeSet.data();
  }
  if(jd->loop.resume)
  {
    // a resumed job: the checkpoint of an earlier run of this grid and kind
    const char *b = static_cast<const char *>(jd->loop.resume);
    j->resumeBlob.assign(b, b + loop_checkpoint_bytes(d.nel, jd->kind));
    j->loop.resume = j->resumeBlob.data();
  }
  j->hist.assign(jd->loop.nsteps, 0.0);
  j->iters.assign(jd->loop.nsteps, 0.0);
  j->x.assign(d.nel, 0.0);
  j->bytes = icb_job_footprint(&g, jd->kind);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if(j->bytes > s->budget)
      throw Error{ICB_ERR_REJECTED, "job needs more device memory than the server budget"};
    j->id = s->nextId++;
    j->submit = s->now();
    s->jobs[j->id] = j;
    s->queue.push_back(j);
  }
  s->cv.notify_all();
  if(id)
    *id = j->id;
  ICB_API_END
}

int icb_server_wait(icb_server s, long long id, double timeout_s, icb_job_info *info)
{
  if(!s)
    return ICB_ERR_BAD_ARG;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if(it == s->jobs.end())
  {
    set_error("unknown job id");
    return ICB_ERR_BAD_ARG;
  }
  auto j = it->second;
  auto pred = [&] { return j->state == ICB_JOB_DONE || j->state == ICB_JOB_CANCELLED; };
  if(timeout_s < 0)
    s->doneCv.wait(lk, pred);
  else if(!s->doneCv.wait_for(lk, std::chrono::duration<double>(timeout_s), pred))
  {
    if(info)
    {
      info->state = j->state;
      info->status = ICB_OK;
    }
    set_error("job still running");
    return ICB_ERR_TIMEOUT;
  }
  if(info)
  {
    info->state = j->state;
    info->status = j->status;
    info->submit_s = j->submit;
    info->start_s = j->start;
    info->end_s = j->end;
    info->bytes = j->bytes;
    info->nsteps = j->loop.nsteps;
  }
  if(j->status != ICB_OK)
    set_error(j->error);
  return j->status;
}

int icb_server_result(icb_server s, long long id, double *hist, double *x, double *iter_seconds)
{
  if(!s)
    return ICB_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if(it == s->jobs.end() || it->second->state != ICB_JOB_DONE)
  {
    set_error("job unknown or not finished");
    return ICB_ERR_STATE;
  }
  auto &j = *it->second;
  if(hist)
    std::memcpy(hist, j.hist.data(), sizeof(double) * j.hist.size());
  if(x)
    std::memcpy(x, j.x.data(), sizeof(double) * j.x.size());
  if(iter_seconds)
    std::memcpy(iter_seconds, j.iters.data(), sizeof(double) * j.iters.size());
  return j.status;
}

int icb_server_cancel(icb_server s, long long id)
{
  if(!s)
    return ICB_ERR_BAD_ARG;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(id);
    if(it == s->jobs.end())
    {
      set_error("unknown job id");
      return ICB_ERR_BAD_ARG;
    }
    auto j = it->second;
    if(j->state != ICB_JOB_QUEUED)
    {
      set_error("only queued jobs can be cancelled");
      return ICB_ERR_STATE;
    }
    s->queue.erase(std::remove(s->queue.begin(), s->queue.end(), j), s->queue.end());
    j->state = ICB_JOB_CANCELLED;
    j->status = ICB_ERR_STATE;
    j->error = "cancelled";
  }
  s->doneCv.notify_all();
  return ICB_OK;
}

int icb_server_forget(icb_server s, long long id)
{
  if(!s)
    return ICB_ERR_BAD_ARG;
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->jobs.find(id);
  if(it == s->jobs.end())
    return ICB_ERR_BAD_ARG;
  if(it->second->state != ICB_JOB_DONE && it->second->state != ICB_JOB_CANCELLED)
    return ICB_ERR_STATE;
  s->jobs.erase(it);
  return ICB_OK;
}

int icb_server_destroy(icb_server s)
{
  if(!s)
    return ICB_OK;
  stopAll(*s);
  delete s;
  return ICB_OK;
}

int icb_run_batch(int n, const icb_problem *probs, const int *kinds, const icb_loop_opts *opts,
                  const double *const *rho0, double *const *hist, double *const *xout,
                  int nworkers, int *status)
{
  ICB_API_BEGIN
  if(n < 0 || !probs || !opts || !rho0 || !hist || nworkers < 1)
    throw Error{ICB_ERR_BAD_ARG, "bad batch arguments"};
  std::atomic<int> next{0};
  std::vector<int> st(n, ICB_OK);
  std::vector<std::string> err(n);
  if(batch_fused_enabled() && oc_fused_eligible(n, probs, kinds, opts))
  {
    // every loop advances together, the solves as batched launches
    run_oc_fused(n, probs, opts, rho0, hist, xout, st.data(), err);
    nworkers = 0;
  }
  auto work = [&] {
    for(int i; (i = next.fetch_add(1)) < n;)
    {
      st[i] = runOne(probs[i], kinds ? kinds[i] : ICB_JOB_OC, opts[i], rho0[i], hist[i],
                     xout ? xout[i] : nullptr);
      if(st[i] != ICB_OK)
        err[i] = icb_last_error();
    }
  };
  std::vector<std::thread> th;
  try
  {
    for(int w = 0; w < std::min(nworkers, std::max(n, 1)); w++)
      th.emplace_back(work);
  }
  catch(const std::system_error &)
  {
    // fewer threads than asked for: the ones that started take every instance
  }
  if(th.empty() && nworkers > 0)
    work();
  for(auto &t : th)
    t.join();
  int first = ICB_OK;
  for(int i = 0; i < n; i++)
  {
    if(status)
      status[i] = st[i];
    if(st[i] != ICB_OK && first == ICB_OK)
    {
      first = st[i];
      set_error("instance " + std::to_string(i) + ": " + err[i]);
    }
  }
  return first;
  ICB_API_END
}

} // extern "C"
