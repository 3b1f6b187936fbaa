// krylov.cu -- device-resident Jacobi-PCG (FP64 for the drop-in path, FP32
// for inner solves) built from three kernels per iteration:
//   A  q = K p            (matrix-free operator, fused p.q reduction)
//   B  r -= alpha q       (fused r.r and r.D^-1 r reductions, convergence test)
//   C  x += alpha p ; p = D^-1 r + beta p
// All scalars live in a device KState; the last block of each reduction
// updates them, so no host round trip is needed inside the loop.  A batch of
// iterations is captured once as a CUDA graph and relaunched; kernels after
// convergence see `stop` and return at once.
#include <algorithm>
#include <cfloat>
#include <cmath>

#include <functional>

#include "krylov.hpp"
#include "reduce.cuh"

namespace icb
{
int matvec_blocks(const Dims &d);

namespace
{
constexpr int VB = 256;
inline int vec_blocks(long long n)
{
  return int(std::max<long long>(1, std::min<long long>((n + VB - 1) / VB, num_sms() * 8LL)));
}

struct FinInit
{
  KState *st;
  double tol;
  int maxit;
  __device__ void operator()(const double *t) const
  {
    st->bb = t[0];
    st->rr = t[0];
    st->rz = t[1];
    st->tol = tol;
    st->thr = fmax(tol * tol * t[0], DBL_MIN);
    st->iter = 0;
    st->pad = 0;
    st->matvecs = 0;
    st->maxit = maxit;
    st->conv = 0;
    st->alpha = st->beta = 0.0;
    st->status = ICB_OK;
    st->stop = 0;
    if(!isfinite(t[0]) || !isfinite(t[1]))
    {
      st->status = ICB_ERR_NAN;
      st->stop = 1;
    }
    else if(t[0] == 0.0 || t[0] < st->thr)
      st->stop = 1;
  }
};

template <typename T>
__global__ void k_pcg_init(long long n, const T *__restrict__ b, T *__restrict__ x,
                           T *__restrict__ r, T *__restrict__ p, const T *__restrict__ dinv,
                           RedScratch red, KState *st, double tol, int maxit)
{
  double v[2] = {0.0, 0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    // b is read on the unknowns only: the inverse diagonal is 0 on
    // constrained DOFs and on the SoA padding past each component's last
    // node, and whatever a caller's b holds there never enters r
    const T di = dinv[i];
    T bi = di != T(0) ? b[i] : T(0);
    T zi = di * bi;
    r[i] = bi;
    p[i] = zi;
    x[i] = T(0);
    v[0] += double(bi) * double(bi);
    v[1] += double(bi) * double(zi);
  }
  block_reduce<2>(v, red, FinInit{st, tol, maxit});
}

struct FinR
{
  KState *st;
  double pq, alpha;
  bool bad;
  __device__ void operator()(const double *t) const
  {
    st->matvecs++;
    if(bad)
    {
      st->status = ICB_ERR_BREAKDOWN;
      st->stop = 1;
      return;
    }
    st->pq = pq;
    st->alpha = alpha;
    st->rr = t[0];
    if(!isfinite(t[0]) || !isfinite(t[1]))
    {
      st->status = ICB_ERR_NAN;
      st->stop = 1;
    }
    else if(t[0] < st->thr)
      st->conv = 1;
    else
    {
      st->beta = t[1] / st->rz;
      st->rz = t[1];
    }
  }
};

template <typename T>
__global__ void k_pcg_r(long long n, T *__restrict__ r, const T *__restrict__ q,
                        const T *__restrict__ dinv, const double *__restrict__ pq,
                        RedScratch red, KState *st)
{
  if(st->stop)
    return;
  const double pqv = *pq;
  const double alpha = st->rz / pqv;
  const bool bad = !(pqv > 0.0) || !isfinite(alpha);
  double v[2] = {0.0, 0.0};
  if(!bad)
  {
    const T a = T(alpha);
    for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
        i += (long long)gridDim.x * blockDim.x)
    {
      T ri = r[i] - a * q[i];
      r[i] = ri;
      T zi = dinv[i] * ri;
      v[0] += double(ri) * double(ri);
      v[1] += double(ri) * double(zi);
    }
  }
  block_reduce<2>(v, red, FinR{st, pqv, alpha, bad});
}

struct FinXP
{
  KState *st;
  LoopCtl L;
  __device__ void operator()(const double *) const
  {
    if(st->conv)
      st->stop = 1;
    else
    {
      st->iter++;
      if(st->iter >= st->maxit)
      {
        st->status = ICB_ERR_MAXITER;
        st->stop = 1;
      }
    }
    loop_end_krylov(L, st);
  }
};

/// the last kernel of an iteration; inside the solve graph it also decides
/// whether the device runs the next one
template <typename T>
__global__ void k_pcg_xp(long long n, T *__restrict__ x, T *__restrict__ p,
                         const T *__restrict__ r, const T *__restrict__ dinv, RedScratch red,
                         KState *st, LoopCtl L)
{
  if(st->stop)
  {
    if(blockIdx.x == 0 && threadIdx.x == 0)
      loop_stop(L);
    return;
  }
  const T a = T(st->alpha), bt = T(st->beta);
  const bool conv = st->conv;
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
  {
    T pi = p[i];
    x[i] += a * pi;
    if(!conv)
      p[i] = dinv[i] * r[i] + bt * pi;
  }
  double v[1] = {0.0};
  block_reduce<1>(v, red, FinXP{st, L});
}

__global__ void k_dot(long long n, const double *__restrict__ a, const double *__restrict__ b,
                      RedScratch red, double *out)
{
  double v[1] = {0.0};
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    v[0] += a[i] * b[i];
  block_reduce<1>(v, red, FinStore{out});
}

__global__ void k_sub(long long n, const double *__restrict__ b, const double *__restrict__ Ku,
                      double *__restrict__ r)
{
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    r[i] = b[i] - Ku[i];
}
__global__ void k_add(long long n, const double *__restrict__ a, const double *__restrict__ b,
                      double *__restrict__ o)
{
  for(long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
      i += (long long)gridDim.x * blockDim.x)
    o[i] = a[i] + b[i];
}
} // namespace

void launch_axpy_sub(long long n, const double *b, const double *Ku, double *r, cudaStream_t s)
{
  k_sub<<<vec_blocks(n), VB, 0, s>>>(n, b, Ku, r);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
void launch_add(long long n, const double *a, const double *b, double *out, cudaStream_t s)
{
  k_add<<<vec_blocks(n), VB, 0, s>>>(n, a, b, out);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
void launch_dot(long long n, const double *a, const double *b, RedScratch &red, double *out,
                cudaStream_t s)
{
  int nb = vec_blocks(n);
  ICB_REQUIRE(nb <= red.maxBlocks, "reduction scratch too small");
  k_dot<<<nb, VB, 0, s>>>(n, a, b, red, out);
  ICB_CUDA(cudaGetLastError());
  count_launch();
}
double device_dot(long long n, const double *a, const double *b, RedScratch &red,
                  double *scratch, cudaStream_t s)
{
  launch_dot(n, a, b, red, scratch, s);
  double h = 0.0;
  ICB_CUDA(cudaMemcpyAsync(&h, scratch, sizeof(double), cudaMemcpyDeviceToHost, s));
  ICB_CUDA(cudaStreamSynchronize(s));
  return h;
}

int reduction_blocks(const Dims &d)
{
  return std::max(matvec_blocks(d), vec_blocks((long long)d.dim * d.ld));
}

// ------------------------------------------------------------ JacobiPcg --
template <typename T> JacobiPcg<T>::JacobiPcg(const Dims &dims, cudaStream_t s) : d(dims)
{
  n = (long long)d.dim * d.ld;
  r.alloc(n);
  p.alloc(n);
  q.alloc(n);
  // every initialisation goes to the owner's stream: the blocking memset
  // would run on the legacy stream, which non-blocking streams do not wait for
  ICB_CUDA(cudaMemsetAsync(r.p, 0, r.bytes(), s));
  ICB_CUDA(cudaMemsetAsync(p.p, 0, p.bytes(), s));
  ICB_CUDA(cudaMemsetAsync(q.p, 0, q.bytes(), s));
  st.alloc(1);
  int mb = reduction_blocks(d);
  partials.alloc((size_t)mb * 2);
  dots.alloc(4);
  counter.alloc(1);
  ICB_CUDA(cudaMemsetAsync(counter.p, 0, sizeof(unsigned), s));
  red.partials = partials.p;
  red.counter = counter.p;
  red.maxBlocks = mb;
  ICB_CUDA(cudaMallocHost(&hst, sizeof(KState)));
}

template <typename T> JacobiPcg<T>::~JacobiPcg()
{
  if(hst)
    cudaFreeHost(hst);
}

template <typename T>
int JacobiPcg<T>::solve(const T *K, const T *E, const uint8_t *fix, const T *invdiag,
                        const T *b, T *x, double tol, int maxit, cudaStream_t s,
                        icb_solve_info *info)
{
  const Dims dd = d;
  RedScratch *rp = &red;
  double *dp = dots.p;
  KState *sp = st.p;
  T *pp = p.p, *qp = q.p;
  auto op = [=](cudaStream_t cs) {
    launch_matvec<T>(dd, K, E, pp, qp, fix, cs, rp, dp, sp);
  };
  return solveOp(op, K, E, fix, invdiag, b, x, tol, maxit, s, info);
}

template <typename T>
int JacobiPcg<T>::solveOp(const std::function<void(cudaStream_t)> &op, const void *opKey0,
                          const void *opKey1, const void *opKey2, const T *invdiag, const T *b,
                          T *x, double tol, int maxit, cudaStream_t s, icb_solve_info *info)
{
  cudaEvent_t e0, e1;
  ICB_CUDA(cudaEventCreate(&e0));
  ICB_CUDA(cudaEventCreate(&e1));
  ICB_CUDA(cudaEventRecord(e0, s));
  const int nb = vec_blocks(n);
  k_pcg_init<T><<<nb, VB, 0, s>>>(n, b, x, r.p, p.p, invdiag, red, st.p, tol, maxit);
  ICB_CUDA(cudaGetLastError());
  count_launch();

  // (re)capture the batch graph when the operands changed: 16 iterations per
  // launch, polled from the host (a device-side WHILE loop was measured at
  // the same speed here, 251 against 249 ms for the c2 solve, and profilers
  // cannot follow its kernels)
  GraphKey key;
  key.add(opKey0).add(opKey1).add(opKey2).add(invdiag).add(x).add((const void *)s);
  key.add((long long)kernel_switches());
  if(loop.exec == nullptr || key != graphKey)
  {
    KState *stp = st.p;
    const long long before = thread_launch_count();
    loop.build(
        [&](cudaStream_t cs, const LoopCtl &L) {
          op(cs); // q = K p with the fused p.q reduction into dots[0]
          k_pcg_r<T><<<nb, VB, 0, cs>>>(n, r.p, q.p, invdiag, dots.p, red, stp);
          k_pcg_xp<T><<<nb, VB, 0, cs>>>(n, x, p.p, r.p, invdiag, red, stp, L);
        },
        false, 16);
    count_launch(before - thread_launch_count()); // recorded, not launched
    graphKey = key;
  }
  long long launched = 0;
  for(;;)
  {
    ICB_CUDA(cudaMemcpyAsync(hst, st.p, sizeof(KState), cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    if(hst->stop)
      break;
    if(launched > (long long)maxit + loop.batch)
      break; // device bookkeeping stops at maxit; this is a host-side backstop
    loop.launch(s);
    launched += loop.batch;
    count_launch(loop.graphNodes);
  }
  ICB_CUDA(cudaEventRecord(e1, s));
  ICB_CUDA(cudaEventSynchronize(e1));
  float ms = 0.f;
  cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if(info)
  {
    info->iters = hst->iter;
    info->matvecs = hst->matvecs;
    info->relres = hst->bb > 0 ? std::sqrt(hst->rr / hst->bb) : 0.0;
    info->seconds = ms * 1e-3;
    info->status = hst->status;
  }
  return hst->status;
}

template struct JacobiPcg<double>;
template struct JacobiPcg<float>;

/// Jacobi-PCG with every buffer supplied by the caller and no CUDA graph:
/// the same three kernels per iteration as JacobiPcg, launched directly, the
/// stop flag polled every 16 iterations into a caller-owned host KState.
int pcg_run_external(const Dims &d, const double *K, const double *E, const uint8_t *fix,
                     const double *invdiag, const double *b, double *x, double *r, double *p,
                     double *q, double *dotOut, KState *st, RedScratch red, double tol,
                     int maxit, cudaStream_t s, KState *hostState)
{
  const long long n = (long long)d.dim * d.ld;
  const int nb = vec_blocks(n);
  ICB_REQUIRE(reduction_blocks(d) <= red.maxBlocks, "reduction scratch too small");
  k_pcg_init<double><<<nb, VB, 0, s>>>(n, b, x, r, p, invdiag, red, st, tol, maxit);
  ICB_CUDA(cudaGetLastError());
  count_launch();
  long long launched = 0;
  for(;;)
  {
    ICB_CUDA(cudaMemcpyAsync(hostState, st, sizeof(KState), cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    if(hostState->stop || launched > (long long)maxit + 16)
      break;
    for(int it = 0; it < 16; it++)
    {
      launch_matvec<double>(d, K, E, p, q, fix, s, &red, dotOut, st);
      k_pcg_r<double><<<nb, VB, 0, s>>>(n, r, q, invdiag, dotOut, red, st);
      k_pcg_xp<double><<<nb, VB, 0, s>>>(n, x, p, r, invdiag, red, st, LoopCtl{});
      count_launch(2);
    }
    ICB_CUDA(cudaGetLastError());
    launched += 16;
  }
  return hostState->status;
}


} // namespace icb
