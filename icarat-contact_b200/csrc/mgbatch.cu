// mgbatch.cu -- the multigrid-preconditioned solves of many independent
// problems as one sequence of batched launches, and the OC loop of many
// problems advancing together (the batched form of icb_run_batch).
//
// ICARAT solves one problem per process (src/analysis/linear.hpp:15-41).  A
// batch of small, uneven 2D designs run one at a time leaves the GPU idle:
// each FCG iteration of a 100k-element problem is ~50 kernels of a few
// microseconds.  Here every kernel of an iteration (the Krylov operator and
// vector updates, and per V-cycle level the smoother, residual, transfers
// and coarse solve) is launched once for all problems: block b of a batched
// launch looks up (problem, block) in a map and runs that block of that
// problem's own launch -- same grid, same arithmetic, same reduction order
// (block_reduce_at) -- so each problem's iterates are bitwise those of its
// own solve.  A problem that has converged is gated out (its blocks return at
// once), as in its own solve.  Problems whose hierarchies have fewer levels
// reach their coarsest solve earlier; a batched launch holds the problems
// that take that step at that point of the V-cycle.
#include <atomic>
#include <chrono>
#include <cstring>
#include <memory>

#include "loopcache.hpp"
#include "batchq.cuh"
#include "mg_impl.cuh"
#include "opt.hpp"

namespace icb
{
namespace
{
/// persistent CTAs take (record, block) items from the queue; block b of a
/// record is block b of that problem's own launch (its own grid)
template <class L>
__global__ void k_batch(const L *__restrict__ D, const int2 *__restrict__ map, BatchQueue q)
{
  batch_queue(
      D, map, q, [](const L &l) { return int(l.g.gx * l.g.gy * l.g.gz); },
      [](const L &l) { return l.skip(); },
      [](const L &l, int bi, bool) {
        const unsigned b = unsigned(bi);
        const Blk B{b % l.g.gx, (b / l.g.gx) % l.g.gy, b / (l.g.gx * l.g.gy), l.g.gx, l.g.gy,
                    l.g.gz};
        l.run(B);
      });
}

// the per-problem launches as records: the kernel's arguments and its grid
template <typename TK, typename TP> struct InitL
{
  Blk g;
  long long n;
  const TK *b;
  TK *x, *r;
  TP *rP;
  RedScratch red;
  KState *st;
  double tol;
  int maxit;
  __device__ bool skip() const { return false; }
  __device__ void run(const Blk &B) const { mg_init_b<TK, TP>(n, b, x, r, rP, red, st, tol, maxit, B); }
};
template <typename TK, typename TP> struct Init2L
{
  Blk g;
  long long n;
  const TK *r;
  const TP *z;
  TK *p;
  RedScratch red;
  KState *st;
  __device__ bool skip() const { return st->stop != 0; }
  __device__ void run(const Blk &B) const { mg_init2_b<TK, TP>(n, r, z, p, red, st, B); }
};
template <typename TK, typename TP> struct RL
{
  Blk g;
  long long n;
  TK *r;
  TP *rP;
  const TK *q;
  const TP *z;
  const double *pq;
  RedScratch red;
  KState *st;
  __device__ bool skip() const { return st->stop != 0; }
  __device__ void run(const Blk &B) const { mg_r_b<TK, TP>(n, r, rP, q, z, pq, red, st, B); }
};
template <typename TK, typename TP> struct RzL
{
  Blk g;
  long long n;
  const TK *r;
  const TP *z;
  RedScratch red;
  KState *st;
  __device__ bool skip() const { return st->stop || st->conv; }
  __device__ void run(const Blk &B) const { mg_rz_b<TK, TP>(n, r, z, red, st, B); }
};
template <typename TK, typename TP> struct XpL
{
  Blk g;
  long long n;
  TK *x, *p;
  const TP *z;
  RedScratch red;
  KState *st;
  __device__ bool skip() const { return st->stop != 0; }
  __device__ void run(const Blk &B) const { mg_xp_b<TK, TP>(n, x, p, z, red, st, LoopCtl{}, B); }
};
template <typename T> struct Jacobi0L
{
  Blk g;
  long long n;
  T c;
  const T *dinv, *b;
  T *x, *x0;
  const KState *gate;
  __device__ bool skip() const { return gated(gate); }
  __device__ void run(const Blk &B) const { jacobi0_b<T>(n, c, dinv, b, x, x0, gate, B); }
};
/// the transfers write each node from its own reads only, so a batched
/// launch may give a block several node rows: g.gy blocks take the ry rows
/// of the per-problem grid (same results, far fewer tiny blocks)
template <typename T> struct RestrictL
{
  Blk g;
  Dims df, dc;
  int3 sh;
  const T *rf;
  T *bc;
  const uint8_t *fixc;
  const KState *gate;
  unsigned ry;
  __device__ bool skip() const { return gated(gate); }
  __device__ void run(const Blk &B) const
  {
    Blk b = B;
#pragma unroll 2
    for(b.y = B.y; b.y < ry; b.y += B.gy)
      restrict_b<T>(df, dc, sh, rf, bc, fixc, gate, b);
  }
};
/// g.gy blocks along y, each ry node rows from its first, kProlongRows at a
/// time
template <typename T> struct ProlongL
{
  Blk g;
  Dims df, dc;
  int3 sh;
  const T *xc;
  T *xf;
  const uint8_t *fixf;
  const KState *gate;
  unsigned ry;
  __device__ bool skip() const { return gated(gate); }
  __device__ void run(const Blk &B) const
  {
    if(gated(gate))
      return;
    const int i = B.x * blockDim.x + threadIdx.x;
    const int j1 = min(df.sy, int((B.y + 1) * ry));
    for(int j = int(B.y * ry); j < j1; j += kProlongRows)
      prolong_rows_b<T>(df, dc, sh, xc, xf, fixf, i, j, B.z);
  }
};
/// Rows per work item of a batched launch whose rows are independent: one
/// while the launch's rows (`rows`, over every problem) fill the GPU's
/// resident warps twice (`capacity`), more as they exceed it, at most `most`.
/// A work item walks its rows in sequence, so on small (coarse) launches one
/// row each keeps them short and parallel, and on large ones several rows
/// each keep the per-item overhead small.
inline unsigned rows_per_item(long long rows, long long capacity, unsigned most)
{
  const long long r = rows / std::max(1LL, 2 * capacity);
  return unsigned(std::max(1LL, std::min<long long>(most, r)));
}
/// blocks along y of a batched transfer over ry node rows, k rows each
inline unsigned transfer_rows(unsigned ry, unsigned k) { return (ry + k - 1) / k; }
/// resident CTAs of a transfer launch (kTB threads) on the whole GPU
inline long long transfer_capacity() { return num_sms() * 16LL; }
template <typename T> struct FillL
{
  Blk g;
  long long n;
  T v;
  T *x;
  __device__ bool skip() const { return false; }
  __device__ void run(const Blk &B) const { fill_b<T>(n, v, x, B); }
};
template <typename T> struct DenseL
{
  Blk g;
  int n;
  const double *A;
  const long long *soa;
  const T *b;
  T *x;
  const KState *gate;
  __device__ bool skip() const { return gated(gate); }
  __device__ void run(const Blk &B) const { dense_apply_b<T>(n, A, soa, b, x, gate, B); }
};
/// y = x over n entries (the V-cycle's result when the smoothing ends in the
/// scratch vector), grid-stride
template <typename T> struct CopyL
{
  Blk g;
  long long n;
  const T *x;
  T *y;
  const KState *gate;
  __device__ bool skip() const { return gated(gate); }
  __device__ void run(const Blk &B) const
  {
    if(gated(gate))
      return;
    for(long long i = B.x * (long long)blockDim.x + threadIdx.x; i < n;
        i += (long long)B.gx * blockDim.x)
      y[i] = x[i];
  }
};

template <typename T> struct CoarsenL
{
  Blk g;
  Dims df, dc;
  int3 sh;
  const T *Ef;
  T *Ec;
  __device__ bool skip() const { return false; }
  __device__ void run(const Blk &B) const { coarsen_E_b<T>(df, dc, sh, Ef, Ec, B); }
};
template <typename T> struct AssembleL
{
  Blk g;
  Dims d;
  KMat<double, 24> K;
  const T *E;
  const int *dense;
  int n;
  double *A;
  __device__ bool skip() const { return false; }
  __device__ void run(const Blk &B) const { dense_assemble_b<T>(d, K, E, dense, n, A, B); }
};
template <bool SMEM> struct InvertL
{
  Blk g;
  int n;
  double *A;
  int *status;
  __device__ bool skip() const { return false; }
  __device__ void run(const Blk &) const { invert_spd_b<SMEM>(n, A, status); }
};

/// number of problems whose solve has not stopped
__global__ void k_count_active(int n, KState *const *st, int *out)
{
  __shared__ int c;
  if(threadIdx.x == 0)
    c = 0;
  __syncthreads();
  int mine = 0;
  for(int i = threadIdx.x; i < n; i += blockDim.x)
    mine += st[i]->stop ? 0 : 1;
  atomicAdd(&c, mine);
  __syncthreads();
  if(threadIdx.x == 0)
    *out = c;
}

using Launch = std::function<void(cudaStream_t)>;

/// records of one batched launch, collected problem by problem
template <class L> struct Builder
{
  std::vector<L> recs;
  std::vector<int2> map;
  void add(L l, unsigned gx, unsigned gy = 1, unsigned gz = 1)
  {
    l.g = Blk{0, 0, 0, gx, gy, gz};
    const int id = int(recs.size());
    recs.push_back(l);
    const long long nb = (long long)gx * gy * gz;
    ICB_REQUIRE((long long)map.size() + nb < (1LL << 31), "batched launch too large");
    for(long long b = 0; b < nb; b++)
      map.push_back(make_int2(id, int(b)));
  }
  /// upload and return the launch (empty when no problem takes this step)
  Launch finish(int threads, int smem, cudaStream_t s, unsigned *counters)
  {
    if(recs.empty())
      return {};
    auto D = std::make_shared<DevBuf<L>>(recs.size());
    auto M = std::make_shared<DevBuf<int2>>(map.size());
    ICB_CUDA(cudaMemcpyAsync(D->p, recs.data(), sizeof(L) * recs.size(), cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaMemcpyAsync(M->p, map.data(), sizeof(int2) * map.size(), cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    BatchQueue q{counters, counters + 1, int(map.size())};
    const int grid = queue_grid((const void *)k_batch<L>, threads, smem, q);
    return [D, M, q, grid, threads, smem](cudaStream_t cs) {
      k_batch<L><<<grid, threads, smem, cs>>>(D->p, M->p, q);
      ICB_CUDA(cudaGetLastError());
      count_launch();
    };
  }
};

/// most rows per work item of a batched Q4 operator launch without a fused dot
constexpr unsigned kQ4BatchRows = 16;

/// the Q4 operator launches of one step (k_matvec_q4_batch)
template <typename T> struct Q4Builder
{
  std::vector<Q4Launch<T>> recs;
  int mode = OP_APPLY;
  bool dot = false;
  void add(const Dims &d, const T *K, const T *E, const T *u, T *y, const uint8_t *fix,
           const OpExtras<T> &x)
  {
    Q4Launch<T> q{};
    std::copy(K, K + 64, q.K.k);
    q.d = d;
    q4_grid(d, q.bx, q.by, q.ychunk);
    q.E = E;
    q.u = u;
    q.y = y;
    q.fix = fix;
    q.red = x.dotRed ? *x.dotRed : RedScratch{};
    q.dotOut = x.dotOut;
    q.gate = x.gate;
    q.gateConv = x.gateConv;
    q.ep = Epi<T>{x.b, x.dinv, T(x.omega), T(x.c1), T(x.c2)};
    if(x.dotRed)
      ICB_REQUIRE(q4_dot_slots(d) <= x.dotRed->maxBlocks, "reduction scratch too small");
    mode = x.mode;
    dot = x.dotRed != nullptr;
    recs.push_back(q);
  }
  Launch finish(cudaStream_t s, unsigned *counters)
  {
    if(recs.empty())
      return {};
    // one element matrix for every launch (the same material and element
    // shape): it goes to the kernel as a parameter
    bool uniform = true;
    for(const Q4Launch<T> &q : recs)
      uniform = uniform && std::memcmp(q.K.k, recs[0].K.k, sizeof(q.K.k)) == 0;
    {
      // the operator's output does not depend on how its rows are cut into
      // blocks (every node is the same sum, computed by its owner), nor does
      // its fused dot (one slot per node row and warp strip, summed in slot
      // order): rows per block from the size of the whole launch -- one on
      // small (coarse) launches, so their blocks stay short and parallel, up
      // to kQ4BatchRows on large ones, so the per-item overhead stays small
      long long rows = 0;
      for(const Q4Launch<T> &q : recs)
        rows += (long long)q.bx * q4_block_warps() * q.d.sy;
      const unsigned k =
          rows_per_item(rows, q4_batch_capacity_warps<T>(mode, dot, uniform), kQ4BatchRows);
      for(Q4Launch<T> &q : recs)
      {
        q.ychunk = std::min<int>(q.d.sy, int(k));
        q.by = (q.d.sy + q.ychunk - 1) / q.ychunk;
      }
    }
    std::vector<int2> map;
    for(size_t id = 0; id < recs.size(); id++)
      for(int b = 0; b < recs[id].bx * recs[id].by; b++)
        map.push_back(make_int2(int(id), b));
    ICB_REQUIRE(map.size() < (1ULL << 31), "batched launch too large");
    auto D = std::make_shared<DevBuf<Q4Launch<T>>>(recs.size());
    auto M = std::make_shared<DevBuf<int2>>(map.size());
    ICB_CUDA(cudaMemcpyAsync(D->p, recs.data(), sizeof(Q4Launch<T>) * recs.size(),
                             cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaMemcpyAsync(M->p, map.data(), sizeof(int2) * map.size(), cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    const int md = mode;
    const bool dt = dot;
    BatchQueue q{counters, counters + 1, int(map.size())};
    const int grid = q4_batch_grid<T>(md, dt, uniform, q);
    const bool uk = uniform;
    const KMat<T, 8> K = recs[0].K;
    return [D, M, q, grid, md, dt, uk, K](cudaStream_t cs) {
      launch_q4_batch<T>(D->p, M->p, q, grid, md, dt, uk ? &K : nullptr, cs);
    };
  }
};

} // namespace

/// The FCG iteration with its V-cycle (MgPcg::iteration / level) for many
/// 2D problems at once, TK = double, V-cycle in TP.
template <typename TP> struct BatchMg
{
  using MG = MgPcg<double, TP>;
  std::vector<MG *> M;
  std::vector<Launch> refresh, init, iter;
  DevBuf<unsigned> qc; ///< the work-queue counters every batched launch uses in turn
  DevBuf<KState *> states;
  DevBuf<int> active;
  int *hActive = nullptr;
  cudaGraphExec_t exec = nullptr;
  int batch = 4; ///< iterations per graph launch
  long long nodes = 0;

  ~BatchMg()
  {
    if(exec)
      cudaGraphExecDestroy(exec);
    if(hActive)
      cudaFreeHost(hActive);
  }

  /// problem i's V-cycle on level l: the state of one problem while the
  /// sequence of steps is emitted
  struct Inst
  {
    int i;
    const TP *b;
    TP *out;
  };

  /// append the batched steps of level(l, b, out) for the problems `set`
  void emitLevel(size_t l, const std::vector<Inst> &set, bool gated, std::vector<Launch> &seq,
                 cudaStream_t s)
  {
    std::vector<Inst> coarse, fine;
    for(const Inst &I : set)
      (l + 1 == M[I.i]->lv.size() ? coarse : fine).push_back(I);
    auto gate = [&](int i) -> const KState * { return gated ? M[i]->st.p : nullptr; };
    auto push = [&](Launch f) {
      if(f)
        seq.push_back(std::move(f));
    };
    if(!coarse.empty())
    {
      // MgPcg::coarseSolve
      Builder<FillL<TP>> f;
      Builder<DenseL<TP>> da;
      int ncmax = 1;
      for(const Inst &I : coarse)
      {
        MG &m = *M[I.i];
        const Level<TP> &C = m.lv.back();
        const long long n = (long long)C.d.dim * C.d.ld;
        f.add(FillL<TP>{{}, n, TP(0), I.out}, unsigned(vblocks(n)));
        if(m.nc)
        {
          da.add(DenseL<TP>{{}, m.nc, m.cA.p, m.cSoa.p, I.b, I.out, gate(I.i)}, 8);
          ncmax = std::max(ncmax, m.nc);
        }
      }
      push(f.finish(VB, 0, s, qc.p));
      push(da.finish(256, int(sizeof(double)) * ncmax, s, qc.p));
    }
    if(fine.empty())
      return;
    struct Cur
    {
      TP *cur, *oth;
    };
    std::vector<Cur> cs(fine.size());
    const int nu = M[fine[0].i]->nu;
    for(const Inst &I : fine)
      ICB_REQUIRE(M[I.i]->nu == nu, "batched problems need the same smoothing degree");
    {
      Builder<Jacobi0L<TP>> j0;
      for(size_t k = 0; k < fine.size(); k++)
      {
        const Inst &I = fine[k];
        MG &m = *M[I.i];
        Level<TP> &L = m.lv[l];
        const long long n = (long long)L.d.dim * L.d.ld;
        cs[k] = Cur{L.t.p, I.out};
        j0.add(Jacobi0L<TP>{{}, n, TP(m.cc2[0]), L.dinv.p, I.b, cs[k].cur, cs[k].oth, gate(I.i)},
               unsigned(vblocks(n)));
      }
      push(j0.finish(VB, 0, s, qc.p));
    }
    auto cheb = [&](int k) {
      Q4Builder<TP> op;
      for(size_t t = 0; t < fine.size(); t++)
      {
        const Inst &I = fine[t];
        MG &m = *M[I.i];
        Level<TP> &L = m.lv[l];
        OpExtras<TP> ch;
        ch.mode = OP_CHEB;
        ch.b = I.b;
        ch.dinv = L.dinv.p;
        ch.gate = gate(I.i);
        ch.gateConv = 1;
        ch.c1 = m.cc1[k];
        ch.c2 = m.cc2[k];
        op.add(L.d, L.K, L.E, cs[t].cur, cs[t].oth, L.fix, ch);
        std::swap(cs[t].cur, cs[t].oth);
      }
      push(op.finish(s, qc.p));
    };
    for(int k = 1; k < nu; k++)
      cheb(k);
    {
      Q4Builder<TP> op;
      Builder<RestrictL<TP>> rs;
      std::vector<Inst> next;
      long long rowsR = 0;
      for(const Inst &I : fine)
      {
        const dim3 g3 = grid3(M[I.i]->lv[l + 1].d);
        rowsR += (long long)g3.x * g3.y * g3.z;
      }
      const unsigned kR = rows_per_item(rowsR, transfer_capacity(), 8);
      for(size_t t = 0; t < fine.size(); t++)
      {
        const Inst &I = fine[t];
        MG &m = *M[I.i];
        Level<TP> &L = m.lv[l];
        Level<TP> &Cn = m.lv[l + 1];
        OpExtras<TP> res;
        res.mode = OP_RESIDUAL;
        res.b = I.b;
        res.gate = gate(I.i);
        res.gateConv = 1;
        op.add(L.d, L.K, L.E, cs[t].cur, L.r.p, L.fix, res);
        const dim3 g3 = grid3(Cn.d);
        rs.add(RestrictL<TP>{{}, L.d, Cn.d, Cn.sh, L.r.p, Cn.b.p, Cn.fix, gate(I.i), g3.y}, g3.x,
               transfer_rows(g3.y, kR), g3.z);
        next.push_back(Inst{I.i, Cn.b.p, Cn.x.p});
      }
      push(op.finish(s, qc.p));
      push(rs.finish(kTB, 0, s, qc.p));
      emitLevel(l + 1, next, gated, seq, s);
    }
    {
      Builder<ProlongL<TP>> pr;
      long long rowsP = 0;
      for(const Inst &I : fine)
      {
        const Dims &d = M[I.i]->lv[l].d;
        const dim3 g3 = grid3(d);
        rowsP += (long long)g3.x * prolong_row_blocks(d) * g3.z;
      }
      // row groups of kProlongRows per work item
      const unsigned kP = rows_per_item(rowsP, transfer_capacity(), 4);
      for(size_t t = 0; t < fine.size(); t++)
      {
        const Inst &I = fine[t];
        MG &m = *M[I.i];
        Level<TP> &L = m.lv[l];
        Level<TP> &Cn = m.lv[l + 1];
        const dim3 g3 = grid3(L.d);
        const unsigned rows = kP * kProlongRows; // node rows per work item
        pr.add(ProlongL<TP>{{}, L.d, Cn.d, Cn.sh, Cn.x.p, cs[t].cur, L.fix, gate(I.i), rows}, g3.x,
               transfer_rows(g3.y, rows), g3.z);
      }
      push(pr.finish(kTB, 0, s, qc.p));
    }
    for(int k = 0; k < nu; k++)
      cheb(k);
    Builder<CopyL<TP>> cp;
    for(size_t t = 0; t < fine.size(); t++)
      if(cs[t].cur != fine[t].out)
      {
        const Level<TP> &L = M[fine[t].i]->lv[l];
        const long long n = (long long)L.d.dim * L.d.ld;
        cp.add(CopyL<TP>{{}, n, cs[t].cur, fine[t].out, gate(fine[t].i)}, unsigned(vblocks(n)));
      }
    push(cp.finish(VB, 0, s, qc.p));
  }

  /// MgPcg::refresh of every problem (coarse moduli level by level, every
  /// level's inverse diagonal, the coarsest matrix and its inverse)
  void buildRefresh(cudaStream_t s)
  {
    refresh.clear();
    auto push = [&](Launch f) {
      if(f)
        refresh.push_back(std::move(f));
    };
    size_t depth = 0;
    for(MG *m : M)
      depth = std::max(depth, m->lv.size());
    for(size_t l = 1; l < depth; l++)
    {
      Builder<CoarsenL<TP>> c;
      for(MG *m : M)
        if(l < m->lv.size())
          c.add(CoarsenL<TP>{{}, m->lv[l - 1].d, m->lv[l].d, m->lv[l].sh, m->lv[l - 1].E,
                             m->lv[l].Eown.p},
                nblocks(m->lv[l].d.nel, 256));
      push(c.finish(256, 0, s, qc.p));
    }
    {
      std::vector<Diag2Launch<TP>> recs;
      std::vector<int2> map;
      for(MG *m : M)
        for(auto &L : m->lv)
        {
          Diag2Launch<TP> q{};
          std::copy(L.K, L.K + 64, q.K.k);
          q.d = L.d;
          q.E = L.E;
          q.fix = L.fix;
          q.invdiag = L.dinv.p;
          const int id = int(recs.size());
          recs.push_back(q);
          for(unsigned b = 0; b < nblocks(L.d.nnode, 256); b++)
            map.push_back(make_int2(id, int(b)));
        }
      auto D = std::make_shared<DevBuf<Diag2Launch<TP>>>(recs.size());
      auto Mp = std::make_shared<DevBuf<int2>>(map.size());
      ICB_CUDA(cudaMemcpyAsync(D->p, recs.data(), sizeof(Diag2Launch<TP>) * recs.size(),
                               cudaMemcpyHostToDevice, s));
      ICB_CUDA(cudaMemcpyAsync(Mp->p, map.data(), sizeof(int2) * map.size(),
                               cudaMemcpyHostToDevice, s));
      ICB_CUDA(cudaStreamSynchronize(s));
      BatchQueue q{qc.p, qc.p + 1, int(map.size())};
      push([D, Mp, q](cudaStream_t cs) { launch_diag2_batch<TP>(D->p, Mp->p, q, cs); });
      // (the refresh steps run outside any capture: the diagonal launch sizes
      // its grid when it runs)
    }
    Builder<FillL<double>> zA;
    Builder<FillL<int>> zS;
    Builder<AssembleL<TP>> as;
    Builder<InvertL<true>> invS;
    Builder<InvertL<false>> invG;
    int smemMax = 0;
    for(MG *m : M)
    {
      if(!m->nc)
        continue;
      const Level<TP> &C = m->lv.back();
      const long long nn = (long long)m->nc * m->nc;
      zA.add(FillL<double>{{}, nn, 0.0, m->cA.p}, unsigned(vblocks(nn)));
      zS.add(FillL<int>{{}, 1, 0, m->cStatus.p}, 1);
      AssembleL<TP> a{};
      for(int i = 0; i < 576; i++)
        a.K.k[i] = double(C.K[i]);
      a.d = C.d;
      a.E = C.E;
      a.dense = m->cDense.p;
      a.n = m->nc;
      a.A = m->cA.p;
      as.add(a, nblocks(C.d.nnode * C.d.dim, 128));
      if(m->nc <= kInvSmemMax)
      {
        invS.add(InvertL<true>{{}, m->nc, m->cA.p, m->cStatus.p}, 1);
        smemMax = std::max(smemMax, int(sizeof(double)) * m->nc * m->nc);
      }
      else
        invG.add(InvertL<false>{{}, m->nc, m->cA.p, m->cStatus.p}, 1);
    }
    push(zA.finish(VB, 0, s, qc.p));
    push(zS.finish(VB, 0, s, qc.p));
    push(as.finish(128, 0, s, qc.p));
    if(smemMax > 0)
      ICB_CUDA(cudaFuncSetAttribute(k_batch<InvertL<true>>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(sizeof(double)) * kInvSmemMax * kInvSmemMax));
    push(invS.finish(1024, smemMax, s, qc.p));
    push(invG.finish(1024, 0, s, qc.p));
  }

  /// the step sequences of MgPcg::solve's set-up (init) and of one iteration
  /// (iter) for problems whose hierarchies are built, solving
  /// K x[i] = b[i]
  void build(const std::vector<MG *> &mgs, const std::vector<const double *> &b,
             const std::vector<double *> &x, const std::vector<double> &tol,
             const std::vector<int> &maxit, cudaStream_t s)
  {
    M = mgs;
    const int n = int(M.size());
    if(!qc.p)
    {
      qc.alloc(2);
      ICB_CUDA(cudaMemsetAsync(qc.p, 0, 2 * sizeof(unsigned), s));
    }
    buildRefresh(s);
    init.clear();
    iter.clear();
    auto push = [](std::vector<Launch> &seq, Launch f) {
      if(f)
        seq.push_back(std::move(f));
    };
    std::vector<Inst> all;
    {
      Builder<InitL<double, TP>> in;
      for(int i = 0; i < n; i++)
      {
        MG &m = *M[i];
        in.add(InitL<double, TP>{{}, m.n, b[i], x[i], m.r.p, MG::same() ? nullptr : m.rP.p, m.red,
                                 m.st.p, tol[i], maxit[i]},
               unsigned(vblocks(m.n)));
        all.push_back(Inst{i, m.rin(), m.z.p});
      }
      push(init, in.finish(VB, 0, s, qc.p));
    }
    emitLevel(0, all, false, init, s);
    {
      Builder<Init2L<double, TP>> in2;
      for(int i = 0; i < n; i++)
      {
        MG &m = *M[i];
        in2.add(Init2L<double, TP>{{}, m.n, m.r.p, m.z.p, m.p.p, m.red, m.st.p},
                unsigned(vblocks(m.n)));
      }
      push(init, in2.finish(VB, 0, s, qc.p));
    }
    // one iteration (MgPcg::iteration)
    {
      Q4Builder<double> op;
      Builder<RL<double, TP>> rb;
      for(int i = 0; i < n; i++)
      {
        MG &m = *M[i];
        OpExtras<double> a;
        a.dotRed = &m.red;
        a.dotOut = m.dots.p;
        a.gate = m.st.p;
        op.add(m.lv[0].d, m.Kk, m.Ek, m.p.p, m.q.p, m.lv[0].fix, a);
        rb.add(RL<double, TP>{{}, m.n, m.r.p, MG::same() ? nullptr : m.rP.p, m.q.p, m.z.p,
                              m.dots.p, m.red, m.st.p},
               unsigned(vblocks(m.n)));
      }
      push(iter, op.finish(s, qc.p));
      push(iter, rb.finish(VB, 0, s, qc.p));
    }
    emitLevel(0, all, true, iter, s);
    {
      Builder<RzL<double, TP>> rz;
      Builder<XpL<double, TP>> xp;
      for(int i = 0; i < n; i++)
      {
        MG &m = *M[i];
        rz.add(RzL<double, TP>{{}, m.n, m.r.p, m.z.p, m.red, m.st.p}, unsigned(vblocks(m.n)));
        xp.add(XpL<double, TP>{{}, m.n, x[i], m.p.p, m.z.p, m.red, m.st.p}, unsigned(vblocks(m.n)));
      }
      push(iter, rz.finish(VB, 0, s, qc.p));
      push(iter, xp.finish(VB, 0, s, qc.p));
    }
    std::vector<KState *> sp(n);
    for(int i = 0; i < n; i++)
      sp[i] = M[i]->st.p;
    states.alloc(n);
    active.alloc(1);
    ICB_CUDA(cudaMemcpyAsync(states.p, sp.data(), sizeof(KState *) * n, cudaMemcpyHostToDevice, s));
    if(!hActive)
      ICB_CUDA(cudaMallocHost(&hActive, sizeof(int)));
    // `batch` iterations and the count of active problems as one graph
    if(exec)
      cudaGraphExecDestroy(exec);
    exec = nullptr;
    cudaStream_t cs;
    ICB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t gr = nullptr;
    const long long before = thread_launch_count();
    ICB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
    for(int k = 0; k < batch; k++)
      for(auto &f : iter)
        f(cs);
    k_count_active<<<1, 256, 0, cs>>>(n, states.p, active.p);
    ICB_CUDA(cudaMemcpyAsync(hActive, active.p, sizeof(int), cudaMemcpyDeviceToHost, cs));
    ICB_CUDA(cudaStreamEndCapture(cs, &gr));
    nodes = thread_launch_count() - before;
    count_launch(-nodes); // recorded, not launched
    ICB_CUDA(cudaGraphInstantiate(&exec, gr, 0));
    cudaGraphDestroy(gr);
    cudaStreamDestroy(cs);
    ICB_CUDA(cudaStreamSynchronize(s));
  }

  /// run the set-up and iterations until every problem has stopped (each
  /// stops at its own tolerance or iteration limit, as its own solve would).
  /// When at most handOff() problems are left, each finishes in its own
  /// solve loop on its own stream (own[i], solving into x[i]): the same
  /// iterations, without the batch's launches over every problem.
  long long iterationsRun = 0; ///< batched iterations of the last run()
  int handedOff = 0;           ///< problems of the last run() finished on their own
  int handOff() const
  {
    const int k = batch_handoff();
    return k > 0 ? k : std::min(32, std::max(1, int(M.size()) / 8));
  }
  void run(int maxit, cudaStream_t s, const std::vector<cudaStream_t> &own,
           const std::vector<double *> &x)
  {
    for(auto &f : refresh)
      f(s);
    for(auto &f : init)
      f(s);
    long long launched = 0;
    const int n = int(M.size());
    handedOff = 0;
    for(;;)
    {
      // the share of the batch still iterating when this launch starts
      const int act = launched == 0 ? n : *hActive;
      const auto t0 = std::chrono::steady_clock::now();
      ICB_CUDA(cudaGraphLaunch(exec, s));
      count_launch(nodes + 1);
      ICB_CUDA(cudaStreamSynchronize(s));
      fused_active_record(act, n, std::chrono::duration<double>(
                                      std::chrono::steady_clock::now() - t0).count());
      launched += batch;
      if(*hActive == 0 || launched > (long long)maxit + batch)
        break;
      if(*hActive <= handOff())
      {
        const int left = *hActive;
        const auto t1 = std::chrono::steady_clock::now();
        finishAlone(maxit, s, own, x);
        fused_active_record(left, n, std::chrono::duration<double>(
                                         std::chrono::steady_clock::now() - t1).count());
        break;
      }
    }
    iterationsRun = launched;
  }

  /// every problem still iterating continues in its own loop on its own
  /// stream (after the batch's work on s), then s waits for them all
  void finishAlone(int maxit, cudaStream_t s, const std::vector<cudaStream_t> &own,
                   const std::vector<double *> &x)
  {
    const int n = int(M.size());
    std::vector<KState> hs(n);
    for(int i = 0; i < n; i++)
      ICB_CUDA(cudaMemcpyAsync(&hs[i], M[i]->st.p, sizeof(KState), cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    std::vector<int> left;
    for(int i = 0; i < n; i++)
      if(!hs[i].stop)
        left.push_back(i);
    // s is idle (synchronised above): the problems' streams may start, and
    // in the device form their loops run side by side
    for(int i : left)
    {
      MG &m = *M[i];
      m.prepareLoop(x[i], own[i]);
      if(m.loop.device)
        m.launchLoop(own[i]);
      else
        m.iterate(x[i], maxit, own[i], nullptr);
    }
    handedOff = int(left.size());
    for(int i : left)
    {
      ICB_CUDA(cudaStreamSynchronize(own[i]));
      if(M[i]->loop.device)
        count_launch((long long)M[i]->hst->pad * M[i]->loop.graphNodes);
    }
  }
};

/// MgPcg of problem p for solve options o, built (not refreshed)
template <typename TP> MgPcg<double, TP> *prepare_mg(icb_problem p, const icb_solve_opts &o);

template <> MgPcg<double, double> *prepare_mg<double>(icb_problem p, const icb_solve_opts &o)
{
  Mixed &M = mixed_of(p, o);
  if(!M.mg64)
  {
    M.mg64 = std::make_unique<MgPcg<double, double>>();
    M.mg64->build(*p->hs, p->K0, p->E.p, p->K0, p->E.p, p->fix.p, o.mg_coarse_dofs, o.mg_smooth,
                  p->stream());
  }
  return M.mg64.get();
}
template <> MgPcg<double, float> *prepare_mg<float>(icb_problem p, const icb_solve_opts &o)
{
  Mixed &M = mixed_of(p, o);
  if(!M.mgmx)
  {
    M.mgmx = std::make_unique<MgPcg<double, float>>();
    M.mgmx->build(*p->hs, p->K0, p->E.p, p->K0f, p->Ef.p, p->fix.p, o.mg_coarse_dofs, o.mg_smooth,
                  p->stream());
  }
  return M.mgmx.get();
}

template struct BatchMg<double>;
template struct BatchMg<float>;

/// the batched solves' graph launches of the last fused run by the share of
/// the batch still iterating when each started: more than half, more than an
/// eighth, at most an eighth (seconds and launches)
static double g_active_s[3];
static long long g_active_n[3];
void fused_active_record(int active, int n, double seconds)
{
  const int k = 2 * active > n ? 0 : (8 * active > n ? 1 : 2);
  g_active_s[k] += seconds;
  g_active_n[k]++;
}
double fused_active_seconds(int k) { return k >= 0 && k < 3 ? g_active_s[k] : -1.0; }
long long fused_active_launches(int k) { return k >= 0 && k < 3 ? g_active_n[k] : -1; }

/// wall time of the fused loop's phases over the last run, in seconds:
/// 0 building the batched launches, 1 per-problem filter and moduli
/// launches, 2 the batched multigrid set-up and solve, 3 compliance,
/// sensitivities and adjoint filters, 4 OC updates and the step's wait
static double g_fused_phase[5];
double fused_phase_seconds(int k) { return k >= 0 && k < 5 ? g_fused_phase[k] : -1.0; }
/// iterations of the last fused run: the batch's (every launch sequence
/// counted once) and the sum over problems of their own
static long long g_fused_iters[2];
long long fused_iterations(int k) { return k >= 0 && k < 2 ? g_fused_iters[k] : -1; }

namespace
{
using PhaseClock = std::chrono::steady_clock;
double since(PhaseClock::time_point t)
{
  return std::chrono::duration<double>(PhaseClock::now() - t).count();
}

/// one problem of the fused OC loop: its loop work space and state
struct OcRun
{
  int idx = 0;
  icb_problem p = nullptr;
  const icb_loop_opts *o = nullptr;
  double *hist = nullptr;
  ConeFilter *cone = nullptr;
  OcUpdater *oc = nullptr;
  DevBuf<double> *x, *xf, *xh, *dxh, *dc, *dv, *dcf, *dvf, *lo, *hi, *V;
  cudaGraphExec_t g3 = nullptr; ///< the step's work after the solve (built in the loop)
  long long g3nodes = 0;
  double V0 = 0.0;
  bool active = true;
  int status = ICB_OK;
  std::string err;
};

/// the opt-macro-oc loop (icb_run_oc, opt_macro_oc.cpp:84-172) of every
/// problem, advanced together: per step the filters, moduli and multigrid
/// set-up run on each problem's own stream, the solves of all problems as
/// one batched sequence (BatchMg), then compliance, sensitivities, adjoint
/// filters and the OC update again per problem, all queued before one wait.
/// Each problem's history and design are bitwise those of its own
/// icb_run_oc.
template <typename TP>
void run_oc_fused_tp(std::vector<OcRun> &R, cudaStream_t sb)
{
  BatchMg<TP> batch;
  OcBatch ocb;
  std::vector<OcRun *> set;
  auto rebuild = [&]() {
    set.clear();
    std::vector<OcBatchItem> ocItems;
    std::vector<MgPcg<double, TP> *> mgs;
    std::vector<const double *> b;
    std::vector<double *> x;
    std::vector<double> tol;
    std::vector<int> maxit;
    for(OcRun &r : R)
      if(r.active)
      {
        set.push_back(&r);
        mgs.push_back(prepare_mg<TP>(r.p, r.o->solve));
        b.push_back(r.p->f.p);
        x.push_back(r.p->x.p);
        tol.push_back(r.o->solve.tol);
        maxit.push_back(r.o->solve.maxit);
        ocItems.push_back(OcBatchItem{r.cone, r.oc, r.x->p, r.dcf->p, r.dvf->p, r.lo->p, r.hi->p,
                                      r.V->p});
      }
    if(!set.empty())
    {
      batch.build(mgs, b, x, tol, maxit, sb);
      ocb.build(ocItems, sb);
    }
  };
  auto fail = [&](OcRun &r, int st, const std::string &msg) {
    r.active = false;
    r.status = st;
    r.err = msg;
  };
  int maxSteps = 0;
  for(OcRun &r : R)
    maxSteps = std::max(maxSteps, r.o->nsteps);
  for(double &v : g_fused_phase)
    v = 0.0;
  for(int k = 0; k < 3; k++)
  {
    g_active_s[k] = 0.0;
    g_active_n[k] = 0;
  }
  g_fused_iters[0] = g_fused_iters[1] = 0;
  {
    auto tb = PhaseClock::now();
    rebuild();
    g_fused_phase[0] += since(tb);
  }
  double *hc = nullptr, *hv = nullptr;
  KState *hs = nullptr;
  const size_t n = R.size();
  ICB_CUDA(cudaMallocHost(&hc, sizeof(double) * n));
  ICB_CUDA(cudaMallocHost(&hv, sizeof(double) * n));
  ICB_CUDA(cudaMallocHost(&hs, sizeof(KState) * n));
  std::vector<cudaEvent_t> ev(n);
  for(auto &e : ev)
    ICB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  try
  {
    for(int step = 1; step <= maxSteps && !set.empty(); step++)
    {
      auto t0 = std::chrono::steady_clock::now();
      // filters, moduli and the multigrid set-up, problem by problem
      for(OcRun *r : set)
      {
        cudaStream_t s = r->p->stream();
        const double beta =
            r->o->use_threshold ? std::min(std::pow(2.0, (int)(step / 40)), 16.0) : 0.0;
        r->cone->forward(r->x->p, r->xf->p, beta, 0.5, r->xh->p, r->dxh->p, s);
        const int rc = icb_set_density_device(r->p, r->xh->p);
        if(rc)
        {
          fail(*r, rc, icb_last_error());
          continue;
        }
        ICB_CUDA(cudaEventRecord(ev[r->idx], s));
      }
      bool lost = false;
      for(OcRun *r : set)
        lost = lost || !r->active;
      if(lost)
      {
        for(OcRun *r : set)
          if(r->active)
            ICB_CUDA(cudaStreamSynchronize(r->p->stream()));
        rebuild();
        step--;
        continue; // the remaining problems redo this step's set-up
      }
      auto tp = PhaseClock::now();
      g_fused_phase[1] += std::chrono::duration<double>(tp - t0).count();
      for(OcRun *r : set)
        ICB_CUDA(cudaStreamWaitEvent(sb, ev[r->idx], 0));
      int maxit = 0;
      for(OcRun *r : set)
        maxit = std::max(maxit, r->o->solve.maxit);
      {
        std::vector<cudaStream_t> own;
        std::vector<double *> xs;
        for(OcRun *r : set)
        {
          own.push_back(r->p->stream());
          xs.push_back(r->p->x.p);
        }
        batch.run(maxit, sb, own, xs);
      }
      for(size_t k = 0; k < set.size(); k++)
        ICB_CUDA(cudaMemcpyAsync(&hs[set[k]->idx], batch.M[k]->st.p, sizeof(KState),
                                 cudaMemcpyDeviceToHost, sb));
      ICB_CUDA(cudaStreamSynchronize(sb));
      g_fused_phase[2] += since(tp);
      g_fused_iters[0] += batch.iterationsRun;
      for(size_t k = 0; k < set.size(); k++)
        g_fused_iters[1] += hs[set[k]->idx].iter;
      tp = PhaseClock::now();
      // compliance, V0 (step 1), sensitivities and adjoint filters
      for(OcRun *r : set)
      {
        const KState &k = hs[r->idx];
        if(k.status != ICB_OK)
        {
          fail(*r, k.status, k.status == ICB_ERR_MAXITER ? "iteration limit reached"
                                                         : "CG breakdown or non-finite values");
          continue;
        }
        icb_problem p = r->p;
        cudaStream_t s = p->stream();
        const long long ne = p->d.nel;
        p->solved = true;
        p->last = icb_solve_info{k.iter, k.matvecs, 1, k.bb > 0 ? std::sqrt(k.rr / k.bb) : 0.0,
                                 -1.0, 0.0, k.status};
        // the step's per-design work after the solve, the same every step: a
        // graph captured at the first step and relaunched (one host call per
        // design instead of ten)
        if(!r->g3)
        {
          const long long before = thread_launch_count();
          ICB_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
          ICB_CUDA(cudaMemcpyAsync(p->u.p, p->x.p, sizeof(double) * p->nsoa,
                                   cudaMemcpyDeviceToDevice, s));
          launch_dot(p->nsoa, p->x.p, p->f.p, p->red, p->scal.p + 2, s);
          ICB_CUDA(cudaMemcpyAsync(&hc[r->idx], p->scal.p + 2, sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
          const icb_grid_desc &g = p->hs->desc;
          launch_sensitivity(p->d, p->K0, g.young1, g.young2, g.penalty, p->rho.p, p->u.p,
                             p->dc.p, s);
          ICB_CUDA(cudaMemcpyAsync(r->dc->p, p->dc.p, sizeof(double) * ne,
                                   cudaMemcpyDeviceToDevice, s));
          launch_scale_mul(ne, r->dc->p, r->dxh->p, 1.0, s);
          ICB_CUDA(cudaMemcpyAsync(r->dv->p, r->V->p, sizeof(double) * ne,
                                   cudaMemcpyDeviceToDevice, s));
          launch_scale_mul(ne, r->dv->p, r->dxh->p, 1.0, s);
          r->cone->adjoint(r->dc->p, r->dcf->p, s);
          r->cone->adjoint(r->dv->p, r->dvf->p, s);
          cudaGraph_t gr = nullptr;
          ICB_CUDA(cudaStreamEndCapture(s, &gr));
          r->g3nodes = thread_launch_count() - before;
          count_launch(-r->g3nodes); // recorded, not launched
          const cudaError_t e = cudaGraphInstantiate(&r->g3, gr, 0);
          cudaGraphDestroy(gr);
          ICB_CUDA(e);
        }
        ICB_CUDA(cudaGraphLaunch(r->g3, s));
        count_launch(r->g3nodes);
        if(step == 1)
        {
          launch_sum(p, r->xh->p, ne, p->scal.p + 8);
          ICB_CUDA(cudaMemcpyAsync(&hv[r->idx], p->scal.p + 8, sizeof(double),
                                   cudaMemcpyDeviceToHost, s));
        }
      }
      if(step == 1)
        for(OcRun *r : set)
          if(r->active)
          {
            ICB_CUDA(cudaStreamSynchronize(r->p->stream()));
            r->V0 = hv[r->idx] * r->p->hs->volume;
          }
      g_fused_phase[3] += since(tp);
      tp = PhaseClock::now();
      // the OC updates: every problem's bisection as one batched sequence
      // (OcBatch) when all of the set is still running, else problem by
      // problem; then one wait
      auto ocParams = [&](const OcRun *r) {
        OcParams P;
        P.move = r->o->move_limit;
        P.beta = r->o->use_threshold ? std::min(std::pow(2.0, (int)(step / 40)), 16.0) : 0.0;
        return P;
      };
      bool allActive = true;
      for(OcRun *r : set)
        allActive = allActive && r->active;
      if(allActive)
      {
        std::vector<double> g;
        std::vector<OcParams> P;
        for(OcRun *r : set)
        {
          ICB_CUDA(cudaEventRecord(ev[r->idx], r->p->stream()));
          ICB_CUDA(cudaStreamWaitEvent(sb, ev[r->idx], 0));
          g.push_back(r->V0);
          P.push_back(ocParams(r));
        }
        ocb.update(g, P, sb);
      }
      else
      {
        for(OcRun *r : set)
          if(r->active)
            r->oc->launch(r->cone, r->x->p, r->dcf->p, r->dvf->p, r->V0, r->lo->p, r->hi->p,
                          r->V->p, ocParams(r), r->p->stream());
        for(OcRun *r : set)
          if(r->active)
          {
            ICB_CUDA(cudaStreamSynchronize(r->p->stream()));
            r->oc->finish();
          }
      }
      bool changed = false;
      g_fused_phase[4] += since(tp);
      const double dt2 =
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      for(OcRun *r : set)
      {
        if(!r->active)
        {
          changed = true;
          continue;
        }
        r->hist[step - 1] = hc[r->idx];
        if(r->o->iter_seconds)
          r->o->iter_seconds[step - 1] = dt2;
        if(step == r->o->nsteps)
        {
          r->active = false;
          changed = true;
        }
      }
      if(changed)
      {
        auto tb = PhaseClock::now();
        rebuild();
        g_fused_phase[0] += since(tb);
      }
    }
  }
  catch(...)
  {
    // the step graphs copy into hc: released before it
    for(OcRun &r : R)
      if(r.g3)
      {
        cudaStreamSynchronize(r.p->stream());
        cudaGraphExecDestroy(r.g3);
        r.g3 = nullptr;
      }
    for(auto &e : ev)
      cudaEventDestroy(e);
    cudaFreeHost(hc);
    cudaFreeHost(hv);
    cudaFreeHost(hs);
    throw;
  }
  for(OcRun &r : R)
    if(r.g3)
    {
      ICB_CUDA(cudaStreamSynchronize(r.p->stream()));
      cudaGraphExecDestroy(r.g3);
      r.g3 = nullptr;
    }
  for(auto &e : ev)
    cudaEventDestroy(e);
  cudaFreeHost(hc);
  cudaFreeHost(hv);
  cudaFreeHost(hs);
}
} // namespace

static std::atomic<int> g_batch_handoff{0};
int batch_handoff() { return g_batch_handoff; }
void set_batch_handoff(int k) { g_batch_handoff = k; }

static std::atomic<bool> g_batch_fused{true};
bool batch_fused_enabled() { return g_batch_fused; }
void set_batch_fused(bool on) { g_batch_fused = on; }

bool oc_fused_eligible(int n, const icb_problem *probs, const int *kinds,
                       const icb_loop_opts *opts)
{
  if(n < 2)
    return false;
  for(int i = 0; i < n; i++)
  {
    const icb_problem p = probs[i];
    const icb_loop_opts &o = opts[i];
    if(!p || !p->hs || !p->hs->finalized || p->d.dim != 2 || p->hasDirichletValues)
      return false;
    if(kinds && kinds[i] != ICB_JOB_OC)
      return false;
    if(o.solve.precond != ICB_PRECOND_GMG ||
       (o.solve.precision != ICB_FP64 && o.solve.precision != ICB_MIXED))
      return false;
    if(o.solve.precision != opts[0].solve.precision || o.solve.mg_smooth != opts[0].solve.mg_smooth ||
       p->ctx->device != probs[0]->ctx->device)
      return false;
    if(o.on_step || o.resume || o.checkpoint || o.conv_eps > 0.0 || o.nsteps <= 0 ||
       !(o.filter_radius > 0.0))
      return false;
  }
  return true;
}

void run_oc_fused(int n, const icb_problem *probs, const icb_loop_opts *opts,
                  const double *const *rho0, double *const *hist, double *const *xout, int *status,
                  std::vector<std::string> &err)
{
  ICB_CUDA(cudaSetDevice(probs[0]->ctx->device));
  std::vector<OcRun> R(n);
  for(int i = 0; i < n; i++)
  {
    // icb_run_oc's set-up (toapi.cu): filter, updater, work vectors
    OcRun &r = R[i];
    r.idx = i;
    r.p = probs[i];
    r.o = &opts[i];
    r.hist = hist[i];
    icb_problem p = r.p;
    cudaStream_t s = p->stream();
    const long long ne = p->d.nel;
    LoopCache &LC = loop_cache(p);
    r.cone = &LC.coneFilter(p->d, p->hs->h, r.o->filter_radius, s);
    r.oc = &LC.ocUpdater(p->d, s);
    r.x = &LC.buf(0, ne);
    r.xf = &LC.buf(1, ne);
    r.xh = &LC.buf(2, ne);
    r.dxh = &LC.buf(3, ne);
    r.dc = &LC.buf(4, ne);
    r.dv = &LC.buf(5, ne);
    r.dcf = &LC.buf(6, ne);
    r.dvf = &LC.buf(7, ne);
    r.lo = &LC.buf(8, ne);
    r.hi = &LC.buf(9, ne);
    r.V = &LC.buf(10, ne);
    ICB_CUDA(cudaMemcpyAsync(r.x->p, rho0[i], sizeof(double) * ne, cudaMemcpyHostToDevice, s));
    launch_fill(ne, 1.0e-4, r.lo->p, s);
    launch_fill(ne, 1.0, r.hi->p, s);
    launch_fill(ne, p->hs->volume, r.V->p, s);
  }
  for(int i = 0; i < n; i++)
    ICB_CUDA(cudaStreamSynchronize(probs[i]->stream()));
  cudaStream_t sb;
  ICB_CUDA(cudaStreamCreateWithFlags(&sb, cudaStreamNonBlocking));
  try
  {
    if(opts[0].solve.precision == ICB_FP64)
      run_oc_fused_tp<double>(R, sb);
    else
      run_oc_fused_tp<float>(R, sb);
  }
  catch(...)
  {
    cudaStreamDestroy(sb);
    throw;
  }
  cudaStreamDestroy(sb);
  for(int i = 0; i < n; i++)
  {
    OcRun &r = R[i];
    if(xout && xout[i] && r.status == ICB_OK)
      ICB_CUDA(cudaMemcpyAsync(xout[i], r.x->p, sizeof(double) * r.p->d.nel,
                               cudaMemcpyDeviceToHost, r.p->stream()));
    ICB_CUDA(cudaStreamSynchronize(r.p->stream()));
    status[i] = r.status;
    err[i] = r.err;
  }
}

} // namespace icb
