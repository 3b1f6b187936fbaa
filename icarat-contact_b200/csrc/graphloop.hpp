// graphloop.hpp -- a CUDA graph whose body repeats on the device while a
// kernel at the end of the body says so (a conditional WHILE node): one
// graph launch and one host wait run a Krylov solve or a bisection to its
// end, with no wasted gated iterations and no host round trip in between.
#pragma once
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <vector>

#include "icb_internal.hpp"

namespace icb
{
/// the loop condition as the last kernel of a body sees it: `on` is 0 when
/// the kernel runs outside a WHILE graph
struct LoopCtl
{
  cudaGraphConditionalHandle h = 0;
  int on = 0;
};

/// A solver loop as a CUDA graph, in one of two forms: on the device, the
/// body is a conditional WHILE node that repeats until the body's last kernel
/// clears the condition (one launch and one host wait per solve); from the
/// host, the graph holds `batch` passes of the body and is relaunched until
/// a polled device flag says stop (the kernels after the stop are gated).
/// Profilers that cannot follow conditional nodes see every kernel of the
/// host form.
struct WhileGraph
{
  cudaGraphExec_t exec = nullptr;
  bool device = true;      ///< the WHILE-node form
  int batch = 1;           ///< passes per launch in the host form
  long long graphNodes = 0; ///< nodes per launch (host) or per pass (device)

  WhileGraph() = default;
  WhileGraph(const WhileGraph &) = delete;
  WhileGraph &operator=(const WhileGraph &) = delete;
  ~WhileGraph() { reset(); }
  void reset();
  /// record the body by stream capture: body(cs, L) launches one pass on cs;
  /// its last kernel sets the condition through L (loop_end_* / loop_stop;
  /// L.on is 0 in the host form)
  void build(const std::function<void(cudaStream_t, const LoopCtl &)> &body, bool onDevice,
             int hostBatch);
  void launch(cudaStream_t s) const;
};

/// process-wide choice of the loop form for the multigrid PCG and the OC
/// bisection (icb_set_option "device_loops"; default on)
bool device_loops_enabled();
void set_device_loops(bool on);

/// the process-wide kernel switches (tc_operator, hex8_modal, device_loops,
/// tc_spin_limit) as bits: a captured graph holds the kernels they chose
unsigned long long kernel_switches();

/// Everything a captured graph bakes in: the device pointers and sizes its
/// kernels were given, the parameter structs passed by value and the kernel
/// switches.  A cached graph is relaunched only when every entry is equal.
/// Keying on the address of a host object is not enough: an object freed and
/// re-created at the same address owns new device buffers, and the old graph
/// would read the freed ones.  With every baked value in the key, a graph is
/// reused only where a fresh capture would record the same launches.
struct GraphKey
{
  std::vector<unsigned long long> v;
  GraphKey &add(const void *p)
  {
    v.push_back((unsigned long long)(uintptr_t)p);
    return *this;
  }
  GraphKey &add(long long x)
  {
    v.push_back((unsigned long long)x);
    return *this;
  }
  /// a trivially copyable parameter struct, byte by byte
  template <typename S> GraphKey &addBytes(const S &s)
  {
    const unsigned char *b = reinterpret_cast<const unsigned char *>(&s);
    for(size_t i = 0; i < sizeof(S); i += 8)
    {
      unsigned long long w = 0;
      std::memcpy(&w, b + i, std::min<size_t>(8, sizeof(S) - i));
      v.push_back(w);
    }
    return *this;
  }
  bool operator==(const GraphKey &o) const { return v == o.v; }
  bool operator!=(const GraphKey &o) const { return v != o.v; }
};

#ifdef __CUDACC__
/// one thread, at the end of a Krylov body: count the pass (st->pad, zeroed by
/// the solver's init kernel), stop a loop that ran st->maxit + 2 passes
/// without stopping (ICB_ERR_MAXITER), and repeat while !st->stop
__device__ __forceinline__ void loop_end_krylov(const LoopCtl &L, KState *st)
{
  if(!L.on)
    return;
  const int n = ++st->pad;
  if(!st->stop && (long long)n >= (long long)st->maxit + 2)
  {
    st->stop = 1;
    st->status = ICB_ERR_MAXITER;
  }
  cudaGraphSetConditional(L.h, st->stop ? 0u : 1u);
}
/// one thread of a body's last kernel that found the loop already finished
__device__ __forceinline__ void loop_stop(const LoopCtl &L)
{
  if(L.on)
    cudaGraphSetConditional(L.h, 0u);
}
#endif

} // namespace icb
