// graphloop.cu -- conditional WHILE graphs for the device-side solver loops.
#include <algorithm>
#include <atomic>

#include "graphloop.hpp"

namespace icb
{

static std::atomic<bool> g_device_loops{true};
bool device_loops_enabled() { return g_device_loops.load(); }
void set_device_loops(bool on) { g_device_loops = on; }
unsigned long long kernel_switches()
{
  return (tc_operator_enabled() ? 1ull : 0ull) | (hex8_modal_enabled() ? 2ull : 0ull) |
         (device_loops_enabled() ? 4ull : 0ull) | (hex8_pair_enabled() ? 8ull : 0ull) |
         ((unsigned long long)tc_spin_limit() << 8);
}

void WhileGraph::reset()
{
  if(exec)
    cudaGraphExecDestroy(exec);
  exec = nullptr;
  graphNodes = 0;
}

void WhileGraph::build(const std::function<void(cudaStream_t, const LoopCtl &)> &body,
                       bool onDevice, int hostBatch)
{
  reset();
  device = onDevice;
  batch = onDevice ? 1 : std::max(1, hostBatch);
  if(!onDevice)
  {
    cudaStream_t cs = nullptr;
    ICB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    try
    {
      ICB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
      for(int k = 0; k < batch; k++)
        body(cs, LoopCtl{});
      ICB_CUDA(cudaStreamEndCapture(cs, &g));
      size_t nn = 0;
      ICB_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
      graphNodes = (long long)nn;
      ICB_CUDA(cudaGraphInstantiate(&exec, g, 0));
    }
    catch(...)
    {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(cs, &junk);
      if(g)
        cudaGraphDestroy(g);
      cudaStreamDestroy(cs);
      exec = nullptr;
      throw;
    }
    cudaGraphDestroy(g);
    cudaStreamDestroy(cs);
    return;
  }
  cudaGraph_t g = nullptr;
  ICB_CUDA(cudaGraphCreate(&g, 0));
  cudaStream_t cs = nullptr;
  try
  {
    // the condition starts at 1 on every launch: the body runs at least once
    LoopCtl L;
    ICB_CUDA(cudaGraphConditionalHandleCreate(&L.h, g, 1, cudaGraphCondAssignDefault));
    L.on = 1;
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = L.h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    ICB_CUDA(cudaGraphAddNode(&node, g, nullptr, 0, &cp));
    cudaGraph_t bodyG = cp.conditional.phGraph_out[0];
    ICB_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    ICB_CUDA(cudaStreamBeginCaptureToGraph(cs, bodyG, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
    body(cs, L);
    cudaGraph_t captured = nullptr;
    ICB_CUDA(cudaStreamEndCapture(cs, &captured));
    size_t nn = 0;
    ICB_CUDA(cudaGraphGetNodes(bodyG, nullptr, &nn));
    graphNodes = (long long)nn;
    ICB_CUDA(cudaGraphInstantiate(&exec, g, 0));
  }
  catch(...)
  {
    if(cs)
    {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(cs, &junk); // leave capture mode if the body threw
      cudaStreamDestroy(cs);
    }
    cudaGraphDestroy(g);
    exec = nullptr;
    throw;
  }
  cudaStreamDestroy(cs);
  cudaGraphDestroy(g);
}

void WhileGraph::launch(cudaStream_t s) const { ICB_CUDA(cudaGraphLaunch(exec, s)); }

} // namespace icb
