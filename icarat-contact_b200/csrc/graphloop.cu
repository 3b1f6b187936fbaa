// graphloop.cu -- conditional WHILE graphs for the device-side solver loops.
#include "graphloop.hpp"

namespace icb
{

void WhileGraph::reset()
{
  if(exec)
    cudaGraphExecDestroy(exec);
  exec = nullptr;
  bodyNodes = 0;
}

void WhileGraph::build(const std::function<void(cudaStream_t, const LoopCtl &)> &body)
{
  reset();
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
    bodyNodes = (long long)nn;
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
