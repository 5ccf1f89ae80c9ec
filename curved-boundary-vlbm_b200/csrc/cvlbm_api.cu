// Library-level entry points of the C ABI: version, error text, graphs.
#include <cuda_runtime.h>

#include <string>

#include "cvlbm_common.cuh"

namespace cv {
namespace {
thread_local std::string g_last_error;
}
void set_error(const char* msg) { g_last_error = msg ? msg : ""; }
}  // namespace cv

extern "C" int cvlbm_version(void) { return 10000; }

extern "C" const char* cvlbm_last_error(void) { return cv::g_last_error.c_str(); }

extern "C" int cvlbm_graph_launch(cvlbm_graph* g, void* stream) {
  if (!g) return cv::fail(CVLBM_ERR_INVALID_ARG, "null graph");
  if (cudaGraphLaunch(g->exec, (cudaStream_t)stream) != cudaSuccess)
    return cv::fail(CVLBM_ERR_CUDA, "cudaGraphLaunch failed");
  return CVLBM_OK;
}

extern "C" void cvlbm_graph_destroy(cvlbm_graph* g) {
  if (!g) return;
  cudaGraphExecDestroy(g->exec);
  cudaGraphDestroy(g->graph);
  delete g;
}
