// Library-level entry points of the C ABI: version, error text, graphs.
#include <cuda_runtime.h>

#include <string>

#include "cvlbm_common.cuh"

#include <atomic>

namespace cv {
namespace {
thread_local std::string g_last_error;
thread_local cvlbm_timer* g_timer = nullptr;
thread_local cvlbm_timer* g_link_timer = nullptr;
std::atomic<long long> g_launches{0};
}  // namespace
void set_error(const char* msg) { g_last_error = msg ? msg : ""; }
void count_launches(int n) { g_launches += n; }
cvlbm_timer* attached_timer() { return g_timer; }
cvlbm_timer* attached_link_timer() { return g_link_timer; }
int attach_timer(cvlbm_timer* t) {
  g_timer = t;
  return CVLBM_OK;
}
}  // namespace cv

extern "C" int64_t cvlbm_launch_count(void) { return (int64_t)cv::g_launches.load(); }

extern "C" int cvlbm_timer_create(int32_t capacity, cvlbm_timer** out) {
  if (!out || capacity <= 0) return cv::fail(CVLBM_ERR_INVALID_ARG, "bad timer capacity");
  cvlbm_timer* t = new cvlbm_timer{capacity, 0, new cudaEvent_t[capacity], new cudaEvent_t[capacity]};
  for (int k = 0; k < capacity; ++k) {
    if (cudaEventCreate(&t->begin[k]) != cudaSuccess || cudaEventCreate(&t->end[k]) != cudaSuccess)
      return cv::fail(CVLBM_ERR_CUDA, "cudaEventCreate failed");
  }
  *out = t;
  return CVLBM_OK;
}

extern "C" void cvlbm_timer_destroy(cvlbm_timer* t) {
  if (!t) return;
  if (cv::g_timer == t) cv::g_timer = nullptr;
  if (cv::g_link_timer == t) cv::g_link_timer = nullptr;
  for (int k = 0; k < t->capacity; ++k) {
    cudaEventDestroy(t->begin[k]);
    cudaEventDestroy(t->end[k]);
  }
  delete[] t->begin;
  delete[] t->end;
  delete t;
}

extern "C" int cvlbm_timer_reset(cvlbm_timer* t) {
  if (!t) return cv::fail(CVLBM_ERR_INVALID_ARG, "null timer");
  t->used = 0;
  return CVLBM_OK;
}

extern "C" int cvlbm_timer_elapsed(cvlbm_timer* t, double* total_ms, int32_t* count) {
  if (!t || !total_ms || !count) return cv::fail(CVLBM_ERR_INVALID_ARG, "null argument");
  double sum = 0.0;
  for (int k = 0; k < t->used; ++k) {
    if (cudaEventSynchronize(t->end[k]) != cudaSuccess)
      return cv::fail(CVLBM_ERR_CUDA, "cudaEventSynchronize failed");
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, t->begin[k], t->end[k]) != cudaSuccess)
      return cv::fail(CVLBM_ERR_CUDA, "cudaEventElapsedTime failed");
    sum += ms;
  }
  *total_ms = sum;
  *count = t->used;
  return CVLBM_OK;
}

extern "C" int cvlbm_timer_attach(cvlbm_timer* t) { return cv::attach_timer(t); }

extern "C" int cvlbm_timer_attach_links(cvlbm_timer* t) {
  cv::g_link_timer = t;
  return CVLBM_OK;
}

extern "C" int cvlbm_version(void) { return 10000; }

extern "C" int64_t cvlbm_struct_size(int32_t which) {
  switch (which) {
    case 0: return (int64_t)sizeof(cvlbm2d_problem);
    case 1: return (int64_t)sizeof(cvlbm2d_fields);
    case 2: return (int64_t)sizeof(cvlbm3d_problem);
    case 3: return (int64_t)sizeof(cvlbm3d_fields);
    case 4: return (int64_t)sizeof(cvlbm3d_stencil_input);
    default: return -1;
  }
}

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
