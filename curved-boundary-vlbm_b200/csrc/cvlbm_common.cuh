// Host-side helpers shared by the 2-D and 3-D translation units: error
// reporting across the C ABI and CUDA-graph capture of a launch sequence.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <string>

#include "cvlbm.h"

struct cvlbm_timer {
  int capacity;
  int used;
  cudaEvent_t* begin;
  cudaEvent_t* end;
};

struct cvlbm_graph {
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};

namespace cv {

void set_error(const char* msg);

// Launch accounting and the optional per-thread timer of the dominant kernel.
void count_launches(int n);
cvlbm_timer* attached_timer();

// Records the begin event of the next timer pair (if a timer is attached and
// has room) and returns its index, else -1.
inline int timer_begin(cudaStream_t s) {
  cvlbm_timer* t = attached_timer();
  if (!t || t->used >= t->capacity) return -1;
  int k = t->used++;
  cudaEventRecordWithFlags(t->begin[k], s, cudaEventRecordExternal);
  return k;
}
inline void timer_end(int k, cudaStream_t s) {
  if (k >= 0) cudaEventRecordWithFlags(attached_timer()->end[k], s, cudaEventRecordExternal);
}

inline int fail(int code, const char* msg) {
  set_error(msg);
  return code;
}

// Reports a launch-configuration error of the preceding launches (does not
// synchronise; asynchronous execution errors surface on the next sync).
inline int check_launch(const char* where) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s: %s", where, cudaGetErrorString(e));
    set_error(buf);
    return CVLBM_ERR_CUDA;
  }
  return CVLBM_OK;
}

template <class F>
int capture_graph(F&& body, cvlbm_graph** out) {
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess)
    return fail(CVLBM_ERR_CUDA, "graph capture: stream creation failed");
  int rc = CVLBM_OK;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
    cudaStreamDestroy(s);
    return fail(CVLBM_ERR_CUDA, "graph capture: begin failed");
  }
  rc = body(s);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  cudaStreamDestroy(s);
  if (rc != CVLBM_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess || !g) return fail(CVLBM_ERR_CUDA, "graph capture: end failed");
  cudaGraphExec_t ex;
  if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(CVLBM_ERR_CUDA, "graph capture: instantiate failed");
  }
  *out = new cvlbm_graph{g, ex};
  return CVLBM_OK;
}

}  // namespace cv
