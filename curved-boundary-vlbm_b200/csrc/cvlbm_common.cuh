// Host-side helpers shared by the 2-D and 3-D translation units: error
// reporting across the C ABI and CUDA-graph capture of a launch sequence.
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <map>
#include <mutex>
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

// Records a timer event on `s`: as an external event node when `s` is being
// captured into a graph (so that every replay records it), else plainly.
inline void record_timer_event(cudaEvent_t e, cudaStream_t s) {
  cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(s, &st) == cudaSuccess && st == cudaStreamCaptureStatusActive)
    cudaEventRecordWithFlags(e, s, cudaEventRecordExternal);
  else
    cudaEventRecord(e, s);
}

// Records the begin event of the next timer pair (if a timer is attached and
// has room) and returns its index, else -1.
inline int timer_begin(cudaStream_t s) {
  cvlbm_timer* t = attached_timer();
  if (!t || t->used >= t->capacity) return -1;
  int k = t->used++;
  record_timer_event(t->begin[k], s);
  return k;
}
inline void timer_end(int k, cudaStream_t s) {
  if (k >= 0) record_timer_event(attached_timer()->end[k], s);
}

// The same for the cut-link kernel (a second per-thread timer).
cvlbm_timer* attached_link_timer();
inline int link_timer_begin(cudaStream_t s) {
  cvlbm_timer* t = attached_link_timer();
  if (!t || t->used >= t->capacity) return -1;
  int k = t->used++;
  record_timer_event(t->begin[k], s);
  return k;
}
inline void link_timer_end(int k, cudaStream_t s) {
  if (k >= 0) record_timer_event(attached_link_timer()->end[k], s);
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

// Captures run one at a time on one persistent stream per device, so that
// per-stream resources the captured code keys on that stream (the second
// stream of an overlapped step) are reused from capture to capture.
inline std::mutex& capture_mutex() {
  static std::mutex mu;
  return mu;
}
inline cudaStream_t capture_stream() {
  static std::map<int, cudaStream_t> streams;
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return nullptr;
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
  streams[dev] = s;
  return s;
}

template <class F>
int capture_graph(F&& body, cvlbm_graph** out) {
  std::lock_guard<std::mutex> lock(capture_mutex());
  cudaStream_t s = capture_stream();
  if (!s) return fail(CVLBM_ERR_CUDA, "graph capture: stream creation failed");
  int rc = CVLBM_OK;
  cudaGraph_t g = nullptr;
  if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    return fail(CVLBM_ERR_CUDA, "graph capture: begin failed");
  rc = body(s);
  cudaError_t e = cudaStreamEndCapture(s, &g);
  if (rc != CVLBM_OK) {
    if (g) cudaGraphDestroy(g);
    return rc;
  }
  if (e != cudaSuccess || !g) return fail(CVLBM_ERR_CUDA, "graph capture: end failed");
  cudaGraphExec_t ex;
  // kernels launched with a priority attribute keep it when replayed
  if (cudaGraphInstantiate(&ex, g, cudaGraphInstantiateFlagUseNodePriority) != cudaSuccess) {
    cudaGraphDestroy(g);
    return fail(CVLBM_ERR_CUDA, "graph capture: instantiate failed");
  }
  *out = new cvlbm_graph{g, ex};
  return CVLBM_OK;
}

}  // namespace cv
