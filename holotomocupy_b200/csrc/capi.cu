// Library-wide entry points: version, last-error message, launch counter and
// CUDA-graph capture of a stream's work.
#include "common.cuh"
#include "holotomo_b200_internal.h"

extern "C" int ht_version(void) { return 100; }

extern "C" const char* ht_last_error(void) { return ht::last_error(); }

extern "C" long ht_launch_count(void) { return ht::launch_count(); }

// ------------------------------------------------------- host memory
// Page-lock host memory for asynchronous copies (the host arrays a chunked
// call streams).  A range that is already page-locked is not an error: it is
// reported with *registered = 0, and the runtime's pending error is cleared.
extern "C" int ht_host_register(void* ptr, long bytes, int* registered) {
  HT_REQUIRE(ptr && registered && bytes > 0, "ht_host_register: null pointer or empty range");
  const cudaError_t e = cudaHostRegister(ptr, (size_t)bytes, cudaHostRegisterDefault);
  if (e == cudaErrorHostMemoryAlreadyRegistered) {
    (void)cudaGetLastError();
    *registered = 0;
    return ht::kOk;
  }
  HT_CHECK_CUDA(e);
  *registered = 1;
  return ht::kOk;
}

extern "C" int ht_host_unregister(void* ptr) {
  HT_REQUIRE(ptr, "ht_host_unregister: null pointer");
  HT_CHECK_CUDA(cudaHostUnregister(ptr));
  return ht::kOk;
}

// ------------------------------------------------------------ graphs
// Record the work issued to `stream` until ht_graph_end into a graph, instead
// of running it.  Relaxed mode: a free of unrelated memory made meanwhile
// (say, by another request's object being destroyed) does not invalidate
// the recording.
extern "C" int ht_graph_begin(void* stream) {
  HT_REQUIRE(stream, "ht_graph_begin: capture needs a non-default stream");
  HT_CHECK_CUDA(cudaStreamBeginCapture(static_cast<cudaStream_t>(stream), cudaStreamCaptureModeRelaxed));
  return ht::kOk;
}

extern "C" int ht_graph_end(void* stream, void** exec) {
  HT_REQUIRE(stream && exec, "ht_graph_end: null pointer");
  cudaGraph_t g = nullptr;
  HT_CHECK_CUDA(cudaStreamEndCapture(static_cast<cudaStream_t>(stream), &g));
  cudaGraphExec_t ex = nullptr;
  const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
  cudaGraphDestroy(g);
  HT_CHECK_CUDA(e);
  *exec = ex;
  return ht::kOk;
}

extern "C" int ht_graph_launch(void* exec, void* stream) {
  HT_REQUIRE(exec, "ht_graph_launch: null graph");
  HT_CHECK_CUDA(cudaGraphLaunch(static_cast<cudaGraphExec_t>(exec), static_cast<cudaStream_t>(stream)));
  return ht::kOk;
}

extern "C" int ht_graph_destroy(void* exec) {
  if (exec) HT_CHECK_CUDA(cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(exec)));
  return ht::kOk;
}
